"""C++ drop-in: the reference's own make_csr_hamiltonian / selected_ci_diag
templates with the B200 generator in the HamiltonianGenerator virtual hook,
compiled against the unmodified reference headers (oracle/ref/dropin_check.cpp,
built into oracle/_ref by oracle/ref/Makefile)."""
import json
import os
import subprocess

import numpy as np
import pytest

from golden_data import constants, water

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "dropin_check")


@pytest.mark.skipif(not os.path.exists(EXE), reason="dropin_check not built")
def test_reference_templates_with_b200_generator(tmp_path):
    norb, T, V, _ = water()
    K = constants()
    (tmp_path / "T.bin").write_bytes(np.ascontiguousarray(T).tobytes())
    (tmp_path / "V.bin").write_bytes(np.ascontiguousarray(V).tobytes())
    out = subprocess.run([EXE, str(tmp_path / "T.bin"), str(tmp_path / "V.bin"),
                          str(norb), "5", "5", "10000"], capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert r["ndets"] == 12636 and r["csr_equal"]
    assert r["e_cpu"] == r["e_hook"]           # identical CSR -> same Davidson
    assert abs(r["e_gpu"] - r["e_cpu"]) < 1e-8
    # the reference's davidson on the shim's matrix-free operator
    assert abs(r["e_matrix_free"] - r["e_cpu"]) < 1e-8
    # form_rdms through the generator hook, against the reference generator
    assert r["rdm_max_diff"] < 1e-11
    assert r["asci_size"] == 10000 and abs(r["asci_norm"] - 1) < 1e-10
    assert abs(r["asci_e0"] - K["water_asci_grow_e0"]) < 1e-8
    # the shim's screened drivers: recording + training leaves every search
    # as it was; pruning (searches 3 and 4, half the units) still grows the
    # same state -- the network's accuracy is tested in test_gpu_screening
    print(f"\nshim screened grow: dE {r['scr_e0'] - r['asci_e0']:.3e} Eh, "
          f"units {r['scr_units_kept']}/{r['scr_units_total']}")
    assert r["rec_size"] == 10000 and r["rec_searches"] == 4
    assert r["rec_trained"] == 4 and abs(r["rec_e0"] - r["asci_e0"]) < 1e-8
    assert r["scr_size"] == 10000 and r["scr_trained"] == 4
    assert 0 < r["scr_units_kept"] <= 0.52 * r["scr_units_total"] + 2
    assert abs(r["scr_e0"] - r["asci_e0"]) < 1e-3   # measured 1.1e-4
