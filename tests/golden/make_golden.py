"""Regenerate the committed golden fixtures from the reference tree.

Run in a container that has the reference mounted (it is read here only):

    python tests/golden/make_golden.py <path to the MACIS source tree>

or with the path in the environment variable MACIS_REFERENCE_DIR.

Outputs (all under tests/golden/):

* ``h2o_ccpvdz_fcidump.npz`` -- the water cc-pVDZ FCIDUMP of the reference
  tests (tests/ref_data/h2o.ccpvdz.fci.dat) transcribed line by line to
  binary: ``idx`` (nline, 4) int8 1-based orbital indices and ``val`` float64.
  The 8-fold fill that turns it into T and V is in tests/golden_data.py and
  follows src/macis/fcidump.cxx:141-174.
* ``h2o_ccpvdz_cisd_rowptr.npz`` -- tests/ref_data/h2o.ccpvdz.cisd.rowptr.bin
  (int32, 12,637 entries), the exact CSR row pointer the reference test
  tests/csr_hamiltonian.cxx:64 checks.
* ``reference_constants.json`` -- the literal golden numbers in the reference
  tests, with the file:line each comes from.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def transcribe_fcidump(path):
    idx, val = [], []
    with open(path) as f:
        for line in f:
            tok = line.split()
            if len(tok) != 5:
                continue
            # fcidump.cxx:28-61: a token is a float if it holds a letter or
            # '.', and the integral is last when the last token is a float.
            is_float = lambda t: any(c.isalpha() or c == "." for c in t)
            if is_float(tok[-1]):
                p, q, r, s = (int(t) for t in tok[:4])
                v = float(tok[4])
            else:
                p, q, r, s = (int(t) for t in tok[1:])
                v = float(tok[0])
            idx.append((p, q, r, s))
            val.append(v)
    return np.asarray(idx, dtype=np.int8), np.asarray(val, dtype=np.float64)


CONSTANTS = {
    "water_nocc": [5, "tests/csr_hamiltonian.cxx:22"],
    "water_ehf_plus_ecore": [-76.0267803489191, "tests/double_loop.cxx:53"],
    "water_single_diag": [-6.488097259228e01, "tests/double_loop.cxx:62"],
    "water_ss_double_diag": [-6.314093508151e01, "tests/double_loop.cxx:71"],
    "water_os_double_diag": [-6.304547887231e01, "tests/double_loop.cxx:81"],
    "water_mp2": [-0.203989305096243, "tests/double_loop.cxx:159"],
    "water_cisd_e0_plus_ecore": [-7.623197835987e01, "tests/davidson.cxx:48"],
    "water_cisd_davidson_max_m": [15, "tests/davidson.cxx:60"],
    "water_cisd_thresh": [1e-16, "tests/csr_hamiltonian.cxx:46"],
    "water_asci_grow_e0": [-8.542926243842e01, "tests/asci.cxx:257"],
    "water_asci_refine_e0": [-8.542925964708e01, "tests/asci.cxx:268"],
    "water_asci_ntdets_max": [10000, "tests/asci.cxx:252"],
    "catch2_approx_rel": [1.1920928955078125e-05,
                          "Catch2 v2 Approx default epsilon float eps*100"],
}


def main(ref):
    idx, val = transcribe_fcidump(
        os.path.join(ref, "tests/ref_data/h2o.ccpvdz.fci.dat"))
    np.savez_compressed(os.path.join(HERE, "h2o_ccpvdz_fcidump.npz"),
                        idx=idx, val=val)
    rp = np.fromfile(os.path.join(ref, "tests/ref_data/h2o.ccpvdz.cisd.rowptr.bin"),
                     dtype=np.int32)
    np.savez_compressed(os.path.join(HERE, "h2o_ccpvdz_cisd_rowptr.npz"),
                        rowptr=rp)
    with open(os.path.join(HERE, "reference_constants.json"), "w") as f:
        json.dump(CONSTANTS, f, indent=1)
    print("lines", len(val), "rowptr", rp.shape, rp[-1])


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get(
        "MACIS_REFERENCE_DIR")
    if not src:
        sys.exit("usage: make_golden.py <path to the MACIS source tree> "
                 "(or set MACIS_REFERENCE_DIR)")
    main(src)
