"""Host-side logic that needs no GPU: determinant spaces, integrals, the
Rayleigh-Ritz eigensolver, the C ABI surface, the row-block partition and
the drivers' use of the screening settings."""
import ctypes
import os
import re

import numpy as np
import pytest

import macis_b200 as mb
import oracle
from macis_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_header_symbols_exported():
    hdr = open(os.path.join(ROOT, "include", "macis_b200.h")).read()
    names = set(re.findall(r"\b(macis_b200_\w+)\s*\(", hdr))
    assert names, "no declarations found"
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for n in sorted(names):
        assert hasattr(lib, n), n
    assert names == set(_lib.EXPORTS)
    assert _lib.LIB.macis_b200_version() == 1


def test_struct_layouts_match_header(tmp_path):
    """ctypes mirrors agree with the C header (compiled here with gcc)."""
    import subprocess
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include "macis_b200.h"\nint main(){'
                   'printf("%zu %zu %zu %zu %zu", sizeof(macis_b200_asci_settings),'
                   'sizeof(macis_b200_asci_stats),'
                   'sizeof(macis_b200_davidson_opts),'
                   'sizeof(macis_b200_build_stats),'
                   'sizeof(macis_b200_asci_screen));return 0;}')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True,
                                          text=True).stdout.split()]
    assert got == [ctypes.sizeof(_lib.AsciSettingsC),
                   ctypes.sizeof(_lib.AsciStatsC),
                   ctypes.sizeof(_lib.DavidsonOptsC),
                   ctypes.sizeof(_lib.BuildStatsC),
                   ctypes.sizeof(_lib.AsciScreenC)]
    assert ctypes.sizeof(_lib.AsciSettingsC) == ctypes.sizeof(
        oracle.AsciSettings)


@pytest.mark.parametrize("nbits", [64, 128, 256])
def test_spaces_match_oracle(port, nbits):
    assert np.array_equal(mb.generate_hilbert_space(7, 3, 2, nbits),
                          port.hilbert_space(nbits, 7, 3, 2))
    hf = mb.canonical_hf_determinant(4, 3, nbits)
    assert np.array_equal(hf, port.hf_det(nbits, 4, 3))
    assert np.array_equal(mb.generate_cisd_hilbert_space(9, hf, nbits),
                          port.cisd_space(nbits, 9, 4, 3))


def test_hilbert_space_matches_reference(ref):
    for nbits in (64, 128):
        assert np.array_equal(mb.generate_hilbert_space(8, 4, 3, nbits),
                              ref.hilbert_space(nbits, 8, 4, 3))
        hf = mb.canonical_hf_determinant(4, 4, nbits)
        assert np.array_equal(mb.generate_cisd_hilbert_space(10, hf, nbits),
                              ref.cisd_space(nbits, 10, 4, 4))


def test_canonical_strings_roundtrip():
    d = mb.sd.make_dets([0b1011], [0b0110], 128)
    s = mb.to_canonical_string(d, 128)
    assert s[:4] == "u22u"[:1] + "2" + "d" + "u"
    assert np.array_equal(mb.from_canonical_string(s, 128), d)


def test_synthetic_integrals():
    T, V = mb.synthetic_integrals(6, seed=3)
    n = 6
    T2 = T.reshape(n, n, order="F")
    V4 = V.reshape(n, n, n, n, order="F")
    assert np.array_equal(T2, T2.T)
    np.testing.assert_allclose(np.diag(T2), -1.5 + 2.5 * np.arange(n) / (n - 1))
    for perm in [(1, 0, 2, 3), (0, 1, 3, 2), (2, 3, 0, 1), (3, 2, 1, 0)]:
        assert np.allclose(V4, V4.transpose(perm), atol=1e-15)
    w = np.linalg.eigvalsh(V.reshape(n * n, n * n, order="F"))
    assert w.min() > -1e-12
    T3, V3 = mb.synthetic_integrals(6, seed=3)
    assert np.array_equal(T, T3) and np.array_equal(V, V3)


def test_water_fcidump_fill():
    from golden_data import water
    norb, T, V, ec = water()
    assert norb == 24 and ec != 0.0
    V4 = V.reshape((norb,) * 4, order="F")
    assert np.allclose(V4, V4.transpose(1, 0, 3, 2))
    assert np.allclose(V4, V4.transpose(2, 3, 0, 1))


def test_small_syev_against_numpy():
    rng = np.random.default_rng(0)
    for k in (1, 3, 17, 64, 250):
        M = rng.standard_normal((k, k))
        S = np.tril(M) + np.tril(M, -1).T
        w, v = np.linalg.eigh(S)
        nw = min(6, k)
        W, Vv = mb.small_syev(np.tril(M), nw)
        np.testing.assert_allclose(W, w[:nw], atol=1e-12 * max(1, abs(w).max()))
        np.testing.assert_allclose(np.abs(np.sum(Vv * v[:, :nw], 0)), 1,
                                   atol=1e-10)
    for M in (np.zeros((4, 4)), np.kron(np.eye(3), [[2., 1.], [1., 2.]])):
        W, Vv = mb.small_syev(np.tril(M), 4)
        assert np.abs(Vv.T @ Vv - np.eye(4)).max() < 1e-12
        assert np.abs(M @ Vv - Vv * W).max() < 1e-12


def test_row_bounds_partition():
    for M in (0, 1, 7, 853776):
        for w in (1, 2, 3, 8):
            b = [mb.row_bounds(M, w, r) for r in range(w)]
            assert b[0][0] == 0 and b[-1][1] == M
            assert all(b[i][1] == b[i + 1][0] for i in range(w - 1))


def test_settings_defaults_match_reference():
    s = mb.ASCISettings()
    o = oracle.AsciSettings.default()
    for f, _ in _lib.AsciSettingsC._fields_:
        if f != "pad_":
            assert getattr(s.c_struct(), f) == getattr(o, f), f
    m = mb.MCSCFSettings()
    assert (m.ci_res_tol, m.ci_max_subspace) == (1e-8, 20)
    assert m.ci_matel_tol == np.finfo(float).eps


class _FakeNet:
    """Stands in for a ScreeningNetwork: records what the drivers ask of it."""

    handle = None

    def __init__(self, trained_steps):
        self.trained_steps = trained_steps
        self.calls = []

    def clamp_samples(self, q):
        self.calls.append(("clamp", q))

    def train(self, X, t, epochs, batch, lr, seed):
        self.calls.append(("train", X, t, epochs, batch, lr, seed))


def test_screening_decision_and_retraining():
    """The drivers' use of ScreenSettings: no pruning before the network is
    trained or during the warm-up searches; retraining (clamped first) only
    after a search that recorded samples, seeded by the search count."""
    from macis_b200.asci import _train_after_search, _use_net
    net = _FakeNet(trained_steps=0)
    sc = mb.ScreenSettings(network=net, min_units=0, warmup_searches=2,
                           clamp_quantile=0.6, seed=5)
    assert not _use_net(None, None, None, 0.0, None)
    assert not _use_net(sc, None, None, 0.0, None)        # untrained
    net.trained_steps = 1
    sc.searches = 1
    assert not _use_net(sc, None, None, 0.0, None)        # warm-up
    sc.searches = 2
    assert _use_net(sc, None, None, 0.0, None)
    assert _train_after_search(sc, {"samples": 0}) == 0.0
    assert net.calls == []
    assert _train_after_search(sc, {"samples": 10}) >= 0.0
    assert net.calls == [("clamp", 0.6),
                         ("train", None, None, sc.epochs, sc.batch, sc.lr, 7)]
    sc.train = False
    net.calls.clear()
    _train_after_search(sc, {"samples": 10})
    assert net.calls == []
    assert sc.c_struct(True).max_samples == 0              # nothing recorded
    sc.train, sc.clamp_quantile = True, 0.0
    _train_after_search(sc, {"samples": 10})
    assert [c[0] for c in net.calls] == ["train"]


def test_recall_check_policy(monkeypatch):
    """The recall check's decisions (asci._recall_check), with stand-ins for
    the searches: no check for unscreened or large searches; the exact
    selection replaces the pruned one; keep_frac doubles below the target
    (at most 1) and otherwise halves through trial searches while they keep
    the target, not below keep_min; training uses the exact search's
    sample count; and topk_recall counts the exact search's new
    determinants found by the other."""
    from macis_b200 import asci
    monkeypatch.setattr(asci, "last_search_stats",
                        lambda h: {"samples": 77})
    ncore = 2
    exact = np.arange(24, dtype=np.uint64).reshape(12, 2)   # 10 new + 2 core
    half = exact.copy()
    half[:5] += 1000                                       # 5 of 10 found
    assert mb.topk_recall(exact, exact, ncore) == 1.0
    assert mb.topk_recall(half, exact, ncore) == 0.5
    net = _FakeNet(trained_steps=1)
    st = {"units_total": 100, "samples": 5}
    trials = []

    def check(sc, got, recall_of_trial):
        def pruned(k):
            trials.append(k)
            return exact if recall_of_trial(k) else half
        return asci._recall_check(sc, True, st, got, ncore, None,
                                  lambda: exact, pruned)

    sc = mb.ScreenSettings(network=net, keep_frac=0.4, keep_min=0.1,
                           check_units_max=1000)
    # not screened, or too many units: no check, the result is kept
    assert asci._recall_check(sc, False, st, half, ncore, None,
                              None, None) == (half, None, st)
    big = dict(st, units_total=10 ** 6)
    assert asci._recall_check(sc, True, big, half, ncore, None, None,
                              None)[1] is None
    # below the target: doubles, no trials, exact selection and samples
    dets, rec, st2 = check(sc, half, lambda k: True)
    assert dets is exact and rec == 0.5 and st2["samples"] == 77
    assert sc.keep_frac == 0.8 and trials == []
    check(sc, half, lambda k: True)
    assert sc.keep_frac == 1.0
    check(sc, half, lambda k: True)
    assert sc.keep_frac == 1.0
    # at the target: halves while the trials keep it (0.8 -> 0.4 -> 0.2)
    sc.keep_frac = 0.8
    dets, rec, _ = check(sc, exact, lambda k: k >= 0.2)
    assert rec == 1.0 and sc.keep_frac == 0.2 and trials == [0.4, 0.2, 0.1]
    # down to keep_min, never below
    trials.clear()
    sc.keep_frac = 0.2
    check(sc, exact, lambda k: True)
    assert sc.keep_frac == 0.1 and trials == [0.1]
    trials.clear()
    check(sc, exact, lambda k: True)
    assert sc.keep_frac == 0.1 and trials == []
    # recall_target 0: the check is off
    sc.recall_target = 0.0
    assert asci._recall_check(sc, True, st, half, ncore, None, None,
                              None)[1] is None


def test_product_does_not_use_the_oracle():
    """The package (the product path) imports neither the oracle nor any
    working file; only the tests, smoke() and bench.py's baseline legs do."""
    pat = re.compile(r"^\s*(import|from)\s+(\.*\s*)?(oracle|_work)\b", re.M)
    pkg = os.path.join(ROOT, "macis_b200")
    for f in sorted(os.listdir(pkg)):
        if f.endswith(".py"):
            with open(os.path.join(pkg, f)) as fh:
                assert not pat.search(fh.read()), f


def test_merge_asci_parts_topk_rules():
    """merge_asci_parts: |score| descending then determinant ascending, cut
    at ndets_max - ncdets (determinant_search.hpp:547, size_t): fewer slots
    than core determinants cut nothing, and a result beyond ndets_max is
    refused as by the search."""
    from macis_b200.asci import merge_asci_parts
    u = lambda *v: np.array(v, dtype=np.uint64).reshape(-1, 1)
    parts = [(u(5, 1, 9), np.array([-0.5, -0.2, -0.5])),
             (u(3, 7), np.array([-0.5, -0.1]))]
    core = u(200, 100)
    assert merge_asci_parts(parts, 5, core, 64)[:, 0].tolist() == \
        [3, 5, 9, 200, 100]
    assert merge_asci_parts(parts, 4, core, 64)[:, 0].tolist() == \
        [3, 5, 200, 100]                       # tie at the cut: smaller dets
    assert merge_asci_parts(parts, 7, core, 64)[:, 0].tolist() == \
        [1, 3, 5, 7, 9, 200, 100]
    with pytest.raises(mb.MacisError, match="exceeds ndets_max"):
        merge_asci_parts(parts, 1, core, 64)    # 1 - 2 wraps: nothing cut
    empty = [(np.zeros((0, 1), dtype=np.uint64), np.zeros(0))]
    assert merge_asci_parts(empty, 1, core, 64)[:, 0].tolist() == [200, 100]
