"""Small, self-contained workloads for kernel profiling (ncu) and timing.

    python profile_cases.py hbuild_c1   # CAS(10e,10o) CSR build
    python profile_cases.py hbuild_c2   # CAS(12e,12o) CSR build
    python profile_cases.py hbuild_c2s  # 12 orbitals, 3a/6b: the
        # beta lists of CAS(12e,12o) at a quarter of its output (3.3 GB)
    python profile_cases.py spmv_c1     # FP64 SpMV on CAS(10e,10o)
    python profile_cases.py hop_c2      # matrix-free H x, CAS(12e,12o)
    python profile_cases.py hbuild_sel  # selected (shuffled) space
    python profile_cases.py asci_n48    # one ASCI search, n = 48
    python profile_cases.py asci_n100 --ncore 10000
        # the same on n = 100, 20a/20b, bitset<256> (C5 shape), 20 x ncore dets
        # (--ncore core determinants, default 10000)
    python profile_cases.py mlp_fwd     # network forward, 2M rows
    python profile_cases.py mlp_train   # one training epoch
    python profile_cases.py asci_iter_n48 --ncore 100000 --ntdets 1e6
        # one ASCI iteration, n = 48: exact FP64 against learned + mixed
    python profile_cases.py c3 --ntdets 1000000 --mode fp64
        # ASCI n = 48, 12a/12b, bitset<128>: grow from HF (factor 8, <= 1e5
        # core dets) then 3 refine iterations; --mode fp64 (exact search,
        # FP64 Davidson) or learned_mixed (screened search, FP32-H Davidson)
    python profile_cases.py c4 --ntdets 1000000 --mode ...
        # the same on n = 64, 16a/16b, bitset<128>; learned_mixed also runs
        # one exact search from its last core set and reports the top-k
        # recall of the screened one
    python profile_cases.py c5 --ntdets 51200 --refine 1 --mode ...
        # n = 100, 20a/20b, bitset<256>, modes as c3

Each case runs its hot call a few times (--reps) and prints one timing line.
"""
import argparse
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import macis_b200 as mb  # noqa: E402

EPS = float(np.finfo(np.float64).eps)


def fci(norb, k, nbits=64, seed=0, kb=None):
    T, V = mb.synthetic_integrals(norb, seed)
    return T, V, mb.generate_hilbert_space(norb, k, k if kb is None else kb,
                                           nbits)


def hbuild(norb, k, reps, shuffle=False, kb=None):
    T, V, dets = fci(norb, k, kb=kb)
    if shuffle:
        dets = dets[np.random.default_rng(1).permutation(len(dets))]
    H = mb.HamiltonianGenerator(T, V, 64)
    for _ in range(reps):
        A = mb.make_csr_hamiltonian(dets, H, EPS)
        st = A.build_stats()
        print(f"build nnz={A.nnz} build_ms={st['build_ms']:.3f} "
              f"fill_ms={st['fill_ms']:.3f} direct={st['direct_product']}")
        del A


def spmv(norb, k, reps):
    T, V, dets = fci(norb, k)
    H = mb.HamiltonianGenerator(T, V, 64)
    A = mb.make_csr_hamiltonian(dets, H, EPS)
    x = np.random.default_rng(0).standard_normal(A.n)
    for _ in range(reps):
        t = time.perf_counter()
        A.spmv(x)
        print(f"spmv host-staged {1e3 * (time.perf_counter() - t):.3f} ms")


def _bench():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "bench", os.path.join(os.path.dirname(os.path.abspath(__file__)),
                              "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    return bench


def asci_n48(reps, ncore=10000, ndets=200000, n=48, k=12, nbits=128):
    """One exact ASCI search on the bench's n = 48 core set (the first run
    grows the memory pool); n = 100, 20 / 20, bitset<256> for asci_n100."""
    bench = _bench()
    n, H, core, C, E0 = bench._n48_core(mb, ncore, n=n, k=k, nbits=nbits)
    s = mb.ASCISettings()
    for _ in range(reps):
        t = time.perf_counter()
        mb.asci_search(s, ndets, core, E0, C, n, H)
        dt = time.perf_counter() - t
        st = mb.last_search_stats(H)
        print(f"asci {dt:.3f} s raw={st['raw_pairs']} "
              f"unique={st['unique_pairs']} batches={st['batches']} "
              f"pairs_ms={st['pairs_ms']:.1f} sort_ms={st['sort_ms']:.1f} "
              f"keep_ms={st['keep_ms']:.1f} "
              f"passes={st['sort_pass_items'] / max(st['raw_pairs'], 1):.2f}")


def hop(norb, k, reps):
    """Matrix-free H x on the FCI list against the CSR product (host-staged
    vectors; the determinant list and the tables stay on the device)."""
    T, V, dets = fci(norb, k)
    H = mb.HamiltonianGenerator(T, V, 64)
    t = time.perf_counter()
    Hm = mb.MatrixFreeHamiltonian(dets, H, EPS)
    print(f"matrix-free setup {1e3 * (time.perf_counter() - t):.1f} ms")
    x = np.random.default_rng(0).standard_normal(len(dets))
    for _ in range(reps):
        t = time.perf_counter()
        y = Hm.spmv(x)
        print(f"matrix-free H x {1e3 * (time.perf_counter() - t):.1f} ms")
    A = mb.make_csr_hamiltonian(dets, H, EPS)
    t = time.perf_counter()
    y0 = A.spmv(x)
    print(f"CSR H x {1e3 * (time.perf_counter() - t):.1f} ms (host-staged), "
          f"max rel diff {np.abs(y - y0).max() / np.abs(y0).max():.2e}")


def _rand_rows(n, din, seed=0):
    rng = np.random.default_rng(seed)
    X = np.zeros((n, din), dtype=np.float32)
    X[:, :din - 64] = rng.integers(0, 2, (n, din - 64))
    X[:, din - 64:] = rng.normal(0, 1, (n, 64))
    u = X.view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16)).astype(np.uint16)


def mlp_fwd(reps, n=1 << 21):
    net = mb.ScreeningNetwork(din=192, seed=0)
    X = _rand_rows(n, 192)
    for _ in range(reps):
        t = time.perf_counter()
        net.forward(X)
        dt = time.perf_counter() - t
        print(f"mlp forward {n} rows {dt * 1e3:.3f} ms (host-staged)")


def mlp_train(reps, n=1 << 18, batch=256):
    net = mb.ScreeningNetwork(din=192, seed=0)
    X = _rand_rows(n, 192)
    t = np.random.default_rng(1).normal(0, 1, n).astype(np.float32)
    for _ in range(reps):
        tt = time.perf_counter()
        loss = net.train(X, t, epochs=1, batch=batch)
        dt = time.perf_counter() - tt
        print(f"mlp train 1 epoch {n} rows batch {batch}: {dt * 1e3:.1f} ms "
              f"({dt * 1e6 / (n / batch):.1f} us/step) loss {loss:.4f}")


def asci_iter_n48(ncore=100000, ndets=1000000):
    """The bench's C3-shaped ASCI iteration (exact FP64 against learned +
    mixed) on its own."""
    import json
    bench = _bench()
    print(json.dumps(bench.asci_iteration(mb, bench.peaks()[0], ncore=ncore,
                                          ndets=ndets), default=float))


def c3(ntdets, mode, refine=3, ncore=100000, seed=0, n=48, k=12, nbits=128,
       compare=False, save=None):
    """One C3-shaped ASCI run (C4 with n = 64, k = 16); prints one JSON line
    with the per-iteration log, the final energy and the wall time."""
    import json
    import logging
    logging.basicConfig(level=logging.INFO, format="%(name)s %(message)s")
    T, V = mb.synthetic_integrals(n, seed)
    H = mb.HamiltonianGenerator(T, V, nbits)
    s = mb.ASCISettings(ntdets_max=int(ntdets), ntdets_min=100,
                        ncdets_max=int(ncore), grow_factor=8, h_el_tol=1e-8,
                        max_refine_iter=int(refine))
    m = mb.MCSCFSettings(ci_max_subspace=40, davidson_restart_keep=8,
                         davidson_max_iter=4000,
                         precision=mb.MIXED if mode == "learned_mixed" else mb.FP64)
    scr = None
    if mode == "learned_mixed":
        scr = mb.ScreenSettings(network=mb.ScreeningNetwork(nbits=nbits,
                                                             seed=seed))
    hf = mb.canonical_hf_determinant(k, k, nbits)
    E0 = float(H.matrix_element(hf, hf))
    t0 = time.perf_counter()
    E, dets, X = mb.asci_grow(s, m, E0, hf, [1.0], H, n, screen=scr)
    t_grow = time.perf_counter() - t0
    Eg = E
    for _ in range(int(refine)):  # refine.hpp:15-66, fixed iteration count
        E, dets, X = mb.asci_iter(s, m, len(dets), E, dets, X, H, n, scr)
    dt = time.perf_counter() - t0
    recall = None
    cmp = None
    if save:  # the final core set (search input of a next iteration)
        core, C = mb.reorder_ci_on_coeff(dets, np.asarray(X))
        nc = min(int(ncore), len(core))
        np.savez(save, dets=core[:nc], C=C[:nc], E=E, n=n, k=k, nbits=nbits)
    if scr is not None and compare:
        # one more iteration from the final wavefunction both ways: exact
        # search + FP64 solve against the trained network's screened search
        # + mixed solve, at equal determinant count
        core, C = mb.reorder_ci_on_coeff(dets, np.asarray(X))
        nc = min(int(ncore), len(core))
        bench = _bench()
        cmp = bench.asci_iteration(mb, bench.peaks()[0],
                                   problem=(n, H, core[:nc], C[:nc], E),
                                   ndets=len(dets), nbits=nbits,
                                   net=scr.network, warm=False,
                                   keep_frac=scr.keep_frac)
    elif scr is not None:
        # top-k recall of the screened search against the exact one, from
        # the same core set (the last iteration's wavefunction)
        core, C = mb.reorder_ci_on_coeff(dets, np.asarray(X))
        nc = min(int(ncore), len(core))
        sc = mb.ScreenSettings(network=scr.network, keep_frac=scr.keep_frac,
                               explore_frac=0.0, train=False)
        got = mb.asci_search(s, len(dets), core[:nc], E, C[:nc], n, H,
                             screen=sc, use_net=True)
        exact = mb.asci_search(s, len(dets), core[:nc], E, C[:nc], n, H)
        recall = mb.topk_recall(got, exact, nc)
    # variational energy of the final wavefunction with the FP64 H (the
    # mixed mode solved with FP32 off-diagonal values)
    # (a stored FP64 H when it fits in device memory, else matrix-free only)
    Xd = np.asarray(X, dtype=np.float64)
    AX, csr_ms = None, None
    try:
        A = mb.make_csr_hamiltonian(dets, H, EPS, np.int64)
        t = time.perf_counter()
        AX = A.spmv(Xd)
        csr_ms = 1e3 * (time.perf_counter() - t)
        del A
    except mb.MacisError as e:
        print(f"stored FP64 H does not fit: {e}", file=sys.stderr)
    # the same product without storing H (host-staged vectors both ways)
    t = time.perf_counter()
    Hm = mb.MatrixFreeHamiltonian(dets, H, EPS)
    hop_setup_ms = 1e3 * (time.perf_counter() - t)
    t = time.perf_counter()
    AXm = Hm.spmv(Xd)
    hop_ms = 1e3 * (time.perf_counter() - t)
    hop_diff = (None if AX is None else
                float(np.abs(AXm - AX).max() / np.abs(AX).max()))
    if AX is None:
        AX = AXm
    E_fp64 = float(Xd @ AX) / float(Xd @ Xd)
    del Hm
    out = {"mode": mode, "ntdets": int(ntdets), "ndets": len(dets),
           "n": n, "electrons": [k, k], "E_grow": Eg, "E_final": E,
           "E_final_fp64_H": E_fp64, "topk_recall_last": recall,
           "seconds": dt, "grow_seconds": t_grow, "compare": cmp,
           "final_product_ms": {"csr": csr_ms, "matrix_free": hop_ms,
                                "matrix_free_setup": hop_setup_ms,
                                "max_rel_diff": hop_diff},
           "iterations": m.iteration_log}
    print(json.dumps(out, default=float))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--ntdets", type=float, default=1e6)
    ap.add_argument("--mode", default="fp64")
    ap.add_argument("--ncore", type=int, default=None,
                    help="core determinants (default 1e4 for the single "
                         "searches, 1e5 for asci_iter_n48 and c3/c4/c5)")
    ap.add_argument("--refine", type=int, default=3)
    ap.add_argument("--compare", action="store_true")
    ap.add_argument("--save", default=None,
                    help="c3/c4/c5: write the final core set to this .npz")
    a = ap.parse_args()
    if a.case == "hbuild_c1":
        hbuild(10, 5, a.reps)
    elif a.case == "hbuild_c2":
        hbuild(12, 6, a.reps)
    elif a.case == "hop_c1":
        hop(10, 5, a.reps)
    elif a.case == "hop_c2":
        hop(12, 6, a.reps)
    elif a.case == "hbuild_c2s":
        hbuild(12, 3, a.reps, kb=6)
    elif a.case == "hbuild_sel":
        hbuild(10, 5, a.reps, shuffle=True)
    elif a.case == "spmv_c1":
        spmv(10, 5, a.reps)
    elif a.case == "asci_n48":
        asci_n48(a.reps, ncore=a.ncore or 10000)
    elif a.case == "asci_n100":
        asci_n48(a.reps, ncore=a.ncore or 10000,
                 ndets=20 * (a.ncore or 10000), n=100, k=20,
                 nbits=256)
    elif a.case == "mlp_fwd":
        mlp_fwd(a.reps)
    elif a.case == "mlp_train":
        mlp_train(a.reps)
    elif a.case == "asci_iter_n48":
        asci_iter_n48(a.ncore or 100000,
                      int(a.ntdets))
    elif a.case in ("c3", "c4", "c5"):
        # --ncore: core determinants per search (default 1e5 for these)
        nc = a.ncore or 100000
        if a.case == "c3":
            c3(a.ntdets, a.mode, refine=a.refine, ncore=nc, compare=a.compare,
               save=a.save)
        elif a.case == "c4":
            c3(a.ntdets, a.mode, refine=a.refine, ncore=nc, n=64, k=16,
               compare=a.compare, save=a.save)
        else:
            # n = 100, 20a/20b, bitset<256> (network input 320 columns)
            c3(a.ntdets, a.mode, refine=a.refine, ncore=nc, n=100, k=20,
               nbits=256, compare=a.compare, save=a.save)
    else:
        raise SystemExit(f"unknown case {a.case}")


if __name__ == "__main__":
    main()
