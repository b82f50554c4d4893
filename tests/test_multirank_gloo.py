"""The multi-rank (N > 1) path on CPU: two gloo ranks, spawned processes.

Each rank computes its row block [lo, hi) of H with the oracle (the stand-in
for the block libmacis_b200 builds on that rank's GPU), and the host logic of
macis_b200.dist is checked: the row partition of make_dist_csr_hamiltonian
(csr_hamiltonian.hpp:49-82), gathering blocks back into the full matrix, the
max / sum reductions the benchmark uses for its timings and counts, and the
parallel Davidson (p_davidson, davidson.hpp:283-394) against the serial
solve on the full matrix."""
import socket
import traceback

import numpy as np
import pytest

from cases import fci

WORLD = 2
TIMEOUT_S = 240


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    # 35 x 35 = 1225 determinants: an odd count, so the last rank gets the
    # extra row
    return fci(7, 3, 3, 64, seed=4)


def _block_op(port, hp, dets, lo, hi):
    import torch
    rp, ci, nz = port.build_csr(hp, dets[lo:hi], dets, np.finfo(float).eps)

    def mv(x_full):
        return torch.from_numpy(port.spmv(rp, ci, nz, x_full.numpy()))
    return (rp, ci, nz), mv


def _asci_parts(port, world=WORLD, ndets_max=300):
    """Parts of a split ASCI search built from the oracle's accumulated
    pairs: core dets and zero scores removed, a disjoint split by a hash of
    the determinant, each part cut at its (ndets_max - ncore)-th |score|
    with every tie kept. Returns [(states, scores, core, ndets_max)]."""
    import oracle
    T, V, d = fci(7, 3, 3, 64, seed=6)
    core = d[:40]
    C = np.random.default_rng(2).standard_normal(len(core))
    C /= np.linalg.norm(C)
    hp = port.ham(64, 7, T, V)
    E0 = float(port.matrix_element(hp, core[:1], core[:1])[0]) - 0.5
    st, rv = port.asci_pairs(hp, oracle.AsciSettings.default(), core, E0, C)
    keep = (rv != 0) & ~np.isin(st[:, 0], core[:, 0])
    st, rv = st[keep], rv[keep]
    k = ndets_max - len(core)
    out = []
    for r in range(world):
        m = (st[:, 0] * np.uint64(0x9E3779B97F4A7C15) >> np.uint64(61)) % \
            np.uint64(world) == np.uint64(r)
        ps, pr = st[m], rv[m]
        if len(pr) > k:
            cut = np.sort(np.abs(pr))[::-1][k - 1]
            ps, pr = ps[np.abs(pr) >= cut], pr[np.abs(pr) >= cut]
        out.append((ps, pr, core, ndets_max))
    return out, (st, rv)


def _sample_targets(n=1000, seed=3):
    """Targets of a whole search's samples and the parts' views of them:
    each unit's largest score lands in one rank's bins; the other ranks see
    a smaller one (or none: the floor target (ln 1e-12 + 20) / 5)."""
    rng = np.random.default_rng(seed)
    floor = np.float32((np.log(1e-12) + 20) / 5)
    whole = rng.uniform(floor, 4.0, n).astype(np.float32)
    owner = rng.integers(0, WORLD, n)
    parts = []
    for r in range(WORLD):
        lower = np.maximum(whole - rng.uniform(0, 1, n).astype(np.float32),
                           floor)
        lower[rng.random(n) < 0.3] = floor
        parts.append(np.where(owner == r, whole, lower).astype(np.float32))
    return whole, parts


class _FakeBlock:
    """A rank's H block on the CPU (the oracle's rows) in place of DistCSR."""

    def __init__(self, md, lo, hi, N, D, mv):
        import torch
        self.md, self.lo, self.hi, self.N = md, lo, hi, N
        self.D, self.mv = torch.from_numpy(D), mv
        self.device = torch.device("cpu")
        self.m_local = hi - lo

    def diagonal(self, device=None):
        return self.D

    def operator(self):
        return self.md.RowBlockOperator(self.mv, self.N)


class _Ham64:
    nbits = 64


def _dist_iter(md, dets, lo, hi, rp, ci, nz, mv):
    """dist.asci_iter's host flow on the CPU: reorder, the search (standing
    in: returns the whole space, records what it was given), the
    distributed solve over the rank's oracle block, the gathered vector."""
    import macis_b200 as mb
    N = len(dets)
    D = np.empty(hi - lo)
    rows = np.repeat(np.arange(hi - lo), np.diff(rp))
    on = ci == rows + lo
    D[rows[on]] = nz[on]
    seen = {}

    def search(s, nmax, cd, E, C, norb, H, group=None, screen=None,
               use_net=False):
        seen.update(cd=np.array(cd), C=np.array(C), nmax=nmax)
        return dets

    def build(d, H, tol, group=None):
        assert len(d) == N and tol == np.finfo(float).eps
        return _FakeBlock(md, lo, hi, N, D, mv)
    saved = md.asci_search, md.make_dist_csr_hamiltonian
    md.asci_search, md.make_dist_csr_hamiltonian = search, build
    try:
        s = mb.ASCISettings()
        s.ncdets_max = 20
        m = mb.MCSCFSettings()
        m.ci_max_subspace = 200
        X0 = np.random.default_rng(5).standard_normal(50)
        E, wfn, X = md.asci_iter(s, m, N, -1.0, dets[:50], X0, _Ham64(), 7)
    finally:
        md.asci_search, md.make_dist_csr_hamiltonian = saved
    return dict(E=E, X=X, nwfn=len(wfn), seen=seen)


def _dist_sci_partial_guess(md, dets, lo, hi, rp, ci, nz, mv, rank):
    """dist.selected_ci_diag where only rank 0 passes its rows of a guess
    (rank 1 passes None): every rank must take the diagonal guess."""
    N = len(dets)
    D = np.empty(hi - lo)
    rows = np.repeat(np.arange(hi - lo), np.diff(rp))
    on = ci == rows + lo
    D[rows[on]] = nz[on]

    def build(d, H, tol, group=None):
        return _FakeBlock(md, lo, hi, N, D, mv)
    saved = md.make_dist_csr_hamiltonian
    md.make_dist_csr_hamiltonian = build
    try:
        C_local = np.full(hi - lo, 0.9) if rank == 0 else None
        E, X = md.selected_ci_diag(dets, _Ham64(), np.finfo(float).eps, 200,
                                   1e-8, C_local=C_local)
    finally:
        md.make_dist_csr_hamiltonian = saved
    return dict(E=E, X=md.allgather_rows(X, N).numpy())


class _FakeNet:
    """Network stand-in: the samples a part search recorded."""
    handle = None

    def __init__(self, X, t):
        self.X, self.t = X, t

    def samples(self):
        return self.X, self.t

    def set_sample_targets(self, t):
        self.t = np.asarray(t, dtype=np.float32)


def _screened_split(rank, parts_in):
    import macis_b200 as mb
    from macis_b200 import asci as masci
    from macis_b200 import dist as md
    states, scores, core, ndets_max = parts_in[rank]
    _, t_parts = _sample_targets()
    X = np.arange(len(t_parts[rank]) * 3, dtype=np.uint16).reshape(-1, 3)
    net = _FakeNet(X, t_parts[rank])
    sc = mb.ScreenSettings(network=net)
    seen = {}

    def part_search(s, nmax, cd, E, C, norb, H, index, count, screen=None,
                    use_net=False):
        seen.update(index=index, count=count, screen=screen, use_net=use_net)
        return states, scores

    class _Ham:
        nbits = 64
    orig = masci.asci_search_part
    masci.asci_search_part = part_search
    try:
        got = md.asci_search(mb.ASCISettings(), ndets_max, core, 0.0,
                             np.ones(len(core)), 7, _Ham(), screen=sc,
                             use_net=True)
    finally:
        masci.asci_search_part = orig
    return dict(merged=got, targets=net.t, part=(seen["index"], seen["count"]),
                passed=(seen["screen"] is sc, seen["use_net"]))


def _rank_main(rank, port_no, case, q):
    import datetime

    import torch
    import torch.distributed as dist
    try:
        dist.init_process_group(
            "gloo", init_method=f"tcp://127.0.0.1:{port_no}", rank=rank,
            world_size=WORLD, timeout=datetime.timedelta(seconds=60))
        import oracle
        from macis_b200 import dist as md
        port = oracle.port()
        T, V, dets = _problem()
        N = len(dets)
        hp = port.ham(64, 7, T, V)
        lo, hi = md.local_rows(N)
        (rp, ci, nz), mv = _block_op(port, hp, dets, lo, hi)
        out = {"rank": rank, "lo": lo, "hi": hi}
        if case == "csr":
            full = md.gather_row_blocks(rp, ci, nz)
            out["full"] = full
            out["max"] = md.reduce_max(10.0 * (rank + 1))
            out["sum"] = md.reduce_sum(float(len(ci)))
            xl = torch.arange(lo, hi, dtype=torch.float64)
            out["gathered"] = md.allgather_rows(xl, N).numpy()
        elif case == "davidson":
            D = np.empty(hi - lo)
            rows = np.repeat(np.arange(hi - lo), np.diff(rp))
            on = ci == rows + lo
            D[rows[on]] = nz[on]
            # guess: unit vector on the globally lowest diagonal element
            allD = md.allgather_rows(torch.from_numpy(D), N).numpy()
            g = int(np.argmin(allD))
            X = torch.zeros(hi - lo, dtype=torch.float64)
            if lo <= g < hi:
                X[g - lo] = 1.0
            out["guess_equal"] = bool(torch.equal(
                md.p_diagonal_guess(torch.from_numpy(D), N), X))
            op = md.RowBlockOperator(mv, N)
            it, E = md.p_davidson(hi - lo, 200, op, torch.from_numpy(D),
                                  1e-8, X)
            out.update(it=it, E=E, X=md.allgather_rows(X, N).numpy(),
                       guess=g)
        elif case == "dist_iter":
            out.update(_dist_iter(md, dets, lo, hi, rp, ci, nz, mv))
        elif case == "sci_partial_guess":
            out.update(_dist_sci_partial_guess(md, dets, lo, hi, rp, ci, nz,
                                               mv, rank))
        elif case == "asci":
            parts_in, _ = _asci_parts(port)
            states, scores, core, ndets_max = parts_in[rank]
            out["merged"] = md.merge_search_parts((states, scores), ndets_max,
                                                  core, 64)
            t_whole, t_parts = _sample_targets()
            out["targets"] = md.merge_sample_targets(t_parts[rank])
            # the whole split search with screening: each rank's part search
            # (standing in: the oracle parts) records the same sample rows
            # with its partial targets; every rank ends with the merged
            # result and the whole search's targets in its network
            out["screened"] = _screened_split(rank, parts_in)
            # guess reuse is one decision for all ranks: only rank 0 holds
            # a coefficient above 1/N = 0.01 in the first case
            out["reuse"] = (
                md.reuse_guess([0.5, 0.0] if rank == 0 else [0.0], 100),
                md.reuse_guess([0.005] if rank == 0 else None, 100))
        dist.barrier()
        dist.destroy_process_group()
        q.put(out)
    except Exception:
        q.put({"rank": rank, "error": traceback.format_exc()})


def _run(case):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, p, case, q))
             for r in range(WORLD)]
    for pr in procs:
        pr.start()
    res = {}
    try:
        for _ in range(WORLD):
            o = q.get(timeout=TIMEOUT_S)
            res[o["rank"]] = o
    finally:
        for pr in procs:
            pr.join(timeout=30)
            if pr.is_alive():
                pr.kill()
    for o in res.values():
        assert "error" not in o, o["error"]
    return res


def test_row_blocks_gather_and_reductions(port):
    res = _run("csr")
    T, V, dets = _problem()
    N = len(dets)
    assert (res[0]["lo"], res[0]["hi"]) == (0, N // 2)
    assert (res[1]["lo"], res[1]["hi"]) == (N // 2, N)
    full = port.build_csr(port.ham(64, 7, T, V), dets, dets,
                          np.finfo(float).eps)
    got = res[0]["full"]
    assert np.array_equal(got[0], full[0])
    assert np.array_equal(got[1], full[1])
    assert np.array_equal(got[2], full[2])
    assert res[1]["full"] is None
    for r in range(WORLD):
        assert res[r]["max"] == 20.0
        assert res[r]["sum"] == float(len(full[1]))
        assert np.array_equal(res[r]["gathered"], np.arange(N, dtype=float))


def test_p_davidson_two_ranks_matches_serial(port):
    res = _run("davidson")
    assert all(res[r]["guess_equal"] for r in range(WORLD))  # p_diagonal_guess
    T, V, dets = _problem()
    rp, ci, nz = port.build_csr(port.ham(64, 7, T, V), dets, dets,
                                np.finfo(float).eps)
    X0 = np.zeros(len(dets))
    X0[res[0]["guess"]] = 1.0
    E, it, X = port.davidson(rp, ci, nz, 200, 1e-8, X0)
    for r in range(WORLD):
        assert res[r]["E"] == res[0]["E"]             # same on every rank
        assert abs(res[r]["E"] - E) < 1e-9
        assert abs(res[r]["it"] - it) <= 1
        Xr = res[r]["X"]
        assert abs(abs(Xr @ X) / (np.linalg.norm(Xr) * np.linalg.norm(X))
                   - 1.0) < 1e-10


def test_p_davidson_single_rank_no_group(port):
    """Without a process group the same code is the serial solver."""
    import torch

    from macis_b200 import dist as md
    T, V, dets = _problem()
    N = len(dets)
    assert md.rank_world() == (0, 1)
    (rp, ci, nz), mv = _block_op(port, port.ham(64, 7, T, V), dets, 0, N)
    D = np.asarray([nz[rp[i]:rp[i + 1]][ci[rp[i]:rp[i + 1]] == i][0]
                    for i in range(N)])
    X = torch.zeros(N, dtype=torch.float64)
    X[int(np.argmin(D))] = 1.0
    X0 = X.numpy().copy()
    it, E = md.p_davidson(N, 200, md.RowBlockOperator(mv, N),
                          torch.from_numpy(D), 1e-8, X)
    E_ref, it_ref, _ = port.davidson(rp, ci, nz, 200, 1e-8, X0)
    assert abs(E - E_ref) < 1e-9 and abs(it - it_ref) <= 1
    with pytest.raises(RuntimeError, match="Did Not Converge"):
        md.p_davidson(N, 3, md.RowBlockOperator(mv, N), torch.from_numpy(D),
                      1e-14, torch.from_numpy(X0.copy()))


def test_split_asci_search_merge_two_ranks(port):
    """merge_search_parts over two gloo ranks returns, on both, the merge of
    the whole candidate list (the result of the unsplit search), and
    merge_sample_targets the whole search's recorded targets."""
    from macis_b200.asci import merge_asci_parts
    res = _run("asci")
    parts, (st, rv) = _asci_parts(port)
    _, _, core, ndets_max = parts[0]
    whole = merge_asci_parts([(st, rv)], ndets_max, core, 64)
    assert len(whole) == ndets_max
    for r in range(WORLD):
        assert np.array_equal(res[r]["merged"], whole)
    for r in range(WORLD):
        assert res[r]["reuse"] == (True, False)
        scr = res[r]["screened"]
        assert scr["part"] == (r, WORLD) and scr["passed"] == (True, True)
        assert np.array_equal(scr["merged"], whole)
        assert np.array_equal(scr["targets"], _sample_targets()[0])
    # recorded sample targets: the elementwise maximum over the ranks
    t_whole, _ = _sample_targets()
    for r in range(WORLD):
        assert res[r]["targets"].dtype == np.float32
        assert np.array_equal(res[r]["targets"], t_whole)


def test_dist_asci_iter_two_ranks(port):
    """dist.asci_iter over two gloo ranks (the search and the H blocks stood
    in on the CPU): the search gets the ncdets_max largest |C| in order, the
    distributed solve with the p_diagonal_guess start matches the serial
    Davidson, and every rank holds the same gathered eigenvector."""
    res = _run("dist_iter")
    T, V, dets = _problem()
    X0 = np.random.default_rng(5).standard_normal(50)
    order = np.argsort(-np.abs(X0), kind="stable")[:20]
    rp, ci, nz = port.build_csr(port.ham(64, 7, T, V), dets, dets,
                                np.finfo(float).eps)
    rows = np.repeat(np.arange(len(dets)), np.diff(rp))
    D = nz[ci == rows]
    G = np.zeros(len(dets))
    G[int(np.argmin(D))] = 1.0
    E, it, X = port.davidson(rp, ci, nz, 200, 1e-8, G)
    for r in range(WORLD):
        o = res[r]
        assert np.array_equal(o["seen"]["cd"], dets[:50][order])
        assert np.array_equal(o["seen"]["C"], X0[order])
        assert o["seen"]["nmax"] == len(dets) and o["nwfn"] == len(dets)
        assert o["E"] == res[0]["E"] and abs(o["E"] - E) < 1e-9
        assert np.array_equal(o["X"], res[0]["X"])
        assert abs(abs(o["X"] @ X) / (np.linalg.norm(o["X"]) *
                                      np.linalg.norm(X)) - 1.0) < 1e-10


def test_dist_selected_ci_diag_guess_on_one_rank_only(port):
    """Only rank 0 passes its rows of the guess: both ranks fall back to the
    p_diagonal_guess start together (no rank fails alone while the other
    waits in a collective) and match the serial Davidson from that start."""
    res = _run("sci_partial_guess")
    T, V, dets = _problem()
    rp, ci, nz = port.build_csr(port.ham(64, 7, T, V), dets, dets,
                                np.finfo(float).eps)
    rows = np.repeat(np.arange(len(dets)), np.diff(rp))
    D = nz[ci == rows]
    G = np.zeros(len(dets))
    G[int(np.argmin(D))] = 1.0
    E, it, X = port.davidson(rp, ci, nz, 200, 1e-8, G)
    for r in range(WORLD):
        o = res[r]
        assert o["E"] == res[0]["E"] and abs(o["E"] - E) < 1e-9
        assert np.array_equal(o["X"], res[0]["X"])
