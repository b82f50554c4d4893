"""Learned screening network on the GPU: tcgen05 forward and backward against
the CPU oracle (oracle/screen_oracle.py), Adam, online training from the
ASCI search's recorded samples, and what the trained network gains over
the exact search and over an untrained network at the same budget."""
import time

import numpy as np
import pytest

import macis_b200 as mb
import oracle
from oracle import screen_oracle as so

pytestmark = pytest.mark.gpu


def _rand_inputs(rng, n, din, nbits_cols):
    """BF16 bit patterns: 0/1 occupation columns + normal features."""
    X = np.zeros((n, din), dtype=np.float32)
    X[:, :nbits_cols] = rng.integers(0, 2, (n, nbits_cols))
    X[:, nbits_cols:] = rng.normal(0, 1, (n, din - nbits_cols))
    return so.bf16_bits(X)


def _rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / max(
        np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("din,n", [(192, 300), (320, 129), (192, 1)])
def test_forward_matches_oracle(din, n):
    rng = np.random.default_rng(din + n)
    net = mb.ScreeningNetwork(din=din, seed=5)
    P = net.params.astype(np.float64)
    # non-zero biases exercise the epilogues
    off, _ = so.layout(din)
    for k in ("b1", "b2", "b3"):
        a, b = off[k]
        P[a:b] = rng.normal(0, 0.1, b - a)
    net.params = P.astype(np.float32)
    Xb = _rand_inputs(rng, n, din, din - 64)
    y = net.forward(Xb)
    yo, _ = so.forward(net.params.astype(np.float64),
                       so.bf16_value(Xb).astype(np.float64), din)
    assert np.all(np.isfinite(y))
    assert np.max(np.abs(y - yo)) <= 1e-4 * max(1.0, np.max(np.abs(yo)))


@pytest.mark.parametrize("din,n", [(192, 517), (320, 256)])
def test_gradients_match_oracle(din, n):
    """Backward kernels (three tcgen05 GEMMs + reductions) against the
    oracle with the same BF16 rounding points; per block relative L2."""
    rng = np.random.default_rng(7 + din)
    net = mb.ScreeningNetwork(din=din, seed=11)
    Xb = _rand_inputs(rng, n, din, din - 64)
    t = rng.normal(0, 1, n).astype(np.float32)
    g, loss = net.gradients(Xb, t)
    go, lo = so.gradients(net.params.astype(np.float64),
                          so.bf16_value(Xb).astype(np.float64), t, din)
    assert abs(loss - lo) <= 1e-5 * max(1.0, abs(lo))
    off, _ = so.layout(din)
    for k, (a, b) in off.items():
        assert _rel(g[a:b], go[a:b]) < 2e-3, k


def test_adam_steps_match_oracle():
    """Three full-batch Adam steps: the GPU update follows the oracle's."""
    din, n, lr = 192, 384, 1e-3
    rng = np.random.default_rng(1)
    net = mb.ScreeningNetwork(din=din, seed=3)
    P0 = net.params.astype(np.float64)
    Xb = _rand_inputs(rng, n, din, 128)
    t = rng.normal(0, 1, n).astype(np.float32)
    net.train(Xb, t, epochs=3, batch=n, lr=lr)
    P1 = net.params.astype(np.float64)
    P, M, V = P0.copy(), np.zeros_like(P0), np.zeros_like(P0)
    Xf = so.bf16_value(Xb).astype(np.float64)
    for step in range(1, 4):
        G, _ = so.gradients(P.astype(np.float32).astype(np.float64), Xf, t,
                            din)
        P, M, V = so.adam(P, G, M, V, step, lr)
    d_gpu, d_or = P1 - P0, P - P0
    assert _rel(d_gpu, d_or) < 0.05
    assert np.max(np.abs(d_gpu)) <= 3 * lr * 1.01


def test_training_fits_a_teacher():
    """Adam on the GPU fits targets made by another network."""
    din, n = 192, 8192
    rng = np.random.default_rng(2)
    teacher = mb.ScreeningNetwork(din=din, seed=99)
    Xb = _rand_inputs(rng, n, din, 128)
    t = teacher.forward(Xb)
    t = (t - t.mean()) / t.std()
    net = mb.ScreeningNetwork(din=din, seed=1)
    y0 = net.forward(Xb)
    l0 = float(np.mean((y0 - t) ** 2) / 2)
    l1 = net.train(Xb, t, epochs=20, batch=512, lr=1e-3)
    y1 = net.forward(Xb)
    l1b = float(np.mean((y1 - t) ** 2) / 2)
    assert l1 < 0.25 * l0 and l1b < 0.25 * l0


def _ham(norb, nbits, seed=0):
    T, V = mb.synthetic_integrals(norb, seed)
    return T, V, mb.HamiltonianGenerator(T, V, nbits)


@pytest.mark.parametrize("nbits,norb,na,nb", [(64, 10, 3, 3), (128, 14, 4, 3),
                                              (256, 70, 3, 2)])
def test_unit_features_match_oracle(port, nbits, norb, na, nb):
    T, V, H = _ham(norb, nbits, seed=4)
    hp = port.ham(nbits, norb, T, V)
    hf = mb.canonical_hf_determinant(na, nb, nbits)
    dets = mb.generate_cisd_hilbert_space(norb, hf, nbits)[:7]
    rng = np.random.default_rng(0)
    C = rng.normal(0, 1, len(dets))
    E0 = -3.21
    X, U = mb.unit_features(H, dets, E0, C)
    Xo = so.unit_features(port, hp, nbits, norb, dets, E0, C, V)
    assert U == len(Xo) == len(X)
    nbc = mb.unit_width(nbits) - 64
    Xg = so.bf16_value(X)
    assert np.array_equal(Xg[:, :nbc], Xo[:, :nbc])
    # features: equal up to one BF16 rounding step (FP64 summation order)
    diff = np.abs(Xg[:, nbc:] - Xo[:, nbc:])
    assert np.all(diff <= 2.0 ** -7 * np.abs(Xo[:, nbc:]) + 1e-30)
    assert np.mean(diff == 0) > 0.99


def test_search_records_samples(port):
    norb, nbits = 12, 64
    T, V, H = _ham(norb, nbits, seed=1)
    hf = mb.canonical_hf_determinant(4, 4, nbits)
    dets = mb.generate_cisd_hilbert_space(norb, hf, nbits)
    C = np.random.default_rng(0).normal(0, 1, len(dets))
    C[0] = 10.0
    E0 = -5.0
    s = mb.ASCISettings(h_el_tol=1e-8)
    net = mb.ScreeningNetwork(nbits=nbits, seed=0)
    scr = mb.ScreenSettings(network=net, max_samples=10 ** 6, train=True)
    exact = mb.asci_search(s, 2000, dets, E0, C, norb, H)
    rec = mb.asci_search(s, 2000, dets, E0, C, norb, H, screen=scr)
    assert np.array_equal(exact, rec)  # recording does not change the search
    st = mb.last_search_stats(H)
    Xs, ts = net.samples()
    na, nva = 4, norb - 4
    assert st["units_total"] == len(dets) * (2 + 3 * na * nva)
    assert st["samples"] == st["units_total"] == len(ts)
    # all units recorded, in unit order: rows equal the unit inputs
    Xu, U = mb.unit_features(H, dets, E0, C)
    assert np.array_equal(Xs, Xu)
    # the largest target is that of the largest |rv| of any raw contribution
    hp = port.ham(nbits, norb, T, V)
    raw_states, raw_rv = port.asci_pairs(hp, oracle.AsciSettings.default(
        h_el_tol=1e-8), dets, E0, C, accumulate=False)
    assert np.isfinite(ts).all()
    want = so.unit_targets([np.abs(raw_rv).max()])[0]
    assert abs(ts.max() - want) <= 1e-5 * abs(want)


def _grow(H, norb, nbits, na, nb, ndets, ncore, screen=None):
    s = mb.ASCISettings(ntdets_max=ndets, ntdets_min=100, ncdets_max=ncore,
                        h_el_tol=1e-8, grow_factor=4)
    m = mb.MCSCFSettings(ci_max_subspace=60, davidson_restart_keep=8,
                         davidson_max_iter=400)
    hf = mb.canonical_hf_determinant(na, nb, nbits)
    E0 = float(H.matrix_element(hf, hf))
    return s, m, mb.asci_grow(s, m, E0, hf, [1.0], H, norb, screen=screen)


def test_trained_network_gains_over_the_search_without_it():
    """At an equal budget of exactly scored units (20% of the full search's),
    the online-trained network finds a better determinant set than the
    method without it -- the exact search over a core set cut to the same
    unit count -- and than an untrained network. Measured: top-k recall
    against the full exact search and the variational energy at equal
    determinant count; raw contributions show the work saved."""
    norb, nbits, na, nb = 16, 64, 5, 5
    T, V, H = _ham(norb, nbits, seed=2)
    net = mb.ScreeningNetwork(nbits=nbits, seed=0)
    scr = mb.ScreenSettings(network=net, warmup_searches=10 ** 6,
                            max_samples=400000)
    s, m, (E, dets, X) = _grow(H, norb, nbits, na, nb, 6000, 1500, scr)
    assert net.trained_steps >= 3
    order = np.argsort(-np.abs(X), kind="stable")
    core, Cc = dets[order][:1500], X[order][:1500]
    k = 24000
    t0 = time.perf_counter()
    exact = mb.asci_search(s, k, core, E, Cc, norb, H)
    t_exact = time.perf_counter() - t0
    st_exact = mb.last_search_stats(H)

    def screened(network):
        sc = mb.ScreenSettings(network=network, keep_frac=0.2,
                               explore_frac=0.0, train=False)
        t0 = time.perf_counter()
        out = mb.asci_search(s, k, core, E, Cc, norb, H, screen=sc,
                             use_net=True)
        return out, mb.last_search_stats(H), time.perf_counter() - t0

    learned, st_l, t_l = screened(net)
    fresh, st_f, _ = screened(mb.ScreeningNetwork(nbits=nbits, seed=123))
    # without the network: every unit of a smaller core set (same units)
    ncut = 300
    cut = mb.asci_search(s, k, core[:ncut], E, Cc[:ncut], norb, H)
    st_c = mb.last_search_stats(H)
    assert st_c["units_total"] == st_exact["units_total"] * ncut // 1500
    assert st_l["units_kept"] <= 0.2 * st_l["units_total"] + 2

    ea = set(map(tuple, exact.tolist()))

    def recall(a):
        return len(ea & set(map(tuple, np.asarray(a).tolist()))) / len(ea)

    def energy(d):
        return mb.selected_ci_diag(d, H, m.ci_matel_tol, 60, 1e-8,
                                   restart_keep=8, max_iter=400)[0]

    Ee = energy(exact)
    r_l, r_f, r_c = recall(learned), recall(fresh), recall(cut)
    dl, df, dc = energy(learned) - Ee, energy(fresh) - Ee, energy(cut) - Ee
    print(f"\nscreening n={norb}: units {st_l['units_kept']}/"
          f"{st_l['units_total']}; raw pairs learned {st_l['raw_pairs']} "
          f"cut-core {st_c['raw_pairs']} exact {st_exact['raw_pairs']}; "
          f"recall learned {r_l:.4f} cut-core {r_c:.4f} untrained {r_f:.4f}; "
          f"dE learned {dl:.3e} cut-core {dc:.3e} untrained {df:.3e} Eh; "
          f"search {t_l * 1e3:.1f} ms vs exact {t_exact * 1e3:.1f} ms")
    assert len(learned) == len(exact) == len(fresh) == len(cut)
    assert st_l["raw_pairs"] <= 0.5 * st_exact["raw_pairs"]
    assert r_l >= r_c + 0.05 and r_l >= r_f + 0.15
    assert dl < 0.7 * dc and dl < df


def test_recall_check_keeps_exact_selections():
    """Pruning searches small enough for the recall check
    (ScreenSettings.check_units_max) also run exactly and keep the exact
    selection: a screened grow follows the unscreened grow determinant for
    determinant, the measured recalls are logged, and keep_frac doubles
    after every check below recall_target (above 1 here, so every check
    fails) until pruning stops at keep_frac 1; a check that passes halves
    keep_frac down to keep_min."""
    norb, nbits, na, nb = 16, 64, 5, 5
    T, V, H = _ham(norb, nbits, seed=2)
    _, _, (E0, d0, X0) = _grow(H, norb, nbits, na, nb, 6000, 1500)
    scr = mb.ScreenSettings(network=mb.ScreeningNetwork(nbits=nbits, seed=0),
                            min_units=0, recall_target=1.01,
                            check_units_max=10 ** 12)
    _, m, (E1, d1, X1) = _grow(H, norb, nbits, na, nb, 6000, 1500, scr)
    assert np.array_equal(d1, d0) and abs(E1 - E0) < 1e-9
    log = m.iteration_log
    checks = [it["recall_check"] for it in log if it["screened"]]
    assert len(checks) >= 2 and all(0.0 <= r <= 1.0 for r in checks)
    assert scr.keep_frac == min(1.0, 0.2 * 2 ** len(checks))
    assert all(it["recall_check"] is None for it in log if not it["screened"])
    # a check that passes leaves keep_frac alone
    sc2 = mb.ScreenSettings(network=scr.network, recall_target=1e-9,
                            min_units=0, check_units_max=10 ** 12)
    sc2.searches = sc2.warmup_searches
    s = mb.ASCISettings(ntdets_max=6000, ntdets_min=100, ncdets_max=1500,
                        h_el_tol=1e-8)
    m2 = mb.MCSCFSettings(ci_max_subspace=60, davidson_restart_keep=8,
                          davidson_max_iter=400)
    mb.asci_iter(s, m2, 6000, E1, d1, X1, H, norb, sc2)
    assert m2.iteration_log[-1]["screened"]
    assert m2.iteration_log[-1]["recall_check"] is not None
    assert sc2.keep_frac == 0.2
    # a check that passes tries halving keep_frac, down to keep_min, while
    # the trial searches keep the recall (here always: a tiny target)
    sc3 = mb.ScreenSettings(network=scr.network, recall_target=1e-9,
                            keep_frac=0.8, keep_min=0.2, min_units=0,
                            check_units_max=10 ** 12)
    sc3.searches = sc3.warmup_searches
    E3, d3, _ = mb.asci_iter(s, m2, 6000, E1, d1, X1, H, norb, sc3)
    assert sc3.keep_frac == 0.2
    # the selection is still the exact search's
    E4, d4, _ = mb.asci_iter(s, m2, 6000, E1, d1, X1, H, norb, None)
    assert np.array_equal(d3, d4) and abs(E3 - E4) < 1e-9
