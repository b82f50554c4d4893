"""ASCI search on the GPU against the oracle (bit-exact pairs and selection,
same summation order) and the compiled reference (pair sets identical, rv to
1e-12 relative, top-k identical outside boundary ties)."""
import os

import numpy as np
import pytest

import macis_b200 as mb
import oracle
from cases import embed, fci
from golden_data import constants, water

pytestmark = pytest.mark.gpu
K = constants()


def _core(port, hp, nbits, norb, na, nb, n_core, ndets, seed=0):
    """A core set from one oracle ASCI iteration starting at HF."""
    s = oracle.AsciSettings.default()
    ci = oracle.CiSettings.default()
    hf = port.hf_det(nbits, na, nb)
    E0 = port.matrix_element(hp, hf, hf)[0]
    E, dets, X = port.asci_iter(hp, s, ci, ndets, E0, hf, np.ones(1))
    order = np.argsort(-np.abs(X), kind="stable")
    return dets[order][:n_core], X[order][:n_core], E


def _settings(**kw):
    s = mb.ASCISettings()
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def _tuples(a):
    return set(map(tuple, np.asarray(a).tolist()))


@pytest.fixture(scope="module")
def wcase(port):
    norb, T, V, _ = water()
    hp = port.ham(64, norb, T, V)
    cd, cc, E = _core(port, hp, 64, norb, 5, 5, 100, 800)
    return norb, T, V, hp, cd, cc, E


def test_pairs_bit_exact_vs_oracle_and_ref(port, ref, wcase):
    norb, T, V, hp, cd, cc, E = wcase
    H = mb.HamiltonianGenerator(T, V, 64, norb)
    st, rv = mb.asci_pairs(_settings(), cd, E, cc, H)
    so, ro = port.asci_pairs(hp, oracle.AsciSettings.default(), cd, E, cc)
    assert np.array_equal(st, so)
    assert np.array_equal(rv, ro)                     # same summation order
    sr, rr = ref.asci_pairs(ref.ham(64, norb, T, V),
                            oracle.AsciSettings.default(), cd, E, cc)
    assert np.array_equal(st, sr)
    assert np.all(np.abs(rv - rr) <= 1e-12 * np.abs(rr) + 1e-15 * np.abs(rr).max())


@pytest.mark.parametrize("ndets", [800, 5000, 30000])
def test_search_matches_oracle_and_ref(port, ref, wcase, ndets):
    norb, T, V, hp, cd, cc, E = wcase
    H = mb.HamiltonianGenerator(T, V, 64, norb)
    got = mb.asci_search(_settings(), ndets, cd, E, cc, norb, H)
    exp = port.asci_search(hp, oracle.AsciSettings.default(), ndets, cd, E, cc)
    assert np.array_equal(got, exp)
    r = ref.asci_search(ref.ham(64, norb, T, V), oracle.AsciSettings.default(),
                        ndets, cd, E, cc)
    assert len(r) == len(got)
    diff = _tuples(got) ^ _tuples(r)
    # only boundary ties may differ: their scores equal the k-th score
    if diff:
        st, rv = port.asci_pairs(hp, oracle.AsciSettings.default(), cd, E, cc)
        score = {tuple(s): abs(v) for s, v in zip(st.tolist(), rv)}
        kth = min(score[t] for t in _tuples(got[:-len(cd)]))
        for t in diff:
            assert abs(score[t] - kth) <= 1e-12 * kth


def test_search_128_and_256_bits(port, wcase):
    norb, T, V, hp, cd, cc, E = wcase
    H64 = mb.HamiltonianGenerator(T, V, 64, norb)
    base = mb.asci_search(_settings(), 5000, cd, E, cc, norb, H64)
    for nbits in (128,):
        H = mb.HamiltonianGenerator(T, V, nbits, norb)
        got = mb.asci_search(_settings(), 5000, embed(cd, 64, nbits), E, cc,
                             norb, H)
        assert _tuples(embed(got, nbits, 64)) == _tuples(base)
    # 256 bits (no reference): oracle restatement on a smaller problem
    T2, V2, d2 = fci(10, 3, 3, 64, seed=2)
    hp2 = port.ham(256, 10, T2, V2)
    cd2 = embed(d2[:40], 64, 256)
    c2 = np.linspace(1.0, 0.1, 40)
    H2 = mb.HamiltonianGenerator(T2, V2, 256)
    E2 = -1.0
    got = mb.asci_search(_settings(), 1000, cd2, E2, c2, 10, H2)
    exp = port.asci_search(hp2, oracle.AsciSettings.default(), 1000, cd2, E2, c2)
    assert np.array_equal(got, exp)


def test_search_edge_cases(port, wcase):
    norb, T, V, hp, cd, cc, E = wcase
    H = mb.HamiltonianGenerator(T, V, 64, norb)
    os_ = oracle.AsciSettings.default
    # just singles
    got = mb.asci_search(_settings(just_singles=True), 300, cd, E, cc, norb, H)
    exp = port.asci_search(hp, os_(just_singles=1), 300, cd, E, cc)
    assert np.array_equal(got, exp)
    # loose screening threshold
    got = mb.asci_search(_settings(h_el_tol=1e-3), 2000, cd, E, cc, norb, H)
    exp = port.asci_search(hp, os_(h_el_tol=1e-3), 2000, cd, E, cc)
    assert np.array_equal(got, exp)
    # k larger than the candidate count: everything kept
    got = mb.asci_search(_settings(), 10 ** 7, cd[:3], E, cc[:3], norb, H)
    exp = port.asci_search(hp, os_(), 10 ** 7, cd[:3], E, cc[:3])
    assert np.array_equal(got, exp)
    # single core determinant, empty core list
    got = mb.asci_search(_settings(), 50, cd[:1], E, cc[:1], norb, H)
    assert np.array_equal(got, port.asci_search(hp, os_(), 50, cd[:1], E, cc[:1]))
    got = mb.asci_search(_settings(), 50, cd[:0], E, cc[:0], norb, H)
    assert len(got) == 0


def test_search_partitioned_ranges(port, wcase, monkeypatch):
    """Splitting the candidates into hash ranges (forced small here) gives
    the unpartitioned result exactly: each range holds complete sums and the
    running top-k keeps every tie until the end."""
    norb, T, V, hp, cd, cc, E = wcase
    H = mb.HamiltonianGenerator(T, V, 64, norb)
    one = mb.asci_search(_settings(), 5000, cd, E, cc, norb, H)
    assert mb.last_search_stats(H)["batches"] == 1
    net = mb.ScreeningNetwork(nbits=64, seed=0)
    rec = mb.ScreenSettings(network=net, max_samples=10 ** 6)
    mb.asci_search(_settings(), 5000, cd, E, cc, norb, H, screen=rec)
    X1, t1 = net.samples()
    monkeypatch.setenv("MACIS_B200_ASCI_BATCH_PAIRS", "50000")
    got = mb.asci_search(_settings(), 5000, cd, E, cc, norb, H)
    st = mb.last_search_stats(H)
    assert st["batches"] > 1
    assert np.array_equal(got, one)
    exp = port.asci_search(hp, oracle.AsciSettings.default(), 5000, cd, E, cc)
    assert np.array_equal(got, exp)
    # per-unit recorded targets are the maximum over all ranges
    mb.asci_search(_settings(), 5000, cd, E, cc, norb, H, screen=rec)
    X2, t2 = net.samples()
    assert np.array_equal(X1, X2) and np.array_equal(t1, t2)
    # tiny top-k: ties resolved towards smaller determinants in both modes
    got_small = mb.asci_search(_settings(), len(cd) + 7, cd, E, cc, norb, H)
    monkeypatch.delenv("MACIS_B200_ASCI_BATCH_PAIRS")
    one_small = mb.asci_search(_settings(), len(cd) + 7, cd, E, cc, norb, H)
    assert np.array_equal(got_small, one_small)


def test_water_grow_refine_golden():
    norb, T, V, _ = water()
    H = mb.HamiltonianGenerator(T, V, 64, norb)
    s = _settings(ntdets_max=K["water_asci_ntdets_max"])
    ci = mb.MCSCFSettings()
    hf = mb.canonical_hf_determinant(5, 5, 64)
    E0 = H.matrix_element(hf, hf)
    E, dets, X = mb.asci_grow(s, ci, E0, hf, np.ones(1), H, norb)
    assert len(dets) == 10000 and abs(X @ X - 1) < 1e-10
    assert abs(E - K["water_asci_grow_e0"]) < 1e-8
    E, dets, X = mb.asci_refine(s, ci, E, dets, X, H, norb)
    assert len(dets) == 10000
    assert abs(E - K["water_asci_refine_e0"]) < 1e-7


@pytest.mark.parametrize("nparts", [1, 2, 4])
def test_split_search_merges_to_whole(port, wcase, monkeypatch, nparts):
    """A search split into parts by the alpha-string bins (one process per
    GPU in a distributed run; run one after another here) merges to the
    whole search's result exactly -- with one range per part, with several
    (small range cap), and with a small top-k whose ties are resolved only in
    the merge."""
    norb, T, V, hp, cd, cc, E = wcase
    H = mb.HamiltonianGenerator(T, V, 64, norb)

    def split(ndets_max):
        parts = [mb.asci_search_part(_settings(), ndets_max, cd, E, cc, norb,
                                     H, i, nparts) for i in range(nparts)]
        assert sum(len(p[1]) for p in parts) > 0
        return mb.merge_asci_parts(parts, ndets_max, cd, 64)

    for ndets_max in (5000, len(cd) + 7):
        whole = mb.asci_search(_settings(), ndets_max, cd, E, cc, norb, H)
        assert np.array_equal(split(ndets_max), whole)
    monkeypatch.setenv("MACIS_B200_ASCI_BATCH_PAIRS", "50000")
    got = split(5000)
    assert mb.last_search_stats(H)["batches"] >= 1
    exp = port.asci_search(hp, oracle.AsciSettings.default(), 5000, cd, E, cc)
    assert np.array_equal(got, exp)


def test_screened_split_search_matches_whole(wcase):
    """Learned screening over a split search (parts run one after another
    here): a recording part stores the whole search's sample rows, and the
    elementwise maximum of the parts' targets is the whole search's targets;
    networks trained on them stay equal to the one-GPU network, and a pruning
    search split into parts merges to the screened whole search."""
    norb, T, V, hp, cd, cc, E = wcase
    H = mb.HamiltonianGenerator(T, V, 64, norb)
    nparts, ndets_max = 3, 5000
    nets = [mb.ScreeningNetwork(nbits=64, seed=0) for _ in range(nparts + 1)]
    scr = [mb.ScreenSettings(network=n, max_samples=10 ** 6) for n in nets]

    def split(use_net):
        parts = [mb.asci_search_part(_settings(), ndets_max, cd, E, cc, norb,
                                     H, i, nparts, screen=scr[i + 1],
                                     use_net=use_net) for i in range(nparts)]
        return mb.merge_asci_parts(parts, ndets_max, cd, 64)

    whole = mb.asci_search(_settings(), ndets_max, cd, E, cc, norb, H,
                           screen=scr[0])
    Xw, tw = nets[0].samples()
    assert len(tw) > 1000
    assert np.array_equal(split(False), whole)
    got = [n.samples() for n in nets[1:]]
    for X, t in got:
        assert np.array_equal(X, Xw)
    tmax = np.maximum.reduce([t for _, t in got])
    assert np.array_equal(tmax, tw)
    assert not all(np.array_equal(t, tw) for _, t in got)
    for n in nets[1:]:
        n.set_sample_targets(tmax)
    for sc in scr:
        sc.network.clamp_samples(sc.clamp_quantile)
        sc.network.train(None, None, sc.epochs, sc.batch, sc.lr,
                         sc.seed + sc.searches)
    P0 = nets[0].params
    for n in nets[1:]:
        assert np.array_equal(n.params, P0)
    for sc in scr:
        sc.train = False
    whole2 = mb.asci_search(_settings(), ndets_max, cd, E, cc, norb, H,
                            screen=scr[0], use_net=True)
    st = mb.last_search_stats(H)
    assert 0 < st["units_kept"] < st["units_total"]
    assert not np.array_equal(whole2, whole)
    assert np.array_equal(split(True), whole2)
    with pytest.raises(mb.MacisError, match="recorded sample count"):
        nets[1].set_sample_targets(tmax[:-1])


def test_onesweep_sort_matches_classic_passes(monkeypatch):
    """The candidate sort with one-sweep digit passes (decoupled look-back,
    MACIS_B200_SORT_ONESWEEP=1) against the classic histogram / scan /
    scatter passes (the default), and with candidate ranges split by bin
    into separately sorted groups: identical accumulated candidates and
    scores, and identical selections, on an n = 48 bitset<128> core set of
    300 determinants (about 8e7 contributions)."""
    from cases import core_set
    monkeypatch.setenv("MACIS_B200_SORT_ONESWEEP", "1")
    n, k = 48, 12
    T, V = mb.synthetic_integrals(n, 0)
    cd, C = core_set(n, k, 300, 128, nalpha=80, top=40)
    H = mb.HamiltonianGenerator(T, V, 128)
    E0 = float(H.matrix_element(cd[:1], cd[:1])) - 0.5
    s1, r1 = mb.asci_pairs(_settings(), cd, E0, C, H)
    sel1 = mb.asci_search(_settings(), 50000, cd, E0, C, n, H)
    assert mb.last_search_stats(H)["raw_pairs"] > 5e7
    # a range split by alpha-string bin into sort groups (forced small
    # here; large searches do it above 1e9 records per range)
    monkeypatch.setenv("MACIS_B200_ASCI_SORT_GROUP", "3000000")
    monkeypatch.setenv("MACIS_B200_ASCI_BATCH_PAIRS", "40000000")
    selg = mb.asci_search(_settings(), 50000, cd, E0, C, n, H)
    assert mb.last_search_stats(H)["batches"] >= 2
    assert np.array_equal(selg, sel1)
    monkeypatch.delenv("MACIS_B200_ASCI_SORT_GROUP")
    monkeypatch.delenv("MACIS_B200_ASCI_BATCH_PAIRS")
    monkeypatch.delenv("MACIS_B200_SORT_ONESWEEP")
    s0, r0 = mb.asci_pairs(_settings(), cd, E0, C, H)
    sel0 = mb.asci_search(_settings(), 50000, cd, E0, C, n, H)
    assert np.array_equal(s1, s0) and np.array_equal(r1, r0)
    assert np.array_equal(sel1, sel0)


@pytest.mark.parametrize("nbits,n,k,ncore,nalpha,top",
                         [(128, 48, 12, 300, 80, 40), (256, 100, 20, 8, 6, 4)])
def test_ranked_keys_and_alpha_lists_match_plain_search(monkeypatch, nbits, n,
                                                        k, ncore, nalpha, top):
    """The candidate paths of a large search against the plain one (one
    range, candidates sorted by their determinant bitsets,
    MACIS_B200_ASCI_RANKS=0): candidates sorted by ranked keys (alpha and
    beta string ranks; the default above 2^22 contributions), and candidate
    ranges that take their alpha-double counts and contributions from
    per-alpha-string lists (the default once a search needs several ranges)
    for the most frequent alpha strings only (MACIS_B200_ASCI_ALPHA_LISTS=3)
    or test every contribution's bin (MACIS_B200_ASCI_ALPHA_LISTS=0), with a
    range cap that leaves every range whole and one small enough to split
    the heaviest alpha-string bin by beta string. Identical accumulated
    candidates and scores, selections (exact and screened) and recorded
    unit targets."""
    from cases import core_set
    T, V = mb.synthetic_integrals(n, 0)
    cd, C = core_set(n, k, ncore, nbits, nalpha=nalpha, top=top)
    H = mb.HamiltonianGenerator(T, V, nbits)
    E0 = float(H.matrix_element(cd[:1], cd[:1])) - 0.5
    keep = mb.ScreenSettings(network=mb.ScreeningNetwork(nbits=nbits, seed=0),
                             keep_frac=0.4, explore_frac=0.0, train=False)
    rec = mb.ScreenSettings(network=mb.ScreeningNetwork(nbits=nbits, seed=1),
                            max_samples=200000)

    def run(ranks, lists=None, cap=None):
        monkeypatch.setenv("MACIS_B200_ASCI_RANKS", ranks)
        if lists is None:
            monkeypatch.delenv("MACIS_B200_ASCI_ALPHA_LISTS", raising=False)
        else:
            monkeypatch.setenv("MACIS_B200_ASCI_ALPHA_LISTS", lists)
        if cap is None:
            monkeypatch.delenv("MACIS_B200_ASCI_BATCH_PAIRS", raising=False)
        else:
            monkeypatch.setenv("MACIS_B200_ASCI_BATCH_PAIRS", str(cap))
        exact = mb.asci_search(_settings(), 40000, cd, E0, C, n, H)
        st = mb.last_search_stats(H)
        scr = mb.asci_search(_settings(), 40000, cd, E0, C, n, H, screen=keep,
                             use_net=True)
        rec.searches = 0  # the same sample draw in every run
        mb.asci_search(_settings(), 40000, cd, E0, C, n, H, screen=rec)
        return exact, scr, rec.network.samples(), st

    def same(a, b):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        assert np.array_equal(a[2][0], b[2][0])
        assert np.array_equal(a[2][1], b[2][1])

    plain = run("0")
    st = plain[3]
    assert st["batches"] == 1 and st["key_bits"] == 0
    assert st["alpha_strings"] == 0
    ranked = run("1")
    assert 0 < ranked[3]["key_bits"] < 2 * n
    same(ranked, plain)
    monkeypatch.setenv("MACIS_B200_ASCI_RANKS", "1")
    pr = mb.asci_pairs(_settings(), cd, E0, C, H)
    monkeypatch.setenv("MACIS_B200_ASCI_RANKS", "0")
    pp = mb.asci_pairs(_settings(), cd, E0, C, H)
    assert np.array_equal(pr[0], pp[0]) and np.array_equal(pr[1], pp[1])
    raw = st["raw_pairs"]
    for cap in (raw // 12, raw // 150):
        for ranks, lists in (("1", None), ("1", "0"), ("0", None), ("1", "3")):
            got = run(ranks, lists, cap)
            assert got[3]["batches"] > 3
            assert (got[3]["alpha_strings"] > 0) == (lists != "0")
            if lists == "3":
                assert got[3]["alpha_strings"] == 3
            assert (got[3]["key_bits"] > 0) == (ranks == "1")
            same(got, plain)
