"""ASCI drivers on the B200.

* ``ASCISettings`` / ``MCSCFSettings`` -- include/macis/asci/
  determinant_search.hpp:34-51 and include/macis/util/mcscf.hpp:15-30
* ``asci_search``  -- determinant_search.hpp:395-663 (GPU search)
* ``reorder_ci_on_coeff`` -- asci/determinant_sort.hpp:19-37 (stable)
* ``asci_iter``    -- asci/iteration.hpp:17-68
* ``asci_grow``    -- asci/grow.hpp:17-171 (the natural-orbital rotation
  branch, grow_with_rot, is not part of this path)
* ``asci_refine``  -- asci/refine.hpp:15-66

The search returns the top-k states in ascending determinant order followed
by the core determinants; the reference returns them in nth_element order.
"""
import ctypes as ct
import dataclasses
import logging
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import LIB, check
from .solvers import FP64, selected_ci_diag

__all__ = ["ASCISettings", "MCSCFSettings", "asci_search", "asci_pairs",
           "asci_search_part", "merge_asci_parts",
           "asci_iter", "asci_grow", "asci_refine", "reorder_ci_on_coeff",
           "last_search_stats", "topk_recall"]


@dataclass
class ASCISettings:
    ntdets_max: int = 100000
    ntdets_min: int = 100
    ncdets_max: int = 100
    h_el_tol: float = 1e-8
    rv_prune_tol: float = 1e-8
    pair_size_max: int = 500000000
    just_singles: bool = False
    grow_factor: int = 8
    max_refine_iter: int = 6
    refine_energy_tol: float = 1e-6
    grow_with_rot: bool = False
    rot_size_start: int = 1000
    constraint_level: int = 2

    def c_struct(self):
        return _lib.AsciSettingsC(
            int(self.ntdets_max), int(self.ntdets_min), int(self.ncdets_max),
            float(self.h_el_tol), float(self.rv_prune_tol),
            int(self.pair_size_max), int(bool(self.just_singles)), 0,
            int(self.grow_factor), int(self.max_refine_iter),
            float(self.refine_energy_tol))


@dataclass
class MCSCFSettings:
    ci_res_tol: float = 1e-8
    ci_max_subspace: int = 20
    ci_matel_tol: float = float(np.finfo(np.float64).eps)
    precision: str = FP64  # FP64 or MIXED Davidson inside asci_iter
    # thick restart of the Davidson (0: the reference solver, no restart)
    davidson_restart_keep: int = 0
    davidson_max_iter: int = 0
    iteration_log: list = field(default_factory=list)


def reorder_ci_on_coeff(dets, C):
    """Sort by |C| descending; equal magnitudes keep their order."""
    order = np.argsort(-np.abs(C), kind="stable")
    return dets[order], C[order]


def _dets(d, nbits):
    return np.ascontiguousarray(d, dtype=np.uint64).reshape(-1, nbits // 64)


def asci_search(asci_settings, ndets_max, cdets, E_ASCI, C, norb, ham_gen,
                screen=None, use_net=False):
    """New determinant list: top-(ndets_max - ncdets) contributions then the
    core determinants (determinant_search.hpp:395-663).

    screen: optional ScreenSettings (macis_b200.screening). Its network
    records (unit input, exact log score) samples of the units this search
    scores; with use_net it also prunes units by prediction first."""
    log = logging.getLogger("asci_search")
    cdets = _dets(cdets, ham_gen.nbits)
    C = np.ascontiguousarray(C, dtype=np.float64)[:len(cdets)]
    s = asci_settings.c_struct()
    out = np.empty((int(ndets_max) + len(cdets), ham_gen.nbits // 64),
                   dtype=np.uint64)
    nout = ct.c_size_t()
    if screen is not None and screen.network is not None:
        sc = screen.c_struct(use_net)
        check(LIB.macis_b200_asci_search_screened(
            ham_gen.handle, ct.byref(s), ct.byref(sc), int(ndets_max),
            cdets.ctypes.data, len(cdets), float(E_ASCI), C.ctypes.data,
            out.ctypes.data, ct.byref(nout), 0))
        screen.searches += 1
    else:
        check(LIB.macis_b200_asci_search(ham_gen.handle, ct.byref(s),
                                         int(ndets_max), cdets.ctypes.data,
                                         len(cdets), float(E_ASCI),
                                         C.ctypes.data, out.ctypes.data,
                                         ct.byref(nout), 0))
    st = last_search_stats(ham_gen)
    log.info("  * ASCI Kept %d Pairs; %d unique; PAIR_DUR = %.2e s, "
             "SORT_ACC_DUR = %.2e s, ASCI_SEARCH DUR = %.2e s",
             st["raw_pairs"], st["unique_pairs"], st["pairs_ms"] / 1e3,
             st["sort_ms"] / 1e3, st["total_ms"] / 1e3)
    return out[:nout.value]


def asci_search_part(asci_settings, ndets_max, cdets, E_ASCI, C, norb,
                     ham_gen, part_index, part_count, screen=None,
                     use_net=False):
    """One part of an exact search split over part_count processes
    (macis_b200_asci_search_part): (states, scores) of the part's candidates,
    cut at the (ndets_max - ncdets)-th |score| with every tie kept.
    merge_asci_parts of all parts gives asci_search's result.

    screen / use_net as in asci_search: parts whose networks are equal keep
    the same units, so the merge gives the screened whole search; recorded
    targets cover the part's bins only (their elementwise maximum over the
    parts is the whole search's, see dist.merge_sample_targets)."""
    cdets = _dets(cdets, ham_gen.nbits)
    C = np.ascontiguousarray(C, dtype=np.float64)[:len(cdets)]
    s = asci_settings.c_struct()
    n = ct.c_size_t()
    if screen is not None and screen.network is not None:
        sc = screen.c_struct(use_net)
        check(LIB.macis_b200_asci_search_part_screened(
            ham_gen.handle, ct.byref(s), ct.byref(sc), int(ndets_max),
            cdets.ctypes.data, len(cdets), float(E_ASCI), C.ctypes.data,
            int(part_index), int(part_count), ct.byref(n), 0))
        screen.searches += 1
    else:
        check(LIB.macis_b200_asci_search_part(
            ham_gen.handle, ct.byref(s), int(ndets_max), cdets.ctypes.data,
            len(cdets), float(E_ASCI), C.ctypes.data, int(part_index),
            int(part_count), ct.byref(n), 0))
    W = ham_gen.nbits // 64
    st = np.empty((max(n.value, 1), W), dtype=np.uint64)
    sc = np.empty(max(n.value, 1))
    check(LIB.macis_b200_asci_part_results(ham_gen.handle, st.ctypes.data,
                                           sc.ctypes.data))
    return st[:n.value], sc[:n.value]


def merge_asci_parts(parts, ndets_max, cdets, nbits):
    """asci_search's result from the parts of a split search: the union of
    the parts' (states, scores) ordered by |score| descending then by
    determinant ascending (bitset order, most significant word first), cut
    at ndets_max - ncdets, listed in ascending determinant order, followed by
    the core determinants in their input order. ndets_max - ncdets is size_t
    arithmetic, as in the search: with fewer slots than core determinants
    nothing is cut, and a result beyond ndets_max raises ECAPACITY, as the
    search does."""
    W = nbits // 64
    cdets = _dets(cdets, nbits)
    st = [np.asarray(p[0], dtype=np.uint64).reshape(-1, W) for p in parts]
    sc = [np.asarray(p[1], dtype=np.float64).ravel() for p in parts]
    st = np.concatenate(st) if st else np.zeros((0, W), dtype=np.uint64)
    sc = np.concatenate(sc) if sc else np.zeros(0)
    k = int(ndets_max) - len(cdets)
    if k < 0:
        k += 1 << 64   # size_t arithmetic, as the search (determinant_search.hpp:547)
    if len(sc) > k:
        # lexsort: the last key is the primary one
        order = np.lexsort(tuple(st[:, w] for w in range(W)) + (-np.abs(sc),))
        st = st[order[:k]]
    if len(st) > int(ndets_max):
        raise _lib.MacisError(_lib.ECAPACITY, "ASCI search result exceeds "
                              "ndets_max + ncdets determinants")
    if len(st):
        st = st[np.lexsort(tuple(st[:, w] for w in range(W)))]
    return np.concatenate([st, cdets]) if len(cdets) else st


def asci_pairs(asci_settings, cdets, E_ASCI, C, ham_gen):
    """Accumulated (states, rv) before the core merge, states ascending."""
    cdets = _dets(cdets, ham_gen.nbits)
    C = np.ascontiguousarray(C, dtype=np.float64)[:len(cdets)]
    s = asci_settings.c_struct()
    n = ct.c_size_t()
    check(LIB.macis_b200_asci_pairs(ham_gen.handle, ct.byref(s),
                                    cdets.ctypes.data, len(cdets),
                                    float(E_ASCI), C.ctypes.data, None, None,
                                    ct.byref(n)))
    st = np.empty((max(n.value, 1), ham_gen.nbits // 64), dtype=np.uint64)
    rv = np.empty(max(n.value, 1))
    check(LIB.macis_b200_asci_pairs(ham_gen.handle, ct.byref(s),
                                    cdets.ctypes.data, len(cdets),
                                    float(E_ASCI), C.ctypes.data,
                                    st.ctypes.data, rv.ctypes.data,
                                    ct.byref(n)))
    return st[:n.value], rv[:n.value]


def last_search_stats(ham_gen):
    st = _lib.AsciStatsC()
    check(LIB.macis_b200_asci_last_stats(ham_gen.handle, ct.byref(st)))
    return {k: getattr(st, k) for k, _ in st._fields_}


def _screened(screen):
    """Whether the next search prunes by prediction."""
    return (screen is not None and screen.network is not None and
            screen.network.trained_steps > 0 and
            screen.searches >= screen.warmup_searches and
            screen.keep_frac < 1.0)


def topk_recall(got, exact, ncore):
    """Fraction of the exact search's new determinants (all but the trailing
    ncore core determinants) that another search of the same core set also
    selected."""
    ne, ng = len(exact) - ncore, len(got) - ncore
    if ne <= 0:
        return 1.0
    W = exact.shape[1]
    key = np.dtype((np.void, 8 * W))
    a = np.ascontiguousarray(exact[:ne]).view(key).ravel()
    b = np.ascontiguousarray(got[:max(ng, 0)]).view(key).ravel()
    return float(np.isin(a, b).sum()) / ne


def _use_net(screen, ham_gen, cdets, E0, C):
    """Whether the next search prunes by prediction: a trained network,
    past the warm-up searches, and (with min_units) a search large enough
    for the network to save time."""
    use_net = _screened(screen)
    if use_net and screen.min_units:
        from .screening import unit_features
        _, nunits = unit_features(ham_gen, cdets, E0, C, 0, 0)
        use_net = nunits >= screen.min_units
    return use_net


def _recall_check(screen, use_net, st, got, ncore, ham_gen, exact_search,
                  pruned_search):
    """The recall check of ScreenSettings after a pruning search `got` with
    statistics st: when it applies, the exact search of the same core set
    (exact_search(), recording unbiased samples for the training that
    follows) replaces the result and the top-k recall of `got` against it
    is measured. Below recall_target keep_frac doubles. At or above it,
    pruned_search(k) (no recording) tries halving keep_frac, down to
    keep_min, while the recall stays at the target; keep_frac becomes the
    smallest fraction that met it. Returns (dets, recall or None,
    statistics for the training)."""
    if not (use_net and screen.recall_target and
            st["units_total"] <= screen.check_units_max):
        return got, None, st
    exact = exact_search()
    st_train = dict(st, samples=last_search_stats(ham_gen)["samples"])
    recall = topk_recall(got, exact, ncore)
    if recall < screen.recall_target:
        screen.keep_frac = min(1.0, 2.0 * screen.keep_frac)
    else:
        k = screen.keep_frac
        while k / 2.0 >= screen.keep_min:
            trial = pruned_search(k / 2.0)
            if topk_recall(trial, exact, ncore) < screen.recall_target:
                break
            k /= 2.0
        screen.keep_frac = k
    return exact, recall, st_train


def _trial_search(screen, search):
    """pruned_search for _recall_check: the same network at keep fraction k,
    without recording samples."""
    def run(k):
        return search(dataclasses.replace(screen, keep_frac=k, train=False))
    return run


def _train_after_search(screen, stats):
    """Retrain the network on the samples the search recorded (clamped
    first); returns the milliseconds it took (0 without training)."""
    if not (screen is not None and screen.network is not None and
            screen.train and stats["samples"] > 0):
        return 0.0
    tt = time.perf_counter()
    if screen.clamp_quantile:
        screen.network.clamp_samples(screen.clamp_quantile)
    screen.network.train(None, None, screen.epochs, screen.batch, screen.lr,
                         screen.seed + screen.searches)
    return (time.perf_counter() - tt) * 1e3


def asci_iter(asci_settings, mcscf_settings, ndets_max, E0, wfn, X, ham_gen,
              norb, screen=None):
    """One ASCI iteration: reorder, search on the ncdets_max largest, then
    rediagonalise without guess reuse (iteration.hpp:17-68). With a
    ScreenSettings the search records samples / prunes units and the
    network is retrained on the recorded samples afterwards."""
    wfn = _dets(wfn, ham_gen.nbits)
    X = np.asarray(X, dtype=np.float64)
    if len(wfn) > 1:
        wfn, X = reorder_ci_on_coeff(wfn, X)
    nkeep = min(int(asci_settings.ncdets_max), len(wfn))
    t0 = time.perf_counter()
    core, Cc = wfn[:nkeep], X[:nkeep]
    use_net = _use_net(screen, ham_gen, core, E0, Cc)
    wfn = asci_search(asci_settings, ndets_max, core, E0, Cc, norb, ham_gen,
                      screen=screen, use_net=use_net)
    st = last_search_stats(ham_gen)
    wfn, recall, st = _recall_check(
        screen, use_net, st, wfn, nkeep, ham_gen,
        lambda: asci_search(asci_settings, ndets_max, core, E0, Cc, norb,
                            ham_gen, screen=screen, use_net=False),
        _trial_search(screen, lambda sc: asci_search(
            asci_settings, ndets_max, core, E0, Cc, norb, ham_gen, screen=sc,
            use_net=True)))
    t1 = time.perf_counter()
    train_ms = _train_after_search(screen, st)
    t1b = time.perf_counter()
    tim = {}
    E, X = selected_ci_diag(wfn, ham_gen, mcscf_settings.ci_matel_tol,
                            mcscf_settings.ci_max_subspace,
                            mcscf_settings.ci_res_tol, None,
                            precision=mcscf_settings.precision,
                            index_t=None, timings=tim,
                            restart_keep=mcscf_settings.davidson_restart_keep,
                            max_iter=mcscf_settings.davidson_max_iter)
    t2 = time.perf_counter()
    mcscf_settings.iteration_log.append(dict(
        ndets=len(wfn), E=E, search_ms=(t1 - t0) * 1e3, train_ms=train_ms,
        diag_ms=(t2 - t1b) * 1e3, screened=bool(use_net),
        units_total=st["units_total"], units_kept=st["units_kept"],
        raw_pairs=st["raw_pairs"], recall_check=recall,
        keep_frac=None if screen is None else screen.keep_frac,
        ranges=st["batches"], alpha_strings=st["alpha_strings"],
        key_bits=st["key_bits"], pairs_ms=st["pairs_ms"],
        sort_ms=st["sort_ms"], **tim))
    return E, wfn, X


def asci_grow(asci_settings, mcscf_settings, E0, wfn, X, ham_gen, norb,
              screen=None):
    log = logging.getLogger("asci_grow")
    wfn = _dets(wfn, ham_gen.nbits)
    if asci_settings.grow_with_rot:
        raise NotImplementedError("grow_with_rot is outside the GPU path")
    it = 1
    while len(wfn) < asci_settings.ntdets_max:
        ndets_new = min(max(asci_settings.ntdets_min,
                            len(wfn) * asci_settings.grow_factor),
                        asci_settings.ntdets_max)
        E, wfn, X = asci_iter(asci_settings, mcscf_settings, ndets_new, E0,
                              wfn, X, ham_gen, norb, screen)
        if ndets_new > len(wfn):
            raise RuntimeError("Wavefunction didn't grow enough...")
        log.info("iter = %4d, E0 = %20.12e, dE = %14.6e, WFN_SIZE = %d", it, E,
                 E - E0, len(wfn))
        it += 1
        E0 = E
    return E0, wfn, X


def asci_refine(asci_settings, mcscf_settings, E0, wfn, X, ham_gen, norb,
                screen=None):
    log = logging.getLogger("asci_refine")
    ndets = len(wfn)
    for it in range(asci_settings.max_refine_iter):
        E, wfn, X = asci_iter(asci_settings, mcscf_settings, ndets, E0, wfn, X,
                              ham_gen, norb, screen)
        if len(wfn) != ndets:
            raise RuntimeError("Wavefunction size can't change in refinement")
        dE = E - E0
        log.info("iter = %4d, E0 = %20.12e, dE = %14.6e", it + 1, E, dE)
        E0 = E
        if abs(dE) < asci_settings.refine_energy_tol:
            return E0, wfn, X
    raise RuntimeError("ACCI Refine did not converge")
