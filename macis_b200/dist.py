"""Row-block distribution of the Hamiltonian and its Davidson solve over
ranks: one process per GPU, torch.distributed for the exchange.

The reference distributes H by rows (make_dist_csr_hamiltonian,
include/macis/csr_hamiltonian.hpp:49-82): every rank holds all determinants
and integrals and builds the rows ``row_bounds(M, world, rank)`` against the
full ket list; the build needs no exchange. Its parallel Davidson
(p_davidson, include/macis/solvers/davidson.hpp:283-394) keeps the local rows
of every subspace vector; the operator first gathers the vector from all
ranks (sparsexx pspmbv), inner products are summed over ranks
(p_gram_schmidt, :228-256), and the k x k Rayleigh-Ritz problem is reduced
over ranks, solved on rank 0 and broadcast (p_rayleigh_ritz, :258-280).

Here the ranks are torch.distributed processes. With NCCL every rank drives
one GPU: its H block is built by libmacis_b200 and the gathered vector and
the local products stay in HBM. The same host logic runs on CPU tensors
over gloo, which is how the multi-rank path is tested without GPUs.
"""
import ctypes as C
import math

import numpy as np

from . import _lib
from .hamiltonian import DeviceCSR, _dev_ptr, _host_dets, row_bounds
from ._lib import LIB, check

__all__ = ["rank_world", "local_rows", "reduce_max", "reduce_sum",
           "allgather_rows", "DistCSR", "make_dist_csr_hamiltonian",
           "RowBlockOperator", "p_gram_schmidt", "p_rayleigh_ritz",
           "p_davidson", "gather_row_blocks", "merge_search_parts",
           "merge_sample_targets", "asci_search", "p_diagonal_guess", "reuse_guess",
           "selected_ci_diag", "asci_iter", "asci_grow", "asci_refine"]


def _dist():
    import torch.distributed as dist
    return dist


def rank_world(group=None):
    """(rank, world size) of this process; (0, 1) without a process group."""
    dist = _dist()
    if not (dist.is_available() and dist.is_initialized()):
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def local_rows(M, group=None):
    """Row block [lo, hi) this rank owns (dist_sparse_matrix default
    partition, sparsexx/matrix_types/dist_sparse_matrix.hpp:47-62)."""
    r, w = rank_world(group)
    return row_bounds(M, w, r)


def _scalar_reduce(x, op, group, device):
    import torch
    r, w = rank_world(group)
    if w == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    _dist().all_reduce(t, op=op, group=group)
    return float(t.item())


def reduce_max(x, group=None, device="cpu"):
    """Maximum of a scalar over ranks (timings: the slowest rank)."""
    return _scalar_reduce(x, _dist().ReduceOp.MAX, group, device)


def reduce_sum(x, group=None, device="cpu"):
    """Sum of a scalar over ranks (counts: nnz, determinants)."""
    return _scalar_reduce(x, _dist().ReduceOp.SUM, group, device)


def allgather_rows(x_local, N, group=None):
    """The full length-N vector from every rank's row block (the gather
    of pspmbv). Blocks differ in length only on the last rank; each is padded
    to the longest so that one all_gather moves them all."""
    import torch
    r, w = rank_world(group)
    if w == 1:
        return x_local
    per = N // w
    longest = per + N % w
    buf = torch.zeros(longest, dtype=x_local.dtype, device=x_local.device)
    buf[:x_local.numel()] = x_local
    parts = [torch.empty_like(buf) for _ in range(w)]
    _dist().all_gather(parts, buf, group=group)
    return torch.cat([p[:row_bounds(N, w, q)[1] - row_bounds(N, w, q)[0]]
                      for q, p in enumerate(parts)])


class DistCSR:
    """This rank's row block of a row-distributed H: ``local`` is the
    DeviceCSR of rows [lo, hi) against all N columns."""

    def __init__(self, local, lo, hi, N, group=None, bra=None):
        self.local, self.lo, self.hi, self.N = local, lo, hi, N
        self.group = group
        self._bra = bra

    @property
    def m_local(self):
        return self.hi - self.lo

    @property
    def device(self):
        """Where the block's vectors live: this rank's CUDA device."""
        import torch
        return torch.device("cuda", torch.cuda.current_device())

    def nnz_total(self, device="cpu"):
        return int(reduce_sum(self.local.nnz, self.group, device))

    def diagonal(self, device=None):
        """H_ii for the local rows i in [lo, hi), as a float64 tensor: the
        diagonal of the block's diagonal tile (columns [lo, hi)), which p_davidson
        preconditions with (the reference takes it from
        H.diagonal_tile()). The block's own stored diagonal is the entry in
        column == local row, the same thing only on the rank with lo = 0."""
        import torch
        if self.lo == 0 or self.m_local == 0:
            d = self.local.diagonal()
        else:
            b = self._bra
            if hasattr(b, "cpu"):
                b = b.cpu().numpy().view(np.uint64)
            d = np.atleast_1d(self.local.ham.matrix_element(b, b))
        d = torch.from_numpy(np.ascontiguousarray(d, dtype=np.float64))
        return d if device is None else d.to(device)

    def local_spmv(self, x_full, y_local):
        """y_local = H[lo:hi, :] x_full on this rank's GPU (device tensors)."""
        import torch
        if not (x_full.is_cuda and y_local.is_cuda):
            raise RuntimeError("local_spmv needs CUDA tensors")
        torch.cuda.current_stream().synchronize()
        check(LIB.macis_b200_spmv(self.local.handle, 1, 1.0,
                                  C.c_void_p(x_full.data_ptr()), self.N, 0.0,
                                  C.c_void_p(y_local.data_ptr()),
                                  max(self.m_local, 1), _lib.DEVICE_PTRS))
        return y_local

    def operator(self):
        """RowBlockOperator over this block for p_davidson."""
        import torch

        def mv(x_full):
            y = torch.empty(self.m_local, dtype=torch.float64,
                            device=x_full.device)
            return self.local_spmv(x_full, y)
        return RowBlockOperator(mv, self.N, self.group)


def make_dist_csr_hamiltonian(dets, ham_gen, H_thresh, index_t=np.int32,
                              value_t=np.float64, group=None):
    """make_dist_csr_hamiltonian (csr_hamiltonian.hpp:49-82): rows
    local_rows(len(dets)) of H against the full determinant list, built on
    this rank's GPU. `dets` is a host array or a CUDA tensor of the full list
    (replicated on every rank, as in the reference)."""
    p = _dev_ptr(dets)
    if p is not None:
        words = ham_gen.nbits // 64
        N = dets.numel() // words
        lo, hi = local_rows(N, group)
        flat = dets.reshape(-1)
        bra = flat[lo * words:hi * words]
        local = DeviceCSR.build(ham_gen, bra, flat, H_thresh, index_t, value_t)
    else:
        d = _host_dets(dets, ham_gen.nbits)
        N = len(d)
        lo, hi = local_rows(N, group)
        bra = d[lo:hi]
        local = DeviceCSR.build(ham_gen, bra, d, H_thresh, index_t, value_t)
    return DistCSR(local, lo, hi, N, group, bra)


class RowBlockOperator:
    """Operator action on row-distributed vectors: gather the full vector,
    then apply this rank's row block (``local_matvec(x_full) -> y_local``)."""

    def __init__(self, local_matvec, N, group=None):
        self.local_matvec, self.N, self.group = local_matvec, N, group

    def __call__(self, x_local):
        return self.local_matvec(allgather_rows(x_local, self.N, self.group))


def _allreduce_(t, group):
    if rank_world(group)[1] > 1:
        _dist().all_reduce(t, group=group)
    return t


def p_gram_schmidt(V, k, v, group=None):
    """Project v (local rows, updated in place) out of the first k columns of
    V twice, then normalise: p_gram_schmidt, davidson.hpp:228-256."""
    Vk = V[:, :k]
    for _ in range(2):
        inner = _allreduce_(Vk.T @ v, group)
        v -= Vk @ inner
    nrm = math.sqrt(_allreduce_((v @ v).reshape(1), group).item())
    v /= nrm
    return v


def p_rayleigh_ritz(V, AV, k, group=None):
    """Eigenpairs of V^T A V over the first k columns, the k x k projection
    summed over ranks, diagonalised on rank 0 and broadcast:
    p_rayleigh_ritz, davidson.hpp:258-280."""
    import torch
    Cm = _allreduce_((V[:, :k].T @ AV[:, :k]).contiguous(), group)
    r, w = rank_world(group)
    lam = torch.empty(k, dtype=Cm.dtype, device=Cm.device)
    vec = torch.empty_like(Cm)
    if r == 0:
        # syev with Uplo::Lower reads the lower triangle only
        lam_, vec_ = torch.linalg.eigh(torch.tril(Cm) + torch.tril(Cm, -1).T)
        lam.copy_(lam_)
        vec.copy_(vec_)
    if w > 1:
        _dist().broadcast(lam, 0, group=group)
        _dist().broadcast(vec, 0, group=group)
    return lam, vec


def p_davidson(N_local, max_m, op, D_local, tol, X_local, group=None,
               log=None):
    """Lowest eigenpair of a row-distributed symmetric operator:
    p_davidson, davidson.hpp:283-394 (no restarts, like the reference).

    `op(x_local) -> y_local` applies A (a RowBlockOperator); D_local holds
    this rank's rows of diag(A); X_local (this rank's rows of the normalised
    guess) is overwritten with the eigenvector. Every rank returns the same
    (iterations, eigenvalue). Raises RuntimeError if the residual norm does
    not reach `tol` within `max_m` subspace vectors."""
    import torch
    if N_local and X_local is None:
        raise RuntimeError("Davidson: No Guess Provided")
    dev, dt = X_local.device, torch.float64
    V = torch.zeros((N_local, max_m + 1), dtype=dt, device=dev)
    AV = torch.zeros((N_local, max_m + 1), dtype=dt, device=dev)
    V[:, 0] = X_local
    AV[:, 0] = op(V[:, 0].contiguous())
    v1 = AV[:, 0].clone()
    p_gram_schmidt(V, 1, v1, group)
    V[:, 1] = v1
    converged = False
    it = 1
    lam0 = 0.0
    for i in range(1, max_m):
        k = i + 1
        AV[:, i] = op(V[:, i].contiguous())
        lam, Cm = p_rayleigh_ritz(V, AV, k, group)
        lam0 = float(lam[0].item())
        c0 = Cm[:, 0]
        X_local.copy_(V[:, :k] @ c0)
        R = AV[:, :k] @ c0 - lam0 * X_local
        res = math.sqrt(_allreduce_((R @ R).reshape(1), group).item())
        if log is not None:
            log.info(f"iter = {i:4d}, LAM(0) = {lam0:20.12e}, "
                     f"RNORM = {res:20.12e}")
        if res < tol:
            converged = True
            break
        R = -R / (D_local - lam0)
        p_gram_schmidt(V, k, R, group)
        V[:, i + 1] = R
        it += 1
    if not converged:
        raise RuntimeError("Davidson Did Not Converge!")
    return it, lam0


def gather_row_blocks(rowptr, colind, nzval, dst=0, group=None):
    """Concatenate every rank's CSR row block (host arrays, blocks in rank
    order) into the full matrix on rank `dst`; other ranks get None."""
    dist = _dist()
    r, w = rank_world(group)
    mine = (np.asarray(rowptr, np.int64), np.asarray(colind, np.int64),
            np.asarray(nzval))
    if w == 1:
        return mine
    got = [None] * w if r == dst else None
    dist.gather_object(mine, got, dst=dst, group=group)
    if r != dst:
        return None
    rps, cis, nzs = [], [], []
    off = 0
    for q, (rp, ci, nz) in enumerate(got):
        rps.append(rp[(1 if q else 0):] - rp[0] + off)
        off += int(rp[-1] - rp[0])
        cis.append(ci)
        nzs.append(nz)
    return np.concatenate(rps), np.concatenate(cis), np.concatenate(nzs)


def merge_search_parts(part, ndets_max, cdets, nbits, group=None):
    """All-gather every rank's (states, scores) part of a split ASCI search
    and merge them (asci.merge_asci_parts) into the whole search's result,
    the same on every rank."""
    from .asci import merge_asci_parts
    r, w = rank_world(group)
    if w == 1:
        parts = [part]
    else:
        parts = [None] * w
        _dist().all_gather_object(parts, (np.asarray(part[0]),
                                          np.asarray(part[1])), group=group)
    return merge_asci_parts(parts, ndets_max, cdets, nbits)


def merge_sample_targets(t, group=None):
    """Elementwise maximum over the ranks of the recorded sample targets of
    a split search (every rank records the same sample rows; each target is
    the unit's largest score over the rank's bins). float32 in and out."""
    t = np.ascontiguousarray(t, dtype=np.float32).ravel()
    r, w = rank_world(group)
    if w == 1:
        return t
    import torch
    x = torch.from_numpy(t.copy()).to(_device(group))
    _dist().all_reduce(x, op=_dist().ReduceOp.MAX, group=group)
    return x.cpu().numpy()


def _device(group):
    """Where collective buffers live: CUDA for NCCL, else the CPU."""
    if rank_world(group)[1] == 1:
        return "cpu"
    return "cuda" if _dist().get_backend(group) == "nccl" else "cpu"


def asci_search(asci_settings, ndets_max, cdets, E_ASCI, C, norb, ham_gen,
                group=None, screen=None, use_net=False):
    """Exact ASCI search split over the ranks of `group`, one GPU each: rank
    r searches part r of world (asci.asci_search_part: its share of the
    alpha-string hash bins, cut by the contribution histogram every rank
    computes alike), then the parts are gathered and merged. The result is
    asci_search's on one GPU, on every rank (the reference's MPI search,
    determinant_search.hpp:145-391, splits by alpha constraints instead).

    screen / use_net: the learned screening (asci.asci_search), with every
    rank holding an equal network. A recording search merges the parts'
    targets (merge_sample_targets) into every rank's network, so each holds
    the one-GPU search's samples and training keeps the networks equal."""
    from .asci import asci_search_part
    r, w = rank_world(group)
    part = asci_search_part(asci_settings, ndets_max, cdets, E_ASCI, C, norb,
                            ham_gen, r, w, screen=screen, use_net=use_net)
    if (w > 1 and screen is not None and screen.network is not None and
            screen.train and screen.max_samples > 0):
        _, t = screen.network.samples()
        dev = _device(group)
        n = reduce_max(len(t), group, dev)     # equal on every rank
        if n != len(t) or reduce_sum(len(t), group, dev) != w * n:
            raise RuntimeError("ranks recorded different sample counts")
        if len(t):
            screen.network.set_sample_targets(merge_sample_targets(t, group))
    return merge_search_parts(part, ndets_max, cdets, ham_gen.nbits, group)


def p_diagonal_guess(D_local, N, group=None):
    """p_diagonal_guess (davidson.hpp:72-110): this rank's rows of the unit
    vector at the first minimum of the full diagonal, which is gathered
    from every rank's rows."""
    import torch
    D = allgather_rows(D_local, N, group)
    g = int(torch.argmin(D).item())     # the first minimum
    lo, hi = local_rows(N, group)
    X = torch.zeros(hi - lo, dtype=torch.float64, device=D_local.device)
    if lo <= g < hi:
        X[g - lo] = 1.0
    return X


def reuse_guess(C_local, N, group=None):
    """Whether the passed vector is the Davidson guess: max |C| over all
    ranks above 1/N (selected_ci_diag.hpp:41-52 and :94-101, decided once for
    all ranks). C_local None or empty counts as zero on this rank."""
    c = np.abs(np.asarray(C_local, dtype=np.float64)) if C_local is not None \
        else np.zeros(0)
    mx = float(c.max()) if c.size else 0.0
    return reduce_max(mx, group, _device(group)) > 1.0 / max(N, 1)


def selected_ci_diag(dets, ham_gen, h_el_tol, davidson_max_m,
                     davidson_res_tol, C_local=None, group=None, log=None):
    """selected_ci_diag over the ranks of `group` (selected_ci_diag.hpp:
    125-206 with a communicator, parallel_selected_ci_diag :23-72): this
    rank's row block of H on its GPU (make_dist_csr_hamiltonian), the guess,
    then p_davidson (no restarts, as the reference). C_local (this rank's
    rows) is the guess when max |C| over all ranks exceeds 1/N; else the
    diagonal guess (p_diagonal_guess), also when any rank lacks its rows of
    C (None or the wrong length). Returns (E0, X_local), X_local this
    rank's rows of the eigenvector as a CUDA tensor.

    The reference compares each rank's own max |C_local| with 1/len(C_local),
    so its ranks can disagree, and only some of them then enter the
    collective p_diagonal_guess; here the test is one over all ranks."""
    import torch
    dets = _host_dets(dets, ham_gen.nbits)
    N = len(dets)
    A = make_dist_csr_hamiltonian(dets, ham_gen, h_el_tol, group=group)
    dev = A.device
    D = A.diagonal(dev)
    ok = C_local is not None and len(C_local) == A.m_local
    # one branch on every rank: the guess is reused only when every rank
    # holds its rows of it (else a rank without them would fail while the
    # others wait in p_davidson's collectives)
    all_ok = reduce_max(0.0 if ok else 1.0, group, dev) == 0.0
    if reuse_guess(C_local if ok else None, N, group) and all_ok:
        X = torch.as_tensor(np.asarray(C_local, dtype=np.float64)).to(dev)
    else:
        X = p_diagonal_guess(D, N, group)
    it, E = p_davidson(A.m_local, int(davidson_max_m), A.operator(), D,
                       davidson_res_tol, X, group, log)
    return E, X


def asci_iter(asci_settings, mcscf_settings, ndets_max, E0, wfn, X, ham_gen,
              norb, group=None, screen=None):
    """asci_iter with a communicator (iteration.hpp:17-68): reorder on |C|,
    the split search over the ranks (asci_search above), the distributed
    rediagonalisation without guess reuse (selected_ci_diag above), and the
    eigenvector all-gathered to every rank. screen as in asci.asci_iter,
    with an equal network on every rank. Only the reference solver is
    distributed: FP64 values, no thick restart."""
    from .asci import (_dets, _recall_check, _train_after_search,
                       _trial_search, _use_net, last_search_stats,
                       reorder_ci_on_coeff)
    from .solvers import FP64
    if mcscf_settings.precision != FP64 or mcscf_settings.davidson_restart_keep:
        raise NotImplementedError(
            "the distributed solve is the reference p_davidson: FP64, no "
            "restart")
    wfn = _dets(wfn, ham_gen.nbits)
    X = np.asarray(X, dtype=np.float64)
    if len(wfn) > 1:
        wfn, X = reorder_ci_on_coeff(wfn, X)
    nkeep = min(int(asci_settings.ncdets_max), len(wfn))
    core, Cc = wfn[:nkeep], X[:nkeep]
    use_net = _use_net(screen, ham_gen, core, E0, Cc)
    wfn = asci_search(asci_settings, ndets_max, core, E0, Cc, norb, ham_gen,
                      group, screen=screen, use_net=use_net)
    if screen is not None:
        # the recall check of asci.asci_iter; every rank holds the merged
        # results and the same statistics, so all take the same branch
        wfn, _, st = _recall_check(
            screen, use_net, last_search_stats(ham_gen), wfn, nkeep, ham_gen,
            lambda: asci_search(asci_settings, ndets_max, core, E0, Cc, norb,
                                ham_gen, group, screen=screen, use_net=False),
            _trial_search(screen, lambda sc: asci_search(
                asci_settings, ndets_max, core, E0, Cc, norb, ham_gen, group,
                screen=sc, use_net=True)))
        _train_after_search(screen, st)
    E, X_local = selected_ci_diag(wfn, ham_gen, mcscf_settings.ci_matel_tol,
                                  mcscf_settings.ci_max_subspace,
                                  mcscf_settings.ci_res_tol, None, group)
    X = allgather_rows(X_local, len(wfn), group).cpu().numpy()
    return E, wfn, X


def asci_grow(asci_settings, mcscf_settings, E0, wfn, X, ham_gen, norb,
              group=None, screen=None):
    """asci_grow (grow.hpp:17-171, without grow_with_rot) over the ranks:
    distributed asci_iter until ntdets_max determinants."""
    from .asci import _dets
    wfn = _dets(wfn, ham_gen.nbits)
    if asci_settings.grow_with_rot:
        raise NotImplementedError("grow_with_rot is outside the GPU path")
    while len(wfn) < asci_settings.ntdets_max:
        ndets_new = min(max(asci_settings.ntdets_min,
                            len(wfn) * asci_settings.grow_factor),
                        asci_settings.ntdets_max)
        E, wfn, X = asci_iter(asci_settings, mcscf_settings, ndets_new, E0,
                              wfn, X, ham_gen, norb, group, screen)
        if ndets_new > len(wfn):
            raise RuntimeError("Wavefunction didn't grow enough...")
        E0 = E
    return E0, wfn, X


def asci_refine(asci_settings, mcscf_settings, E0, wfn, X, ham_gen, norb,
                group=None, screen=None):
    """asci_refine (refine.hpp:15-66) over the ranks."""
    ndets = len(wfn)
    for _ in range(asci_settings.max_refine_iter):
        E, wfn, X = asci_iter(asci_settings, mcscf_settings, ndets, E0, wfn,
                              X, ham_gen, norb, group, screen)
        if len(wfn) != ndets:
            raise RuntimeError("Wavefunction size can't change in refinement")
        dE = E - E0
        E0 = E
        if abs(dE) < asci_settings.refine_energy_tol:
            return E0, wfn, X
    raise RuntimeError("ACCI Refine did not converge")
