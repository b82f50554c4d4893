"""Learned screening of the ASCI search (no MACIS counterpart).

``ScreeningNetwork`` owns the device network (din -> 256 -> 256 -> 1, GELU,
BF16 tcgen05 GEMMs with FP32 accumulation, FP32 master weights, Adam).
``ScreenSettings`` tells ``asci_search`` / ``asci_iter`` / ``asci_grow`` /
``asci_refine`` (macis_b200.asci) how to use it: record (unit input, exact
log score) samples from each search, prune units by prediction once the
network has been trained, and retrain after every search.

A unit is one core determinant with one excitation class and, for doubles,
one outer (occupied, virtual) pair -- the inner loop of
append_ss_doubles / append_os_doubles_asci_contributions
(include/macis/asci/determinant_contributions.hpp:68-160) for fixed (i, a),
or all singles of one spin (:25-66). Pruning a unit skips its contributions
before they are generated, scored, sorted or merged.
"""
import ctypes as ct
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import LIB, check

__all__ = ["ScreeningNetwork", "ScreenSettings", "unit_width",
           "unit_features"]


def unit_width(nbits):
    """Network input width of the units of nbits-wide determinants."""
    return int(LIB.macis_b200_asci_unit_width(int(nbits)))


class ScreeningNetwork:
    def __init__(self, nbits=None, din=None, seed=0):
        if din is None:
            din = unit_width(nbits if nbits is not None else 64)
        self.din = int(din)
        h = ct.c_void_p()
        check(LIB.macis_b200_mlp_create(self.din, int(seed), ct.byref(h)))
        self.handle = h
        n = ct.c_size_t()
        check(LIB.macis_b200_mlp_num_params(self.handle, ct.byref(n)))
        self.num_params = n.value
        self.trained_steps = 0
        self.history = []

    def __del__(self):
        if getattr(self, "handle", None):
            LIB.macis_b200_mlp_destroy(self.handle)
            self.handle = None

    # parameters: W1 [256][din], b1, W2 [256][256], b2, w3, b3 (FP32)
    @property
    def params(self):
        P = np.empty(self.num_params, dtype=np.float32)
        check(LIB.macis_b200_mlp_get_params(self.handle, P.ctypes.data))
        return P

    @params.setter
    def params(self, P):
        P = np.ascontiguousarray(P, dtype=np.float32)
        assert P.size == self.num_params
        check(LIB.macis_b200_mlp_set_params(self.handle, P.ctypes.data))

    def _x(self, X):
        X = np.ascontiguousarray(X, dtype=np.uint16)
        assert X.ndim == 2 and X.shape[1] == self.din
        return X

    def forward(self, X):
        """Predictions for BF16 inputs given as uint16 bit patterns."""
        X = self._x(X)
        y = np.empty(len(X), dtype=np.float32)
        check(LIB.macis_b200_mlp_forward(self.handle, X.ctypes.data, len(X),
                                         y.ctypes.data, 0))
        return y

    def gradients(self, X, t):
        """(gradient, loss) of sum (y - t)^2 / (2 n) over all rows."""
        X = self._x(X)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.empty(self.num_params, dtype=np.float32)
        loss = ct.c_double()
        check(LIB.macis_b200_mlp_gradients(self.handle, X.ctypes.data,
                                           t.ctypes.data, len(X),
                                           g.ctypes.data, ct.byref(loss), 0))
        return g, loss.value

    def train(self, X=None, t=None, epochs=2, batch=1024, lr=1e-3, seed=0):
        """Adam over shuffled minibatches; X None = the recorded samples.
        Returns the mean loss of the last epoch."""
        loss = ct.c_double()
        if X is None:
            check(LIB.macis_b200_mlp_train(self.handle, None, None, 0,
                                           int(epochs), int(batch), float(lr),
                                           int(seed), ct.byref(loss), 0))
        else:
            X = self._x(X)
            t = np.ascontiguousarray(t, dtype=np.float32)
            check(LIB.macis_b200_mlp_train(self.handle, X.ctypes.data,
                                           t.ctypes.data, len(X), int(epochs),
                                           int(batch), float(lr), int(seed),
                                           ct.byref(loss), 0))
        self.trained_steps += 1
        self.history.append(loss.value)
        return loss.value

    def clamp_samples(self, q):
        """Raise recorded targets below their q-quantile to it."""
        f = ct.c_float()
        check(LIB.macis_b200_mlp_clamp_samples(self.handle, float(q),
                                               ct.byref(f)))
        return f.value

    def set_sample_targets(self, t):
        """Overwrite the targets of the recorded samples (same count)."""
        t = np.ascontiguousarray(t, dtype=np.float32).ravel()
        check(LIB.macis_b200_mlp_set_sample_targets(self.handle,
                                                    t.ctypes.data, t.size))

    def samples(self):
        """(X, t) recorded by the last search that recorded samples."""
        n = ct.c_size_t()
        check(LIB.macis_b200_mlp_samples(self.handle, ct.byref(n), None, None))
        X = np.empty((n.value, self.din), dtype=np.uint16)
        t = np.empty(n.value, dtype=np.float32)
        if n.value:
            check(LIB.macis_b200_mlp_samples(self.handle, ct.byref(n),
                                             X.ctypes.data, t.ctypes.data))
        return X, t


@dataclass
class ScreenSettings:
    """How the ASCI drivers use a ScreeningNetwork."""
    network: ScreeningNetwork = None
    keep_frac: float = 0.2        # units kept by prediction
    explore_frac: float = 0.02    # extra random units (unbiased training data)
    max_samples: int = 1_000_000  # samples recorded per search
    epochs: int = 2
    lr: float = 1e-3
    batch: int = 1024
    clamp_quantile: float = 0.6   # recorded targets below it are raised to it
    min_units: int = 20000        # searches with fewer units run exact
    warmup_searches: int = 1      # exact (recording) searches before pruning
    train: bool = True            # retrain after every search
    seed: int = 0
    searches: int = 0             # searches run so far (updated)
    # Recall check: a pruning search of asci_iter / asci_grow / asci_refine
    # with at most check_units_max units is also run exactly; its top-k
    # recall against the exact selection is measured and the exact
    # selection is kept. Below recall_target keep_frac doubles (at 1 pruning
    # stops); at or above it, pruned searches of the same core set at half
    # the fraction (down to keep_min) are tried, and keep_frac becomes the
    # smallest that meets the target. recall_target 0 turns the check off.
    recall_target: float = 0.95
    check_units_max: int = 20_000_000
    keep_min: float = 0.2

    def c_struct(self, use_net):
        return _lib.AsciScreenC(
            self.network.handle if self.network is not None else None,
            int(bool(use_net)), 0, float(self.keep_frac),
            float(self.explore_frac),
            int(self.max_samples) if self.train else 0,
            int(self.seed + 7919 * self.searches))


def unit_features(ham_gen, cdets, E0, C, first=0, n=None):
    """Network inputs (uint16 BF16 bits) of units [first, first + n) of the
    search over cdets, and the search's unit count."""
    cdets = np.ascontiguousarray(cdets, dtype=np.uint64).reshape(
        -1, ham_gen.nbits // 64)
    C = np.ascontiguousarray(C, dtype=np.float64)[:len(cdets)]
    nu = ct.c_size_t()
    check(LIB.macis_b200_asci_unit_features(
        ham_gen.handle, cdets.ctypes.data, len(cdets), float(E0),
        C.ctypes.data, 0, 0, None, ct.byref(nu)))
    if n is None:
        n = nu.value - first
    X = np.empty((max(n, 0), unit_width(ham_gen.nbits)), dtype=np.uint16)
    if n > 0:
        check(LIB.macis_b200_asci_unit_features(
            ham_gen.handle, cdets.ctypes.data, len(cdets), float(E0),
            C.ctypes.data, int(first), int(n), X.ctypes.data, ct.byref(nu)))
    return X, nu.value
