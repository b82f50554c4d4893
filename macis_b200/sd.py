"""Determinant spaces and string helpers on the host (numpy).

Determinant arrays are uint64 of shape (ndets, nbits // 64) in the
std::bitset<nbits> word layout (alpha string first; see include/macis_b200.h).
These helpers reproduce the orders of the reference so that CSR rows and
columns line up with it:

* ``generate_hilbert_space`` -- alpha strings outer, beta inner, each in
  std::prev_permutation order (include/macis/sd_operations.hpp:440-476),
  which is lexicographic order of the occupied-index tuples.
* ``generate_cisd_hilbert_space`` -- HF, singles, doubles, mixed
  (sd_operations.hpp:361-430).
"""
from itertools import combinations

import numpy as np

__all__ = ["spin_words", "make_dets", "split_dets", "canonical_hf_determinant",
           "generate_combs", "generate_hilbert_space",
           "generate_cisd_hilbert_space", "to_canonical_string",
           "from_canonical_string", "det_less_order"]


def spin_words(nbits):
    return 2 if nbits == 256 else 1


def _spin_to_int(row, nbits, beta):
    if nbits == 64:
        w = int(row[0])
        return (w >> 32) if beta else (w & 0xFFFFFFFF)
    if nbits == 128:
        return int(row[1 if beta else 0])
    o = 2 if beta else 0
    return int(row[o]) | (int(row[o + 1]) << 64)


def make_dets(alpha, beta, nbits):
    """Pack python-int (or uint64) spin strings into determinant words."""
    alpha = [int(a) for a in np.atleast_1d(alpha)]
    beta = [int(b) for b in np.atleast_1d(beta)]
    n = len(alpha)
    nw = nbits // 64
    out = np.zeros((n, nw), dtype=np.uint64)
    m64 = (1 << 64) - 1
    for i, (a, b) in enumerate(zip(alpha, beta)):
        if nbits == 64:
            out[i, 0] = (a & 0xFFFFFFFF) | ((b & 0xFFFFFFFF) << 32)
        elif nbits == 128:
            out[i, 0] = a & m64
            out[i, 1] = b & m64
        else:
            out[i] = (a & m64, a >> 64, b & m64, b >> 64)
    return out


def split_dets(dets, nbits):
    """(alpha, beta) python ints of each determinant."""
    dets = np.asarray(dets, dtype=np.uint64).reshape(-1, nbits // 64)
    return ([_spin_to_int(r, nbits, False) for r in dets],
            [_spin_to_int(r, nbits, True) for r in dets])


def canonical_hf_determinant(nalpha, nbeta, nbits=64):
    """sd_operations.hpp:31-37: lowest nalpha / nbeta orbitals occupied."""
    return make_dets([(1 << nalpha) - 1], [(1 << nbeta) - 1], nbits)


def generate_combs(nbits, nset):
    """sd_operations.hpp:440-458 as python ints, prev_permutation order."""
    return [sum(1 << i for i in c) for c in combinations(range(nbits), nset)]


def generate_hilbert_space(norbs, nalpha, nbeta, nbits=64):
    a = generate_combs(norbs, nalpha)
    b = generate_combs(norbs, nbeta)
    if nbits == 64:
        av = np.asarray(a, dtype=np.uint64)
        bv = np.asarray(b, dtype=np.uint64)
        return (av[:, None] | (bv[None, :] << np.uint64(32))).reshape(-1, 1)
    if nbits == 128:
        out = np.empty((len(a) * len(b), 2), dtype=np.uint64)
        out[:, 0] = np.repeat(np.asarray(a, dtype=np.uint64), len(b))
        out[:, 1] = np.tile(np.asarray(b, dtype=np.uint64), len(a))
        return out
    return make_dets(np.repeat(np.array(a, dtype=object), len(b)),
                     np.tile(np.array(b, dtype=object), len(a)), nbits)


def _singles(norb, s):
    occ = [i for i in range(norb) if s >> i & 1]
    vir = [i for i in range(norb) if not s >> i & 1]
    return [s ^ (1 << o) ^ (1 << v) for v in vir for o in occ]


def _doubles(norb, s):
    occ = [i for i in range(norb) if s >> i & 1]
    vir = [i for i in range(norb) if not s >> i & 1]
    out = []
    for a in range(len(vir)):
        for i in range(len(occ)):
            for b in range(a + 1, len(vir)):
                for j in range(i + 1, len(occ)):
                    out.append(s ^ (1 << occ[i]) ^ (1 << vir[a]) ^
                               (1 << occ[j]) ^ (1 << vir[b]))
    return out


def generate_cisd_hilbert_space(norb, state, nbits=64):
    (a,), (b,) = split_dets(state, nbits)
    sa, sb = _singles(norb, a), _singles(norb, b)
    da, db = _doubles(norb, a), _doubles(norb, b)
    al = [a] + sa + [a] * len(sb) + da + [a] * len(db)
    be = [b] + [b] * len(sa) + sb + [b] * len(da) + db
    for x in sa:
        for y in sb:
            al.append(x)
            be.append(y)
    return make_dets(al, be, nbits)


def to_canonical_string(det, nbits=64):
    """sd_operations.hpp:596-613 ('2', 'u', 'd', '0' per orbital)."""
    (a,), (b,) = split_dets(det, nbits)
    out = []
    for i in range(nbits // 2):
        x, y = a >> i & 1, b >> i & 1
        out.append("2" if x and y else "u" if x else "d" if y else "0")
    return "".join(out)


def from_canonical_string(s, nbits=64):
    a = b = 0
    for i, ch in enumerate(s):
        if ch in "2u":
            a |= 1 << i
        if ch in "2d":
            b |= 1 << i
    return make_dets([a], [b], nbits)


def det_less_order(dets):
    """Permutation sorting determinants by bitset_less (most significant word
    first, include/macis/bitset_operations.hpp:289-306)."""
    dets = np.asarray(dets, dtype=np.uint64)
    return np.lexsort(tuple(dets[:, j] for j in range(dets.shape[1])))
