"""The reference's file formats, host side.

* FCIDUMP integrals: ``read_fcidump`` / ``write_fcidump``
  (src/macis/fcidump.cxx:78-200).
* ASCII CI wavefunctions: ``read_wavefunction`` / ``write_wavefunction``
  (include/macis/wavefunction_io.hpp:39-114).
* Binary RDMs: ``read_rdms_binary`` / ``write_rdms_binary``
  (src/macis/fcidump.cxx:202-280).

Integrals and RDMs are flat column-major float64 arrays, the layout the
rest of the package (and the reference's spans) use.
"""
import re
import struct

import numpy as np

from .sd import from_canonical_string, split_dets, to_canonical_string

__all__ = ["read_fcidump", "write_fcidump", "read_wavefunction",
           "write_wavefunction", "read_rdms_binary", "write_rdms_binary"]

_INT = re.compile(r"\s*[+-]?\d+")
_FLT = re.compile(r"\s*[+-]?(\d+\.?\d*([eE][+-]?\d+)?|\.\d+([eE][+-]?\d+)?|"
                  r"inf|infinity|nan)", re.IGNORECASE)


def _stoi(tok):
    """Leading integer of a token, as std::stoi reads it."""
    m = _INT.match(tok)
    if not m:
        raise ValueError(f"stoi: no conversion of {tok!r}")
    return int(m.group(0))


def _stod(tok):
    """Leading number of a token, as std::stod reads it."""
    m = _FLT.match(tok)
    if not m:
        raise ValueError(f"stod: no conversion of {tok!r}")
    return float(m.group(0))


def _is_float(tok):
    # fcidump.cxx:31-34: a letter or a '.' marks the integral value
    return any(c.isalpha() or c == "." for c in tok)


def _fcidump_lines(fname):
    """(p, q, r, s, value) of every line with five space-separated tokens
    (fcidump.cxx:36-62, 78-94); other lines are skipped."""
    with open(fname) as f:
        for line in f:
            tokens = [t for t in line.rstrip("\n").split(" ") if t]
            if len(tokens) != 5:
                continue
            idx_first = _is_float(tokens[-1])
            if idx_first and _is_float(tokens[0]):
                raise RuntimeError("Invalid FCIDUMP Line")
            if idx_first:
                p, q, r, s = (_stoi(t) for t in tokens[:4])
                v = _stod(tokens[4])
            else:
                p, q, r, s = (_stoi(t) for t in tokens[1:])
                v = _stod(tokens[0])
            if min(p, q, r, s) < 0:
                raise RuntimeError("Invalid Orb Idx")
            yield p, q, r, s, v


def read_fcidump(fname):
    """(norb, T, V, E_core) from an FCIDUMP file: norb is the largest
    orbital index (read_fcidump_norb), E_core the first all-zero-index line
    (read_fcidump_core, 0 without one), one-body lines fill T symmetrically
    and two-body lines V with its eight-fold symmetry (read_fcidump_1body /
    _2body, fcidump.cxx:96-174)."""
    lines = list(_fcidump_lines(fname))
    n = max((max(l[:4]) for l in lines), default=0)
    T = np.zeros((n, n), order="F")
    V = np.zeros((n, n, n, n), order="F")
    ecore = None
    for p, q, r, s, v in lines:
        if not (p or q or r or s):
            if ecore is None:
                ecore = v
        elif p and q and r and s:
            p, q, r, s = p - 1, q - 1, r - 1, s - 1
            for a, b, c, d in ((p, q, r, s), (p, q, s, r), (q, p, r, s),
                               (q, p, s, r), (r, s, p, q), (s, r, p, q),
                               (r, s, q, p), (s, r, q, p)):
                V[a, b, c, d] = v
        else:
            if not (p and q):
                raise RuntimeError("Invalid Orb Idx")
            T[p - 1, q - 1] = v
            T[q - 1, p - 1] = v
    return (n, np.ascontiguousarray(T.ravel(order="F")),
            np.ascontiguousarray(V.ravel(order="F")),
            0.0 if ecore is None else ecore)


def write_fcidump(fname, norb, T, V, E_core):
    """Every two-body element (i outermost), every one-body element, then
    the core energy, one '{:8} {:8} {:8} {:8} {:25.16e}' line each
    (write_fcidump, fcidump.cxx:186-200)."""
    n = int(norb)
    T = np.asarray(T, dtype=np.float64).reshape(-1, order="F")
    V = np.asarray(V, dtype=np.float64).reshape(-1, order="F")
    if T.size != n * n or V.size != n ** 4:
        raise RuntimeError("T / V have incorrect dimensions")
    Vm = V.reshape(n, n, n, n, order="F")
    with open(fname, "w") as f:
        for i in range(n):
            for j in range(n):
                for k in range(n):
                    row = Vm[i, j, k, :]
                    f.write("".join(f"{i + 1:8d} {j + 1:8d} {k + 1:8d} "
                                    f"{l + 1:8d} {row[l]:25.16e}\n"
                                    for l in range(n)))
        Tm = T.reshape(n, n, order="F")
        for i in range(n):
            for j in range(n):
                f.write(f"{i + 1:8d} {j + 1:8d} {0:8d} {0:8d} "
                        f"{Tm[i, j]:25.16e}\n")
        f.write(f"{0:8d} {0:8d} {0:8d} {0:8d} {float(E_core):25.16e}\n")


def _counts(det, nbits):
    a, b = split_dets(np.asarray(det).reshape(1, -1), nbits)
    return (sum(bin(int(x)).count("1") for x in np.ravel(a)),
            sum(bin(int(x)).count("1") for x in np.ravel(b)))


def write_wavefunction(fname, norb, dets, coeffs, nbits=64):
    """'<NSTATE> <NORB> <NALPHA> <NBETA>' then one '<COEFF> <STR> ' line per
    determinant, COEFF in %30.16e and STR the canonical string of all N/2
    spin orbitals (write_wavefunction, wavefunction_io.hpp:88-114; NALPHA /
    NBETA from the first determinant). Nothing is written for no states."""
    dets = np.asarray(dets, dtype=np.uint64).reshape(-1, nbits // 64)
    coeffs = np.asarray(coeffs, dtype=np.float64)
    if len(dets) != len(coeffs):
        raise RuntimeError("Invalid Wave Function Dimensions")
    if not len(dets):
        return
    na, nb = _counts(dets[0], nbits)
    with open(fname, "w") as f:
        f.write(f"{len(dets)} {int(norb)} {na} {nb}\n")
        for d, c in zip(dets, coeffs):
            f.write(f"{c:30.16e} {to_canonical_string(d, nbits)} \n")


def read_wavefunction(fname, nbits=64):
    """(dets, coeffs) of an ASCII wavefunction file (read_wavefunction,
    wavefunction_io.hpp:39-74): the header line, whose four fields must
    parse as integers, then one '<COEFF> <STR>' line per determinant. As
    there, every later line is a determinant: a blank one has no
    coefficient and raises, a missing string is the empty determinant."""
    dets, coeffs = [], []
    with open(fname) as f:
        head = f.readline().split()
        for tok in (head + [""] * 4)[:4]:
            _stoi(tok)
        for line in f:
            tok = line.split() + ["", ""]
            dets.append(from_canonical_string(tok[1], nbits)[0])
            coeffs.append(_stod(tok[0]))
    W = nbits // 64
    out = (np.asarray(dets, dtype=np.uint64).reshape(-1, W) if dets
           else np.zeros((0, W), dtype=np.uint64))
    return out, np.asarray(coeffs, dtype=np.float64)


def write_rdms_binary(fname, norb, ordm, trdm):
    """int32 norb, the norb^2 1-RDM and the norb^4 2-RDM as raw
    column-major float64 (write_rdms_binary, fcidump.cxx:252-280)."""
    n = int(norb)
    o = np.asarray(ordm, dtype=np.float64).reshape(-1, order="F")
    t = np.asarray(trdm, dtype=np.float64).reshape(-1, order="F")
    if o.size != n * n or t.size != n ** 4:
        raise RuntimeError("RDMs have incorrect dimensions")
    with open(fname, "wb") as f:
        f.write(struct.pack("i", n))
        f.write(o.tobytes())
        f.write(t.tobytes())


def read_rdms_binary(fname, norb):
    """(ordm, trdm) flat column-major from a binary RDM file; the stored
    norb must match (read_rdms_binary, fcidump.cxx:209-250). Both reads go
    into one zero-initialised norb^4 buffer, as there, so a short file
    leaves the bytes it lacks as that buffer held them: zeros, or for the
    2-RDM the 1-RDM bytes read before."""
    n = int(norb)
    with open(fname, "rb") as f:
        head = f.read(4)
        if len(head) != 4:
            raise RuntimeError(f"{fname} not available")
        nr = struct.unpack("i", head)[0]
        if nr != n:
            raise RuntimeError(f"NORB in RDM file doesn't match {n} {nr}")
        raw = bytearray(n ** 4 * 8)
        b = f.read(n * n * 8)
        raw[:len(b)] = b
        o = np.frombuffer(bytes(raw[:n * n * 8]), dtype=np.float64).copy()
        b = f.read(n ** 4 * 8)
        raw[:len(b)] = b
        t = np.frombuffer(bytes(raw), dtype=np.float64).copy()
    return o, t
