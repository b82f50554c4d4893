"""CPU restatement of the learned screening network and of its ASCI unit
inputs -- TEST INFRASTRUCTURE ONLY (imported by ``tests/`` as the checker).

The network has no MACIS counterpart, so this file is its specification:

* ``forward`` / ``gradients`` -- din -> 256 -> 256 -> 1 with GELU (erf form),
  loss sum_i (y_i - t_i)^2 / (2 n). With ``bf16=True`` the rounding points of
  the device kernels are reproduced: W1, W2 and the inputs are BF16, H1 is
  rounded to BF16 before layer 2, dZ2 and dZ1 are rounded to BF16 before the
  weight-gradient and dH1 products (the BF16 tensor-core operands); all
  other arithmetic is float64 here (FP32 on the device). With ``bf16=False``
  it is the plain float64 network, whose gradient ``tests/`` checks against
  finite differences.
* ``adam`` -- the Adam update (beta1 0.9, beta2 0.999, eps 1e-8, bias
  corrected).
* ``unit_features`` -- the network input of every unit of an ASCI search,
  in the unit order of the search: per core det the alpha singles, the beta
  singles, the (i, a) outer pairs of append_ss_doubles (alpha, then beta) and
  of append_os_doubles (include/macis/asci/determinant_contributions.hpp:
  26-160). Orbital energies and diagonals come from the C port
  (single_orbital_ens, fast_diagonals.hpp:34-53; matrix_element diag); the
  outer-pair integral bounds from ``pair_bounds``.

Parity is unpinned against MACIS (the network is not part of it); it is
pinned by the finite-difference check of the float64 gradient.
"""
import numpy as np
from scipy.special import erf

H = 256
NFEAT = 64
EPS_ORBS = 48


# ------------------------------------------------------------------ BF16
def bf16_round(x):
    """float32 -> nearest BF16 value (round half to even), as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(
        np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def bf16_bits(x):
    u = bf16_round(x).view(np.uint32)
    return (u >> 16).astype(np.uint16)


def bf16_value(bits):
    return (np.asarray(bits, dtype=np.uint32) << 16).view(np.float32)


# -------------------------------------------------------------- network
def layout(din):
    off = {}
    o = 0
    for name, size in (("W1", H * din), ("b1", H), ("W2", H * H), ("b2", H),
                       ("w3", H), ("b3", 1)):
        off[name] = (o, o + size)
        o += size
    return off, o


def unpack(P, din):
    off, _ = layout(din)
    P = np.asarray(P, dtype=np.float64)
    g = {k: P[a:b] for k, (a, b) in off.items()}
    return (g["W1"].reshape(H, din), g["b1"], g["W2"].reshape(H, H), g["b2"],
            g["w3"], g["b3"][0])


def pack(din, W1, b1, W2, b2, w3, b3):
    return np.concatenate([np.ravel(W1), b1, np.ravel(W2), b2, w3,
                           [b3]]).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(
        -0.5 * z * z) / np.sqrt(2.0 * np.pi)


def _r(x, on):
    return bf16_round(x).astype(np.float64) if on else x


def forward(P, X, din, bf16=True):
    """X: float array [n][din] (BF16 values when bf16). Returns y, cache."""
    W1, b1, W2, b2, w3, b3 = unpack(P, din)
    if bf16:
        W1 = _r(W1, True)
        W2 = _r(W2, True)
    X = np.asarray(X, dtype=np.float64)
    z1 = X @ W1.T + b1
    h1 = _r(gelu(z1), bf16)
    z2 = h1 @ W2.T + b2
    h2 = gelu(z2)
    y = h2 @ w3 + b3
    return y, dict(X=X, W1=W1, W2=W2, w3=w3, z1=z1, h1=h1, z2=z2, h2=h2)


def gradients(P, X, t, din, bf16=True):
    """Gradient of sum (y - t)^2 / (2 n); returns (grad in the parameter
    layout, loss)."""
    y, c = forward(P, X, din, bf16)
    n = len(y)
    e = y - np.asarray(t, dtype=np.float64)
    loss = float(e @ e) / (2 * n)
    dy = e / n
    dw3 = c["h2"].T @ dy
    db3 = dy.sum()
    dz2 = dy[:, None] * c["w3"][None, :] * gelu_grad(c["z2"])
    db2 = dz2.sum(axis=0)
    dz2o = _r(dz2, bf16)
    dW2 = dz2o.T @ c["h1"]
    dh1 = dz2o @ c["W2"]
    dz1 = dh1 * gelu_grad(c["z1"])
    db1 = dz1.sum(axis=0)
    dW1 = _r(dz1, bf16).T @ c["X"]
    return pack(din, dW1, db1, dW2, db2, dw3, db3), loss


def adam(P, G, M, V, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (step counts from 1); returns new (P, M, V)."""
    M = b1 * M + (1 - b1) * G
    V = b2 * V + (1 - b2) * G * G
    P = P - lr * (M / (1 - b1 ** step)) / (np.sqrt(V / (1 - b2 ** step)) + eps)
    return P, M, V


# ----------------------------------------------------------- unit inputs
def unit_width(nbits):
    nsw = 2 if nbits == 256 else 1
    return 2 * 64 * nsw + NFEAT


def _spins(det, nbits):
    w = [int(x) for x in det]
    if nbits == 64:
        return w[0] & 0xFFFFFFFF, w[0] >> 32
    if nbits == 128:
        return w[0], w[1]
    return w[0] | (w[1] << 64), w[2] | (w[3] << 64)


def _unit_list(na, nb, nva, nvb):
    units = [(0, 0, 0, na * nva), (1, 0, 0, nb * nvb)]
    units += [(2, i, a, (na - 1 - i) * (nva - 1 - a))
              for i in range(na) for a in range(nva)]
    units += [(3, i, a, (nb - 1 - i) * (nvb - 1 - a))
              for i in range(nb) for a in range(nvb)]
    units += [(4, i, a, nb * nvb) for i in range(na) for a in range(nva)]
    return units


def pair_bounds(V, norb):
    """maxG[i, a] = max_{b,j} |G(b,j,a,i)|, maxV[i, a] = max_{b,j}
    |V(a,i,b,j)| with G(i,j,k,l) = V(i,j,k,l) - V(i,l,k,j) (the G
    intermediate of hamiltonian_generator/impl.hpp:26-43)."""
    V4 = np.asarray(V, dtype=np.float64).reshape((norb,) * 4, order="F")
    G4 = V4 - V4.transpose(0, 3, 2, 1)
    maxG = np.abs(G4).max(axis=(0, 1)).T   # [a, i] -> [i, a]
    maxV = np.abs(V4).max(axis=(2, 3)).T
    return maxG, maxV


def unit_features(port, h, nbits, norb, cdets, E0, C, V):
    """Float32 inputs [U][width] (BF16 values) of every unit, in order."""
    nsw = 2 if nbits == 256 else 1
    width = unit_width(nbits)
    maxG, maxV = pair_bounds(V, norb)
    rows = []
    for c, det in enumerate(np.asarray(cdets, dtype=np.uint64)):
        sp = list(_spins(det, nbits))
        occ = [[p for p in range(norb) if (s >> p) & 1] for s in sp]
        vir = [[p for p in range(norb) if not (s >> p) & 1] for s in sp]
        eps = [port.single_orbital_ens(h, occ[0], occ[1]),
               port.single_orbital_ens(h, occ[1], occ[0])]
        hd = port.matrix_element(h, det[None, :], det[None, :])[0]
        lnC = np.log(abs(float(C[c])) + 1e-300) / 10.0
        for kind, ii, aa, ninner in _unit_list(len(occ[0]), len(occ[1]),
                                               len(vir[0]), len(vir[1])):
            s2 = list(sp)
            S, hole, part = 0, -1, -1
            if kind >= 2:
                S = 1 if kind == 3 else 0
                hole, part = occ[S][ii], vir[S][aa]
                s2[S] ^= (1 << hole) | (1 << part)
            x = np.zeros(width, dtype=np.float64)
            for s in range(2):
                for p in range(64 * nsw):
                    x[s * 64 * nsw + p] = (s2[s] >> p) & 1
            eh = eps[S][hole] if hole >= 0 else 0.0
            ep = eps[S][part] if part >= 0 else 0.0
            f = np.zeros(NFEAT)
            f[0] = 1.0
            f[1] = lnC
            f[2 + kind] = 1.0
            f[7], f[8], f[9] = eh, ep, ep - eh
            f[10] = E0 - hd
            f[11] = np.log(1.0 + ninner) / 10.0
            lnc = np.log(abs(float(C[c])) + 1e-300)
            if hole >= 0:
                f[12] = np.float32(hole + 1) / np.float32(norb)
                f[13] = np.float32(part + 1) / np.float32(norb)
                bound = (maxV if kind == 4 else maxG)[hole, part]
                lb = np.log(bound + 1e-300)
                f[14] = lb / 10.0
                f[15] = (lnc + lb - np.log(abs(E0 - hd - (ep - eh)) + 1e-3)) \
                    / 10.0
            else:
                f[15] = (lnc - np.log(abs(E0 - hd) + 1e-3)) / 10.0
            for p in range(min(norb, EPS_ORBS)):
                e = 0.0
                if (s2[0] >> p) & 1:
                    e += eps[0][p]
                if (s2[1] >> p) & 1:
                    e += eps[1][p]
                f[16 + p] = e
            x[2 * 64 * nsw:] = f
            rows.append(x)
    X = np.array(rows, dtype=np.float64).reshape(-1, width)
    return bf16_round(X.astype(np.float32))


def unit_targets(umax):
    """(ln max(|rv|, 1e-12) + 20) / 5 per unit."""
    return (np.log(np.maximum(np.asarray(umax, np.float32), 1e-12)) + 20) / 5
