"""File formats (macis_b200.io) on the CPU: FCIDUMP (fcidump.cxx:78-200),
ASCII wavefunctions (wavefunction_io.hpp:39-114), binary RDMs
(fcidump.cxx:202-280)."""
import struct

import numpy as np
import pytest

import macis_b200 as mb
from macis_b200 import io as mio
from golden_data import water


def test_fcidump_round_trip_water(tmp_path, ref):
    norb, T, V, ecore = water()
    f = tmp_path / "FCIDUMP"
    mio.write_fcidump(f, norb, T, V, ecore)
    # the reference's writer (fcidump.cxx:184-207) writes the same bytes
    ref.write_fcidump(tmp_path / "FCIDUMP.ref", norb, T, V, ecore)
    assert f.read_bytes() == (tmp_path / "FCIDUMP.ref").read_bytes()
    n, T2, V2, e2 = mio.read_fcidump(f)
    assert n == norb and e2 == ecore
    assert np.array_equal(T2, np.asarray(T).ravel(order="F"))
    assert np.array_equal(V2, np.asarray(V).ravel(order="F"))
    lines = f.read_text().splitlines()
    assert len(lines) == norb ** 4 + norb ** 2 + 1
    assert lines[0] == f"{1:8d} {1:8d} {1:8d} {1:8d} {V2[0]:25.16e}"
    assert lines[-1].split()[:4] == ["0", "0", "0", "0"]


def test_fcidump_reader_rules(tmp_path, ref):
    f = tmp_path / "FCIDUMP"
    f.write_text(
        " &FCI NORB=  3,NELEC=2,MS2=0,\n"
        "  ORBSYM=1,1,1,\n"
        "  ISYM=1,\n"
        " &END\n"
        "  0.5 1 1 2 2\n"                  # value first
        "3 3 1 1   0.25\n"                 # value last, extra spaces
        "  -1.0 1 2 0 0\n"                 # one-body, symmetric fill
        "   2.0 3 3 0 0\n"
        "   7.5 0 0 0 0\n"                 # core: the first one counts
        "   9.9 0 0 0 0\n")
    n, T, V, e = mio.read_fcidump(f)
    assert n == 3 and e == 7.5
    Tm = T.reshape(3, 3, order="F")
    Vm = V.reshape(3, 3, 3, 3, order="F")
    assert Tm[0, 1] == Tm[1, 0] == -1.0 and Tm[2, 2] == 2.0
    assert Vm[0, 0, 1, 1] == Vm[1, 1, 0, 0] == 0.5
    assert Vm[2, 2, 0, 0] == Vm[0, 0, 2, 2] == 0.25
    assert np.count_nonzero(V) == 4
    # the same file through the reference's readers (fcidump.cxx:78-182)
    nr, Tr, Vr, er = ref.read_fcidump(f)
    assert (nr, er) == (n, e)
    assert np.array_equal(Tr, T) and np.array_equal(Vr, V)
    bad = tmp_path / "BAD"
    bad.write_text("1.0 1 1 1 2.0\n")     # value at both ends
    with pytest.raises(RuntimeError, match="Invalid FCIDUMP Line"):
        mio.read_fcidump(bad)
    with pytest.raises(RuntimeError, match="Invalid FCIDUMP Line"):
        ref.read_fcidump(bad)


@pytest.mark.parametrize("nbits", [64, 128, 256])
def test_wavefunction_round_trip(tmp_path, nbits):
    dets = mb.generate_hilbert_space(6, 3, 2, nbits)[:40]
    c = np.random.default_rng(0).standard_normal(len(dets))
    f = tmp_path / "wfn.dat"
    mio.write_wavefunction(f, 6, dets, c, nbits)
    lines = f.read_text().splitlines()
    assert lines[0] == f"{len(dets)} 6 3 2"
    assert lines[1] == f"{c[0]:30.16e} {mb.to_canonical_string(dets[0], nbits)} "
    assert len(lines[1].split()[1]) == nbits // 2
    d2, c2 = mio.read_wavefunction(f, nbits)
    assert np.array_equal(d2, np.asarray(dets).reshape(len(dets), -1))
    assert np.array_equal(c2, c)
    with pytest.raises(RuntimeError, match="Invalid Wave Function"):
        mio.write_wavefunction(f, 6, dets, c[:-1], nbits)


def test_wavefunction_reader_rules(tmp_path, ref):
    """wavefunction_io.hpp:39-74: stoi of the four header fields, then
    every line a determinant (stod of its coefficient) -- checked against
    the compiled reference reader on the same files."""
    f = tmp_path / "wfn.dat"

    def both(text):
        f.write_text(text)
        return mio.read_wavefunction(f), ref.read_wavefunction(f)

    (d, c), (dr, cr) = both("2 4 1 1\n  0.5e0 2000 \n-0.25 ud\n")
    assert np.array_equal(c, [0.5, -0.25])
    assert np.array_equal(d[:, 0], [1 | (1 << 32), 1 | (2 << 32)])
    assert np.array_equal(d, dr) and np.array_equal(c, cr)
    # no string: the empty determinant; extra tokens ignored
    (d, c), (dr, cr) = both("2 4 1 1\n0.5 2000 x y\n0.7\n")
    assert d[1, 0] == 0 and c[1] == 0.7
    assert np.array_equal(d, dr) and np.array_equal(c, cr)
    # the writers agree byte for byte (64-bit determinants)
    dets = mb.generate_hilbert_space(6, 3, 2, 64)[:25]
    cf = np.random.default_rng(2).standard_normal(len(dets)) * 1e-3
    mio.write_wavefunction(tmp_path / "a.dat", 6, dets, cf)
    ref.write_wavefunction(tmp_path / "b.dat", 6, dets, cf)
    assert (tmp_path / "a.dat").read_bytes() == (tmp_path / "b.dat").read_bytes()
    with pytest.raises(RuntimeError, match="Invalid Wave Function"):
        ref.write_wavefunction(tmp_path / "b.dat", 6, dets, cf[:-1])
    # a blank line, a short header: both readers raise
    for text in ("2 4 1 1\n0.5 2000\n\n0.1 ud\n", "2 4 1\n0.5 2000\n"):
        f.write_text(text)
        with pytest.raises(ValueError):
            mio.read_wavefunction(f)
        with pytest.raises(RuntimeError):
            ref.read_wavefunction(f)


def test_rdms_binary_round_trip(tmp_path, ref):
    n = 4
    rng = np.random.default_rng(1)
    o, t = rng.standard_normal(n * n), rng.standard_normal(n ** 4)
    f = tmp_path / "rdms.bin"
    mio.write_rdms_binary(f, n, o, t)
    raw = f.read_bytes()
    ref.write_rdms_binary(tmp_path / "rdms.ref", n, o, t)
    assert (tmp_path / "rdms.ref").read_bytes() == raw
    assert struct.unpack("i", raw[:4])[0] == n
    assert len(raw) == 4 + 8 * (n * n + n ** 4)
    o2, t2 = mio.read_rdms_binary(f, n)
    assert np.array_equal(o2, o) and np.array_equal(t2, t)
    with pytest.raises(RuntimeError, match="NORB in RDM file"):
        mio.read_rdms_binary(f, n + 1)
    # short files (fcidump.cxx:235-249 reads into one zeroed buffer): a
    # missing 2-RDM keeps the 1-RDM bytes at its start, the rest is zero
    f.write_bytes(raw[:4 + 8 * n * n])
    o3, t3 = mio.read_rdms_binary(f, n)
    assert np.array_equal(o3, o)
    assert np.array_equal(t3[:n * n], o) and not t3[n * n:].any()
    f.write_bytes(raw[:4 + 8 * (n * n + 5)])
    o4, t4 = mio.read_rdms_binary(f, n)
    assert np.array_equal(o4, o)
    assert np.array_equal(t4[:5], t[:5]) and np.array_equal(t4[5:n * n], o[5:])
    assert not t4[n * n:].any()
    f.write_bytes(raw[:4 + 8 * 3])
    o5, t5 = mio.read_rdms_binary(f, n)
    assert np.array_equal(o5[:3], o[:3]) and not o5[3:].any()
    assert np.array_equal(t5[:3], o[:3]) and not t5[3:].any()
    # the reference reader on the same short files
    for k in (4 + 8 * n * n, 4 + 8 * (n * n + 5), 4 + 8 * 3, len(raw)):
        f.write_bytes(raw[:k])
        ours, theirs = mio.read_rdms_binary(f, n), ref.read_rdms_binary(f, n)
        assert np.array_equal(ours[0], theirs[0])
        assert np.array_equal(ours[1], theirs[1])
    with pytest.raises(RuntimeError, match="NORB in RDM file"):
        ref.read_rdms_binary(f, n + 1)
