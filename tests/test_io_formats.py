"""On-disk formats on the host (no GPU): the formatter of the engine library
(mdff_io_format) against the reference's own CONTFF of examples/ex1/ref
byte for byte, Fortran edit-descriptor corner cases, and write -> read round
trips of every format and form through mdff_b200.io's readers.
"""
import hashlib
import os

import numpy as np
import pytest

from mdff_b200 import io

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REF = os.environ.get("MDFF_REFERENCE", "/root/reference")


def ex1_frame():
    d = np.load(os.path.join(GOLD, "ex1_final.npz"))
    n = len(d["pos"])
    h = io.header("UNKNOWN", ["A"], natmi=[n], cell=d["cell"], natm=n)
    cols = np.concatenate([d["pos"].T, d["vel"].T, d["force"].T])
    return h, np.ones(n, np.int32), cols


def test_contff_matches_reference_bytes():
    # write_CONTFF (src/config.f90:206-250) of the ex1 final state: the
    # reference's CONTFF, 12-digit values re-printed from their parsed doubles
    h, it, cols = ex1_frame()
    out = io.format_frame("CONTFF", 1, "rvf", h, it, cols)
    head = open(os.path.join(GOLD, "ex1_contff_head.txt"), "rb").read()
    assert out[:len(head)] == head
    digest = open(os.path.join(GOLD, "ex1_contff.sha256")).read().split()[0]
    assert hashlib.sha256(out).hexdigest() == digest


def E(v, w=20, d=12):
    h = io.header("x", ["A"], natmi=[1], cell=np.eye(3), natm=1)
    out = io.format_frame("TRAJFF", 1, "rnn", h, [1], np.array([[v], [0.0], [0.0]])).decode()
    return out.split("\n")[9][3:3 + w]


def test_edit_descriptor_E():
    assert E(1.5) == "  0.150000000000E+01"
    assert E(-1.5) == " -0.150000000000E+01"
    assert E(0.0) == "  0.000000000000E+00"
    assert E(9.9999999999995) == "  0.100000000000E+02"      # rounds up into the next decade
    assert E(1.0e120) == "  0.100000000000+121"            # three-digit exponent drops the letter
    assert E(-2.5e-100) == " -0.250000000000E-99"
    assert E(-2.5e-101) == " -0.250000000000-100"
    assert E(123456.789) == "  0.123456789000E+06"


def test_trajff_header_layout():
    h = io.header("MgO test", ["O", "Mg"], natmi=[2, 1], cell=np.diag([4.2, 4.3, 4.4]), natm=3)
    out = io.format_frame("TRAJFF", 1, "rnn", h, [1, 1, 2], np.zeros((3, 3))).decode().split("\n")
    assert out[0] == "     3"                                  # (i6)
    assert out[1] == "MgO test".ljust(60)                      # (a) of character(len=60)
    assert out[2] == "      4.200000000000      0.000000000000      0.000000000000"   # (3f20.12)
    assert out[5] == "   2"                                    # (i4)
    assert out[6] == " O   Mg "                                # list-directed labels
    assert out[7] == "           2           1"                # list-directed integers
    assert out[8] == "Cartesian"
    assert out[11].startswith("Mg   0.000000000000E+00")


def rand_frame(rng, n=7, ntype=2):
    it = rng.integers(1, ntype + 1, n).astype(np.int32)
    natmi = [int(np.sum(it == t)) for t in range(1, ntype + 1)]
    cell = np.diag(rng.uniform(8, 12, 3)) + rng.normal(0, 0.3, (3, 3))
    h = io.header("round trip", ["O", "Mg"][:ntype], natmi=natmi, cell=cell, natm=n)
    return h, it, natmi, cell


@pytest.mark.parametrize("data", ["rvf", "rvn", "rnf", "rnn"])
@pytest.mark.parametrize("iformat", [0, 1])
def test_trajff_round_trip(tmp_path, data, iformat):
    rng = np.random.default_rng(3)
    h, it, natmi, cell = rand_frame(rng)
    ncol = 3 + 3 * (data[1] == "v") + 3 * (data[2] == "f")
    frames = [rng.normal(0, 5, (ncol, 7)) for _ in range(3)]
    p = tmp_path / "TRAJFF"
    with open(p, "wb") as f:
        for c in frames:
            f.write(io.format_frame("TRAJFF", iformat, data, h, it, c))
    got = io.read_trajff(p, iformat, data)
    assert len(got) == 3
    tol = 0 if iformat == 0 else 5e-12
    for fr, c in zip(got, frames):
        assert fr["natm"] == 7 and fr["labels"] == ["O", "Mg"] and fr["natmi"] == natmi
        assert fr["system"] == "round trip"
        # write_trajff_xyz writes the rows of simu_cell%A: read back as columns
        assert np.allclose(fr["cell"], cell.T, rtol=0, atol=1e-12 if iformat else 0)
        assert np.allclose(fr["r"], c[0:3].T, rtol=tol, atol=0)
        k = 3
        if data[1] == "v":
            assert np.allclose(fr["v"], c[k:k + 3].T, rtol=tol, atol=0)
            k += 3
        if data[2] == "f":
            assert np.allclose(fr["f"], c[k:k + 3].T, rtol=tol, atol=0)
        if iformat:
            assert fr["atype"] == [["O", "Mg"][t - 1] for t in it]


@pytest.mark.parametrize("iformat", [0, 1])
def test_efgall_round_trip(tmp_path, iformat):
    rng = np.random.default_rng(4)
    h, it, natmi, cell = rand_frame(rng)
    efg = rng.normal(0, 2, (6, 7))
    p = tmp_path / "EFGALL"
    p.write_bytes(io.format_frame("EFGALL", iformat, 0, h, it, efg) * 2)
    got = io.read_efgall(p, iformat)
    assert len(got) == 2
    for fr in got:
        assert np.allclose(fr["efg"], efg.T, rtol=0 if iformat == 0 else 1e-15, atol=0)
        assert np.allclose(fr["cell"], cell, rtol=0, atol=0 if iformat == 0 else 1e-15)
        assert fr["natmi"] == natmi


@pytest.mark.parametrize("kind", ["DIPFF", "EFALL"])
def test_vector_files_round_trip(tmp_path, kind):
    rng = np.random.default_rng(5)
    h, it, natmi, cell = rand_frame(rng)
    v = rng.normal(0, 1, (3, 7))
    p = tmp_path / kind
    p.write_bytes(io.format_frame(kind, 1, 0, h, it, v))
    (fr,) = io.read_vectors(p)
    assert np.allclose(fr["values"], v.T, rtol=1e-15, atol=0)
    assert fr["atype"] == [["O", "Mg"][t - 1] for t in it]
    # the reference writes these formatted only
    with pytest.raises(ValueError):
        io.format_frame(kind, 0, 0, h, it, v)


def test_bad_type_index_rejected():
    h = io.header("x", ["A"], natmi=[1], cell=np.eye(3), natm=1)
    with pytest.raises(ValueError):
        io.format_frame("TRAJFF", 1, "rnn", h, [2], np.zeros((3, 1)))


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
def test_reads_reference_inputs():
    # the reference's own input files parse as read_traj reads them
    two = io.read_trajff(os.path.join(REF, "examples/ex4/TRAJFF.twocharges"), 1, "rvf")[0]
    assert two["natm"] == 2 and two["labels"] == ["A", "B"] and two["r"][0, 0] == 0.5
    pos = io.read_trajff(os.path.join(REF, "examples/ex1/POSFF"), 1, "rnn")[0]
    assert pos["natm"] == 256 and pos["coord"] == "Direct"
    assert abs(pos["r"][1, 0] - 0.125 * 20.993868) < 1e-12


@pytest.mark.parametrize("kind,w,d", [("TRAJFF", 20, 12), ("DIPFF", 24, 16)])
def test_digits_are_correctly_rounded(kind, w, d):
    # the formatter's fast digit path against Python's correctly rounded
    # conversion, over 60 decades and at rounding ties of the last digit
    rng = np.random.default_rng(11)
    v = rng.normal(0, 1, 6000) * 10.0 ** rng.integers(-30, 30, 6000)
    ties = np.array([float(f"1.{'2' * (d - 2)}35e{k}") for k in range(-8, 9)])
    v = np.concatenate([v, ties, -ties, [1e-25, 3e24, 9.9999999999995, 0.5]])
    n = len(v)
    h = io.header("x", ["A"], natmi=[n], cell=np.eye(3), natm=n)
    text = io.format_frame(kind, 1, "rnn", h, np.ones(n, np.int32), np.stack([v, v, v])).decode().split("\n")
    rows = text[9:9 + n]
    for x, line in zip(v, rows):
        field = line[3:3 + w] if kind == "TRAJFF" else line[13:13 + w]
        m = f"{abs(x):.{d - 1}e}"
        e = int(m.split("e")[1]) + 1
        ex = f"E{e:+03d}" if abs(e) <= 99 else f"{e:+04d}"
        want = ("-" if x < 0 else "") + "0." + m[0] + m[2:d + 1] + ex
        assert field.strip() in (want, want.replace("0.", ".", 1)), (x, field, want)
