"""MDFF's on-disk formats: readers, the host formatter and the streaming writer.

Formats, each as the reference reads or writes it:

* TRAJFF: write_trajff_xyz / read_traj (src/config.f90:539-788). Formatted (itraj_format != 0) or Fortran unformatted sequential (== 0), with trajff_data rvf, rvn, rnf or rnn. POSFF uses the same layout.
* CONTFF: write_CONTFF (src/config.f90:206-250), formatted rvf.
* EFGALL: write_EFGALL (src/field.f90:4140-4195) and efg_stat's reader (src/efg.f90:2183-2222). Formatted has six components per site; unformatted has the full efg_t(natm, 3, 3).
* DIPFF and EFALL: write_DIPFF / write_EFALL (src/field.f90:4051-4240).

The writers are in the engine library: mdff_io_format formats a frame from host arrays, and Writer streams frames from the device. The readers here parse the formats back, with list-directed fields split on blanks as a Fortran list-directed READ does.
"""
import ctypes as C
import struct

import numpy as np

from . import abi

KINDS = {"TRAJFF": abi.FILE_TRAJFF, "CONTFF": abi.FILE_CONTFF, "EFGALL": abi.FILE_EFGALL,
         "DIPFF": abi.FILE_DIPFF, "EFALL": abi.FILE_EFALL}


def _kind(kind):
    return KINDS[kind] if isinstance(kind, str) else int(kind)


def _data(data):
    return abi.TRAJ_DATA[data] if isinstance(data, str) else int(data)


def header(system, labels, natmi=(), cell=None, natm=0):
    """mdff_frame_header from Python values: labels are the type names
    (atypei, at most 3 characters), cell rows are the lattice vectors."""
    h = abi.FrameHeader()
    h.natm = int(natm)
    h.ntype = len(labels)
    h.system = system.encode()[:60].ljust(60)
    for t, name in enumerate(labels):
        h.atypei[t].raw = name.encode()[:3].ljust(3)
    for t, k in enumerate(natmi):
        h.natmi[t] = int(k)
    if cell is not None:
        A = np.asarray(cell, dtype=np.float64)     # rows = lattice vectors -> column-major simu_cell%A
        for i in range(3):
            for j in range(3):
                h.A[i + 3 * j] = A[j, i]
    return h


def format_frame(kind, iformat, data, h, itype, cols):
    """One frame as bytes (mdff_io_format).  itype 1-based; cols [ncol][natm]."""
    from . import lib
    it = np.ascontiguousarray(itype, dtype=np.int32)
    c = np.ascontiguousarray(cols, dtype=np.float64)
    n = C.c_size_t()
    L = lib()
    args = (_kind(kind), int(iformat), _data(data), C.byref(h), it.ctypes.data_as(C.POINTER(C.c_int)),
            c.ctypes.data_as(C.POINTER(C.c_double)))
    guess = 4096 + c.size * 26 + it.size * 16          # above any frame's length: one formatting pass
    buf = C.create_string_buffer(guess)
    rc = L.mdff_io_format(*args, buf, guess, C.byref(n))
    if rc == abi.E_ARG and n.value > guess:
        buf = C.create_string_buffer(n.value)
        rc = L.mdff_io_format(*args, buf, n.value, C.byref(n))
    if rc != 0:
        raise ValueError(f"mdff_io_format failed ({rc})")
    return buf.raw[:n.value]


class Writer:
    """Streaming writer of an Engine's frames (mdff_writer_open / frame / close)."""

    def __init__(self, engine, path, kind, iformat=1, data="rvf", system="", labels=(), nslot=4):
        from . import lib
        self._e = engine
        self._w = C.c_void_p()
        h = header(system, labels)
        engine._check(lib().mdff_writer_open(engine._h, str(path).encode(), _kind(kind), int(iformat), _data(data),
                                             C.byref(h), int(nslot), C.byref(self._w)))

    def frame(self):
        from . import lib
        self._e._check(lib().mdff_writer_frame(self._w))

    def close(self):
        from . import lib
        if self._w:
            w, self._w = self._w, C.c_void_p()
            self._e._check(lib().mdff_writer_close(w))

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# ---- readers ----------------------------------------------------------------
def fortran_records(path):
    """Records of a Fortran unformatted sequential file (4-byte markers)."""
    raw = open(path, "rb").read()
    k = 0
    while k < len(raw):
        (m,) = struct.unpack_from("<i", raw, k)
        body = raw[k + 4:k + 4 + m]
        (m2,) = struct.unpack_from("<i", raw, k + 4 + m)
        if m2 != m:
            raise ValueError(f"{path}: record markers {m} / {m2} differ at byte {k}")
        yield body
        k += 8 + m


def _ffloat(tok):
    """A Fortran real field (E or D exponent, or a three-digit exponent
    written without the letter)."""
    t = tok.replace("D", "E").replace("d", "e")
    try:
        return float(t)
    except ValueError:
        for k in range(len(t) - 1, 0, -1):
            if t[k] in "+-" and t[k - 1].isdigit():
                return float(t[:k] + "E" + t[k:])
        raise


def _header_formatted(lines, k):
    natm = int(lines[k].split()[0])
    system = lines[k + 1].strip()
    A = np.array([[_ffloat(x) for x in lines[k + 2 + r].split()[:3]] for r in range(3)])
    ntype = int(lines[k + 5].split()[0])
    labels = lines[k + 6].split()[:ntype]
    natmi = [int(x) for x in lines[k + 7].split()[:ntype]]
    return {"natm": natm, "system": system, "cell": A, "ntype": ntype, "labels": labels, "natmi": natmi}, k + 8


def _dirkar(cell, s):
    """dirkar (src/lattice.f90:229-257): direct to Cartesian; cell rows are the
    lattice vectors."""
    A = np.asarray(cell).T
    return np.stack([s[:, 0] * A[0, 0] + s[:, 1] * A[0, 1] + s[:, 2] * A[0, 2],
                     s[:, 0] * A[1, 0] + s[:, 1] * A[1, 1] + s[:, 2] * A[1, 2],
                     s[:, 0] * A[2, 0] + s[:, 1] * A[2, 1] + s[:, 2] * A[2, 2]], axis=1)


def read_trajff(path, iformat=1, data="rvf"):
    """Frames of a TRAJFF (or POSFF / CONTFF with data 'rnn' / 'rvf') as
    read_traj reads them: dicts with natm, system, cell (row r = the three
    values of header line r, which read_traj takes as simu_cell%A(:, r)),
    ntype, labels, natmi, coord, atype (per-atom labels of formatted files),
    r, and v and f when data has them; Direct coordinates converted to
    Cartesian."""
    want_v, want_f = data[1] == "v", data[2] == "f"
    frames = []
    if iformat != 0:
        lines = open(path).read().split("\n")
        k = 0
        while k < len(lines) and lines[k].strip():
            fr, k = _header_formatted(lines, k)
            fr["coord"] = lines[k].split()[0]
            k += 1
            n = fr["natm"]
            rows = [lines[k + i].split() for i in range(n)]
            k += n
            fr["atype"] = [r[0] for r in rows]
            vals = np.array([[_ffloat(x) for x in r[1:]] for r in rows])
            c = 0
            fr["r"] = vals[:, c:c + 3]
            c += 3
            if want_v:
                fr["v"] = vals[:, c:c + 3]
                c += 3
            if want_f:
                fr["f"] = vals[:, c:c + 3]
            if fr["coord"] in ("Direct", "D"):
                fr["r"] = _dirkar(fr["cell"], fr["r"])
            frames.append(fr)
        return frames
    recs = list(fortran_records(path))
    k = 0
    while k < len(recs):
        natm = struct.unpack("<i", recs[k])[0]
        ntype = struct.unpack("<i", recs[k + 5])[0]
        arr = np.frombuffer(recs[k + 9], dtype="<f8").reshape(-1, natm)
        fr = {"natm": natm, "system": recs[k + 1].decode().strip(),
              "cell": np.array([struct.unpack("<3d", recs[k + 2 + r]) for r in range(3)]), "ntype": ntype,
              "labels": [recs[k + 6][3 * t:3 * t + 3].decode().strip() for t in range(ntype)],
              "natmi": list(struct.unpack(f"<{ntype}i", recs[k + 7])), "coord": recs[k + 8].decode().strip(),
              "r": arr[0:3].T.copy()}
        c = 3
        if want_v:
            fr["v"] = arr[c:c + 3].T.copy()
            c += 3
        if want_f:
            fr["f"] = arr[c:c + 3].T.copy()
        if fr["coord"] in ("Direct", "D"):
            fr["r"] = _dirkar(fr["cell"], fr["r"])
        frames.append(fr)
        k += 10
    return frames


def read_efgall(path, iformat=1):
    """Frames of an EFGALL: the header fields and efg [natm][6] (xx yy zz xy
    xz yz), as efg_stat reads them (src/efg.f90:2183-2222)."""
    frames = []
    if iformat != 0:
        lines = open(path).read().split("\n")
        k = 0
        while k < len(lines) and lines[k].strip():
            fr, k = _header_formatted(lines, k)
            k += 1   # column titles
            n = fr["natm"]
            rows = [lines[k + i].split() for i in range(n)]
            k += n
            fr["atype"] = [r[1] for r in rows]
            fr["efg"] = np.array([[_ffloat(x) for x in r[2:8]] for r in rows])
            frames.append(fr)
        return frames
    recs = list(fortran_records(path))
    k = 0
    while k < len(recs):
        natm = struct.unpack("<i", recs[k])[0]
        ntype = struct.unpack("<i", recs[k + 5])[0]
        t = np.frombuffer(recs[k + 8], dtype="<f8").reshape(3, 3, natm)   # efg_t(ia, i, j) -> [j][i][ia]
        frames.append({"natm": natm, "system": recs[k + 1].decode().strip(),
                       "cell": np.array([struct.unpack("<3d", recs[k + 2 + r]) for r in range(3)]),
                       "ntype": ntype,
                       "labels": [recs[k + 6][3 * i:3 * i + 3].decode().strip() for i in range(ntype)],
                       "natmi": list(struct.unpack(f"<{ntype}i", recs[k + 7])),
                       "efg": np.stack([t[0, 0], t[1, 1], t[2, 2], t[1, 0], t[2, 0], t[2, 1]], axis=1)})
        k += 9
    return frames


def read_vectors(path):
    """Frames of a DIPFF or EFALL: the header fields and the three values per
    site ([natm][3])."""
    frames = []
    lines = open(path).read().split("\n")
    k = 0
    while k < len(lines) and lines[k].strip():
        fr, k = _header_formatted(lines, k)
        k += 1
        n = fr["natm"]
        rows = [lines[k + i].split() for i in range(n)]
        k += n
        fr["atype"] = [r[1] for r in rows]
        fr["values"] = np.array([[_ffloat(x) for x in r[2:5]] for r in rows])
        frames.append(fr)
    return frames
