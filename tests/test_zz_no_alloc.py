"""mdff_rec_energy_noalloc (reciprocal energy with a fixed device scratch,
no allocation) against the engine's own reciprocal energy, mdff_engforce's
u_rec, on the same charges-only system; two calls in a row."""
import ctypes as C

import numpy as np
import pytest

import mdff_b200
from mdff_b200 import abi, systems

pytestmark = pytest.mark.gpu


def _noalloc():
    L = mdff_b200.lib()
    f = L.mdff_rec_energy_noalloc
    dp = C.POINTER(C.c_double)
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, dp, C.c_double,
                  C.POINTER(C.c_int), C.c_void_p, dp, C.POINTER(C.c_longlong)]
    f.restype = C.c_int
    return f


def test_noalloc_rec_energy_matches_engine():
    import torch
    s = systems.silica_bmh()
    p = s["params"]
    p.device = 0
    eng = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    u_engine = eng.engforce()["e"]["u_rec"]
    pos = eng.positions()
    dev = torch.device("cuda", 0)
    r = [torch.tensor(np.ascontiguousarray(pos[:, k]), dtype=torch.float64, device=dev) for k in range(3)]
    q = torch.tensor([p.qch[t - 1] for t in s["itype"]], dtype=torch.float64, device=dev)
    A = np.ascontiguousarray(np.asarray(s["cell"], dtype=np.float64).T.reshape(9))
    kmax = (C.c_int * 3)(*p.kES)
    f = _noalloc()
    torch.cuda.synchronize(dev)
    vals = []
    for _ in range(2):
        u = C.c_double()
        need = C.c_longlong()
        rc = f(0, len(s["itype"]), r[0].data_ptr(), r[1].data_ptr(), r[2].data_ptr(), q.data_ptr(),
               A.ctypes.data_as(C.POINTER(C.c_double)), p.alphaES, kmax, None, C.byref(u), C.byref(need))
        assert rc == abi.OK, rc
        assert 0 < need.value <= 1 << 21
        vals.append(u.value)
    assert vals[0] == vals[1]
    assert abs(vals[0] - u_engine) <= 1e-12 * abs(u_engine), (vals[0], u_engine)


def test_noalloc_rejects_oversize_problem():
    import torch
    n = 300000
    dev = torch.device("cuda", 0)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    A = np.ascontiguousarray((np.eye(3) * 200.0).T.reshape(9))
    kmax = (C.c_int * 3)(40, 40, 40)
    u = C.c_double()
    need = C.c_longlong()
    rc = _noalloc()(0, n, x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(),
                    A.ctypes.data_as(C.POINTER(C.c_double)), 0.3, kmax, None, C.byref(u), C.byref(need))
    assert rc == abi.E_NOMEM
    assert need.value > 1 << 21
