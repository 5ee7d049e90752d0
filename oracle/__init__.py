"""CPU FP64 oracle of MDFF's force-and-integration path -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
this module; the engine (mdff_b200) never imports it.  The C++ restatement in
mdff_oracle.cpp follows the reference routine by routine (file:line cited
there); this wrapper only marshals arrays through ctypes.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from mdff_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(abi.Params), C.c_int, ip, dp, dp, dp, dp]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_erfc_mode.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_errfc.restype = C.c_double
        L.orc_errfc.argtypes = [C.c_double]
        L.orc_tt_damp.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, dp, dp]
        L.orc_lattice.argtypes = [dp, dp, dp, dp, dp]
        L.orc_ewald_info.argtypes = [C.c_void_p, dp, ip, ip, dp]
        L.orc_set_positions.argtypes = [C.c_void_p, dp, dp, dp]
        L.orc_get_positions.argtypes = [C.c_void_p, dp, dp, dp]
        L.orc_nlist_build.argtypes = [C.c_void_p]
        L.orc_nlist_get.argtypes = [C.c_void_p, C.c_int, ip, ip, C.c_int, ip]
        L.orc_engforce.argtypes = [C.c_void_p, dp, dp, dp, C.POINTER(abi.Energies), dp, dp, dp, dp, dp]
        L.orc_coulomb_field.argtypes = [C.c_void_p, dp, dp, C.c_int, dp, dp, dp]
        L.orc_field_time.argtypes = [C.c_void_p, C.c_int, dp, dp, dp]
        L.orc_max_threads.restype = C.c_int
        L.orc_md_start.argtypes = [C.c_void_p, dp, dp, dp, C.POINTER(abi.Thermo)]
        L.orc_loss_grad.argtypes = [C.c_void_p, dp, dp, dp, dp, C.c_double, C.c_double, dp,
                                    C.POINTER(abi.ParamGrad), ip]
        L.orc_step.argtypes = [C.c_void_p, C.c_int, dp, dp, dp, dp, dp, dp, dp, dp, dp, C.POINTER(abi.Thermo)]
        L.orc_opt_sastry.argtypes = [C.c_void_p, C.c_int, C.POINTER(abi.OptResult)]
        L.orc_opt_lbfgs.argtypes = [C.c_void_p, C.c_int, C.c_double, C.POINTER(abi.OptResult)]
        L.orc_opt_m1qn3.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.POINTER(abi.OptResult)]
        L.orc_gr.argtypes = [C.c_void_p, C.c_double, C.c_double, dp, C.POINTER(C.c_int)]
        L.orc_rmc.argtypes = [C.c_void_p, C.POINTER(abi.RmcParams), dp, dp, C.c_longlong, dp,
                              C.POINTER(abi.RmcResult)]
        L.orc_rmc_efg.argtypes = [C.c_void_p, C.POINTER(abi.RmcParams), C.POINTER(abi.RmcEfgParams), dp, dp, dp, dp,
                                  dp, C.c_longlong, dp, dp, dp, dp, C.POINTER(abi.RmcResult)]
        L.orc_efg_rmc.argtypes = [C.c_void_p, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int)) if a is not None else None


def max_threads():
    return lib().orc_max_threads()


def set_threads(n):
    lib().orc_set_threads(int(n))


def errfc(x):
    return lib().orc_errfc(float(x))


def tt_damp(b, c, r, order):
    f = C.c_double()
    fd = C.c_double()
    lib().orc_tt_damp(b, c, r, order, C.byref(f), C.byref(fd))
    return f.value, fd.value


class Oracle:
    """Same call shape as mdff_b200.Engine, computed on the CPU in FP64."""

    def __init__(self, params, itype, pos, cell, erfc_mode=1):
        self.n = len(itype)
        self.itype = np.ascontiguousarray(itype, dtype=np.int32)
        pos = np.asarray(pos, dtype=np.float64)
        rx, ry, rz = (np.ascontiguousarray(pos[:, k]) for k in range(3))
        A = np.ascontiguousarray(np.asarray(cell, dtype=np.float64).T.reshape(9))  # column-major
        self._p = params
        self._h = lib().orc_create(C.byref(params), self.n, _ip(self.itype), _dp(rx), _dp(ry), _dp(rz), _dp(A))
        lib().orc_set_erfc_mode(self._h, erfc_mode)

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def ewald_info(self):
        a = C.c_double()
        km = (C.c_int * 3)()
        nk = C.c_int()
        cl = C.c_double()
        lib().orc_ewald_info(self._h, C.byref(a), km, C.byref(nk), C.byref(cl))
        return {"alpha": a.value, "kmax": tuple(km), "nk": nk.value, "cutlongrange": cl.value}

    def positions(self):
        r = [np.empty(self.n) for _ in range(3)]
        lib().orc_get_positions(self._h, *(_dp(a) for a in r))
        return np.stack(r, axis=1)

    def set_positions(self, pos):
        pos = np.asarray(pos, dtype=np.float64)
        r = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
        lib().orc_set_positions(self._h, *(_dp(a) for a in r))

    def nlist_build(self):
        lib().orc_nlist_build(self._h)

    def nlist(self, which):
        point = np.empty(self.n + 1, dtype=np.int32)
        cnt = C.c_int()
        cap = 0
        rc = lib().orc_nlist_get(self._h, which, _ip(point), None, 0, C.byref(cnt))
        cap = cnt.value
        lst = np.empty(max(cap, 1), dtype=np.int32)
        rc = lib().orc_nlist_get(self._h, which, _ip(point), _ip(lst), cap, C.byref(cnt))
        assert rc == 0, rc
        return point, lst[:cnt.value]

    def engforce(self):
        n = self.n
        f = [np.empty(n) for _ in range(3)]
        e = abi.Energies()
        tn = np.empty(9)
        tc = np.empty(9)
        ef = np.empty(3 * n)
        efg = np.empty(6 * n)
        mu = np.empty(3 * n)
        lib().orc_engforce(self._h, *(_dp(a) for a in f), C.byref(e), _dp(tn), _dp(tc), _dp(ef), _dp(efg), _dp(mu))
        return {
            "f": np.stack(f, axis=1),
            "e": e.as_dict(),
            "tau_nonb": tn.reshape(3, 3).T.copy(),
            "tau_coul": tc.reshape(3, 3).T.copy(),
            "ef": ef.reshape(3, n).T.copy(),
            "efg": efg.reshape(6, n).T.copy(),
            "mu": mu.reshape(3, n).T.copy(),
        }

    def coulomb_field(self, q, mu, damp=False):
        n = self.n
        q = np.ascontiguousarray(q, dtype=np.float64)
        m = np.ascontiguousarray(np.asarray(mu, dtype=np.float64).T.reshape(3 * n))
        ef = np.empty(3 * n)
        efg = np.empty(6 * n)
        u = C.c_double()
        lib().orc_coulomb_field(self._h, _dp(q), _dp(m), int(damp), _dp(ef), _dp(efg), C.byref(u))
        return ef.reshape(3, n).T.copy(), efg.reshape(6, n).T.copy(), u.value

    def field_time(self, kstride=1):
        """Seconds of one Ewald field evaluation (real space, reciprocal space
        over every kstride-th k-vector) and one short-range pair loop."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        lib().orc_field_time(self._h, int(kstride), C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def loss_grad(self, f_target, tau_target, c_force, c_stress, grad=None):
        """Force-matching loss c_force*sum|F-F*|^2 + c_stress*sum(tau-tau*)^2
        of this configuration (a fresh induced-dipole solve) and its gradient
        with respect to the force-field tables, accumulated into grad (an
        abi.ParamGrad, created zeroed when None).  Returns (loss, grad,
        (forward iterations, adjoint iterations))."""
        ft = np.asarray(f_target, dtype=np.float64)
        f = [np.ascontiguousarray(ft[:, k]) for k in range(3)]
        tt = np.ascontiguousarray(np.asarray(tau_target, dtype=np.float64).T.reshape(9))
        if grad is None:
            grad = abi.ParamGrad()
        loss = C.c_double(0.0)
        it = (C.c_int * 2)()
        lib().orc_loss_grad(self._h, *(_dp(a) for a in f), _dp(tt), float(c_force), float(c_stress),
                            C.byref(loss), C.byref(grad), it)
        return loss.value, grad, (it[0], it[1])

    def opt_sastry(self, itmax=10000):
        """Structure optimisation from the current positions (sastry,
        src/opt.f90:452-849); the positions are left at the minimum."""
        r = abi.OptResult()
        lib().orc_opt_sastry(self._h, int(itmax), C.byref(r))
        return r.as_dict()

    def opt_lbfgs(self, itmax=10000, eps=abi.EPSREL_OPT):
        """Structure optimisation by L-BFGS (lbfgs_driver, src/opt.f90:972-1194,
        over LBFGS/MCSRCH/MCSTEP of src/lbfgs.f90)."""
        r = abi.OptResult()
        lib().orc_opt_lbfgs(self._h, int(itmax), float(eps), C.byref(r))
        return r.as_dict()

    def opt_m1qn3(self, niter=6000, nsim=6000, epsg=abi.EPSREL_OPT):
        """Structure optimisation by M1QN3 (m1qn3_driver, src/opt.f90:1203-1330,
        over m1qn3a/dd/mlis3/ecube of src/m1qn3.f90)."""
        r = abi.OptResult()
        lib().orc_opt_m1qn3(self._h, int(niter), int(nsim), float(epsg), C.byref(r))
        return r.as_dict()

    def gr(self, cut, res):
        """g(r) as rmc_gr forms it (gr_main, src/radial_distrib.f90)."""
        nb = C.c_int()
        lib().orc_gr(self._h, float(cut), float(res), None, C.byref(nb))
        npairs = self._p.ntype * (self._p.ntype + 1) // 2
        g = np.empty((npairs + 1, nb.value))
        lib().orc_gr(self._h, float(cut), float(res), _dp(g), C.byref(nb))
        return g

    def rmc(self, rp, gexp, uniforms):
        """rmc_main on the g(r) chi^2 with the given uniforms; returns
        (result, g(r) of the final configuration)."""
        gexp = np.ascontiguousarray(gexp, dtype=np.float64)
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        g = np.empty_like(gexp)
        r = abi.RmcResult()
        lib().orc_rmc(self._h, C.byref(rp), _dp(gexp), _dp(u), len(u), _dp(g), C.byref(r))
        return r.as_dict(), g

    def rmc_efg(self, rp, ep, gexp, dibU_exp=None, dibvzz_exp=None, dibeta_exp=None, uniforms=()):
        """rmc_main with the EFG chi^2 terms (rmc_efg over multipole_efg_ES,
        eval_chisq_Uefg/vzz/eta) on the given uniforms; returns (result, g(r),
        U, Vzz, eta distributions of the last accepted configuration)."""
        su, sv, se = ep.shapes(self._p.ntype)
        gexp = np.ascontiguousarray(gexp, dtype=np.float64)
        ex = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
              for a in (dibU_exp, dibvzz_exp, dibeta_exp)]
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        g = np.empty_like(gexp)
        U, V, E = np.zeros(su), np.zeros(sv), np.zeros(se)
        r = abi.RmcResult()
        lib().orc_rmc_efg(self._h, C.byref(rp), C.byref(ep), _dp(gexp), *(_dp(a) for a in ex), _dp(u), len(u),
                          _dp(g), _dp(U), _dp(V), _dp(E), C.byref(r))
        return r.as_dict(), g, U, V, E

    def efg_rmc(self):
        """multipole_efg_ES of the current positions for point charges, [n][6]
        (xx yy zz xy xz yz) without coul_unit."""
        out = np.empty((6, self.n))
        lib().orc_efg_rmc(self._h, _dp(out))
        return out.T.copy()

    def md_start(self, vel):
        vel = np.asarray(vel, dtype=np.float64)
        v = [np.ascontiguousarray(vel[:, k]) for k in range(3)]
        t0 = abi.Thermo()
        lib().orc_md_start(self._h, *(_dp(a) for a in v), C.byref(t0))
        return t0.as_dict()

    def step(self, nsteps):
        n = self.n
        r = [np.empty(n) for _ in range(3)]
        v = [np.empty(n) for _ in range(3)]
        f = [np.empty(n) for _ in range(3)]
        th = (abi.Thermo * max(nsteps, 1))()
        # positions/velocities are read back only: pass buffers filled from the current state
        pos = self.positions()
        for k in range(3):
            r[k][:] = pos[:, k]
        lib().orc_step(self._h, nsteps, *(_dp(a) for a in r), None, None, None, *(_dp(a) for a in f), th)
        return {
            "pos": np.stack(r, axis=1),
            "f": np.stack(f, axis=1),
            "thermo": [th[i].as_dict() for i in range(nsteps)],
        }
