"""B200 force engine for MDFF's force-and-integration hot path.

Python binding of the C ABI in include/mdff_engine.h.  The compute runs in the
CUDA library mdff_b200/lib/libmdff_engine.so (sm_100a); there is no CPU
fallback: importing works without a GPU, but creating an Engine without the
library or without a CUDA device raises.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libmdff_engine.so")
_lib = None


class EngineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mdff engine error {code}: {msg}")
        self.code = code


def build(force=False):
    """Compile the CUDA engine library in place (nvcc, sm_100a)."""
    args = ["make", "-s", "-C", os.path.join(_HERE, "csrc")]
    if force:
        subprocess.run(args + ["clean"], check=True)
    subprocess.run(args, check=True)


def lib():
    """Load the engine library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EngineError(abi.E_STATE, f"engine library missing: {LIB_PATH} (run mdff_b200.build())")
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        vp = C.c_void_p
        L.mdff_params_default.argtypes = [C.POINTER(abi.Params)]
        L.mdff_params_default.restype = None
        L.mdff_create.argtypes = [C.POINTER(abi.Params), C.POINTER(vp)]
        L.mdff_destroy.argtypes = [vp]
        L.mdff_destroy.restype = None
        L.mdff_last_error.argtypes = [vp]
        L.mdff_last_error.restype = C.c_char_p
        L.mdff_set_system.argtypes = [vp, C.c_int, ip, dp, dp, dp, dp]
        L.mdff_set_positions.argtypes = [vp, dp, dp, dp]
        L.mdff_set_cell.argtypes = [vp, dp]
        L.mdff_gr.argtypes = [vp, C.c_double, C.c_double, dp, ip]
        L.mdff_rmc.argtypes = [vp, C.POINTER(abi.RmcParams), dp, dp, C.c_longlong, C.c_ulonglong, dp,
                               C.POINTER(abi.RmcResult)]
        L.mdff_rmc_efg.argtypes = [vp, C.POINTER(abi.RmcParams), C.POINTER(abi.RmcEfgParams), dp, dp, dp, dp, dp,
                                   C.c_longlong, C.c_ulonglong, dp, dp, dp, dp, C.POINTER(abi.RmcResult)]
        L.mdff_get_positions.argtypes = [vp, dp, dp, dp]
        L.mdff_engforce.argtypes = [vp, dp, dp, dp, C.POINTER(abi.Energies), dp, dp, dp, dp, dp]
        L.mdff_nlist_build.argtypes = [vp]
        L.mdff_nlist_get.argtypes = [vp, C.c_int, ip, ip, C.c_int, ip]
        L.mdff_md_start.argtypes = [vp, dp, dp, dp, C.POINTER(abi.Thermo)]
        L.mdff_step.argtypes = [vp, C.c_int, dp, dp, dp, dp, dp, dp, dp, dp, dp, C.POINTER(abi.Thermo)]
        L.mdff_get_velocities.argtypes = [vp, dp, dp, dp]
        L.mdff_stream.argtypes = [vp, C.POINTER(vp)]
        L.mdff_profile.argtypes = [vp, C.c_int]
        L.mdff_profile_get.argtypes = [vp, dp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.c_int]
        L.mdff_measure_pipes.argtypes = [C.c_int, dp]
        L.mdff_measure_tensor.argtypes = [C.c_int, dp]
        L.mdff_opt_sastry.argtypes = [vp, C.c_int, C.POINTER(abi.OptResult)]
        L.mdff_opt_lbfgs.argtypes = [vp, C.c_int, C.c_double, C.POINTER(abi.OptResult)]
        L.mdff_opt_m1qn3.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.POINTER(abi.OptResult)]
        L.mdff_profile_detail.argtypes = [vp, dp, C.POINTER(C.c_longlong), dp]
        L.mdff_io_format.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(abi.FrameHeader), ip, dp, C.c_char_p,
                                     C.c_size_t, C.POINTER(C.c_size_t)]
        L.mdff_writer_open.argtypes = [vp, C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(abi.FrameHeader),
                                       C.c_int, C.POINTER(vp)]
        L.mdff_writer_frame.argtypes = [vp]
        L.mdff_writer_close.argtypes = [vp]
        L.mdff_checkpoint_save.argtypes = [vp, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]
        L.mdff_checkpoint_load.argtypes = [vp, C.c_void_p, C.c_size_t]
        L.mdff_efg_nmr.argtypes = [vp, C.c_int, dp, dp, dp, dp]
        L.mdff_efg_dist.argtypes = [vp, C.c_int, dp, C.POINTER(abi.EfgDistParams), dp, dp, dp, ip, ip, ip, ip]
        L.mdff_struct_size.argtypes = [C.c_int]
        L.mdff_kspace_info.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.mdff_graph_info.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.mdff_kspace_mode.argtypes = [vp, C.POINTER(C.c_int)]
        L.mdff_erfc_check.argtypes = [C.c_int, C.c_int, dp, dp, dp]
        L.mdff_launch_shape.argtypes = [vp, C.POINTER(C.c_int)]
        L.mdff_batch_create.argtypes = [C.POINTER(abi.Params), C.c_int, ip, ip, dp, dp, dp, dp, dp, dp, ip, C.POINTER(vp)]
        L.mdff_batch_destroy.argtypes = [vp]
        L.mdff_batch_destroy.restype = None
        L.mdff_batch_last_error.argtypes = [vp]
        L.mdff_batch_last_error.restype = C.c_char_p
        L.mdff_batch_stream.argtypes = [vp, C.POINTER(vp)]
        L.mdff_batch_set_params.argtypes = [vp, C.POINTER(abi.Params)]
        L.mdff_batch_forces.argtypes = [vp, dp, dp, dp, dp, dp, ip]
        L.mdff_batch_set_targets.argtypes = [vp, dp, dp, dp, dp, C.c_double, C.c_double]
        L.mdff_batch_loss_grad.argtypes = [vp, dp, C.POINTER(abi.ParamGrad), ip]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int)) if a is not None else None


PROFILE_GROUPS = ("nlist", "pair", "dir", "sfac", "kfield", "solver", "integrate", "other")


def measure_tensor(device=0):
    """Measured tcgen05 kind::i8 throughput (TOPS, dense): (N=256 peak, N=96, N=64)."""
    out = np.zeros(3)
    rc = lib().mdff_measure_tensor(int(device), _dp(out))
    if rc != 0:
        raise EngineError(rc, "mdff_measure_tensor failed")
    return tuple(float(x) for x in out)


def measure_pipes(device=0):
    """Measured FMA throughput (TFLOP/s): (fp64, fp32, fp32x2)."""
    out = np.zeros(3)
    rc = lib().mdff_measure_pipes(int(device), _dp(out))
    if rc != 0:
        raise EngineError(rc, "mdff_measure_pipes failed")
    return tuple(float(x) for x in out)


def erfc_check(x, device=0):
    """The real-space kernels' erfc and CUDA's erfc at the points x, both
    evaluated on the device (mdff_erfc_check): (erfc_ex2, erfc)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    a, b = np.empty_like(x), np.empty_like(x)
    rc = lib().mdff_erfc_check(int(device), len(x), _dp(x), _dp(a), _dp(b))
    if rc != 0:
        raise EngineError(rc, "mdff_erfc_check failed")
    return a, b


def params_default():
    p = abi.Params()
    lib().mdff_params_default(C.byref(p))
    return p


class Engine:
    """One engine context on one GPU: the state engforce_driver and md_run
    share through module globals in the reference."""

    def __init__(self, params, itype, pos, cell):
        L = lib()
        self._h = C.c_void_p()
        self.params = params
        rc = L.mdff_create(C.byref(params), C.byref(self._h))
        self._check(rc)
        self.n = len(itype)
        self.itype = np.ascontiguousarray(itype, dtype=np.int32)
        pos = np.asarray(pos, dtype=np.float64)
        r = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
        A = np.ascontiguousarray(np.asarray(cell, dtype=np.float64).T.reshape(9))   # rows = vectors -> column-major
        self._check(L.mdff_set_system(self._h, self.n, _ip(self.itype), *(_dp(a) for a in r), _dp(A)))

    def _check(self, rc):
        if rc != 0:
            msg = lib().mdff_last_error(self._h).decode() if self._h else "no context"
            raise EngineError(rc, msg)

    def kspace_info(self):
        """k-vector counts: rectangle, reference half space, the path's main
        set (mixed: the FP32 / tensor-core set; FP64: the half space or its
        part inside the fp64_keps sphere), mixed FP64 low set."""
        out = (C.c_longlong * 4)()
        self._check(lib().mdff_kspace_info(self._h, out))
        return {"rect": out[0], "half": out[1], "main": out[2], "low": out[3]}

    def kspace_mode(self):
        """Which reciprocal kernels the mixed path uses: the main set and the
        low-|k| set on the tensor cores (mdff_kspace_mode)."""
        out = (C.c_int * 2)()
        self._check(lib().mdff_kspace_mode(self._h, out))
        return {"main_tc": bool(out[0]), "low_tc": bool(out[1])}

    def graph_info(self):
        """How the MD steps ran: replayed from a CUDA graph, captures made,
        plain launches (mdff_graph_info)."""
        out = (C.c_longlong * 3)()
        self._check(lib().mdff_graph_info(self._h, out))
        return {"graph_steps": out[0], "captures": out[1], "plain_steps": out[2]}

    def launch_shape(self):
        """Launch shape in use: real-space lanes per atom (FP64, FP32) and the
        FP32 structure-factor / field splits (in halves of the default)."""
        out = (C.c_int * 4)()
        self._check(lib().mdff_launch_shape(self._h, out))
        return {"g_dir": out[0], "g_dd32": out[1], "sfac_split_x2": out[2], "field_split_x2": out[3]}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().mdff_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def positions(self):
        r = [np.empty(self.n) for _ in range(3)]
        self._check(lib().mdff_get_positions(self._h, *(_dp(a) for a in r)))
        return np.stack(r, axis=1)

    def gr(self, cut, res):
        """g(r) of the current positions as rmc_gr forms it: [npairs+1][nbins]
        (row 0 all pairs, then type pairs it1 <= it2)."""
        nb = C.c_int()
        self._check(lib().mdff_gr(self._h, float(cut), float(res), None, C.byref(nb)))
        npairs = self.params.ntype * (self.params.ntype + 1) // 2
        g = np.empty((npairs + 1, nb.value))
        self._check(lib().mdff_gr(self._h, float(cut), float(res), _dp(g), C.byref(nb)))
        return g

    def rmc(self, rp, gexp, uniforms=None, seed=0):
        """Reverse Monte Carlo on g(r) (mdff_rmc); returns (result, g(r) of the
        final configuration).  The engine's positions become the chain's last."""
        gexp = np.ascontiguousarray(gexp, dtype=np.float64)
        u = None if uniforms is None else np.ascontiguousarray(uniforms, dtype=np.float64)
        g = np.empty_like(gexp)
        r = abi.RmcResult()
        self._check(lib().mdff_rmc(self._h, C.byref(rp), _dp(gexp), _dp(u), 0 if u is None else len(u),
                                   int(seed), _dp(g), C.byref(r)))
        return r.as_dict(), g

    def rmc_efg(self, rp, ep, gexp, dibU_exp=None, dibvzz_exp=None, dibeta_exp=None, uniforms=None, seed=0):
        """Reverse Monte Carlo with rmc_main's EFG chi^2 terms (mdff_rmc_efg);
        returns (result, g(r), U, Vzz, eta distributions of the last accepted
        configuration), the distributions shaped as RmcEfgParams.shapes."""
        su, sv, se = ep.shapes(self.params.ntype)
        gexp = np.ascontiguousarray(gexp, dtype=np.float64)
        ex = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
              for a in (dibU_exp, dibvzz_exp, dibeta_exp)]
        for a, shp in zip(ex, (su, sv, se)):
            if a is not None and a.shape != shp:
                raise ValueError(f"distribution shape {a.shape}, expected {shp}")
        u = None if uniforms is None else np.ascontiguousarray(uniforms, dtype=np.float64)
        g = np.empty_like(gexp)
        U, V, E = np.empty(su), np.empty(sv), np.empty(se)
        r = abi.RmcResult()
        self._check(lib().mdff_rmc_efg(self._h, C.byref(rp), C.byref(ep), _dp(gexp), *(_dp(a) for a in ex), _dp(u),
                                       0 if u is None else len(u), int(seed), _dp(g), _dp(U), _dp(V), _dp(E),
                                       C.byref(r)))
        return r.as_dict(), g, U, V, E

    def set_cell(self, cell):
        """A new cell (rows = lattice vectors) for the same atoms (mdff_set_cell)."""
        A = np.ascontiguousarray(np.asarray(cell, dtype=np.float64).T.reshape(9))
        self._check(lib().mdff_set_cell(self._h, _dp(A)))

    def set_positions(self, pos):
        pos = np.asarray(pos, dtype=np.float64)
        r = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
        self._check(lib().mdff_set_positions(self._h, *(_dp(a) for a in r)))

    def velocities(self):
        v = [np.empty(self.n) for _ in range(3)]
        self._check(lib().mdff_get_velocities(self._h, *(_dp(a) for a in v)))
        return np.stack(v, axis=1)

    state_velocities = velocities

    def stream(self):
        """The engine's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        ptr = C.c_void_p()
        self._check(lib().mdff_stream(self._h, C.byref(ptr)))
        return ptr.value or 0

    def enable_profile(self, on=True):
        self._check(lib().mdff_profile(self._h, int(bool(on))))

    def profile(self, reset=False):
        ms = np.zeros(8)
        cnt = (C.c_longlong * 8)()
        tot = C.c_longlong()
        self._check(lib().mdff_profile_get(self._h, _dp(ms), cnt, C.byref(tot), int(bool(reset))))
        out = {k: {"ms": float(ms[i]), "count": int(cnt[i])} for i, k in enumerate(PROFILE_GROUPS)}
        out["_launches"] = {"ms": 0.0, "count": int(tot.value)}
        return out

    def profile_reset(self):
        self.profile(reset=True)

    def opt_sastry(self, itmax=10000):
        """Structure optimisation from the current positions (conjugate
        gradients with cubic line minimisation, the reference's sastry);
        the engine's positions are left at the minimum."""
        r = abi.OptResult()
        self._check(lib().mdff_opt_sastry(self._h, int(itmax), C.byref(r)))
        return r.as_dict()

    def opt_lbfgs(self, itmax=10000, eps=abi.EPSREL_OPT):
        """Structure optimisation from the current positions by limited-memory
        BFGS (the reference's lbfgs_driver; eps is epsrel_lbfgs, itmax bounds
        the force evaluations); the engine's positions are left at the last
        evaluated point."""
        r = abi.OptResult()
        self._check(lib().mdff_opt_lbfgs(self._h, int(itmax), float(eps), C.byref(r)))
        return r.as_dict()

    def opt_m1qn3(self, niter=6000, nsim=6000, epsg=abi.EPSREL_OPT):
        """Structure optimisation from the current positions by M1QN3 in
        diagonal-initial-scaling mode (the reference's m1qn3_driver); the
        positions are left at the returned point, evaluated there."""
        r = abi.OptResult()
        self._check(lib().mdff_opt_m1qn3(self._h, int(niter), int(nsim), float(epsg), C.byref(r)))
        return r.as_dict()

    def _efg_input(self, efg):
        """[nconf][6][natm] contiguous from [natm][6] or [nconf][natm][6]; None stays None."""
        if efg is None:
            return None, 1
        e = np.asarray(efg, dtype=np.float64)
        if e.ndim == 2:
            e = e[None]
        return np.ascontiguousarray(e.transpose(0, 2, 1)), e.shape[0]

    def efg_nmr(self, efg=None):
        """Per-site EFG analysis (efg_stat, src/efg.f90:2225-2270).  efg:
        [natm][6] or [nconf][natm][6] (xx yy zz xy xz yz), or None for the
        tensors of the last engforce (doefg).  Returns nmr [..][natm][4]
        (Vxx, Vyy, Vzz, eta in the NMR convention), U [..][natm][5] (Czjzek
        components) and S [..][natm], with the configuration axis only when
        efg has one."""
        n = self.n
        e6, nc = self._efg_input(efg)
        nmr, U, S = np.empty(4 * n * nc), np.empty(5 * n * nc), np.empty(n * nc)
        self._check(lib().mdff_efg_nmr(self._h, nc, _dp(e6), _dp(nmr), _dp(U), _dp(S)))
        nmr = nmr.reshape(nc, 4, n).transpose(0, 2, 1).copy()
        U = U.reshape(nc, 5, n).transpose(0, 2, 1).copy()
        S = S.reshape(nc, n)
        if efg is None or np.ndim(efg) == 2:
            return nmr[0], U[0], S[0]
        return nmr, U, S

    def efg_dist(self, dist, efg=None):
        """efg_stat's statistics and distributions (src/efg.f90:2272-2440)
        over one configuration ([natm][6]) or several ([nconf][natm][6]); None
        for the context's own EFG.  dist: abi.EfgDistParams.  Rows 0 (all
        sites), 1..ntype.  Returns a dict with stats [nconf][ntype+1][8]
        (vzzmin, vzzmax, <Vzz>, <|Vzz|>, <eta>, P(Vzz>=0), rho_z, sigma per
        configuration, as the reference's loop forms them), mU [ntype+1][5],
        m2U [ntype+1][5][5] and the integer histograms summed over the
        configurations: vzz, eta, u [6][ntype+1][PANU+1], s."""
        nt1 = self.params.ntype + 1
        PV, PE, PU, PS = dist.bins()
        e6, nc = self._efg_input(efg)
        stats, mU, m2U = np.empty((nc, nt1, 8)), np.empty((nt1, 5)), np.empty((nt1, 5, 5))
        hv = np.empty((nt1, PV + 1), dtype=np.int32)
        he = np.empty((nt1, PE + 1), dtype=np.int32)
        hu = np.empty((6, nt1, PU + 1), dtype=np.int32)
        hs = np.empty((nt1, PS + 1), dtype=np.int32)
        self._check(lib().mdff_efg_dist(self._h, nc, _dp(e6), C.byref(dist), _dp(stats), _dp(mU), _dp(m2U),
                                        _ip(hv), _ip(he), _ip(hu), _ip(hs)))
        return {"stats": stats, "mU": mU, "m2U": m2U, "vzz": hv, "eta": he, "u": hu, "s": hs}

    def efgcalc(self, frames, dist=None, efgall=None, iformat=1, system="", labels=()):
        """calc = 'efg' (efgcalc, src/efg.f90:325-660): for each configuration
        of a TRAJFF -- frames from io.read_trajff, or a path to read -- the
        Ewald EFG of the engine's system at those positions (with induced
        dipoles where the system is polarisable, as get_moments gives them),
        written to an EFGALL when efgall names one (write_EFGALL's layout,
        iformat 1 formatted / 0 unformatted), then efg_stat over all of them
        when dist (abi.EfgDistParams) is given.  Returns (efg [nconf][natm][6]
        with coul_unit, efg_dist's result or None).  The engine needs
        doefg = 1."""
        from . import io as _io
        if isinstance(frames, (str, os.PathLike)):
            frames = _io.read_trajff(frames)
        out = np.empty((len(frames), self.n, 6))
        w = open(efgall, "wb") if efgall else None
        try:
            for k, fr in enumerate(frames):
                if fr["natm"] != self.n:
                    raise ValueError(f"configuration {k}: {fr['natm']} atoms, the engine has {self.n}")
                self.set_cell(np.asarray(fr["cell"], dtype=np.float64))
                self.set_positions(fr["r"])
                out[k] = self.engforce()["efg"]
                if w is not None:
                    h = _io.header(system or fr.get("system", ""), labels or fr.get("labels", ()),
                                   natmi=fr.get("natmi", ()), cell=fr["cell"], natm=self.n)
                    w.write(_io.format_frame("EFGALL", iformat, 0, h, self.itype, out[k].T))
        finally:
            if w is not None:
                w.close()
        return out, (self.efg_dist(dist, out) if dist is not None else None)

    def checkpoint(self):
        """The whole time-integration state as bytes (mdff_checkpoint_save)."""
        n = C.c_size_t()
        self._check(lib().mdff_checkpoint_save(self._h, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        self._check(lib().mdff_checkpoint_save(self._h, buf, n.value, C.byref(n)))
        return buf.raw[:n.value]

    def restore(self, data):
        """Continue from a checkpoint of an engine with the same parameters
        and system (mdff_checkpoint_load), in place of md_start."""
        buf = C.create_string_buffer(bytes(data), len(data))
        self._check(lib().mdff_checkpoint_load(self._h, buf, len(data)))

    def writer(self, path, kind, iformat=1, data="rvf", system="", labels=(), nslot=4):
        """A streaming writer of this engine's frames (mdff_writer_open)."""
        from .io import Writer
        return Writer(self, path, kind, iformat, data, system, labels, nslot)

    def efg_dist_ptr(self, dist, ptr, nconf):
        """efg_dist over tensors at a raw address of [nconf][6][natm] float64:
        this GPU's memory (read in place, e.g. a torch CUDA tensor's
        data_ptr()) or host memory (uploaded; pinned memory copies fastest)."""
        nt1 = self.params.ntype + 1
        PV, PE, PU, PS = dist.bins()
        stats, mU, m2U = np.empty((nconf, nt1, 8)), np.empty((nt1, 5)), np.empty((nt1, 5, 5))
        hv = np.empty((nt1, PV + 1), dtype=np.int32)
        he = np.empty((nt1, PE + 1), dtype=np.int32)
        hu = np.empty((6, nt1, PU + 1), dtype=np.int32)
        hs = np.empty((nt1, PS + 1), dtype=np.int32)
        self._check(lib().mdff_efg_dist(self._h, int(nconf), C.cast(C.c_void_p(ptr), C.POINTER(C.c_double)),
                                        C.byref(dist), _dp(stats), _dp(mU), _dp(m2U), _ip(hv), _ip(he), _ip(hu),
                                        _ip(hs)))
        return {"stats": stats, "mU": mU, "m2U": m2U, "vzz": hv, "eta": he, "u": hu, "s": hs}

    def profile_detail(self):
        """Single-kernel detail timers: the tensor-core k-space kernels (mixed
        path; ops = int8 digit-product operations) and the EFG site kernel
        (ops = bytes it reads): accumulated ms, launches and work."""
        ms, ops = np.zeros(5), np.zeros(5)
        cnt = (C.c_longlong * 5)()
        self._check(lib().mdff_profile_detail(self._h, _dp(ms), cnt, _dp(ops)))
        return {k: {"ms": float(ms[i]), "count": int(cnt[i]), "ops": float(ops[i])}
                for i, k in enumerate(("sfac_tc", "kfield_tc", "efg_sites", "sfac_tc4", "kfield_tc4"))}

    def nlist_build(self):
        self._check(lib().mdff_nlist_build(self._h))

    def nlist(self, which):
        point = np.empty(self.n + 1, dtype=np.int32)
        cnt = C.c_int()
        rc = lib().mdff_nlist_get(self._h, which, _ip(point), None, 0, C.byref(cnt))
        if rc not in (0, abi.E_LISTOVF):
            self._check(rc)
        lst = np.empty(max(cnt.value, 1), dtype=np.int32)
        self._check(lib().mdff_nlist_get(self._h, which, _ip(point), _ip(lst), cnt.value, C.byref(cnt)))
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
        self._check(lib().mdff_engforce(self._h, *(_dp(a) for a in f), C.byref(e), _dp(tn), _dp(tc), _dp(ef),
                                        _dp(efg), _dp(mu)))
        return {
            "f": np.stack(f, axis=1),
            "e": e.as_dict(),
            "tau_nonb": tn.reshape(3, 3).T.copy(),
            "tau_coul": tc.reshape(3, 3).T.copy(),
            "ef": ef.reshape(3, n).T.copy(),
            "efg": efg.reshape(6, n).T.copy(),
            "mu": mu.reshape(3, n).T.copy(),
        }

    def md_start(self, vel):
        vel = np.asarray(vel, dtype=np.float64)
        v = [np.ascontiguousarray(vel[:, k]) for k in range(3)]
        t0 = abi.Thermo()
        self._check(lib().mdff_md_start(self._h, *(_dp(a) for a in v), C.byref(t0)))
        return t0.as_dict()

    def step(self, nsteps, thermo=True):
        """Advance nsteps; return final positions, velocities, forces and the
        per-step thermodynamics."""
        n = self.n
        r = [np.empty(n) for _ in range(3)]
        v = [np.empty(n) for _ in range(3)]
        f = [np.empty(n) for _ in range(3)]
        th = (abi.Thermo * max(nsteps, 1))() if thermo else None
        # no upload (NULL position/velocity inputs would skip the download too),
        # so advance first, then read the state back
        self._check(lib().mdff_step(self._h, nsteps, None, None, None, None, None, None, *(_dp(a) for a in f),
                                    th if thermo else None))
        pos = self.positions()
        return {
            "pos": pos,
            "f": np.stack(f, axis=1),
            "thermo": [th[i].as_dict() for i in range(nsteps)] if thermo else [],
        }

    def advance(self, nsteps):
        """Advance nsteps with the state left on the device (nothing read back)."""
        self._check(lib().mdff_step(self._h, int(nsteps), None, None, None, None, None, None, None, None, None,
                                    None))

    def step_host(self, nsteps, pos, vel, thermo=None):
        """The host-buffer form of mdff_step: positions and velocities are
        uploaded from, and written back to, the given (N,3)-shaped SoA arrays."""
        n = self.n
        f = [np.empty(n) for _ in range(3)]
        self._check(lib().mdff_step(self._h, nsteps, *(_dp(pos[k]) for k in range(3)), *(_dp(vel[k]) for k in range(3)),
                                    *(_dp(a) for a in f), thermo))
        return f


class Batch:
    """A batch of fixed configurations sharing one force field: forces and
    stress of all of them, and the force-matching loss with its adjoint
    gradient, each in one set of launches (mdff_batch_* in
    include/mdff_engine.h).

    confs: list of dicts with itype (1-based), pos [n,3], cell [3,3] (rows
    are the basis vectors), rc, alpha, kmax (int or 3 ints)."""

    def __init__(self, params, confs):
        L = lib()
        self.params = params
        self.nconf = len(confs)
        self.natm = np.array([len(c["itype"]) for c in confs], dtype=np.int32)
        self.N = int(self.natm.sum())
        self.offsets = np.concatenate([[0], np.cumsum(self.natm)])
        itype = np.ascontiguousarray(np.concatenate([c["itype"] for c in confs]), dtype=np.int32)
        pos = np.concatenate([np.asarray(c["pos"], dtype=np.float64) for c in confs])
        r = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
        cells = np.ascontiguousarray(np.concatenate(
            [np.asarray(c["cell"], dtype=np.float64).T.reshape(9) for c in confs]))
        rc = np.ascontiguousarray([float(c["rc"]) for c in confs])
        alpha = np.ascontiguousarray([float(c["alpha"]) for c in confs])
        km = np.ascontiguousarray(np.concatenate(
            [np.broadcast_to(np.asarray(c["kmax"], dtype=np.int32), (3,)) for c in confs]), dtype=np.int32)
        self._h = C.c_void_p()
        rc_ = L.mdff_batch_create(C.byref(params), self.nconf, _ip(self.natm), _ip(itype), *(_dp(a) for a in r),
                                  _dp(cells), _dp(rc), _dp(alpha), _ip(km), C.byref(self._h))
        self._check(rc_)

    def _check(self, rc):
        if rc != 0:
            msg = lib().mdff_batch_last_error(self._h).decode() if self._h else "no batch"
            raise EngineError(rc, msg)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().mdff_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stream(self):
        s = C.c_void_p()
        self._check(lib().mdff_batch_stream(self._h, C.byref(s)))
        return s.value or 0

    def set_params(self, params):
        self.params = params
        self._check(lib().mdff_batch_set_params(self._h, C.byref(params)))

    def split(self, a):
        return [a[self.offsets[c]:self.offsets[c + 1]] for c in range(self.nconf)]

    def forces(self):
        """Per configuration: forces [n,3] (eV/A), total stress [3,3] (GPa)
        and potential energy (eV); and the dipole-solve iterations."""
        f = [np.empty(self.N) for _ in range(3)]
        tau = np.empty(9 * self.nconf)
        e = np.empty(self.nconf)
        it = C.c_int()
        self._check(lib().mdff_batch_forces(self._h, *(_dp(a) for a in f), _dp(tau), _dp(e), C.byref(it)))
        F = np.stack(f, axis=1)
        taus = [tau[9 * c:9 * c + 9].reshape(3, 3).T.copy() for c in range(self.nconf)]
        return {"f": self.split(F), "tau": taus, "energy": e, "iters": it.value}

    def set_targets(self, f_target, tau_target, w_force=1.0, w_stress=1.0):
        """Targets of the loss: forces per configuration [n,3] and stresses [3,3]."""
        F = np.concatenate([np.asarray(x, dtype=np.float64) for x in f_target])
        f = [np.ascontiguousarray(F[:, k]) for k in range(3)]
        tau = np.ascontiguousarray(np.concatenate(
            [np.asarray(t, dtype=np.float64).T.reshape(9) for t in tau_target]))
        self._check(lib().mdff_batch_set_targets(self._h, *(_dp(a) for a in f), _dp(tau), float(w_force),
                                                 float(w_stress)))

    def loss_grad(self, want_grad=True):
        """(loss, abi.ParamGrad or None, (forward iterations, adjoint iterations))."""
        loss = C.c_double()
        g = abi.ParamGrad() if want_grad else None
        it = (C.c_int * 2)()
        self._check(lib().mdff_batch_loss_grad(self._h, C.byref(loss), C.byref(g) if g is not None else None, it))
        return loss.value, g, (it[0], it[1])
