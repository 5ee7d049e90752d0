#!/usr/bin/env python
"""Benchmark: atom-steps/s of the polarisable-ion Ewald NVT production run.

Workload (one replica per GPU, weak scaling): 32440-ion MgO polarisable-ion
model, 16^3 rock-salt cells with 1 % vacancies, rc 10 A, Ewald alpha 0.3
A^-1, kmax 23 (nk = 51911), induced dipoles by PCG to an RMS residual of
1e-8, Nose-Hoover chain of length 3 at 2000 K, dt 1 fs, EFG every 10 steps
(mdff_b200.systems.mgo_production).  A step is one full MD step: Verlet-list
check, short-range pair loop, dipole solve, Ewald forces / stress / EFG and
the integrator.  Inputs are synthetic (seeded), no dataset is involved.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
  python bench.py --impl reference ...   CPU oracle (C++ port of the reference path)

Prints one JSON line on rank 0.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s PIM-Ewald 32k atoms, mixed vs FP64 GPU at <=1e-6 rel force err"

# DRAM traffic per launch (MB, read + write) of the tensor-core k-space
# kernels on the 32 440-ion production cell, from one ncu capture of each
# (the launch list and sections are summarised under profiles/).
TC_TRAFFIC_MB = {"sfac_tc": 58.0, "kfield_tc": 29.3, "sfac_tc4": 31.5, "kfield_tc4": 17.8}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true",
                    help="skip the FP64 arms and the mixed-vs-FP64 errors of the default (mixed) run")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-stream", action="store_true",
                    help="skip the trajectory-streaming measurement of the production workload")
    ap.add_argument("--ncell", type=int, default=16)
    ap.add_argument("--ext", default="aspc", choices=["aspc", "poly"],
                    help="induced-dipole predictor (algo_ext_dipole)")
    ap.add_argument("--ext-order", type=int, default=5, help="extrapolate_order of the predictor (ASPC 5: 7.5 PCG iterations per step against 7.9 at 3)")
    ap.add_argument("--ksplit", type=float, default=None,
                    help="mixed path: |k| below ksplit*alpha summed in FP64 (default: the library's)")
    ap.add_argument("--keps", type=float, default=None,
                    help="mixed path: leave out k with exp(-k^2/4 alpha^2) below keps (0: all; default: the library's)")
    ap.add_argument("--autotune", type=int, default=1, choices=[0, 1], help="autotune the launch shapes")
    ap.add_argument("--tc", type=int, default=2, choices=[0, 1, 2],
                    help="mixed path: k-space on the tensor cores (1), with the low-|k| set too (2), or the FP32 CUDA-core kernels (0)")
    ap.add_argument("--reuse", default="auto", choices=["auto", "0", "1"],
                    help="kspace_reuse (auto: on for the mixed path, off for the plain FP64 path)")
    ap.add_argument("--opt-iters", type=int, default=10,
                    help="opt workload: iterations (sastry), 5x as many force evaluations (lbfgs) or iterations (m1qn3)")
    ap.add_argument("--rmc-var-moves", type=int, default=50,
                    help="rmc workload: trial moves with the distance-variance term (0: skip)")
    ap.add_argument("--rmc-efg-moves", type=int, default=100,
                    help="rmc workload: trial moves of the chain with the EFG chi^2 terms (0: skip)")
    ap.add_argument("--optalgo", default="sastry", choices=["sastry", "lbfgs", "m1qn3"],
                    help="opt workload: minimiser (the reference's optalgo)")
    ap.add_argument("--workload", default="production", choices=["production", "batch", "opt", "efg", "rmc"],
                    help="production: the 32 440-ion PIM NVT cell (the headline metric); batch: the 64-configuration "
                         "force-matching loss and adjoint gradient; opt: conjugate-gradient structure optimisation; "
                         "efg: EFG statistics and distributions over many configurations")
    ap.add_argument("--efg-conf", type=int, default=128, help="efg workload: configurations per step")
    ap.add_argument("--rmc-moves", type=int, default=20000, help="rmc workload: trial moves per step")
    ap.add_argument("--ensemble", default="nvt", choices=["nvt", "npt"],
                    help="production workload: Nose-Hoover chains at constant volume (the headline) or the "
                         "isotropic barostat at 0 GPa (timesca_baro 0.5 ps)")
    ap.add_argument("--accuracy", action="store_true",
                    help="error of the mixed path against the FP64 path on snapshots of an FP64 trajectory")
    ap.add_argument("--snapshots", type=int, default=3)
    ap.add_argument("--snap-every", type=int, default=100)
    return ap.parse_args()


class ClockSampler:
    """SM clock and throttle reasons sampled by one streaming nvidia-smi
    process (every 50 ms) while the timed region runs."""

    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._proc = None
        self._th = None

    def _reader(self):
        for line in self._proc.stdout:
            f = [x.strip() for x in line.strip().split(",")]
            if len(f) >= 7:
                self.samples.append(f)

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                           "--format=csv,noheader,nounits", "-lms", "50"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._th = threading.Thread(target=self._reader, daemon=True)
            self._th.start()
            time.sleep(0.3)   # first sample lands before the timed region starts
        except OSError:
            self._proc = None
        return self

    def __exit__(self, *a):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
            self._th.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        num = lambda x: x.replace(".", "", 1).isdigit()
        sm = [float(s[0]) for s in self.samples if num(s[0])]
        mx = [float(s[1]) for s in self.samples if num(s[1])]
        reasons = sorted({self.NAMES[k] for s in self.samples for k in range(4) if s[3 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup(n_gpus, backend="nccl"):
    """One process per GPU under torchrun: the process group is used only for
    the barrier around the timed region and the max/sum over ranks (each rank
    runs an independent replica; there is no data-path collective)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local, dist


def _reduce(v, dist, device, op):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(v, dist, device):
    return _reduce(v, dist, device, dist.ReduceOp.MAX if dist is not None else None)


def whole_job_rate(units, seconds, dist, device):
    """Whole-job throughput: the units all ranks processed divided by the
    slowest rank's time."""
    if dist is None:
        return units / seconds
    return _reduce(units, dist, device, dist.ReduceOp.SUM) / max_over_ranks(seconds, dist, device)


def barrier(dist, device):
    if dist is not None:
        if device.type == "cuda":
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


def copy_params(p):
    from mdff_b200 import abi
    q = abi.Params()
    C.pointer(q)[0] = p
    return q


def timed_md(eng, vel, steps, warmup, device, dist):
    """md_start, W untimed steps, then K timed MD steps between CUDA events on
    the engine's own stream (barrier + synchronize on both sides).  Returns the
    device milliseconds of the K steps and their thermodynamics."""
    import torch
    ext = torch.cuda.ExternalStream(eng.stream(), device=device)
    eng.md_start(vel)
    if warmup:
        eng.step(warmup, thermo=False)
    barrier(dist, device)
    torch.cuda.synchronize(device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(ext)
    out = eng.step(steps, thermo=True)
    ev1.record(ext)
    ev1.synchronize()
    torch.cuda.synchronize(device)
    return ev0.elapsed_time(ev1), out


def fp64_arms(s, pm, args, device, dist):
    """The plain FP64 GPU path on the same cell, steps and warm-up as the mixed
    arm, twice: (a) the reference's whole half space of k-vectors and its
    sequence of reciprocal evaluations (kspace_reuse off), and (b) the same
    k sphere (fp64_keps = mixed_keps) and structure-factor reuse as the mixed
    arm, so that the ratio (b) isolates precision.  Then, at the positions the
    FP64 trajectory (a) reached, one force evaluation of each path: the errors
    of the mixed path (and of the FP64 sphere) against plain FP64 as global
    relative norms ||x - x_fp64|| / ||x_fp64||."""
    import mdff_b200
    from mdff_b200 import abi
    natm = len(s["itype"])
    arms, last = {}, None
    cases = (("fp64", 0.0, 0), ("fp64_sphere_reuse", pm.mixed_keps, 1))
    for name, keps, reuse in cases:
        pf = copy_params(pm)
        pf.precision = abi.PREC_FP64
        pf.fp64_keps = keps
        pf.kspace_reuse = reuse
        e = mdff_b200.Engine(pf, s["itype"], s["pos"], s["cell"])
        e.enable_profile(False)
        ms, out = timed_md(e, s["vel"], args.steps, args.warmup, device, dist)
        ki = e.kspace_info()
        arms[name] = {"value": whole_job_rate(natm * args.steps, ms / 1e3, dist, device), "unit": "atom-steps/s",
                      "ms_per_step": max_over_ranks(ms, dist, device) / args.steps, "steps": args.steps,
                      "warmup": args.warmup, "k_vectors": ki["main"], "fp64_keps": keps, "kspace_reuse": reuse,
                      "solver_iters_mean": float(np.mean([t["scf_iter"] for t in out["thermo"]]))}
        if name == "fp64":
            last = e.positions()
        e.close()
    res = {}
    for name, pp in (("fp64", None), ("fp64_sphere_reuse", None), ("fp64_kmax_plus4", None), ("mixed", pm)):
        if pp is None:
            pp = copy_params(pm)
            pp.precision = abi.PREC_FP64
            pp.fp64_keps = pm.mixed_keps if name == "fp64_sphere_reuse" else 0.0
            pp.kspace_reuse = 1 if name == "fp64_sphere_reuse" else 0
        pp = copy_params(pp)
        pp.doefg = 1
        pp.efg_period = 0
        if name == "fp64_kmax_plus4":
            for d in range(3):
                pp.kES[d] = pm.kES[d] + 4
        e = mdff_b200.Engine(pp, s["itype"], last, s["cell"])
        res[name] = e.engforce()
        e.close()
    rel = lambda x, y: float(np.linalg.norm(x - y) / np.linalg.norm(y))
    b = res["fp64"]

    def errs(a):
        return {"eps_F": rel(a["f"], b["f"]), "eps_mu": rel(a["mu"], b["mu"]), "eps_efg": rel(a["efg"], b["efg"]),
                "eps_tau_coul": rel(a["tau_coul"], b["tau_coul"]),
                "eps_tau_total": rel(a["tau_coul"] + a["tau_nonb"], b["tau_coul"] + b["tau_nonb"]),
                "rel_u_coul": abs(a["e"]["u_coul"] - b["e"]["u_coul"]) / abs(b["e"]["u_coul"])}
    acc = {"positions": "the FP64 trajectory's after %d + %d steps" % (args.warmup, args.steps),
           "against": "plain FP64 path (whole half space, %d k-vectors)" % arms["fp64"]["k_vectors"],
           "mixed": errs(res["mixed"]), "fp64_sphere_reuse": errs(res["fp64_sphere_reuse"]),
           "fp64_kmax_plus4": errs(res["fp64_kmax_plus4"]),
           "definition": "global relative norms over all atoms and components (stress: 3x3 Frobenius; the "
                         "total stress nearly cancels between Coulomb and short range in this cell); "
                         "fp64_kmax_plus4 is the plain FP64 path's own k truncation (kmax+4 against kmax)"}
    return arms, acc


def run_engine(args):
    import torch
    world, rank, local, dist = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    import mdff_b200
    from mdff_b200 import abi, systems
    s = systems.mgo_production(ncell=args.ncell)
    p = s["params"]
    p.precision = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    p.device = local
    if args.ensemble == "npt":
        p.integrator = abi.NPT_NHCNP
        p.press = 0.0
        p.timesca_baro = 0.5
    p.algo_ext_dipole = abi.EXT_ASPC if args.ext == "aspc" else abi.EXT_POLY
    p.extrapolate_order = args.ext_order
    p.kspace_reuse = (1 if args.precision == "mixed" else 0) if args.reuse == "auto" else int(args.reuse)
    if args.ksplit is not None:
        p.mixed_ksplit = args.ksplit
    if args.keps is not None:
        p.mixed_keps = args.keps
    p.autotune = args.autotune
    p.kspace_tc = args.tc
    natm = len(s["itype"])
    eng = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    # the timed region runs without the per-kernel-group CUDA events (they
    # cost ~0.7 ms of gaps per step); a separate profiled pass afterwards
    # gives the kernel breakdown and the roofline's detail timers
    eng.enable_profile(False)
    stream_ptr = eng.stream()
    ext = torch.cuda.ExternalStream(stream_ptr, device=device)
    t0 = eng.md_start(s["vel"])
    if args.warmup:
        eng.step(args.warmup, thermo=False)
    eng.profile_reset()
    # L2: the per-step working set (k-space partials ~100 MB, lists ~60 MB,
    # per-atom arrays) exceeds the 126 MB L2 and is rewritten every step.
    barrier(dist, device)
    torch.cuda.synchronize(device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    g0 = eng.graph_info()
    with ClockSampler(local) as clk:
        ev0.record(ext)
        out = eng.step(args.steps, thermo=True)
        ev1.record(ext)
        ev1.synchronize()
    torch.cuda.synchronize(device)
    g1 = eng.graph_info()
    graph_timed = {k: int(g1[k] - g0[k]) for k in g1}   # how the timed steps ran (replays, captures, plain)
    ms = ev0.elapsed_time(ev1)
    launches = eng.profile()["_launches"]["count"]   # counted with the timers off too
    ms_max = max_over_ranks(ms, dist, device)
    value = whole_job_rate(natm * args.steps, ms / 1e3, dist, device)
    iters = [t["scf_iter"] for t in out["thermo"]]
    h = [t["h_tot"] for t in out["thermo"]]
    # end to end through the C ABI with host buffers (pinned), one call per step
    e2e = None
    if not args.no_e2e:
        pos = [torch.empty(natm, dtype=torch.float64, pin_memory=True).numpy() for _ in range(3)]
        vel = [torch.empty(natm, dtype=torch.float64, pin_memory=True).numpy() for _ in range(3)]
        cur = eng.positions()
        for k in range(3):
            pos[k][:] = cur[:, k]
        st = eng.state_velocities()
        for k in range(3):
            vel[k][:] = st[:, k]
        ke = max(2, min(args.steps, 10))
        eng.step_host(1, pos, vel)
        barrier(dist, device)
        torch.cuda.synchronize(device)
        t1 = time.perf_counter()
        for _ in range(ke):
            eng.step_host(1, pos, vel)
        t2 = time.perf_counter()
        e2e = {"value": whole_job_rate(natm * ke, t2 - t1, dist, device), "unit": "atom-steps/s", "steps": ke,
               "h2d_bytes_per_step": 6 * 8 * natm, "d2h_bytes_per_step": 9 * 8 * natm}
    # trajectory streaming: the same steps with TRAJFF frames written through
    # the engine's writer (device snapshot, copy stream, writer thread), against
    # the same loop without frames.  wall_ms_per_step runs to the end of the
    # last step on the device (frames that the writer could not keep up with
    # block frame() and show there); drain_ms_after_last_step is the writer's
    # tail, the frames still being formatted or written when the steps end
    stream = None
    if not args.no_stream:
        import shutil
        import tempfile
        tmpd = tempfile.mkdtemp(prefix="mdff_stream_")
        ks = max(40, args.steps)

        shm = tempfile.mkdtemp(prefix="mdff_stream_", dir="/dev/shm") if os.path.isdir("/dev/shm") else None

        def run_stream(iformat, every, where=None):
            w = None
            if every:
                w = eng.writer(os.path.join(where or tmpd, f"TRAJFF{iformat}"), "TRAJFF", iformat, "rvf",
                               system="MgO", labels=["O", "Mg"], nslot=4)
            torch.cuda.synchronize(device)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            t1 = time.perf_counter()
            a.record(ext)
            for k in range(ks):
                eng.advance(1)
                if w is not None and (k + 1) % every == 0:
                    w.frame()
            b.record(ext)
            b.synchronize()
            t2 = time.perf_counter()
            if w is not None:
                w.close()
            t3 = time.perf_counter()
            return a.elapsed_time(b), (t2 - t1) * 1e3, (t3 - t2) * 1e3

        base_ms, base_wall, _ = run_stream(1, 0)
        stream = {"steps": ks, "dir": tmpd, "no_frames": {"device_ms_per_step": base_ms / ks,
                                                          "wall_ms_per_step": base_wall / ks}}
        cases = [("trajff_rvf_unformatted_every_step", 0, 1, tmpd),
                 ("trajff_rvf_formatted_every_10_steps", 1, 10, tmpd)]
        if shm:
            cases += [("trajff_rvf_unformatted_every_step_to_dev_shm", 0, 1, shm),
                      ("trajff_rvf_formatted_every_10_steps_to_dev_shm", 1, 10, shm)]
        for label, iformat, every, where in cases:
            d_ms, w_ms, drain_ms = run_stream(iformat, every, where)
            nbytes = os.path.getsize(os.path.join(where, f"TRAJFF{iformat}"))
            stream[label] = {"device_ms_per_step": d_ms / ks, "wall_ms_per_step": w_ms / ks,
                             "wall_overhead_vs_no_frames": w_ms / base_wall - 1.0,
                             "drain_ms_after_last_step": drain_ms,
                             "bytes_written": nbytes,
                             "file_mb_per_s": nbytes / ((w_ms + drain_ms) / 1e3) / 1e6}
        shutil.rmtree(tmpd, ignore_errors=True)
        if shm:
            shutil.rmtree(shm, ignore_errors=True)
    # profiled pass (not part of the timed region)
    kp = max(2, min(args.steps, 10))
    eng.enable_profile(True)
    eng.profile_reset()
    outp = eng.step(kp, thermo=True)
    prof = eng.profile()
    det = eng.profile_detail()
    eng.enable_profile(False)
    iters_p = [t["scf_iter"] for t in outp["thermo"]]
    arms = acc = None
    if args.precision == "mixed" and not args.no_fp64:
        arms, acc = fp64_arms(s, p, args, device, dist)
    result = None
    if rank == 0:
        pipes = mdff_b200.measure_pipes(local)
        ki = eng.kspace_info()
        # algorithmic k-vectors per evaluation: the reference's half space on
        # the FP64 path; the FP32 set plus the FP64 low set on the mixed path
        nk_eff = ki["main"] + ki["low"]
        mean_it = float(np.mean(iters))
        mean_it_p = float(np.mean(iters_p))
        kern = {k: v for k, v in prof.items() if v["count"] > 0 and not k.startswith("_")}
        ksf = kern.get("sfac", {"ms": 0.0, "count": 0})
        kkf = kern.get("kfield", {"ms": 0.0, "count": 0})
        # algorithmic flops of the dominant pair of kernels over the timed region.
        # Evaluations per step: plain sequence: structure factor for the static
        # field, the first residual, each iteration and the forces; field for
        # all but the forces (E) plus one with the field gradient.  With
        # kspace_reuse the static field and first residual share one
        # evaluation and the forces take no structure-factor pass.
        if p.kspace_reuse:
            n_sf, n_e = 1 + mean_it_p, 1 + mean_it_p
        else:
            n_sf, n_e = 3 + mean_it_p, 2 + mean_it_p
        sf_flops = natm * nk_eff * 15.0 * n_sf * kp
        kf_flops = natm * nk_eff * (18.0 * n_e + 36.0) * kp
        k_ms = ksf["ms"] + kkf["ms"]
        total_ms = sum(v["ms"] for v in kern.values())
        tc_ms = det["sfac_tc"]["ms"] + det["kfield_tc"]["ms"]
        if args.precision == "mixed" and det["sfac_tc"]["count"] > 0:
            # dominant kernels: the tensor-core structure factor and field,
            # timed alone (CUDA events around each launch); achieved = the int8
            # digit-product operations of the unpadded GEMMs / their time
            tens = mdff_b200.measure_tensor(local)
            ops = det["sfac_tc"]["ops"] + det["kfield_tc"]["ops"]
            achieved = ops / (tc_ms / 1e3) / 1e12
            per = {}
            for k, v in det.items():
                if v["count"] and k != "efg_sites":
                    per[k] = {"launches": v["count"], "ms_per_launch": v["ms"] / v["count"],
                              "tops": v["ops"] / (v["ms"] / 1e3) / 1e12,
                              "traffic_mb": TC_TRAFFIC_MB.get(k)}
            # DRAM bytes per (structure factor + field) pair of the two main
            # kernels, weighted by their launch counts in the profiled pass
            n_s, n_f = det["sfac_tc"]["count"], det["kfield_tc"]["count"]
            traffic = (TC_TRAFFIC_MB["sfac_tc"] * n_s + TC_TRAFFIC_MB["kfield_tc"] * n_f) / max(1, n_s + n_f) * 1e6
            roof = {
                "bound": "tensor",
                "kernels": "k_sfac_tc + k_kfield_tc (tcgen05 kind::i8 digit GEMMs of the reciprocal sum)",
                "achieved": achieved,
                "peak": tens[0],
                "unit": "TOPS (int8, dense)",
                "frac": achieved / tens[0],
                "peak_source": "measured tcgen05 kind::i8 throughput on this GPU (mdff_measure_tensor): "
                               "N=256 %.0f, N=96 %.0f, N=64 %.0f TOPS" % tuple(tens),
                "per_kernel": per,
                "share_of_step": tc_ms / total_ms if total_ms else None,
                # algorithmic FP32-equivalent rate of the k-space sum these two kernels perform
                "kspace_fp32_equiv_tflops": (sf_flops + kf_flops) / (tc_ms / 1e3) / 1e12,
                "traffic": traffic,
                "traffic_note": "bytes per launch averaged over the two kernels' launches: ncu "
                                "dram__bytes_read.sum + dram__bytes_write.sum of one capture of each "
                                "(32 440 ions, kmax 23), per kernel in per_kernel.traffic_mb; the tensor "
                                "kernels are not memory-bound (a few % of HBM)",
            }
        else:
            achieved = (sf_flops + kf_flops) / (k_ms / 1e3) / 1e12 if k_ms > 0 else None
            peak = pipes[1] if args.precision == "mixed" else pipes[0]
            roof = {
                "bound": "fp32" if args.precision == "mixed" else "fp64",
                "kernels": "k-space structure factor + field (k_sfac*, k_kfield*)",
                "achieved": achieved,
                "peak": peak,
                "unit": "TFLOP/s",
                "frac": achieved / peak if achieved and peak else None,
                "peak_source": "measured FMA throughput on this GPU (mdff_measure_pipes): fp64 %.1f, fp32 %.1f, "
                               "fp32x2 %.1f TFLOP/s" % tuple(pipes),
                "share_of_step": k_ms / total_ms if total_ms else None,
                "traffic": None,
            }
        result = {
            "metric": METRIC,
            "value": value,
            "unit": "atom-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "fp32+fp64" if args.precision == "mixed" else "fp64",
            "data": "synthetic (seeded MgO polarisable-ion cell, mdff_b200.systems.mgo_production)",
            "config": {"workload": "mgo-pim-production", "natm": natm, "kmax": list(p.kES), "k_vectors": ki,
                       "rc": p.cutlongrange, "alpha": p.alphaES,
                       "ensemble": "npt-nhcnp (0 GPa)" if args.ensemble == "npt" else "nvt-nhcn", "nhc_n": p.nhc_n,
                       "dt_ps": p.dt, "efg_period": p.efg_period, "solver": "pcg", "tol": p.conv_tol_ind,
                       "predictor": "%s order %d" % (args.ext, args.ext_order),
                       "kspace_reuse": int(p.kspace_reuse),
                       "mixed_ksplit": p.mixed_ksplit if args.precision == "mixed" else None,
                       "mixed_keps": p.mixed_keps if args.precision == "mixed" else None,
                       "kspace_tc": int(p.kspace_tc) if args.precision == "mixed" else None,
                       "precision": args.precision, "parallelism": f"replicas{world}",
                       "l2": "per-step working set > 126 MB L2 (Verlet and pair-table lists, k-space digit "
                             "images, partials)"},
            "gpu_launches": int(launches),
            "graph_timed_steps": graph_timed,
            "launch_shape": eng.launch_shape(),
            "solver_iters_mean": mean_it,
            "h_tot_drift_per_step": (h[-1] - h[0]) / max(1, len(h) - 1) / natm,
            "profile_steps": kp,
            "kernels_ms_per_step": {k: round(v["ms"] / kp, 4) for k, v in kern.items()},
            "roofline": roof,
            "e2e": e2e,
            "fp64_arms": arms,
            "speedup_vs_fp64": value / arms["fp64"]["value"] if arms else None,
            "speedup_vs_fp64_sphere_reuse": value / arms["fp64_sphere_reuse"]["value"] if arms else None,
            "accuracy_vs_fp64": acc,
            "stream": stream,
            "step0": {"h_tot": t0["h_tot"], "temp_r": t0["temp_r"], "scf_iter": t0["scf_iter"]},
        }
        if not args.no_cpu:
            result["cpu_baseline"] = cpu_baseline(s, p, mean_it)
        result["clocks"] = clk.summary()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return result


def cpu_baseline(s, p, iters_per_step, kstride=16):
    """The CPU oracle (C++ FP64 restatement of the reference path) timed on
    all host cores: one Ewald field evaluation (real space over the Coulomb
    list, reciprocal space over every kstride-th k-vector, scaled back) and
    one BMHFTD pair loop; an MD step is (iterations + 2) field evaluations plus
    the pair loop."""
    import oracle
    o = oracle.Oracle(p, s["itype"], s["pos"], s["cell"])
    cores = oracle.max_threads()
    td, tr, tp = o.field_time(kstride)
    t_eval = td + tr * kstride
    t_step = (iters_per_step + 2) * t_eval + tp
    natm = len(s["itype"])
    return {"value": natm / t_step, "unit": "atom-steps/s", "cores": cores, "kind": "port", "host": host_cpu(),
            "sample": "one Ewald field evaluation of the 32440-ion cell (real space + every %dth k-vector, scaled) "
                      "and one BMHFTD pair loop, x (%.1f solver iterations + 2) evaluations per MD step"
                      % (kstride, iters_per_step),
            "seconds": {"dir": td, "rec_sampled": tr, "pair": tp}}


def run_accuracy(args):
    """Error of each mixed-precision result against the FP64 path at identical
    positions: snapshots every --snap-every steps of an FP64 NVT trajectory of
    the production cell.  Global relative norms ||x_mixed - x_fp64|| / ||x_fp64||
    for forces, dipoles, EFG, stresses; energies relative; also the per-atom
    maximum force deviation relative to the RMS force."""
    import torch
    import mdff_b200
    from mdff_b200 import abi, systems
    s = systems.mgo_production(ncell=args.ncell)
    p = s["params"]
    p.precision = abi.PREC_FP64
    traj = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    traj.md_start(s["vel"])
    pm = abi.Params()
    C.pointer(pm)[0] = p
    pm.precision = abi.PREC_MIXED
    pm.kspace_reuse = 1 if args.reuse in ("auto", "1") else 0
    if args.ksplit is not None:
        pm.mixed_ksplit = args.ksplit
    if args.keps is not None:
        pm.mixed_keps = args.keps
    pm.kspace_tc = args.tc
    pf = abi.Params()
    C.pointer(pf)[0] = p
    snaps = []
    for k in range(args.snapshots + 1):
        if k > 0:
            traj.step(args.snap_every, thermo=False)
        pos = traj.positions()
        res = {}
        for name, pp in (("fp64", pf), ("mixed", pm)):
            e = mdff_b200.Engine(pp, s["itype"], pos, s["cell"])
            res[name] = e.engforce()
            e.close()
        a, b = res["mixed"], res["fp64"]
        rel = lambda x, y: float(np.linalg.norm(x - y) / np.linalg.norm(y))
        df = np.linalg.norm(a["f"] - b["f"], axis=1)
        snaps.append({
            "step": k * args.snap_every,
            "eps_F": rel(a["f"], b["f"]),
            "max_atom_dF_over_rms_F": float(df.max() / np.sqrt((b["f"] ** 2).sum(1).mean())),
            "rms_F_eV_per_A": float(np.sqrt((b["f"] ** 2).sum(1).mean())),
            "eps_mu": rel(a["mu"], b["mu"]),
            "eps_efg": rel(a["efg"], b["efg"]),
            "eps_tau_coul": rel(a["tau_coul"], b["tau_coul"]),
            "rel_u_coul": abs(a["e"]["u_coul"] - b["e"]["u_coul"]) / abs(b["e"]["u_coul"]),
            "rel_u_bmhft": abs(a["e"]["u_bmhft"] - b["e"]["u_bmhft"]) / abs(b["e"]["u_bmhft"]),
            "du_per_atom_eV": abs(a["e"]["u_coul"] - b["e"]["u_coul"]) / len(pos),
            "iters": [a["e"]["scf_iter"], b["e"]["scf_iter"]],
        })
    return {"mode": "accuracy", "workload": "mgo-pim-production", "natm": len(s["itype"]),
            "mixed": {"kspace_reuse": int(pm.kspace_reuse), "mixed_ksplit": pm.mixed_ksplit,
                      "mixed_keps": pm.mixed_keps, "kspace_tc": int(pm.kspace_tc)}, "snapshots": snaps,
            "eps_F_max": max(x["eps_F"] for x in snaps)}


def host_cpu():
    """The host's logical CPU count and model name (from /proc/cpuinfo)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "model": model}


def run_reference(args):
    """Reference arm: the CPU oracle (C++ FP64 restatement of the reference's
    path; the Fortran/MPI reference cannot be built on this image) on all host
    cores, same 32 440-ion cell.  A whole MD step of the reference (its
    fixed-point SCF: about 35 multipole Ewald evaluations over all 51 911
    k-vectors) takes minutes on the host, so each timed step here is ONE
    complete multipole Ewald evaluation of the cell (real space over the
    Coulomb list and reciprocal space over every k-vector of the reference's
    half space, nothing sampled or scaled) plus one BMHFTD pair loop, and
    ms_per_step is its measured time.  value is the MD rate this implies:
    natm / ((SCF iterations + 2) x evaluation + pair loop), with the SCF
    iteration count of the reference's solver at the same tolerance measured
    on an 8^3-site replica of the model."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    import oracle
    from mdff_b200 import abi, systems
    s = systems.mgo_production(ncell=args.ncell)
    p = s["params"]
    small = systems.mgo_pim(grid=(8, 8, 8), rc=8.0, alpha=0.3, kmax=8, temp=2000.0, seed=11)
    sp = small["params"]
    sp.algo_moment_from_pola = abi.POLA_SCF
    sp.conv_tol_ind = p.conv_tol_ind
    sp.max_scf_pol_iter = 500
    so = oracle.Oracle(sp, small["itype"], small["pos"], small["cell"])
    so.md_start(small["vel"])
    st = so.step(2)
    iters = float(np.mean([t["scf_iter"] for t in st["thermo"]]))
    o = oracle.Oracle(p, s["itype"], s["pos"], s["cell"])
    natm = len(s["itype"])
    for _ in range(args.warmup):
        o.field_time(64)   # untimed warm-up: threads and caches, a 1/64 k sample
    samples = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        samples.append(o.field_time(1))
    wall = time.perf_counter() - t0
    td, tr, tp = (float(np.mean([x[k] for x in samples])) for k in range(3))
    t_eval = td + tr
    t_md = (iters + 2) * t_eval + tp
    v = natm / t_md
    cores = oracle.max_threads()
    cpu = host_cpu()
    k1, k2, k3 = p.kES
    nk = k3 + k2 * (2 * k3 + 1) + k1 * (2 * k2 + 1) * (2 * k3 + 1)   # the half space (src/field.f90:1648)
    sample = ("each timed step: one complete multipole Ewald evaluation of the %d-ion cell (real space + all "
              "%d k-vectors) and one BMHFTD pair loop; value = natm / ((%.1f SCF iterations + 2) x evaluation + "
              "pair loop)" % (natm, nk, iters))
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": "atom-steps/s",
        "n_gpus": 0,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp64",
        "data": "synthetic (seeded MgO polarisable-ion cell, mdff_b200.systems.mgo_production)",
        "config": {"workload": "mgo-pim-production", "natm": natm, "kmax": list(p.kES), "solver": "scf (reference)",
                   "solver_iters": iters, "precision": "fp64",
                   "step_unit": "one multipole Ewald evaluation + one pair loop (1/%.1f of an MD step's "
                                "evaluations)" % (iters + 2)},
        "md_step_derived": {"seconds_per_md_step": t_md, "evaluation_s": t_eval, "real_space_s": td,
                            "reciprocal_s": tr, "pair_loop_s": tp, "extrapolated": True,
                            "from": "measured evaluations x measured SCF iteration count"},
        "consistency": {"steps_timed": args.steps, "wall_s": wall,
                        "ms_per_step_x_steps_s": wall / args.steps * args.steps,
                        "fits_in_driver_run": wall < 600.0,
                        "note": "ms_per_step is the measured wall time of each timed step as run (one "
                                "evaluation + one pair loop); value is the MD rate derived from it"},
        "host": cpu,
        "cpu_baseline": {"value": v, "unit": "atom-steps/s", "cores": cores, "kind": "port", "sample": sample,
                         "host": cpu},
        "e2e": {"value": v, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_batch(args):
    """Force-matching workload: one evaluation = the loss of 64 MgO PIM
    configurations (200-2000 ions each, rc <= 10 A, PCG 1e-8) and its adjoint
    gradient with respect to the 12 force-field parameters, all configurations
    in one set of launches.  Targets are the FP64 forces and stresses at
    parameters perturbed 5 % from the seed values.  Timed on the FP64 batch
    and on the mixed one (the dipole operator's pair table in FP32); value is
    the one --precision names, and the mixed loss and gradient are compared
    with the FP64 ones.  Under torchrun the configurations are sharded over the
    ranks (balanced by atom count) and each evaluation ends with one all-reduce
    of the loss and the 12 gradient components: strong scaling of one batch."""
    import torch
    world, rank, local, dist = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    import mdff_b200
    from mdff_b200 import abi, fit, systems
    confs_all = systems.mgo_batch()
    confs, _ = fit.shard(confs_all, rank, world)
    base = systems.mgo_params(6.0, 0.5, 6)
    base.conv_tol_ind = 1e-8
    base.max_scf_pol_iter = 300
    base.device = local
    space = fit.mgo_space(base)
    theta0 = space.get(base)
    theta_t = theta0 * (1.0 + 0.05 * np.random.default_rng(7).standard_normal(len(theta0)))
    bt = mdff_b200.Batch(space.apply(base, theta_t), confs)
    tgt = bt.forces()
    bt.close()
    runs = {}
    clk_summary = None
    natm_local = int(sum(len(c["itype"]) for c in confs))
    natm = int(sum(len(c["itype"]) for c in confs_all))
    nat = (int(min(len(c["itype"]) for c in confs_all)), int(max(len(c["itype"]) for c in confs_all)))
    for prec_name, prec in (("fp64", abi.PREC_FP64), ("mixed", abi.PREC_MIXED)):
        bp = copy_params(base)
        bp.precision = prec
        b = mdff_b200.Batch(bp, confs)
        b.set_targets(tgt["f"], tgt["tau"], 1.0, 0.01)

        def evaluate():
            L, g, it = b.loss_grad()
            L, gt = fit.allreduce_loss_grad(L, space.project(g, theta0), len(confs), len(confs_all), dist, device)
            return L, gt, it

        for _ in range(max(args.warmup, 1)):
            evaluate()
        barrier(dist, device)
        torch.cuda.synchronize(device)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        its = []
        with ClockSampler(local) as clk:
            ev0.record()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                L, gt, it = evaluate()
                its.append(it)
            ev1.record()
            ev1.synchronize()
            t1 = time.perf_counter()
        ms = ev0.elapsed_time(ev1)
        if prec_name == args.precision:
            clk_summary = clk.summary()
        ms_max = max_over_ranks(ms, dist, device)
        wall_max = max_over_ranks(t1 - t0, dist, device)
        runs[prec_name] = {"value": args.steps / (ms_max / 1e3),
                           "ms_per_step": ms_max / args.steps,
                           "e2e": args.steps / wall_max,
                           "solve_iterations": {"forward": float(np.mean([i[0] for i in its])),
                                                "adjoint": float(np.mean([i[1] for i in its]))},
                           "loss": L, "grad": gt}
        b.close()
    sel = runs[args.precision]
    gm, gd = runs["mixed"]["grad"], runs["fp64"]["grad"]
    acc = {"rel_loss": abs(runs["mixed"]["loss"] - runs["fp64"]["loss"]) / abs(runs["fp64"]["loss"]),
           "rel_grad": float(np.linalg.norm(gm - gd) / np.linalg.norm(gd)),
           "max_component_rel_grad": float(np.max(np.abs(gm - gd) / np.abs(gd)))}
    result = None
    if rank == 0:
        result = {
            "metric": "force-matching loss+gradient evaluations/s, 64-configuration MgO PIM batch",
            "value": sel["value"],
            "unit": "evaluations/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": sel["ms_per_step"],
            "higher_is_better": True,
            "scaling": "strong",
            "vs_baseline": None,
            "dtype": "fp32+fp64" if args.precision == "mixed" else "fp64",
            "data": "synthetic (seeded rock-salt MgO snapshots, mdff_b200.systems.mgo_batch)",
            "config": {"workload": "mgo-pim-force-matching-batch", "nconf": len(confs_all), "natm_total": natm,
                       "natm_range": list(nat), "parameters": space.names, "precision": args.precision,
                       "solver": "pcg", "tol": base.conv_tol_ind,
                       "parallelism": f"dp{world}" if world > 1 else "dp1",
                       "sharding": "configurations over ranks, balanced by atoms; one all-reduce of 13 doubles "
                                   "per evaluation" if world > 1 else None,
                       "rank0_configurations": len(confs), "rank0_atoms": natm_local,
                       "l2": "each evaluation rewrites > 126 MB (k-space partials, lists of 69k ions)"},
            "atom_evaluations_per_s": natm * sel["value"],
            "solve_iterations": sel["solve_iterations"],
            "fp64": {k: v for k, v in runs["fp64"].items() if k not in ("grad",)},
            "mixed": {k: v for k, v in runs["mixed"].items() if k not in ("grad",)},
            "mixed_vs_fp64": acc,
            "e2e": {"value": sel["e2e"], "unit": "evaluations/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 8 + 82048},
            "clocks": clk_summary,
        }
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return result


def run_opt(args):
    """Structure-optimisation workload: the reference's conjugate-gradient
    minimiser (sastry) on the production cell from its jittered start, capped
    at --opt-iters iterations.  Every line-search point is one full force
    evaluation (pair loop, real and reciprocal Ewald, induced-dipole solve), so
    value = atoms x force evaluations / device time; e2e adds loading the
    positions from host memory and reading the minimised ones back."""
    import torch
    world, rank, local, dist = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    import mdff_b200
    from mdff_b200 import abi, systems
    s = systems.mgo_production(ncell=args.ncell)
    p = s["params"]
    p.precision = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    p.device = local
    p.kspace_reuse = (1 if args.precision == "mixed" else 0) if args.reuse == "auto" else int(args.reuse)
    p.autotune = args.autotune
    p.kspace_tc = args.tc
    natm = len(s["itype"])
    pos0 = np.ascontiguousarray(s["pos"])
    eng = mdff_b200.Engine(p, s["itype"], pos0, s["cell"])
    ext = torch.cuda.ExternalStream(eng.stream(), device=device)
    if args.optalgo == "lbfgs":
        def minimise(cap):   # cap: force evaluations, the driver's itmax
            return eng.opt_lbfgs(cap)
        cap = args.opt_iters * 5
    elif args.optalgo == "m1qn3":
        def minimise(cap):   # cap: M1QN3 iterations (niter), simulations 5x that
            return eng.opt_m1qn3(cap, 5 * cap)
        cap = args.opt_iters * 5
    else:
        def minimise(cap):   # cap: conjugate-gradient iterations
            return eng.opt_sastry(cap)
        cap = args.opt_iters
    for _ in range(max(args.warmup, 1)):
        eng.set_positions(pos0)
        minimise(2)
    eng.set_positions(pos0)
    barrier(dist, device)
    torch.cuda.synchronize(device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(ext)
        r = minimise(cap)
        ev1.record(ext)
        ev1.synchronize()
    torch.cuda.synchronize(device)
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, dist, device)
    value = whole_job_rate(natm * r["nforce"], ms / 1e3, dist, device)
    # end to end: positions from pinned host memory in, minimised positions out
    hp = torch.empty((natm, 3), dtype=torch.float64, pin_memory=True).numpy()
    hp[:] = pos0
    barrier(dist, device)
    t1 = time.perf_counter()
    eng.set_positions(hp)
    r2 = minimise(cap)
    out = eng.positions()
    t2 = time.perf_counter()
    e2e_v = whole_job_rate(natm * r2["nforce"], t2 - t1, dist, device)
    result = None
    if rank == 0:
        result = {
            "metric": "structure-optimisation atom-force-evaluations/s, 32k-ion MgO PIM (" +
                      {"lbfgs": "limited-memory BFGS, More-Thuente line search)",
                       "m1qn3": "M1QN3 diagonal initial scaling, Wolfe line search mlis3)",
                       "sastry": "conjugate gradients, cubic line search)"}[args.optalgo],
            "value": value,
            "unit": "atom-evaluations/s",
            "n_gpus": world,
            "steps": r["iterations"],
            "warmup": args.warmup,
            "ms_per_step": ms_max / max(r["nforce"], 1),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "fp32+fp64" if args.precision == "mixed" else "fp64",
            "data": "synthetic (seeded MgO polarisable-ion cell, mdff_b200.systems.mgo_production)",
            "config": {"workload": "mgo-pim-opt", "natm": natm,
                       "algorithm": {"lbfgs": "lbfgs (m = 5, More-Thuente line search)",
                                     "m1qn3": "m1qn3 (DIS, m = 5, mlis3)",
                                     "sastry": "sastry (cg + cubic line search)"}[args.optalgo],
                       "cap": {"lbfgs": "force evaluations", "m1qn3": "iterations",
                               "sastry": "iterations"}[args.optalgo] + f" <= {cap}", "precision": args.precision, "kspace_tc": int(p.kspace_tc),
                       "parallelism": f"replicas{world}",
                       "l2": "per-evaluation working set > 126 MB L2"},
            "opt": r,
            "e2e": {"value": e2e_v, "unit": "atom-evaluations/s", "h2d_bytes_per_step": 24 * natm,
                    "d2h_bytes_per_step": 24 * natm + 48},
            "clocks": clk.summary(),
        }
        if not args.no_cpu:
            cb = cpu_baseline(s, p, 8.0)
            cb["unit"] = "atom-evaluations/s"
            cb["sample"] = cb["sample"].replace("per MD step", "per force evaluation")
            result["cpu_baseline"] = cb
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return result


def run_efg(args):
    """EFG post-processing workload (efg_stat over an EFGALL of --efg-conf
    configurations of the production cell): per site the Czjzek components,
    principal values in the NMR convention, per-type statistics and the Vzz,
    eta, U and S distributions.  The tensors are the production cell's EFG from
    one force evaluation plus seeded traceless noise of 20 % of their scale per
    configuration (synthetic configurations of the same shape and value
    distribution).  One step = all configurations, 128 x 32 440 sites, 199 MB of
    tensors (> 126 MB L2, re-read every step).  value: the tensors resident in
    device memory; e2e: from pinned host memory through the same call, with the
    histograms and statistics read back."""
    import torch
    world, rank, local, dist = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    import mdff_b200
    from mdff_b200 import abi, systems
    s = systems.mgo_production(ncell=args.ncell)
    p = s["params"]
    p.precision = abi.PREC_MIXED
    p.device = local
    p.doefg = 1
    natm = len(s["itype"])
    eng = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    base = eng.engforce()["efg"]                         # [natm][6]
    nc = args.efg_conf
    scale = float(np.abs(base).max())
    rng = np.random.default_rng(11)
    host = torch.empty((nc, 6, natm), dtype=torch.float64, pin_memory=True)
    hn = host.numpy()
    for c in range(nc):
        noise = rng.normal(0.0, 0.2 * scale, (natm, 6))
        noise[:, 2] = -(noise[:, 0] + noise[:, 1])
        hn[c] = (base + noise).T
    dev = host.to(device)
    torch.cuda.synchronize(device)
    vz = 3.0 * scale
    dp = abi.EfgDistParams()
    dp.vzzmin, dp.resvzz, dp.reseta, dp.umin, dp.resu, dp.smax = -vz, vz / 150, 0.01, -vz, vz / 150, 2 * vz
    ext = torch.cuda.ExternalStream(eng.stream(), device=device)
    for _ in range(max(args.warmup, 3)):
        eng.efg_dist_ptr(dp, dev.data_ptr(), nc)
    barrier(dist, device)
    torch.cuda.synchronize(device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(ext)
        for _ in range(args.steps):
            out = eng.efg_dist_ptr(dp, dev.data_ptr(), nc)
        ev1.record(ext)
        ev1.synchronize()
    torch.cuda.synchronize(device)
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, dist, device)
    sites = natm * nc
    value = whole_job_rate(sites * args.steps, ms / 1e3, dist, device)
    # end to end: tensors from pinned host memory each step
    barrier(dist, device)
    t1 = time.perf_counter()
    for _ in range(args.steps):
        out_h = eng.efg_dist_ptr(dp, host.data_ptr(), nc)
    t2 = time.perf_counter()
    e2e_v = whole_job_rate(sites * args.steps, t2 - t1, dist, device)
    same = all(np.array_equal(out[k], out_h[k]) for k in ("vzz", "eta", "u", "s"))
    # the site kernel alone (detail timer) for the roofline
    eng.enable_profile(True)
    eng.profile_reset()
    kp = min(args.steps, 10)
    for _ in range(kp):
        eng.efg_dist_ptr(dp, dev.data_ptr(), nc)
    det = eng.profile_detail()["efg_sites"]
    eng.enable_profile(False)
    result = None
    if rank == 0:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        ach = det["ops"] / (det["ms"] / 1e3) / 1e9
        nbins = sum(int(np.prod(out[k].shape)) for k in ("vzz", "eta", "u", "s"))
        result = {
            "metric": "EFG post-processing sites/s (efg_stat: NMR principal values, statistics, distributions), "
                      "32k-ion MgO PIM configurations",
            "value": value,
            "unit": "sites/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": max(args.warmup, 3),
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "fp64",
            "data": "synthetic (production-cell EFG of one force evaluation + seeded traceless noise per "
                    "configuration)",
            "config": {"workload": "mgo-pim-efg-stat", "natm": natm, "nconf": nc, "ntype": int(p.ntype),
                       "bins": nbins, "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (%.0f MB of tensors per step)" % (48.0 * sites / 1e6)},
            "gpu_launches": 2 * args.steps,
            "roofline": {"bound": "hbm", "kernels": "k_efg_sites (one pass: tensor read once)",
                         "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": ach / peaks["hbm_gbs"],
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                         "algorithmic_bytes_per_site": 52, "ms_per_launch": det["ms"] / max(det["count"], 1),
                         "share_of_step": (det["ms"] / kp) / (ms_max / args.steps), "traffic": None},
            "e2e": {"value": e2e_v, "unit": "sites/s", "h2d_bytes_per_step": 48 * sites,
                    "d2h_bytes_per_step": 4 * (nbins + 1) + 8 * nc * (p.ntype + 1) * 28,
                    "same_histograms_as_device_input": bool(same)},
            "clocks": clk.summary(),
        }
        if not args.no_cpu:
            from oracle import efg_stat
            sub_n = 4096
            t0 = time.perf_counter()
            efg_stat.efg_dist(hn[0].T[:sub_n], s["itype"][:sub_n], int(p.ntype), dp.vzzmin, dp.resvzz, dp.reseta,
                              dp.umin, dp.resu, dp.smax)
            dt = time.perf_counter() - t0
            result["cpu_baseline"] = {"value": sub_n / dt, "unit": "sites/s", "cores": 1, "kind": "port",
                                      "sample": f"{sub_n} sites of one configuration through the numpy "
                                                "restatement (LAPACK eigvalsh per site)"}
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return result


def run_rmc(args):
    """Reverse Monte Carlo workload (rmc_main on the g(r) chi^2): the
    32 440-ion production cell fitted to the g(r) (cut 10 A, 0.05 A bins, two
    types) of a seeded perturbation of itself (synthetic target of the same
    shape).  One step = --rmc-moves trial moves of one chain on the device;
    value = trial moves / device time.  e2e adds loading the positions and the
    target from host memory and reading the chain's g(r) and positions back.
    The reference recounts every pair at every move (O(N^2) per move); the
    device chain updates the counts from the moved atom's N - 1 pairs."""
    import torch
    world, rank, local, dist = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    import mdff_b200
    from mdff_b200 import abi, systems
    s = systems.mgo_production(ncell=args.ncell)
    p = s["params"]
    p.device = local
    natm = len(s["itype"])
    pos0 = np.ascontiguousarray(s["pos"])
    eng = mdff_b200.Engine(p, s["itype"], pos0, s["cell"])
    cut, res = 10.0, 0.05
    tgt = pos0 + np.random.default_rng(21).normal(0.0, 0.12, pos0.shape)
    eng.set_positions(tgt)
    gexp = eng.gr(cut, res)
    eng.set_positions(pos0)
    rp = abi.RmcParams()
    rp.max_displacement = 0.1
    rp.resolution_gr = res
    rp.cut_rmc = cut
    for q in range(6):
        rp.temp_rmc[q] = 1e-4
    rp.acceptance_max = 10 ** 12
    rp.max_trials = args.rmc_moves + 1
    ext = torch.cuda.ExternalStream(eng.stream(), device=device)
    for _ in range(max(args.warmup, 3)):
        eng.rmc(rp, gexp, seed=1)
    eng.set_positions(pos0)
    barrier(dist, device)
    torch.cuda.synchronize(device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    moves = 0
    chis = []
    with ClockSampler(local) as clk:
        ev0.record(ext)
        for k in range(args.steps):
            r, g = eng.rmc(rp, gexp, seed=1000 + k)
            moves += r["kall"] - 1
            chis.append(r["chisq"][0])
        ev1.record(ext)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, dist, device)
    value = whole_job_rate(moves, ms / 1e3, dist, device)
    # end to end: positions in from host memory, g(r) and positions out, each step
    barrier(dist, device)
    t1 = time.perf_counter()
    for k in range(args.steps):
        eng.set_positions(pos0)
        r2, g2 = eng.rmc(rp, gexp, seed=2000 + k)
        eng.positions()
    t2 = time.perf_counter()
    e2e_v = whole_job_rate(args.steps * (rp.max_trials - 1), t2 - t1, dist, device)
    result = None
    if rank == 0:
        result = {
            "metric": "reverse Monte Carlo trial moves/s (g(r) chi^2), 32k-ion MgO PIM cell",
            "value": value,
            "unit": "moves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": max(args.warmup, 3),
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "fp64",
            "data": "synthetic (target g(r) of a seeded perturbation of the production cell)",
            "config": {"workload": "mgo-pim-rmc-gr", "natm": natm, "cut_rmc": cut, "resolution_gr": res,
                       "moves_per_step": rp.max_trials - 1, "parallelism": f"replicas{world}",
                       "l2": "positions (0.8 MB) L2-resident by design: the chain reads them at every move"},
            "gpu_launches": 4 * args.steps,
            "pair_distances_per_s": value * 2.0 * (natm - 1),
            "chisq_last": chis[-1],
            "roofline": {"bound": "hbm", "kernels": "k_rmc_chain (one CTA: the Markov chain is sequential)",
                         "achieved": value * 2.0 * (natm - 1) * 24.0 / 1e9,
                         "peak": json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"],
                         "unit": "GB/s", "frac": None, "traffic": None,
                         "note": "latency-bound by design: each move depends on the previous one; achieved counts "
                                 "the 24 bytes of coordinates read per pair distance (from L2)"},
            "e2e": {"value": e2e_v, "unit": "moves/s", "h2d_bytes_per_step": 24 * natm,
                    "d2h_bytes_per_step": 24 * natm + 8 * gexp.size},
            "clocks": clk.summary(),
        }
        roof = result["roofline"]
        roof["frac"] = roof["achieved"] / roof["peak"]
    if args.rmc_efg_moves > 0:
        # the EFG chi^2 terms (rmc_efg): the same cell as rigid ions (the
        # reference's rmc_efg takes point charges), U, Vzz and eta fitted to
        # the distributions of the perturbed target, every trial one Ewald
        # EFG of the whole trial configuration; on the FP64 path and on the
        # mixed one, Verlet lists with the chain's own validity tracking
        efg_runs = {}
        for prec_name, prec in (("fp64", abi.PREC_FP64), ("mixed", abi.PREC_MIXED)):
            pr = type(p).from_buffer_copy(p)
            for t in range(pr.ntype):
                pr.ldip_polar[t] = 0
                pr.poldip_iso[t] = 0.0
            pr.doefg = 1
            pr.precision = prec
            pr.lvnlist = 1
            pr.skindiff = max(pr.skindiff, 1.0)
            er = mdff_b200.Engine(pr, s["itype"], tgt, s["cell"])
            ep = abi.RmcEfgParams()
            ep.lrmc_u = ep.lrmc_vzz = ep.lrmc_eta = 1
            ep.resolution_u_efg, ep.u_efg_min = 0.02, -1.0
            ep.resolution_vzz_efg, ep.vzz_efg_min = 0.02, -2.0
            ep.resolution_eta_efg = 0.02
            su, sv, se = ep.shapes(pr.ntype)
            r1 = abi.RmcParams.from_buffer_copy(rp)
            r1.acceptance_max, r1.max_trials = 1, 1
            _, _, Ux, Vx, Ex = er.rmc_efg(r1, ep, gexp, np.zeros(su), np.zeros(sv), np.zeros(se))
            er.set_positions(pos0)
            r1.acceptance_max, r1.max_trials = 10 ** 12, 4
            er.rmc_efg(r1, ep, gexp, Ux, Vx, Ex, seed=5)   # warm-up
            er.set_positions(pos0)
            r1.max_trials = args.rmc_efg_moves + 1
            ext2 = torch.cuda.ExternalStream(er.stream(), device=device)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(device)
            e0.record(ext2)
            rr, *_ = er.rmc_efg(r1, ep, gexp, Ux, Vx, Ex, seed=7)
            e1.record(ext2)
            e1.synchronize()
            ems = e0.elapsed_time(e1)
            # where a move's time goes: a profiled pass of the same length
            er.set_positions(pos0)
            er.enable_profile(True)
            er.profile_reset()
            t0 = time.perf_counter()
            rq, *_ = er.rmc_efg(r1, ep, gexp, Ux, Vx, Ex, seed=7)
            wall_ms = (time.perf_counter() - t0) * 1e3
            kprof = {k: round(v["ms"] / max(1, rq["kall"] - 1), 4) for k, v in er.profile().items()
                     if v["count"] > 0 and not k.startswith("_")}
            er.enable_profile(False)
            er.close()
            efg_runs[prec_name] = {"value": (rr["kall"] - 1) / (ems / 1e3), "moves": rr["kall"] - 1,
                                   "accepted": rr["kacc"] - 1, "ms_per_move": ems / max(1, rr["kall"] - 1),
                                   "chisq_last": rr["chisq"], "kernels_ms_per_move": kprof,
                                   "profiled_wall_ms_per_move": wall_ms / max(1, rq["kall"] - 1)}
        if result is not None:
            result["efg_terms"] = {
                "metric": "reverse Monte Carlo trial moves/s with the g(r), U, Vzz and eta chi^2 terms, 32k-ion "
                          "rigid-ion MgO",
                "value": efg_runs["mixed"]["value"], "unit": "moves/s", "bins": {"U": su, "vzz": sv, "eta": se},
                "fp64": efg_runs["fp64"], "mixed": efg_runs["mixed"],
                "note": "one full-device Ewald EFG evaluation of the trial configuration per move, as rmc_efg "
                        "computes it (multipole_efg_ES); value = the mixed path"}
    if args.rmc_var_moves > 0:
        # the distance-variance term (eval_chisq_var_distance): the sorted
        # distance lists of all 32k ions (natm^2 doubles, 8.4 GB) built once
        # per call and kept on the device; per trial the moved ion's lists are
        # sorted again and one value moves in every other ion's list
        ev = mdff_b200.Engine(p, s["itype"], pos0, s["cell"])
        ep = abi.RmcEfgParams()
        ep.lrmc_var = 1
        ep.resolution_u_efg = ep.resolution_vzz_efg = ep.resolution_eta_efg = 0.1
        ep.u_efg_min = ep.vzz_efg_min = -1.0
        su, sv, se = ep.shapes(p.ntype)
        z = (np.zeros(su), np.zeros(sv), np.zeros(se))
        r1 = abi.RmcParams.from_buffer_copy(rp)
        r1.acceptance_max, r1.max_trials = 10 ** 12, 1
        t0 = time.perf_counter()
        ev.rmc_efg(r1, ep, gexp, *z, seed=5)   # the set-up alone: lists, sort, first chi^2
        setup_s = time.perf_counter() - t0
        r1.max_trials = args.rmc_var_moves + 1
        t0 = time.perf_counter()
        rv, *_ = ev.rmc_efg(r1, ep, gexp, *z, seed=7)
        wall = time.perf_counter() - t0
        ev.close()
        moves = rv["kall"] - 1
        if result is not None:
            result["variance_term"] = {
                "metric": "reverse Monte Carlo trial moves/s with the g(r) and distance-variance chi^2 terms, 32k ions",
                "value": moves / max(1e-9, wall - setup_s), "unit": "moves/s", "moves": moves,
                "accepted": rv["kacc"] - 1, "setup_s": setup_s, "wall_s_with_setup": wall,
                "chisq_var_last": rv["chisq"][1],
                "note": "value = moves / (wall time of the call - its set-up, both timed on the host around the "
                        "synchronous call); the reference recounts all natm^2 distances and sorts every list at "
                        "each trial"}
    if result is not None:
        if not args.no_cpu:
            import oracle
            o = oracle.Oracle(p, s["itype"], pos0, s["cell"])
            u = np.random.default_rng(3).random(64)
            rq = abi.RmcParams()
            ctypes_copy = C.pointer(rq)
            ctypes_copy[0] = rp
            rq.max_trials = 3
            t0 = time.perf_counter()
            ro, _ = o.rmc(rq, gexp, u)
            dt = time.perf_counter() - t0
            result["cpu_baseline"] = {"value": (ro["kall"] - 1) / dt, "unit": "moves/s", "cores": 1, "kind": "port",
                                      "sample": "2 trial moves of the oracle's chain (full O(N^2) recount per move, "
                                                "as the reference)"}
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return result


def main():
    args = parse()
    if args.accuracy:
        r = run_accuracy(args)
    elif args.impl == "reference":
        r = run_reference(args)
    elif args.workload == "batch":
        r = run_batch(args)
    elif args.workload == "opt":
        r = run_opt(args)
    elif args.workload == "efg":
        r = run_efg(args)
    elif args.workload == "rmc":
        r = run_rmc(args)
    else:
        r = run_engine(args)
    if r is not None:
        print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
