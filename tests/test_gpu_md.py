"""Short MD trajectories on the GPU against the oracle: NVE velocity Verlet
(prop_velocity_verlet), the Nose-Hoover chain (nhcn / chain_nhcn) and the
polarisable-ion model with dipole extrapolation, step by step."""
import numpy as np
import pytest

import mdff_b200
import oracle
from mdff_b200 import abi, systems

from helpers import rel

pytestmark = pytest.mark.gpu


def run_both(s, nsteps):
    p = s["params"]
    e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    o = oracle.Oracle(p, s["itype"], s["pos"], s["cell"])
    te0 = e.md_start(s["vel"])
    to0 = o.md_start(s["vel"])
    re = e.step(nsteps)
    ro = o.step(nsteps)
    return te0, to0, re, ro


def test_lj_nve_100_steps():
    s = systems.lj_argon()
    te0, to0, re, ro = run_both(s, 100)
    assert abs(te0["e_tot"] - to0["e_tot"]) < 1e-12 * abs(to0["e_tot"])
    for a, b in zip(re["thermo"], ro["thermo"]):
        assert abs(a["e_tot"] - b["e_tot"]) < 1e-9 * abs(b["e_tot"])
        assert abs(a["u_tot"] - b["u_tot"]) < 1e-9 * abs(b["u_tot"])
        assert a["nlist_rebuilt"] == b["nlist_rebuilt"]
    assert rel(re["pos"], ro["pos"]) < 1e-10
    assert rel(re["f"], ro["f"]) < 1e-8
    assert sum(t["nlist_rebuilt"] for t in re["thermo"]) > 0


def test_silica_nhc_chain():
    # the BKS-type pairs collapse from random starts within a few fs at 3000 K;
    # a 0.1 fs step keeps these 10 steps finite, which is all a parity check needs
    s = systems.silica_bmh()
    p = s["params"]
    p.dt = 0.0001
    te0, to0, re, ro = run_both(s, 10)
    for a, b in zip(re["thermo"], ro["thermo"]):
        assert abs(a["h_tot"] - b["h_tot"]) < 1e-9 * abs(b["h_tot"])
        assert abs(a["e_nvt"] - b["e_nvt"]) < 1e-9 * max(1.0, abs(b["e_nvt"]))
        assert abs(a["temp_r"] - b["temp_r"]) < 1e-9 * b["temp_r"]
    assert rel(re["pos"], ro["pos"]) < 1e-11


def test_lj_nhc_chain_300_steps():
    s = systems.lj_argon(ncell=4)
    p = s["params"]
    p.integrator = abi.NVT_NHCN
    p.nhc_n = 3
    p.temp = 1.2
    p.timesca_thermo = 0.5
    te0, to0, re, ro = run_both(s, 300)
    for a, b in zip(re["thermo"], ro["thermo"]):
        assert abs(a["h_tot"] - b["h_tot"]) < 1e-8 * abs(b["h_tot"])
        assert a["nlist_rebuilt"] == b["nlist_rebuilt"]


@pytest.mark.parametrize("literal", [0, 1])
def test_lj_nhc2_300_steps(literal):
    """nvt-nhc2 (nhc2 + chain_nhc2, src/integration.f90:205-324) step by step
    against the oracle, with the corrected and with the reference's literal
    thermostat energy."""
    s = systems.lj_argon(ncell=4)
    p = s["params"]
    p.integrator = abi.NVT_NHC2
    p.temp = 1.2
    p.timesca_thermo = 0.5
    p.nhc_literal = literal
    te0, to0, re, ro = run_both(s, 300)
    for a, b in zip(re["thermo"], ro["thermo"]):
        assert abs(a["h_tot"] - b["h_tot"]) < 1e-8 * abs(b["h_tot"])
        assert abs(a["e_nvt"] - b["e_nvt"]) < 1e-8 * max(1.0, abs(b["h_tot"]))
        assert abs(a["temp_r"] - b["temp_r"]) < 1e-8 * b["temp_r"]
        assert a["nlist_rebuilt"] == b["nlist_rebuilt"]
    assert rel(re["pos"], ro["pos"]) < 1e-10


def test_pim_nhc2_fp64_and_mixed():
    """nhc2 on the polarisable-ion model: FP64 engine against the oracle, and
    the mixed path tracking the FP64 path."""
    s = systems.mgo_pim(grid=(6, 6, 6), rc=6.0, alpha=0.55, kmax=8, temp=1000.0)
    p = s["params"]
    p.integrator = abi.NVT_NHC2
    p.timesca_thermo = 0.05
    p.conv_tol_ind = 1e-10
    te0, to0, re, ro = run_both(s, 10)
    for a, b in zip(re["thermo"], ro["thermo"]):
        assert abs(a["h_tot"] - b["h_tot"]) < 1e-9 * abs(b["h_tot"])
        assert abs(a["temp_r"] - b["temp_r"]) < 1e-8 * b["temp_r"]
    p.precision = abi.PREC_MIXED
    m = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    m.md_start(s["vel"])
    rm = m.step(10)
    for a, b in zip(rm["thermo"], re["thermo"]):
        assert abs(a["h_tot"] - b["h_tot"]) < 1e-6 * abs(b["h_tot"])


@pytest.mark.parametrize("ext", [(abi.EXT_POLY, 0), (abi.EXT_POLY, 1), (abi.EXT_POLY, 3), (abi.EXT_ASPC, 2)])
def test_pim_nve_with_extrapolation(ext):
    s = systems.mgo_pim(grid=(6, 6, 6), rc=6.0, alpha=0.55, kmax=8, temp=1000.0)
    p = s["params"]
    p.algo_ext_dipole, p.extrapolate_order = ext
    p.algo_moment_from_pola = abi.POLA_SCF
    p.conv_tol_ind = 1e-9
    te0, to0, re, ro = run_both(s, 8)
    for a, b in zip(re["thermo"], ro["thermo"]):
        assert abs(a["e_tot"] - b["e_tot"]) < 1e-9 * abs(b["e_tot"])
        assert a["scf_iter"] == b["scf_iter"]
    assert rel(re["f"], ro["f"]) < 1e-8


@pytest.mark.parametrize("ext", [(abi.EXT_POLY, 0), (abi.EXT_ASPC, 3)])
def test_pim_pcg_kspace_reuse_vs_oracle(ext):
    """kspace_reuse (one reciprocal evaluation for the static field and the
    first residual; final structure factor from the solver's by linearity):
    the same trajectory as the oracle's plain sequence of evaluations."""
    s = systems.mgo_pim(grid=(6, 6, 6), rc=6.0, alpha=0.55, kmax=8, temp=1000.0)
    p = s["params"]
    p.algo_ext_dipole, p.extrapolate_order = ext
    p.algo_moment_from_pola = abi.POLA_PCG
    p.conv_tol_ind = 1e-11
    p.doefg = 1
    p.kspace_reuse = 1
    te0, to0, re, ro = run_both(s, 8)
    assert abs(te0["e_tot"] - to0["e_tot"]) < 1e-10 * abs(to0["e_tot"])
    for a, b in zip(re["thermo"], ro["thermo"]):
        assert abs(a["e_tot"] - b["e_tot"]) < 1e-9 * abs(b["e_tot"])
        assert abs(a["pressure_tot"] - b["pressure_tot"]) < 1e-8 * max(1.0, abs(b["pressure_tot"]))
    assert rel(re["f"], ro["f"]) < 1e-8



def _pim_pcg_nhc():
    s = systems.mgo_pim(grid=(8, 8, 8), rc=6.0, alpha=0.5, kmax=8, temp=1500.0, integrator=abi.NVT_NHCN)
    p = s["params"]
    p.algo_moment_from_pola = abi.POLA_PCG
    p.algo_ext_dipole = abi.EXT_ASPC
    p.extrapolate_order = 3
    p.kspace_reuse = 1
    p.conv_tol_ind = 1e-9
    p.doefg = 1
    return s


def _run(s, nsteps, profile=False, **over):
    p = s["params"]
    for k, v in over.items():
        setattr(p, k, v)
    e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    e.enable_profile(profile)
    e.md_start(s["vel"])
    out = e.step(nsteps)
    return e, out


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_graph_steps_equal_plain_steps(prec):
    """Steps replayed from the captured CUDA graph (the whole step, the PCG as a
    conditional loop on the device) leave bit for bit the state, forces and
    thermodynamics of the same steps run as plain launches (profiling keeps a
    context on plain launches)."""
    s = _pim_pcg_nhc()
    runs = {}
    for prof in (False, True):
        e, out = _run(s, 20, profile=prof, precision=prec)
        runs[prof] = (e.positions(), e.velocities(), out, e.graph_info())
    g, pl = runs[False], runs[True]
    assert g[3]["graph_steps"] >= 10 and g[3]["captures"] >= 1, g[3]
    assert pl[3]["graph_steps"] == 0 and pl[3]["plain_steps"] == 20, pl[3]
    assert np.array_equal(g[0], pl[0]) and np.array_equal(g[1], pl[1])
    assert np.array_equal(g[2]["f"], pl[2]["f"])
    for a, b in zip(g[2]["thermo"], pl[2]["thermo"]):
        assert a["h_tot"] == b["h_tot"] and a["scf_iter"] == b["scf_iter"] and a["scf_rmsd"] == b["scf_rmsd"]


@pytest.mark.parametrize("integ", [abi.NVE_VV, abi.NVT_NHC2])
def test_graph_steps_lj_and_nhc2(integ):
    """The graph path of the pair-only integrators: LJ NVE and nvt-nhc2 against
    the oracle, with the steps replayed from graphs."""
    s = systems.lj_argon(ncell=4)
    p = s["params"]
    p.integrator = integ
    p.temp = 1.2
    p.timesca_thermo = 0.5
    te0, to0, re, ro = run_both(s, 50)
    for a, b in zip(re["thermo"], ro["thermo"]):
        assert abs(a["h_tot"] - b["h_tot"]) < 1e-8 * abs(b["h_tot"])
        assert a["nlist_rebuilt"] == b["nlist_rebuilt"]
    e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    e.md_start(s["vel"])
    e.step(10)
    assert e.graph_info()["graph_steps"] >= 9


def test_efg_period():
    """efg_period = 10: the EFG is written on steps 10, 20, ...; forces and
    the trajectory are bit for bit those of EFG at every step, and after step
    15 the context's EFG is still that of step 10."""
    s = _pim_pcg_nhc()
    e1, _ = _run(s, 10, efg_period=1)
    nmr10 = e1.efg_nmr()[0]
    out1 = e1.step(5)
    e10, out10 = _run(s, 15, efg_period=10)
    assert np.array_equal(e1.positions(), e10.positions())
    assert np.array_equal(out1["f"], out10["f"])
    assert np.array_equal(e10.efg_nmr()[0], nmr10)
    assert not np.array_equal(e1.efg_nmr()[0], nmr10)
    out1b = e1.step(5)
    out10b = e10.step(5)
    assert np.array_equal(e1.efg_nmr()[0], e10.efg_nmr()[0])   # step 20 writes the EFG in both


def test_lj_nve_1000_steps():
    """Config 1 at its length: 500-atom LJ argon, NVE velocity Verlet, 1000
    steps of dt 0.005, engine against the oracle.  The two sum the pair forces
    in different orders, so the trajectories drift apart at the rate of the
    system's chaos from last-bit differences; energies stay within 1e-7 and
    both conserve e_tot."""
    s = systems.lj_argon()
    te0, to0, re, ro = run_both(s, 1000)
    e = np.array([t["e_tot"] for t in re["thermo"]])
    o = np.array([t["e_tot"] for t in ro["thermo"]])
    assert np.abs(e - o).max() < 1e-7 * np.abs(o).max()
    assert np.abs(e - te0["e_tot"]).max() < 2e-3 * abs(te0["e_tot"])
    assert sum(t["nlist_rebuilt"] for t in re["thermo"]) > 10


def test_config3_pim_3000_ions_nve_200_steps():
    """Config 3's cell (3000 ions, 10 x 10 x 30 sites, rc 10, alpha 0.3,
    kmax 10^3): 200 NVE steps of the mixed path tracking the FP64 path's
    energy, with the EFG of every step."""
    s = systems.mgo_pim()
    res = {}
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        p = s["params"]
        p.precision = prec
        p.kspace_reuse = 1
        p.algo_ext_dipole = abi.EXT_ASPC
        p.extrapolate_order = 3
        e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
        t0 = e.md_start(s["vel"])
        out = e.step(200)
        res[prec] = (t0, np.array([t["e_tot"] for t in out["thermo"]]), out)
    (t0, ed, od), (_, em, om) = res[abi.PREC_FP64], res[abi.PREC_MIXED]
    assert np.abs(em - ed).max() < 1e-6 * abs(t0["e_tot"])
    assert np.abs(ed - t0["e_tot"]).max() < 1e-3 * abs(t0["e_tot"])
