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

