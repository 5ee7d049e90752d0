"""The oracle's structure optimisation, the three optalgo of opt_main: sastry
(src/opt.f90:452-849), lbfgs (lbfgs_driver :972-1194 over src/lbfgs.f90) and
m1qn3 (m1qn3_driver :1203-1330 over src/m1qn3.f90).  From a jittered LJ FCC
crystal each minimiser must return to the perfect lattice (its energy is the
known minimum), stop on the reference's own test and report its exits as the
reference does."""
import numpy as np

import oracle
from mdff_b200 import abi, systems


def test_lj_crystal_relaxes_to_the_lattice():
    s = systems.lj_argon()
    perfect = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"]).engforce()["e"]["u_lj"]
    rng = np.random.default_rng(3)
    o = oracle.Oracle(s["params"], s["itype"], s["pos"] + rng.normal(0, 0.08, s["pos"].shape), s["cell"])
    r = o.opt_sastry()
    assert r["status"] == 0
    assert r["u_initial"] > perfect + 100.0
    assert abs(r["u_final"] - perfect) < 1e-11 * abs(perfect)
    assert np.abs(o.engforce()["f"]).max() < 1e-4
    assert r["nforce"] > 2 * r["iterations"]


def _jittered_lj():
    s = systems.lj_argon()
    perfect = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"]).engforce()["e"]["u_lj"]
    pos = s["pos"] + np.random.default_rng(3).normal(0, 0.08, s["pos"].shape)
    return s, pos, perfect


def test_lbfgs_relaxes_to_the_lattice():
    # optalgo = 'lbfgs' (lbfgs_driver, src/opt.f90:972-1194) with the default
    # epsrel_lbfgs = 1e-5: the same minimum as sastry, in far fewer
    # force evaluations
    s, pos, perfect = _jittered_lj()
    o = oracle.Oracle(s["params"], s["itype"], pos, s["cell"])
    r = o.opt_lbfgs()
    assert r["status"] == 0 and r["info"] == 0
    assert abs(r["u_final"] - perfect) < 1e-10 * abs(perfect)
    f = o.engforce()["f"]
    gnorm = np.sqrt(np.sum(f * f))
    xnorm = max(1.0, np.sqrt(np.sum(o.positions() ** 2)))
    assert gnorm / xnorm <= 1e-5                      # the LBFGS termination test
    cg = oracle.Oracle(s["params"], s["itype"], pos, s["cell"]).opt_sastry()
    assert r["nforce"] < cg["nforce"] / 3
    assert r["nforce"] >= r["iterations"] + 1


def test_lbfgs_evaluation_budget_and_line_search_exit():
    s, pos, _ = _jittered_lj()
    o = oracle.Oracle(s["params"], s["itype"], pos, s["cell"])
    r = o.opt_lbfgs(itmax=7)
    assert r["status"] == 1 and r["nforce"] == 7
    assert r["u_final"] < r["u_initial"]
    # a tolerance below what rounding allows ends in MCSRCH's rounding exit
    # (info 6) or its interval test (info 2), as the reference reports it
    r = oracle.Oracle(s["params"], s["itype"], pos, s["cell"]).opt_lbfgs(eps=1e-14)
    assert r["status"] == 3 and r["info"] in (2, 6)


def test_m1qn3_relaxes_to_the_lattice():
    # optalgo = 'm1qn3' (m1qn3_driver, src/opt.f90:1203-1330): DIS mode,
    # m = 5, stop when |G| / |G_0| < epsrel_m1qn3; the driver evaluates once
    # more at the returned point, so phigrad is |G|^2 there
    s, pos, perfect = _jittered_lj()
    o = oracle.Oracle(s["params"], s["itype"], pos, s["cell"])
    g0 = np.sqrt(np.sum(o.engforce()["f"] ** 2))
    r = o.opt_m1qn3()
    assert r["status"] == 0 and r["info"] == 1
    assert np.sqrt(r["phigrad"]) / g0 < abi.EPSREL_OPT
    assert abs(r["u_final"] - perfect) < 1e-9 * abs(perfect)
    f = o.engforce()
    assert abs(f["e"]["u_lj"] - r["u_final"]) < 1e-12 * abs(perfect)
    cg = oracle.Oracle(s["params"], s["itype"], pos, s["cell"]).opt_sastry()
    assert r["nforce"] < cg["nforce"] / 3


def test_m1qn3_iteration_cap_and_rounding_exit():
    s, pos, _ = _jittered_lj()
    r = oracle.Oracle(s["params"], s["itype"], pos, s["cell"]).opt_m1qn3(niter=4)
    assert r["status"] == 1 and r["info"] == 4 and r["iterations"] == 4
    assert r["u_final"] < r["u_initial"]
    # below what rounding allows: mlis3's dxmin/precision exit, omode 6,
    # which the reference's driver accepts with a warning
    r = oracle.Oracle(s["params"], s["itype"], pos, s["cell"]).opt_m1qn3(epsg=1e-13)
    assert r["status"] == 3 and r["info"] == 6
    # epsg >= 1: no progress asked for, only the driver's evaluations
    r = oracle.Oracle(s["params"], s["itype"], pos, s["cell"]).opt_m1qn3(epsg=1.0)
    assert r["status"] == 0 and r["iterations"] == 0 and r["nforce"] == 2
    assert r["u_final"] == r["u_initial"]
