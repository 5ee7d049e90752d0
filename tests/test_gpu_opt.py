"""Structure optimisation on the device (mdff_opt_sastry: the reference's
sastry conjugate-gradient minimiser over the engine's force evaluations)
against the oracle's restatement, from jittered LJ and polarisable-ion MgO
starts.  Both follow the same scalar control flow; their dot products are
summed in different orders, so the line searches can take slightly
different paths near the end -- the minima must agree, not the step counts."""
import numpy as np
import pytest

import mdff_b200
import oracle
from mdff_b200 import abi, systems

pytestmark = pytest.mark.gpu


def _min_image(d, cell):
    inv = np.linalg.inv(cell)
    f = d @ inv.T
    f -= np.rint(f)
    return f @ cell.T


def test_lj_minimum_matches_oracle_and_lattice():
    s = systems.lj_argon()
    perfect = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"]).engforce()["e"]["u_lj"]
    rng = np.random.default_rng(3)
    pos = s["pos"] + rng.normal(0, 0.08, s["pos"].shape)
    e = mdff_b200.Engine(s["params"], s["itype"], pos, s["cell"])
    o = oracle.Oracle(s["params"], s["itype"], pos, s["cell"])
    re, ro = e.opt_sastry(), o.opt_sastry()
    assert re["status"] == 0 and ro["status"] == 0
    assert abs(re["u_initial"] - ro["u_initial"]) < 1e-12 * abs(ro["u_initial"])
    assert abs(re["u_final"] - ro["u_final"]) < 1e-11 * abs(ro["u_final"])
    assert abs(re["u_final"] - perfect) < 1e-11 * abs(perfect)
    d = _min_image(e.positions() - o.positions(), np.asarray(s["cell"]))
    assert np.abs(d).max() < 1e-5
    assert abs(re["iterations"] - ro["iterations"]) <= 5


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_pim_minimum_matches_oracle(prec):
    s = systems.mgo_pim(grid=(6, 6, 6), rc=6.0, alpha=0.55, kmax=8, temp=1000.0, jitter=0.1, seed=5)
    p = s["params"]
    p.algo_moment_from_pola = abi.POLA_PCG
    p.conv_tol_ind = 1e-10
    o = oracle.Oracle(p, s["itype"], s["pos"], s["cell"])
    ro = o.opt_sastry()
    p.precision = prec
    e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    re = e.opt_sastry()
    assert ro["status"] == 0 and re["status"] in (0, 3)
    tol = 1e-10 if prec == abi.PREC_FP64 else 1e-7
    assert abs(re["u_initial"] - ro["u_initial"]) < tol * abs(ro["u_initial"])
    assert abs(re["u_final"] - ro["u_final"]) < tol * abs(ro["u_final"])
    d = _min_image(e.positions() - o.positions(), np.asarray(s["cell"]))
    assert np.abs(d).max() < (1e-5 if prec == abi.PREC_FP64 else 1e-3)
    f = e.engforce()["f"]
    assert np.abs(f).max() < 1e-3


def test_lbfgs_lj_matches_oracle():
    # mdff_opt_lbfgs (device vectors, two-loop recursion with device-side
    # coefficients) against the oracle's reverse-communication restatement of
    # lbfgs_driver/LBFGS/MCSRCH: the same evaluations up to rounding of the
    # dot products, the same minimum
    s = systems.lj_argon()
    perfect = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"]).engforce()["e"]["u_lj"]
    pos = s["pos"] + np.random.default_rng(3).normal(0, 0.08, s["pos"].shape)
    e = mdff_b200.Engine(s["params"], s["itype"], pos, s["cell"])
    o = oracle.Oracle(s["params"], s["itype"], pos, s["cell"])
    re, ro = e.opt_lbfgs(), o.opt_lbfgs()
    assert re["status"] == ro["status"] == 0
    assert abs(re["u_initial"] - ro["u_initial"]) < 1e-12 * abs(ro["u_initial"])
    assert abs(re["u_final"] - ro["u_final"]) < 1e-11 * abs(ro["u_final"])
    assert abs(re["u_final"] - perfect) < 1e-10 * abs(perfect)
    assert abs(re["nforce"] - ro["nforce"]) <= 2 and abs(re["iterations"] - ro["iterations"]) <= 2
    d = _min_image(e.positions() - o.positions(), np.asarray(s["cell"]))
    assert np.abs(d).max() < 1e-5
    # the evaluation budget: itmax force evaluations, then status 1
    e2 = mdff_b200.Engine(s["params"], s["itype"], pos, s["cell"])
    r7, o7 = e2.opt_lbfgs(itmax=7), oracle.Oracle(s["params"], s["itype"], pos, s["cell"]).opt_lbfgs(itmax=7)
    assert r7["status"] == o7["status"] == 1 and r7["nforce"] == o7["nforce"] == 7
    assert abs(r7["u_final"] - o7["u_final"]) < 1e-10 * abs(o7["u_final"])


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_lbfgs_pim_minimum_matches_oracle(prec):
    s = systems.mgo_pim(grid=(6, 6, 6), rc=6.0, alpha=0.55, kmax=8, temp=1000.0, jitter=0.1, seed=5)
    p = s["params"]
    p.algo_moment_from_pola = abi.POLA_PCG
    p.conv_tol_ind = 1e-10
    ro = oracle.Oracle(p, s["itype"], s["pos"], s["cell"]).opt_lbfgs()
    p.precision = prec
    e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    re = e.opt_lbfgs()
    assert ro["status"] == 0 and re["status"] == 0
    tol = 1e-10 if prec == abi.PREC_FP64 else 1e-7
    assert abs(re["u_initial"] - ro["u_initial"]) < tol * abs(ro["u_initial"])
    assert abs(re["u_final"] - ro["u_final"]) < max(tol, 1e-9) * abs(ro["u_final"])
    # the termination test |G| / max(1, |X|) <= epsrel_lbfgs holds at the
    # returned point with the oracle's FP64 forces too
    o = oracle.Oracle(p, s["itype"], e.positions(), s["cell"])
    f = o.engforce()["f"]
    assert np.sqrt(np.sum(f * f)) / max(1.0, np.sqrt(np.sum(e.positions() ** 2))) <= 1e-5 * (1.0 + 10 * tol)
