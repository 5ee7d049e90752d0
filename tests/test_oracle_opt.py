"""The oracle's structure optimisation (sastry, src/opt.f90:452-849): from a
jittered LJ FCC crystal the conjugate-gradient minimiser must return to the
perfect lattice (its energy is the known minimum), stop on the reference's
energy test and leave the forces at zero."""
import numpy as np

import oracle
from mdff_b200 import systems


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
