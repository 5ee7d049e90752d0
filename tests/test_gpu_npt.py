"""Constant pressure on the GPU (MDFF_NPT_NHCNP) against the oracle's
restatement of nhcnp (with its corrections D14-D17), and mdff_set_cell: the
cell-dependent state (lattice, tail corrections, Ewald k tables) of a moved
cell must give the forces of a system built at that cell.

Tolerances as the NVT trajectory tests: FP64 energies 1e-9 relative per
step, positions 1e-9 global relative; the mixed path within its force
tolerance (1e-6) of the FP64 path.
"""
import numpy as np
import pytest

import mdff_b200
import oracle
from mdff_b200 import abi, systems

from helpers import rel

pytestmark = pytest.mark.gpu


def npt(s, press, tb=0.5):
    p = s["params"]
    p.integrator = abi.NPT_NHCNP
    p.nhc_n = 3
    p.timesca_baro = tb
    p.press = press
    return s


def lj():
    s = systems.lj_argon(ncell=4, temp=1.2)
    s["params"].temp = 1.2
    s["params"].timesca_thermo = 0.5
    return npt(s, 3.0, tb=1.0)


def pim(precision=abi.PREC_FP64):
    s = systems.mgo_pim(grid=(8, 8, 8), rc=6.0, alpha=0.5, kmax=8, temp=1500.0, integrator=abi.NVT_NHCN, seed=2)
    p = s["params"]
    p.precision = precision
    p.timesca_thermo = 0.05
    p.conv_tol_ind = 1e-10
    p.max_scf_pol_iter = 300
    return npt(s, 5.0, tb=0.2)


def both(s, nsteps):
    p = s["params"]
    e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    o = oracle.Oracle(p, s["itype"], s["pos"], s["cell"])
    te0, to0 = e.md_start(s["vel"]), o.md_start(s["vel"])
    return (te0, e.step(nsteps)), (to0, o.step(nsteps))


def test_lj_npt_matches_oracle():
    s = lj()
    (te0, re), (to0, ro) = both(s, 200)
    assert abs(te0["h_tot"] - to0["h_tot"]) < 1e-12 * abs(to0["h_tot"])
    for a, b in zip(re["thermo"], ro["thermo"]):
        assert abs(a["h_tot"] - b["h_tot"]) < 1e-9 * abs(b["h_tot"])
        assert abs(a["volume"] - b["volume"]) < 1e-9 * b["volume"]
        assert abs(a["e_nvt"] - b["e_nvt"]) < 1e-9 * max(1.0, abs(b["e_nvt"]))
    assert rel(re["pos"], ro["pos"]) < 1e-9
    vols = [t["volume"] for t in re["thermo"]]
    assert np.ptp(vols) > 0.01 * np.mean(vols)
    h = [t["h_tot"] for t in re["thermo"]]
    assert np.ptp(h) < 0.02 * np.std([t["e_kin"] for t in re["thermo"]])


def test_pim_npt_ewald_matches_oracle():
    # the cell moves every step: the k tables refreshed on the device must be
    # the ones the oracle recomputes from its new cell
    s = pim()
    (te0, re), (to0, ro) = both(s, 10)
    for a, b in zip(re["thermo"], ro["thermo"]):
        assert abs(a["volume"] - b["volume"]) < 1e-10 * b["volume"]
        assert abs(a["u_coul"] - b["u_coul"]) < 1e-9 * abs(b["u_coul"])
        assert abs(a["h_tot"] - b["h_tot"]) < 1e-9 * abs(b["h_tot"])
    assert abs(re["thermo"][-1]["volume"] / te0["volume"] - 1.0) > 1e-5
    assert rel(re["f"], ro["f"]) < 1e-8


def test_pim_npt_mixed_tracks_fp64():
    sm, sd = pim(abi.PREC_MIXED), pim(abi.PREC_FP64)
    em = mdff_b200.Engine(sm["params"], sm["itype"], sm["pos"], sm["cell"])
    ed = mdff_b200.Engine(sd["params"], sd["itype"], sd["pos"], sd["cell"])
    em.md_start(sm["vel"])
    ed.md_start(sd["vel"])
    rm, rd = em.step(6), ed.step(6)
    assert rel(rm["f"], rd["f"]) < 1e-6
    assert abs(rm["thermo"][-1]["volume"] / rd["thermo"][-1]["volume"] - 1.0) < 1e-9


@pytest.mark.parametrize("mixed", [False, True])
def test_set_cell_gives_the_forces_of_that_cell(mixed):
    s = pim(abi.PREC_MIXED if mixed else abi.PREC_FP64)
    p = s["params"]
    p.integrator = abi.NVE_VV
    e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    g = 1.012
    cell2 = np.asarray(s["cell"]) * g
    pos2 = np.asarray(s["pos"]) * g
    e.set_cell(cell2)
    e.set_positions(pos2)
    got = e.engforce()
    o = oracle.Oracle(p, s["itype"], pos2, cell2)
    ref = o.engforce()
    tol = 1e-6 if mixed else 1e-10
    assert rel(got["f"], ref["f"]) < tol
    assert abs(got["e"]["u_coul"] - ref["e"]["u_coul"]) < tol * abs(ref["e"]["u_coul"])
    assert rel(got["tau_coul"], ref["tau_coul"]) < (1e-6 if mixed else 1e-9)


@pytest.mark.parametrize("case", ["lj", "pim_mixed"])
def test_npt_checkpoint_restart_is_bit_identical(case):
    s = lj() if case == "lj" else pim(abi.PREC_MIXED)
    n1, n2 = (25, 25) if case == "lj" else (5, 5)

    def fresh():
        return mdff_b200.Engine(s["params"], s["itype"], s["pos"], s["cell"])

    a = fresh()
    a.md_start(s["vel"])
    a.step(n1, thermo=False)
    ra, va = a.step(n2), a.velocities()
    b = fresh()
    b.md_start(s["vel"])
    b.step(n1, thermo=False)
    ck = b.checkpoint()
    b.close()
    c = fresh()
    c.restore(ck)
    rc, vc = c.step(n2), c.velocities()
    assert np.array_equal(ra["pos"], rc["pos"])
    assert np.array_equal(va, vc)
    assert ra["thermo"] == rc["thermo"]
