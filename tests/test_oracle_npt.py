"""Constant-pressure MD in the oracle (nhcnp, src/integration.f90:715-1160,
with the corrections D14-D17 of the oracle's header), on LJ argon in reduced
units: the reference's conserved quantity e_tot + e_npt holds, the barostat
brings the internal pressure (1 + 3/Nf) 2K/3V + pvirial to its target, and
with an infinitely heavy barostat the run is the NVT chain's run.
"""
import numpy as np

import oracle
from mdff_b200 import abi, systems


def npt_lj(press=3.0, tb=1.0, ncell=3):
    s = systems.lj_argon(ncell=ncell, temp=1.2)
    p = s["params"]
    p.integrator = abi.NPT_NHCNP
    p.nhc_n = 3
    p.temp = 1.2
    p.timesca_thermo = 0.5
    p.timesca_baro = tb
    p.press = press
    return s


def run(s, nsteps):
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    t0 = o.md_start(s["vel"])
    return t0, o.step(nsteps)


def test_extended_energy_is_conserved():
    s = npt_lj()
    t0, r = run(s, 400)
    h = np.array([t0["h_tot"]] + [t["h_tot"] for t in r["thermo"]])
    ek = np.array([t["e_kin"] for t in r["thermo"]])
    V = np.array([t["volume"] for t in r["thermo"]])
    assert np.ptp(V) > 0.05 * V.mean()              # the cell really moves
    assert np.ptp(h) < 0.02 * ek.std()               # conserved to 2 % of the kinetic fluctuation


def test_barostat_reaches_the_target_pressure():
    press = 3.0
    s = npt_lj(press=press)
    t0, r = run(s, 2500)
    n = len(s["itype"])
    th = r["thermo"][500:]
    V = np.array([t["volume"] for t in th])
    ek = np.array([t["e_kin"] for t in th]) * n       # reduced output divides by natm
    pv = np.array([t["pvirial_tot"] for t in th]) * n
    p_int = (1.0 + 1.0 / n) * 2.0 * ek / (3.0 * V) + pv
    err = p_int.std() / np.sqrt(len(p_int) / 50.0)   # correlated samples: ~50 steps apart
    assert abs(p_int.mean() - press) < 4.0 * err + 0.05


def test_infinitely_heavy_barostat_is_nvt():
    s = npt_lj(tb=1e7)
    _, r = run(s, 150)
    s2 = npt_lj()
    p2 = s2["params"]
    p2.integrator = abi.NVT_NHCN
    _, r2 = run(s2, 150)
    assert abs(r["thermo"][-1]["volume"] / r2["thermo"][-1]["volume"] - 1.0) < 1e-12
    assert np.max(np.abs(r["pos"] - r2["pos"])) < 1e-9
