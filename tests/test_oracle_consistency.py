"""Internal-consistency checks of the CPU oracle where the reference ships no
golden data (BMHFTD, Tang-Toennies damping, dipole Ewald, induced dipoles,
Nose-Hoover chain): forces are minus the energy gradient, the total force
vanishes, the Ewald total does not depend on alpha, the SCF and PCG solves
agree, translations change nothing, the conserved quantities are conserved.
"""
import numpy as np
import pytest

import oracle
from mdff_b200 import abi, systems

from helpers import rel


def small_pim(**kw):
    s = systems.mgo_pim(grid=(6, 6, 6), rc=6.0, alpha=0.55, kmax=8, **kw)
    s["params"].conv_tol_ind = 1e-11
    return s


def total_u(r):
    e = r["e"]
    return e["u_lj"] + e["u_bmhft"] + e["u_morse"] + e["u_coul"]


def test_tt_damping_derivative():
    for order in (4, 6, 8):
        for r in (0.5, 1.7, 3.0):
            h = 1e-6
            f, fd = oracle.tt_damp(1.8, 1.3, r, order)
            fp, _ = oracle.tt_damp(1.8, 1.3, r + h, order)
            fm, _ = oracle.tt_damp(1.8, 1.3, r - h, order)
            assert abs((fp - fm) / (2 * h) - fd) < 1e-8


@pytest.mark.parametrize("algo", [abi.POLA_SCF, abi.POLA_PCG])
def test_pim_forces_are_energy_gradient(algo):
    s = small_pim()
    p = s["params"]
    p.algo_moment_from_pola = algo
    p.max_scf_pol_iter = 500
    o = oracle.Oracle(p, s["itype"], s["pos"], s["cell"])
    pos0 = o.positions()
    r0 = o.engforce()
    assert np.abs(r0["f"].sum(axis=0)).max() < 1e-9
    h = 1e-4
    for (i, c) in [(0, 0), (7, 1), (120, 2), (200, 0)]:
        pp = pos0.copy(); pp[i, c] += h
        o.set_positions(pp); up = total_u(o.engforce())
        pm = pos0.copy(); pm[i, c] -= h
        o.set_positions(pm); um = total_u(o.engforce())
        fd = -(up - um) / (2 * h)
        assert abs(fd - r0["f"][i, c]) < 2e-5 * max(1.0, abs(r0["f"][i, c]))


def test_scf_and_pcg_agree():
    s = small_pim()
    out = {}
    for algo in (abi.POLA_SCF, abi.POLA_PCG):
        p = s["params"]
        p.algo_moment_from_pola = algo
        p.max_scf_pol_iter = 500
        o = oracle.Oracle(p, s["itype"], s["pos"], s["cell"])
        out[algo] = o.engforce()
    a, b = out[abi.POLA_SCF], out[abi.POLA_PCG]
    assert rel(a["mu"], b["mu"]) < 1e-8
    assert rel(a["f"], b["f"]) < 1e-9
    assert abs(a["e"]["u_coul"] - b["e"]["u_coul"]) < 1e-8 * abs(b["e"]["u_coul"])


def test_ewald_alpha_independence_rigid_ions():
    s = systems.silica_bmh()
    res = []
    for alpha, kmax in ((0.42, 14), (0.46, 15), (0.50, 16)):
        p = s["params"]
        p.alphaES = alpha
        p.kES[0] = p.kES[1] = p.kES[2] = kmax
        p.lbmhft = 0
        o = oracle.Oracle(p, s["itype"], s["pos"], s["cell"])
        res.append(o.engforce())
    for r in res[1:]:
        assert abs(r["e"]["u_coul"] - res[0]["e"]["u_coul"]) < 1e-5 * abs(res[0]["e"]["u_coul"])
        assert rel(r["f"], res[0]["f"]) < 2e-4


def test_translation_invariance():
    s = small_pim()
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    r0 = o.engforce()
    o2 = oracle.Oracle(s["params"], s["itype"], s["pos"] + np.array([0.37, -1.1, 2.3]), s["cell"])
    r1 = o2.engforce()
    assert rel(r1["f"], r0["f"]) < 1e-9
    assert abs(total_u(r1) - total_u(r0)) < 1e-9 * abs(total_u(r0))


def test_virial_matches_stress_trace():
    s = systems.silica_bmh()
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    r = o.engforce()
    vol = abs(np.linalg.det(s["cell"]))
    press = 0.00624150964712042
    assert abs(np.trace(r["tau_nonb"]) / 3.0 - r["e"]["vir_bmhft"] / vol / press) < 1e-9 * abs(np.trace(r["tau_nonb"]))


def test_nve_energy_conservation_lj():
    s = systems.lj_argon(ncell=4)
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    t0 = o.md_start(s["vel"])
    out = o.step(200)
    e = np.array([t["e_tot"] for t in out["thermo"]])
    assert np.abs(e - t0["e_tot"]).max() < 2e-3 * abs(t0["e_tot"])


def test_nhc_conserved_quantity_lj():
    s = systems.lj_argon(ncell=4)
    p = s["params"]
    p.integrator = abi.NVT_NHCN
    p.nhc_n = 3
    p.temp = 1.2
    p.timesca_thermo = 0.5
    o = oracle.Oracle(p, s["itype"], s["pos"], s["cell"])
    t0 = o.md_start(s["vel"])
    out = o.step(300)
    h = np.array([t["h_tot"] for t in out["thermo"]])
    t = np.array([t["temp_r"] for t in out["thermo"]])
    assert np.abs(h - t0["h_tot"]).max() < 2e-3 * abs(t0["h_tot"])
    assert t[-100:].mean() > t[:100].mean() + 0.1   # the thermostat heats towards T* = 1.2


def test_nhc2_conserved_quantity_lj():
    """nhc2 / chain_nhc2 (src/integration.f90:205-324): with the thermostat
    energy Q vxi^2 / 2 + L T xi1 + T xi2 (D23) the extended energy holds; the
    reference's literal vxi^2 / (2 Q) does not; the chain heats towards T* = 1.2."""
    def run(literal):
        s = systems.lj_argon(ncell=4)
        p = s["params"]
        p.integrator = abi.NVT_NHC2
        p.nhc_n = 7          # ignored: nhc2 always has two thermostats
        p.temp = 1.2
        p.timesca_thermo = 0.5
        p.nhc_literal = literal
        o = oracle.Oracle(p, s["itype"], s["pos"], s["cell"])
        t0 = o.md_start(s["vel"])
        out = o.step(300)
        h = np.array([t["h_tot"] for t in out["thermo"]])
        t = np.array([t["temp_r"] for t in out["thermo"]])
        e = np.array([t["e_nvt"] for t in out["thermo"]])
        return t0, h, t, e
    t0, h, t, e = run(0)
    assert np.abs(h - t0["h_tot"]).max() < 2e-3 * abs(t0["h_tot"])
    assert t[-100:].mean() > t[:100].mean() + 0.05   # heating towards T* = 1.2
    assert np.abs(e).max() > 1e-2 * abs(t0["h_tot"])   # the thermostat does work
    _, hl, _, _ = run(1)
    assert np.abs(hl - t0["h_tot"]).max() > 10 * np.abs(h - t0["h_tot"]).max()


def test_nlist_matches_all_pairs_brute_force():
    s = systems.silica_bmh()
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    point, lst = o.nlist(0)
    pos = o.positions()
    L = s["cell"][0, 0]
    n = len(pos)
    rsk = (8.0 + 0.15) ** 2
    for i in (0, 17, 800, n - 1):
        row = sorted(lst[point[i] - 1:point[i + 1] - 1])
        want = []
        for j in range(n):
            I, J = i + 1, j + 1
            if (I > J and (I + J) % 2 == 0) or (I < J and (I + J) % 2 != 0):
                d = pos[i] - pos[j]
                d -= L * np.round(d / L)
                if d @ d <= rsk:
                    want.append(J)
        assert row == want
