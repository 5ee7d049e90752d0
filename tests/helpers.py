"""Shared helpers for the parity tests."""
import numpy as np

from mdff_b200 import abi


def rel(a, b):
    """Global relative difference ||a-b|| / ||b|| (the engine's error norm)."""
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def lj_params_ex1():
    d = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "ex1_final.npz"))
    p = abi.default_params()
    p.ntype = 1
    p.lnmlj = 1
    p.cutshortrange = float(d["cutshortrange"])
    p.trunc = abi.TRUNC_LINEAR
    p.epslj[0][0] = float(d["epslj"])
    p.sigmalj[0][0] = float(d["sigmalj"])
    p.mass[0] = float(d["mass"])
    return p, d


def copy_params(p):
    q = abi.Params()
    __import__("ctypes").pointer(q)[0] = p
    return q


def _golden(name):
    import os
    return np.load(os.path.join(os.path.dirname(__file__), "golden", name))


def ex4_cluster_case():
    """examples/ex4's cluster (9 ions in a 10 A box, qch 0.1 / -0.8) with the
    example's Ewald settings (cutlongrange 5, lautoES, epsw 1e-8) and GULP's
    table: params, itype, pos, cell, gulp [9][4] (Vxx Vyy Vzz eta)."""
    d = _golden("ex4_cluster.npz")
    p = abi.default_params()
    p.ntype = 2
    p.lcoulomb = 1
    p.cutlongrange = float(d["cutlongrange"])
    p.lautoES = 1
    p.epsw = float(d["epsw"])
    p.doefg = 1
    p.qch[0], p.qch[1] = (float(x) for x in d["qch"])
    return p, d["itype"].astype(np.int32), d["pos"], d["cell"], d["gulp"]


def ex0_fcc_case():
    """examples/ex0: 256-atom FCC argon, LJ 12-6 untruncated at rc 10 A, and
    DL_POLY's static energy, virial and long-range corrections for it."""
    d = _golden("ex0_fcc.npz")
    p = abi.default_params()
    p.ntype = 1
    p.lnmlj = 1
    p.cutshortrange = float(d["cutshortrange"])
    p.trunc = abi.TRUNC_NONE
    p.epslj[0][0] = float(d["epslj"])
    p.sigmalj[0][0] = float(d["sigmalj"])
    p.mass[0] = float(d["mass"])
    pos = d["frac"] @ d["cell"]
    return p, np.ones(len(pos), np.int32), pos, d["cell"], d


# GULP prints 4 decimals and uses its own Coulomb constant and Ewald
# convergence; the reference's restatement agrees with its table to 1.2e-5 of
# the largest |Vzz| (5.6e-4 V/A^2) and 1e-4 on eta
EX4_TOL_V = 1.0e-3    # V/A^2
EX4_TOL_ETA = 2.0e-4
KATM_TO_GPA = 0.101325
PRESS_UNIT = 0.00624150964712042   # eV/A^3 per GPa (src/constants.f90:85)


def check_ex0(e, volume, d):
    """DL_POLY's static LJ result (examples/ex0/dl_poly) from an engforce
    energy record: eng_vdw = u_lj + tail (DL_POLY tabulates its potential and
    prints 7 digits: 3e-6 relative); the tail corrections as printed (6
    digits); vir_vdw = -(sum r.f) - 3 V p_tail, DL_POLY's sign, to 1e-3 eV
    (2e-4 of the pair sum, DL_POLY's tabulated forces)."""
    assert abs(e["utail"] - float(d["elrc_ev"])) < 1e-6
    assert abs(e["ptail"] - float(d["plrc_katm"]) * KATM_TO_GPA) < 3e-6 * abs(e["ptail"])
    u = e["u_lj"] + e["utail"]
    assert abs(u - float(d["eng_vdw"])) < 3e-6 * abs(float(d["eng_vdw"])), u
    w = -3.0 * e["vir_lj"] - 3.0 * volume * e["ptail"] * PRESS_UNIT
    assert abs(w - float(d["vir_vdw"])) < 1e-3, w
