"""Pin the CPU oracle against the reference's own outputs and known answers.

ex1 (examples/ex1/ref): LJ argon final configuration, forces, energy,
virial pressure and stress from the reference's 2014 run (fixture made by
tests/golden/make_fixtures.py).  ex2 (examples/ex2): Lennard-Jones cluster
energies against the Cambridge Cluster Database values the reference ships,
read in place when the reference tree is present.  ex4
(examples/ex4/run_ex4.sh:78-79): electric field gradient of two opposite
unit charges in a 10 A box (Nymand & Linse values printed by the reference's
example script), and the 9-ion cluster against the GULP table the same script
prints (run_ex4.sh:159-170).  ex0 (examples/ex0/dl_poly): DL_POLY's static
energy, virial and long-range corrections of the 256-atom FCC argon
configuration.  The ex4 cluster and ex0 fixtures are made by
tests/golden/make_fixtures.py.
"""
import os

import numpy as np
import pytest

import oracle
from mdff_b200 import abi

from conftest import REFERENCE, has_reference
from helpers import EX4_TOL_ETA, EX4_TOL_V, check_ex0, ex0_fcc_case, ex4_cluster_case, lj_params_ex1, rel
from oracle import efg_stat


def test_ex1_lj_forces_energy_stress():
    p, d = lj_params_ex1()
    n = len(d["pos"])
    o = oracle.Oracle(p, np.ones(n, np.int32), d["pos"], d["cell"])
    r = o.engforce()
    # energy: OSZIFF prints 8 significant digits
    assert abs(r["e"]["u_lj"] - float(d["u_lj"])) < 5e-6
    # forces: CONTFF prints 12 significant digits
    assert np.abs(r["f"] - d["force"]).max() < 1e-9
    assert rel(r["f"], d["force"]) < 1e-9
    # virial pressure (Pvir_vdw, GPa) = vir / V / press_unit
    pvir = r["e"]["vir_lj"] / abs(np.linalg.det(d["cell"])) / 0.00624150964712042
    assert abs(pvir - float(d["pvir_gpa"])) < 1e-8
    # stress: the 2014 build printed twice the current source's tau_nonb
    assert np.abs(2.0 * r["tau_nonb"] - d["tau_nonb_printed"]).max() < 1e-7


def test_ex1_tail_correction():
    # examples/ex1/ref/stdout:79 prints the long-range correction -1.42129648126362
    # (same potential and cutoff, 256 atoms in the 21.62 A box)
    p, d = lj_params_ex1()
    n = len(d["pos"])
    o = oracle.Oracle(p, np.ones(n, np.int32), d["pos"], d["cell"])
    e = o.engforce()["e"]
    assert abs(e["utail"] - (-1.42129648126362)) < 1e-11


@pytest.mark.skipif(not has_reference(), reason="reference tree not present")
@pytest.mark.parametrize("name", ["3", "5", "13", "26", "38", "55", "75", "100", "147", "38i", "104i"])
def test_ex2_cluster_energies(name):
    refs = {}
    for line in open(os.path.join(REFERENCE, "examples", "ex2", "REFERENCE")):
        t = line.split()
        if len(t) == 2 and not line.startswith("#"):
            refs[t[0]] = float(t[1])
    xyz = np.loadtxt(os.path.join(REFERENCE, "examples", "ex2", "clusters", name))
    p = abi.default_params()
    p.lnmlj = 1
    p.cutshortrange = 100.0
    p.trunc = abi.TRUNC_LINEAR
    p.epslj[0][0] = 1.0
    p.sigmalj[0][0] = 1.0
    o = oracle.Oracle(p, np.ones(len(xyz), np.int32), xyz, np.eye(3) * 100.0)
    u = o.engforce()["e"]["u_lj"]
    assert abs(u - refs[name]) < 2e-6   # REFERENCE prints 6 decimals


def two_charges_params():
    p = abi.default_params()
    p.ntype = 2
    p.lcoulomb = 1
    p.lreduced = 1
    p.cutlongrange = 1000.0
    p.qch[0] = 1.0
    p.qch[1] = -1.0
    p.alphaES = 0.8
    p.kES[0] = p.kES[1] = p.kES[2] = 11
    p.doefg = 1
    return p


@pytest.mark.parametrize("erfc_mode", [0, 1])
def test_ex4_two_charges_efg(erfc_mode):
    p = two_charges_params()
    o = oracle.Oracle(p, np.array([1, 2], np.int32), np.array([[0.5, 0, 0], [-0.5, 0, 0]]), np.eye(3) * 10.0,
                      erfc_mode=erfc_mode)
    info = o.ewald_info()
    assert info["cutlongrange"] == 5.0          # clamped to half the box width (field.f90:875-881)
    assert info["nk"] == 11 + 11 * 23 + 11 * 23 * 23
    efg = o.engforce()["efg"]
    assert abs(efg[0, 0] - 2.0003749) < 1e-7
    assert abs(efg[0, 1] - (-1.0001874)) < 1e-7
    assert abs(efg[0, 2] - (-1.0001874)) < 1e-7
    # the field gradient is traceless
    assert abs(efg[0, 0] + efg[0, 1] + efg[0, 2]) < 1e-9


def test_errfc_matches_reference_fit_accuracy():
    from math import erfc
    xs = np.linspace(0.0, 5.0, 501)
    err = max(abs(oracle.errfc(x) - erfc(x)) / erfc(x) for x in xs)
    assert err < 1.3e-7   # the fit's documented relative accuracy
    assert abs(oracle.errfc(-1.0) - (2.0 - oracle.errfc(1.0))) < 1e-15


def test_ex4_cluster_efg_vs_gulp():
    """Ewald EFG of the ex4 cluster (point charges 0.1 / -0.8, lautoES at
    epsw 1e-8, lefg_vasp_sign), principal values in the NMR convention,
    against GULP's diagonalised EFGs and asymmetries."""
    p, itype, pos, cell, gulp = ex4_cluster_case()
    o = oracle.Oracle(p, itype, pos, cell)
    efg = -o.engforce()["efg"]   # lefg_vasp_sign (src/efg.f90:486-488)
    nmr = efg_stat.efg_nmr(efg)[0]
    assert np.abs(nmr[:, :3] - gulp[:, :3]).max() < EX4_TOL_V
    assert np.abs(nmr[:, 3] - gulp[:, 3]).max() < EX4_TOL_ETA


def test_ex0_dl_poly_static_lj():
    p, itype, pos, cell, d = ex0_fcc_case()
    o = oracle.Oracle(p, itype, pos, cell)
    check_ex0(o.engforce()["e"], abs(np.linalg.det(cell)), d)
