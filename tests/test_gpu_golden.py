"""The engine against the reference's own golden data, through the C ABI:
the ex4 cluster's Ewald EFG and its NMR principal values (mdff_efg_nmr)
against the GULP table of examples/ex4/run_ex4.sh:159-170, and the ex0 FCC
argon static LJ energy, virial and tail corrections against DL_POLY
(examples/ex0/dl_poly).  Fixtures: tests/golden/ex4_cluster.npz and
ex0_fcc.npz (tests/golden/make_fixtures.py)."""
import numpy as np
import pytest

import mdff_b200
import oracle
from mdff_b200 import abi

from helpers import EX4_TOL_ETA, EX4_TOL_V, check_ex0, ex0_fcc_case, ex4_cluster_case, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_ex4_cluster_efg_vs_gulp(prec):
    p, itype, pos, cell, gulp = ex4_cluster_case()
    p.precision = prec
    e = mdff_b200.Engine(p, itype, pos, cell)
    r = e.engforce()
    efg = -r["efg"]   # lefg_vasp_sign (src/efg.f90:486-488)
    nmr = e.efg_nmr(efg)[0]
    assert np.abs(nmr[:, :3] - gulp[:, :3]).max() < EX4_TOL_V
    assert np.abs(nmr[:, 3] - gulp[:, 3]).max() < EX4_TOL_ETA
    if prec == abi.PREC_FP64:
        o = oracle.Oracle(p, itype, pos, cell)
        assert rel(r["efg"], o.engforce()["efg"]) < 1e-10


def test_ex0_dl_poly_static_lj():
    p, itype, pos, cell, d = ex0_fcc_case()
    e = mdff_b200.Engine(p, itype, pos, cell)
    check_ex0(e.engforce()["e"], abs(np.linalg.det(cell)), d)
