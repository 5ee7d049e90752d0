"""Verlet lists built on the GPU equal the reference's lists bit for bit.

The reference stores half lists with the parity ownership rule and ascending
j (vnlist_pbc, src/tools.f90:274-370); mdff_nlist_get returns that layout.
The oracle restates vnlist_pbc's all-pairs loop with the same FP64 operation
order; the engine bins atoms into cells and tests candidates with the same
expression.  point[] and list[] must be identical arrays.
"""
import numpy as np
import pytest

import mdff_b200
import oracle
from mdff_b200 import abi, systems

pytestmark = pytest.mark.gpu


def compare_lists(p, itype, pos, cell, whiches=(0,)):
    e = mdff_b200.Engine(p, itype, pos, cell)
    o = oracle.Oracle(p, itype, pos, cell)
    for w in whiches:
        pe, le = e.nlist(w)
        po, lo = o.nlist(w)
        assert np.array_equal(pe, po), f"point differs (list {w})"
        assert np.array_equal(le, lo), f"list differs (list {w})"
    return e, o


def test_lj_fcc():
    s = systems.lj_argon()
    compare_lists(s["params"], s["itype"], s["pos"], s["cell"])


def test_silica_both_lists():
    s = systems.silica_bmh()
    p = s["params"]
    p.cutlongrange = 7.0    # different cutoffs: two lists from one pass
    compare_lists(p, s["itype"], s["pos"], s["cell"], whiches=(0, 1))


def test_pim_thin_box_fewer_than_three_cells():
    # 21.06 x 21.06 x 63.18 A box with a 10.15 A list radius: two cells across x and y
    s = systems.mgo_pim()
    compare_lists(s["params"], s["itype"], s["pos"], s["cell"], whiches=(0, 1))


def test_triclinic_cell():
    rng = np.random.default_rng(5)
    cell = np.array([[14.0, 0.0, 0.0], [3.1, 13.2, 0.0], [-2.2, 1.7, 12.5]])
    n = 700
    frac = rng.random((n, 3))
    pos = frac @ cell
    p = abi.default_params()
    p.lnmlj = 1
    p.cutshortrange = 3.9
    p.epslj[0][0] = 0.01
    p.sigmalj[0][0] = 2.0
    compare_lists(p, np.ones(n, np.int32), pos, cell)


@pytest.mark.parametrize("n", [2, 3, 7])
def test_ragged_tiny_systems(n):
    rng = np.random.default_rng(n)
    pos = rng.random((n, 3)) * 6.0
    p = abi.default_params()
    p.lnmlj = 1
    p.cutshortrange = 2.9
    p.epslj[0][0] = 0.01
    p.sigmalj[0][0] = 1.0
    compare_lists(p, np.ones(n, np.int32), pos, np.eye(3) * 6.0)


def test_cutoff_beyond_half_box():
    # ex2-style: cutoff larger than half the box, every pair within one image
    rng = np.random.default_rng(3)
    pos = rng.normal(0.0, 1.0, (40, 3))
    p = abi.default_params()
    p.lnmlj = 1
    p.cutshortrange = 100.0
    p.epslj[0][0] = 1.0
    p.sigmalj[0][0] = 1.0
    compare_lists(p, np.ones(40, np.int32), pos, np.eye(3) * 100.0)


def test_pairs_on_the_boundary():
    # atoms placed exactly at the list radius along axes and diagonals
    L = 20.0
    rl = 4.0 + 0.15
    pos = [[1.0, 1.0, 1.0], [1.0 + rl, 1.0, 1.0], [1.0, 1.0 + rl, 1.0], [1.0, 1.0, 1.0 + rl],
           [1.0 + rl / np.sqrt(3)] * 3, [1.0 - rl, 1.0, 1.0], [1.0 + rl * (1 + 1e-16), 5.0, 5.0]]
    pos = np.array(pos)
    p = abi.default_params()
    p.lnmlj = 1
    p.cutshortrange = 4.0
    p.epslj[0][0] = 0.01
    p.sigmalj[0][0] = 1.0
    compare_lists(p, np.ones(len(pos), np.int32), pos, np.eye(3) * L)


def test_rebuild_after_motion_matches():
    s = systems.lj_argon()
    p = s["params"]
    e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    rng = np.random.default_rng(0)
    moved = e.positions() + rng.normal(0.0, 0.4, (len(s["pos"]), 3))   # unwrapped, some leave the box
    e.set_positions(moved)
    e.nlist_build()
    o = oracle.Oracle(p, s["itype"], s["pos"], s["cell"])
    o.set_positions(moved)
    o.nlist_build()
    pe, le = e.nlist(0)
    po, lo = o.nlist(0)
    assert np.array_equal(pe, po) and np.array_equal(le, lo)
