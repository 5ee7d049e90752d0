"""The mixed-precision path (FP32 reciprocal space with exact fixed-point
phases and FP64 accumulation; FP64 real space, solver, integrator) against
the FP64 path on identical inputs.

Error measure (global): eps_F = ||F_mixed - F_fp64||_2 / ||F_fp64||_2 over all
atoms and components; the same form for dipoles, EFG (6 components), field.
Bound: eps_F <= 1e-6 (the workload's force-error target); energies and
stress to 1e-6 relative (the reciprocal energy sum_k A_k |S(k)|^2 is summed in
FP64 but S(k) carries the FP32 terms' ~1e-7 error).
"""
import ctypes as C

import numpy as np
import pytest

import mdff_b200
from mdff_b200 import abi, systems

from helpers import rel

pytestmark = pytest.mark.gpu


def pair(s, **over):
    out = {}
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        p = s["params"]
        p.precision = prec
        for k, v in over.items():
            setattr(p, k, v)
        e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
        out[prec] = e.engforce()
    return out[abi.PREC_MIXED], out[abi.PREC_FP64]


def test_mixed_rigid_ions_silica():
    m, d = pair(systems.silica_bmh(), doefield=1)
    assert rel(m["f"], d["f"]) < 1e-6
    assert rel(m["ef"], d["ef"]) < 1e-6
    assert abs(m["e"]["u_coul"] - d["e"]["u_coul"]) < 1e-6 * abs(d["e"]["u_coul"])


def test_mixed_pim_production_model():
    s = systems.mgo_pim(grid=(16, 16, 16), rc=10.0, alpha=0.3, kmax=12, vacancy_frac=0.01, seed=3, jitter=0.1)
    m, d = pair(s, doefg=1, conv_tol_ind=1e-10)
    eps_f = rel(m["f"], d["f"])
    assert eps_f < 1e-6, eps_f
    assert rel(m["mu"], d["mu"]) < 1e-6
    assert rel(m["efg"], d["efg"]) < 1e-6
    assert abs(m["e"]["u_coul"] - d["e"]["u_coul"]) < 1e-6 * abs(d["e"]["u_coul"])
    assert rel(m["tau_coul"], d["tau_coul"]) < 1e-6


def test_mixed_md_energy_tracks_fp64():
    s = systems.mgo_pim(grid=(8, 8, 8), rc=8.0, alpha=0.4, kmax=9, temp=1500.0)
    res = {}
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        p = s["params"]
        p.precision = prec
        p.conv_tol_ind = 1e-10
        e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
        e.md_start(s["vel"])
        res[prec] = e.step(20)
    for a, b in zip(res[abi.PREC_MIXED]["thermo"], res[abi.PREC_FP64]["thermo"]):
        assert abs(a["e_tot"] - b["e_tot"]) < 1e-6 * abs(b["e_tot"])


def test_mixed_kspace_reuse_matches_fp64():
    """The mixed path with kspace_reuse and the FP32 real-space dipole operator
    against the plain FP64 path."""
    s = systems.mgo_pim(grid=(16, 16, 16), rc=10.0, alpha=0.3, kmax=12, vacancy_frac=0.01, seed=3, jitter=0.1)
    out = {}
    for prec, reuse in ((abi.PREC_FP64, 0), (abi.PREC_MIXED, 1)):
        p = s["params"]
        p.precision = prec
        p.kspace_reuse = reuse
        p.doefg = 1
        p.conv_tol_ind = 1e-10
        out[prec] = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"]).engforce()
    m, d = out[abi.PREC_MIXED], out[abi.PREC_FP64]
    assert rel(m["f"], d["f"]) < 1e-6
    assert rel(m["mu"], d["mu"]) < 1e-6
    assert rel(m["efg"], d["efg"]) < 1e-6
    assert abs(m["e"]["u_coul"] - d["e"]["u_coul"]) < 1e-6 * abs(d["e"]["u_coul"])
    assert rel(m["tau_coul"], d["tau_coul"]) < 1e-6


@pytest.mark.parametrize("prec,tol", [(abi.PREC_FP64, 1e-12), (abi.PREC_MIXED, 1e-8)])
def test_autotuned_launch_shapes_same_results(prec, tol):
    """The autotuner's launch shapes change only the summation order."""
    s = systems.mgo_pim(grid=(12, 12, 12), rc=8.0, alpha=0.4, kmax=10, vacancy_frac=0.01, seed=5, jitter=0.1)
    out, shape = {}, None
    for at in (0, 1):
        p = s["params"]
        p.precision = prec
        p.autotune = at
        p.kspace_reuse = 1
        p.conv_tol_ind = 1e-11
        e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
        out[at] = e.engforce()
        if at:
            shape = e.launch_shape()
    assert shape["g_dir"] in (8, 16, 32) and shape["g_dd32"] in (8, 16, 32)
    assert shape["sfac_split_x2"] in (1, 2, 4) and shape["field_split_x2"] in (1, 2, 4)
    assert rel(out[1]["f"], out[0]["f"]) < tol
    assert rel(out[1]["mu"], out[0]["mu"]) < tol


@pytest.mark.parametrize("case", ["mgo_pim", "silica_rigid", "mgo_small_kz"])
def test_tensor_core_structure_factor(case):
    """The tensor-core structure factor (exact int8 digit products of 24-bit
    fixed point) against the FP64 path, and no less accurate than the FP32
    CUDA-core kernel it replaces.  Covers charges with dipoles and field
    gradient, charges only, atom counts that are not a multiple of the
    16-atom pipeline block, and a short nz range."""
    if case == "mgo_pim":
        s = systems.mgo_pim(grid=(16, 16, 16), rc=10.0, alpha=0.3, kmax=12, vacancy_frac=0.01, seed=3, jitter=0.1)
        over = dict(doefg=1, conv_tol_ind=1e-10)
    elif case == "silica_rigid":
        s = systems.silica_bmh()
        over = dict(doefield=1)
    else:
        s = systems.mgo_pim(grid=(10, 10, 6), rc=6.0, alpha=0.5, kmax=9, vacancy_frac=0.02, seed=5, jitter=0.1)
        s["params"].kES[2] = 4
        over = dict(doefg=1, conv_tol_ind=1e-10)
    assert len(s["itype"]) % 16 != 0 or case == "silica_rigid"
    out = {}
    for key, prec, tc in (("fp64", abi.PREC_FP64, 0), ("fp32", abi.PREC_MIXED, 0), ("tc", abi.PREC_MIXED, 1)):
        p = s["params"]
        p.precision = prec
        p.kspace_tc = tc
        for k, v in over.items():
            setattr(p, k, v)
        out[key] = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"]).engforce()
    d = out["fp64"]
    e_tc = rel(out["tc"]["f"], d["f"])
    e_32 = rel(out["fp32"]["f"], d["f"])
    assert e_tc < 1e-6, (e_tc, e_32)
    assert e_tc < 2.0 * e_32 + 1e-8, (e_tc, e_32)
    assert abs(out["tc"]["e"]["u_coul"] - d["e"]["u_coul"]) < 1e-6 * abs(d["e"]["u_coul"])
    assert rel(out["tc"]["tau_coul"], d["tau_coul"]) < 1e-6
    if over.get("doefg"):
        assert rel(out["tc"]["mu"], d["mu"]) < 1e-6
        assert rel(out["tc"]["efg"], d["efg"]) < 1e-6


@pytest.mark.parametrize("case", ["mgo_pim", "silica_rigid", "mgo_small_kz"])
def test_low_set_on_tensor_cores(case):
    """kspace_tc = 2: the low-|k| set as int8 digit GEMMs of 32-bit fixed
    point (FP64 operands, ten digit products in four exact S32 levels) against
    the same set in FP64 on the CUDA cores (kspace_tc = 1), and against the
    FP64 path.  The 32-bit quantisation is 2.3e-10 of each operand's scale;
    a field value sums ~1 700 (column, nz) terms, so its error is about
    sqrt(1700) x 4.7e-10 = 2e-8 of the term size (measured 1.2e-8 on the
    forces and 1.8e-8 on the dipoles of the 4 055-ion PIM cell), a tenth of
    the mixed path's own error (~1.5e-7): forces, dipoles, field and EFG to
    5e-8.  The energy sums |S(k)|^2, where the quantisation errors average
    out: 1e-9 (measured 1.5e-12 on the PIM cell, 1.5e-10 on rigid-ion
    silica, whose few ions average less).  Covers dipoles with the field gradient (EFG), charges only,
    and a short nz range."""
    if case == "mgo_pim":
        s = systems.mgo_pim(grid=(16, 16, 16), rc=10.0, alpha=0.3, kmax=12, vacancy_frac=0.01, seed=3, jitter=0.1)
        over = dict(doefg=1, conv_tol_ind=1e-10)
    elif case == "silica_rigid":
        s = systems.silica_bmh()
        over = dict(doefield=1)
    else:
        s = systems.mgo_pim(grid=(10, 10, 6), rc=6.0, alpha=0.5, kmax=9, vacancy_frac=0.02, seed=5, jitter=0.1)
        s["params"].kES[2] = 4
        over = dict(doefg=1, conv_tol_ind=1e-10)
    out, mode = {}, {}
    for key, prec, tc in (("fp64", abi.PREC_FP64, 0), ("low64", abi.PREC_MIXED, 1), ("low32", abi.PREC_MIXED, 2)):
        p = s["params"]
        p.precision = prec
        p.kspace_tc = tc
        for k, v in over.items():
            setattr(p, k, v)
        e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
        out[key] = e.engforce()
        mode[key] = e.kspace_mode()
        e.close()
    assert mode["low32"] == {"main_tc": True, "low_tc": True}, mode
    assert mode["low64"] == {"main_tc": True, "low_tc": False}, mode
    a, b, d = out["low32"], out["low64"], out["fp64"]
    errs = {"F": rel(a["f"], b["f"]), "u": abs(a["e"]["u_coul"] - b["e"]["u_coul"]) / abs(b["e"]["u_coul"]),
            "tau": rel(a["tau_coul"], b["tau_coul"])}
    if over.get("doefg"):
        errs.update(mu=rel(a["mu"], b["mu"]), efg=rel(a["efg"], b["efg"]))
    else:
        errs.update(ef=rel(a["ef"], b["ef"]))
    print(case, errs)
    assert 0.0 < errs["F"] < 5e-8, errs
    assert max(v for k, v in errs.items() if k != "u") < 5e-8, errs
    assert errs["u"] < 1e-9, errs
    assert rel(a["f"], d["f"]) < 1e-6
    assert abs(a["e"]["u_coul"] - d["e"]["u_coul"]) < 1e-6 * abs(d["e"]["u_coul"])


def _production_run(pos, s, prec, kadd=0):
    p = s["params"]
    p.precision = prec
    p.kspace_reuse = 1 if prec == abi.PREC_MIXED else 0
    p.doefg = 1
    p.efg_period = 0
    k0 = list(p.kES)
    p.kES = (C.c_int * 3)(*[k + kadd for k in k0])
    e = mdff_b200.Engine(p, s["itype"], pos, s["cell"])
    r = e.engforce()
    e.close()
    p.kES = (C.c_int * 3)(*k0)
    return r


def _production_errors(pos, s):
    """Mixed path (the production settings: tensor-core k-space, mixed_keps
    sphere, FP64 low-|k| set, structure-factor reuse) against the plain FP64
    path (the reference's whole half space, no reuse) at identical positions,
    and the plain FP64 path's own k truncation (kmax 23 against kmax 27) on
    the Coulomb stress."""
    m = _production_run(pos, s, abi.PREC_MIXED)
    d = _production_run(pos, s, abi.PREC_FP64)
    w = _production_run(pos, s, abi.PREC_FP64, kadd=4)
    dn = np.linalg.norm
    return {"F": rel(m["f"], d["f"]), "mu": rel(m["mu"], d["mu"]), "efg": rel(m["efg"], d["efg"]),
            "tau_coul": rel(m["tau_coul"], d["tau_coul"]),
            "dtau_mixed": float(dn(m["tau_coul"] - d["tau_coul"])),
            "dtau_kmax": float(dn(w["tau_coul"] - d["tau_coul"])),
            "tau_total": rel(m["tau_coul"] + m["tau_nonb"], d["tau_coul"] + d["tau_nonb"]),
            "u": abs(m["e"]["u_coul"] - d["e"]["u_coul"]) / abs(d["e"]["u_coul"])}


def test_mixed_error_at_production_cell():
    """The graded configuration itself: the 32 440-ion cell with kmax 23 (the
    mixed path leaves out the 16 974 vectors of the half space outside its
    exp(-k^2/4 alpha^2) >= 1e-7 sphere).  Bound 1e-6 on forces, dipoles, EFG,
    the Coulomb energy and the Coulomb stress, at the start positions and at a
    snapshot of an FP64 NVT trajectory 50 steps in.  The stress sum weights
    each k by an extra (1 - kcoe k^2), about k^2 / 2 alpha^2 = 32 at the
    sphere, so the stress carries most of the sphere's error (measured
    5.7e-7, ten times the change the reference's own kmax 23 -> 27 makes);
    the total stress (Coulomb plus short range) nearly cancels in this cell,
    so its relative error is larger and only reported."""
    s = systems.mgo_production()
    e0 = _production_errors(s["pos"], s)
    assert max(e0["F"], e0["mu"], e0["efg"], e0["tau_coul"], e0["u"]) < 1e-6, e0
    p = s["params"]
    p.precision = abi.PREC_FP64
    traj = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    traj.md_start(s["vel"])
    traj.step(50, thermo=False)
    pos50 = traj.positions()
    traj.close()
    e50 = _production_errors(pos50, s)
    assert max(e50["F"], e50["mu"], e50["efg"], e50["tau_coul"], e50["u"]) < 1e-6, e50


def test_fp64_sphere_matches_mixed_set():
    """fp64_keps: the FP64 path over the same k sphere as the mixed path (the
    like-for-like FP64 arm).  Against the plain FP64 path the sphere costs at
    most the left-out Gaussian weight; against the mixed path (same sphere)
    what is left is the mixed path's own arithmetic."""
    s = systems.mgo_pim(grid=(16, 16, 16), rc=10.0, alpha=0.3, kmax=12, vacancy_frac=0.01, seed=3, jitter=0.1)
    res = {}
    for name, prec, keps in (("full", abi.PREC_FP64, 0.0), ("sphere", abi.PREC_FP64, 1e-7),
                             ("mixed", abi.PREC_MIXED, 0.0)):
        p = s["params"]
        p.precision = prec
        p.fp64_keps = keps
        p.kspace_reuse = 1
        p.doefg = 1
        p.conv_tol_ind = 1e-10
        e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
        res[name] = e.engforce()
        res[name + "_k"] = e.kspace_info()
        e.close()
    assert res["sphere_k"]["main"] < res["full_k"]["main"] == res["full_k"]["half"]
    assert res["sphere_k"]["main"] == res["mixed_k"]["main"] + res["mixed_k"]["low"]
    assert rel(res["sphere"]["f"], res["full"]["f"]) < 1e-6
    assert rel(res["sphere"]["efg"], res["full"]["efg"]) < 1e-6
    assert rel(res["mixed"]["f"], res["sphere"]["f"]) < 1e-6
    assert abs(res["sphere"]["e"]["u_coul"] - res["full"]["e"]["u_coul"]) < 1e-7 * abs(res["full"]["e"]["u_coul"])


def test_mixed_triclinic_cell():
    """A sheared (triclinic) PIM cell: the tensor-core k-space in 24-bit and
    32-bit fixed point uses the reciprocal basis B in its column constants
    and the factorised phases X[nx] Y[ny] Z[nz] of the fractional
    coordinates, so a non-orthogonal B exercises both.  Mixed (both k sets on
    the tensor cores) against FP64 on forces, dipoles and EFG to 1e-6, and the
    32-bit low set against the FP64 low set to 5e-8."""
    s = systems.mgo_pim(grid=(16, 16, 16), rc=10.0, alpha=0.3, kmax=12, vacancy_frac=0.01, seed=4, jitter=0.08)
    L = np.diag(s["cell"]).copy()
    frac = s["pos"] / L
    cell = np.diag(L)
    cell[1, 0] = 0.07 * L[1]
    cell[2, 0] = -0.05 * L[2]
    cell[2, 1] = 0.04 * L[2]
    pos = frac @ cell
    out = {}
    for key, prec, tc in (("fp64", abi.PREC_FP64, 0), ("low64", abi.PREC_MIXED, 1), ("low32", abi.PREC_MIXED, 2)):
        p = s["params"]
        p.precision = prec
        p.kspace_tc = tc
        p.doefg = 1
        p.conv_tol_ind = 1e-10
        e = mdff_b200.Engine(p, s["itype"], pos, cell)
        out[key] = e.engforce()
        if tc == 2:
            assert e.kspace_mode() == {"main_tc": True, "low_tc": True}
        e.close()
    d, a, b = out["fp64"], out["low32"], out["low64"]
    assert rel(a["f"], d["f"]) < 1e-6
    assert rel(a["mu"], d["mu"]) < 1e-6
    assert rel(a["efg"], d["efg"]) < 1e-6
    assert abs(a["e"]["u_coul"] - d["e"]["u_coul"]) < 1e-6 * abs(d["e"]["u_coul"])
    assert rel(a["f"], b["f"]) < 5e-8 and rel(a["mu"], b["mu"]) < 5e-8
