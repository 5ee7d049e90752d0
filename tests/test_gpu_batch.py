"""Batched forces and the adjoint force-matching gradient on the GPU.

Checked against the CPU oracle (forces, stress, energy, loss and the
hand-derived gradient, FP64 on both sides), against central finite
differences of the engine's own loss (h = 1e-5 relative), for batch
consistency (a batch equals its configurations run one by one) and through
the torch.autograd.Function.
"""
import numpy as np
import pytest

import oracle
from mdff_b200 import abi, fit, systems

pytestmark = pytest.mark.gpu


def _base(tol=1e-12):
    p = systems.mgo_params(6.0, 0.5, 6)
    p.conv_tol_ind = tol
    p.max_scf_pol_iter = 500
    p.device = 0
    return p


def _cfg_params(p, c):
    q = fit.ParamSpace([]).apply(p, [])
    q.cutshortrange = q.cutlongrange = c["rc"]
    q.alphaES = c["alpha"]
    for d in range(3):
        q.kES[d] = c["kmax"][d]
    return q


def _targets(base, space, confs, theta_t):
    import mdff_b200
    b = mdff_b200.Batch(space.apply(base, theta_t), confs)
    out = b.forces()
    b.close()
    return out["f"], out["tau"]


@pytest.fixture(scope="module")
def small():
    confs = systems.mgo_batch(nconf=4, nmin=120, nmax=420, seed=21)
    base = _base()
    space = fit.mgo_space(base)
    theta0 = space.get(base)
    rng = np.random.default_rng(4)
    theta_t = theta0 * (1.0 + 0.05 * rng.standard_normal(len(theta0)))
    ft, tt = _targets(base, space, confs, theta_t)
    return confs, base, space, theta0, ft, tt


def test_batch_forces_match_oracle(small):
    import mdff_b200
    confs, base, space, theta0, _, _ = small
    b = mdff_b200.Batch(base, confs)
    out = b.forces()
    assert out["iters"] > 0
    for c, conf in enumerate(confs):
        r = oracle.Oracle(_cfg_params(base, conf), conf["itype"], conf["pos"], conf["cell"]).engforce()
        df = np.linalg.norm(out["f"][c] - r["f"]) / np.linalg.norm(r["f"])
        tau_o = r["tau_nonb"] + r["tau_coul"]
        dt = np.linalg.norm(out["tau"][c] - tau_o) / np.linalg.norm(tau_o)
        u_o = r["e"]["u_bmhft"] + r["e"]["u_coul"]
        du = abs(out["energy"][c] - u_o) / abs(u_o)
        assert df < 1e-10 and dt < 1e-10 and du < 1e-11, (c, df, dt, du)


def test_batch_loss_grad_matches_oracle(small):
    import mdff_b200
    confs, base, space, theta0, ft, tt = small
    b = mdff_b200.Batch(base, confs)
    b.set_targets(ft, tt, 1.0, 0.01)
    loss, g, its = b.loss_grad()
    assert its[0] > 0 and its[1] > 0
    consts = fit.batch_constants([len(c["itype"]) for c in confs], 1.0, 0.01)
    go = abi.ParamGrad()
    lo = 0.0
    for conf, f, t, (cf, cs) in zip(confs, ft, tt, consts):
        o = oracle.Oracle(_cfg_params(base, conf), conf["itype"], conf["pos"], conf["cell"])
        l, go, _ = o.loss_grad(f, t, cf, cs, go)
        lo += l
    assert abs(loss - lo) / abs(lo) < 1e-9, (loss, lo)
    ge = space.project(g, theta0)
    gr = space.project(go, theta0)
    scale = np.abs(gr * theta0).max()
    err = np.abs(ge - gr) * np.abs(theta0) / scale
    assert err.max() < 1e-8, list(zip(space.names, ge, gr))
    rel = np.abs(ge - gr) / np.abs(gr)
    assert np.median(rel) < 1e-8, list(zip(space.names, rel))


def test_batch_grad_vs_central_differences(small):
    import mdff_b200
    confs, base, space, theta0, ft, tt = small
    b = mdff_b200.Batch(base, confs)
    b.set_targets(ft, tt, 1.0, 0.01)
    L0, g, _ = b.loss_grad()
    ge = space.project(g, theta0)
    fd = np.empty_like(ge)
    for k in range(len(theta0)):
        h = 1e-5 * abs(theta0[k])
        vals = []
        for sgn in (1.0, -1.0):
            th = theta0.copy()
            th[k] += sgn * h
            b.set_params(space.apply(base, th))
            vals.append(b.loss_grad(want_grad=False)[0])
        fd[k] = (vals[0] - vals[1]) / (2.0 * h)
    floor = 50.0 * np.finfo(float).eps * abs(L0) / (1e-5 * np.abs(theta0))
    ok = np.abs(ge - fd) <= np.maximum(1e-5 * np.abs(fd), floor)
    assert ok.all(), list(zip(space.names, ge, fd, floor))


def test_batch_is_sum_of_single_configurations(small):
    import mdff_b200
    confs, base, space, theta0, ft, tt = small
    b = mdff_b200.Batch(base, confs)
    b.set_targets(ft, tt, 1.0, 0.01)
    L, g, _ = b.loss_grad()
    gb = space.project(g, theta0)
    B = len(confs)
    Ls, gs = 0.0, np.zeros_like(gb)
    for c in range(B):
        s = mdff_b200.Batch(base, [confs[c]])
        s.set_targets([ft[c]], [tt[c]], 1.0, 0.01)
        l, gg, _ = s.loss_grad()
        Ls += l / B          # each single batch normalises by its own size 1
        gs += space.project(gg, theta0) / B
    assert abs(L - Ls) / abs(Ls) < 1e-11
    np.testing.assert_allclose(gb, gs, rtol=1e-8, atol=1e-12 * np.abs(gs).max())


def test_batch_deterministic(small):
    import mdff_b200
    confs, base, space, theta0, ft, tt = small
    b = mdff_b200.Batch(base, confs)
    b.set_targets(ft, tt, 1.0, 0.01)
    l1, g1, _ = b.loss_grad()
    l2, g2, _ = b.loss_grad()
    assert l1 == l2
    assert np.array_equal(space.project(g1, theta0), space.project(g2, theta0))


def test_autograd_function(small):
    import torch
    import mdff_b200
    confs, base, space, theta0, ft, tt = small
    b = mdff_b200.Batch(base, confs)
    b.set_targets(ft, tt, 1.0, 0.01)
    theta = torch.tensor(theta0 * 1.01, dtype=torch.float64, requires_grad=True)
    loss = fit.force_match_loss(theta, b, space, base)
    (2.0 * loss).backward()
    b.set_params(space.apply(base, theta0 * 1.01))
    l, g, _ = b.loss_grad()
    assert loss.item() == l
    np.testing.assert_allclose(theta.grad.numpy(), 2.0 * space.project(g, theta0 * 1.01), rtol=1e-14)


def test_batch_64_uneven_configurations():
    """The force-matching workload: 64 configurations of 200-2000 ions."""
    import mdff_b200
    confs = systems.mgo_batch()
    base = _base(1e-8)
    space = fit.mgo_space(base)
    theta0 = space.get(base)
    theta_t = theta0 * (1.0 + 0.05 * np.random.default_rng(7).standard_normal(len(theta0)))
    b = mdff_b200.Batch(space.apply(base, theta_t), confs)
    out = b.forces()
    b.set_params(base)
    b.set_targets(out["f"], out["tau"], 1.0, 0.01)
    L, g, its = b.loss_grad()
    ge = space.project(g, theta0)
    assert np.isfinite(L) and L > 0 and np.all(np.isfinite(ge))
    assert 0 < its[0] < 200 and 0 < its[1] < 200
    # at the target parameters the loss and gradient vanish
    b.set_params(space.apply(base, theta_t))
    L1, g1, _ = b.loss_grad()
    assert L1 < 1e-18 * max(1.0, L)


def test_batch_64_matches_oracle_and_central_differences():
    """The force-matching workload itself (64 configurations of 200-2000 ions,
    69 642 in all, targets from parameters perturbed 5 %): the engine's loss and
    12-parameter gradient against the oracle's summed over the 64
    configurations (induced dipoles to 1e-10 on both sides), and against
    central differences of the batch loss (h = 1e-5 relative, dipoles to
    1e-12 so that the differences resolve the gradient to 1e-5)."""
    import mdff_b200
    confs = systems.mgo_batch()
    rng = np.random.default_rng(7)
    for tol in (1e-10, 1e-12):
        base = _base(tol)
        space = fit.mgo_space(base)
        theta0 = space.get(base)
        theta_t = theta0 * (1.0 + 0.05 * np.random.default_rng(7).standard_normal(len(theta0)))
        ft, tt = _targets(base, space, confs, theta_t)
        b = mdff_b200.Batch(base, confs)
        b.set_targets(ft, tt, 1.0, 0.01)
        L, g, its = b.loss_grad()
        ge = space.project(g, theta0)
        if tol == 1e-10:
            consts = fit.batch_constants([len(c["itype"]) for c in confs], 1.0, 0.01)
            go = abi.ParamGrad()
            lo = 0.0
            for conf, f, t, (cf, cs) in zip(confs, ft, tt, consts):
                o = oracle.Oracle(_cfg_params(base, conf), conf["itype"], conf["pos"], conf["cell"])
                l, go, _ = o.loss_grad(f, t, cf, cs, go)
                lo += l
            assert abs(L - lo) / abs(lo) < 1e-8, (L, lo)
            gr = space.project(go, theta0)
            err = np.abs(ge - gr) * np.abs(theta0) / np.abs(gr * theta0).max()
            assert err.max() < 1e-7, list(zip(space.names, ge, gr))
        else:
            fd = np.empty_like(ge)
            for k in range(len(theta0)):
                h = 1e-5 * abs(theta0[k])
                vals = []
                for sgn in (1.0, -1.0):
                    th = theta0.copy()
                    th[k] += sgn * h
                    b.set_params(space.apply(base, th))
                    vals.append(b.loss_grad(want_grad=False)[0])
                fd[k] = (vals[0] - vals[1]) / (2.0 * h)
            floor = 50.0 * np.finfo(float).eps * abs(L) / (1e-5 * np.abs(theta0))
            ok = np.abs(ge - fd) <= np.maximum(1e-5 * np.abs(fd), floor)
            assert ok.all(), list(zip(space.names, ge, fd, floor))
        b.close()


def test_mixed_batch_against_fp64_batch():
    """The mixed batch (the dipole operator's pair table in FP32, its products
    in FP32 and sums in FP64) against the FP64 batch on the force-matching
    workload: forces to 1e-6 (global relative), and the loss and gradient to
    2e-5 -- the loss squares the force residual, which is ~5 % of the force, so
    a force error e moves the loss by ~2e / 0.05."""
    import mdff_b200
    confs = systems.mgo_batch()
    base = _base(1e-10)
    space = fit.mgo_space(base)
    theta0 = space.get(base)
    theta_t = theta0 * (1.0 + 0.05 * np.random.default_rng(7).standard_normal(len(theta0)))
    ft, tt = _targets(base, space, confs, theta_t)
    out = {}
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        p = fit.ParamSpace([]).apply(base, [])
        p.precision = prec
        b = mdff_b200.Batch(p, confs)
        fo = b.forces()
        b.set_targets(ft, tt, 1.0, 0.01)
        L, g, _ = b.loss_grad()
        out[prec] = (np.concatenate([f.ravel() for f in fo["f"]]), L, space.project(g, theta0))
        b.close()
    (fd, Ld, gd), (fm, Lm, gm) = out[abi.PREC_FP64], out[abi.PREC_MIXED]
    assert np.linalg.norm(fm - fd) / np.linalg.norm(fd) < 1e-6
    assert abs(Lm - Ld) < 2e-5 * abs(Ld)
    assert np.linalg.norm(gm - gd) < 2e-5 * np.linalg.norm(gd)
