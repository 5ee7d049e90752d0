"""The oracle's force-matching gradient (hand-derived adjoint through the pair
loop, the multipole Ewald sum and the induced-dipole solve) against central
finite differences of the oracle's own loss, h = 1e-5 relative.

This pins the derivation on the CPU; the engine's adjoint kernels are then
checked against this gradient and against their own finite differences on
the GPU (test_gpu_adjoint.py).
"""
import numpy as np
import pytest

import oracle
from mdff_b200 import abi, fit, systems


def _setup(nconf=1, nmin=120, nmax=160, seed=5):
    confs = systems.mgo_batch(nconf=nconf, nmin=nmin, nmax=nmax, seed=seed)
    base = systems.mgo_params(6.0, 0.5, 6)
    base.conv_tol_ind = 1e-13
    base.max_scf_pol_iter = 500
    space = fit.mgo_space(base)
    return confs, base, space


def _cfg_params(p, c):
    q = fit.ParamSpace([]).apply(p, [])
    q.cutshortrange = q.cutlongrange = c["rc"]
    q.alphaES = c["alpha"]
    for d in range(3):
        q.kES[d] = c["kmax"][d]
    return q


def _loss(confs, base, space, targets, consts, theta):
    p = space.apply(base, theta)
    g = abi.ParamGrad()
    L = 0.0
    for c, (ft, tt), (cf, cs) in zip(confs, targets, consts):
        o = oracle.Oracle(_cfg_params(p, c), c["itype"], c["pos"], c["cell"])
        l, g, _ = o.loss_grad(ft, tt, cf, cs, g)
        L += l
    return L, space.project(g, theta)


def test_space_roundtrip():
    _, base, space = _setup()
    th = space.get(base)
    assert len(th) == 12
    p2 = space.apply(base, th * 1.1)
    np.testing.assert_allclose(space.get(p2), th * 1.1, rtol=1e-15)
    # the symmetric counterpart of a pair entry moves with it
    assert p2.Abmhftd[1][0] == p2.Abmhftd[0][1]
    assert p2.dip_pol_damp_b[0][1][0] == p2.dip_pol_damp_b[0][0][1]


def test_adjoint_vs_central_differences():
    confs, base, space = _setup(nconf=2)
    theta0 = space.get(base)
    rng = np.random.default_rng(3)
    theta_t = theta0 * (1.0 + 0.05 * rng.standard_normal(len(theta0)))
    targets = []
    for c in confs:
        r = oracle.Oracle(_cfg_params(space.apply(base, theta_t), c), c["itype"], c["pos"], c["cell"]).engforce()
        targets.append((r["f"], r["tau_nonb"] + r["tau_coul"]))
    consts = fit.batch_constants([len(c["itype"]) for c in confs], 1.0, 0.01)
    L0, g = _loss(confs, base, space, targets, consts, theta0)
    fd = np.empty_like(g)
    for k in range(len(theta0)):
        h = 1e-5 * abs(theta0[k])
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += h
        tm[k] -= h
        fd[k] = (_loss(confs, base, space, targets, consts, tp)[0] -
                 _loss(confs, base, space, targets, consts, tm)[0]) / (2.0 * h)
    # errors on the dL/dln(theta) scale, normalised by its largest component
    sens = np.abs(fd * theta0)
    err = np.abs(g - fd) * np.abs(theta0)
    assert err.max() / sens.max() < 1e-5, (err / sens.max())
    # per component: within 1e-5 relative, or within the central-difference
    # round-off floor eps*L/h (a few components are 1e-8 of the loss scale)
    floor = 50.0 * np.finfo(float).eps * abs(L0) / (1e-5 * np.abs(theta0))
    ok = np.abs(g - fd) <= np.maximum(1e-5 * np.abs(fd), floor)
    assert ok.all(), list(zip(space.names, g, fd, floor))


def test_adjoint_morse_pair_terms():
    """Morse derivatives (not in the MgO set) on a Morse + BMHFTD system."""
    confs, base, _ = _setup(nconf=1, nmin=100, nmax=110, seed=8)
    base.lmorse = 1
    for (i, j) in ((0, 0), (0, 1), (1, 1)):
        for a, b in ((i, j), (j, i)):
            base.epsmor[a][b] = 0.05
            base.rhomor[a][b] = 1.6
            base.sigmamor[a][b] = 2.8
    space = fit.ParamSpace([fit.Tie("eps", [("epsmor", (0, 1))]), fit.Tie("rho", [("rhomor", (0, 1))]),
                            fit.Tie("sig", [("sigmamor", (0, 1))]), fit.Tie("eps_OO", [("epsmor", (0, 0))])])
    theta0 = space.get(base)
    c = confs[0]
    tgt = oracle.Oracle(_cfg_params(space.apply(base, theta0 * 1.03), c), c["itype"], c["pos"], c["cell"]).engforce()
    targets = [(tgt["f"], tgt["tau_nonb"] + tgt["tau_coul"])]
    consts = fit.batch_constants([len(c["itype"])], 1.0, 0.01)
    L0, g = _loss(confs, base, space, targets, consts, theta0)
    for k in range(len(theta0)):
        h = 1e-5 * abs(theta0[k])
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += h
        tm[k] -= h
        fd = (_loss(confs, base, space, targets, consts, tp)[0] - _loss(confs, base, space, targets, consts, tm)[0]) / (2 * h)
        floor = 50.0 * np.finfo(float).eps * abs(L0) / h
        assert abs(g[k] - fd) <= max(1e-5 * abs(fd), floor), (space.names[k], g[k], fd)
