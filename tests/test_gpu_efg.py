"""EFG post-processing on the GPU (mdff_efg_nmr / mdff_efg_dist) against the
CPU restatement of efg_stat and nmr_convention (oracle/efg_stat.py) on the
same tensors.

Tolerances: Czjzek components 1e-15 relative (the same products; FMA
contraction in S); principal values 1e-12 of the tensor scale (cyclic Jacobi
against LAPACK); eta 1e-10 absolute; statistics 1e-12 relative (summation
order); integer histograms exact.
"""
import numpy as np
import pytest

import mdff_b200
from mdff_b200 import abi, systems
from oracle import efg_stat

pytestmark = pytest.mark.gpu


def dist_params(**kw):
    d = abi.EfgDistParams()
    d.vzzmin, d.resvzz, d.reseta, d.umin, d.resu, d.smax = (kw.get(k) for k in
                                                          ("vzzmin", "resvzz", "reseta", "umin", "resu", "smax"))
    return d


def engine_for(grid=(8, 8, 8), doefg=1):
    s = systems.mgo_pim(grid=grid, rc=6.0, alpha=0.5, kmax=7)
    s["params"].doefg = doefg
    return mdff_b200.Engine(s["params"], s["itype"], s["pos"], s["cell"]), s


def random_traceless(n, rng, scale=1.0):
    a = rng.normal(0, scale, (n, 6))
    a[:, 2] = -(a[:, 0] + a[:, 1])
    return a


def check_nmr(e, efg):
    nmr, U, S = e.efg_nmr(efg)
    on, oU, oS = efg_stat.efg_nmr(efg)
    scale = np.abs(efg).max()
    assert np.max(np.abs(U - oU)) <= 1e-15 * scale
    assert np.max(np.abs(S - oS)) <= 2e-15 * scale
    assert np.max(np.abs(nmr[:, :3] - on[:, :3])) <= 1e-12 * scale
    assert np.max(np.abs(nmr[:, 3] - on[:, 3])) <= 1e-10
    return nmr


def test_nmr_random_tensors():
    e, s = engine_for()
    rng = np.random.default_rng(11)
    check_nmr(e, random_traceless(e.n, rng))
    # axial tensors (eta = 0) rotated, and exact diagonal ones
    t = np.zeros((e.n, 6))
    for i in range(e.n):
        q, r = np.linalg.qr(rng.normal(size=(3, 3)))
        m = q @ np.diag([-1.0, -1.0, 2.0]) * rng.uniform(0.1, 3) @ q.T
        t[i] = [m[0, 0], m[1, 1], m[2, 2], m[0, 1], m[0, 2], m[1, 2]]
    nmr = check_nmr(e, t)
    assert np.max(np.abs(nmr[:, 3])) < 1e-10
    d = np.zeros((e.n, 6))
    d[:, :3] = [2.0003749, -1.0001874, -1.0001874]
    nmr, _, _ = e.efg_nmr(d)
    assert np.all(nmr[:, 2] == 2.0003749) and np.all(nmr[:, 3] == 0.0)


def test_dist_matches_oracle():
    e, s = engine_for()
    rng = np.random.default_rng(5)
    efg = random_traceless(e.n, rng)
    kw = dict(vzzmin=-8.0, resvzz=0.05, reseta=0.02, umin=-6.0, resu=0.05, smax=8.0)
    got = e.efg_dist(dist_params(**kw), efg)
    ref = efg_stat.efg_dist(efg, s["itype"], s["params"].ntype, **kw)
    for k in ("vzz", "eta", "u", "s"):
        assert got[k].shape == ref[k].shape, k
        assert np.array_equal(got[k], ref[k]), k
    assert np.allclose(got["stats"], ref["stats"], rtol=1e-12, atol=1e-14)
    assert np.allclose(got["mU"], ref["mU"], rtol=1e-12, atol=1e-14)
    assert np.allclose(got["m2U"], ref["m2U"], rtol=1e-12, atol=1e-14)


def test_dist_over_configurations():
    # several configurations in one call: histograms summed, statistics formed
    # as the reference's configuration loop forms them
    e, s = engine_for()
    rng = np.random.default_rng(8)
    efg = np.stack([random_traceless(e.n, rng, scale=0.5 + 0.25 * c) for c in range(5)])
    kw = dict(vzzmin=-10.0, resvzz=0.05, reseta=0.02, umin=-8.0, resu=0.05, smax=10.0)
    got = e.efg_dist(dist_params(**kw), efg)
    ref = efg_stat.efg_dist(efg, s["itype"], s["params"].ntype, **kw)
    for k in ("vzz", "eta", "u", "s"):
        assert np.array_equal(got[k], ref[k]), k
    assert got["stats"].shape == (5, 3, 8)
    for k in ("stats", "mU", "m2U"):
        assert np.allclose(got[k], ref[k], rtol=1e-12, atol=1e-14), k
    nmr, U, S = e.efg_nmr(efg)
    assert nmr.shape == (5, e.n, 4)
    assert np.max(np.abs(nmr[:, :, 2] - ref["nmr"][:, :, 2])) <= 1e-12 * np.abs(efg).max()
    assert np.max(np.abs(U - ref["U"])) <= 1e-15 * np.abs(efg).max()


def test_dist_many_bins_global_histograms():
    # more bins than fit the block-private shared-memory histograms
    e, s = engine_for()
    efg = random_traceless(e.n, np.random.default_rng(12))
    kw = dict(vzzmin=-8.0, resvzz=0.002, reseta=0.001, umin=-6.0, resu=0.002, smax=8.0)
    got = e.efg_dist(dist_params(**kw), efg)
    ref = efg_stat.efg_dist(efg, s["itype"], s["params"].ntype, **kw)
    assert got["u"].size > 12288
    for k in ("vzz", "eta", "u", "s"):
        assert np.array_equal(got[k], ref[k]), k


def test_dist_from_device_memory():
    # tensors already on the GPU are read in place and give the same answer
    import torch
    e, s = engine_for()
    efg = np.stack([random_traceless(e.n, np.random.default_rng(c), scale=0.8) for c in range(3)])
    kw = dict(vzzmin=-8.0, resvzz=0.05, reseta=0.02, umin=-6.0, resu=0.05, smax=8.0)
    t = torch.from_numpy(np.ascontiguousarray(efg.transpose(0, 2, 1))).cuda()
    got = e.efg_dist_ptr(dist_params(**kw), t.data_ptr(), 3)
    ref = e.efg_dist(dist_params(**kw), efg)
    for k in ("vzz", "eta", "u", "s", "stats", "mU", "m2U"):
        assert np.array_equal(got[k], ref[k]), k


def test_dist_of_engine_efg():
    # tensors of a PIM force evaluation (doefg) taken from the context itself
    s = systems.mgo_pim(grid=(8, 8, 8), rc=6.0, alpha=0.5, kmax=7, vacancy_frac=0.02, seed=4)
    p = s["params"]
    p.doefg = 1
    pos = s["pos"] + np.random.default_rng(3).normal(0, 0.05, s["pos"].shape)
    e = mdff_b200.Engine(p, s["itype"], pos, s["cell"])
    efg = e.engforce()["efg"]
    check_nmr(e, efg)
    v = np.abs(efg).max()
    kw = dict(vzzmin=-4 * v, resvzz=v / 50, reseta=0.05, umin=-4 * v, resu=v / 50, smax=4 * v)
    got = e.efg_dist(dist_params(**kw))                 # None: the context's own EFG
    ref = efg_stat.efg_dist(efg, s["itype"], p.ntype, **kw)
    for k in ("vzz", "eta", "u", "s"):
        assert np.array_equal(got[k], ref[k]), k
    assert np.allclose(got["stats"], ref["stats"], rtol=1e-11, atol=1e-14)


def test_dist_out_of_range_is_an_error():
    e, s = engine_for()
    efg = random_traceless(e.n, np.random.default_rng(1), scale=5.0)
    with pytest.raises(mdff_b200.EngineError) as ei:
        e.efg_dist(dist_params(vzzmin=-0.5, resvzz=0.1, reseta=0.1, umin=-40.0, resu=0.1, smax=80.0), efg)
    assert ei.value.code == abi.E_ARG
    with pytest.raises(mdff_b200.EngineError):
        e.efg_dist(dist_params(vzzmin=-0.5, resvzz=0.0, reseta=0.1, umin=-4.0, resu=0.1, smax=8.0), efg)


def test_nmr_without_efg_state_is_an_error():
    e, s = engine_for(doefg=0)
    with pytest.raises(mdff_b200.EngineError) as ei:
        e.efg_nmr(None)
    assert ei.value.code == abi.E_STATE
