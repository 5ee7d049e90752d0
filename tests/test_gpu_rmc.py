"""g(r) and reverse Monte Carlo on the GPU (mdff_gr, mdff_rmc) against the
oracle's restatement of gr_main / rmc_gr / rmc_main.

g(r): the same integer counts and the same normalisation, so the rows agree
bit for bit.  RMC: given the same random stream the device chain (incremental
counts in one persistent CTA) and the oracle's (full recount every move, as
the reference) take the same decisions: the same trial and acceptance counts,
the same stream consumption, the same chi^2 and final configuration.
"""
import numpy as np
import pytest

import mdff_b200
import oracle
from mdff_b200 import abi, systems

pytestmark = pytest.mark.gpu


def lj(ncell=3, jitter=0.0, seed=1):
    s = systems.lj_argon(ncell=ncell)
    if jitter:
        s["pos"] = s["pos"] + np.random.default_rng(seed).normal(0, jitter, s["pos"].shape)
    return s


def mgo(jitter=0.0, seed=2):
    s = systems.mgo_pim(grid=(6, 6, 6), rc=5.0, alpha=0.6, kmax=6, vacancy_frac=0.02, seed=seed)
    if jitter:
        s["pos"] = s["pos"] + np.random.default_rng(seed).normal(0, jitter, s["pos"].shape)
    return s


def pair(s):
    return (mdff_b200.Engine(s["params"], s["itype"], s["pos"], s["cell"]),
            oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"]))


@pytest.mark.parametrize("system,cut,res", [("lj", 2.2, 0.03), ("mgo", 6.0, 0.05)])
def test_gr_matches_oracle_bitwise(system, cut, res):
    s = lj(jitter=0.05) if system == "lj" else mgo(jitter=0.1)
    e, o = pair(s)
    ge, go = e.gr(cut, res), o.gr(cut, res)
    assert ge.shape == go.shape
    assert np.array_equal(ge, go)


def rmc_params(acc, trials, cut, res, temp=1e-3, disp=0.1):
    rp = abi.RmcParams()
    rp.max_displacement = disp
    rp.resolution_gr = res
    rp.cut_rmc = cut
    for q in range(6):
        rp.temp_rmc[q] = temp
    rp.acceptance_max = acc
    rp.max_trials = trials
    return rp


@pytest.mark.parametrize("system", ["lj", "mgo"])
def test_rmc_chain_matches_oracle(system):
    if system == "lj":
        s, t, cut, res = lj(), lj(jitter=0.08), 2.0, 0.05
    else:
        s, t, cut, res = mgo(), mgo(jitter=0.15, seed=9), 6.0, 0.1
    gexp = oracle.Oracle(t["params"], t["itype"], t["pos"], t["cell"]).gr(cut, res)
    e, o = pair(s)
    rp = rmc_params(150, 3000, cut, res)
    u = np.random.default_rng(7).random(40000)
    re, ge = e.rmc(rp, gexp, u)
    ro, go = o.rmc(rp, gexp, u)
    assert re["status"] == ro["status"] == 0
    assert (re["kall"], re["kacc"], re["uniforms_used"]) == (ro["kall"], ro["kacc"], ro["uniforms_used"])
    assert re["chisq"] == ro["chisq"]
    assert np.array_equal(ge, go)
    assert np.max(np.abs(e.positions() - o.positions())) < 1e-12
    # the chain's chi^2 is that of its final configuration's g(r)
    assert abs(re["chisq"][0] - float(np.sum((go - gexp) ** 2))) <= 1e-12 * max(1.0, re["chisq"][0])


def test_rmc_internal_stream_lowers_chi2():
    s, t = lj(ncell=4), lj(ncell=4, jitter=0.08)
    gexp = oracle.Oracle(t["params"], t["itype"], t["pos"], t["cell"]).gr(2.0, 0.05)
    e = mdff_b200.Engine(s["params"], s["itype"], s["pos"], s["cell"])
    chi0 = float(np.sum((e.gr(2.0, 0.05) - gexp) ** 2))
    r, g = e.rmc(rmc_params(1500, 100000, 2.0, 0.05), gexp, seed=12345)
    assert r["status"] == 0 and r["kacc"] > 500
    assert r["chisq"][0] < 0.1 * chi0
    assert abs(float(np.sum((g - gexp) ** 2)) - r["chisq"][0]) < 1e-12 * chi0


def test_rmc_rejects_bad_parameters():
    s = lj()
    e = mdff_b200.Engine(s["params"], s["itype"], s["pos"], s["cell"])
    rp = rmc_params(10, 10, 2.0, 0.05, temp=0.0)
    with pytest.raises(mdff_b200.EngineError):
        e.rmc(rp, np.zeros((2, 41)))


# ---- the EFG chi^2 terms: mdff_rmc_efg against the oracle's rmc_efg chain ----

from test_oracle_rmc import distributions, efg_params, rigid_mgo, rmc_par   # noqa: E402


@pytest.mark.parametrize("terms", ["all", "vzz_eta"])
def test_rmc_efg_chain_matches_oracle(terms):
    # the same uniforms: the same decisions, the same final configuration and
    # distributions.  The engine's EFG (the MD path within rc) and the
    # oracle's multipole_efg_ES (every minimum image) agree to ~1e-10 at
    # alpha rc ~ 5, far inside the bins; the histograms then agree exactly
    ep = efg_params()
    if terms == "vzz_eta":
        ep.lrmc_u = 0
    t = rigid_mgo(seed=7, jitter=0.15)
    g, U, V, E, _ = distributions(t, efg_params())
    s = rigid_mgo()
    u = np.random.default_rng(11).random(20000)
    rp = rmc_par(60, 800)
    e = mdff_b200.Engine(s["params"], s["itype"], s["pos"], s["cell"])
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    re, ge, Ue, Ve, Ee = e.rmc_efg(rp, ep, g, U, V, E, u)
    ro, go, Uo, Vo, Eo = o.rmc_efg(rp, ep, g, U, V, E, u)
    assert re["status"] == ro["status"] == 0
    assert (re["kall"], re["kacc"], re["uniforms_used"]) == (ro["kall"], ro["kacc"], ro["uniforms_used"])
    assert re["kacc"] > 5
    assert re["chisq"][0] == ro["chisq"][0]
    for q in range(2, 6):
        assert abs(re["chisq"][q] - ro["chisq"][q]) <= 1e-12 * max(1.0, ro["chisq"][q])
    assert np.array_equal(ge, go)
    assert np.array_equal(Ve, Vo) and np.array_equal(Ee, Eo)
    if ep.lrmc_u:
        assert np.array_equal(Ue, Uo)
    assert np.max(np.abs(e.positions() - o.positions())) < 1e-12


def test_rmc_efg_rejects_polarisable_systems():
    s = mgo()
    e = mdff_b200.Engine(s["params"], s["itype"], s["pos"], s["cell"])
    ep = efg_params()
    su, sv, se = ep.shapes(s["params"].ntype)
    with pytest.raises(mdff_b200.EngineError):
        e.rmc_efg(rmc_params(10, 10, 6.0, 0.1), ep, np.zeros((4, 61)), np.zeros(su), np.zeros(sv), np.zeros(se))


# ---- the distance-variance term: device lists against the oracle's full recount ----

from test_oracle_rmc import chisq_var_numpy, var_params   # noqa: E402


@pytest.mark.parametrize("with_efg", [False, True])
def test_rmc_variance_chain_matches_oracle(with_efg):
    # given the same uniforms the device chain (sorted lists kept on the device,
    # one value moved per atom and trial) and the oracle's full recount every
    # trial take the same decisions; the variance chi^2 agrees to 1e-11 (its
    # final sum runs per atom and by a fixed tree, the reference's left to right)
    ep = efg_params()
    if not with_efg:
        ep.lrmc_u = ep.lrmc_vzz = ep.lrmc_eta = 0
    ep.lrmc_var = 1
    t = rigid_mgo(seed=7, jitter=0.15)
    g, U, V, E, _ = distributions(t, efg_params())
    s = rigid_mgo()
    u = np.random.default_rng(13).random(20000)
    rp = rmc_par(60, 800)
    e = mdff_b200.Engine(s["params"], s["itype"], s["pos"], s["cell"])
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    re, ge, Ue, Ve, Ee = e.rmc_efg(rp, ep, g, U, V, E, u)
    ro, go, Uo, Vo, Eo = o.rmc_efg(rp, ep, g, U, V, E, u)
    assert re["status"] == ro["status"] == 0
    assert (re["kall"], re["kacc"], re["uniforms_used"]) == (ro["kall"], ro["kacc"], ro["uniforms_used"])
    assert re["kacc"] > 5
    assert ro["chisq"][1] > 0
    assert abs(re["chisq"][1] - ro["chisq"][1]) <= 1e-11 * ro["chisq"][1]
    assert np.array_equal(ge, go)
    assert np.max(np.abs(e.positions() - o.positions())) < 1e-12
    # rejected moves are undone, so the last accepted configuration is the
    # final one: its chi^2 is the numpy recount of the final positions
    fin = dict(s)
    fin["pos"] = o.positions()
    assert abs(re["chisq"][1] - chisq_var_numpy(fin)) < 1e-9 * ro["chisq"][1]


def test_rmc_variance_rejects_oversized_types():
    # more than 16384 atoms of one type: the device sort's limit
    s = systems.lj_argon(ncell=17)
    e = mdff_b200.Engine(s["params"], s["itype"], s["pos"], s["cell"])
    ep = var_params()
    su, sv, se = ep.shapes(s["params"].ntype)
    with pytest.raises(mdff_b200.EngineError) as exc:
        e.rmc_efg(rmc_params(10, 10, 2.0, 0.1), ep, np.zeros((2, 21)), np.zeros(su), np.zeros(sv), np.zeros(se))
    assert exc.value.code == abi.E_UNSUPPORTED
