"""g(r) and reverse Monte Carlo in the oracle (gr_main, src/radial_distrib.f90;
rmc_gr / rmc_main, src/rmc.f90): the normalisation of rmc_gr on an ideal gas
and on the FCC lattice's first shell, and the chain's behaviour -- chi^2
falls, the stream is consumed as the reference consumes it.
"""
import numpy as np

import oracle
from mdff_b200 import abi, systems


def lj(ncell=3, jitter=0.0, seed=1):
    s = systems.lj_argon(ncell=ncell)
    if jitter:
        s["pos"] = s["pos"] + np.random.default_rng(seed).normal(0, jitter, s["pos"].shape)
    return s


def test_ideal_gas_normalisation():
    rng = np.random.default_rng(3)
    n, L = 800, 12.0
    s = lj()
    o = oracle.Oracle(s["params"], np.ones(n, np.int32), rng.random((n, 3)) * L, np.eye(3) * L)
    g = o.gr(5.0, 0.25)
    # beyond the first bins g(r) of uncorrelated points is (N-1)/N on average;
    # the last of the INT(cut/res) + 1 bins holds r >= cut and stays empty
    assert abs(g[0, 8:-1].mean() - (n - 1) / n) < 0.03
    assert g[0, -1] == 0.0
    assert np.array_equal(g[0], g[1])           # one type: the type row is the all-pairs row


def test_fcc_first_shell_holds_twelve_neighbours():
    s = lj(ncell=4)
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    res = 0.02
    g = o.gr(1.5, res)
    n = len(s["itype"])
    V = float(np.linalg.det(s["cell"]))
    rr = (np.arange(g.shape[1]) + 0.5) * res
    vol = 4.0 * np.pi * (res * rr * rr + res ** 3 / 12.0) / V
    counts = g[0] * vol * n * n                  # ordered pairs per bin
    assert abs(counts.sum() / n - 12.0) < 1e-9   # 12 nearest neighbours within 1.5 sigma
    a = (4.0 / 0.844) ** (1.0 / 3.0)
    assert abs(rr[np.argmax(counts)] - a / np.sqrt(2.0)) < res


def rmc_params(acc, trials, temp=1e-3):
    rp = abi.RmcParams()
    rp.max_displacement = 0.1
    rp.resolution_gr = 0.05
    rp.cut_rmc = 2.0
    for q in range(6):
        rp.temp_rmc[q] = temp
    rp.acceptance_max = acc
    rp.max_trials = trials
    return rp


def test_chain_reduces_chi2_and_consumes_the_stream_in_order():
    s, t = lj(), lj(jitter=0.08)
    gexp = oracle.Oracle(t["params"], t["itype"], t["pos"], t["cell"]).gr(2.0, 0.05)
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    g0 = o.gr(2.0, 0.05)
    chi0 = float(np.sum((g0 - gexp) ** 2))
    r, g = o.rmc(rmc_params(300, 5000), gexp, np.random.default_rng(5).random(60000))
    assert r["status"] == 0 and r["kacc"] == 300
    assert r["chisq"][0] < 0.2 * chi0
    assert abs(float(np.sum((g - gexp) ** 2)) - r["chisq"][0]) < 1e-12 * chi0
    # per trial: particle + 3 displacements + one draw for each of the four
    # zero components (their change is 0, not negative) + two when g(r)'s
    # chi^2 (and so the total's) did not fall
    moves = r["kall"] - 1
    assert 8 * moves <= r["uniforms_used"] <= 10 * moves


def test_stream_running_out_stops_cleanly():
    s, t = lj(), lj(jitter=0.08)
    gexp = oracle.Oracle(t["params"], t["itype"], t["pos"], t["cell"]).gr(2.0, 0.05)
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    r, _ = o.rmc(rmc_params(10 ** 6, 10 ** 6), gexp, np.random.default_rng(2).random(103))
    assert r["status"] == 1 and r["uniforms_used"] <= 103
