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


# ---- the EFG chi^2 terms (rmc_efg, src/rmc.f90:1499-1660) ----

def rigid_mgo(grid=(4, 4, 4), rc=4.1, alpha=1.25, kmax=12, seed=2, jitter=0.05):
    """Rigid-ion MgO (the PIM cell without polarisabilities): rmc_main's EFG
    is that of the point charges.  alpha * rc ~ 5 makes the real-space terms
    beyond rc negligible, so the MD path's EFG (within rc) and
    multipole_efg_ES (every minimum image) agree to ~1e-10.  An even grid
    keeps the cell neutral (a charged one gives every tensor a trace)."""
    s = systems.mgo_pim(grid=grid, rc=rc, alpha=alpha, kmax=kmax, vacancy_frac=0.0, seed=seed, jitter=jitter)
    p = s["params"]
    for t in range(p.ntype):
        p.ldip_polar[t] = 0
        p.poldip_iso[t] = 0.0
    p.doefg = 1
    return s


def efg_params():
    ep = abi.RmcEfgParams()
    ep.lrmc_u = ep.lrmc_vzz = ep.lrmc_eta = 1
    ep.efg_start = 0
    ep.resolution_u_efg, ep.u_efg_min = 0.05, -3.0
    ep.resolution_vzz_efg, ep.vzz_efg_min = 0.05, -4.0
    ep.resolution_eta_efg = 0.05
    return ep


def rmc_par(acc, trials, cut=4.0, res=0.1, temp=1e-3):
    rp = abi.RmcParams()
    rp.max_displacement, rp.resolution_gr, rp.cut_rmc = 0.1, res, cut
    for q in range(6):
        rp.temp_rmc[q] = temp
    rp.acceptance_max, rp.max_trials = acc, trials
    return rp


def distributions(s, ep):
    """rmc_efg's distributions of a configuration: the chain's start with no trial."""
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    su, sv, se = ep.shapes(s["params"].ntype)
    g = o.gr(4.0, 0.1)
    r, _, U, V, E = o.rmc_efg(rmc_par(1, 1), ep, g, np.zeros(su), np.zeros(sv), np.zeros(se), [])
    return g, U, V, E, r


def test_efg_of_rmc_is_the_point_charge_ewald_efg():
    # multipole_efg_ES (every minimum image, no coul_unit) against the MD
    # path's Ewald EFG (within rc, times coul_unit)
    s = rigid_mgo()
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    V = o.efg_rmc()
    md = o.engforce()["efg"]
    cu = 14.399645   # e^2 / (4 pi eps0 A) in eV
    assert np.max(np.abs(md / cu - V)) < 1e-6 * np.max(np.abs(V))
    ratio = md[np.abs(V) > 0.1] / V[np.abs(V) > 0.1]
    assert np.ptp(ratio) < 1e-8 * np.mean(ratio)


def test_rmc_efg_distributions_and_quirks():
    s = rigid_mgo()
    ep = efg_params()
    _, U, V, E, r = distributions(s, ep)
    n, natmi = len(s["itype"]), np.bincount(np.asarray(s["itype"]) - 1)   # itype is 1-based
    # every site inside the Vzz and eta ranges: the all-sites rows integrate to 1
    assert abs(V[:, 0].sum() * ep.resolution_vzz_efg - 1.0) < 1e-12
    assert abs(E[:, 0].sum() * ep.resolution_eta_efg - 1.0) < 1e-12
    for t in range(2):
        assert abs(V[:, 1 + t].sum() * ep.resolution_vzz_efg - 1.0) < 1e-12
    # the reference's per-type U rows divide the all-types U1 counts
    for t in range(2):
        assert np.allclose(U[:, 1 + t, :5], (U[:, 0, 0] * n / natmi[t])[:, None], rtol=1e-14, atol=0)
    assert not U[:, :, 5].any() and not E[-1].any()
    # chi^2 against itself is zero; the total is the sum of the terms
    g, U2, V2, E2, r2 = distributions(s, ep)
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    r3, *_ = o.rmc_efg(rmc_par(1, 1), ep, g, U, V, E, [])
    assert r3["chisq"] == [0.0] * 6
    assert r["chisq"][5] == sum(r["chisq"][:5])


def test_rmc_efg_chain_fits_the_target():
    ep = efg_params()
    t = rigid_mgo(seed=7, jitter=0.15)
    g, U, V, E, _ = distributions(t, ep)
    s = rigid_mgo()
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    r0, *_ = o.rmc_efg(rmc_par(1, 1), ep, g, U, V, E, [])
    u = np.random.default_rng(7).random(40000)
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    r, g1, U1, V1, E1 = o.rmc_efg(rmc_par(200, 3000), ep, g, U, V, E, u)
    assert r["status"] == 0 and r["kacc"] > 10
    assert r["chisq"][5] < 0.5 * r0["chisq"][5]
    # the reported chi^2 and distributions are those of the final configuration
    o2 = oracle.Oracle(s["params"], s["itype"], o.positions(), s["cell"])
    rf, gf, Uf, Vf, Ef = o2.rmc_efg(rmc_par(1, 1), ep, g, U, V, E, [])
    assert np.array_equal(Uf, U1) and np.array_equal(Vf, V1) and np.array_equal(Ef, E1)
    assert abs(rf["chisq"][5] - r["chisq"][5]) <= 1e-9 * r["chisq"][5]


def test_rmc_efg_start_delays_the_efg_terms():
    ep = efg_params()
    ep.efg_start = 10 ** 6
    t = rigid_mgo(seed=7, jitter=0.15)
    g, U, V, E, _ = distributions(t, efg_params())
    s = rigid_mgo()
    u = np.random.default_rng(3).random(5000)
    a = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"]).rmc_efg(rmc_par(20, 300), ep, g, U, V, E, u)
    b = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"]).rmc(rmc_par(20, 300), g, u)
    assert a[0]["chisq"][2:5] == [0.0, 0.0, 0.0]
    assert (a[0]["kall"], a[0]["kacc"], a[0]["uniforms_used"]) == (b[0]["kall"], b[0]["kacc"], b[0]["uniforms_used"])
    assert np.array_equal(a[1], b[1])


# ---- the distance-variance term (eval_chisq_var_distance, src/rmc.f90:778-1063) ----

def var_params():
    ep = abi.RmcEfgParams()
    ep.lrmc_var = 1
    ep.resolution_u_efg = ep.resolution_vzz_efg = ep.resolution_eta_efg = 0.1
    ep.u_efg_min = ep.vzz_efg_min = -1.0
    return ep


def chisq_var_numpy(s):
    """eval_chisq_var_distance restated in numpy: per atom and type the sorted
    minimum-image distances to the other atoms of that type, the mean of the
    m-th smallest over the atoms of each type, and
    sum (d_m - mean_m)^2 / mean_m^2 over atoms, types and ranks."""
    pos = np.asarray(s["pos"], float)
    cell = np.asarray(s["cell"], float)
    it = np.asarray(s["itype"]) - 1
    frac = pos @ np.linalg.inv(cell)
    frac -= np.floor(frac)
    n, nt = len(pos), it.max() + 1
    lists = {}
    for a in range(n):
        d = frac[a] - frac
        d -= np.round(d)
        r = np.sqrt(((d @ cell) ** 2).sum(1))
        for t in range(nt):
            sel = (it == t) & (np.arange(n) != a)
            lists[a, t] = np.sort(r[sel])
    chi = 0.0
    for t1 in range(nt):
        atoms = np.where(it == t1)[0]
        for t2 in range(nt):
            L = np.array([lists[a, t2] for a in atoms])
            mean = L.sum(0) / len(atoms)
            chi += (((L - mean) / mean) ** 2).sum()
    return chi


def gexp_of(s, cut=2.0, res=0.05):
    return oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"]).gr(cut, res)


def test_variance_term_against_numpy_and_zero_on_a_lattice():
    # a two-type jittered cell: the oracle's chi^2 (no trial move) against the
    # numpy restatement; on the perfect FCC lattice every atom sees the same
    # sorted distances, so the term vanishes
    t = rigid_mgo(grid=(4, 4, 4), jitter=0.12, seed=3)
    o = oracle.Oracle(t["params"], t["itype"], t["pos"], t["cell"])
    rp = rmc_params(10, 1)
    rp.cut_rmc = 4.0
    rp.resolution_gr = 0.1
    g = o.gr(4.0, 0.1)
    ep = var_params()
    su, sv, se = ep.shapes(t["params"].ntype)
    r, *_ = o.rmc_efg(rp, ep, g, np.zeros(su), np.zeros(sv), np.zeros(se), np.zeros(0))
    ref = chisq_var_numpy(t)
    assert abs(r["chisq"][1] - ref) < 1e-10 * ref
    s = lj(ncell=3)
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    su, sv, se = ep.shapes(s["params"].ntype)
    r, *_ = o.rmc_efg(rmc_params(10, 1), ep, gexp_of(s), np.zeros(su), np.zeros(sv), np.zeros(se), np.zeros(0))
    assert r["chisq"][1] < 1e-20


def test_variance_term_drives_the_chain_towards_equal_environments():
    # with the variance term alone deciding (g(r) at a high temperature), the
    # chain from a jittered lattice makes the atoms' distance lists more alike
    s = lj(ncell=3, jitter=0.06, seed=4)
    o = oracle.Oracle(s["params"], s["itype"], s["pos"], s["cell"])
    rp = rmc_params(100, 6000)
    rp.temp_rmc[0] = 1e6
    ep = var_params()
    su, sv, se = ep.shapes(s["params"].ntype)
    chi0 = chisq_var_numpy(s)
    r, *_ = o.rmc_efg(rp, ep, gexp_of(s), np.zeros(su), np.zeros(sv), np.zeros(se),
                      np.random.default_rng(9).random(40000))
    assert r["status"] == 0 and r["kacc"] == 100
    assert r["chisq"][1] < 0.9 * chi0
