"""The EFG post-processing restatement (oracle/efg_stat.py) on closed-form
cases: principal values of rotated diagonal tensors, the NMR ordering, eta,
the Czjzek invariant S^2 = Vzz^2 (1 + eta^2/3) / 4 of a traceless tensor, the
two-charge known answer of examples/ex4/run_ex4.sh:78-79, the per-type
statistics and the histogram bookkeeping of efg_stat (src/efg.f90:2272-2440).
"""
import math

import numpy as np
import pytest

from oracle import efg_stat


def rot(rng):
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    return q * np.sign(np.diag(r))


def tensor6(m):
    return np.array([m[0, 0], m[1, 1], m[2, 2], m[0, 1], m[0, 2], m[1, 2]])


def rotated(vals, rng):
    R = rot(rng)
    return tensor6(R @ np.diag(vals) @ R.T)


def test_rotated_principal_values_and_eta():
    rng = np.random.default_rng(1)
    for _ in range(200):
        vzz = rng.uniform(-3, 3)
        eta = rng.uniform(0, 1)
        vxx, vyy = -vzz * (1 - eta) / 2, -vzz * (1 + eta) / 2
        t = rotated([vyy, vzz, vxx], rng)
        nmr, U, S = efg_stat.efg_nmr(t[None, :])
        assert abs(nmr[0, 2] - vzz) < 1e-12 * 3
        assert abs(nmr[0, 3] - eta) < 1e-11 / abs(vzz)
        assert abs(nmr[0, 0] - vxx) < 1e-12 * 3 and abs(nmr[0, 1] - vyy) < 1e-12 * 3
        # rotation invariant of the Czjzek components
        assert abs(S[0] - abs(vzz) / 2 * math.sqrt(1 + eta * eta / 3)) < 1e-12 * 3


def test_axial_tensor_eta_zero_and_ordering():
    nmr = efg_stat.nmr_convention([-1.0, -1.0, 2.0])
    assert nmr == (-1.0, -1.0, 2.0, 0.0)
    nmr = efg_stat.nmr_convention([-2.0, 1.0, 1.0])
    assert nmr == (1.0, 1.0, -2.0, 0.0)
    # all three below 1e-5: eta forced to 0
    assert efg_stat.nmr_convention([-2e-6, 0.5e-6, 1.5e-6])[3] == 0.0
    # |Vzz| >= |Vyy| >= |Vxx| for a generic set, eta in [0, 1]
    vxx, vyy, vzz, eta = efg_stat.nmr_convention([-3.0, 0.5, 2.5])
    assert (vxx, vyy, vzz) == (0.5, 2.5, -3.0) and abs(eta - (0.5 - 2.5) / -3.0) < 1e-16


def test_non_traceless_large_trace_uses_zero_shift():
    # trace/3 above 1e-3: the reference resets diso to 0 and orders by |V|
    vxx, vyy, vzz, eta = efg_stat.nmr_convention([1.0, 2.0, 4.0])
    assert (vxx, vyy, vzz) == (1.0, 2.0, 4.0)


def test_two_charges_known_answer():
    # examples/ex4/run_ex4.sh:78-79: V1,xx = 2.0003749, V1,yy = V1,zz = -1.0001874
    t = np.array([[2.0003749, -1.0001874, -1.0001874, 0.0, 0.0, 0.0]])
    nmr, U, S = efg_stat.efg_nmr(t)
    assert nmr[0, 2] == 2.0003749 and nmr[0, 3] == 0.0
    assert U[0, 0] == -1.0001874 * 0.5


def test_czjzek_components():
    t = np.array([[1.0, 2.0, -3.0, 0.5, -0.25, 0.75]])
    U, S = efg_stat.czjzek(t)
    s3 = 1 / math.sqrt(3)
    assert np.allclose(U[0], [-1.5, -0.25 * s3, 0.75 * s3, 0.5 * s3, -1.0 * s3 / 2], rtol=0, atol=1e-16)
    assert abs(S[0] - math.sqrt(np.sum(U[0] ** 2))) < 1e-15


def random_traceless(n, rng, scale=1.0):
    a = rng.normal(0, scale, (n, 6))
    a[:, 2] = -(a[:, 0] + a[:, 1])
    return a


def test_statistics_and_histograms_bookkeeping():
    rng = np.random.default_rng(7)
    n, ntype = 300, 2
    itype = np.where(np.arange(n) % 3 == 0, 1, 2)
    efg = random_traceless(n, rng)
    d = efg_stat.efg_dist(efg, itype, ntype, vzzmin=-8.0, resvzz=0.1, reseta=0.05, umin=-6.0, resu=0.1, smax=8.0)
    counts = [n, int(np.sum(itype == 1)), int(np.sum(itype == 2))]
    for r in range(ntype + 1):
        assert d["vzz"][r].sum() == counts[r]
        assert d["eta"][r].sum() == counts[r]
        assert d["s"][r].sum() == counts[r]
        for k in range(5):
            assert d["u"][k, r].sum() == counts[r]
        assert d["u"][5, r].sum() == 4 * counts[r]
    # row statistics from the per-site values
    nmr = d["nmr"][0]
    for r in range(ntype + 1):
        sel = np.ones(n, bool) if r == 0 else itype == r
        v = nmr[sel, 2]
        st = d["stats"][0, r]
        assert abs(st[0] - min(0.0, v.min())) < 1e-15 and abs(st[1] - max(0.0, v.max())) < 1e-15
        assert abs(st[2] - v.mean()) < 1e-13 and abs(st[3] - np.abs(v).mean()) < 1e-13
        assert abs(st[4] - nmr[sel, 3].mean()) < 1e-13
        assert abs(st[5] - np.mean(v >= 0)) < 1e-15
        sig = math.sqrt(np.mean(v * v) - np.abs(v).mean() ** 2)
        assert abs(st[7] - sig) < 1e-12 and abs(st[6] - sig / np.abs(v).mean()) < 1e-12
        U = d["U"][0][sel]
        assert np.allclose(d["mU"][r], U.mean(axis=0), rtol=0, atol=1e-13)
        m2 = np.triu(U.T @ U)
        if r > 0:
            m2 = m2 / sel.sum()
        assert np.allclose(d["m2U"][r], m2, rtol=1e-12, atol=1e-12)
    # bins of one site by hand
    ia = 5
    kv = int((nmr[ia, 2] + 8.0) / 0.1) + 1
    assert d["vzz"][0, kv] >= 1 and d["vzz"][itype[ia], kv] >= 1


def test_configurations_carry_the_previous_averages():
    # two configurations: the reference zeroes its sums once, so the second
    # configuration's averages include the first configuration's averages
    rng = np.random.default_rng(9)
    n = 60
    itype = np.ones(n, int)
    e = np.stack([random_traceless(n, rng), random_traceless(n, rng)])
    kw = dict(vzzmin=-8.0, resvzz=0.1, reseta=0.05, umin=-6.0, resu=0.1, smax=8.0)
    d2 = efg_stat.efg_dist(e, itype, 1, **kw)
    a = efg_stat.efg_dist(e[0], itype, 1, **kw)
    b = efg_stat.efg_dist(e[1], itype, 1, **kw)
    assert np.array_equal(d2["stats"][0], a["stats"][0])
    v1 = a["nmr"][0][:, 2]
    v2 = b["nmr"][0][:, 2]
    assert abs(d2["stats"][1, 0, 2] - (v1.mean() + v2.sum()) / n) < 1e-13
    assert d2["stats"][1, 0, 0] == min(0.0, v1.min(), v2.min())
    for k in ("vzz", "eta", "u", "s"):
        assert np.array_equal(d2[k], a[k] + b[k])
    assert np.allclose(d2["mU"], (a["mU"] + b["mU"]) / 2, rtol=0, atol=1e-14)


def test_out_of_range_raises():
    rng = np.random.default_rng(2)
    efg = random_traceless(10, rng, scale=5.0)
    with pytest.raises(efg_stat.OutOfRange):
        efg_stat.efg_dist(efg, np.ones(10, int), 1, vzzmin=-0.5, resvzz=0.1, reseta=0.1, umin=-20, resu=0.1,
                          smax=40)


def test_bins_follow_check_tag():
    assert efg_stat.bins(-4.0, 0.1, 0.1, -3.0, 0.1, 5.0) == (80, 10, 60, 50)
