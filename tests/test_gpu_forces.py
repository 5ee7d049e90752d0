"""Force evaluations on the GPU (FP64 path) against the reference's golden
data and the CPU oracle on identical seeded inputs.

Tolerances (FP64, different summation order and FMA contraction):
forces 1e-10 global relative, energies 1e-11 relative, stresses 1e-10,
dipoles / fields / EFG 1e-10 relative.
"""
import numpy as np
import pytest

import mdff_b200
import oracle
from mdff_b200 import abi, systems

from helpers import lj_params_ex1, rel

pytestmark = pytest.mark.gpu

F_TOL = 1e-10
E_TOL = 1e-11


def jittered(s, sigma=0.05, seed=0):
    """A lattice has zero net forces by symmetry; displace the atoms so the
    relative force norm is meaningful."""
    s = dict(s)
    s["pos"] = s["pos"] + np.random.default_rng(seed).normal(0.0, sigma, s["pos"].shape)
    return s


def both(p, s, erfc_mode=1):
    e = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"])
    o = oracle.Oracle(p, s["itype"], s["pos"], s["cell"], erfc_mode=erfc_mode)
    return e.engforce(), o.engforce()


def assert_energies(re, ro, keys, tol=E_TOL):
    for k in keys:
        a, b = re["e"][k], ro["e"][k]
        assert abs(a - b) <= tol * max(1.0, abs(b)), (k, a, b)


def test_ex1_golden_through_engine():
    p, d = lj_params_ex1()
    n = len(d["pos"])
    e = mdff_b200.Engine(p, np.ones(n, np.int32), d["pos"], d["cell"])
    r = e.engforce()
    assert abs(r["e"]["u_lj"] - float(d["u_lj"])) < 5e-6
    assert np.abs(r["f"] - d["force"]).max() < 1e-9
    assert np.abs(2.0 * r["tau_nonb"] - d["tau_nonb_printed"]).max() < 1e-7
    assert abs(r["e"]["utail"] - (-1.42129648126362)) < 1e-11


@pytest.mark.parametrize("trunc", [abi.TRUNC_NONE, abi.TRUNC_LINEAR, abi.TRUNC_QUADRATIC])
def test_lj_vs_oracle(trunc):
    s = jittered(systems.lj_argon(trunc=trunc))
    re, ro = both(s["params"], s)
    assert rel(re["f"], ro["f"]) < F_TOL
    assert_energies(re, ro, ["u_lj", "vir_lj"])
    assert rel(re["tau_nonb"], ro["tau_nonb"]) < 1e-10


def test_lj_nm_non_integer_exponents():
    s = jittered(systems.lj_argon())
    p = s["params"]
    p.plj[0][0] = 5.5
    p.qlj[0][0] = 9.0
    re, ro = both(p, s)
    assert rel(re["f"], ro["f"]) < F_TOL
    assert_energies(re, ro, ["u_lj"])


def test_morse_vs_oracle():
    s = jittered(systems.lj_argon())
    p = s["params"]
    p.lnmlj = 0
    p.lmorse = 1
    p.epsmor[0][0] = 0.8
    p.sigmamor[0][0] = 1.1
    p.rhomor[0][0] = 3.0
    re, ro = both(p, s)
    assert rel(re["f"], ro["f"]) < F_TOL
    assert_energies(re, ro, ["u_morse", "vir_morse"])


def test_silica_bmh_ewald_vs_oracle():
    s = systems.silica_bmh()
    p = s["params"]
    p.doefield = 1
    re, ro = both(p, s)
    assert rel(re["f"], ro["f"]) < F_TOL
    assert_energies(re, ro, ["u_bmhft", "u_coul", "u_dir", "u_rec", "u_self", "vir_bmhft"])
    assert rel(re["tau_nonb"], ro["tau_nonb"]) < 1e-10
    assert rel(re["tau_coul"], ro["tau_coul"]) < 1e-10
    assert rel(re["ef"], ro["ef"]) < 1e-10


@pytest.mark.parametrize("algo", [abi.POLA_SCF, abi.POLA_PCG])
def test_pim_vs_oracle(algo):
    s = systems.mgo_pim(grid=(8, 8, 8), rc=8.0, alpha=0.4, kmax=9)
    p = s["params"]
    p.algo_moment_from_pola = algo
    p.conv_tol_ind = 1e-10
    p.max_scf_pol_iter = 300
    p.doefield = 1
    p.doefg = 1
    re, ro = both(p, s)
    assert rel(re["mu"], ro["mu"]) < 1e-9
    assert rel(re["f"], ro["f"]) < 1e-9
    assert rel(re["efg"], ro["efg"]) < 1e-9
    assert rel(re["ef"], ro["ef"]) < 1e-9
    assert_energies(re, ro, ["u_bmhft", "u_coul", "u_pol", "u_dir", "u_rec", "u_self"], tol=1e-10)
    assert rel(re["tau_coul"], ro["tau_coul"]) < 1e-9
    assert re["e"]["scf_iter"] == ro["e"]["scf_iter"]


def test_pim_production_cell_scaled_down_pcg():
    # the production model at 1/8 of the cell (8^3 rock-salt cells, 1 % vacancies)
    s = systems.mgo_pim(grid=(16, 16, 16), rc=10.0, alpha=0.3, kmax=12, vacancy_frac=0.01, seed=3)
    p = s["params"]
    re, ro = both(p, s)
    assert rel(re["f"], ro["f"]) < 1e-9
    assert rel(re["mu"], ro["mu"]) < 1e-8
    assert_energies(re, ro, ["u_coul", "u_bmhft"], tol=1e-10)


def test_two_charges_efg_known_answer():
    p = abi.default_params()
    p.ntype = 2
    p.lcoulomb = 1
    p.lreduced = 1
    p.cutlongrange = 1000.0
    p.qch[0] = 1.0
    p.qch[1] = -1.0
    p.alphaES = 0.8
    p.kES[0] = p.kES[1] = p.kES[2] = 11
    p.doefg = 1
    e = mdff_b200.Engine(p, np.array([1, 2], np.int32), np.array([[0.5, 0, 0], [-0.5, 0, 0]]), np.eye(3) * 10.0)
    efg = e.engforce()["efg"]
    # examples/ex4/run_ex4.sh:78-79 (Nymand & Linse): V1,xx = 2.0003749, V1,yy = -1.0001874
    assert abs(efg[0, 0] - 2.0003749) < 1e-7
    assert abs(efg[0, 1] - (-1.0001874)) < 1e-7


def test_reference_erfc_mode_matches_oracle():
    s = systems.silica_bmh()
    p = s["params"]
    p.erfc_ref = 1
    re, ro = both(p, s, erfc_mode=0)
    assert rel(re["f"], ro["f"]) < F_TOL
    assert_energies(re, ro, ["u_coul"])


def test_no_verlet_list_all_pairs():
    s = systems.silica_bmh()
    p = s["params"]
    p.lvnlist = 0
    re, ro = both(p, s)
    assert rel(re["f"], ro["f"]) < F_TOL
    assert_energies(re, ro, ["u_coul", "u_bmhft"])


def test_static_dipoles_and_polarisable():
    s = systems.mgo_pim(grid=(6, 6, 6), rc=6.0, alpha=0.55, kmax=8)
    p = s["params"]
    p.dip[1][0] = 0.05
    p.dip[1][2] = -0.02
    p.conv_tol_ind = 1e-11
    p.doefg = 1
    re, ro = both(p, s)
    assert rel(re["f"], ro["f"]) < 1e-9
    assert rel(re["efg"], ro["efg"]) < 1e-9
    assert_energies(re, ro, ["u_coul"], tol=1e-10)


def test_config3_pim_3000_ion_cell_vs_oracle():
    """Config 3's cell itself: 3000 MgO ions on the 10 x 10 x 30 site grid
    (21.06 x 21.06 x 63.18 A), rc 10 A, alpha 0.3, kmax 10^3 (4630 k-vectors),
    polarisable O with Tang-Toennies damping, dipoles by PCG: forces,
    energies, stress, dipoles and EFG of the FP64 engine against the oracle."""
    s = systems.mgo_pim()
    p = s["params"]
    p.conv_tol_ind = 1e-11
    p.doefg = 1
    assert len(s["itype"]) == 3000
    a = mdff_b200.Engine(p, s["itype"], s["pos"], s["cell"]).engforce()
    b = oracle.Oracle(p, s["itype"], s["pos"], s["cell"]).engforce()
    assert rel(a["f"], b["f"]) < 1e-9
    assert rel(a["mu"], b["mu"]) < 1e-9
    assert rel(a["efg"], b["efg"]) < 1e-9
    assert rel(a["tau_coul"], b["tau_coul"]) < 1e-9
    assert abs(a["e"]["u_coul"] - b["e"]["u_coul"]) < 1e-11 * abs(b["e"]["u_coul"])
    assert abs(a["e"]["u_bmhft"] - b["e"]["u_bmhft"]) < 1e-11 * abs(b["e"]["u_bmhft"])
