"""Streaming of frames from the device (mdff_writer_*) and whole-state
checkpoints (mdff_checkpoint_*), through the C ABI.

Writer: frames written during MD must hold exactly the engine's state at the
moment of mdff_writer_frame -- velocities and forces bit for bit, positions
folded into the cell (a lattice translation of the engine's, fractional
coordinates in [-1/2, 1/2]) -- and the formatted files must be byte for
byte the host formatter's output of the same values.

Checkpoint: a run stopped, saved, restored into a fresh engine and continued
must reproduce the uninterrupted run bit for bit (positions, velocities,
thermodynamics), on the FP64 path (LJ, Nose-Hoover chain) and on the mixed
path (polarisable-ion MgO, tensor-core k-space, ASPC predictor, NHC).
"""
import numpy as np
import pytest

import mdff_b200
from mdff_b200 import abi, io, systems

pytestmark = pytest.mark.gpu


def lj():
    s = systems.lj_argon(ncell=4)
    p = s["params"]
    p.integrator = abi.NVT_NHCN
    p.nhc_n = 3
    p.temp = 1.2
    p.timesca_thermo = 0.5
    return s


def pim(mixed=True):
    s = systems.mgo_pim(grid=(8, 8, 8), rc=6.0, alpha=0.5, kmax=8, temp=1500.0, integrator=abi.NVT_NHCN,
                        vacancy_frac=0.02, seed=5)
    p = s["params"]
    p.precision = abi.PREC_MIXED if mixed else abi.PREC_FP64
    p.algo_ext_dipole = abi.EXT_ASPC
    p.extrapolate_order = 3
    p.doefg = 1
    p.doefield = 1
    return s


def engine(s):
    return mdff_b200.Engine(s["params"], s["itype"], s["pos"], s["cell"])


def test_trajff_stream_holds_the_engine_state(tmp_path):
    s = lj()
    e = engine(s)
    e.md_start(s["vel"])
    pf, pb, pc = tmp_path / "TRAJFF.txt", tmp_path / "TRAJFF.bin", tmp_path / "CONTFF"
    wf = e.writer(pf, "TRAJFF", 1, "rvf", system="LJ argon", labels=["Ar"], nslot=3)
    wb = e.writer(pb, "TRAJFF", 0, "rvf", system="LJ argon", labels=["Ar"], nslot=2)
    wc = e.writer(pc, "CONTFF", 1, system="LJ argon", labels=["Ar"])
    states = []
    for _ in range(6):
        r = e.step(3, thermo=False)
        states.append((r["pos"], e.velocities(), r["f"]))
        wf.frame()
        wb.frame()
        wc.frame()
    for w in (wf, wb, wc):
        w.close()
    frames = io.read_trajff(pb, 0, "rvf")
    assert len(frames) == 6
    cell = np.asarray(s["cell"])
    for fr, (pos, vel, f) in zip(frames, states):
        assert np.array_equal(fr["v"], vel)
        assert np.array_equal(fr["f"], f)
        frac = fr["r"] @ np.linalg.inv(cell)
        assert np.all(np.abs(frac) <= 0.5 + 1e-12)
        shift = (fr["r"] - pos) @ np.linalg.inv(cell)
        assert np.max(np.abs(shift - np.round(shift))) < 1e-9
        assert fr["natm"] == e.n and fr["labels"] == ["Ar"] and fr["system"] == "LJ argon"
    # the formatted stream and CONTFF are the host formatter's text of the same values
    h = io.header("LJ argon", ["Ar"], natmi=[e.n], cell=frames[0]["cell"].T, natm=e.n)
    it = np.ones(e.n, np.int32)
    cols = [np.concatenate([fr["r"].T, fr["v"].T, fr["f"].T]) for fr in frames]
    assert pf.read_bytes() == b"".join(io.format_frame("TRAJFF", 1, "rvf", h, it, c) for c in cols)
    hc = io.header("LJ argon", ["Ar"], natmi=[e.n], cell=frames[0]["cell"], natm=e.n)
    assert pc.read_bytes() == io.format_frame("CONTFF", 1, "rvf", hc, it, cols[-1])


def test_field_files_stream(tmp_path):
    s = pim(mixed=False)
    e = engine(s)
    out = e.engforce()
    paths = {k: tmp_path / k for k in ("EFGALL.bin", "EFGALL.txt", "DIPFF", "EFALL")}
    ws = [e.writer(paths["EFGALL.bin"], "EFGALL", 0, system="MgO", labels=["O", "Mg"]),
          e.writer(paths["EFGALL.txt"], "EFGALL", 1, system="MgO", labels=["O", "Mg"]),
          e.writer(paths["DIPFF"], "DIPFF", 1, system="MgO", labels=["O", "Mg"]),
          e.writer(paths["EFALL"], "EFALL", 1, system="MgO", labels=["O", "Mg"])]
    for w in ws:
        w.frame()
        w.close()
    (b,) = io.read_efgall(paths["EFGALL.bin"], 0)
    assert np.array_equal(b["efg"], out["efg"])
    (t,) = io.read_efgall(paths["EFGALL.txt"], 1)
    assert np.allclose(t["efg"], out["efg"], rtol=2e-16 * 8, atol=1e-300)
    assert t["natmi"] == [int(np.sum(s["itype"] == 1)), int(np.sum(s["itype"] == 2))]
    (d,) = io.read_vectors(paths["DIPFF"])
    assert np.allclose(d["values"], out["mu"], rtol=1e-15, atol=1e-300)
    (f,) = io.read_vectors(paths["EFALL"])
    assert np.allclose(f["values"], out["ef"], rtol=1e-15, atol=1e-300)


def test_one_slot_ring_keeps_every_frame_in_order(tmp_path):
    s = lj()
    e = engine(s)
    e.md_start(s["vel"])
    p = tmp_path / "TRAJFF"
    w = e.writer(p, "TRAJFF", 0, "rvn", system="ring", labels=["Ar"], nslot=1)
    vels = []
    for _ in range(25):
        e.step(1, thermo=False)
        vels.append(e.velocities())
        w.frame()
    w.close()
    frames = io.read_trajff(p, 0, "rvn")
    assert len(frames) == 25
    for fr, v in zip(frames, vels):
        assert np.array_equal(fr["v"], v)


def test_writer_refuses_what_the_reference_cannot_write(tmp_path):
    s = lj()
    e = engine(s)
    with pytest.raises(mdff_b200.EngineError) as ei:
        e.writer(tmp_path / "EFGALL", "EFGALL", 1, labels=["Ar"])      # no Coulomb, no EFG
    assert ei.value.code == abi.E_STATE
    s2 = pim(mixed=False)
    e2 = engine(s2)
    with pytest.raises(mdff_b200.EngineError) as ei:
        e2.writer(tmp_path / "DIPFF", "DIPFF", 0, labels=["O", "Mg"])  # formatted only
    assert ei.value.code == abi.E_UNSUPPORTED


def continued(s, n1, n2):
    e = engine(s)
    e.md_start(s["vel"])
    e.step(n1, thermo=False)
    r = e.step(n2)
    return r, e.velocities()


def restarted(s, n1, n2):
    e = engine(s)
    e.md_start(s["vel"])
    e.step(n1, thermo=False)
    ck = e.checkpoint()
    e.close()
    e2 = engine(s)
    e2.restore(ck)
    r = e2.step(n2)
    return r, e2.velocities()


@pytest.mark.parametrize("case", ["lj_fp64_nhc", "pim_fp64_aspc_nhc", "pim_mixed_aspc_nhc"])
def test_checkpoint_restart_is_bit_identical(case):
    s = {"lj_fp64_nhc": lj, "pim_fp64_aspc_nhc": lambda: pim(False), "pim_mixed_aspc_nhc": lambda: pim(True)}[case]()
    n1, n2 = (30, 30) if case.startswith("lj") else (7, 8)
    (ra, va), (rb, vb) = continued(s, n1, n2), restarted(s, n1, n2)
    assert np.array_equal(ra["pos"], rb["pos"])
    assert np.array_equal(va, vb)
    assert np.array_equal(ra["f"], rb["f"])
    assert ra["thermo"] == rb["thermo"]
    assert sum(t["nlist_rebuilt"] for t in ra["thermo"]) >= 0


def test_checkpoint_of_another_setup_is_refused():
    s = lj()
    e = engine(s)
    e.md_start(s["vel"])
    ck = e.checkpoint()
    s2 = lj()
    s2["params"].temp = 1.5
    e2 = engine(s2)
    with pytest.raises(mdff_b200.EngineError) as ei:
        e2.restore(ck)
    assert ei.value.code == abi.E_ARG
    with pytest.raises(mdff_b200.EngineError):
        e.restore(ck[:-8])


def test_efgcalc_over_a_trajff(tmp_path):
    # calc = 'efg' (efgcalc, src/efg.f90:325-660): the configurations of a
    # TRAJFF, the EFG of each (FP64, with induced dipoles) against the
    # oracle's, EFGALL written and read back, efg_stat over all of them
    import oracle
    s = pim(mixed=False)
    s["params"].conv_tol_ind = 1e-12      # both dipole solves well below the comparison
    s["params"].max_scf_pol_iter = 500
    e = engine(s)
    rng = np.random.default_rng(4)
    confs = [np.asarray(s["pos"]) + rng.normal(0.0, 0.05, np.shape(s["pos"])) for _ in range(3)]
    labels = ["O", "Mg"]
    it = np.asarray(s["itype"], dtype=np.int32)
    natmi = [int(np.sum(it == 1)), int(np.sum(it == 2))]
    h = io.header("MgO", labels, natmi=natmi, cell=np.asarray(s["cell"]).T, natm=e.n)
    traj = tmp_path / "TRAJFF"
    traj.write_bytes(b"".join(io.format_frame("TRAJFF", 1, "rnn", h, it, np.ascontiguousarray(r.T)) for r in confs))
    dist = abi.EfgDistParams()
    # ranges wide enough for every site (the tensors carry coul_unit, V/A^2)
    dist.vzzmin, dist.resvzz, dist.reseta, dist.umin, dist.resu, dist.smax = -200.0, 0.5, 0.05, -200.0, 0.5, 300.0
    efg, st = e.efgcalc(str(traj), dist, efgall=str(tmp_path / "EFGALL"), labels=labels, system="MgO")
    assert efg.shape == (3, e.n, 6)
    for k, r in enumerate(io.read_trajff(str(traj))):
        ref = oracle.Oracle(s["params"], s["itype"], r["r"], r["cell"]).engforce()["efg"]
        assert np.max(np.abs(efg[k] - ref)) < 1e-8 * np.max(np.abs(ref))
    back = io.read_efgall(str(tmp_path / "EFGALL"), 1)
    assert len(back) == 3
    for k in range(3):
        assert np.max(np.abs(back[k]["efg"] - efg[k])) <= 1e-11 * np.max(np.abs(efg[k]))
    direct = e.efg_dist(dist, efg)
    for key in ("vzz", "eta", "u", "s"):
        assert np.array_equal(st[key], direct[key])
    assert np.array_equal(st["stats"], direct["stats"])
