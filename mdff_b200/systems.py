"""Seeded synthetic systems for the engine's five workloads.

The reference ships no input decks for these workloads, so each generator
builds the positions, cell, types, parameters and Maxwell-Boltzmann
velocities from a seed (numpy PCG64).  Where a workload description leaves a
value open, the value chosen here is stated in the generator's docstring and
used identically by the engine, the CPU oracle and the benchmark.

Every generator returns a dict with keys
  params  abi.Params (control-file units, see include/mdff_engine.h)
  itype   int32[N], 1-based, grouped by type as typeinfo_init requires
          (src/read_pos.f90:181-190)
  pos     float64[N,3] Cartesian positions (Angstrom, or sigma in reduced units)
  cell    float64[3,3], rows are the basis vectors a, b, c
  vel     float64[N,3] velocities in the reference's internal units
  meta    dict of the choices made
"""
import math

import numpy as np

from . import abi

AMU_G = 1.66053906660e-24        # grams per amu
BOLTZ_EV = 8.61734229648141e-05   # boltz_unit, src/constants.f90:86
MASS_O, MASS_MG, MASS_SI = 15.999, 24.305, 28.0855


def maxwell_boltzmann(rng, mass, temp_energy):
    """Velocities at temperature kB*T = temp_energy (energy units), zero net
    momentum, rescaled to the exact target like init_velocities
    (src/kinetic.f90:28-120)."""
    n = len(mass)
    v = rng.standard_normal((n, 3)) * np.sqrt(temp_energy / mass)[:, None]
    p = (v * mass[:, None]).sum(axis=0)
    v -= p / mass.sum()
    ekin = 0.5 * (mass[:, None] * v * v).sum()
    t_eff = 2.0 * ekin / (3.0 * n)
    v *= math.sqrt(temp_energy / t_eff)
    return v


def fcc_lattice(ncell, a):
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.arange(ncell)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    return ((cells[:, None, :] + base[None, :, :]).reshape(-1, 3)) * a


def lj_argon(ncell=5, rho=0.844, temp=0.72, seed=1234, trunc=abi.TRUNC_LINEAR):
    """Plain LJ argon, reduced units, NVE velocity Verlet.

    fcc ncell^3 cells (500 atoms at ncell=5), reduced density rho,
    epsilon = sigma = mass = 1, rc 2.5 sigma, Verlet skin 0.3 sigma,
    dt 0.005, Maxwell-Boltzmann velocities at T* = temp.  The truncation is
    'linear' (energy shifted at rc, src/field.f90:974-983)."""
    a = (4.0 / rho) ** (1.0 / 3.0)
    pos = fcc_lattice(ncell, a)
    L = ncell * a
    n = len(pos)
    p = abi.default_params()
    p.ntype = 1
    p.lnmlj = 1
    p.lreduced = 1
    p.cutshortrange = 2.5
    p.skindiff = 0.3
    p.trunc = trunc
    p.epslj[0][0] = 1.0
    p.sigmalj[0][0] = 1.0
    p.mass[0] = 1.0
    p.integrator = abi.NVE_VV
    p.dt = 0.005
    p.temp = temp
    rng = np.random.default_rng(seed)
    vel = maxwell_boltzmann(rng, np.ones(n), temp)
    return dict(params=p, itype=np.ones(n, np.int32), pos=pos, cell=np.eye(3) * L, vel=vel,
                meta=dict(workload="lj-argon", natm=n, box=L))


def random_min_sep(rng, n, L, dmin, max_tries=2000):
    """Uniform random positions in a cubic box with a minimum (periodic)
    separation, by sequential rejection on a cell grid."""
    nc = max(1, int(L // dmin))
    cw = L / nc
    grid = {}
    pos = np.empty((n, 3))
    k = 0
    tries = 0
    while k < n:
        tries += 1
        if tries > max_tries * n:
            raise RuntimeError("could not place atoms with the requested minimum separation")
        x = rng.random(3) * L
        c = tuple((x // cw).astype(int) % nc)
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in grid.get(((c[0] + dx) % nc, (c[1] + dy) % nc, (c[2] + dz) % nc), ()):
                        d = pos[j] - x
                        d -= L * np.round(d / L)
                        if d @ d < dmin * dmin:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            pos[k] = x
            grid.setdefault(c, []).append(k)
            k += 1
    return pos


def silica_bmh(n_si=512, density=2.2, temp=3000.0, seed=2024, dmin=1.2):
    """Rigid-ion Ewald silica melt: 512 Si (q=+2.4) + 1024 O (q=-1.2) placed
    uniformly at random with a 1.2 A minimum separation in a cubic box at
    2.2 g/cm3.  BMH pairs without damping (lbmhft): O-O A=1388.8 eV,
    rho=0.362 A, C=175 eV A^6; Si-O A=18003.8 eV, rho=0.2052 A,
    C=133.5 eV A^6; Si-Si A=0 (skipped, src/field.f90:2953).  rc 8 A,
    Ewald alpha 0.35 A^-1, kmax 8^3.  NVT Nose-Hoover chain 'nvt-nhcn' with
    nhc_n=2 (the reference refuses a chain of length 1, src/md.f90:302-305),
    Yoshida order 3, 2 multiple steps, thermostat time scale 0.1 ps; dt 1 fs.
    Type 1 = O, type 2 = Si."""
    n_o = 2 * n_si
    mass_tot = n_si * MASS_SI + n_o * MASS_O
    vol = mass_tot * AMU_G / density * 1e24
    L = vol ** (1.0 / 3.0)
    rng = np.random.default_rng(seed)
    pos = random_min_sep(rng, n_si + n_o, L, dmin)
    itype = np.array([1] * n_o + [2] * n_si, np.int32)
    p = abi.default_params()
    p.ntype = 2
    p.lbmhft = 1
    p.lcoulomb = 1
    p.cutshortrange = 8.0
    p.cutlongrange = 8.0
    p.mass[0], p.mass[1] = MASS_O, MASS_SI
    p.qch[0], p.qch[1] = -1.2, 2.4
    for (i, j, A, rho, Cc) in [(0, 0, 1388.8, 0.362, 175.0), (0, 1, 18003.8, 0.2052, 133.5)]:
        p.Abmhftd[i][j] = A
        p.Bbmhftd[i][j] = 1.0 / rho
        p.Cbmhftd[i][j] = Cc
        p.Dbmhftd[i][j] = 0.0
    p.alphaES = 0.35
    p.kES[0] = p.kES[1] = p.kES[2] = 8
    p.integrator = abi.NVT_NHCN
    p.nhc_n = 2
    p.nhc_yosh_order = 3
    p.nhc_mults = 2
    p.timesca_thermo = 0.1
    p.dt = 0.001
    p.temp = temp
    mass = np.where(itype == 1, MASS_O, MASS_SI)
    vel = maxwell_boltzmann(rng, mass, temp * BOLTZ_EV)
    return dict(params=p, itype=itype, pos=pos, cell=np.eye(3) * L, vel=vel,
                meta=dict(workload="silica-bmh", natm=len(itype), box=L))


# MgO polarisable-ion parameters.  The workload fixes the charges, the O
# polarisability and the damping constants but not the short-range
# constants; these are Lewis-Catlow-type formal-charge Buckingham constants
# with small added C6/C8 so that every one of the 12 fitted parameters has a
# non-zero value.
MGO_PARAMS = {
    "A": {("O", "O"): 22764.0, ("O", "Mg"): 1428.5},
    "rho": {("O", "O"): 0.149, ("O", "Mg"): 0.2945},
    "C6": {("O", "O"): 27.88, ("O", "Mg"): 5.0},
    "C8": {("O", "O"): 50.0, ("O", "Mg"): 10.0},
    "b_disp": 1.5,          # Tang-Toennies dispersion damping, A^-1
    "alpha_O": 1.6,         # A^3
    "b_dip": 1.8,           # Tang-Toennies dipole damping, A^-1
    "c_dip": 1.0,
    "k_dip": 4,
}


def mgo_params(rc, alpha, kmax, mp=None):
    """abi.Params of the MgO polarisable-ion model (type 1 = O, type 2 = Mg):
    BMHFTD pairs with Tang-Toennies dispersion damping (n = 6, 8), O
    polarisability with Tang-Toennies dipole damping for O-Mg and O-O."""
    mp = mp or MGO_PARAMS
    p = abi.default_params()
    p.ntype = 2
    p.lbmhftd = 1
    p.lcoulomb = 1
    p.cutshortrange = rc
    p.cutlongrange = rc
    p.mass[0], p.mass[1] = MASS_O, MASS_MG
    p.qch[0], p.qch[1] = -2.0, 2.0
    for (a, b), (i, j) in {("O", "O"): (0, 0), ("O", "Mg"): (0, 1)}.items():
        p.Abmhftd[i][j] = mp["A"][(a, b)]
        p.Bbmhftd[i][j] = 1.0 / mp["rho"][(a, b)]
        p.Cbmhftd[i][j] = mp["C6"][(a, b)]
        p.Dbmhftd[i][j] = mp["C8"][(a, b)]
        p.BDbmhftd[i][j] = mp["b_disp"]
    p.ldip_polar[0] = 1
    p.poldip_iso[0] = mp["alpha_O"]
    for other in (0, 1):
        p.ldip_damping[0][0][other] = 1
        p.dip_pol_damp_b[0][0][other] = mp["b_dip"]
        p.dip_pol_damp_c[0][0][other] = mp["c_dip"]
        p.dip_pol_damp_k[0][0][other] = mp["k_dip"]
    p.alphaES = alpha
    p.kES[0] = p.kES[1] = p.kES[2] = kmax
    p.algo_moment_from_pola = abi.POLA_PCG
    p.conv_tol_ind = 1e-8
    p.max_scf_pol_iter = 200
    p.doefg = 1
    return p


def rocksalt_sites(nx, ny, nz, a):
    """Simple-cubic grid of spacing a/2 with alternating O / Mg occupation."""
    h = a / 2.0
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), axis=-1).reshape(-1, 3)
    is_o = (g.sum(axis=1) % 2) == 0
    return g * h, is_o


def mgo_pim(grid=(10, 10, 30), a=4.212, jitter=0.05, rc=10.0, alpha=0.3, kmax=10, vacancy_frac=0.0,
            temp=2000.0, seed=7, integrator=abi.NVE_VV, nhc_n=3):
    """Polarisable-ion MgO.

    Sites on a simple-cubic grid of spacing a/2 (rock-salt occupation),
    grid=(10,10,30) gives the 3000-ion cell of 21.06 x 21.06 x 63.18 A
    (a '10x10x15 cell' of 3000 ions read as 10x10x30 sites of a/2);
    grid=(32,32,32) gives the 16^3 rock-salt conventional cells = 32768 sites.
    A fraction of sites is removed as equal numbers of O and Mg (charge
    neutral); positions are jittered by N(0, jitter^2).  Charges -2 (O) and
    +2 (Mg); BMHFTD + Tang-Toennies dispersion damping; O polarisability
    1.6 A^3 with Tang-Toennies dipole damping b=1.8, c=1.0, order 4; induced
    dipoles by PCG to an RMS residual of 1e-8."""
    rng = np.random.default_rng(seed)
    sites, is_o = rocksalt_sites(*grid, a)
    nvac = int(round(vacancy_frac * len(sites) / 2.0))
    keep = np.ones(len(sites), bool)
    if nvac:
        o_idx = np.flatnonzero(is_o)
        m_idx = np.flatnonzero(~is_o)
        keep[rng.choice(o_idx, nvac, replace=False)] = False
        keep[rng.choice(m_idx, nvac, replace=False)] = False
    sites, is_o = sites[keep], is_o[keep]
    order = np.concatenate([np.flatnonzero(is_o), np.flatnonzero(~is_o)])
    pos = sites[order] + rng.normal(0.0, jitter, (len(order), 3))
    n_o = int(is_o.sum())
    itype = np.array([1] * n_o + [2] * (len(order) - n_o), np.int32)
    cell = np.diag(np.array(grid, float) * a / 2.0)
    p = mgo_params(rc, alpha, kmax)
    p.integrator = integrator
    p.nhc_n = nhc_n
    p.nhc_yosh_order = 3
    p.nhc_mults = 2
    p.timesca_thermo = 0.1
    p.dt = 0.001
    p.temp = temp
    mass = np.where(itype == 1, MASS_O, MASS_MG)
    vel = maxwell_boltzmann(rng, mass, temp * BOLTZ_EV)
    return dict(params=p, itype=itype, pos=pos, cell=cell, vel=vel,
                meta=dict(workload="mgo-pim", natm=len(itype), grid=grid, box=np.diag(cell).tolist()))


def ewald_kmax_for(alpha, L, eps, rc):
    """kmax of the reference's DL_POLY-style estimate (src/field.f90:882-888)
    for a cubic box of side L at fixed alpha, accuracy eps and real-space
    cutoff rc (the clamped cutlongrange)."""
    tol = math.sqrt(abs(math.log(eps * rc)))
    tol1 = math.sqrt(-math.log(eps * rc * (2.0 * tol * alpha) ** 2))
    return int(round(0.25 + L * alpha * tol1 / math.pi))


def mgo_production(ncell=16, vacancy_frac=0.01, seed=11):
    """32768-site PIM MgO NVT production cell: 16^3 rock-salt cells, 1 %
    vacancies as equal Mg/O counts (N = 32440), rc 10 A, alpha 0.3 A^-1,
    kmax from the reference's estimate at eps 1e-7 (23 at this box), Nose-Hoover
    chain of length 3 at 2000 K, dt 1 fs, EFG every 10 steps."""
    L = ncell * 4.212
    kmax = ewald_kmax_for(0.3, L, 1e-7, 10.0)
    s = mgo_pim(grid=(2 * ncell,) * 3, rc=10.0, alpha=0.3, kmax=kmax, vacancy_frac=vacancy_frac,
                temp=2000.0, seed=seed, integrator=abi.NVT_NHCN, nhc_n=3)
    s["params"].efg_period = 10
    s["meta"].update(workload="mgo-pim-production", kmax=kmax)
    return s


def _grid_for(n, max_aspect=2.0):
    """Even site-grid dimensions (nx <= ny <= nz, nz/nx <= max_aspect) whose
    product P >= n is smallest, P - n even."""
    best = None
    for nx in range(2, 40, 2):
        for ny in range(nx, 40, 2):
            for nz in range(ny, int(max_aspect * nx) + 1, 2):
                P = nx * ny * nz
                if P < n or (P - n) % 2:
                    continue
                if best is None or P < best[0]:
                    best = (P, (nx, ny, nz))
    return best[1]


def mgo_batch(nconf=64, nmin=200, nmax=2000, dens=(3.3, 3.8), seed=99, jitter=0.12):
    """Batch of MgO PIM configurations for force matching.

    Atom counts are drawn uniformly from [nmin, nmax] (rounded down to even,
    half O and half Mg) and densities uniformly from dens (g/cm3).  Each
    configuration is a rock-salt site grid (spacing h, rock-salt occupation)
    in the smallest orthorhombic box of even grid dimensions holding at least
    n sites, with the surplus sites removed as equal numbers of O and Mg
    vacancies, h scaled so that the n atoms have the drawn density, and
    positions jittered by N(0, jitter^2): disordered hot-crystal snapshots,
    which keep the induced-dipole system well conditioned (uniformly random
    positions put O-O pairs within the polarisation-catastrophe distance).
    rc = min(10, half the smallest box width), alpha = 3.2 / rc, kmax from
    the reference's estimate at 1e-6."""
    rng = np.random.default_rng(seed)
    confs = []
    for c in range(nconf):
        n = int(rng.integers(nmin, nmax + 1)) // 2 * 2
        d = float(rng.uniform(*dens))
        nx, ny, nz = _grid_for(n)
        m = (n // 2) * (MASS_O + MASS_MG)
        vol = m * AMU_G / d * 1e24
        h = (vol / (nx * ny * nz)) ** (1.0 / 3.0)
        sites, is_o = rocksalt_sites(nx, ny, nz, 2.0 * h)
        nvac = (len(sites) - n) // 2
        keep = np.ones(len(sites), bool)
        if nvac:
            keep[rng.choice(np.flatnonzero(is_o), nvac, replace=False)] = False
            keep[rng.choice(np.flatnonzero(~is_o), nvac, replace=False)] = False
        sites, is_o = sites[keep], is_o[keep]
        order = np.concatenate([np.flatnonzero(is_o), np.flatnonzero(~is_o)])
        pos = sites[order] + rng.normal(0.0, jitter, (n, 3))
        box = np.array([nx, ny, nz], float) * h
        rc = min(10.0, 0.5 * box.min() - 1e-9)
        alpha = 3.2 / rc
        kmax = [max(3, ewald_kmax_for(alpha, float(L), 1e-6, rc)) for L in box]
        itype = np.array([1] * (n // 2) + [2] * (n // 2), np.int32)
        confs.append(dict(itype=itype, pos=pos, cell=np.diag(box), rc=rc, alpha=alpha, kmax=kmax, density=d))
    return confs
