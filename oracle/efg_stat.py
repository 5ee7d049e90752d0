"""CPU restatement of MDFF's EFG post-processing (efg_stat and nmr_convention,
src/efg.f90:2057-2650) over one or more configurations.

Test infrastructure: tests and the bench's CPU leg use it as the checker of the
engine's mdff_efg_nmr / mdff_efg_dist; nothing in the product imports it.

The reference ships no efg_stat output for any example, so this restatement is
pinned by closed-form cases instead (tests/test_oracle_efg.py): diagonal
tensors rotated by known rotations, whose principal values, Vzz and eta are
known exactly.  Principal values come from LAPACK through numpy's eigvalsh in
place of the reference's DSYEV (both return them ascending).

Arrays follow the reference's index meaning with 0-based rows: nmr[:, 0..3] =
Vxx, Vyy, Vzz, eta; U[:, 0..4] = U1..U5; per-type rows 0 (all sites), 1..ntype
from 1-based itype.
"""
import math

import numpy as np


def czjzek(efg):
    """U and S of the tensors efg [n][6] (xx yy zz xy xz yz): src/efg.f90:2235-2244."""
    sq3 = 1.0 / math.sqrt(3.0)
    sq32 = sq3 * 0.5
    xx, yy, zz, xy, xz, yz = (efg[:, k] for k in range(6))
    U = np.stack([zz * 0.5, xz * sq3, yz * sq3, xy * sq3, (xx - yy) * sq32], axis=1)
    S = np.zeros(len(efg))
    for k in range(5):
        S = S + U[:, k] * U[:, k]
    return U, np.sqrt(S)


def nmr_convention(eig):
    """src/efg.f90:2546-2620: (Vxx, Vyy, Vzz, eta) from three principal values."""
    e1, e2, e3 = (float(x) for x in eig)
    diso = (e1 + e2 + e3) / 3.0
    if abs(diso) != 0.0 and abs(diso) > 1e-3:
        diso = 0.0
    a1, a2, a3 = abs(e1 - diso), abs(e2 - diso), abs(e3 - diso)
    if a1 >= a2 and a1 >= a3:
        d11 = e1
        d22, d33 = (e2, e3) if a2 >= a3 else (e3, e2)
    elif a2 >= a1 and a2 >= a3:
        d11 = e2
        d22, d33 = (e1, e3) if a1 >= a3 else (e3, e1)
    else:
        d11 = e3
        d22, d33 = (e1, e2) if a1 >= a2 else (e2, e1)
    vxx, vyy, vzz = d33, d22, d11
    eta = (vxx - vyy) / vzz if vzz != 0.0 else 0.0
    if vxx == vyy:
        eta = 0.0
    if vzz == 0.0:
        eta = 0.0
    if abs(vxx) < 1.0e-5 and abs(vyy) < 1.0e-5 and abs(vzz) < 1.0e-5:
        eta = 0.0
    return vxx, vyy, vzz, eta


def efg_nmr(efg):
    """Per site (src/efg.f90:2225-2270): nmr [n][4], U [n][5], S [n]."""
    efg = np.asarray(efg, dtype=np.float64)
    U, S = czjzek(efg)
    nmr = np.empty((len(efg), 4))
    for i, t in enumerate(efg):
        m = np.array([[t[0], t[3], t[4]], [t[3], t[1], t[5]], [t[4], t[5], t[2]]])
        nmr[i] = nmr_convention(np.linalg.eigvalsh(m))
    return nmr, U, S


def bins(vzzmin, resvzz, reseta, umin, resu, smax):
    """efg_check_tag (src/efg.f90:233-236): PANvzz, PANeta, PANU, PANS."""
    return (int((2.0 * abs(vzzmin)) / resvzz), int(1.0 / reseta), int((2.0 * abs(umin)) / resu),
            int(smax / resu))


class OutOfRange(ValueError):
    """A site outside a distribution's range (the reference STOPs there)."""


def efg_dist(efg, itype, ntype, vzzmin, resvzz, reseta, umin, resu, smax):
    """Statistics and distributions over configurations (src/efg.f90:2159-2440).

    efg: [natm][6] or [nconf][natm][6]; itype is 1-based.  Returns dict:
    stats [nconf][ntype+1][8] (vzzmin, vzzmax, <Vzz>, <|Vzz|>, <eta>,
    P(Vzz>=0), rho_z, sigma) formed as the reference's configuration loop forms
    them: the sums are zeroed once before the loop, so each configuration's
    sums add to the previous configuration's averages before the division, and
    the extrema run over all configurations starting from 0; mU [ntype+1][5] and
    m2U [ntype+1][5][5] over all configurations (row 0 of m2U the plain sum, as
    the reference leaves it); the integer histograms vzz, eta, u
    [6][ntype+1][PANU+1], s, summed over the configurations; and the per-site
    nmr, U, S of every configuration.
    """
    efg = np.asarray(efg, dtype=np.float64)
    if efg.ndim == 2:
        efg = efg[None]
    nconf = efg.shape[0]
    itype = np.asarray(itype, dtype=np.int64)
    n = len(itype)
    nt1 = ntype + 1
    PV, PE, PU, PS = bins(vzzmin, resvzz, reseta, umin, resu, smax)
    vzzm = np.zeros(nt1); vzzma = np.zeros(nt1); etam = np.zeros(nt1); vzzsq = np.zeros(nt1)
    pvzz = np.zeros(nt1); vmin = np.zeros(nt1); vmax = np.zeros(nt1)
    natmi = np.array([n] + [int(np.sum(itype == t)) for t in range(1, nt1)], dtype=float)
    mU = np.zeros((nt1, 5)); m2U = np.zeros((nt1, 5, 5))
    hv = np.zeros((nt1, PV + 1), dtype=np.int32)
    he = np.zeros((nt1, PE + 1), dtype=np.int32)
    hu = np.zeros((6, nt1, PU + 1), dtype=np.int32)
    hs = np.zeros((nt1, PS + 1), dtype=np.int32)
    stats = np.zeros((nconf, nt1, 8))
    nmrs, Us, Ss = [], [], []
    for ic in range(nconf):
        nmr, U, S = efg_nmr(efg[ic])
        nmrs.append(nmr); Us.append(U); Ss.append(S)
        for ia in range(n):
            it = int(itype[ia])
            v, e = nmr[ia, 2], nmr[ia, 3]
            for r in (0, it):
                mU[r] += U[ia]
                for a in range(5):
                    for b in range(a, 5):
                        m2U[r, a, b] += U[ia, a] * U[ia, b]
                vzzm[r] += v
                etam[r] += e
                vzzma[r] += abs(v)
                if v <= vmin[r]:
                    vmin[r] = v
                if v >= vmax[r]:
                    vmax[r] = v
                if v >= 0.0:
                    pvzz[r] += 1.0
                vzzsq[r] += v * v
        for r in range(nt1):
            c = natmi[r]
            if c > 0:
                vzzm[r] /= c; vzzsq[r] /= c; vzzma[r] /= c; etam[r] /= c; pvzz[r] /= c
            sig = math.sqrt(vzzsq[r] - vzzma[r] * vzzma[r])
            rho = sig / vzzma[r] if vzzma[r] != 0.0 else 0.0
            stats[ic, r] = (vmin[r], vmax[r], vzzm[r], vzzma[r], etam[r], pvzz[r], rho, sig)
        for ia in range(n):
            it = int(itype[ia])
            for ui in range(5):
                ku = int((U[ia, ui] - umin) / resu) + 1
                if ku < 0 or ku > PU:
                    raise OutOfRange(f"U{ui + 1} of site {ia + 1}: bin {ku} outside 0..{PU}")
                hu[ui, 0, ku] += 1
                hu[ui, it, ku] += 1
                if ui != 0:
                    hu[5, 0, ku] += 1
                    hu[5, it, ku] += 1
            ks = int(S[ia] / resu) + 1
            if ks < 0 or ks > PS:
                raise OutOfRange(f"S of site {ia + 1}: bin {ks} outside 0..{PS}")
            hs[0, ks] += 1
            hs[it, ks] += 1
            kv = int((nmr[ia, 2] - vzzmin) / resvzz) + 1
            ke = int(nmr[ia, 3] / reseta)
            if kv < 0 or kv > PV:
                raise OutOfRange(f"Vzz of site {ia + 1}: bin {kv} outside 0..{PV}")
            if ke < 0 or ke > PE:
                raise OutOfRange(f"eta of site {ia + 1}: bin {ke} outside 0..{PE}")
            hv[0, kv] += 1
            hv[it, kv] += 1
            he[0, ke] += 1
            he[it, ke] += 1
    for r in range(nt1):
        den = nconf * natmi[r]
        if den > 0:
            mU[r] /= den
            if r > 0:
                m2U[r] /= den
    return {"nmr": np.array(nmrs), "U": np.array(Us), "S": np.array(Ss), "stats": stats, "mU": mU, "m2U": m2U,
            "vzz": hv, "eta": he, "u": hu, "s": hs}
