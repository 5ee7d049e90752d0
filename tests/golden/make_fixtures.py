"""Generate the golden fixtures of the reference's own outputs.

Reads the reference tree (default /root/reference, or $MDFF_REFERENCE) and
writes small .npz files next to this script.  Run once where the reference is
available; the fixtures are committed so the GPU tests never read the
reference at run time.

ex1_contff_head.txt, ex1_contff.sha256 -- the first 24 lines of
examples/ex1/ref/CONTFF and the SHA-256 of the whole file.

ex1_final.npz -- examples/ex1/ref: the final configuration of the 256-atom
LJ argon NVE run (CONTFF: positions, velocities and forces at step 5000,
12 significant digits), its energy (OSZIFF line of step 5000), virial
pressure and final stress tensor (stdout).  The run used ctrunc='linear',
rc 8.5 A, eps 0.010323576 eV, sigma 3.405 A.  That build printed
TAU_NONB without the 0.5 factor the current source has
(src/field.f90:1306-1314), i.e. twice the virial stress.

ex4_cluster.npz -- examples/ex4: the 9-ion cluster of TRAJFF.cluster (8 A
ions, 1 B ion) in its 10 A cubic box, the charges of the example's Ewald run
(qch = 0.1 -0.8, cutlongrange 5, lautoES, epsw 1e-8, lefg_vasp_sign) and the
GULP table run_ex4.sh prints for it (diagonalised EFG xx yy zz in V/A^2 and
the asymmetry, 4 decimals).

ex0_fcc.npz -- examples/ex0: the 256-atom FCC argon configuration of POSFF
(direct coordinates, 20.993868 A box), the LJ 12-6 potential of control.F
(eps 0.010323576 eV, sigma 3.405 A, no truncation, rc 10 A) and DL_POLY's
static result for it in examples/ex0/dl_poly: STATIS's eng_vdw and vir_vdw
(7 digits) and OUTPUT's long-range corrections (energy in eV, pressure in
katm).
"""
import os
import re
import sys

import numpy as np

REF = os.environ.get("MDFF_REFERENCE", "/root/reference")
OUT = os.path.dirname(os.path.abspath(__file__))


def ex1():
    base = os.path.join(REF, "examples", "ex1", "ref")
    lines = open(os.path.join(base, "CONTFF")).read().split("\n")
    n = int(lines[0])
    cell = np.array([[float(x) for x in lines[k].split()] for k in (2, 3, 4)])
    data = np.array([[float(x) for x in l.split()[1:]] for l in lines[9:9 + n]])
    osz = open(os.path.join(base, "OSZIFF")).read().split("\n")
    last = [l for l in osz if l.startswith(" step =      5000") and "Utot" in l][0]
    u = float(re.search(r"Utot\s+=\s+(\S+)", last).group(1))
    last2 = [l for l in osz if l.startswith(" step =      5000") and "Pvir_vdw" in l][0]
    pvir = float(re.search(r"Pvir_vdw\s+=\s+(\S+)", last2).group(1))
    out = open(os.path.join(base, "stdout")).read().split("\n")
    k = [i for i, l in enumerate(out) if "stress tensor of final configuration" in l][0]
    k = [i for i in range(k, len(out)) if out[i].strip() == "TAU_NONB"][0]
    tau = np.array([[float(x) for x in out[k + 1 + r].split()] for r in range(3)])
    np.savez(os.path.join(OUT, "ex1_final.npz"), cell=cell, pos=data[:, 0:3], vel=data[:, 3:6], force=data[:, 6:9],
             u_lj=u, pvir_gpa=pvir, tau_nonb_printed=tau, cutshortrange=8.5, epslj=0.010323576, sigmalj=3.405,
             mass=39.95)
    print("ex1_final.npz", n, u, pvir)
    # the CONTFF text itself (write_CONTFF's layout): its first lines and the
    # digest of the whole file, for the formatter's byte-for-byte check
    import hashlib
    raw = open(os.path.join(base, "CONTFF"), "rb").read()
    head = b"\n".join(raw.split(b"\n")[:24]) + b"\n"
    open(os.path.join(OUT, "ex1_contff_head.txt"), "wb").write(head)
    open(os.path.join(OUT, "ex1_contff.sha256"), "w").write(hashlib.sha256(raw).hexdigest() + "\n")
    print("ex1_contff_head.txt", len(raw))


def ex4_cluster():
    base = os.path.join(REF, "examples", "ex4")
    lines = open(os.path.join(base, "TRAJFF.cluster")).read().split("\n")
    n = int(lines[0])
    cell = np.array([[float(x) for x in lines[k].split()] for k in (2, 3, 4)])
    labels = lines[6].split()
    rows = [l.split() for l in lines[9:9 + n]]
    itype = np.array([labels.index(r[0]) + 1 for r in rows], np.int32)
    pos = np.array([[float(x) for x in r[1:4]] for r in rows])
    script = open(os.path.join(base, "run_ex4.sh")).read().split("\n")
    k = [i for i, l in enumerate(script) if "Diagonalised EFGs" in l][0]
    table = []
    for l in script[k + 1:]:
        m = re.match(r'echo "\s+(\d+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)"', l)
        if m:
            table.append([float(m.group(j)) for j in range(2, 6)])
        elif table:
            break
    np.savez(os.path.join(OUT, "ex4_cluster.npz"), cell=cell, pos=pos, itype=itype, qch=np.array([0.1, -0.8]),
             cutlongrange=5.0, epsw=1e-8, gulp=np.array(table))
    print("ex4_cluster.npz", n, len(table))


def ex0_fcc():
    base = os.path.join(REF, "examples", "ex0")
    lines = open(os.path.join(base, "POSFF")).read().split("\n")
    n = int(lines[0])
    cell = np.array([[float(x) for x in lines[k].split()] for k in (2, 3, 4)])
    frac = np.array([[float(x) for x in l.split()[1:4]] for l in lines[9:9 + n]])
    st = open(os.path.join(base, "dl_poly", "STATIS")).read().split("\n")
    v = [float(x) for x in " ".join(st[3:6]).split()]
    eng_vdw, vir_vdw = v[3], v[12]
    out = open(os.path.join(base, "dl_poly", "OUTPUT")).read()
    elrc = float(re.search(r"vdw energy\s+(\S+)", out).group(1))
    plrc = float(re.search(r"vdw pressure\s+(\S+)", out).group(1))
    np.savez(os.path.join(OUT, "ex0_fcc.npz"), cell=cell, frac=frac, epslj=0.010323576, sigmalj=3.405,
             cutshortrange=10.0, mass=39.95, eng_vdw=eng_vdw, vir_vdw=vir_vdw, elrc_ev=elrc, plrc_katm=plrc)
    print("ex0_fcc.npz", n, eng_vdw, vir_vdw, elrc, plrc)


if __name__ == "__main__":
    if not os.path.isdir(REF):
        sys.exit(f"reference tree not found at {REF}")
    ex1()
    ex4_cluster()
    ex0_fcc()
