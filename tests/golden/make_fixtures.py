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


if __name__ == "__main__":
    if not os.path.isdir(REF):
        sys.exit(f"reference tree not found at {REF}")
    ex1()
