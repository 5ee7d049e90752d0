"""Shared helpers for the parity tests."""
import numpy as np

from mdff_b200 import abi


def rel(a, b):
    """Global relative difference ||a-b|| / ||b|| (the engine's error norm)."""
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def lj_params_ex1():
    d = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "ex1_final.npz"))
    p = abi.default_params()
    p.ntype = 1
    p.lnmlj = 1
    p.cutshortrange = float(d["cutshortrange"])
    p.trunc = abi.TRUNC_LINEAR
    p.epslj[0][0] = float(d["epslj"])
    p.sigmalj[0][0] = float(d["sigmalj"])
    p.mass[0] = float(d["mass"])
    return p, d


def copy_params(p):
    q = abi.Params()
    __import__("ctypes").pointer(q)[0] = p
    return q
