"""Force matching: a named parameter vector over the force-field tables, and
the loss + adjoint gradient behind torch.autograd.Function.

The reference fits nothing; this module is the host side of the engine's
differentiable path.  A ParamSpace ties each named scalar to one or more
entries of the mdff_params tables (all entries of one tie move together, and
the symmetric counterpart [b][a] of every pair entry is written too, as
field_check_tag's symmetrisation does, src/field.f90:316-339).  Its
gradient is the sum over the tied entries of the table derivatives that
mdff_batch_loss_grad returns (include/mdff_engine.h, mdff_param_grad).

The loss of a batch of B configurations (c) is

    L = 1/B sum_c [ w_force/(3 N_c) sum_i |F_i - F*_i|^2 + w_stress/9 sum_ab (tau_ab - tau*_ab)^2 ]

with F the total force (eV/A) and tau = tau_nonb + tau_coul (GPa).
"""
import copy
import ctypes as C

import numpy as np

from . import abi

# table name -> (kind, ParamGrad field)
_PAIR_TABLES = ("Abmhftd", "Bbmhftd", "Cbmhftd", "Dbmhftd", "BDbmhftd", "epsmor", "sigmamor", "rhomor")
_DAMP_TABLES = ("dip_pol_damp_b", "dip_pol_damp_c")


class Tie:
    """One named scalar: entries [(table, index tuple), ...] set to
    transform(value).  transform is 'id' or 'inv' (the table holds 1/value,
    e.g. Bbmhftd = 1/rho)."""

    def __init__(self, name, entries, transform="id"):
        self.name = name
        self.entries = list(entries)
        self.transform = transform

    def table_value(self, v):
        return 1.0 / v if self.transform == "inv" else v

    def dtable_dv(self, v):
        return -1.0 / (v * v) if self.transform == "inv" else 1.0


def _upper(idx):
    if len(idx) == 2:
        a, b = idx
        return (min(a, b), max(a, b))
    if len(idx) == 3:
        p, a, b = idx
        return (p, min(a, b), max(a, b))
    return idx


class ParamSpace:
    def __init__(self, ties):
        self.ties = list(ties)
        self.names = [t.name for t in self.ties]

    def __len__(self):
        return len(self.ties)

    def get(self, params):
        """Current values of the named parameters in params."""
        out = np.empty(len(self.ties))
        for k, t in enumerate(self.ties):
            tab, idx = t.entries[0]
            v = getattr(params, tab)
            for i in idx:
                v = v[i]
            out[k] = 1.0 / v if t.transform == "inv" else v
        return out

    def apply(self, params, theta):
        """A copy of params with the named parameters set to theta."""
        p = copy.deepcopy(params)
        for t, v in zip(self.ties, np.asarray(theta, dtype=np.float64)):
            tv = t.table_value(float(v))
            for tab, idx in t.entries:
                arr = getattr(p, tab)
                if len(idx) == 1:
                    arr[idx[0]] = tv
                elif len(idx) == 2:
                    a, b = idx
                    arr[a][b] = tv
                    arr[b][a] = tv
                else:
                    q, a, b = idx
                    arr[q][a][b] = tv
                    arr[q][b][a] = tv
        return p

    def project(self, grad, theta):
        """dL/dtheta from the table derivatives (abi.ParamGrad)."""
        out = np.zeros(len(self.ties))
        for k, t in enumerate(self.ties):
            s = 0.0
            for tab, idx in t.entries:
                arr = np.ctypeslib.as_array(getattr(grad, tab))
                s += arr[_upper(idx)] if len(idx) > 1 else arr[idx[0]]
            out[k] = s * t.dtable_dv(float(theta[k]))
        return out


def mgo_space(params):
    """The 12 force-matching parameters of the MgO polarisable-ion model
    (type 1 = O, type 2 = Mg): A, rho, C6, C8 for O-O and O-Mg, the O
    polarisability, the Tang-Toennies dipole damping b and c (every entry
    flagged in ldip_damping), and the dispersion damping b (BDbmhftd of every
    pair with A != 0)."""
    ties = []
    for lab, (i, j) in (("OO", (0, 0)), ("MgO", (0, 1))):
        ties.append(Tie("A_" + lab, [("Abmhftd", (i, j))]))
        ties.append(Tie("rho_" + lab, [("Bbmhftd", (i, j))], "inv"))
        ties.append(Tie("C6_" + lab, [("Cbmhftd", (i, j))]))
        ties.append(Tie("C8_" + lab, [("Dbmhftd", (i, j))]))
    ties.append(Tie("alpha_O", [("poldip_iso", (0,))]))
    nt = params.ntype
    damp = sorted({_upper((q, a, b)) for q in range(nt) for a in range(nt) for b in range(nt)
                   if params.ldip_damping[q][a][b]})
    ties.append(Tie("b_dip", [("dip_pol_damp_b", e) for e in damp]))
    ties.append(Tie("c_dip", [("dip_pol_damp_c", e) for e in damp]))
    disp = sorted({_upper((a, b)) for a in range(nt) for b in range(nt) if params.Abmhftd[a][b] != 0.0})
    ties.append(Tie("b_disp", [("BDbmhftd", e) for e in disp]))
    return ParamSpace(ties)


def batch_constants(natm, w_force, w_stress):
    """Per-configuration weights (c_force, c_stress) of the batch loss."""
    B = len(natm)
    return [(w_force / (3.0 * n * B), w_stress / (9.0 * B)) for n in natm]


def shard(confs, rank, world):
    """The configurations rank `rank` of `world` data-parallel ranks takes of
    a force-matching batch: largest first to the rank with the fewest atoms so
    far (ties to the lower rank), so every rank gets about the same number of
    atoms.  Returns (the rank's configurations, their indices in confs)."""
    order = sorted(range(len(confs)), key=lambda c: (-len(confs[c]["itype"]), c))
    load = [0] * world
    mine = []
    for c in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += len(confs[c]["itype"])
        if r == rank:
            mine.append(c)
    mine.sort()
    return [confs[c] for c in mine], mine


def allreduce_loss_grad(loss, grad, n_local, n_total, dist, device):
    """Whole-batch loss and dL/dtheta from each rank's shard.  A rank's Batch
    normalises by its own configuration count (the 1/B of the loss), so the
    whole batch's value is the sum over ranks of (n_local / n_total) times
    the shard's: one all-reduce of 1 + len(grad) doubles.  With dist None
    (one rank) the values come back unchanged."""
    import torch
    g = np.asarray(grad, dtype=np.float64)
    if dist is None:
        return float(loss), g.copy()
    w = float(n_local) / float(n_total)
    t = torch.tensor(np.concatenate([[w * float(loss)], w * g]), dtype=torch.float64, device=device)
    dist.all_reduce(t)
    v = t.cpu().numpy()
    return float(v[0]), v[1:].copy()


def _autograd_function():
    import torch

    class ForceMatchLoss(torch.autograd.Function):
        """loss(theta) of a Batch at the force field space.apply(base, theta).
        The forward pass runs the batch's forward and adjoint solves once and
        keeps dL/dtheta; backward returns it times the incoming gradient."""

        @staticmethod
        def forward(ctx, theta, batch, space, base):
            th = theta.detach().cpu().double().numpy()
            batch.set_params(space.apply(base, th))
            loss, g, _ = batch.loss_grad(want_grad=True)
            grad = torch.as_tensor(space.project(g, th), dtype=theta.dtype, device=theta.device)
            ctx.save_for_backward(grad)
            return theta.new_tensor(loss)

        @staticmethod
        def backward(ctx, gout):
            (grad,) = ctx.saved_tensors
            return gout * grad, None, None, None

    return ForceMatchLoss


_FML = None


def force_match_loss(theta, batch, space, base):
    """Differentiable force-matching loss (torch scalar) of batch at theta."""
    global _FML
    if _FML is None:
        _FML = _autograd_function()
    return _FML.apply(theta, batch, space, base)
