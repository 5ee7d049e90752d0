"""The multi-rank paths, run as two gloo ranks on the CPU: the plumbing of
bench.py (one process per GPU under torchrun: process group set-up, the
barrier, the max over ranks of the timed region and the whole-job
throughput), and the data-parallel force-matching batch (configurations
sharded over the ranks, one all-reduce of the loss and its gradient)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import torch
    import bench
    w, r, local, dist = bench.dist_setup(world, backend="gloo")
    dev = torch.device("cpu")
    bench.barrier(dist, dev)
    # rank r processed (r + 1) * 1000 units in (r + 1) * 0.5 s
    units, secs = (r + 1) * 1000.0, (r + 1) * 0.5
    rate = bench.whole_job_rate(units, secs, dist, dev)
    tmax = bench.max_over_ranks(secs, dist, dev)
    bench.barrier(dist, dev)
    dist.destroy_process_group()
    out.put((r, w, rate, tmax))


def test_two_gloo_ranks_whole_job_rate():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, rate, tmax in res:
        assert w == world
        assert tmax == 1.0                      # slowest rank
        assert rate == pytest.approx(3000.0)    # (1000 + 2000) units / 1.0 s


def test_single_process_needs_no_group():
    import bench
    w, r, local, dist = bench.dist_setup(1)
    assert dist is None and w == 1
    assert bench.whole_job_rate(500.0, 2.0, None, None) == 250.0
    assert bench.max_over_ranks(3.0, None, None) == 3.0


def _cfg_params(p, c):
    from mdff_b200 import fit
    q = fit.ParamSpace([]).apply(p, [])
    q.cutshortrange = q.cutlongrange = c["rc"]
    q.alphaES = c["alpha"]
    for d in range(3):
        q.kES[d] = c["kmax"][d]
    return q


def _shard_problem():
    import numpy as np
    import oracle
    from mdff_b200 import fit, systems
    confs = systems.mgo_batch(nconf=5, nmin=60, nmax=130, seed=9)
    base = systems.mgo_params(6.0, 0.5, 6)
    base.conv_tol_ind = 1e-12
    base.max_scf_pol_iter = 300
    space = fit.mgo_space(base)
    theta0 = space.get(base)
    theta_t = theta0 * (1.0 + 0.05 * np.random.default_rng(2).standard_normal(len(theta0)))
    targets = []
    for c in confs:
        r = oracle.Oracle(_cfg_params(space.apply(base, theta_t), c), c["itype"], c["pos"], c["cell"]).engforce()
        targets.append((r["f"], r["tau_nonb"] + r["tau_coul"]))
    return confs, base, space, theta0, targets


def _shard_loss(confs, targets, base, space, theta0):
    """The batch loss and dL/dtheta of confs (normalised by their own count),
    through the oracle's adjoint."""
    import oracle
    from mdff_b200 import abi, fit
    consts = fit.batch_constants([len(c["itype"]) for c in confs], 1.0, 0.01)
    g = abi.ParamGrad()
    L = 0.0
    for c, (ft, tt), (cf, cs) in zip(confs, targets, consts):
        o = oracle.Oracle(_cfg_params(base, c), c["itype"], c["pos"], c["cell"])
        l, g, _ = o.loss_grad(ft, tt, cf, cs, g)
        L += l
    return L, space.project(g, theta0)


def _batch_rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import torch
    import bench
    from mdff_b200 import fit
    w, r, local, dist = bench.dist_setup(world, backend="gloo")
    confs, base, space, theta0, targets = _shard_problem()
    mine, idx = fit.shard(confs, r, w)
    L, g = _shard_loss(mine, [targets[i] for i in idx], base, space, theta0)
    L, g = fit.allreduce_loss_grad(L, g, len(mine), len(confs), dist, torch.device("cpu"))
    dist.destroy_process_group()
    out.put((r, L, list(g), idx, sum(len(c["itype"]) for c in mine)))


def test_sharded_force_matching_batch_two_gloo_ranks():
    """Data-parallel force matching: the configurations of one batch split
    over two ranks (balanced by atoms), each rank's loss and gradient
    normalised by its own count, then one all-reduce of the 13 values weighted
    by the ranks' shares.  Equals the whole batch on one rank (oracle adjoint
    on both sides) to rounding."""
    import numpy as np
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=600) for _ in range(world)])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    confs, base, space, theta0, targets = _shard_problem()
    L1, g1 = _shard_loss(confs, targets, base, space, theta0)
    idx = sorted(i for r in res for i in r[3])
    assert idx == list(range(len(confs)))                       # every configuration once
    atoms = [r[4] for r in res]
    assert max(atoms) - min(atoms) <= max(len(c["itype"]) for c in confs)
    for r, L, g, _, _ in res:
        assert L == res[0][1] and g == res[0][2]                 # every rank holds the same result
        assert abs(L - L1) <= 1e-12 * abs(L1)
        assert np.linalg.norm(np.asarray(g) - g1) <= 1e-11 * np.linalg.norm(g1)


def test_shard_single_rank_is_identity():
    from mdff_b200 import fit, systems
    confs = systems.mgo_batch(nconf=6, nmin=60, nmax=130, seed=9)
    mine, idx = fit.shard(confs, 0, 1)
    assert idx == list(range(6)) and len(mine) == 6
    L, g = fit.allreduce_loss_grad(2.5, [1.0, 2.0], 6, 6, None, None)
    assert L == 2.5 and list(g) == [1.0, 2.0]
