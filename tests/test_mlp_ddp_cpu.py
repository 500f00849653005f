"""Data-parallel training loop of the warm-start MLP (bevy_xpbd_b200/mlp_train.py) on CPU: two gloo ranks with
different local samples, the numpy oracle standing in for the gradient and Adam kernels. Both ranks must end with the
same parameters, equal to a single process that averages the two ranks' minibatch gradients at every step."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

STEPS, BATCH, LR, SEED = 4, 64, 1e-3, 7


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _local_data(rank):
    rng = np.random.default_rng(100 + rank)
    f = rng.normal(size=(500, 9)).astype(np.float32)
    f[:, 5:] = 0.0
    f[:, 5] = 1.0
    t = (rng.normal(size=500) * 0.5).astype(np.float32)
    return f, t


def _init():
    from oracle import mlp_oracle as MO
    p = (np.random.default_rng(0).normal(size=MO.N_PARAMS) * 0.1).astype(np.float32)
    norm = np.zeros(MO.N_NORM, np.float32)
    norm[9:18] = 1.0
    norm[19] = 1.0
    return p, norm


def _worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    from bevy_xpbd_b200 import mlp_train
    from oracle import mlp_oracle as MO
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        f, t = _local_data(rank)
        p, norm = _init()
        state = dict(p=p, m1=np.zeros_like(p), m2=np.zeros_like(p), step=0)

        def grad_fn(g, batch, seed):
            idx = MO.xorshift_indices(seed, batch, len(t))
            grad, loss = MO.gradients(state["p"], norm, f[idx], t[idx])
            g.copy_(torch.from_numpy(grad.astype(np.float32)))
            return loss

        def apply_fn(g, scale, lr):
            state["step"] += 1
            state["p"], state["m1"], state["m2"] = MO.adam(state["p"], state["m1"], state["m2"],
                                                          g.numpy() * np.float32(scale), state["step"], lr)

        g = torch.zeros(MO.N_PARAMS, dtype=torch.float32)
        losses = mlp_train.train_data_parallel(grad_fn, dist.all_reduce, apply_fn, STEPS, BATCH, LR, SEED, rank,
                                               world, g)
        out[rank] = dict(p=state["p"].tolist(), losses=losses)
    finally:
        dist.destroy_process_group()


def test_two_rank_training_keeps_parameters_identical():
    from bevy_xpbd_b200 import mlp_train
    from oracle import mlp_oracle as MO
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=300)
        assert pr.exitcode == 0
    p0, p1 = np.array(out[0]["p"], np.float32), np.array(out[1]["p"], np.float32)
    assert np.array_equal(p0, p1)
    # single-process reference: average of both ranks' gradients per step
    data = [_local_data(r) for r in range(world)]
    p, norm = _init()
    m1 = np.zeros_like(p)
    m2 = np.zeros_like(p)
    for step in range(STEPS):
        gs = []
        for r, (f, t) in enumerate(data):
            idx = MO.xorshift_indices(mlp_train.minibatch_seed(SEED, r, step), BATCH, len(t))
            gs.append(MO.gradients(p, norm, f[idx], t[idx])[0].astype(np.float32))
        g = (gs[0] + gs[1]) * np.float32(0.5)
        p, m1, m2 = MO.adam(p, m1, m2, g, step + 1, LR)
    np.testing.assert_allclose(p0, p, rtol=0, atol=1e-7)
    assert not np.array_equal(p, _init()[0])


def test_minibatch_seeds_distinct():
    from bevy_xpbd_b200 import mlp_train
    seeds = {mlp_train.minibatch_seed(3, r, s) for r in range(8) for s in range(1000)}
    assert len(seeds) == 8000
