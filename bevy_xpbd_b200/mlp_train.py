"""Data-parallel training of the warm-start MLP: one process per GPU.

Each rank collects samples from its own shard of cloths (`ClothComputePlugin.mlp_collect`). Per optimizer step every
rank computes the gradient of a minibatch drawn from its own samples, the 4,865 gradient values are summed over the
ranks with one all-reduce, and every rank applies the same Adam step with the sum scaled by 1/ranks — so the
parameters stay identical on all ranks without ever being broadcast after the start. The normalisation (feature and
target mean/std) is fitted on rank 0's samples and broadcast once, before the first step.

The loop is written against three callables (gradient, all-reduce, apply) so the same code runs with the CUDA
library and NCCL (`train_on_gpus`) and, in the tests, with CPU stand-ins over `gloo`.
"""
from __future__ import annotations

from typing import Callable

MLP_PARAMS = 4865


def minibatch_seed(seed: int, rank: int, step: int) -> int:
    """Seed of rank `rank`'s minibatch at `step`: distinct per rank and step, reproducible."""
    return (seed * 1_000_003 + rank * 7_919 + step) & 0xFFFFFFFFFFFFFFFF


def train_data_parallel(grad_fn: Callable, all_reduce: Callable, apply_fn: Callable, steps: int, batch: int,
                        lr: float, seed: int, rank: int, world: int, grads) -> list:
    """grad_fn(grads, batch, seed) fills `grads` with this rank's minibatch gradient (returns a loss handle or None);
    all_reduce(grads) sums it over the ranks in place; apply_fn(grads, scale, lr) applies one Adam step."""
    losses = []
    for step in range(steps):
        losses.append(grad_fn(grads, batch, minibatch_seed(seed, rank, step)))
        if world > 1:
            all_reduce(grads)
        apply_fn(grads, 1.0 / world, lr)
    return losses


def train_on_gpus(plugin, steps: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0, group=None):
    """Data-parallel training of `plugin`'s MLP over the ranks of `group` (torch.distributed, NCCL), one GPU per
    rank. The plugin must hold samples (`mlp_collect`) and an initialised network with the same seed on every rank.
    Returns this rank's per-step mean squared errors (standardised targets)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    device = torch.device("cuda", torch.cuda.current_device())
    # normalisation from rank 0, identical everywhere
    params, norm = plugin.mlp_params()
    if rank == 0:
        plugin.mlp_fit_normalization()
        params, norm = plugin.mlp_params()
    if world > 1:
        t = torch.tensor(norm, device=device)
        dist.broadcast(t, 0, group=group)
        norm = t.cpu().numpy()
        plugin.mlp_set_params(params, norm)
    stream = torch.cuda.Stream(device)
    grads = torch.zeros(MLP_PARAMS, dtype=torch.float32, device=device)
    loss = torch.zeros(steps, dtype=torch.float32, device=device)
    plugin.set_stream(stream.cuda_stream)  # library launches and the all-reduce share one stream
    try:
        with torch.cuda.stream(stream):
            def grad_fn(g, b, s):
                k = grad_fn.step
                grad_fn.step += 1
                plugin.mlp_minibatch_gradients(b, s, g.data_ptr(), loss[k:].data_ptr())
            grad_fn.step = 0
            train_data_parallel(grad_fn, lambda g: dist.all_reduce(g, group=group),
                                lambda g, scale, rate: plugin.mlp_apply_gradients(g.data_ptr(), scale, rate),
                                steps, batch, lr, seed, rank, world, grads)
        stream.synchronize()
    finally:
        plugin.set_stream(None)
    return (loss.cpu().numpy() / batch).tolist()
