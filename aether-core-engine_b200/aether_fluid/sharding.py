"""Ensembles sharded over the GPUs of one node: one process per GPU.

The instances of an ensemble are independent simulations, so nothing of the
data path crosses GPUs.  Each rank takes a share of the instances, balanced by
cell count, and advances it as one batched `Ensemble` on its own device.  At
the end a host-side gather returns every instance's telemetry and solver
reports to rank 0, in the order of the original instance list.  No collective
touches device memory; the only exchange is `gather_object` over the process
group's backend (gloo or NCCL).
"""
from __future__ import annotations

import numpy as np


def shard_instances(cells: list[int], world: int) -> list[list[int]]:
    """Instance indices per rank, balanced by cell count: largest first, each
    to the rank with the fewest cells so far (lowest rank on ties).  Every
    index appears exactly once; each rank's list is in increasing order.  A
    rank may get no instance when there are fewer instances than ranks."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    if any(c <= 0 for c in cells):
        raise ValueError("every instance needs a positive cell count")
    load = [0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for idx in sorted(range(len(cells)), key=lambda i: (-cells[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(idx)
        load[r] += cells[idx]
    return [sorted(s) for s in shards]


def run_sharded(specs, steps: int, dist=None, runner=None, **ensemble_kw):
    """Advances `specs` for `steps` steps over the ranks of `dist` (the
    torch.distributed module with an initialised process group, or None for one
    process).  Returns, on rank 0, (telemetry [steps, len(specs), 8], solve
    infos [steps][len(specs)], per-rank results) in the original instance order;
    other ranks return None.

    `runner(local_specs, steps)` advances one rank's share and returns
    (telemetry [steps, k, 8], infos [steps][k], extra dict); the default builds
    an `Ensemble` on the current device (the runner is a parameter so that the
    partition and gather can be exercised without a GPU)."""
    world = dist.get_world_size() if dist else 1
    rank = dist.get_rank() if dist else 0
    shards = shard_instances([s.cells for s in specs], world)
    mine = shards[rank]
    if runner is None:
        runner = _ensemble_runner(**ensemble_kw)
    if mine:
        tel, infos, extra = runner([specs[i] for i in mine], steps)
    else:
        tel, infos, extra = np.zeros((steps, 0, 8)), [[] for _ in range(steps)], {}
    part = {"rank": rank, "indices": mine, "tel": np.asarray(tel), "infos": infos,
            "extra": extra}
    if dist is None:
        parts = [part]
    else:
        parts = [None] * world if rank == 0 else None
        dist.gather_object(part, parts, dst=0)
    if rank != 0:
        return None
    n = len(specs)
    tel_all = np.zeros((steps, n, 8))
    info_all = [[None] * n for _ in range(steps)]
    for p in parts:
        for k, idx in enumerate(p["indices"]):
            tel_all[:, idx, :] = p["tel"][:, k, :]
            for t in range(steps):
                info_all[t][idx] = p["infos"][t][k]
    return tel_all, info_all, [{"rank": p["rank"], "indices": p["indices"], **p["extra"]}
                               for p in parts]


def _ensemble_runner(precision=None, autotune=True, **kw):
    """Builds this rank's `Ensemble`, autotunes it (the tuner restores the
    state it times on), and advances it; `run_seconds` is the host time of the
    advance alone, which returns only once the telemetry is on the host."""
    def run(local_specs, steps):
        import time
        from .ensemble import Ensemble
        from .solver import Precision
        ens = Ensemble(local_specs, precision=Precision.MIXED if precision is None
                       else precision, **kw)
        try:
            choice = ens.autotune() if autotune else None
            t0 = time.perf_counter()
            tel, infos = ens.run(steps)
            seconds = time.perf_counter() - t0
            return tel, infos, {"autotune_choice": choice, "info": ens.info(),
                                "run_seconds": seconds,
                                "cells": int(sum(s.cells for s in local_specs))}
        finally:
            ens.close()
    return run
