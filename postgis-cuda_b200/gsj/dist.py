"""ST_ClusterIntersecting across GPUs: one process per GPU (torch.distributed), every rank holding the same layer.

Each rank clusters its probe shard (gsj_cluster with shard = rank: every intersecting pair is found by exactly one
shard), the ranks all-gather their root arrays (the one exchange of the path: NCCL on GPUs, gloo on CPU), and every
rank joins the gathered forests on its GPU (gsj_cluster_merge) into the whole layer's roots.
"""
from __future__ import annotations

import numpy as np


def gather_forests(root: np.ndarray, device: int | None = None) -> list[np.ndarray]:
    """Every rank's root array, in rank order (all-gather over the default process group). With NCCL the exchange
    runs on CUDA device ``device`` (default: the current one), which must be this rank's GPU."""
    import torch
    import torch.distributed as dist
    ws = dist.get_world_size()
    if dist.get_backend() == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    else:
        dev = torch.device("cpu")
    t = torch.from_numpy(root.astype(np.int64, copy=False)).to(dev)
    parts = [torch.empty_like(t) for _ in range(ws)]
    dist.all_gather(parts, t)
    return [p.cpu().numpy().astype(np.uint32) for p in parts]


def cluster_sharded(engine, layer, nparent: int | None = None, refine_mode=1):
    """(roots of the whole layer, this rank's stats): this rank's shard clustered, forests gathered and joined."""
    import torch.distributed as dist
    rank, ws = dist.get_rank(), dist.get_world_size()
    root, st = engine.cluster(layer, nparent, refine_mode=refine_mode, shard=rank, nshards=ws)
    return engine.cluster_merge(gather_forests(root, engine.device)), st
