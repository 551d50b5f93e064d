"""Work across ranks (one process per GPU, torch.distributed).

One graph's multilevel pipeline does not shard: every rank runs whole
partitions on its own GPU. What spreads over ranks is the independent work:

* the ncuts attempts of one call, striped as in the reference's MPI path
  (src/partition/kway.rs:54-138): rank r runs the attempts a with
  a = r (mod world) (seed + a), keeps its first strict minimum, and the
  ranks agree on the global minimum cut with an all-reduce(min). The
  partition of the lowest rank that holds that minimum is the result (the
  reference gathers the holders' partitions on rank 0 and takes the first
  non-empty one in rank order, then broadcasts it; broadcasting from that
  rank directly gives the same partition);
* the graphs of a batch, assigned to ranks by estimated footprint (largest
  first, to the rank with the least assigned so far), each rank running its
  share as one batch on its own GPU.

The partition function is a parameter so that the rank logic can be checked
with any single-process partitioner; by default it is the GPU library's.
"""
from __future__ import annotations

import copy
from typing import Callable, Sequence

import numpy as np
import torch
import torch.distributed as dist

INT32_MAX = 2**31 - 1


def _default_partition(graph, nparts, tpwgts, ubvec, options):
    import rmetis_b200 as rmb
    return rmb.part_graph_kway(graph, nparts, tpwgts=tpwgts, ubvec=ubvec, options=options)


def _tensor_device(group) -> torch.device:
    backend = dist.get_backend(group)
    if backend == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def part_graph_kway_ranks(graph, nparts: int, tpwgts=None, ubvec=None, options=None, group=None,
                          partition: Callable | None = None):
    """Best of options.ncuts attempts, striped over the ranks of `group`
    (src/partition/kway.rs:54-138). Every rank returns the same
    PartitionResult."""
    import rmetis_b200 as rmb
    partition = partition or _default_partition
    options = options or rmb.Options()
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    dev = _tensor_device(group)

    if options.seed != 0 and options.seed + max(1, options.ncuts) - 1 > INT32_MAX:
        raise ValueError("seed + ncuts - 1 does not fit the options array's 32-bit seed slot")
    best = None
    for a in range(rank, max(1, options.ncuts), world):
        o = copy.copy(options)
        o.ncuts = 1
        # Seed of attempt a (kway.rs:55-61); seed 0 draws fresh entropy per attempt.
        o.seed = options.seed + a if options.seed != 0 else int(np.random.SeedSequence().generate_state(1)[0] >> 1)
        res = partition(graph, nparts, tpwgts, ubvec, o)
        if best is None or res.objval < best.objval:
            best = res

    local = best.objval if best is not None else INT32_MAX
    t = torch.tensor([local], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    gmin = int(t.item())
    holder = torch.tensor([rank if (best is not None and best.objval == gmin) else world], dtype=torch.int64,
                          device=dev)
    dist.all_reduce(holder, op=dist.ReduceOp.MIN, group=group)
    winner = int(holder.item())
    if rank == winner:
        part = torch.from_numpy(np.ascontiguousarray(best.part, dtype=np.int32)).to(dev)
    else:
        part = torch.empty(graph.nvtxs, dtype=torch.int32, device=dev)
    src = dist.get_global_rank(group, winner) if group is not None else winner
    dist.broadcast(part, src=src, group=group)
    return rmb.PartitionResult(part=part.cpu().numpy(), objval=gmin)


def assign_by_footprint(sizes: Sequence[tuple[int, int, int, int]], world: int) -> list[int]:
    """Rank of each graph (n, m, nparts, ncon): largest estimated footprint
    first, each to the rank with the least footprint assigned so far (ties to
    the lower rank)."""
    fp = [4 * (n + 1) * 2.5 + 8 * m * 2.5 + 4 * n * c * 2.5 + 88 * n + 8 * m + 24 * k * c for n, m, k, c in sizes]
    order = sorted(range(len(sizes)), key=lambda i: (-fp[i], i))
    load = [0.0] * world
    owner = [0] * len(sizes)
    for i in order:
        r = min(range(world), key=lambda j: (load[j], j))
        owner[i] = r
        load[r] += fp[i]
    return owner


def part_graph_kway_batch_ranks(graphs, nparts, ubvec=None, options=None, group=None,
                                batch: Callable | None = None):
    """Partition the graphs of a batch over the ranks of `group`, each rank
    running its share as one batch (by default part_graph_kway_batch on its
    GPU). Returns, on every rank, the list of all results in input order."""
    import rmetis_b200 as rmb
    batch = batch or (lambda gs, ks, ub, o: rmb.part_graph_kway_batch(gs, ks, ubvec=ub, options=o))
    graphs = list(graphs)
    ks = [nparts] * len(graphs) if np.isscalar(nparts) else [int(k) for k in nparts]
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    owner = assign_by_footprint([(g.nvtxs, len(g.adjncy), k, g.ncon) for g, k in zip(graphs, ks)], world)
    mine = [i for i in range(len(graphs)) if owner[i] == rank]
    local = batch([graphs[i] for i in mine], [ks[i] for i in mine], ubvec, options) if mine else []
    payload = [(i, r.objval, np.asarray(r.part, dtype=np.int32)) for i, r in zip(mine, local)]
    gathered = [None] * world
    dist.all_gather_object(gathered, payload, group=group)
    out = [None] * len(graphs)
    for items in gathered:
        for i, obj, part in items:
            out[i] = rmb.PartitionResult(part=part, objval=int(obj))
    return out
