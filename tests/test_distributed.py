"""Rank logic of rmetis_b200.distributed on CPU: gloo process groups of 2 and 3
ranks, with the oracle as the single-process partitioner. The striping of
attempts, the choice of the winning rank (src/partition/kway.rs:54-138) and
the footprint sharding of a batch are checked against the rules applied
directly to every attempt."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from rmetis_b200 import generators as G


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_partition(graph, nparts, tpwgts, ubvec, options):
    import rmetis_b200 as rmb
    from oracle import oracle as O
    rc, part, obj = O.part_graph_kway(graph.xadj, graph.adjncy, nparts, vwgt=graph.vwgt, adjwgt=graph.adjwgt,
                                      ncon=graph.ncon, tpwgts=tpwgts, ubvec=ubvec, options=options.c_array())
    assert rc == 1
    return rmb.PartitionResult(part=part, objval=int(obj))


def _graph():
    import rmetis_b200 as rmb
    x, a, v, w = G.grid3d(9, 8, 7, weights_seed=3)
    return rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w)


def _worker_ncuts(rank, world, port, ncuts, out_dir, rtype="greedy"):
    import torch.distributed as dist
    import rmetis_b200 as rmb
    from rmetis_b200 import distributed as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = _graph()
        rt = rmb.RType.Fm if rtype == "fm" else rmb.RType.Greedy
        o = rmb.Options(rtype=rt, seed=5, ncuts=ncuts, iptype=rmb.IpType.Random)
        res = D.part_graph_kway_ranks(g, 6, options=o, partition=_oracle_partition)
        np.save(os.path.join(out_dir, f"part{rank}.npy"), res.part)
        np.save(os.path.join(out_dir, f"obj{rank}.npy"), np.array([res.objval]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,ncuts,rtype", [(2, 5, "greedy"), (3, 7, "greedy"), (2, 1, "greedy"), (2, 4, "fm")])
def test_ncuts_striped_over_ranks(tmp_path, world, ncuts, rtype):
    import rmetis_b200 as rmb
    mp.spawn(_worker_ncuts, args=(world, _free_port(), ncuts, str(tmp_path), rtype), nprocs=world, join=True)
    parts = [np.load(tmp_path / f"part{r}.npy") for r in range(world)]
    objs = [int(np.load(tmp_path / f"obj{r}.npy")[0]) for r in range(world)]
    assert len(set(objs)) == 1 and all((p == parts[0]).all() for p in parts)
    # The reference's rule applied to every attempt directly.
    g = _graph()
    runs = []
    for a in range(ncuts):
        rt = rmb.RType.Fm if rtype == "fm" else rmb.RType.Greedy
        o = rmb.Options(rtype=rt, seed=5 + a, ncuts=1, iptype=rmb.IpType.Random)
        runs.append(_oracle_partition(g, 6, None, None, o))
    local = {}
    for r in range(world):
        for a in range(r, ncuts, world):
            if r not in local or runs[a].objval < local[r].objval:
                local[r] = runs[a]
    gmin = min(x.objval for x in local.values())
    winner = min(r for r, x in local.items() if x.objval == gmin)
    assert objs[0] == gmin
    assert (parts[0] == local[winner].part).all()


def _worker_batch(rank, world, port, out_dir):
    import torch.distributed as dist
    import rmetis_b200 as rmb
    from rmetis_b200 import distributed as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        graphs, ks = _batch()
        o = rmb.Options(rtype=rmb.RType.Greedy, seed=2)
        seen = []

        def batch(gs, kk, ub, opts):
            seen.extend(g.nvtxs for g in gs)
            return [_oracle_partition(g, k, None, ub, opts) for g, k in zip(gs, kk)]
        res = D.part_graph_kway_batch_ranks(graphs, ks, options=o, batch=batch)
        np.save(os.path.join(out_dir, f"objs{rank}.npy"), np.array([r.objval for r in res]))
        np.save(os.path.join(out_dir, f"seen{rank}.npy"), np.array(seen))
    finally:
        dist.destroy_process_group()


def _batch():
    import rmetis_b200 as rmb
    graphs, ks = [], []
    for i, n in enumerate([400, 1500, 900, 2500, 300, 1200, 700]):
        x, a, w, _ = G.rgg2d(n, 10 + i, 8.0)
        graphs.append(rmb.Graph(n, 1, x, a, adjwgt=w))
        ks.append(2 + i % 4)
    return graphs, ks


def test_batch_sharded_over_ranks(tmp_path):
    import rmetis_b200 as rmb
    from rmetis_b200 import distributed as D
    world = 2
    mp.spawn(_worker_batch, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    graphs, ks = _batch()
    objs = [np.load(tmp_path / f"objs{r}.npy") for r in range(world)]
    assert (objs[0] == objs[1]).all()
    o = rmb.Options(rtype=rmb.RType.Greedy, seed=2)
    expect = [_oracle_partition(g, k, None, None, o).objval for g, k in zip(graphs, ks)]
    assert list(objs[0]) == expect
    # Every graph ran on exactly one rank, the one the footprint rule names.
    owner = D.assign_by_footprint([(g.nvtxs, len(g.adjncy), k, 1) for g, k in zip(graphs, ks)], world)
    for r in range(world):
        seen = sorted(np.load(tmp_path / f"seen{r}.npy").tolist())
        assert seen == sorted(g.nvtxs for g, o_ in zip(graphs, owner) if o_ == r)


def test_assign_by_footprint_balances():
    from rmetis_b200 import distributed as D
    sizes = [(10_000 * (i + 1), 60_000 * (i + 1), 8, 1) for i in range(9)]
    owner = D.assign_by_footprint(sizes, 3)
    load = [sum(s[0] for s, o in zip(sizes, owner) if o == r) for r in range(3)]
    assert max(load) - min(load) <= 10_000 * 3
    assert D.assign_by_footprint(sizes, 1) == [0] * 9
