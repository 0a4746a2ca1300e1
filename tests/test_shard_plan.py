"""Host side of the sharded run, on the CPU with two gloo processes: every rank
partitions the same mesh, and the exchange plans agree pairwise (the block a
rank sends to a neighbour lists the same mortars, in the same order, as the
block that neighbour receives into its ghost faces)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from dsem_b200 import mesh
    from dsem_b200.shard import partition
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        box = mesh.Box(4, 3, 2, 2)
        part = np.random.default_rng(7).integers(0, world, box.nel)
        mine = partition(box.desc(), part)[rank]
        info = {"rank": rank, "plan": mine["plan"], "ghosts": mine["ghosts"],
                "elements": mine["elements"].tolist(), "nmort": int(mine["desc"]["nmort"])}
        allinfo = [None] * world
        dist.all_gather_object(allinfo, info)
        ok = True
        for a in allinfo:
            for nb, g0, n in a["plan"]:
                b = allinfo[nb]
                seg = [x for x in b["plan"] if x[0] == a["rank"]]
                ok &= len(seg) == 1 and seg[0][2] == n
                ok &= a["ghosts"][g0:g0 + n] == b["ghosts"][seg[0][1]:seg[0][1] + n]
        els = sorted(e for a in allinfo for e in a["elements"])
        ok &= els == list(range(box.nel))
        # every global mortar appears once (local) or twice (cut, once per side)
        cnt = sum(a["nmort"] for a in allinfo)
        ncut = sum(len(a["ghosts"]) for a in allinfo)
        ok &= cnt == box.nmort + ncut // 2 and ncut % 2 == 0
        q.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


def test_exchange_plans_agree_across_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {0: True, 1: True}
