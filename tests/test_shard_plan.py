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


def test_plan_of_dsem_metis_partition(box22):
    """The planner on DSEM's own partition of the 22^3 case: the 100-way METIS split it ships
    (DNS-22p8.graph.part.100, read by metis_file.f90; kept in tests/golden/mesh_22cube_p8.json).
    Every element lands in exactly one part, every mortar whose elements share a part appears
    once and every mortar between parts on both sides, as one ghost face each, and for every
    pair of neighbouring parts the block one sends lists the same mortars, in the same order,
    as the block the other receives.  Each part numbers its elements as DSEM's ranks do: the
    local indices equal grid_distribution.dat, which DSEM wrote for this partition
    (read_restart, restart.f90:486-496)."""
    import base64
    import json

    from dsem_b200.shard import partition
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mesh_22cube_p8.json")) as f:
        fx = json.load(f)
    decode = lambda k: np.frombuffer(base64.b64decode(fx[k]), dtype=np.uint8).astype(np.int64)
    part, dsem_local = decode("metis_part_100_b64"), decode("grid_distribution_local_b64")
    assert part.shape == (box22.nel,) and part.max() == 99
    parts = partition(box22.desc(), part)
    els = np.concatenate([p["elements"] for p in parts])
    assert np.array_equal(np.sort(els), np.arange(box22.nel))
    local = np.zeros(box22.nel, dtype=np.int64)
    for p in parts:
        local[p["elements"]] = np.arange(1, len(p["elements"]) + 1)
    assert np.array_equal(local, dsem_local)
    m = box22.mortar
    crossing = part[m[:, 0] - 1] != part[m[:, 1] - 1]
    count = np.zeros(box22.nmort, dtype=int)
    for p in parts:
        count[p["mortars"]] += 1
    assert np.all(count[~crossing] == 1) and np.all(count[crossing] == 2)
    assert sum(len(p["ghosts"]) for p in parts) == 2 * int(crossing.sum())
    for r, p in enumerate(parts):
        assert sorted(p["ghosts"]) == sorted(np.where(crossing & ((part[m[:, 0] - 1] == r) |
                                                                  (part[m[:, 1] - 1] == r)))[0].tolist())
        for nb, g0, n in p["plan"]:
            back = [x for x in parts[nb]["plan"] if x[0] == r]
            assert len(back) == 1 and back[0][2] == n
            assert p["ghosts"][g0:g0 + n] == parts[nb]["ghosts"][back[0][1]:back[0][1] + n]
