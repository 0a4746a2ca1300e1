"""One case sharded over two processes (shard.run_rank), the multi-rank form of
DSEM's MPI decomposition (send_q_to_mortars_mpi / send_flux_to_mortars_mpi:
send_q.f90:771-895, send_flux.f90:464-692).  Every call here gets one GPU, so
both ranks run on cuda:0 and exchange their cut-mortar blocks over gloo (host
staged); no kernel waits on another rank's kernel, the exchange is the host's.
The gathered state is held against the CPU oracle's single-case run, bit for
bit, and the all-reduced diagnostic sums against the oracle's KE and
dissipation."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dsem_b200 import mesh

pytestmark = pytest.mark.gpu

RE = 1100.0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _case():
    box = mesh.Box(4, 3, 3, 4)
    q = mesh.random_isotropic(box, seed=21, k0=2.0, mach_t=0.25)
    dt = 0.4 * mesh.dtcalc(box, q)
    return box, q, dt


def _worker(rank, world, port, kind, nsteps, out):
    import datetime

    import torch
    import torch.distributed as dist

    from dsem_b200.shard import run_rank, slab_partition
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        box, q, dt = _case()
        part = slab_partition(box, world) if kind == "slab" else np.random.default_rng(5).integers(0, world, box.nel)
        qs, els, sums = run_rank(box.desc(), part, rank, q, dt, nsteps, diag=True, re=RE)
        out.put((rank, qs, els, sums))
    except Exception as e:  # reported to the parent, which fails the test
        out.put((rank, None, None, repr(e)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["slab", "random"])
def test_two_ranks_match_oracle(oracle_mod, kind):
    nsteps = 3
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, kind, nsteps, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        r, qs, els, sums = out.get(timeout=300)
        res[r] = (qs, els, sums)
    for p in procs:
        p.join(timeout=60)
    for r in (0, 1):
        assert res[r][0] is not None, res[r][2]
    box, q, dt = _case()
    full = np.zeros_like(q)
    for r in (0, 1):
        full[res[r][1]] = res[r][0]
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=RE)
    c.set_q(q)
    c.step(0.0, dt, nsteps)
    ref = c.get_q()
    assert np.array_equal(full, ref), float(np.abs(full - ref).max())
    # the all-reduced sums give the oracle's kinetic energy and dissipation
    sums = res[0][2]
    assert np.array_equal(sums, res[1][2])
    ke, _, eps = c.diag(dt, True)
    ke_s = 0.5 * (sums[0] + sums[1] + sums[2]) / sums[5] / (8.0 * np.pi ** 3)  # DSEM divides by 8 pi^3
    eps_s = 100.0 * (sums[3] / sums[4]) / RE
    assert abs(ke_s - ke) <= 1e-13 * abs(ke)
    assert abs(eps_s - eps) <= 1e-13 * abs(eps)
