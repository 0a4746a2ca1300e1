"""One case sharded over several GPUs: partitioning, exchange plan, drivers.

The replacement for DSEM's MPI decomposition (grid_partition.f90:46-79, the
METIS path of metis_file.f90) and its face exchange (send_q_to_mortars_mpi,
send_flux_to_mortars_mpi: send_q.f90:771-895, send_flux.f90:464-692).  Each
shard gets a descriptor of its own elements in the C-ABI layout; a mortar
whose two elements sit on different shards appears on both, with the remote
side's element id replaced by -(g+1), g numbering the shard's ghost faces.
Ghost faces are grouped by neighbouring shard and ordered by global mortar
number, so the two shards of every pair list their common mortars in the
same order: one contiguous block per neighbour in `send` on one side is the
block in `ghost` on the other.

Drivers
  ShardedRun   all shards in one process on one GPU, the exchange a device
               copy (used by the tests: the sharded run must reproduce the
               single-context run bit for bit);
  run_rank     one shard per process under torch.distributed: with NCCL
               (one GPU per rank) the blocks move by send/recv ordered on the
               library's stream, with gloo they are staged through host
               memory (the form the tests run, two ranks on one GPU).
"""
import numpy as np

from .solver import Solver, lib

MORTAR_INTS = 17


def slab_partition(box, nparts, axis=0):
    """Part of each element of a mesh.Box: contiguous slabs along axis (0: x)."""
    n = (box.nex, box.ney, box.nez)[axis]
    if nparts > n:
        raise ValueError("more parts than element layers")
    idx = np.arange(box.nel)
    # Box numbering: e = iy + ney * (ix + nex * iz)
    iy = idx % box.ney
    ix = (idx // box.ney) % box.nex
    iz = idx // (box.ney * box.nex)
    c = (ix, iy, iz)[axis]
    return np.minimum(c * nparts // n, nparts - 1).astype(np.int64)


def partition(desc, part):
    """Per-part descriptors and exchange plans.

    Returns a list over parts of dicts {desc, elements (global ids), mortars
    (global ids of the part's mortar rows), plan: [(neighbour, ghost_start,
    count)], ghosts: [global mortar ids]}.  Boundary mortars (id(2) = 0) go
    with their element."""
    part = np.asarray(part, dtype=np.int64)
    ne, nm, ldx = int(desc["ngrid"]), int(desc["nmort"]), int(desc["ldx"])
    nparts = int(part.max()) + 1
    L3 = ldx ** 3
    mort = np.asarray(desc["mortar"]).reshape(nm, MORTAR_INTS)
    nh = np.asarray(desc["n_hat"]).reshape(nm, ldx * ldx * 3)
    nr = np.asarray(desc["norm"]).reshape(nm, ldx * ldx)
    jac = np.asarray(desc["jacob"]).reshape(ne, L3)
    gg = np.asarray(desc["gmetg"]).reshape(ne, L3 * 9)
    gm = np.asarray(desc["gmet"]).reshape(ne, L3 * 9)
    ncg = np.asarray(desc["ncg"]).reshape(ne, 3)
    bcond = None if desc.get("bcond") is None else np.asarray(desc["bcond"], dtype=np.int32).reshape(ne, 6)
    out = []
    for r in range(nparts):
        els = np.where(part == r)[0]
        local = -np.ones(ne, dtype=np.int64)
        local[els] = np.arange(len(els))
        rows, geo_h, geo_n, ghosts_of = [], [], [], {}
        cut = []
        for j in range(nm):
            e1, e2 = int(mort[j, 0]) - 1, int(mort[j, 1]) - 1
            if e2 < 0:  # boundary face: stays with its element
                if part[e1] == r:
                    t = mort[j].copy()
                    t[0] = local[e1] + 1
                    rows.append((j, t))
                continue
            p1, p2 = part[e1], part[e2]
            if p1 != r and p2 != r:
                continue
            t = mort[j].copy()
            if p1 == r and p2 == r:
                t[0], t[1] = local[e1] + 1, local[e2] + 1
                rows.append((j, t))
            else:
                nb = p2 if p1 == r else p1
                cut.append((int(nb), j, t, p1 == r))
        # ghost numbering: by neighbour, then global mortar number
        cut.sort(key=lambda x: (x[0], x[1]))
        plan, ghosts = [], []
        for g, (nb, j, t, lm) in enumerate(cut):
            e1, e2 = int(mort[j, 0]) - 1, int(mort[j, 1]) - 1
            if lm:
                t[0], t[1] = local[e1] + 1, -(g + 1)
            else:
                t[0], t[1] = -(g + 1), local[e2] + 1
            rows.append((j, t))
            ghosts.append(j)
            if plan and plan[-1][0] == nb:
                plan[-1][2] += 1
            else:
                plan.append([nb, g, 1])
        rows.sort(key=lambda x: x[0])
        js = [j for j, _ in rows]
        d = dict(ngrid=len(els), nmort=len(rows), ldx=ldx,
                 ncg=np.ascontiguousarray(ncg[els].ravel().astype(np.int32)),
                 jacob=np.ascontiguousarray(jac[els].ravel()),
                 gmetg=np.ascontiguousarray(gg[els].ravel()),
                 gmet=np.ascontiguousarray(gm[els].ravel()),
                 mortar=np.ascontiguousarray(np.array([t for _, t in rows], dtype=np.int32).ravel()),
                 n_hat=np.ascontiguousarray(nh[js].ravel()),
                 norm=np.ascontiguousarray(nr[js].ravel()),
                 bcond=None if bcond is None else np.ascontiguousarray(bcond[els].ravel()))
        out.append(dict(desc=d, elements=els, mortars=np.asarray(js, dtype=np.int64), plan=[tuple(p) for p in plan],
                        ghosts=ghosts))
    return out


class _DevArray:
    """__cuda_array_interface__ view of library device memory (torch.as_tensor)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None}


def _buffers(solver):
    import ctypes as C
    import torch
    ng, per = C.c_int(), C.c_int()
    sp, gp = C.POINTER(C.c_double)(), C.POINTER(C.c_double)()
    lib().dsem_shard_info(solver.h, C.byref(ng), C.byref(per), C.byref(sp), C.byref(gp))
    n = ng.value * per.value
    if n == 0:
        return None, None, per.value
    send = torch.as_tensor(_DevArray(C.cast(sp, C.c_void_p).value, n), device="cuda")
    ghost = torch.as_tensor(_DevArray(C.cast(gp, C.c_void_p).value, n), device="cuda")
    return send, ghost, per.value


def _check(solver, rc):
    solver._check(rc)


class ShardedRun:
    """All shards of one case in this process on the current GPU."""

    def __init__(self, desc, part, **phys):
        self.parts = partition(desc, part)
        self.shards = [Solver(p["desc"], **phys) for p in self.parts]
        self.kord = self.shards[0].kord
        self.bufs = [_buffers(s) for s in self.shards]

    def set_les(self, cs, numax):
        for s in self.shards:
            s.set_les(cs, numax)

    def set_boundary(self, twall, Qext=None, fvext=None):
        """As Solver.set_boundary, with the unsharded mesh's [nmort][5][ldx][ldx] arrays."""
        for p, s in zip(self.parts, self.shards):
            s.set_boundary(twall, None if Qext is None else Qext[p["mortars"]],
                           None if fvext is None else fvext[p["mortars"]])

    def upload(self, JQ):
        for p, s in zip(self.parts, self.shards):
            s.upload(JQ[p["elements"]])

    def download(self):
        out = None
        for p, s in zip(self.parts, self.shards):
            q = s.download()
            if out is None:
                out = np.zeros((sum(len(x["elements"]) for x in self.parts),) + q.shape[1:])
            out[p["elements"]] = q
        return out

    def _exchange(self):
        import torch
        for r, p in enumerate(self.parts):
            send_r, ghost_r, per = self.bufs[r]
            for nb, g0, n in p["plan"]:
                # the neighbour's block for this pair
                qn = [x for x in self.parts[nb]["plan"] if x[0] == r][0]
                assert qn[2] == n
                send_n = self.bufs[nb][0]
                ghost_r[g0 * per:(g0 + n) * per].copy_(send_n[qn[1] * per:(qn[1] + n) * per])
        torch.cuda.synchronize()

    def step(self, dt, nsteps=1):
        L = lib()
        for _ in range(nsteps):
            for kk in range(1, self.kord + 1):
                for phase in range(3):
                    for s in self.shards:
                        _check(s, L.dsem_shard_stage(s.h, float(dt), kk, phase))
                    if phase < 2:
                        self._exchange()

    def diag_sums(self):
        import ctypes as C
        tot = np.zeros(7)
        for i, s in enumerate(self.shards):
            v = (C.c_double * 7)()
            _check(s, lib().dsem_diag_sums(s.h, v))
            a = np.array(v[:])
            tot[:5] += a[:5]
            if i == 0:
                tot[5:] = a[5:]
        return tot


def _diag_sums(solver):
    import ctypes as C
    v = (C.c_double * 7)()
    _check(solver, lib().dsem_diag_sums(solver.h, v))
    return np.array(v[:])


def run_rank(desc, part, rank, JQ, dt, nsteps, diag=False, **phys):
    """This process's shard under torch.distributed (initialised by the caller):
    advances nsteps and returns (the shard's final state, its global element ids,
    the all-reduced diagnostic sums or None).

    The exchange after phases 0 and 1 of every stage (send_q_to_mortars_mpi,
    send_flux_to_mortars_mpi: send_q.f90:771-895, send_flux.f90:464-692):
      nccl  one send/recv per neighbour block, issued on the library's own CUDA
            stream (dsem_get_stream, a torch external stream) between the
            enqueued phases (dsem_shard_enqueue): no host wait inside a step; the
            step ends with one dsem_shard_finish (its non-finite check);
      gloo  (a CPU transport, e.g. ranks that share one GPU) the blocks are
            staged through host memory; copies run on the library's stream.
    diag: the shard keeps the last stage's gradients; after the last step its
    seven diagnostic sums are added over the ranks (all-reduce), element-1
    jacobian and validity taken from rank 0, as dsem_diag_sums documents."""
    import ctypes as C

    import torch
    import torch.distributed as dist
    p = partition(desc, part)[rank]
    s = Solver(p["desc"], **phys)
    s.upload(JQ[p["elements"]])
    if diag:
        _diag_sums(s)  # asks the shard to keep the last stage's gradients
    send, ghost, per = _buffers(s)
    L = lib()
    nccl = dist.get_backend() == "nccl"
    sp = C.c_void_p()
    _check(s, L.dsem_get_stream(s.h, C.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value)

    def exchange():
        if not p["plan"]:
            return
        with torch.cuda.stream(stream):
            if nccl:
                ops = []
                for nb, g0, n in p["plan"]:
                    ops.append(dist.P2POp(dist.isend, send[g0 * per:(g0 + n) * per], nb))
                    ops.append(dist.P2POp(dist.irecv, ghost[g0 * per:(g0 + n) * per], nb))
                for w in dist.batch_isend_irecv(ops):
                    w.wait()  # orders the library stream after the transfer; no host wait
            else:
                hs = send.cpu()  # waits for the stream (the packed blocks)
                hg = torch.empty_like(hs)
                reqs = []
                for nb, g0, n in p["plan"]:
                    reqs.append(dist.isend(hs[g0 * per:(g0 + n) * per], nb))
                    reqs.append(dist.irecv(hg[g0 * per:(g0 + n) * per], nb))
                for w in reqs:
                    w.wait()
                ghost.copy_(hg)

    for _ in range(nsteps):
        for kk in range(1, s.kord + 1):
            for phase in range(3):
                _check(s, L.dsem_shard_enqueue(s.h, float(dt), kk, phase))
                if phase < 2:
                    exchange()
        _check(s, L.dsem_shard_finish(s.h))
    sums = None
    if diag:
        a = _diag_sums(s)
        t = torch.tensor(a[:5], dtype=torch.float64, device="cuda" if nccl else "cpu")
        dist.all_reduce(t)
        head = torch.tensor(a[5:], dtype=torch.float64, device=t.device)
        dist.broadcast(head, 0)
        sums = np.concatenate([t.cpu().numpy(), head.cpu().numpy()])
    return s.download(), p["elements"], sums
