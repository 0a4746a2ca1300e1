"""dsem_rhs_noalloc: the right-hand side for callers that cannot allocate device
memory (applications whose GPU memory belongs to their own pool allocator or
is fixed at start-up).  The caller owns every input and output buffer -- here
torch allocates them, standing in for such an application -- and the library
works in its static scratch array.  The result must equal dsem_rhs on the same
state, on two calls in a row (the second call reuses the scratch array the
first one left behind).

This file is collected last so that a failure here cannot hide the result of
any other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from dsem_b200 import mesh

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12


def internal_arrays(box, q):
    """Device-layout inputs: element-major, x fastest, no padding."""
    G, L, ldx, ne = int(box.G[0]), int(box.G[0]) + 1, box.ldx, box.nel
    jq = np.ascontiguousarray(q[:, :, :G, :G, :G])
    jac = np.ascontiguousarray(box.jacob.reshape(ne, ldx, ldx, ldx)[:, :G, :G, :G])
    gmg = box.gmetg.reshape(ne, ldx, ldx, ldx, 9)
    gg = np.ascontiguousarray(np.stack([gmg[:, :G, :G, :G, d + 3 * d] for d in range(3)], axis=1))
    gm5 = box.gmet.reshape(ne, ldx, ldx, ldx, 9)
    gm = np.stack([gm5[:, :G, :G, :L, 0].reshape(ne, -1), gm5[:, :G, :L, :G, 4].reshape(ne, -1),
                   gm5[:, :L, :G, :G, 8].reshape(ne, -1)], axis=1)
    nh = np.ascontiguousarray(box.n_hat[:, :G, :G, :])
    nrm = np.ascontiguousarray(box.norm[:, :G, :G])
    return dict(JQ=jq, jac=jac, gg=gg, gm=np.ascontiguousarray(gm), nh=nh, nrm=nrm,
                mortar=np.ascontiguousarray(box.mortar))


def call_noalloc(lib, box, arrs, torch, p, re=1600.0):
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in arrs.items()}
    G = p + 1
    qt = torch.zeros((box.nel, 5, G, G, G), dtype=torch.float64, device="cuda")
    dp = lambda t: C.c_void_p(t.data_ptr())
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.dsem_rhs_noalloc(box.nel, p, box.nmort, dp(dev["mortar"]), dp(dev["nh"]), dp(dev["nrm"]), dp(dev["JQ"]),
                              dp(dev["jac"]), dp(dev["gg"]), dp(dev["gm"]), C.c_double(1.4), C.c_double(re),
                              C.c_double(0.72), C.c_double(1.0), dp(qt), stream)
    return rc, qt.cpu().numpy()


@pytest.fixture(scope="module")
def lib():
    from dsem_b200 import solver
    L = solver.lib()
    L.dsem_rhs_noalloc.restype = C.c_int
    L.dsem_rhs_noalloc.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 7 + [C.c_double] * 4 + \
        [C.c_void_p, C.c_void_p]
    return L


@pytest.mark.parametrize("n,p", [(3, 4), (2, 8)])
def test_noalloc_matches_rhs_twice(lib, n, p):
    import torch
    from dsem_b200.solver import Solver
    box = mesh.Box(n, n, n, p)
    q = mesh.taylor_green(box)
    s = Solver(box.desc(), re=1600.0)
    s.upload(q)
    G = p + 1
    ref = s.rhs()[:, :, :G, :G, :G]
    arrs = internal_arrays(box, q)
    for call in range(2):
        rc, got = call_noalloc(lib, box, arrs, torch, p)
        assert rc == 0, lib.dsem_last_error(None)
        err = float(np.abs(got - ref).max() / np.abs(ref).max())
        assert err <= RHS_TOL, (call, err)


def test_noalloc_rejects_oversized_mesh(lib):
    """Sizes beyond the static scratch are refused with a clear message, before any device work.
    The buffers are real (one double each), so even a call that went past the size check could
    only fail, never touch an invalid address."""
    import torch
    p = 8
    nel = 96  # 96 * (90*81 + 5*729) + 1 > 2^20
    bufs = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in range(5)]
    dp = lambda t: C.c_void_p(t.data_ptr())
    rc = lib.dsem_rhs_noalloc(nel, p, 0, None, None, None, dp(bufs[0]), dp(bufs[1]), dp(bufs[2]), dp(bufs[3]),
                              C.c_double(1.4), C.c_double(1600.0), C.c_double(0.72), C.c_double(1.0), dp(bufs[4]),
                              None)
    assert rc == -1
    assert b"too large" in lib.dsem_last_error(None)


@pytest.mark.parametrize("field,value", [(0, 0), (1, 9), (2, 7), (10, 8)])
def test_noalloc_rejects_out_of_range_mortar_rows(lib, field, value):
    """A mortar row naming an element outside 1..nel, a face outside 1..6 or an
    orientation outside 0..7 is skipped by the face kernels and reported."""
    import torch
    box = mesh.Box(2, 2, 2, 3)
    arrs = internal_arrays(box, mesh.taylor_green(box))
    rows = arrs["mortar"].reshape(box.nmort, -1).copy()
    rows[1, field] = value
    arrs["mortar"] = rows
    rc, _ = call_noalloc(lib, box, arrs, torch, 3)
    assert rc == -1
    assert b"out of range" in lib.dsem_last_error(None)
    rc, _ = call_noalloc(lib, box, internal_arrays(box, mesh.taylor_green(box)), torch, 3)
    assert rc == 0


@pytest.mark.parametrize("field,value", [(13, 0), (16, 0), (4, 3), (8, 5)])
def test_noalloc_rejects_nonconforming_rows(lib, field, value):
    """A row that dsem_rhs would send through the p-nonconforming projections (a conforming
    flag of 0) or whose lengths do not match the order is refused, not evaluated as a
    conforming mortar; the next call with valid rows succeeds."""
    import torch
    box = mesh.Box(2, 2, 2, 3)
    arrs = internal_arrays(box, mesh.taylor_green(box))
    rows = arrs["mortar"].reshape(box.nmort, -1).copy()
    rows[2, field] = value
    arrs["mortar"] = rows
    rc, _ = call_noalloc(lib, box, arrs, torch, 3)
    assert rc == -5
    assert b"conforming" in lib.dsem_last_error(None)
    rc, _ = call_noalloc(lib, box, internal_arrays(box, mesh.taylor_green(box)), torch, 3)
    assert rc == 0
