"""dsem_create / dsem_create_batch reject malformed inputs with an error code
before touching a device (no GPU needed): the C-ABI never aborts."""
import ctypes

import numpy as np
import pytest

from dsem_b200 import mesh


def _md(desc):
    from dsem_b200.solver import _mesh_desc
    md, keep = _mesh_desc(desc)
    return md, keep


def _create(desc, **phys):
    from dsem_b200 import solver
    L = solver.lib()
    md, keep = _md(desc)
    ph = solver.Phys(phys.get("gamma", 1.4), phys.get("re", 1600.0), 0.72, 1.0, 0.0, 0.0, 0, 4)
    h = ctypes.c_void_p()
    rc = L.dsem_create(ctypes.byref(md), ctypes.byref(ph), ctypes.byref(h))
    return rc, L.dsem_last_error(None).decode()


def test_anisotropic_orders_rejected():
    box = mesh.Box(2, 2, 2, 3)
    d = box.desc()
    d["ncg"] = d["ncg"].copy()
    d["ncg"][1] = 5  # element 0: ncg = (4, 5, 4)
    rc, msg = _create(d)
    assert rc == -5 and "anisotropic" in msg


def test_order_out_of_range_rejected():
    box = mesh.Box(2, 2, 2, 3)
    d = box.desc()
    d["ncg"] = np.full_like(d["ncg"], 10)  # p = 9
    rc, msg = _create(d)
    assert rc == -5 and "order" in msg


def test_padding_too_small_rejected():
    box = mesh.Box(2, 2, 2, 3)
    d = box.desc()
    d["ldx"] = 4  # ncg + 1 = 5 needed
    rc, msg = _create(d)
    assert rc == -1 and "ldx" in msg


def test_empty_mesh_rejected():
    box = mesh.Box(2, 2, 2, 3)
    d = box.desc()
    d["ngrid"] = 0
    rc, msg = _create(d)
    assert rc == -1


def test_batch_physics_mismatch_rejected():
    from dsem_b200 import solver
    L = solver.lib()
    b1, b2 = mesh.Box(2, 2, 2, 3), mesh.Box(2, 2, 2, 4)
    m1, k1 = _md(b1.desc())
    m2, k2 = _md(b2.desc())
    mds = (solver.MeshDesc * 2)(m1, m2)
    phs = (solver.Phys * 2)(solver.Phys(1.4, 800.0, 0.72, 1.0, 0.0, 0.0, 0, 4),
                            solver.Phys(1.3, 800.0, 0.72, 1.0, 0.0, 0.0, 0, 4))
    h = ctypes.c_void_p()
    rc = L.dsem_create_batch(2, mds, phs, ctypes.byref(h))
    assert rc == -5 and b"share gamma" in L.dsem_last_error(None)
    phs[1] = solver.Phys(1.4, -1.0, 0.72, 1.0, 0.0, 0.0, 0, 4)
    rc = L.dsem_create_batch(2, mds, phs, ctypes.byref(h))
    assert rc == -1 and b"re must be positive" in L.dsem_last_error(None)
    rc = L.dsem_create_batch(0, mds, phs, ctypes.byref(h))
    assert rc == -1


def test_null_context_calls_return_errors():
    from dsem_b200 import solver
    L = solver.lib()
    assert L.dsem_step(None, 0.0, 1e-3, 1) == -1
    assert L.dsem_rhs(None, 0.0, None, 10) == -1
    assert L.dsem_step_batch(None, None, 1) == -1
    assert L.dsem_adjoint(None, 1e-3, 1, 1, 0, None, None, 10, None, None) == -1
    assert L.dsem_batch_size(None) == -1
