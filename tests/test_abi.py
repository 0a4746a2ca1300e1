"""The C-ABI library loads and exports every function include/dsem_gpu.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "dsem_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dsem_[a-z_]+)\s*\(", txt)))


def test_header_parses():
    fns = header_functions()
    assert "dsem_create" in fns and "dsem_step" in fns and len(fns) >= 10


def test_library_exports_all_symbols():
    from dsem_b200 import solver
    L = solver.lib()
    for fn in header_functions():
        assert hasattr(L, fn), fn
    assert set(solver.EXPORTS) <= set(header_functions())


def test_create_without_device_fails_cleanly():
    """On a machine without a usable CUDA device dsem_create returns an error code, never aborts."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from dsem_b200 import mesh
    from dsem_b200.solver import DsemError, Solver
    box = mesh.Box(2, 2, 2, 2)
    with pytest.raises(DsemError) as ei:
        Solver(box.desc())
    assert ei.value.code in (-2,)


def test_invalid_descriptor_rejected():
    from dsem_b200 import solver
    L = solver.lib()
    h = ctypes.c_void_p()
    rc = L.dsem_create(None, None, ctypes.byref(h))
    assert rc == -1
    assert b"null" in L.dsem_last_error(None)
