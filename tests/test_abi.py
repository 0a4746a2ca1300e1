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


def test_header_is_strict_c_and_links(tmp_path):
    """A C caller (what DSEM's iso_c_binding interface binds to): include/dsem_gpu.h compiles
    as strict C99 and as C++11 (-pedantic -Werror), every declared function links against the
    library, and the program runs a call that needs no device."""
    import shutil
    import subprocess
    if not shutil.which("gcc") or not shutil.which("g++"):
        pytest.skip("no host C compiler")
    from dsem_b200 import solver
    solver.lib()  # builds the library if it is missing
    libdir = os.path.dirname(solver.LIB)
    fns = header_functions()
    src = tmp_path / "caller.c"
    src.write_text('#include "dsem_gpu.h"\n#include <stdio.h>\nint main(void) {\n'
                   "  void (*fp[])(void) = {\n" + ",\n".join(f"    (void (*)(void))&{f}" for f in fns) +
                   "\n  };\n  const char *e = dsem_last_error(NULL);\n"
                   '  printf("%d %s\\n", (int)(sizeof fp / sizeof fp[0]), e ? "ok" : "null");\n  return 0;\n}\n')
    inc = os.path.join(ROOT, "include")
    for cc, std, lang in (("gcc", "-std=c99", []), ("g++", "-std=c++11", ["-x", "c++"])):
        exe = tmp_path / f"caller_{cc}"
        r = subprocess.run([cc, std, "-Wall", "-Wextra", "-pedantic", "-Werror", *lang, "-I", inc, str(src),
                            "-x", "none", "-L", libdir, "-ldsem_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
        assert out.returncode == 0 and out.stdout.split() == [str(len(fns)), "ok"], (out.stdout, out.stderr)
