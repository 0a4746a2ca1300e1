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


def _c_kind(decl):
    decl = decl.strip()
    if "*" in decl:
        return "ptr"
    return "double" if re.match(r"(const\s+)?double\b", decl) else ("int" if re.match(r"(const\s+)?int\b", decl)
                                                                    else decl)


def _header_structs_and_functions():
    txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "dsem_gpu.h")).read(), flags=re.S)
    structs = {}
    for body, name in re.findall(r"typedef struct\s*\{(.*?)\}\s*(\w+)\s*;", txt, flags=re.S):
        fields = []
        for stmt in body.split(";"):
            stmt = stmt.strip()
            if not stmt:
                continue
            m = re.match(r"((?:const\s+)?\w+)\s*(.*)", stmt)
            base, names = m.group(1), m.group(2)
            for nm in names.split(","):
                nm = nm.strip()
                fields.append((nm.lstrip("*").strip(), "ptr" if nm.startswith("*") else _c_kind(base)))
        structs[name] = fields
    funcs = {}
    for ret, name, params in re.findall(r"([\w\s\*]+?)\b(dsem_\w+)\s*\(([^)]*)\)\s*;", txt):
        ps = [x for x in params.split(",") if x.strip() and x.strip() != "void"]
        funcs[name] = ("ptr" if "*" in ret else ret.strip().split()[-1], len(ps))
    return structs, funcs


def test_integration_fortran_binding_matches_header():
    """The iso_c_binding module a DSEM maintainer adds agrees with
    include/dsem_gpu.h: its BIND(C) derived types list the C structs' fields in the same order
    with matching kinds (c_int / c_double / c_ptr), and each interface binds a declared
    function with the same number of arguments and the same kind of result."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    block = re.search(r"```fortran\n(MODULE dsem_cuda.*?END MODULE dsem_cuda)\n```", text, flags=re.S).group(1)
    block = re.sub(r"!.*", "", block)
    structs, funcs = _header_structs_and_functions()
    kinds = {"INTEGER(c_int)": "int", "REAL(c_double)": "double", "TYPE(c_ptr)": "ptr"}
    types = re.findall(r"TYPE, BIND\(C\) :: (\w+)\n(.*?)END TYPE", block, flags=re.S)
    assert {t for t, _ in types} == {"dsem_mesh_desc", "dsem_phys"}
    for tname, body in types:
        fields = []
        for line in body.strip().splitlines():
            decl, names = line.split("::")
            fields += [(n.strip(), kinds[decl.strip()]) for n in names.split(",")]
        assert fields == structs[tname], (tname, fields, structs[tname])
    bound = re.findall(r"(INTEGER\(c_int\) FUNCTION|TYPE\(c_ptr\) FUNCTION|SUBROUTINE) (\w+)\(([^)]*)\) "
                       r"BIND\(C, name='(\w+)'\)", block)
    assert len(bound) >= 7
    for kind, fname, args, cname in bound:
        assert fname == cname and cname in funcs, cname
        ret, nparams = funcs[cname]
        assert nparams == len([a for a in args.split(",") if a.strip()]), cname
        assert ret == {"INTEGER(c_int) FUNCTION": "int", "TYPE(c_ptr) FUNCTION": "ptr", "SUBROUTINE": "void"}[kind], cname
