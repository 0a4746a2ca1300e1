"""DSEM restart file layout on the host (dsem_b200.restart_file): the records
write_restart produces (restart.f90:19-312) for a small box, framed as Fortran
unformatted sequential records, and the state read back from them."""
import numpy as np

from dsem_b200 import mesh, restart_file


def test_record_layout_round_trip(tmp_path):
    box = mesh.Box(2, 3, 2, 3)
    rng = np.random.default_rng(3)
    q = rng.standard_normal(box.qshape())
    lob = rng.standard_normal((box.nel, 3, 5, box.ldx, box.ldx, box.ldx))
    sz = restart_file.Sizes(nx=box.ldx)
    recs = restart_file.restart_records(box, q, sz, lob, time=1.25)
    # header 13 records, 24 per element, 13 per mortar, num_prop, max_materials, case time
    assert len(recs) == 13 + 24 * box.nel + 13 * box.nmort + 1 + sz.max_materials + 1
    n3 = box.ldx ** 3
    assert len(recs[13 + 6]) == 5 * n3 * 8  # Q(nx,ny,nz,neq)
    assert len(recs[13 + 5]) == 24  # nc, ncg
    assert len(recs[13 + 22]) == 54 and len(recs[13 + 23]) == 8  # bcond CHARACTER(9)*6, domain_type
    p = tmp_path / "a.rst"
    restart_file.write(p, recs)
    raw = p.read_bytes()
    # every record framed by its length before and after
    assert len(raw) == sum(len(r) + 8 for r in recs)
    assert restart_file.records(p) == recs
    q2, lob2, t = restart_file.state(p, box, sz)
    assert np.array_equal(q2, q) and np.array_equal(lob2, lob) and t == 1.25


def test_fixture_script_writes_the_oracle_state(oracle_mod, tmp_path):
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location(
        "mkrst", os.path.join(os.path.dirname(__file__), "golden", "make_restart_fixture.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    p = tmp_path / "f.rst"
    box, q0, dt, c = mk.make(p, 2)
    q, lob, t = restart_file.state(p, box, restart_file.Sizes(nx=box.ldx))
    assert np.array_equal(q, c.get_q())
    ref, ok = c.lobatto()
    assert ok and np.array_equal(lob, ref) and np.abs(lob).max() > 0
    assert t == 2 * dt
    # a zero-step file carries zeroed Lobatto arrays (DSEM's zero_domain)
    p0 = tmp_path / "z.rst"
    mk.make(p0, 0)
    _, lob0, _ = restart_file.state(p0, box, restart_file.Sizes(nx=box.ldx))
    assert not lob0.any()
