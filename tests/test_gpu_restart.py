"""DSEM restart files from and into the device state (dsem_write_restart,
dsem_read_restart: write_restart / read_restart, restart.f90:19-312,
319-929), against files built from the documented record layout by
tests/golden/make_restart_fixture.py and against the CPU oracle.  Entropy
viscosity is on, so a continued run needs the Lobatto arrays the file carries."""
import importlib.util
import os

import numpy as np
import pytest

from dsem_b200 import restart_file

pytestmark = pytest.mark.gpu

_spec = importlib.util.spec_from_file_location(
    "mkrst", os.path.join(os.path.dirname(__file__), "golden", "make_restart_fixture.py"))
mk = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(mk)


def _solver(box):
    from dsem_b200.solver import Solver
    return Solver(box.desc(), **mk.PHYS)


def test_read_file_written_after_steps_continues_like_the_oracle(oracle_mod, tmp_path):
    """A file written after 3 steps (state and Lobatto arrays): the GPU reads it and runs 3 more
    steps; the oracle simply continues.  Entropy viscosity and state to 1e-12."""
    p = tmp_path / "s3.rst"
    box, q0, dt, c = mk.make(p, 3)
    s = _solver(box)
    t = s.read_restart(p)
    assert t == 3 * dt
    assert np.array_equal(s.download(), c.get_q())
    s.step(dt, 3)
    c.step(0.0, dt, 3)
    mo = c.muhg()
    assert np.abs(mo).max() > 0
    assert np.abs(s.muhg() - mo).max() <= 1e-12 * np.abs(mo).max()
    qo = c.get_q()
    assert np.abs(s.download() - qo).max() <= 1e-12 * np.abs(qo).max()


def test_zero_step_file_is_a_fresh_start(tmp_path):
    """DSEM's zero-step file holds zeroed Lobatto arrays: no gradients, mu_EV = 0 on step 1, as
    for a context that uploads the same state."""
    p = tmp_path / "s0.rst"
    box, q0, dt, _ = mk.make(p, 0)
    a = _solver(box)
    a.read_restart(p)
    b = _solver(box)
    b.upload(q0)
    a.step(dt, 2)
    b.step(dt, 2)
    assert np.array_equal(a.download(), b.download())


def test_written_file_holds_the_state_and_restarts_bit_for_bit(oracle_mod, tmp_path):
    """The GPU writes a file after 3 steps (template: the zero-step file): its Q and Lobatto
    records are the oracle's after the same 3 steps; a second context reads it and its next 3
    steps equal the first context's."""
    tpl = tmp_path / "s0.rst"
    box, q0, dt, _ = mk.make(tpl, 0)
    a = _solver(box)
    a.keep_lobatto(True)
    a.upload(q0)
    a.step(dt, 3)
    out = tmp_path / "gpu3.rst"
    a.write_restart(tpl, out, time=3 * dt)
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(**mk.PHYS)
    c.set_q(q0)
    c.step(0.0, dt, 3)
    sz = restart_file.Sizes(nx=box.ldx)
    q, lob, t = restart_file.state(out, box, sz)
    ref_lob, ok = c.lobatto()
    assert ok and t == 3 * dt
    qo = c.get_q()
    assert np.abs(q - qo).max() <= 1e-12 * np.abs(qo).max()
    assert np.abs(lob - ref_lob).max() <= 1e-12 * np.abs(ref_lob).max()
    # every record outside the state passes through unchanged
    r_t, r_o = restart_file.records(tpl), restart_file.records(out)
    assert len(r_t) == len(r_o)
    changed = {13 + 24 * e + k for e in range(box.nel) for k in (6, 7, 8, 9, 13)} | {len(r_t) - 1}
    assert all(r_t[i] == r_o[i] for i in range(len(r_t)) if i not in changed)
    b = _solver(box)
    assert b.read_restart(out) == 3 * dt
    a.step(dt, 3)
    b.step(dt, 3)
    assert np.array_equal(a.download(), b.download())


def test_restart_rejects_a_mismatched_mesh(tmp_path):
    from dsem_b200 import mesh
    from dsem_b200.solver import DsemError, Solver
    p = tmp_path / "s0.rst"
    mk.make(p, 0)
    other = Solver(mesh.Box(2, 2, 2, 3).desc(), **mk.PHYS)
    with pytest.raises(DsemError):
        other.read_restart(p)
