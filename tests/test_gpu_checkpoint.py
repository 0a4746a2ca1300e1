"""Checkpoint / resume of the device state (dsem_save_state / dsem_load_state):
a run resumed from a snapshot continues bit for bit, including the entropy
viscosity and the Smagorinsky model, which read the previous step's
gradients, and the diagnostics' previous kinetic energy."""
import numpy as np
import pytest

from dsem_b200 import mesh

pytestmark = pytest.mark.gpu


def test_resume_continues_bit_for_bit():
    from dsem_b200.solver import Solver
    box = mesh.Box(2, 2, 2, 4)
    q = mesh.random_isotropic(box, seed=8, k0=2.0, mach_t=0.3)
    dt = 0.02 * mesh.dtcalc(box, q)
    phys = dict(re=1000.0, cmu=0.5, mumax=2.0, shock=1)
    a = Solver(box.desc(), **phys)
    a.set_les(0.1, 1e3)
    a.upload(q)
    a.diag(dt, first=True)
    a.step(dt, 3)
    a.diag(dt)
    snap = a.save_state()
    a.step(dt, 4)
    da = a.diag(dt)
    ref = a.download()
    b = Solver(box.desc(), **phys)
    b.set_les(0.1, 1e3)
    b.load_state(snap)
    b.step(dt, 4)
    db = b.diag(dt)
    assert np.array_equal(b.download(), ref)
    assert da == db
    assert np.array_equal(b.muhg(), a.muhg())
    assert np.array_equal(b.nut(), a.nut())


def test_snapshot_rejects_another_mesh():
    from dsem_b200.solver import DsemError, Solver
    a = Solver(mesh.Box(2, 2, 2, 3).desc())
    a.upload(mesh.taylor_green(mesh.Box(2, 2, 2, 3)))
    snap = a.save_state()
    b = Solver(mesh.Box(2, 2, 2, 4).desc())
    with pytest.raises(DsemError) as e:
        b.load_state(snap)
    assert e.value.code == -1
    with pytest.raises(DsemError):
        a.load_state(snap[:40])
    bad = snap.copy()
    bad[0] = ord("X")
    with pytest.raises(DsemError):
        a.load_state(bad)
