"""Autotuning of the volume kernel's launch shape (dsem_autotune): every shape
gives the same results bit for bit, the tuner keeps one of the timed shapes
per order, and a tuned context (single case or ensemble) reproduces an untuned
one exactly."""
import numpy as np
import pytest

from dsem_b200 import mesh

pytestmark = pytest.mark.gpu


def _run(box, q, dt, variant=None, tune=False, steps=2):
    from dsem_b200.solver import Solver
    s = Solver(box.desc(), re=900.0)
    s.upload(q)
    p = int(box.orders[0])
    if variant is not None:
        s.set_vol_variant(p, variant)
    if tune:
        choice, ms = s.autotune(reps=2)
        assert set(choice) == {p}
        nv = 5 if p in (4, 6, 8) else 1
        assert 0 <= choice[p] < nv
        assert np.all(ms[p - 1, :nv] > 0) and np.all(ms[p - 1, nv:] == -1)
        assert np.all(np.delete(ms, p - 1, axis=0) == -1)
    rhs = s.rhs()
    s.step(dt, steps)
    out = s.download()
    s.close()
    return rhs, out


@pytest.mark.parametrize("p", [4, 6, 8])
def test_every_launch_shape_gives_identical_results(p):
    box = mesh.Box(3, 2, 2, p)
    q = mesh.random_isotropic(box, seed=p, k0=2.0, mach_t=0.3)
    dt = 0.3 * mesh.dtcalc(box, q)
    ref_rhs, ref = _run(box, q, dt, variant=0)
    for v in (1, 2, 3, 4):
        rhs, out = _run(box, q, dt, variant=v)
        assert np.array_equal(rhs, ref_rhs), v
        assert np.array_equal(out, ref), v
    rhs, out = _run(box, q, dt, tune=True)
    assert np.array_equal(rhs, ref_rhs) and np.array_equal(out, ref)


def test_order_with_one_shape():
    box = mesh.Box(2, 2, 2, 3)
    q = mesh.random_isotropic(box, seed=1, k0=1.0, mach_t=0.2)
    dt = 0.3 * mesh.dtcalc(box, q)
    _, ref = _run(box, q, dt)
    _, out = _run(box, q, dt, tune=True)
    assert np.array_equal(out, ref)


def test_ensemble_tunes_each_order():
    from dsem_b200.solver import Ensemble
    boxes = [mesh.Box(2, 2, 2, 4), mesh.Box(2, 2, 3, 8), mesh.Box(3, 2, 2, 6)]
    qs = [mesh.random_isotropic(b, seed=i + 3, k0=2.0, mach_t=0.2) for i, b in enumerate(boxes)]
    dts = np.array([0.3 * mesh.dtcalc(b, q) for b, q in zip(boxes, qs)])

    def run(tune):
        e = Ensemble([b.desc() for b in boxes], res=[500.0, 900.0, 1500.0])
        for k, q in enumerate(qs):
            e.upload_case(k, q)
        if tune:
            choice, _ = e.autotune(reps=2)
            assert set(choice) == {4, 6, 8}
        e.step_batch(dts, 2)
        out = [e.download_case(k) for k in range(len(boxes))]
        e.close()
        return out

    for a, b in zip(run(False), run(True)):
        assert np.array_equal(a, b)


def test_shape_arguments_are_checked():
    from dsem_b200.solver import DsemError, Solver
    box = mesh.Box(2, 2, 2, 3)
    s = Solver(box.desc())
    with pytest.raises(DsemError):
        s.set_vol_variant(3, 1)  # p = 3 has one shape
    with pytest.raises(DsemError):
        s.set_vol_variant(9, 0)
    with pytest.raises(DsemError):
        s.set_vol_variant(4, 5)
    s.set_vol_variant(4, 4)  # an order the context does not use: accepted, unused
    s.close()
