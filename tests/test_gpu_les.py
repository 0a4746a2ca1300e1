"""Static Smagorinsky LES (dsem_set_les) against the oracle's restatement of
simpleSmag / nut_prolong (turbulence/staticSmago/staticSmag.f90) and the
viscosity amu = 1 + nu_t rho (+ mu_EV) of Vis_Fluxes_new.f90:123-125.
Bit for bit: the evaluation order follows the oracle."""
import numpy as np
import pytest

from dsem_b200 import mesh

pytestmark = pytest.mark.gpu


def _pair(oracle_mod, box, q, cs, numax, **phys):
    from dsem_b200.solver import Solver
    s = Solver(box.desc(), **phys)
    s.set_les(cs, numax)
    s.upload(q)
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(**phys)
    c.set_les(cs, numax)
    c.set_q(q)
    return s, c


@pytest.mark.parametrize("n,p,numax", [(2, 4, 1e3), (3, 3, 5.0), (2, 6, 1e3)])
def test_les_steps_match_oracle(oracle_mod, n, p, numax):
    box = mesh.Box(n, n, n, p)
    q = mesh.random_isotropic(box, seed=21, k0=2.0, mach_t=0.2)
    dt = 0.02 * mesh.dtcalc(box, q)
    s, c = _pair(oracle_mod, box, q, 0.1, numax, re=1600.0)
    for _ in range(3):  # the first step has no gradients yet (nu_t = 0), the next two do
        s.step(dt, 1)
        c.step(0.0, dt, 1)
        assert np.array_equal(s.download(), c.get_q())
    nu = s.nut()
    assert np.array_equal(nu, c.nut())
    assert nu.max() > 0.0
    if numax < 100:
        assert nu.max() <= numax
    # graph replays of several steps agree too
    s.step(dt, 2)
    c.step(0.0, dt, 2)
    assert np.array_equal(s.download(), c.get_q())


def test_les_with_entropy_viscosity(oracle_mod):
    box = mesh.Box(2, 2, 2, 4)
    q = mesh.random_isotropic(box, seed=5, k0=2.0, mach_t=0.3)
    dt = 0.02 * mesh.dtcalc(box, q)
    phys = dict(re=800.0, cmu=0.5, mumax=2.0, shock=1)
    s, c = _pair(oracle_mod, box, q, 0.12, 1e3, **phys)
    s.step(dt, 3)
    c.step(0.0, dt, 3)
    assert np.array_equal(s.download(), c.get_q())


def test_les_off_changes_nothing(oracle_mod):
    from dsem_b200.solver import DsemError, Solver
    box = mesh.Box(2, 2, 2, 3)
    q = mesh.random_isotropic(box, seed=2, k0=2.0, mach_t=0.2)
    dt = 0.1 * mesh.dtcalc(box, q)
    a = Solver(box.desc(), re=1600.0)
    b = Solver(box.desc(), re=1600.0)
    b.set_les(0.1, 1e3)
    b.set_les(0.0, 0.0)
    for s in (a, b):
        s.upload(q)
        s.step(dt, 2)
    assert np.array_equal(a.download(), b.download())
    with pytest.raises(DsemError):
        b.nut()
    rot = [0] * 27
    rot[13] = 7
    rbox = mesh.Box(3, 3, 3, 3, rot=rot)
    r = Solver(rbox.desc(), re=1600.0)
    with pytest.raises(DsemError) as e:
        r.set_les(0.1, 1e3)
    assert e.value.code == -5


@pytest.mark.parametrize("shock_sensor,rho_sensor,ev", [(True, False, True), (False, True, True), (True, True, True),
                                                         (True, True, False)])
def test_les_sensors_match_oracle(oracle_mod, shock_sensor, rho_sensor, ev):
    """DSEM's shockSensor / rhoSensor (staticSmag.f90:68-69): nu_t scaled by (1 - Ducros sensor) and by
    the density-based sensor that the step's entropy viscosity evaluates (RHS.f90:264-275).  Without
    entropy viscosity both stay zero, as DSEM's zeroed arrays (the density sensor then zeroes nu_t)."""
    box = mesh.Box(3, 3, 3, 4)
    q = mesh.random_isotropic(box, seed=33, k0=1.5, mach_t=0.3)
    phys = dict(re=1600.0, cmu=1.0, mumax=0.5, shock=1) if ev else dict(re=1600.0)
    dt = 0.05 * mesh.dtcalc(box, q)
    s, c = _pair(oracle_mod, box, q, 0.12, 1e3, **phys)
    s.set_les_sensors(shock_sensor, rho_sensor)
    c.set_les_sensors(shock_sensor, rho_sensor)
    plain = _pair(oracle_mod, box, q, 0.12, 1e3, **phys)[1]
    for _ in range(3):
        s.step(dt, 1)
        c.step(0.0, dt, 1)
        plain.step(0.0, dt, 1)
    qo = c.get_q()
    assert np.abs(s.download() - qo).max() <= 1e-12 * np.abs(qo).max()
    nu, nuo, nup = s.nut(), c.nut(), plain.nut()
    assert np.abs(nu - nuo).max() <= 1e-12 * max(np.abs(nuo).max(), 1e-300)
    if rho_sensor and not ev:
        assert not nuo.any()
    else:
        assert nuo.max() > 0.0
        assert not np.array_equal(nuo, nup)  # the sensors change the viscosity
