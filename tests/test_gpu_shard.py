"""One case sharded over several contexts (dsem_shard_stage): the sharded run
reproduces the single-context run bit for bit, and the CPU oracle's run.  All shards run in this
process on one GPU and exchange their cut-mortar blocks by device copies,
the same blocks NCCL moves between GPUs in a multi-GPU run."""
import numpy as np
import pytest

from dsem_b200 import mesh

pytestmark = pytest.mark.gpu


def _single(box, q, dt, nsteps, diag=False, **phys):
    from dsem_b200.solver import Solver
    s = Solver(box.desc(), **phys)
    s.upload(q)
    if diag:
        s.diag(dt, first=True)  # asks for the last stage's gradients
    s.step(dt, nsteps)
    return s


@pytest.mark.parametrize("parts,kind", [(2, "slab"), (3, "slab"), (3, "random"), (4, "random")])
def test_sharded_steps_match_single_context(oracle_mod, parts, kind):
    from dsem_b200.shard import ShardedRun, slab_partition
    box = mesh.Box(4, 4, 4, 3)
    q = mesh.random_isotropic(box, seed=11, k0=2.0, mach_t=0.2)
    dt = 0.5 * mesh.dtcalc(box, q)
    part = slab_partition(box, parts) if kind == "slab" else np.random.default_rng(parts).integers(0, parts, box.nel)
    run = ShardedRun(box.desc(), part, re=1200.0)
    run.upload(q)
    run.diag_sums()  # asks every shard for the last stage's gradients
    run.step(dt, 3)
    ref = _single(box, q, dt, 3, diag=True, re=1200.0)
    got = run.download()
    assert np.array_equal(got, ref.download())
    # and the CPU oracle's single-case run
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=1200.0)
    c.set_q(q)
    c.step(0.0, dt, 3)
    assert np.array_equal(got, c.get_q())
    # diagnostics: shard sums add up to the single context's
    sums = run.diag_sums()
    assert sums[6] == 1.0
    ke, _, eps = ref.diag(dt)
    us = (sums[0] + sums[1] + sums[2]) / sums[5]
    ke_s = 0.5 * us / (8.0 * np.pi ** 3)
    eps_s = 100.0 * (sums[3] / sums[4]) / 1200.0
    assert abs(ke_s - ke) <= 1e-14 * abs(ke)
    assert abs(eps_s - eps) <= 1e-13 * abs(eps)


def test_sharded_rotated_elements_and_ev(oracle_mod):
    """Cut mortars through rotated elements (all orientation codes) with entropy viscosity."""
    from dsem_b200.shard import ShardedRun
    rot = [0] * 27
    rot[13] = 7  # the interior element (the box builder rotates interior elements only)
    box = mesh.Box(3, 3, 3, 3, rot=rot)
    q = mesh.random_isotropic(box, seed=4, k0=1.0, mach_t=0.2)
    dt = 0.02 * mesh.dtcalc(box, q)
    part = np.arange(box.nel) % 2
    phys = dict(re=900.0, cmu=0.5, mumax=2.0, shock=1)
    run = ShardedRun(box.desc(), part, **phys)
    run.upload(q)
    run.step(dt, 2)
    ref = _single(box, q, dt, 2, **phys)
    got = run.download()
    assert np.array_equal(got, ref.download())
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(**phys)
    c.set_q(q)
    c.step(0.0, dt, 2)
    assert np.abs(got - c.get_q()).max() <= 1e-12 * np.abs(c.get_q()).max()


def test_sharded_les_matches_single_context():
    """Smagorinsky viscosity is element-local: a sharded LES run is the single run bit for bit."""
    from dsem_b200.shard import ShardedRun, slab_partition
    from dsem_b200.solver import Solver
    box = mesh.Box(4, 3, 3, 4)
    q = mesh.random_isotropic(box, seed=8, k0=2.0, mach_t=0.3)
    dt = 0.3 * mesh.dtcalc(box, q)
    run = ShardedRun(box.desc(), slab_partition(box, 2), re=3000.0)
    run.set_les(0.17, 0.05)
    run.upload(q)
    run.step(dt, 3)
    ref = Solver(box.desc(), re=3000.0)
    ref.set_les(0.17, 0.05)
    ref.upload(q)
    ref.step(dt, 3)
    assert np.array_equal(run.download(), ref.download())


def test_shard_rejects_plain_stepping():
    from dsem_b200.shard import partition, slab_partition
    from dsem_b200.solver import DsemError, Solver
    box = mesh.Box(4, 2, 2, 2)
    p = partition(box.desc(), slab_partition(box, 2))[0]
    s = Solver(p["desc"])
    s.upload(mesh.taylor_green(box)[p["elements"]])
    with pytest.raises(DsemError):
        s.step(1e-3, 1)
    with pytest.raises(DsemError):
        s.rhs()
    with pytest.raises(DsemError):
        s.adjoint(1e-3, 2, 1)
