"""Discrete adjoint (dsem_adjoint) against complex-step derivatives of the oracle.

J = sum over the last `window` of `nsteps` steps of dt * eps_n, eps_n being the
enstrophy dissipation of the diagnostics after step n.  The oracle evaluates
J in complex arithmetic from JQ0 + i h dq (h = 1e-30), which gives dJ/dJQ0 . dq
to rounding; the adjoint's gradient must agree along seeded directions.  The
derivative with respect to 1/Re is checked against central differences of
the oracle's J.  The bar is 1e-6 relative (the adjoint and complex step are
both exact up to rounding; they agree to ~1e-14 on these cases).
"""
import numpy as np
import pytest

from dsem_b200 import mesh

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _case(n, p, re, seed=3):
    box = mesh.Box(n, n, n, p)
    q = mesh.random_isotropic(box, seed=seed, k0=2.0, mach_t=0.2)
    dt = 0.5 * mesh.dtcalc(box, q)
    return box, q, dt


def _directions(q, G, k, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        d = rng.standard_normal(q.shape)
        d[:, :, G:] = 0.0
        d[:, :, :, G:] = 0.0
        d[:, :, :, :, G:] = 0.0
        out.append(d)
    return out


@pytest.mark.parametrize("n,p,nsteps,window", [(2, 3, 4, 2), (2, 6, 3, 3)])
def test_adjoint_matches_complex_step(oracle_mod, n, p, nsteps, window):
    from dsem_b200.solver import Solver
    re = 400.0
    box, q, dt = _case(n, p, re)
    s = Solver(box.desc(), re=re)
    s.upload(q)
    J, g, lr, _ = s.adjoint(dt, nsteps, window, snapshots=0)
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=re)
    c.set_q(q)
    for d in _directions(q, p + 1, 8, seed=p):  # eight seeded directions
        Jc, dJ = c.objective_cs(dt, nsteps, window, d, 1e-30)
        assert abs(J - Jc) <= 1e-12 * abs(Jc)
        ga = float(np.sum(g * d))
        assert abs(ga - dJ) <= TOL * abs(dJ), (ga, dJ)
    # d/d(1/Re): central differences of the oracle's J
    r = 1.0 / re
    h = 1e-5 * r
    vals = []
    for rr in (r + h, r - h):
        cc = oracle_mod.Case.from_desc(box.desc())
        cc.set_phys(re=1.0 / rr)
        cc.set_q(q)
        vals.append(cc.objective_cs(dt, nsteps, window, None, 0.0)[0])
    fd = (vals[0] - vals[1]) / (2 * h)
    assert abs(lr - fd) <= TOL * abs(fd), (lr, fd)
    s.close()


def test_adjoint_checkpointing_gives_the_same_gradient():
    """Binomial checkpointing recomputes the same steps: same gradient bit for bit."""
    from dsem_b200.solver import Solver
    box, q, dt = _case(2, 4, 800.0, seed=5)
    s = Solver(box.desc(), re=800.0)
    s.upload(q)
    J0, g0, lr0, _ = s.adjoint(dt, 7, 3, snapshots=0)
    for snaps in (1, 2, 3):
        J1, g1, lr1, _ = s.adjoint(dt, 7, 3, snapshots=snaps)
        assert J1 == J0 and lr1 == lr0
        assert np.array_equal(g1, g0)
    s.close()


@pytest.mark.parametrize("snaps", [1, 2, 3, 6, 7, 10])
def test_adjoint_segments_give_the_same_gradient(snaps):
    """Two-level checkpointing (DSEM_ADJ_SEGMENTS: snapshots at segment starts, one
    segment's stage states and traces kept while it is reversed): segments of 7, 4, 3, 2
    and 1 steps, the last one shorter, the window (3 steps) across a segment boundary.
    Same J, dJ/dJQ0 and dJ/d(1/Re) as store-all, bit for bit."""
    from dsem_b200.solver import Solver
    box, q, dt = _case(2, 4, 800.0, seed=5)
    s = Solver(box.desc(), re=800.0)
    s.upload(q)
    J0, g0, lr0, _ = s.adjoint(dt, 7, 3, snapshots=0)
    J1, g1, lr1, _ = s.adjoint(dt, 7, 3, snapshots=snaps, scheme="segments")
    assert J1 == J0 and lr1 == lr0
    assert np.array_equal(g1, g0)
    assert np.array_equal(s.download(), q)  # the state is restored
    s.close()


@pytest.mark.parametrize("snaps", [0, 2])
def test_adjoint_low_memory_paths_give_the_same_gradient(monkeypatch, snaps):
    """Without the optional trace and saved-gradient slots (DSEM_ADJOINT_LEAN=1,
    the paths taken when device memory is short) the reverse sweep recomputes
    the face traces and the window's saved gradients: same gradient bit for bit."""
    from dsem_b200.solver import Solver
    box, q, dt = _case(2, 4, 800.0, seed=7)
    s = Solver(box.desc(), re=800.0)
    s.upload(q)
    J0, g0, lr0, _ = s.adjoint(dt, 6, 3, snapshots=snaps)
    monkeypatch.setenv("DSEM_ADJOINT_LEAN", "1")
    J1, g1, lr1, _ = s.adjoint(dt, 6, 3, snapshots=snaps)
    monkeypatch.delenv("DSEM_ADJOINT_LEAN")
    assert J1 == J0 and lr1 == lr0
    assert np.array_equal(g1, g0)
    s.close()


def test_adjoint_objective_is_the_diagnostic_sum():
    """J equals the sum of dt * eps reported by dsem_diag over the window, and
    the context's state is restored afterwards."""
    from dsem_b200.solver import Solver
    box, q, dt = _case(2, 3, 600.0, seed=9)
    s = Solver(box.desc(), re=600.0)
    s.upload(q)
    before = s.download()
    J, _, _, _ = s.adjoint(dt, 5, 3, snapshots=0, want_grad=False)
    assert np.array_equal(s.download(), before)
    ref = 0.0
    s.diag(dt, first=True)
    for n in range(5):
        s.step(dt, 1)
        _, _, eps = s.diag(dt)
        if n >= 2:
            ref += dt * eps
    assert abs(J - ref) <= 1e-13 * abs(ref)
    s.close()


def test_adjoint_rejects_unsupported_cases():
    from dsem_b200.solver import DsemError, Ensemble, Solver
    boxes = [mesh.Box(2, 2, 2, 3), mesh.Box(2, 2, 2, 4)]
    ens = Ensemble([b.desc() for b in boxes], [400.0, 800.0])  # several cases
    for k, b in enumerate(boxes):
        ens.upload_case(k, mesh.taylor_green(b))
    with pytest.raises(DsemError) as e:
        ens.adjoint(1e-3, 2, 1)
    assert e.value.code == -5
    ens.close()
    rot = [0] * 27
    rot[13] = 7
    box = mesh.Box(3, 3, 3, 3, rot=rot)
    s = Solver(box.desc(), re=400.0)
    s.upload(mesh.taylor_green(box))
    with pytest.raises(DsemError) as e:
        s.adjoint(1e-3, 2, 1)
    assert e.value.code == -5
    s.close()


EV = dict(cmu=4.0, mumax=2.0, shock=1)


@pytest.mark.parametrize("n,p,nsteps,window,prestep", [(2, 3, 4, 2, 0), (2, 4, 3, 3, 2)])
def test_adjoint_with_entropy_viscosity(oracle_mod, n, p, nsteps, window, prestep):
    """Entropy viscosity (tstep.f90:36-38): each step's viscosity comes from its
    start state and the gradients saved by the previous step's last stage; the
    adjoint carries both dependencies.  With prestep > 0 the run starts after
    some steps, so the first step's viscosity uses gradients from before the
    run (held fixed, as the complex step holds them)."""
    from dsem_b200.solver import Solver
    re = 400.0
    box, q, dt = _case(n, p, re, seed=11)
    s = Solver(box.desc(), re=re, **EV)
    s.upload(q)
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=re, **EV)
    c.set_q(q)
    if prestep:
        s.step(dt, prestep)
        c.step(0.0, dt, prestep)
        assert np.array_equal(s.download(), c.get_q())
    q0 = s.download()
    J, g, lr, _ = s.adjoint(dt, nsteps, window, snapshots=0)
    for d in _directions(q, p + 1, 4, seed=p + 20):
        Jc, dJ = c.objective_cs(dt, nsteps, window, d, 1e-30)
        assert abs(J - Jc) <= 1e-12 * abs(Jc)
        ga = float(np.sum(g * d))
        assert abs(ga - dJ) <= TOL * abs(dJ), (ga, dJ)
    if not prestep:  # d/d(1/Re): central differences of the oracle's J
        r = 1.0 / re
        h = 1e-5 * r
        vals = []
        for rr in (r + h, r - h):
            cc = oracle_mod.Case.from_desc(box.desc())
            cc.set_phys(re=1.0 / rr, **EV)
            cc.set_q(q0)
            vals.append(cc.objective_cs(dt, nsteps, window, None, 0.0)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(lr - fd) <= TOL * abs(fd), (lr, fd)
    s.close()


@pytest.mark.parametrize("prestep", [0, 2])
def test_entropy_viscosity_adjoint_with_checkpoints(prestep):
    """Checkpointing with entropy viscosity, binomial and two-level: each checkpoint also keeps
    the gradients its step's viscosity reads, and the step (or segment) being reversed keeps its
    own copy before recomputation.  Every snapshot count gives the store-all gradient bit for bit."""
    from dsem_b200.solver import Solver
    box, q, dt = _case(2, 3, 400.0, seed=13)
    s = Solver(box.desc(), re=400.0, **EV)
    s.upload(q)
    if prestep:
        s.step(dt, prestep)
    q0 = s.download()
    J0, g0, lr0, _ = s.adjoint(dt, 7, 3, snapshots=0)
    assert np.abs(g0).max() > 0
    for snaps in (1, 2, 3, 6):
        for scheme in ("revolve", "segments"):
            s.upload(q0)
            if prestep:  # the same gradients behind the first step's viscosity
                s.upload(q)
                s.step(dt, prestep)
            J1, g1, lr1, _ = s.adjoint(dt, 7, 3, snapshots=snaps, scheme=scheme)
            assert J1 == J0, (snaps, scheme)
            assert lr1 == lr0, (snaps, scheme)
            assert np.array_equal(g1, g0), (snaps, scheme)
    s.close()


DUCROS = dict(cmu=40.0, mumax=2.0, shock=3)


@pytest.mark.parametrize("n,p,nsteps,window,prestep", [(2, 3, 4, 2, 2), (2, 4, 3, 3, 2), (2, 3, 3, 2, 0)])
def test_adjoint_with_ducros_sensor(oracle_mod, n, p, nsteps, window, prestep):
    """Entropy viscosity scaled by the Ducros sensor (shock = 3, RHS.f90:180-207):
    mu = min(max(cmu Re rho h^2 |D| duc, 0), mumax), duc = min(max(div^2 / (div^2 +
    |curl u|^2 + 1e-9), 0), 1), both from the gradients the previous step saved.  cmu = 40
    puts about a tenth of the points at the cap.  Against complex-step derivatives of the
    oracle, and bit for bit across the storage schemes."""
    from dsem_b200.solver import Solver
    re = 400.0
    box, q, dt = _case(n, p, re, seed=11)
    s = Solver(box.desc(), re=re, **DUCROS)
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=re, **DUCROS)
    c.set_q(q)

    def start():
        s.upload(q)
        if prestep:
            s.step(dt, prestep)

    start()
    if prestep:
        c.step(0.0, dt, prestep)
        assert np.array_equal(s.download(), c.get_q())
        G = p + 1
        mu = s.muhg()[:, :G, :G, :G]
        assert mu.max() == DUCROS["mumax"] and mu.min() < DUCROS["mumax"]
    J, g, lr, _ = s.adjoint(dt, nsteps, window, snapshots=0)
    assert np.abs(g).max() > 0
    for d in _directions(q, p + 1, 4, seed=p + 60):
        Jc, dJ = c.objective_cs(dt, nsteps, window, d, 1e-30)
        assert abs(J - Jc) <= 1e-12 * abs(Jc)
        ga = float(np.sum(g * d))
        assert abs(ga - dJ) <= TOL * abs(dJ), (ga, dJ)
    for snaps, scheme in ((2, "revolve"), (2, "segments")):
        start()
        J1, g1, lr1, _ = s.adjoint(dt, nsteps, window, snapshots=snaps, scheme=scheme)
        assert J1 == J and lr1 == lr and np.array_equal(g1, g), (snaps, scheme)
    s.close()


LES = dict(cs=0.15, numax=1e3)


@pytest.mark.parametrize("n,p,nsteps,window,prestep,numax", [(2, 3, 4, 2, 0, 1e3), (2, 4, 3, 3, 2, 1e3),
                                                              (2, 3, 3, 2, 2, 30.0)])
def test_adjoint_with_smagorinsky(oracle_mod, n, p, nsteps, window, prestep, numax):
    """Static Smagorinsky LES (simpleSmag, nut_prolong, amu = 1 + nu_t rho,
    staticSmag.f90:191-261, Vis_Fluxes_new.f90:123-125): each step's nu_t comes from
    its start state and the gradients saved by the previous step's last stage; the
    adjoint carries both dependencies, the density weight, the clip at 0 of the
    prolonged nu_t and, with numax = 0.5, the cap at numax.  nu_t = Re (Cs h)^2 |S|
    depends on Re itself, so dJ/d(1/Re) carries that term too."""
    from dsem_b200.solver import Solver
    re = 400.0
    box, q, dt = _case(n, p, re, seed=17)
    s = Solver(box.desc(), re=re)
    s.set_les(LES["cs"], numax)
    s.upload(q)
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=re)
    c.set_les(LES["cs"], numax)
    c.set_q(q)
    if prestep:
        s.step(dt, prestep)
        c.step(0.0, dt, prestep)
        assert np.array_equal(s.download(), c.get_q())
        G = p + 1
        nu = s.nut()[:, :G, :G, :G]
        assert nu.max() > 0.0
        if numax < 100.0:  # the cap is active at some points, not all
            assert nu.max() == numax and nu.min() < numax
    q0 = s.download()
    J, g, lr, _ = s.adjoint(dt, nsteps, window, snapshots=0)
    assert np.abs(g).max() > 0
    for d in _directions(q, p + 1, 4, seed=p + 40):
        Jc, dJ = c.objective_cs(dt, nsteps, window, d, 1e-30)
        assert abs(J - Jc) <= 1e-12 * abs(Jc)
        ga = float(np.sum(g * d))
        assert abs(ga - dJ) <= TOL * abs(dJ), (ga, dJ)
    if not prestep:  # d/d(1/Re): central differences of the oracle's J
        r = 1.0 / re
        h = 1e-5 * r
        vals = []
        for rr in (r + h, r - h):
            cc = oracle_mod.Case.from_desc(box.desc())
            cc.set_phys(re=1.0 / rr)
            cc.set_les(LES["cs"], numax)
            cc.set_q(q0)
            vals.append(cc.objective_cs(dt, nsteps, window, None, 0.0)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(lr - fd) <= TOL * abs(fd), (lr, fd)
    s.close()


@pytest.mark.parametrize("prestep", [0, 2])
def test_smagorinsky_adjoint_with_checkpoints(prestep):
    """Binomial and two-level checkpointing with LES: the same gradient as store-all, bit
    for bit (each checkpoint keeps the gradients its step's nu_t reads)."""
    from dsem_b200.solver import Solver
    box, q, dt = _case(2, 3, 400.0, seed=19)
    s = Solver(box.desc(), re=400.0)
    s.set_les(LES["cs"], LES["numax"])

    def start():
        s.upload(q)
        if prestep:
            s.step(dt, prestep)

    start()
    J0, g0, lr0, _ = s.adjoint(dt, 7, 3, snapshots=0)
    assert np.abs(g0).max() > 0
    for snaps in (1, 2, 3, 6):
        for scheme in ("revolve", "segments"):
            start()
            J1, g1, lr1, _ = s.adjoint(dt, 7, 3, snapshots=snaps, scheme=scheme)
            assert J1 == J0, (snaps, scheme)
            assert lr1 == lr0, (snaps, scheme)
            assert np.array_equal(g1, g0), (snaps, scheme)
    s.close()


def test_smagorinsky_adjoint_limits():
    """LES together with entropy viscosity, or with the shock / density sensors, is refused."""
    from dsem_b200.solver import DsemError, Solver
    box, q, dt = _case(2, 3, 400.0)
    s = Solver(box.desc(), re=400.0, **EV)
    s.set_les(LES["cs"], LES["numax"])
    s.upload(q)
    with pytest.raises(DsemError) as e:
        s.adjoint(dt, 2, 1)
    assert e.value.code == -5
    s.close()
    s = Solver(box.desc(), re=400.0)
    s.set_les(LES["cs"], LES["numax"])
    s.set_les_sensors(shock_sensor=True)
    s.upload(q)
    with pytest.raises(DsemError) as e:
        s.adjoint(dt, 2, 1)
    assert e.value.code == -5
    s.close()


BND_CASES = [
    {"y": ("walladiab", "walladiab")},
    {"y": ("wallisoth", "walladiab")},
    {"x": ("inflow", "outflow")},
    {"z": ("outflow", "wallisoth"), "x": ("inflow", "walladiab")},
]


def _bnd_pair(oracle_mod, bc, p, re, **phys):
    from dsem_b200.solver import Solver
    box = mesh.Box(2, 3, 2, p, bc=bc)
    q = mesh.random_isotropic(box, seed=5, k0=2.0, mach_t=0.3)
    dt = 0.3 * mesh.dtcalc(box, q)
    qx = mesh.boundary_state(box, 1.0, (0.3, 0.1, -0.2), 100.0 / 1.4, seed=3, amp=0.05)
    fx = 0.01 * np.random.default_rng(4).standard_normal(qx.shape)
    s = Solver(box.desc(), re=re, **phys)
    s.upload(q)
    s.set_boundary(100.0, qx, fx)
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=re, **phys)
    c.set_q(q)
    c.set_boundary(100.0, qx, fx)
    return box, q, dt, s, c


@pytest.mark.parametrize("bc", BND_CASES)
def test_adjoint_with_boundary_faces(oracle_mod, bc):
    """Walls (adiabatic: Roe against the mirror state; isothermal: osher), inflow and outflow
    (Roe against the external state, riemann_solution's Dirichlet state) and their viscous
    conditions (boundary_flux, DirichletBC, Vis_Neumann; ViscousBC_slide.f90:9-420), reversed
    by forward-mode passes through each boundary point's flux and state.  Against
    complex-step derivatives of the oracle, d/d(1/Re) against its central differences (the
    external viscous flux of inflow and outflow faces carries its own 1/Re term), and bit for
    bit across the storage schemes."""
    re = 500.0
    box, q, dt, s, c = _bnd_pair(oracle_mod, bc, 3, re)
    nsteps, window = 3, 2
    J, g, lr, _ = s.adjoint(dt, nsteps, window, snapshots=0)
    assert np.abs(g).max() > 0
    for d in _directions(q, 4, 3, seed=70):
        Jc, dJ = c.objective_cs(dt, nsteps, window, d, 1e-30)
        assert abs(J - Jc) <= 1e-10 * abs(Jc)
        ga = float(np.sum(g * d))
        assert abs(ga - dJ) <= TOL * abs(dJ), (ga, dJ)
    r = 1.0 / re
    h = 1e-5 * r
    vals = []
    for rr in (r + h, r - h):
        _, _, _, _, cc = _bnd_pair(oracle_mod, bc, 3, 1.0 / rr)
        vals.append(cc.objective_cs(dt, nsteps, window, None, 0.0)[0])
    fd = (vals[0] - vals[1]) / (2 * h)
    assert abs(lr - fd) <= TOL * abs(fd), (lr, fd)
    for snaps, scheme in ((1, "revolve"), (2, "revolve"), (2, "segments")):
        s.upload(q)
        J1, g1, lr1, _ = s.adjoint(dt, nsteps, window, snapshots=snaps, scheme=scheme)
        assert J1 == J and lr1 == lr and np.array_equal(g1, g), (snaps, scheme)
    s.close()


def test_adjoint_with_boundary_faces_and_entropy_viscosity(oracle_mod):
    """Walls with entropy viscosity: the saved gradients the viscosity reads are recomputed
    with the boundary faces' Dirichlet states at the element ends."""
    re = 400.0
    box, q, dt, s, c = _bnd_pair(oracle_mod, {"y": ("walladiab", "walladiab")}, 3, re, **EV)
    s.step(dt, 2)
    c.step(0.0, dt, 2)
    assert np.array_equal(s.download(), c.get_q())
    J, g, lr, _ = s.adjoint(dt, 3, 2, snapshots=0)
    for d in _directions(q, 4, 3, seed=71):
        Jc, dJ = c.objective_cs(dt, 3, 2, d, 1e-30)
        assert abs(J - Jc) <= 1e-12 * abs(Jc)
        ga = float(np.sum(g * d))
        assert abs(ga - dJ) <= TOL * abs(dJ), (ga, dJ)
    s.close()


@pytest.mark.parametrize("p,ev", [(7, False), (8, False), (8, True)])
def test_adjoint_high_order(oracle_mod, p, ev):
    """p = 7 and 8: the volume adjoint keeps its element's Gauss gradients, their adjoints
    and the interpolated-gradient adjoints in a per-element device scratch (the working set
    is twice an SM's shared memory).  Against complex-step derivatives of the oracle, with
    and without entropy viscosity, and bit for bit under checkpointing."""
    from dsem_b200.solver import Solver
    re = 600.0
    phys = dict(EV) if ev else {}
    box, q, dt = _case(2, p, re, seed=23)
    s = Solver(box.desc(), re=re, **phys)
    s.upload(q)
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=re, **phys)
    c.set_q(q)
    if ev:
        s.step(dt, 1)
        c.step(0.0, dt, 1)
    q0 = s.download()
    J, g, lr, _ = s.adjoint(dt, 2, 2, snapshots=0)
    for d in _directions(q, p + 1, 3, seed=p + 80):
        Jc, dJ = c.objective_cs(dt, 2, 2, d, 1e-30)
        assert abs(J - Jc) <= 1e-12 * abs(Jc)
        ga = float(np.sum(g * d))
        assert abs(ga - dJ) <= TOL * abs(dJ), (ga, dJ)
    s.upload(q0 if not ev else q)
    if ev:
        s.step(dt, 1)
    J1, g1, lr1, _ = s.adjoint(dt, 2, 2, snapshots=1, scheme="segments")
    assert J1 == J and lr1 == lr and np.array_equal(g1, g)
    s.close()


def _band(n, p_out, p_in):
    """Orders of an n^3 box: p_out, with the middle third in x at p_in (p-nonconforming mortars
    between the two)."""
    orders = np.full(n ** 3, p_out)
    for iz in range(n):
        for ix in range(n):
            for iy in range(n):
                if n // 3 <= ix < n - n // 3:
                    orders[iy + n * (ix + n * iz)] = p_in
    return orders


@pytest.mark.parametrize("p_out,p_in,phys,bc", [(3, 4, {}, None), (4, 6, {}, None), (3, 4, EV, None),
                                                 (3, 4, {}, {"y": ("walladiab", "walladiab")})])
def test_adjoint_nonconforming_band(oracle_mod, p_out, p_in, phys, bc):
    """Two element orders joined by p-nonconforming mortars (mortar_operations.f90:151-758:
    prolongation to the mortar, Roe flux and average there, restriction back): the stage
    adjoint runs per order group and per face list, and k_face_nc_inv_adj / k_face_nc_vis_adj
    transpose the projections.  Against complex-step derivatives of the oracle, and bit for
    bit under checkpointing."""
    from dsem_b200.solver import Solver
    re = 500.0
    box = mesh.Box(3, 3, 3, _band(3, p_out, p_in), bc=bc)
    assert (~box.mortar[:, 13:17].all(axis=1)).sum() > 0  # nonconforming mortars present
    q = mesh.random_isotropic(box, seed=29, k0=2.0, mach_t=0.2)
    dt = 0.4 * mesh.dtcalc(box, q)
    s = Solver(box.desc(), re=re, **phys)
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=re, **phys)
    c.set_q(q)
    s.upload(q)
    if phys:
        s.step(dt, 1)
        c.step(0.0, dt, 1)
    q0 = s.download()
    J, g, lr, _ = s.adjoint(dt, 3, 2, snapshots=0)
    assert np.abs(g).max() > 0
    for d in _directions(q, p_in + 1, 3, seed=p_out + 90):
        Jc, dJ = c.objective_cs(dt, 3, 2, d, 1e-30)
        assert abs(J - Jc) <= 1e-12 * abs(Jc)
        ga = float(np.sum(g * d))
        assert abs(ga - dJ) <= TOL * abs(dJ), (ga, dJ)
    if not phys:  # d/d(1/Re): central differences of the oracle's J
        r = 1.0 / re
        h = 1e-5 * r
        vals = []
        for rr in (r + h, r - h):
            cc = oracle_mod.Case.from_desc(box.desc())
            cc.set_phys(re=1.0 / rr)
            cc.set_q(q0)
            vals.append(cc.objective_cs(dt, 3, 2, None, 0.0)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(lr - fd) <= TOL * abs(fd), (lr, fd)
    for snaps in (1, 2):
        s.upload(q)
        if phys:
            s.step(dt, 1)
        J1, g1, lr1, _ = s.adjoint(dt, 3, 2, snapshots=snaps)
        assert J1 == J and lr1 == lr and np.array_equal(g1, g), snaps
    s.close()
