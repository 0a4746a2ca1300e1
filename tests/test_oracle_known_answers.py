"""Known-answer tests that pin the CPU oracle.

DSEM ships no test suite, fixtures or golden vectors, and its Fortran cannot
be built here, so the restatement is pinned by properties of the mathematics
the reference implements: exactness of the spectral operators, the mortar L2
projections and the quadrature; Roe-flux consistency and symmetry; freestream
preservation and discrete conservation of the full right-hand side; invariance
under rotated element frames; analytic Taylor-Green invariants; spectral
convergence of the full right-hand side to the exact time derivatives of an
advected density wave (convection, heat conduction) and of a viscous shear
wave (viscous stress and its work); the temporal order of the stage loop.
"""
import math

import numpy as np
import pytest

from dsem_b200 import mesh


def cheb(G):
    return mesh.gauss_points(G), mesh.lobatto_points(G + 1)


@pytest.mark.parametrize("p", [1, 2, 4, 6, 8])
def test_derivative_matrix_exact(oracle_mod, p):
    """dmx differentiates polynomials of degree <= p+1 exactly (dermat, matrices.f90:144-178)."""
    dmx, bx = oracle_mod.operators(p)
    xg, xl = cheb(p + 1)
    for deg in range(p + 2):
        f = xl ** deg
        df = deg * xg ** (deg - 1) if deg else 0 * xg
        assert np.abs(dmx @ f - df).max() <= 1e-11 * max(1, deg * deg)
    assert np.abs(dmx.sum(axis=1)).max() <= 1e-12


@pytest.mark.parametrize("p", [1, 3, 5, 8])
def test_interpolation_matrix_exact(oracle_mod, p):
    """bx interpolates polynomials of degree <= p exactly (intrpmat, matrices.f90:185-207)."""
    dmx, bx = oracle_mod.operators(p)
    xg, xl = cheb(p + 1)
    for deg in range(p + 1):
        assert np.abs(bx @ xg ** deg - xl ** deg).max() <= 1e-13
    assert np.abs(bx.sum(axis=1) - 1).max() <= 1e-13


@pytest.mark.parametrize("nin,nout", [(5, 7), (7, 9), (4, 9)])
def test_mortar_projection(oracle_mod, nin, nout):
    """Prolongation is exact interpolation; restriction(prolongation) = identity;
    restriction is the L2 projection (compute_pmat, mortarLib.f90:242-420)."""
    P, R = oracle_mod.projection(nin, nout)
    xi = mesh.gauss_points(nin)
    xo = mesh.gauss_points(nout)
    for deg in range(nin):
        assert np.abs(P @ xi ** deg - xo ** deg).max() <= 1e-12
    assert np.abs(R @ P - np.eye(nin)).max() <= 1e-12
    # R keeps polynomials of degree < nin
    for deg in range(nin):
        assert np.abs(R @ xo ** deg - xi ** deg).max() <= 1e-12


@pytest.mark.parametrize("G", [3, 5, 9])
def test_ke_weights_integrate(oracle_mod, G):
    """bmatu1b integrates the Gauss-node interpolant over the unit cube exactly."""
    w = oracle_mod.ke_weights(G)
    assert abs(w.sum() - 1.0) <= 1e-14
    x = mesh.gauss_points(G)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f = X ** (G - 1) * Y * (1 - Z) ** 2
    exact = (1.0 / G) * 0.5 * (1.0 / 3.0)
    assert abs(np.sum(w * f) - exact) <= 1e-14


def _state(rng):
    rho = 0.5 + rng.random()
    u = rng.standard_normal(3) * 0.3
    p = 1.0 + rng.random()
    return np.array([rho, rho * u[0], rho * u[1], rho * u[2], p / 0.4 + 0.5 * rho * u @ u])


def test_roe_consistency_and_symmetry(oracle_mod):
    """riemann(n, ds, Q, Q) = ds n.F(Q); swapping sides and flipping n negates the flux."""
    rng = np.random.default_rng(3)
    for _ in range(20):
        n = rng.standard_normal(3)
        n /= np.linalg.norm(n)
        ds = 0.3 + rng.random()
        Q = _state(rng)
        f, g, h = oracle_mod.euler(Q)
        ref = ds * (n[0] * f + n[1] * g + n[2] * h)
        assert np.allclose(oracle_mod.riemann(n, ds, Q, Q), ref, rtol=1e-13, atol=1e-13)
        Q2 = _state(rng)
        a = oracle_mod.riemann(n, ds, Q, Q2)
        b = oracle_mod.riemann(-n, ds, Q2, Q)
        assert np.allclose(a, -b, rtol=1e-11, atol=1e-12)


def test_roe_upwinds_supersonic_states(oracle_mod):
    """When both states move through the face faster than sound (normal Mach 2-3, any
    tangential velocity), every Roe wave speed has one sign, so the Roe flux (riemann,
    PhysLib.f90:231-320; the entropy fix only touches near-zero speeds) is the physical flux
    of the upstream state: ds n.F(QL) for flow along n, ds n.F(QR) against it."""
    g = 1.4
    rng = np.random.default_rng(5)

    def cons(rho, u, p):
        return np.array([rho, rho * u[0], rho * u[1], rho * u[2], p / (g - 1.0) + 0.5 * rho * (u @ u)])

    def flux(n, ds, Q):
        f, gf, h = oracle_mod.euler(Q)
        return ds * (n[0] * f + n[1] * gf + n[2] * h)

    for _ in range(100):
        n = rng.standard_normal(3)
        n /= np.linalg.norm(n)
        ds = 0.5 + rng.random()
        (rl, rr), (pl, pr) = 0.5 + rng.random(2), 0.5 + rng.random(2)
        un = (2.0 + rng.random()) * max(math.sqrt(g * pl / rl), math.sqrt(g * pr / rr))
        tl, tr = rng.standard_normal(3), rng.standard_normal(3)
        tl -= (tl @ n) * n
        tr -= (tr @ n) * n
        ul, ur = un * n + 0.3 * tl, un * (1.0 + 0.1 * rng.random()) * n + 0.3 * tr
        QL, QR = cons(rl, ul, pl), cons(rr, ur, pr)
        ref = flux(n, ds, QL)
        assert np.abs(oracle_mod.riemann(n, ds, QL, QR) - ref).max() <= 1e-14 * np.abs(ref).max()
        QL, QR = cons(rl, -ul, pl), cons(rr, -ur, pr)
        ref = flux(n, ds, QR)
        assert np.abs(oracle_mod.riemann(n, ds, QL, QR) - ref).max() <= 1e-14 * np.abs(ref).max()


def _case(oracle_mod, box, re=400.0):
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=re)
    return c


@pytest.mark.parametrize("rot", [None, 13])
def test_freestream_preservation(oracle_mod, rot):
    n, p = 3, 4
    r = None
    if rot is not None:
        r = [0] * 27
        r[13] = rot
    box = mesh.Box(n, n, n, p, rot=r)
    c = _case(oracle_mod, box)
    q = np.zeros(box.qshape()).reshape(box.nel, 5, -1)
    st = np.array([1.1, 0.2, -0.3, 0.4, 0.0])
    st[4] = 2.0 / 0.4 + 0.5 * (st[1] ** 2 + st[2] ** 2 + st[3] ** 2) / st[0]
    m = box.jacob != 0
    for v in range(5):
        q[:, v][m] = st[v] / box.jacob[m]
    c.set_q(q.reshape(box.qshape()))
    qt = c.rhs()
    scale = np.abs(q).max()
    assert np.abs(qt).max() <= 1e-13 * scale


def test_conservation(oracle_mod):
    """Sum over elements of the quadrature-weighted Qt vanishes (periodic box)."""
    n, p = 3, 5
    box = mesh.Box(n, n, n, p)
    c = _case(oracle_mod, box)
    c.set_q(mesh.taylor_green(box))
    qt = c.rhs()
    G = p + 1
    w = oracle_mod.ke_weights(G)  # (i, j, l) = (x, y, z)
    q5 = qt[:, :, :G, :G, :G]  # [e][v][z][y][x]
    tot = np.einsum("evzyx,xyz->v", q5, w)
    mag = np.einsum("evzyx,xyz->v", np.abs(q5), w)
    assert np.all(np.abs(tot) <= 1e-12 * mag)


def test_rotated_frame_invariance(oracle_mod):
    """An interior element with a rotated local frame gives the same RHS at the same physical points."""
    n, p = 3, 4
    r = [0] * 27
    r[13] = 17
    b1, b0 = mesh.Box(n, n, n, p, rot=r), mesh.Box(n, n, n, p)
    c1, c0 = _case(oracle_mod, b1), _case(oracle_mod, b0)
    c1.set_q(mesh.taylor_green(b1))
    c0.set_q(mesh.taylor_green(b0))
    q1, q0 = c1.rhs(), c0.rhs()
    scale = np.abs(q0).max()
    x1, x0 = b1.xg[13], b0.xg[13]
    idx = {tuple(np.round(x, 11)): i for i, x in enumerate(x0) if b0.jacob[13, i] != 0}
    diff = 0.0
    for i in np.where(b1.jacob[13] != 0)[0]:
        j = idx[tuple(np.round(x1[i], 11))]
        diff = max(diff, np.abs(q1[13].reshape(5, -1)[:, i] - q0[13].reshape(5, -1)[:, j]).max())
    assert diff <= 1e-10 * scale
    assert np.abs(np.delete(q1, 13, 0) - np.delete(q0, 13, 0)).max() <= 1e-10 * scale


def test_taylor_green_invariants(oracle_mod):
    """KE0 = 1/8 and 100 <|w|^2>/Re = 75/Re at t = 0 (spectral accuracy)."""
    box = mesh.Box(4, 4, 4, 6)
    c = _case(oracle_mod, box, re=1600.0)
    c.set_q(mesh.taylor_green(box))
    c.rhs()
    ke, _, eps = c.diag(1.0, True)
    assert abs(ke - 0.125) <= 1e-10
    assert abs(eps - 75.0 / 1600.0) <= 1e-3 * 75.0 / 1600.0


def test_kinetic_energy_decays(oracle_mod):
    box = mesh.Box(3, 3, 3, 4)
    c = _case(oracle_mod, box, re=100.0)
    c.set_q(mesh.taylor_green(box))
    dt = 0.5 * c.dtcalc()
    kes = []
    for k in range(6):
        c.step(0.0, dt, 1)
        kes.append(c.diag(dt, k == 0)[0])
    assert all(b < a for a, b in zip(kes, kes[1:]))


def test_rk_coefficients(oracle_mod):
    """Carpenter-Kennedy 2N-storage (iord 4) integrates y' = y to fourth order per step."""
    box = mesh.Box(2, 2, 2, 2)
    c = _case(oracle_mod, box)
    a, b, cc = c.rk()
    assert c.kord() == 5
    for h in (0.1, 0.05):
        y, g = 1.0, 0.0
        for k in range(5):
            g = a[k] * g + y
            y = y + cc[k] * h * g
        err = abs(y - math.exp(h))
        assert err <= 2e-3 * h ** 5 * 10


def band_orders(n, p_out=6, p_in=8):
    """cfg 3 layout: the middle third in x at a higher order (p-nonconforming band)."""
    orders = np.full(n ** 3, p_out)
    for iz in range(n):
        for ix in range(n):
            for iy in range(n):
                if n // 3 <= ix < n - n // 3:
                    orders[iy + n * (ix + n * iz)] = p_in
    return orders


def test_nonconforming_band_freestream_and_conservation(oracle_mod):
    n = 3
    box = mesh.Box(n, n, n, band_orders(n, 4, 6))
    assert (~box.mortar[:, 13:17].all(axis=1)).any()
    c = _case(oracle_mod, box)
    # freestream
    q = np.zeros(box.qshape()).reshape(box.nel, 5, -1)
    st = np.array([1.0, 0.3, 0.1, -0.2, 0.0])
    st[4] = 2.0 / 0.4 + 0.5 * (st[1] ** 2 + st[2] ** 2 + st[3] ** 2) / st[0]
    m = box.jacob != 0
    for v in range(5):
        q[:, v][m] = st[v] / box.jacob[m]
    c.set_q(q.reshape(box.qshape()))
    assert np.abs(c.rhs()).max() <= 1e-12 * np.abs(q).max()
    # conservation across the nonconforming faces
    c.set_q(mesh.taylor_green(box))
    qt = c.rhs()
    tot = np.zeros(5)
    mag = np.zeros(5)
    for e in range(box.nel):
        G = int(box.G[e])
        w = oracle_mod.ke_weights(G)
        q5 = qt[e, :, :G, :G, :G]
        tot += np.einsum("vzyx,xyz->v", q5, w)
        mag += np.einsum("vzyx,xyz->v", np.abs(q5), w)
    assert np.all(np.abs(tot) <= 1e-12 * mag)


def test_entropy_viscosity_bounds(oracle_mod):
    box = mesh.Box(3, 3, 3, 4)
    c = _case(oracle_mod, box, re=400.0)
    c.set_phys(re=400.0, cmu=1.0, mumax=0.5, shock=1)
    c.set_q(mesh.random_isotropic(box, seed=7))
    dt = 0.3 * c.dtcalc()
    c.step(0.0, dt, 1)
    assert np.all(c.muhg() == 0.0)  # no Lobatto arrays before the first Fluxes call
    c.step(0.0, dt, 2)
    mu = c.muhg()[:, :5, :5, :5]
    assert mu.max() > 0.0 and mu.min() >= 0.0 and mu.max() <= 0.5


def _rhs_dqdt(oracle_mod, box, rho, u, p, re, gamma=1.4):
    """dQ/dt at the Gauss points from the oracle's right-hand side (Qt is d(Q/jacob)/dt)."""
    c = _case(oracle_mod, box, re=re)
    c.set_q(mesh._jq(box, rho, u, p, gamma))
    qt = c.rhs().reshape(box.nel, 5, -1)
    return qt * box.jacob[:, None, :], box.jacob != 0


def _density_wave_errors(oracle_mod, box, re=100.0, a=0.2, gamma=1.4, pr=0.72):
    """Max errors of the oracle's dQ/dt against the exact derivatives of the advected density
    wave (test_density_wave_spectral_convergence): (continuity and momentum, energy), each
    relative to the largest exact value."""
    p0 = 1.0 / gamma
    U = np.array([0.3, -0.2, 0.1])
    s = box.xg[..., 0] + box.xg[..., 1] + box.xg[..., 2]
    rho = 1.0 + a * np.sin(s)
    u = np.broadcast_to(U, rho.shape + (3,)).copy()
    dq, m = _rhs_dqdt(oracle_mod, box, rho, u, np.full_like(rho, p0), re)
    drho = -a * np.cos(s) * U.sum()
    lap = 3.0 * p0 * (a * np.sin(s) / rho ** 2 + 2.0 * a * a * np.cos(s) ** 2 / rho ** 3)
    de = -0.5 * (U @ U) * a * np.cos(s) * U.sum() + gamma / (pr * (gamma - 1.0)) * lap / re
    e_cm = max(np.abs(dq[:, v][m] - ex[m]).max() for v, ex in
               enumerate([drho, U[0] * drho, U[1] * drho, U[2] * drho])) / np.abs(drho[m]).max()
    return e_cm, np.abs(dq[:, 4][m] - de[m]).max() / np.abs(de[m]).max()


def test_density_wave_spectral_convergence(oracle_mod):
    """A density wave advected at uniform velocity and pressure, rho = 1 + a sin(x + y + z):
    the exact time derivatives are d rho/dt = -u.grad rho, d(rho u)/dt = u d rho/dt (the
    viscous stress of a uniform velocity vanishes, whatever Re is) and
    dE/dt = -|u|^2/2 u.grad rho + gamma/(Pr (gamma - 1)) lap(p/rho) / Re (heat conduction;
    the Mach number cancels between T = gamma M^2 p/rho and the conductivity).  On a periodic
    3^3 box the full right-hand side (Int_fluxes, Vis_Fluxes, the Roe and BR1 mortars,
    update_interior) converges to them spectrally as p grows."""
    e_cm, e_en = zip(*[_density_wave_errors(oracle_mod, mesh.Box(3, 3, 3, p)) for p in (2, 4, 6, 8)])
    for k in range(1, 4):
        assert e_cm[k] <= 0.1 * e_cm[k - 1], e_cm
        assert e_en[k] <= 0.2 * e_en[k - 1], e_en
    assert e_cm[-1] <= 1e-5 and e_en[-1] <= 1e-3, (e_cm, e_en)


def _shear_wave_errors(oracle_mod, box, re=50.0, A=0.1, gamma=1.4):
    """Errors of the oracle's dQ/dt against the shear wave's exact derivatives
    (test_shear_wave_viscous_stress): (density, x/y momentum, energy) relative to 2A/Re,
    2A/Re and 4A^2/Re, and the largest z-momentum rate relative to 2A/Re."""
    d = np.array([1.0, -1.0, 0.0])
    s = box.xg[..., 0] + box.xg[..., 1]
    u = A * np.sin(s)[..., None] * d
    dq, m = _rhs_dqdt(oracle_mod, box, np.ones_like(s), u, np.full_like(s, 1.0 / gamma), re)
    sm, se = 2.0 * A / re, 4.0 * A * A / re
    e = (np.abs(dq[:, 0][m]).max() / sm,
         max(np.abs(dq[:, 1 + i][m] + 2.0 / re * A * np.sin(s[m]) * d[i]).max() for i in (0, 1)) / sm,
         np.abs(dq[:, 4][m] - se * np.cos(2.0 * s[m])).max() / se)
    return np.array(e), np.abs(dq[:, 3][m]).max() / sm


def test_shear_wave_viscous_stress(oracle_mod):
    """A divergence-free shear wave at uniform density and pressure, u = A sin(x + y) (1, -1, 0):
    the convective terms and the heat flux vanish, so d rho/dt = 0, d(rho u)/dt = -(2/Re) u
    (mu lap u with |k|^2 = 2) and dE/dt = div(tau.u)/Re = 4 A^2 cos(2(x + y))/Re.  The viscous
    stress, its work and the BR1 viscous mortars of the full right-hand side converge to them
    spectrally; the z momentum, untouched by the wave, stays zero to rounding."""
    errs = []
    for p in (2, 4, 6, 8):
        e, ez = _shear_wave_errors(oracle_mod, mesh.Box(3, 3, 3, p))
        assert ez <= 1e-10
        errs.append(e)
    errs = np.array(errs)
    for k in range(1, 4):
        assert np.all(errs[k] <= 0.1 * errs[k - 1]), errs
    assert np.all(errs[-1] <= [1e-3, 1e-3, 1e-2]), errs


def test_density_wave_general_curved_and_nonconforming(oracle_mod):
    """The density wave's exact derivatives hold in physical coordinates, so the same
    convergence pins the general-metric path, curved elements and p-nonconforming mortars:
    a rotated middle element reproduces the axis-aligned box's errors (the scheme is
    invariant under the element's frame); curved elements (a smooth periodic warp of every
    element's map, as general_hex_map gives DSEM's curved meshes) converge spectrally; a
    middle-third band of order p_in inside order p_out (L2 mortar projections,
    mortar_operations.f90:249-758) stays within 2.5x of the uniform order p_out, for the
    density wave and for the viscous shear wave."""
    rot = [0] * 27
    rot[13] = 17
    e_warp = []
    for p in (2, 4, 6, 8):
        plain = _density_wave_errors(oracle_mod, mesh.Box(3, 3, 3, p))
        rotated = _density_wave_errors(oracle_mod, mesh.Box(3, 3, 3, p, rot=rot))
        assert np.allclose(rotated, plain, rtol=1e-6, atol=1e-12), (p, rotated, plain)
        e_warp.append(_density_wave_errors(oracle_mod, mesh.Box(3, 3, 3, p, warp=0.03)))
    e_warp = np.array(e_warp)
    for k in range(1, 4):
        assert np.all(e_warp[k] <= 0.3 * e_warp[k - 1]), e_warp
    assert np.all(e_warp[-1] <= [2e-3, 5e-3]), e_warp
    for p_out, p_in in ((4, 6), (6, 8)):
        orders = np.full(27, p_out)
        for iz in range(3):
            for iy in range(3):
                orders[iy + 3 * (1 + 3 * iz)] = p_in  # ix = 1, the middle third in x
        band = _density_wave_errors(oracle_mod, mesh.Box(3, 3, 3, orders))
        uniform = _density_wave_errors(oracle_mod, mesh.Box(3, 3, 3, p_out))
        assert np.all(np.array(band) <= 2.5 * np.array(uniform)), (p_out, p_in, band, uniform)
        # the viscous mortar projections (k_face_nc_vis's restatement): the shear wave too
        band, _ = _shear_wave_errors(oracle_mod, mesh.Box(3, 3, 3, orders))
        uniform, _ = _shear_wave_errors(oracle_mod, mesh.Box(3, 3, 3, p_out))
        assert np.all(band <= 2.5 * uniform), (p_out, p_in, band, uniform)


@pytest.mark.parametrize("iord,lo,hi", [(4, 12.0, 20.0), (3, 6.5, 10.0)])
def test_time_integration_order(oracle_mod, iord, lo, hi):
    """The stage loop itself (tstep.f90:66-114: g = a g + Qt, JQ += c dt g, tk = t + b dt) has
    the order of its coefficients: on an acoustic wave (p' / p = rho' / rho * gamma = 0.05,
    u' = rho'/rho c along (1,1,1)/sqrt 3) over a fixed time, halving dt divides the error
    against a 32x finer run by about 2^4 for Carpenter-Kennedy (iord 4) and 2^3 for
    Williamson (iord 3)."""
    gamma = 1.4
    box = mesh.Box(2, 2, 2, 4)
    s = box.xg[..., 0] + box.xg[..., 1] + box.xg[..., 2]
    w = 0.05 * np.sin(s)
    k = np.ones(3) / math.sqrt(3.0)
    jq = mesh._jq(box, 1.0 + w / gamma, (w / gamma)[..., None] * k, (1.0 + w) / gamma, gamma)

    def run(n, dt):
        c = oracle_mod.Case.from_desc(box.desc())
        c.set_phys(re=1e4, iord=iord)
        c.set_q(jq)
        c.step(0.0, dt, n)
        return c.get_q(), c

    _, c0 = run(0, 1.0)
    T = 20 * 0.5 * c0.dtcalc()
    ref, _ = run(640, T / 640)
    errs = [np.abs(run(n, T / n)[0] - ref).max() / np.abs(ref).max() for n in (20, 40, 80)]
    for a, b in zip(errs, errs[1:]):
        assert lo <= a / b <= hi, errs


def test_kinetic_energy_budget(oracle_mod):
    """Taylor-Green at Mach 0.1, Re = 100, resolved (3^3 elements, p = 6): the kinetic energy's
    decay rate -dKE/dt, taken from the KE history (do_user_stuff,
    BackstepProblem-stoch.f90:463-709), equals the enstrophy dissipation <|w|^2>/Re
    (energydissipation.f90:2-89, reported x100) to 1e-4 over the first steps: the viscous
    terms of the right-hand side dissipate exactly what the diagnostic measures (pressure
    work and numerical dissipation are O(1e-5) here)."""
    box = mesh.Box(3, 3, 3, 6)
    c = _case(oracle_mod, box, re=100.0)
    c.set_q(mesh.taylor_green(box))
    dt = 0.5 * c.dtcalc()
    h = []
    for k in range(12):
        c.step(0.0, dt, 1)
        h.append(c.diag(dt, k == 0))
    h = np.array(h)[1:]  # the first call has no previous KE
    assert np.all(h[:, 1] > 0)
    assert np.abs(100.0 * h[:, 1] / h[:, 2] - 1.0).max() <= 1e-4


def test_smagorinsky_viscosity_of_a_shear_wave(oracle_mod):
    """Static Smagorinsky (simpleSmag, staticSmag.f90:32-118) on the shear wave
    u = A sin(x + y) (1, -1, 0) at uniform density: |S| = sqrt(2 S_ij S_ij) = 2 A |cos(x + y)|
    exactly, so the subgrid viscosity (in units of 1/Re) is Re (Cs Delta)^2 2 A |cos(x + y)|
    with Delta = J^(1/3) / G (delta_g, :191-201).  It is formed at a step's start from the
    previous right-hand side's Lobatto arrays and converges to that spectrally; values above
    numax are capped at numax."""
    gamma, re, A, cs = 1.4, 400.0, 0.1, 0.17
    d = np.array([1.0, -1.0, 0.0])

    def nut(p, numax):
        box = mesh.Box(3, 3, 3, p)
        s = box.xg[..., 0] + box.xg[..., 1]
        c = _case(oracle_mod, box, re=re)
        c.set_les(cs, numax)
        c.set_q(mesh._jq(box, np.ones_like(s), A * np.sin(s)[..., None] * d, np.full_like(s, 1.0 / gamma), gamma))
        c.rhs()
        c.step(0.0, 1e-6, 1)
        m = box.jacob != 0
        delta = np.abs(1.0 / box.jacob[m]) ** (1.0 / 3.0) / (p + 1)
        return c.nut().reshape(box.nel, -1)[m], re * (cs * delta) ** 2 * 2.0 * A * np.abs(np.cos(s[m]))

    errs = []
    for p in (2, 4, 6, 8):
        got, ex = nut(p, 1e6)
        errs.append(np.abs(got - ex).max() / ex.max())
    for k in range(1, 4):
        assert errs[k] <= 0.05 * errs[k - 1], errs
    assert errs[-1] <= 1e-5, errs
    got, ex = nut(8, 0.06)
    assert got.max() == 0.06 and np.all(got >= 0.0)
    low = ex < 0.05
    assert np.abs(got[low] - ex[low]).max() <= 1e-5 * ex.max()
