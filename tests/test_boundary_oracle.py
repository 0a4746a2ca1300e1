"""Boundary faces (mortars with id(2) = 0) on the CPU: the mesh builder's
boundary mortars, and properties of the oracle's restatement of DSEM's wall,
inflow and outflow conditions (caseFiles/tgv/BackstepProblem-stoch.f90:1602-1729
with NS/BCs/stac3m) that hold for the reference algorithm itself:

* free-stream preservation: a uniform state at rest between walls (adiabatic,
  or isothermal at the state's own temperature), and a uniform stream through
  inflow/outflow faces whose external state is that stream, has a zero
  right-hand side up to rounding;
* a wall without normal velocity passes no mass: the Roe flux of two equal
  states has a zero mass component, so the domain's mass changes only by
  rounding;
* a parallel shear flow decaying between no-slip walls, and a density wave
  convected through inflow and outflow faces that carry the exact external
  state, have exact time derivatives, and the full right-hand side converges
  to them spectrally."""
import numpy as np
import pytest

from dsem_b200 import mesh

TWALL = 100.0
GAMMA = 1.4


def _weights(G):
    """Interpolatory quadrature weights on [0, 1] at the Gauss points (exact to degree G-1)."""
    x = mesh.gauss_points(G)
    V = np.array([np.polynomial.legendre.Legendre.basis(k)(2.0 * x - 1.0) for k in range(G)])
    rhs = np.zeros(G)
    rhs[0] = 1.0
    return np.linalg.solve(V, rhs)


def _uniform(box, rho, vel, p):
    q = np.zeros(box.qshape())
    u, v, w = vel
    cons = [rho, rho * u, rho * v, rho * w, p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v + w * w)]
    jac = box.jacob.reshape(box.nel, box.ldx, box.ldx, box.ldx)
    for e in range(box.nel):
        G = int(box.G[e])
        for k in range(5):
            q[e, k, :G, :G, :G] = cons[k] / jac[e, :G, :G, :G]
    return q


def test_box_boundary_mortars():
    box = mesh.Box(2, 3, 2, 3, bc={"y": ("walladiab", "wallisoth")})
    b = box.boundary_mortars()
    assert len(b) == 2 * 2 * 2  # nex * nez faces on each of the two y sides
    rows = box.mortar[b]
    assert np.all(rows[:, 1] == 0) and np.all(rows[:, 10] == 0) and np.all(rows[:, 12] == 1)
    bc = box.bcond
    for r in rows:
        e, f = r[0] - 1, r[2]
        assert f in (1, 2)  # y faces of unrotated elements
        assert bc[e, f - 1] == (1 if f == 1 else 2)
    assert int((bc > 0).sum()) == len(b)
    # x and z stay periodic (12 + 12 mortars), y has 8 interior and 8 boundary mortars
    assert box.nmort == 12 + 12 + 8 + 8
    with pytest.raises(ValueError):
        mesh.Box(2, 2, 2, 3, bc={"y": ("walladiab", "slip")})
    assert mesh.Box(2, 2, 2, 3).desc()["bcond"] is None


@pytest.mark.parametrize("bc", [{"y": ("walladiab", "walladiab")}, {"y": ("wallisoth", "walladiab")},
                                {"x": ("inflow", "outflow"), "z": ("wallisoth", "wallisoth")}])
def test_free_stream_preserved(oracle_mod, bc):
    box = mesh.Box(2, 3, 2, 4, bc=bc)
    rho, p = 1.0, TWALL / GAMMA  # T = twall with mach = 1: E = rho twall / (gamma (gamma-1))
    q = _uniform(box, rho, (0.0, 0.0, 0.0), p)
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=400.0)
    c.set_q(q)
    c.set_boundary(TWALL, mesh.boundary_state(box, rho, (0.0, 0.0, 0.0), p),
                   np.zeros((box.nmort, 5, box.ldx, box.ldx)))
    qt = c.rhs()
    assert np.abs(qt).max() <= 1e-10 * p


def test_free_stream_through_inflow_outflow(oracle_mod):
    box = mesh.Box(3, 2, 2, 3, bc={"x": ("inflow", "outflow")})
    rho, vel, p = 1.2, (0.3, 0.05, -0.1), TWALL / GAMMA
    q = _uniform(box, rho, vel, p)
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=400.0)
    c.set_q(q)
    c.set_boundary(TWALL, mesh.boundary_state(box, rho, vel, p), None)
    assert np.abs(c.rhs()).max() <= 1e-10 * p


def test_wall_without_normal_velocity_passes_no_mass(oracle_mod):
    box = mesh.Box(2, 3, 2, 4, bc={"y": ("walladiab", "wallisoth")})
    x, y, z = (box.xg[..., k].reshape(box.nel, box.ldx, box.ldx, box.ldx) for k in range(3))
    G = 5
    q = np.zeros(box.qshape())
    jac = box.jacob.reshape(box.nel, box.ldx, box.ldx, box.ldx)
    s = np.s_[:, :G, :G, :G]
    rho = 1.0 + 0.1 * np.sin(x[s]) * np.cos(z[s]) + 0.05 * np.cos(y[s])
    u, w = 0.4 * np.sin(z[s]), 0.2 * np.cos(x[s])
    pr = TWALL / GAMMA * (1.0 + 0.02 * np.cos(y[s] + x[s]))
    for k, val in enumerate([rho, rho * u, 0.0 * rho, rho * w, pr / (GAMMA - 1.0) + 0.5 * rho * (u * u + w * w)]):
        q[:, k, :G, :G, :G] = val / jac[s]
    c = oracle_mod.Case.from_desc(box.desc())
    c.set_phys(re=300.0)
    c.set_q(q)
    c.set_boundary(TWALL)
    qt = c.rhs()[:, 0, :G, :G, :G]
    w1 = _weights(G)
    W = w1[:, None, None] * w1[None, :, None] * w1[None, None, :]
    total = float((qt * W).sum())
    scale = float((np.abs(qt) * W).sum())
    assert scale > 1.0
    assert abs(total) <= 1e-13 * scale, (total, scale)


@pytest.mark.parametrize("wall", ["walladiab", "wallisoth"])
def test_wall_shear_decay_spectral_convergence(oracle_mod, wall):
    """u = A sin(y/2) along x between no-slip walls at y = 0 and 2 pi (uniform density and
    pressure, the walls' temperature): u vanishes on both walls, so the walls' Roe flux, wall
    state and viscous wall flux (wallbc_Inv / wallbc_isoth, wall_vis_flux) see the exact
    solution, whose time derivatives are d(rho u)/dt = -A sin(y/2)/(4 Re) (mu u_yy),
    dE/dt = A^2 cos(y)/(4 Re) (the stress's work) and zero for the other components.  On
    2 x 3 x 2 elements the right-hand side converges to them spectrally as p grows."""
    re, A = 50.0, 0.5
    errs = []
    for p in (2, 4, 6, 8):
        box = mesh.Box(2, 3, 2, p, bc={"y": (wall, wall)})
        y = box.xg[..., 1]
        u = np.zeros(y.shape + (3,))
        u[..., 0] = A * np.sin(y / 2.0)
        c = oracle_mod.Case.from_desc(box.desc())
        c.set_phys(re=re)
        c.set_q(mesh._jq(box, np.ones_like(y), u, np.full_like(y, TWALL / GAMMA), GAMMA))
        c.set_boundary(TWALL)
        dq = c.rhs().reshape(box.nel, 5, -1) * box.jacob[:, None, :]
        m = box.jacob != 0
        sm, se = A / (4.0 * re), A * A / (4.0 * re)
        assert np.abs(dq[:, 3][m]).max() <= 1e-8 * sm  # z momentum: rounding only
        errs.append([np.abs(dq[:, 0][m]).max() / sm,
                     np.abs(dq[:, 1][m] + sm * np.sin(y[m] / 2.0)).max() / sm,
                     np.abs(dq[:, 2][m]).max() / sm,
                     np.abs(dq[:, 4][m] - se * np.cos(y[m])).max() / se])
    errs = np.array(errs)
    for k in range(1, 4):
        assert np.all(errs[k] <= 0.1 * errs[k - 1]), errs
    assert np.all(errs[-1] <= [1e-5, 1e-5, 1e-4, 1e-3]), errs


def test_inflow_outflow_density_wave_convergence(oracle_mod):
    """A density wave rho = 1 + a sin(x + 2y + z) convected at uniform velocity and pressure
    through an inflow face (x = 0) and an outflow face (x = 2 pi) whose external states are the
    exact solution at each mortar point (mrtr%Q(:,:,:,2), filled point by point in the
    mortar_xyz layout): continuity and momentum have the exact derivatives d rho/dt =
    -u.grad rho and d(rho u)/dt = u d rho/dt (no viscous stress), and the full right-hand
    side, inflow_specAll / outflow_specAll Riemann fluxes included, converges to them
    spectrally as p grows."""
    a, re = 0.2, 400.0
    U = np.array([0.4, 0.1, -0.1])
    p0 = TWALL / GAMMA

    def wave(xyz):
        s = xyz[..., 0] + 2.0 * xyz[..., 1] + xyz[..., 2]
        return 1.0 + a * np.sin(s), s

    errs = []
    for p in (2, 4, 6, 8):
        box = mesh.Box(3, 3, 2, p, bc={"x": ("inflow", "outflow")})
        rho, s = wave(box.xg)
        u = np.broadcast_to(U, rho.shape + (3,)).copy()
        c = oracle_mod.Case.from_desc(box.desc())
        c.set_phys(re=re)
        c.set_q(mesh._jq(box, rho, u, np.full_like(rho, p0), GAMMA))
        mx = box.mortar_xyz()
        qext = np.zeros((box.nmort, 5, box.ldx, box.ldx))
        for j in box.boundary_mortars():
            G = int(box.mortar[j, 8])
            r, _ = wave(mx[j, :G, :G])
            qext[j, :, :G, :G] = [r, r * U[0], r * U[1], r * U[2], p0 / (GAMMA - 1.0) + 0.5 * r * (U @ U)]
        c.set_boundary(TWALL, qext, None)
        dq = c.rhs().reshape(box.nel, 5, -1) * box.jacob[:, None, :]
        m = box.jacob != 0
        drho = -a * np.cos(s) * (U[0] + 2.0 * U[1] + U[2])
        errs.append(max(np.abs(dq[:, v][m] - ex[m]).max() for v, ex in
                        enumerate([drho, U[0] * drho, U[1] * drho, U[2] * drho])) / np.abs(drho[m]).max())
    for k in range(1, 4):
        assert errs[k] <= 0.15 * errs[k - 1], errs
    assert errs[-1] <= 5e-4, errs


def test_boundary_needs_its_condition(oracle_mod):
    box = mesh.Box(2, 2, 2, 3, bc={"z": ("walladiab", "outflow")})
    d = box.desc()
    d["bcond"] = np.zeros_like(d["bcond"])
    with pytest.raises(ValueError):
        oracle_mod.Case.from_desc(d)
