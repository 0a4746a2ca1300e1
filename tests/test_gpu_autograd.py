"""The adjoint through torch.autograd (dsem_b200.autograd): J.backward() returns
the library's adjoint gradients, and they agree with central differences of
the same objective evaluated through the autograd function (1e-6 relative, the
bar of the adjoint tests)."""
import numpy as np
import pytest

from dsem_b200 import mesh

pytestmark = pytest.mark.gpu


def _setup(re=500.0):
    box = mesh.Box(2, 2, 2, 3)
    q = mesh.random_isotropic(box, seed=7, k0=2.0, mach_t=0.2)
    dt = 0.5 * mesh.dtcalc(box, q)
    return box, q, dt


def test_backward_returns_the_adjoint_gradients():
    import torch
    from dsem_b200.autograd import AdjointCase, objective
    box, q, dt = _setup()
    case = AdjointCase(box.desc(), 500.0, dt, nsteps=4, window=2)
    jq0 = torch.tensor(q, dtype=torch.float64, requires_grad=True)
    inv_re = torch.tensor(1.0 / 500.0, dtype=torch.float64, requires_grad=True)
    J = objective(jq0, inv_re, case)
    J.backward()
    case.solver.upload(q)
    J_ref, g_ref, lr_ref, _ = case.solver.adjoint(dt, 4, 2)
    assert float(J.detach()) == J_ref
    assert np.array_equal(jq0.grad.numpy(), g_ref)
    assert float(inv_re.grad) == lr_ref
    # a scaled upstream gradient scales both
    jq0.grad = None
    inv_re.grad = None
    (3.0 * objective(jq0, inv_re, case)).backward()
    assert np.allclose(jq0.grad.numpy(), 3.0 * g_ref, rtol=0, atol=0)
    case.close()


def test_gradients_match_central_differences():
    import torch
    from dsem_b200.autograd import AdjointCase, objective
    re = 500.0
    box, q, dt = _setup(re)
    case = AdjointCase(box.desc(), re, dt, nsteps=3, window=3)
    jq0 = torch.tensor(q, dtype=torch.float64, requires_grad=True)
    inv_re = torch.tensor(1.0 / re, dtype=torch.float64, requires_grad=True)
    J = objective(jq0, inv_re, case)
    gq, gr = torch.autograd.grad(J, (jq0, inv_re))
    rng = np.random.default_rng(2)
    G = 4
    for _ in range(3):
        d = rng.standard_normal(q.shape)
        d[:, :, G:] = 0.0
        d[:, :, :, G:] = 0.0
        d[:, :, :, :, G:] = 0.0
        h = 1e-6 * np.abs(q[:, :, :G, :G, :G]).max() / np.abs(d).max()
        with torch.no_grad():
            jp = float(objective(torch.tensor(q + h * d), inv_re, case))
            jm = float(objective(torch.tensor(q - h * d), inv_re, case))
        fd = (jp - jm) / (2 * h)
        ad = float((gq * torch.tensor(d)).sum())
        assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)
    case.close()
    # d/d(1/Re): one context per Reynolds number
    r = 1.0 / re
    hr = 1e-5 * r
    vals = []
    for rr in (r + hr, r - hr):
        c2 = AdjointCase(box.desc(), 1.0 / rr, dt, nsteps=3, window=3)
        with torch.no_grad():
            vals.append(float(objective(torch.tensor(q), torch.tensor(rr, dtype=torch.float64), c2)))
        c2.close()
    fd = (vals[0] - vals[1]) / (2 * hr)
    assert abs(float(gr) - fd) <= 1e-6 * abs(fd), (float(gr), fd)


def test_inv_re_must_match_the_solver():
    import torch
    from dsem_b200.autograd import AdjointCase, objective
    box, q, dt = _setup()
    case = AdjointCase(box.desc(), 500.0, dt, nsteps=2, window=1)
    with pytest.raises(ValueError):
        objective(torch.tensor(q), torch.tensor(1.0 / 400.0, dtype=torch.float64), case)
    case.close()
