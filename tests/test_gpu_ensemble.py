"""Ensembles (dsem_create_batch): independent cases advanced by shared launches.

Every case of an ensemble must give bit for bit what its own single-case
context gives (and so what the oracle gives): the batch only changes which
elements share a launch, never the arithmetic of an element.  Cases mix
orders (several order groups run as parallel graph branches), Reynolds
numbers, time steps, sizes and initial conditions, like the 64-case ensemble
benchmark (E in {4^3..12^3}, p in {4,6,8}, Re in [400,3200]).
"""
import numpy as np
import pytest

from dsem_b200 import mesh

pytestmark = pytest.mark.gpu

CASES = [  # (n, p, Re, initial condition)
    (2, 4, 800.0, "tgv"),
    (3, 3, 1600.0, "iso"),
    (2, 6, 2400.0, "tgv"),
    (2, 4, 400.0, "iso"),
    (3, 2, 3200.0, "tgv"),
]


def _build(cases):
    boxes, qs, dts = [], [], []
    for k, (n, p, re, ic) in enumerate(cases):
        box = mesh.Box(n, n, n, p)
        q = mesh.taylor_green(box) if ic == "tgv" else mesh.random_isotropic(box, seed=100 + k, k0=2.0, mach_t=0.2)
        boxes.append(box)
        qs.append(q)
        dts.append(0.5 * mesh.dtcalc(box, q))
    return boxes, qs, np.array(dts)


def _singles(boxes, qs, dts, cases, nsteps):
    from dsem_b200.solver import Solver
    out, diags = [], []
    for box, q, dt, (n, p, re, ic) in zip(boxes, qs, dts, cases):
        s = Solver(box.desc(), re=re)
        s.upload(q)
        d0 = s.diag(dt, first=True)
        s.step(dt, nsteps)
        d1 = s.diag(dt)
        out.append(s.download())
        diags.append((d0, d1))
        s.close()
    return out, diags


def test_ensemble_matches_single_runs():
    from dsem_b200.solver import Ensemble
    boxes, qs, dts = _build(CASES)
    ens = Ensemble([b.desc() for b in boxes], [c[2] for c in CASES])
    assert ens.ncase == len(CASES)
    for k, q in enumerate(qs):
        ens.upload_case(k, q)
    ke0, dk0, ep0 = ens.diag_batch(dts, first=True)
    ens.step_batch(dts, 3)
    ke1, dk1, ep1 = ens.diag_batch(dts)
    ref, diags = _singles(boxes, qs, dts, CASES, 3)
    for k in range(len(CASES)):
        got = ens.download_case(k)
        assert np.isfinite(got).all()
        assert np.array_equal(got, ref[k]), k
        (a0, b0, c0), (a1, b1, c1) = diags[k]
        assert (ke0[k], dk0[k], ep0[k]) == (a0, b0, c0), k
        assert (ke1[k], dk1[k], ep1[k]) == (a1, b1, c1), k
    ens.close()


def test_ensemble_one_dt_and_concatenated_state(oracle_mod):
    """dsem_step (one dt for all cases) and the concatenated upload/download."""
    from dsem_b200.solver import Ensemble
    cases = [(2, 4, 1600.0, "tgv"), (2, 4, 800.0, "iso")]
    boxes, qs, dts = _build(cases)
    dt = float(dts.min())
    ens = Ensemble([b.desc() for b in boxes], [c[2] for c in cases])
    ens.upload(np.concatenate(qs))
    ens.step(dt, 2)
    got = ens.download()
    ref, _ = _singles(boxes, qs, np.full(len(cases), dt), cases, 2)
    assert np.array_equal(got, np.concatenate(ref))
    # and case 1 against the oracle
    c = oracle_mod.Case.from_desc(boxes[1].desc())
    c.set_phys(re=800.0)
    c.set_q(qs[1])
    c.step(0.0, dt, 2)
    assert np.array_equal(ens.download_case(1), c.get_q())
    ens.close()


def test_ensemble_cases_of_every_order_match_oracle(oracle_mod):
    """One case of each order the 64-case benchmark draws (p = 4, 6, 8), in one ensemble with
    different Re, dt and initial conditions: each case after 3 steps against the CPU oracle's
    run of that case alone, bit for bit (tstep.f90:36-116 per case)."""
    from dsem_b200.solver import Ensemble
    cases = [(3, 4, 2900.0, "iso"), (2, 6, 450.0, "tgv"), (2, 8, 1700.0, "iso")]
    boxes, qs, dts = _build(cases)
    ens = Ensemble([b.desc() for b in boxes], [c[2] for c in cases])
    for k, q in enumerate(qs):
        ens.upload_case(k, q)
    ens.step_batch(dts, 3)
    for k, (box, q, dt, (n, p, re, ic)) in enumerate(zip(boxes, qs, dts, cases)):
        c = oracle_mod.Case.from_desc(box.desc())
        c.set_phys(re=re)
        c.set_q(q)
        c.step(0.0, float(dt), 3)
        assert np.array_equal(ens.download_case(k), c.get_q()), (k, p)
    ens.close()
