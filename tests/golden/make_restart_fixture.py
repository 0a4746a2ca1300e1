"""Writes DSEM restart files in write_restart's record layout
(src/Parabolic3D/stac3m/restart.f90:19-312, through dsem_b200.restart_file)
for the restart tests: a 3 x 3 x 2 periodic box at p = 3 (padding nx = 5),
a seeded isotropic state, entropy viscosity on, advanced `steps` RK steps by
the CPU oracle; the file carries the oracle's state and, after at least one
step, its three Lobatto arrays (d%Qlgg, d%Qglg, d%Qggl), as DSEM's
write_restart would after the same steps.

    python tests/golden/make_restart_fixture.py OUT.rst [--steps N]
"""
import argparse
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PHYS = dict(re=500.0, cmu=1.0, mumax=0.5, shock=1)


def case():
    from dsem_b200 import mesh
    box = mesh.Box(3, 3, 2, 3)
    q0 = mesh.random_isotropic(box, seed=17, k0=1.5, mach_t=0.3)
    dt = 0.3 * mesh.dtcalc(box, q0)
    return box, q0, dt


def make(path, steps):
    """Writes the file; returns (box, q0, dt, oracle case after `steps` steps)."""
    from dsem_b200 import restart_file
    from oracle import oracle
    box, q0, dt = case()
    c = oracle.Case.from_desc(box.desc())
    c.set_phys(**PHYS)
    c.set_q(q0)
    if steps:
        c.step(0.0, dt, steps)
    lob, ok = c.lobatto()
    recs = restart_file.restart_records(box, c.get_q(), restart_file.Sizes(nx=box.ldx), lob if ok else None,
                                        time=steps * dt)
    restart_file.write(path, recs)
    return box, q0, dt, c


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("out")
    ap.add_argument("--steps", type=int, default=3)
    a = ap.parse_args()
    make(a.out, a.steps)
