"""ctypes front end of the CPU oracle (test infrastructure, the checker).

Loads oracle/_build/libdsem_oracle.so, building it with `make` when it is
missing.  Arrays use the C-ABI layout of include/dsem_gpu.h: per element,
Fortran column-major blocks padded to an extent ``ldx``.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libdsem_oracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.orc_build_box.restype = vp
        L.orc_build_box.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [_ip, vp]
        L.orc_from_desc.restype = vp
        L.orc_from_desc.argtypes = [C.c_int, C.c_int, C.c_int, _ip, _dp, _dp, _dp, _ip, _dp, _dp]
        L.orc_free.argtypes = [vp]
        L.orc_set_phys.argtypes = [vp] + [C.c_double] * 6 + [C.c_int, C.c_int]
        for f in ("orc_nel", "orc_nmort", "orc_kord"):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = C.c_int
        L.orc_ncg.argtypes = [vp, C.c_int]
        L.orc_ncg.restype = C.c_int
        L.orc_export_desc.argtypes = [vp, C.c_int, _ip, _dp, _dp, _dp, _ip, _dp, _dp, _dp]
        L.orc_operators.argtypes = [C.c_int, _dp, _dp]
        L.orc_projection.argtypes = [C.c_int, C.c_int, _dp, _dp]
        L.orc_ke_weights.argtypes = [C.c_int, _dp]
        L.orc_init_tgv.argtypes = [vp, C.c_double, C.c_double]
        L.orc_set_q.argtypes = [vp, _dp, C.c_int]
        L.orc_get_q.argtypes = [vp, _dp, C.c_int]
        L.orc_get_lobatto.argtypes = [vp, _dp, C.c_int]
        L.orc_get_lobatto.restype = C.c_int
        L.orc_dtcalc.argtypes = [vp]
        L.orc_dtcalc.restype = C.c_double
        L.orc_rhs.argtypes = [vp, C.c_double, _dp, C.c_int]
        L.orc_stage.argtypes = [vp, C.c_double, C.c_double, C.c_int, vp, C.c_int]
        L.orc_stage.restype = C.c_int
        L.orc_step.argtypes = [vp, C.c_double, C.c_double, C.c_int]
        L.orc_step.restype = C.c_int
        L.orc_diag.argtypes = [vp, C.c_double, C.c_int] + [C.POINTER(C.c_double)] * 3
        L.orc_get_muhg.argtypes = [vp, _dp, C.c_int]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_threads.restype = C.c_int
        L.orc_rk.argtypes = [vp, _dp, _dp, _dp]
        L.orc_set_les.argtypes = [vp, C.c_double, C.c_double]
        L.orc_set_les_sensors.argtypes = [vp, C.c_int, C.c_int]
        L.orc_set_bcond.argtypes = [vp, _ip]
        L.orc_set_bcond.restype = C.c_int
        L.orc_set_boundary.argtypes = [vp, C.c_double, vp, vp, C.c_int]
        L.orc_get_nut.argtypes = [vp, _dp, C.c_int]
        L.orc_objective_cs.argtypes = [vp, C.c_double, C.c_int, C.c_int, vp, C.c_double, C.c_int,
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_riemann.argtypes = [_dp, C.c_double, _dp, _dp, C.c_double, _dp]
        L.orc_euler.argtypes = [_dp, C.c_double, _dp, _dp, _dp]
        L.orc_vis.argtypes = [_dp] * 4 + [C.c_double] * 4 + [_dp] * 3
        _lib = L
    return _lib


def operators(p):
    G, L = p + 1, p + 2
    d = np.zeros(G * L)
    b = np.zeros(L * G)
    lib().orc_operators(p, d, b)
    return d.reshape(G, L), b.reshape(L, G)


def projection(nin, nout):
    P = np.zeros(nout * nin)
    R = np.zeros(nin * nout)
    lib().orc_projection(nin, nout, P, R)
    return P.reshape(nout, nin), R.reshape(nin, nout)


def ke_weights(G):
    w = np.zeros(G ** 3)
    lib().orc_ke_weights(G, w)
    return w.reshape(G, G, G, order="F")


def riemann(n_hat, ds, Ql, Qr, gamma=1.4):
    f = np.zeros(5)
    lib().orc_riemann(np.ascontiguousarray(n_hat, float), ds, np.ascontiguousarray(Ql, float),
                      np.ascontiguousarray(Qr, float), gamma, f)
    return f


def euler(Q, gamma=1.4):
    f, g, h = np.zeros(5), np.zeros(5), np.zeros(5)
    lib().orc_euler(np.ascontiguousarray(Q, float), gamma, f, g, h)
    return f, g, h


def set_threads(n):
    return lib().orc_set_threads(n)


class Case:
    """One oracle case (mesh + state + physics)."""

    def __init__(self, handle):
        self.h = C.c_void_p(handle)
        L = lib()
        self.nel = L.orc_nel(self.h)
        self.nmort = L.orc_nmort(self.h)
        self.ncg = np.array([L.orc_ncg(self.h, e) for e in range(self.nel)], dtype=np.int32)
        self.ldx = int(self.ncg.max()) + 1

    @classmethod
    def box(cls, nex, ney, nez, orders, length=2 * np.pi, rot=None):
        orders = np.ascontiguousarray(np.broadcast_to(np.asarray(orders, dtype=np.int32), (nex * ney * nez,)))
        rp = None
        if rot is not None:
            rot = np.ascontiguousarray(rot, dtype=np.int32)
            rp = rot.ctypes.data_as(C.c_void_p)
        lx = ly = lz = length
        h = lib().orc_build_box(nex, ney, nez, lx, ly, lz, orders, rp)
        c = cls(h)
        c._keep = rot
        return c

    @classmethod
    def from_desc(cls, d):
        h = lib().orc_from_desc(d["ngrid"], d["nmort"], d["ldx"], d["ncg"], d["jacob"], d["gmetg"], d["gmet"],
                                d["mortar"], d["n_hat"], d["norm"])
        c = cls(h)
        if d.get("bcond") is not None:
            c.set_bcond(d["bcond"])
        return c

    def set_bcond(self, bcond):
        """d%bcond per element face ([ngrid][6] codes: 1 walladiab, 2 wallisoth, 3 inflow, 4 outflow)."""
        b = np.ascontiguousarray(bcond, dtype=np.int32).ravel()
        if lib().orc_set_bcond(self.h, b) != 0:
            raise ValueError("a boundary mortar's master face has no boundary condition")

    def set_boundary(self, twall, Qx=None, fvx=None):
        """twall and the external states of the boundary mortars ([nmort][5][ldx][ldx])."""
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (Qx, fvx)]
        ldx = next((a.shape[-1] for a in keep if a is not None), self.ldx)
        for a in keep:
            if a is not None and a.shape != (self.nmort, 5, ldx, ldx):
                raise ValueError("external states are [nmort][5][ldx][ldx]")
        ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        lib().orc_set_boundary(self.h, float(twall), ptr(keep[0]), ptr(keep[1]), ldx)

    def __del__(self):
        try:
            lib().orc_free(self.h)
        except Exception:
            pass

    def set_phys(self, gamma=1.4, re=1600.0, pr=0.72, mach=1.0, cmu=0.0, mumax=0.0, shock=0, iord=4):
        lib().orc_set_phys(self.h, gamma, re, pr, mach, cmu, mumax, int(shock), int(iord))

    def export_desc(self, ldx=None):
        ldx = ldx or self.ldx
        n = self.nel
        L3 = ldx ** 3
        d = dict(ngrid=n, nmort=self.nmort, ldx=ldx,
                 ncg=np.zeros(3 * n, np.int32), jacob=np.zeros(n * L3), gmetg=np.zeros(n * L3 * 9),
                 gmet=np.zeros(n * L3 * 9), mortar=np.zeros(17 * self.nmort, np.int32),
                 n_hat=np.zeros(self.nmort * ldx * ldx * 3), norm=np.zeros(self.nmort * ldx * ldx),
                 xg=np.zeros(n * L3 * 3))
        lib().orc_export_desc(self.h, ldx, d["ncg"], d["jacob"], d["gmetg"], d["gmet"], d["mortar"], d["n_hat"],
                              d["norm"], d["xg"])
        return d

    def qshape(self):
        return (self.nel, 5, self.ldx, self.ldx, self.ldx)

    def init_tgv(self, twall=100.0, v0=1.0):
        lib().orc_init_tgv(self.h, twall, v0)

    def set_q(self, JQ):
        JQ = np.ascontiguousarray(JQ, dtype=np.float64)
        lib().orc_set_q(self.h, JQ.ravel(), self.ldx)

    def get_q(self):
        q = np.zeros(self.qshape())
        lib().orc_get_q(self.h, q.ravel(), self.ldx)
        return q

    def lobatto(self):
        """Lobatto arrays of the last Fluxes call (d%Qlgg, d%Qglg, d%Qggl) as
        [nel][grid d][5][ldx][ldx][ldx] (x fastest, DSEM's padded layout), and
        whether they were ever computed."""
        out = np.zeros((self.nel, 3, 5, self.ldx, self.ldx, self.ldx))
        ok = lib().orc_get_lobatto(self.h, out.ravel(), self.ldx)
        return out, bool(ok)

    def dtcalc(self):
        return lib().orc_dtcalc(self.h)

    def rhs(self, tk=0.0):
        q = np.zeros(self.qshape())
        lib().orc_rhs(self.h, tk, q.ravel(), self.ldx)
        return q

    def stage(self, time, dt, kk, want_qt=True):
        q = np.zeros(self.qshape()) if want_qt else None
        st = lib().orc_stage(self.h, time, dt, kk, q.ctypes.data_as(C.c_void_p) if want_qt else None, self.ldx)
        return st, q

    def step(self, time, dt, nsteps=1):
        return lib().orc_step(self.h, time, dt, nsteps)

    def diag(self, dt, first):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        lib().orc_diag(self.h, dt, int(first), C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def muhg(self):
        m = np.zeros((self.nel, self.ldx, self.ldx, self.ldx))
        lib().orc_get_muhg(self.h, m.ravel(), self.ldx)
        return m

    def kord(self):
        return lib().orc_kord(self.h)

    def set_les(self, cs, numax):
        lib().orc_set_les(self.h, float(cs), float(numax))

    def set_les_sensors(self, shock_sensor, rho_sensor):
        lib().orc_set_les_sensors(self.h, int(bool(shock_sensor)), int(bool(rho_sensor)))

    def nut(self):
        m = np.zeros((self.nel, self.ldx, self.ldx, self.ldx))
        lib().orc_get_nut(self.h, m.ravel(), self.ldx)
        return m

    def objective_cs(self, dt, nsteps, window, dq=None, h=1e-30):
        """(J, dJ/dJQ . dq) of J = sum over the last `window` steps of dt * eps,
        by complex step from the current state; the case is not modified."""
        J, dJ = C.c_double(), C.c_double()
        dqa = None if dq is None else np.ascontiguousarray(dq, dtype=np.float64)
        lib().orc_objective_cs(self.h, float(dt), int(nsteps), int(window),
                               None if dqa is None else dqa.ctypes.data_as(C.c_void_p), float(h), self.ldx,
                               C.byref(J), C.byref(dJ))
        return J.value, dJ.value

    def rk(self):
        a, b, c = np.zeros(5), np.zeros(5), np.zeros(5)
        lib().orc_rk(self.h, a, b, c)
        return a, b, c
