"""ctypes front end of libdsem_b200.so (include/dsem_gpu.h).

`Solver` mirrors the Fortran call sites the library replaces: construction
packs the geometry (after 3DDriver_parfmdf.f90:307), `step` replaces the body
of tstep (src/tstep.f90:36-116), `diag` the KE/dissipation diagnostics.
There is no CPU fallback: a missing library or CUDA device raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libdsem_b200.so")

DSEM_OK = 0
ERRORS = {-1: "INVALID_ARG", -2: "CUDA", -3: "NONFINITE", -4: "TIMEOUT", -5: "UNSUPPORTED", -6: "NOMEM"}
VOL_VARIANTS = 5  # DSEM_VOL_VARIANTS: launch shapes of the volume kernel per order
EXPORTS = ("dsem_create", "dsem_destroy", "dsem_last_error", "dsem_upload_q", "dsem_download_q", "dsem_step",
           "dsem_stage", "dsem_rhs", "dsem_diag", "dsem_get_muhg", "dsem_last_timing", "dsem_profile_rhs",
           "dsem_create_batch", "dsem_batch_size", "dsem_upload_q_case", "dsem_download_q_case", "dsem_step_batch",
           "dsem_diag_batch", "dsem_adjoint", "dsem_set_les", "dsem_get_nut", "dsem_state_size",
           "dsem_save_state", "dsem_load_state", "dsem_shard_info", "dsem_shard_stage", "dsem_diag_sums",
           "dsem_set_boundary", "dsem_autotune", "dsem_set_vol_variant", "dsem_shard_enqueue", "dsem_shard_finish",
           "dsem_get_stream", "dsem_keep_lobatto", "dsem_write_restart", "dsem_read_restart",
           "dsem_set_les_sensors", "dsem_set_adjoint_scheme", "dsem_create_snapped")


class DsemError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dsem error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class MeshDesc(C.Structure):
    _fields_ = [("ngrid", C.c_int), ("nmort", C.c_int), ("ldx", C.c_int), ("ncg", C.POINTER(C.c_int)),
                ("jacob", C.POINTER(C.c_double)), ("gmetg", C.POINTER(C.c_double)), ("gmet", C.POINTER(C.c_double)),
                ("mortar", C.POINTER(C.c_int)), ("n_hat", C.POINTER(C.c_double)), ("norm", C.POINTER(C.c_double)),
                ("bcond", C.POINTER(C.c_int))]


class Phys(C.Structure):
    _fields_ = [("gamma", C.c_double), ("re", C.c_double), ("pr", C.c_double), ("mach", C.c_double),
                ("cmu", C.c_double), ("mumax", C.c_double), ("shock", C.c_int), ("iord", C.c_int)]


_lib = None


def lib(path=None):
    """Loads the in-tree library (building it with nvcc when it is missing)."""
    global _lib
    if _lib is None:
        p = path or LIB
        if not os.path.exists(p):
            from . import build
            build.build()
        L = C.CDLL(p)
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.dsem_create.argtypes = [C.POINTER(MeshDesc), C.POINTER(Phys), C.POINTER(vp)]
        L.dsem_create_snapped.argtypes = [C.POINTER(MeshDesc), C.POINTER(Phys), C.c_double, C.POINTER(vp)]
        L.dsem_destroy.argtypes = [vp]
        L.dsem_last_error.argtypes = [vp]
        L.dsem_last_error.restype = C.c_char_p
        L.dsem_upload_q.argtypes = [vp, dp, C.c_int]
        L.dsem_download_q.argtypes = [vp, dp, C.c_int]
        L.dsem_step.argtypes = [vp, C.c_double, C.c_double, C.c_int]
        L.dsem_stage.argtypes = [vp, C.c_double, C.c_double, C.c_int, dp, C.c_int]
        L.dsem_rhs.argtypes = [vp, C.c_double, dp, C.c_int]
        L.dsem_diag.argtypes = [vp, C.c_double, C.c_int, dp, dp, dp]
        L.dsem_get_muhg.argtypes = [vp, dp, C.c_int]
        L.dsem_last_timing.argtypes = [vp, dp, C.POINTER(C.c_longlong)]
        L.dsem_profile_rhs.argtypes = [vp, C.c_int, dp]
        L.dsem_create_batch.argtypes = [C.c_int, C.POINTER(MeshDesc), C.POINTER(Phys), C.POINTER(vp)]
        L.dsem_batch_size.argtypes = [vp]
        L.dsem_upload_q_case.argtypes = [vp, C.c_int, dp, C.c_int]
        L.dsem_download_q_case.argtypes = [vp, C.c_int, dp, C.c_int]
        L.dsem_step_batch.argtypes = [vp, dp, C.c_int]
        L.dsem_diag_batch.argtypes = [vp, dp, C.c_int, dp, dp, dp]
        L.dsem_set_les.argtypes = [vp, C.c_double, C.c_double]
        L.dsem_set_les_sensors.argtypes = [vp, C.c_int, C.c_int]
        L.dsem_set_adjoint_scheme.argtypes = [vp, C.c_int]
        L.dsem_set_boundary.argtypes = [vp, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]
        L.dsem_autotune.argtypes = [vp, C.c_int, C.POINTER(C.c_int), dp]
        L.dsem_set_vol_variant.argtypes = [vp, C.c_int, C.c_int]
        L.dsem_shard_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(dp), C.POINTER(dp)]
        L.dsem_shard_stage.argtypes = [vp, C.c_double, C.c_int, C.c_int]
        L.dsem_shard_enqueue.argtypes = [vp, C.c_double, C.c_int, C.c_int]
        L.dsem_shard_finish.argtypes = [vp]
        L.dsem_get_stream.argtypes = [vp, C.POINTER(vp)]
        L.dsem_keep_lobatto.argtypes = [vp, C.c_int]
        L.dsem_write_restart.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_int, C.c_double]
        L.dsem_read_restart.argtypes = [vp, C.c_char_p, C.c_int, C.POINTER(C.c_double)]
        L.dsem_diag_sums.argtypes = [vp, dp]
        L.dsem_state_size.argtypes = [vp, C.POINTER(C.c_longlong)]
        L.dsem_save_state.argtypes = [vp, C.c_void_p, C.c_longlong]
        L.dsem_load_state.argtypes = [vp, C.c_void_p, C.c_longlong]
        L.dsem_get_nut.argtypes = [vp, dp, C.c_int]
        L.dsem_adjoint.argtypes = [vp, C.c_double, C.c_int, C.c_int, C.c_int, dp, dp, C.c_int, dp, dp]
        _lib = L
    return _lib


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _mesh_desc(desc):
    """(MeshDesc, arrays kept alive while the descriptor is in use)."""
    a = {k: np.ascontiguousarray(desc[k]) for k in ("ncg", "jacob", "gmetg", "gmet", "mortar", "n_hat", "norm")}
    assert a["ncg"].dtype == np.int32 and a["mortar"].dtype == np.int32
    bc = desc.get("bcond")
    if bc is not None:
        a["bcond"] = np.ascontiguousarray(bc, dtype=np.int32)
    md = MeshDesc(int(desc["ngrid"]), int(desc["nmort"]), int(desc["ldx"]), _iptr(a["ncg"]), _dptr(a["jacob"]),
                  _dptr(a["gmetg"]), _dptr(a["gmet"]), _iptr(a["mortar"]), _dptr(a["n_hat"]), _dptr(a["norm"]),
                  _iptr(a["bcond"]) if bc is not None else None)
    return md, a


class Solver:
    """One device context: geometry + state resident in HBM."""

    def __init__(self, desc, gamma=1.4, re=1600.0, pr=0.72, mach=1.0, cmu=0.0, mumax=0.0, shock=0, iord=4,
                 metric_snap=0.0):
        """metric_snap > 0: dsem_create_snapped (metric rounding noise up to that relative
        size is treated as zero, so noisy axis-aligned elements take the diagonal kernel)."""
        L = lib()
        md, self._arrays = _mesh_desc(desc)
        self.ngrid, self.nmort, self.ldx = int(desc["ngrid"]), int(desc["nmort"]), int(desc["ldx"])
        ph = Phys(gamma, re, pr, mach, cmu, mumax, int(shock), int(iord))
        h = C.c_void_p()
        if metric_snap:
            rc = L.dsem_create_snapped(C.byref(md), C.byref(ph), float(metric_snap), C.byref(h))
        else:
            rc = L.dsem_create(C.byref(md), C.byref(ph), C.byref(h))
        if rc != DSEM_OK:
            raise DsemError(rc, L.dsem_last_error(None).decode())
        self.h = h
        self.kord = 5 if iord == 4 else iord

    def _check(self, rc):
        if rc != DSEM_OK:
            raise DsemError(rc, lib().dsem_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            lib().dsem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def qshape(self, ldx=None):
        ldx = ldx or self.ldx
        return (self.ngrid, 5, ldx, ldx, ldx)

    def upload(self, JQ):
        JQ = np.ascontiguousarray(JQ, dtype=np.float64)
        self._check(lib().dsem_upload_q(self.h, _dptr(JQ), JQ.shape[-1]))

    def download(self, out=None, ldx=None):
        out = np.zeros(self.qshape(ldx)) if out is None else out
        self._check(lib().dsem_download_q(self.h, _dptr(out), out.shape[-1]))
        return out

    def step(self, dt, nsteps=1, time=0.0):
        self._check(lib().dsem_step(self.h, time, dt, nsteps))

    def stage(self, dt, kk, time=0.0, want_qt=True):
        q = np.zeros(self.qshape()) if want_qt else None
        self._check(lib().dsem_stage(self.h, time, dt, kk, _dptr(q) if want_qt else None, self.ldx))
        return q

    def rhs(self, tk=0.0):
        q = np.zeros(self.qshape())
        self._check(lib().dsem_rhs(self.h, tk, _dptr(q), self.ldx))
        return q

    def diag(self, dt, first=False):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        self._check(lib().dsem_diag(self.h, dt, int(first), C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def muhg(self):
        m = np.zeros((self.ngrid, self.ldx, self.ldx, self.ldx))
        self._check(lib().dsem_get_muhg(self.h, _dptr(m), self.ldx))
        return m

    def profile_rhs(self, reps=5):
        """Mean device milliseconds per RHS of {inviscid face, volume, viscous face, update}."""
        ms = np.zeros(4)
        self._check(lib().dsem_profile_rhs(self.h, int(reps), _dptr(ms)))
        return ms

    def keep_lobatto(self, on=True):
        """The last stage of every step keeps its Lobatto arrays (d%Qlgg/Qglg/Qggl) for restart files."""
        self._check(lib().dsem_keep_lobatto(self.h, int(bool(on))))

    def write_restart(self, template, out, time=0.0, max_materials=1):
        """DSEM restart file `out`: `template` (a DSEM restart file of the same mesh) with this
        context's state (dsem_write_restart)."""
        self._check(lib().dsem_write_restart(self.h, str(template).encode(), str(out).encode(), int(max_materials),
                                             float(time)))

    def read_restart(self, path, max_materials=1):
        """State (and, when present, the Lobatto arrays the next step's viscosity models read)
        from a DSEM restart file; returns its time (dsem_read_restart)."""
        t = C.c_double()
        self._check(lib().dsem_read_restart(self.h, str(path).encode(), int(max_materials), C.byref(t)))
        return t.value

    def save_state(self):
        """Snapshot of the device state (bytes) for dsem_load_state."""
        n = C.c_longlong()
        self._check(lib().dsem_state_size(self.h, C.byref(n)))
        buf = np.zeros(n.value, dtype=np.uint8)
        self._check(lib().dsem_save_state(self.h, buf.ctypes.data_as(C.c_void_p), n.value))
        return buf

    def load_state(self, buf):
        buf = np.ascontiguousarray(buf, dtype=np.uint8)
        self._check(lib().dsem_load_state(self.h, buf.ctypes.data_as(C.c_void_p), buf.size))

    def set_boundary(self, twall, Qext=None, fvext=None):
        """Wall temperature and external states of the boundary mortars
        ([nmort][5][ldx][ldx] each, or None)."""
        keep = [None if x is None else np.ascontiguousarray(x, dtype=np.float64) for x in (Qext, fvext)]
        ldx = next((x.shape[-1] for x in keep if x is not None), self.ldx)
        for x in keep:
            if x is not None and x.shape != (self.nmort, 5, ldx, ldx):
                raise ValueError("external states are [nmort][5][ldx][ldx]")
        self._check(lib().dsem_set_boundary(self.h, float(twall), None if keep[0] is None else _dptr(keep[0]),
                                            None if keep[1] is None else _dptr(keep[1]), int(ldx)))

    def autotune(self, reps=5):
        """Times the volume kernel's launch shapes per element order and keeps the
        fastest: returns {p: chosen shape} and ms[p-1][shape] (-1: not timed)."""
        choice = np.zeros(8, dtype=np.int32)
        ms = np.zeros((8, VOL_VARIANTS))
        self._check(lib().dsem_autotune(self.h, int(reps), choice.ctypes.data_as(C.POINTER(C.c_int)), _dptr(ms)))
        orders = sorted({p for p in range(1, 9) if ms[p - 1, 0] >= 0})
        return {p: int(choice[p - 1]) for p in orders}, ms

    def set_vol_variant(self, p, variant):
        self._check(lib().dsem_set_vol_variant(self.h, int(p), int(variant)))

    def set_les(self, cs, numax):
        """Static Smagorinsky model (cs = 0: off)."""
        self._check(lib().dsem_set_les(self.h, float(cs), float(numax)))

    def set_les_sensors(self, shock_sensor=False, rho_sensor=False):
        """DSEM's shockSensor / rhoSensor scaling of the Smagorinsky viscosity."""
        self._check(lib().dsem_set_les_sensors(self.h, int(bool(shock_sensor)), int(bool(rho_sensor))))

    def nut(self):
        m = np.zeros((self.ngrid, self.ldx, self.ldx, self.ldx))
        self._check(lib().dsem_get_nut(self.h, _dptr(m), self.ldx))
        return m

    ADJ_SCHEMES = {"revolve": 0, "segments": 1}

    def adjoint(self, dt, nsteps, window, snapshots=0, want_grad=True, scheme="revolve"):
        """J = sum of eps*dt over the last `window` of `nsteps` steps and its
        gradient: returns (J, dJ/dJQ0 in the upload layout or None, dJ/d(1/Re), ms).
        snapshots > 0 recomputes steps by `scheme`: "revolve" (binomial
        checkpointing) or "segments" (snapshots at segment starts plus the stage
        states of the segment being reversed); see dsem_set_adjoint_scheme."""
        self._check(lib().dsem_set_adjoint_scheme(self.h, self.ADJ_SCHEMES[scheme]))
        J, lr, ms = C.c_double(), C.c_double(), C.c_double()
        g = np.zeros(self.qshape()) if want_grad else None
        self._check(lib().dsem_adjoint(self.h, float(dt), int(nsteps), int(window), int(snapshots), C.byref(J),
                                       _dptr(g) if want_grad else None, self.ldx, C.byref(lr), C.byref(ms)))
        return J.value, g, lr.value, ms.value

    def last_timing(self):
        ms, n = C.c_double(), C.c_longlong()
        self._check(lib().dsem_last_timing(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value


class Ensemble(Solver):
    """Several independent cases advanced together (dsem_create_batch).

    descs: mesh descriptors (each with its own order and padding); res: one
    Reynolds number per case; the other physics parameters are shared.
    """

    def __init__(self, descs, res, gamma=1.4, pr=0.72, mach=1.0, cmu=0.0, mumax=0.0, shock=0, iord=4):
        L = lib()
        n = len(descs)
        assert len(res) == n and n > 0
        mds = (MeshDesc * n)()
        phs = (Phys * n)()
        self._keep = []
        for k, d in enumerate(descs):
            md, arrs = _mesh_desc(d)
            self._keep.append(arrs)
            mds[k] = md
            phs[k] = Phys(gamma, float(res[k]), pr, mach, cmu, mumax, int(shock), int(iord))
        h = C.c_void_p()
        rc = L.dsem_create_batch(n, mds, phs, C.byref(h))
        if rc != DSEM_OK:
            raise DsemError(rc, L.dsem_last_error(None).decode())
        self.h = h
        self.ncase = n
        self.case_ngrid = [int(d["ngrid"]) for d in descs]
        self.case_ldx = [int(d["ldx"]) for d in descs]
        self.ngrid = sum(self.case_ngrid)
        self.ldx = max(self.case_ldx)
        self.kord = 5 if iord == 4 else iord

    def upload_case(self, k, JQ):
        JQ = np.ascontiguousarray(JQ, dtype=np.float64)
        self._check(lib().dsem_upload_q_case(self.h, int(k), _dptr(JQ), JQ.shape[-1]))

    def download_case(self, k, ldx=None):
        ldx = ldx or self.case_ldx[k]
        out = np.zeros((self.case_ngrid[k], 5, ldx, ldx, ldx))
        self._check(lib().dsem_download_q_case(self.h, int(k), _dptr(out), ldx))
        return out

    def step_batch(self, dts, nsteps=1):
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        assert dts.shape == (self.ncase,)
        self._check(lib().dsem_step_batch(self.h, _dptr(dts), int(nsteps)))

    def diag_batch(self, dts, first=False):
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        ke, dk, ep = (np.zeros(self.ncase) for _ in range(3))
        self._check(lib().dsem_diag_batch(self.h, _dptr(dts), int(first), _dptr(ke), _dptr(dk), _dptr(ep)))
        return ke, dk, ep
