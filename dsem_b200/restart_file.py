"""DSEM's restart file layout on the host: write_restart / read_restart
(src/Parabolic3D/stac3m/restart.f90:19-312, 319-929), the branch without
`defined_resolution`.

The file is Fortran unformatted sequential: one record per WRITE statement,
framed by its length in bytes as a 4-byte little-endian integer before and
after.  INTEGER and LOGICAL are 4 bytes, DOUBLE PRECISION 8, CHARACTER(n) n
bytes; arrays are column-major.  Sizes come from DSEM's size.f90 (`Sizes`).

    records(path)                 every record of a file, as bytes
    write(path, records)          a file from records
    restart_records(box, q, ...)  the records write_restart produces for a
                                  mesh.Box, its J*Q state and (optionally) its
                                  three Lobatto arrays and the time
    state(path, box, sizes)       (Q, Lobatto arrays, time) read back from a file

The library reads and writes these files from device state (dsem_write_restart
and dsem_read_restart in include/dsem_gpu.h); this module lets a test or a user
build one from the documented layout and look inside one.
"""
import struct
from dataclasses import dataclass

import numpy as np


@dataclass
class Sizes:
    """size.f90 parameters the layout depends on (DSEM's Taylor-Green case:
    caseFiles/tgv/size.f90): padding nx = ny = nz = nmax, max_orders,
    max_materials, mxprops; neq = 5."""
    nx: int
    max_orders: int = 3
    max_materials: int = 1
    num_prop: int = 1

    @property
    def max_mrtr_mat(self):
        return self.max_orders * self.max_orders // 2 + 1


def records(path):
    out = []
    with open(path, "rb") as f:
        while True:
            h = f.read(4)
            if not h:
                return out
            n = struct.unpack("<i", h)[0]
            data = f.read(n)
            t = struct.unpack("<i", f.read(4))[0]
            if t != n or len(data) != n:
                raise ValueError("malformed record")
            out.append(data)


def write(path, recs):
    with open(path, "wb") as f:
        for r in recs:
            f.write(struct.pack("<i", len(r)))
            f.write(r)
            f.write(struct.pack("<i", len(r)))


def _i(*v):
    return np.asarray(v, dtype="<i4").tobytes()


def _d(a):
    return np.ascontiguousarray(a, dtype="<f8").tobytes()


def restart_records(box, q, sizes, lobatto=None, time=0.0):
    """The records write_restart writes for box (single order per element,
    nx >= p+2) with state q (J*Q as [nel][5][ldx]^3, ldx = nx) and optional
    Lobatto arrays [nel][3][5][nx]^3 (DSEM's d%Qlgg, d%Qglg, d%Qggl; zero when
    absent, as after zero_domain).  Records outside the hot path (operator
    matrices, fluxes f/g/h, mortar states, statistics) are zero-filled: only
    their sizes matter to a reader."""
    nx, mo = sizes.nx, sizes.max_orders
    if box.ldx != nx:
        raise ValueError("box.ldx must equal the padding nx")
    n3 = nx ** 3
    recs = [_i(box.nel, box.nmort), _i(1, 1, 1), _i(*([0] * (3 * mo)))]
    recs += [_d(np.zeros(nx * nx * mo))] * 6  # bx by bz dmx dmy dmz
    recs += [_i(0), _i(*([0] * (2 * sizes.max_mrtr_mat)))]
    recs += [_d(np.zeros(nx * nx * sizes.max_mrtr_mat))] * 2  # prolong restrict
    q = np.asarray(q).reshape(box.nel, 5 * n3)
    lob = np.zeros((box.nel, 3, 5 * n3)) if lobatto is None else np.asarray(lobatto).reshape(box.nel, 3, 5 * n3)
    zero5 = _d(np.zeros(5 * n3))
    for e in range(box.nel):
        G = int(box.G[e])
        mort = np.zeros((6, 2), dtype=np.int32)  # (2,6): mortar # and side per face
        mort[:, 0] = box.emort[e] + 1
        mort[:, 1] = box.mside[e]
        recs += [_i(8), _i(*(list(box.node[e] + 1) + [0] * 18)), _i(*([0] * 6)), _i(*mort.ravel()),
                 _i(*([0] * 6)), _i(G + 1, G + 1, G + 1, G, G, G), _d(q[e]),
                 _d(lob[e, 0]), _d(lob[e, 1]), _d(lob[e, 2]), zero5, zero5, zero5, zero5, _i(1),
                 _d(np.zeros(2 * 3 * nx)), _d(box.xg[e]), _d(box.jacob[e]), _d(box.gmet[e]), _d(box.gmetg[e]),
                 _d(box.corner[e].ravel()), _i(*([0] * 6)),
                 b"".join((b"interface" if not box.boundary[e, f] else b"wall     ") for f in range(6)),
                 b"hex8    "]
    mrt = np.asarray(box.mortar).reshape(box.nmort, 17)
    nh = np.asarray(box.n_hat).reshape(box.nmort, -1)
    nr = np.asarray(box.norm).reshape(box.nmort, -1)
    for j in range(box.nmort):
        t = mrt[j]
        recs += [_i(t[8], t[9]), _i(t[4], t[5], t[6], t[7]), _i(t[0], t[1]), _i(t[2], t[3]), _i(t[10]), _i(t[11]),
                 _i(t[12]), _d(nh[j]), _d(nr[j]), _d(np.zeros(nx * nx * 10)), _d(np.zeros(nx * nx * 10)),
                 _d(np.zeros(3 * nx * nx)), _i(*(int(x != 0) for x in t[13:17]))]
    recs.append(_i(sizes.num_prop))
    recs += [_d(np.zeros(sizes.num_prop))] * sizes.max_materials
    recs.append(_d([time]))  # write_restart_case (caseFiles/tgv/BackstepProblem-stoch.f90:1876-1895)
    return recs


def state(path, box, sizes):
    """(J*Q [nel][5][nx]^3, Lobatto arrays [nel][3][5][nx]^3, time) of a restart file."""
    r = records(path)
    nx, n3 = sizes.nx, sizes.nx ** 3
    hdr = np.frombuffer(r[0], dtype="<i4")
    if int(hdr[0]) != box.nel:
        raise ValueError("element count differs")
    q = np.zeros((box.nel, 5, nx, nx, nx))
    lob = np.zeros((box.nel, 3, 5, nx, nx, nx))
    base = 13
    for e in range(box.nel):
        rr = r[base + 24 * e: base + 24 * (e + 1)]
        q[e] = np.frombuffer(rr[6], dtype="<f8").reshape(5, nx, nx, nx)
        for d in range(3):
            lob[e, d] = np.frombuffer(rr[7 + d], dtype="<f8").reshape(5, nx, nx, nx)
    k = base + 24 * box.nel + 13 * int(hdr[1]) + 1 + sizes.max_materials
    time = struct.unpack("<d", r[k])[0] if k < len(r) and len(r[k]) == 8 else 0.0
    return q, lob, time
