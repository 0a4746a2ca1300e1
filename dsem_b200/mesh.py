"""Mesh descriptors for standalone runs: periodic boxes of hex8 elements, straight or
curved by a smooth periodic deformation (Box(warp=...)).

DSEM's Fortran driver computes the geometry itself and packs it into the
descriptor of include/dsem_gpu.h.  For runs without it this module builds the
same arrays with the same rules:

* element numbering of the shipped TGV mesh (y fastest, then x, then z) and
  hex8 corner order (Grid_Routines/read_mesh.f90:459-506);
* mortars from shared faces, master = first element to present the face,
  orientation from the corner correspondence (Grid_Routines/set_mortars.f90:20-224,
  Grid_Routines/face_operations.f90:404-456);
* periodic pairing of boundary faces z (3 -> 5), y (1 -> 2), x (4 <- 6)
  (caseFiles/tgv/BackstepProblem-stoch.f90:173-278);
* metrics at Gauss points and on the three staggered grids, mortar normals
  from the master element (Grid_Routines/set_domain_geometry.f90:8-348,
  Grid_Routines/GeomLib3D.f90:60-146,685-734);
* nsign from the face normals (Grid_Routines/set_mortars.f90:240-372).

Arrays are returned in the C-ABI layout (Fortran column-major, padded to ldx).
"""
import math

import numpy as np

NV = 5
CORNER_XYZ = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])
FACE_MAP = [(0, 1, 5, 4), (3, 2, 6, 7), (0, 1, 2, 3), (1, 2, 6, 5), (4, 5, 6, 7), (0, 3, 7, 4)]
SIGN_LOW = {1: -1, 3: -1, 6: -1, 2: 1, 4: 1, 5: 1}
END_VALS = [0.0, 1.0, 0.0, 1.0, 1.0, 0.0]
FACE_DIR = {1: 1, 2: 1, 3: 2, 5: 2, 4: 0, 6: 0}


def lobatto_points(L):
    return np.array([0.5 * (1.0 - math.cos(float(n) * math.pi / float(L - 1))) for n in range(L)])


def gauss_points(G):
    return np.array([0.5 * (1.0 - math.cos((2.0 * n - 1.0) * math.pi / (2.0 * (float(G) - 1.0) + 2.0)))
                     for n in range(1, G + 1)])


def rotations():
    """The 24 proper rotations of the reference cube as signed permutation matrices."""
    out = []
    for perm in ([0, 1, 2], [0, 2, 1], [1, 0, 2], [1, 2, 0], [2, 0, 1], [2, 1, 0]):
        for s in range(8):
            M = np.zeros((3, 3), dtype=int)
            for i in range(3):
                M[i, perm[i]] = -1 if (s >> i) & 1 else 1
            if round(np.linalg.det(M)) == 1:
                out.append(M)
    return out


_ROT = rotations()


def _side_map(a, b):
    sm = [[-99, 1, -99, 2], [-1, -99, 2, -99], [-99, -2, -99, -1], [-2, -99, 1, -99]]
    return sm[a][b]


_ORIENT = {(1, 2): 0, (-1, 2): 1, (-1, -2): 2, (1, -2): 3, (2, 1): 4, (-2, 1): 5, (-2, -1): 6, (2, -1): 7}


def faces_match(tn, sn):
    c = [sn.index(x) for x in tn]
    return _ORIENT[(_side_map(c[0], c[1]), _side_map(c[0], c[3]))]


def grad_hex8(c, cx, cy, cz):
    """grad_hex8_map for corners c[..., 8, 3] at computational points (broadcast)."""
    g = np.empty(np.broadcast(cx, cy, cz, c[..., 0, 0]).shape + (3, 3))
    for i in range(3):
        c0, c1, c2, c3, c4, c5, c6, c7 = (c[..., k, i] for k in range(8))
        g[..., i, 0] = (-c0 * (1.0 - cy) * (1.0 - cz) + c1 * (1.0 - cy) * (1.0 - cz) + c2 * cy * (1.0 - cz)
                        - c3 * cy * (1.0 - cz) - c4 * (1.0 - cy) * cz + c5 * (1.0 - cy) * cz + c6 * cy * cz
                        - c7 * cy * cz)
        g[..., i, 1] = (-c0 * (1.0 - cx) * (1.0 - cz) - c1 * cx * (1.0 - cz) + c2 * cx * (1.0 - cz)
                        + c3 * (1.0 - cx) * (1.0 - cz) - c4 * (1.0 - cx) * cz - c5 * cx * cz + c6 * cx * cz
                        + c7 * (1.0 - cx) * cz)
        g[..., i, 2] = (-c0 * (1.0 - cx) * (1.0 - cy) - c1 * cx * (1.0 - cy) - c2 * cx * cy
                        - c3 * (1.0 - cx) * cy + c4 * (1.0 - cx) * (1.0 - cy) + c5 * cx * (1.0 - cy)
                        + c6 * cx * cy + c7 * (1.0 - cx) * cy)
    return g


def hex8(c, cx, cy, cz):
    x = np.empty(np.broadcast(cx, cy, cz, c[..., 0, 0]).shape + (3,))
    for j in range(3):
        c0, c1, c2, c3, c4, c5, c6, c7 = (c[..., k, j] for k in range(8))
        x[..., j] = (c0 * (1.0 - cx) * (1.0 - cy) * (1.0 - cz) + c1 * cx * (1.0 - cy) * (1.0 - cz)
                     + c2 * cx * cy * (1.0 - cz) + c3 * (1.0 - cx) * cy * (1.0 - cz)
                     + c4 * (1.0 - cx) * (1.0 - cy) * cz + c5 * cx * (1.0 - cy) * cz
                     + c6 * cx * cy * cz + c7 * (1.0 - cx) * cy * cz)
    return x


def invert_metric(gx):
    """Invert_Metric_Tensor: returns grad_cx[..., i, j] = dX_i/dx_j and J."""
    small = 100 * np.finfo(float).eps
    comp = {(i, j): np.ascontiguousarray(gx[..., i, j]) for i in range(3) for j in range(3)}
    g = lambda i, j: comp[i, j]
    J = (g(0, 0) * g(1, 1) * g(2, 2) - g(0, 1) * g(1, 0) * g(2, 2) - g(0, 0) * g(1, 2) * g(2, 1)
         + g(0, 2) * g(1, 0) * g(2, 1) + g(0, 1) * g(1, 2) * g(2, 0) - g(0, 2) * g(1, 1) * g(2, 0))
    gc = np.empty_like(gx)
    gc[..., 0, 0] = (g(1, 1) * g(2, 2) - g(1, 2) * g(2, 1)) / J
    gc[..., 1, 0] = (-g(1, 0) * g(2, 2) + g(1, 2) * g(2, 0)) / J
    gc[..., 2, 0] = (g(1, 0) * g(2, 1) - g(2, 0) * g(1, 1)) / J
    gc[..., 0, 1] = (-g(0, 1) * g(2, 2) + g(0, 2) * g(2, 1)) / J
    gc[..., 1, 1] = (g(0, 0) * g(2, 2) - g(0, 2) * g(2, 0)) / J
    gc[..., 2, 1] = (-g(0, 0) * g(2, 1) + g(0, 1) * g(2, 0)) / J
    gc[..., 0, 2] = (g(0, 1) * g(1, 2) - g(1, 1) * g(0, 2)) / J
    gc[..., 1, 2] = (-g(0, 0) * g(1, 2) + g(0, 2) * g(1, 0)) / J
    gc[..., 2, 2] = (g(0, 0) * g(1, 1) - g(0, 1) * g(1, 0)) / J
    gc[np.abs(gc) <= small] = 0.0
    return gc, J


# d%bcond codes of faces without a neighbour (the C-ABI's DSEM_BC_*)
BC_CODES = {"interface": 0, "walladiab": 1, "wallisoth": 2, "inflow": 3, "outflow": 4}


class Box:
    """Box of nex*ney*nez hex8 elements with per-element orders, periodic in
    every direction that `bc` does not name.  bc maps an axis ("x", "y", "z")
    to the conditions of its low and high faces, e.g. {"y": ("walladiab",
    "wallisoth")}; those faces become boundary mortars (id(2) = 0)."""

    def __init__(self, nex, ney, nez, orders, length=2 * np.pi, rot=None, ldx=None, bc=None, warp=0.0):
        self.nex, self.ney, self.nez = nex, ney, nez
        self.length = float(length)
        self.warp = float(warp)
        self.bc = {}
        for ax, pair in (bc or {}).items():
            codes = tuple(BC_CODES.get(x, -1) if isinstance(x, str) else int(x) for x in pair)
            if len(codes) != 2 or not all(1 <= x <= 4 for x in codes):
                raise ValueError("bc: two boundary conditions (low, high) per axis")
            self.bc["xyz".index(ax)] = codes
        ne = nex * ney * nez
        self.nel = ne
        self.orders = np.broadcast_to(np.asarray(orders, dtype=np.int32), (ne,)).copy()
        self.G = self.orders + 1
        self.ldx = int(ldx or (self.G.max() + 1))
        rot = np.zeros(ne, dtype=int) if rot is None else np.asarray(rot, dtype=int)
        lx = ly = lz = float(length)
        self.corner = np.empty((ne, 8, 3))
        self.node = np.empty((ne, 8), dtype=np.int64)
        nid = lambda ix, iy, iz: iy + (ney + 1) * (ix + (nex + 1) * iz)
        for iz in range(nez):
            for ix in range(nex):
                for iy in range(ney):
                    e = iy + ney * (ix + nex * iz)
                    R = _ROT[rot[e] % 24]
                    for k in range(8):
                        v = 2 * CORNER_XYZ[k] - 1
                        src = (R.T @ v + 1) // 2
                        kk = int(np.where((CORNER_XYZ == src).all(axis=1))[0][0])
                        a, b, c = ix + CORNER_XYZ[kk][0], iy + CORNER_XYZ[kk][1], iz + CORNER_XYZ[kk][2]
                        self.node[e, k] = nid(a, b, c)
                        self.corner[e, k] = (a * (lx / nex), b * (ly / ney), c * (lz / nez))
        self._connect()
        self._geometry()

    # ------------------------------------------------------------ topology
    def _connect(self):
        ne = self.nel
        faces = {}
        mort = []  # [id1, id2, f1, f2, orient, sign]
        self.emort = -np.ones((ne, 6), dtype=int)
        self.boundary = np.zeros((ne, 6), dtype=bool)
        self.mside = np.zeros((ne, 6), dtype=int)
        for e in range(ne):
            for f in range(6):
                fn = [int(self.node[e, k]) for k in FACE_MAP[f]]
                key = tuple(sorted(fn))
                if key not in faces:
                    faces[key] = len(mort)
                    mort.append([e, -1, f + 1, 0, 0, 1])
                    self.emort[e, f] = faces[key]
                    self.mside[e, f] = 1
                    self.boundary[e, f] = True
                else:
                    j = faces[key]
                    M = mort[j]
                    mn = [int(self.node[M[0], k]) for k in FACE_MAP[M[2] - 1]]
                    M[1], M[3], M[4] = e, f + 1, faces_match(mn, fn)
                    M[5] = -SIGN_LOW[M[2]] * SIGN_LOW[f + 1]
                    self.emort[e, f] = j
                    self.mside[e, f] = 2
                    self.boundary[M[0], M[2] - 1] = False
        self._mort_pre = [list(m) for m in mort]
        removed = set()
        C = self.corner

        def pair(idm, fm, ids, fs, master_is_m):
            keep = self.emort[idm, fm - 1] if master_is_m else self.emort[ids, fs - 1]
            drop = self.emort[ids, fs - 1] if master_is_m else self.emort[idm, fm - 1]
            mel, sel = (idm, ids) if master_is_m else (ids, idm)
            mf, sf = (fm, fs) if master_is_m else (fs, fm)
            M = mort[keep]
            M[0], M[2], M[1], M[3] = mel, mf, sel, sf
            removed.add(drop)
            self.emort[sel, sf - 1] = keep
            self.mside[sel, sf - 1] = 2
            self.boundary[idm, fm - 1] = False
            self.boundary[ids, fs - 1] = False

        def first_match(fm, fs, cm, cs, comps):
            idx = {}
            for ids in range(ne):
                if self.boundary[ids, fs - 1]:
                    idx.setdefault(tuple(C[ids, cs, comps]), ids)
            for idm in range(ne):
                if self.boundary[idm, fm - 1]:
                    ids = idx.get(tuple(C[idm, cm, comps]))
                    if ids is not None and self.boundary[ids, fs - 1]:
                        yield idm, ids

        if 2 not in self.bc:
            for idm, ids in list(first_match(3, 5, 0, 4, [0, 1])):
                pair(idm, 3, ids, 5, True)
        if 1 not in self.bc:
            for idm, ids in list(first_match(1, 2, 0, 3, [0, 2])):
                pair(idm, 1, ids, 2, True)
        if 0 not in self.bc:
            for idm, ids in list(first_match(6, 4, 0, 1, [2, 1])):
                pair(idm, 6, ids, 4, False)
        keep = [j for j in range(len(mort)) if j not in removed]
        newid = {j: i for i, j in enumerate(keep)}
        self.mort_raw = [mort[j] for j in keep]
        self.mort_geo_src = keep
        self.emort = np.vectorize(lambda j: newid.get(j, -1))(self.emort)
        # faces left without a neighbour lie on a non-periodic side: d%bcond
        self.bcond = np.zeros((ne, 6), dtype=np.int32)
        tol = 1e-9 * self.length
        for m in self.mort_raw:
            if m[1] >= 0:
                continue
            ctr = C[m[0], list(FACE_MAP[m[2] - 1])].mean(axis=0)
            code = 0
            for a, (lo, hi) in self.bc.items():
                if abs(ctr[a]) < tol:
                    code = lo
                elif abs(ctr[a] - self.length) < tol:
                    code = hi
            if code == 0:
                raise ValueError("unpaired boundary faces remain")
            self.bcond[m[0], m[2] - 1] = code

    # ------------------------------------------------------------ geometry
    def _map(self, c, X, Y, Z):
        """Physical points and d(x)/d(X) of the element map at computational points: the
        hex8 map (hex8, grad_hex8) followed, when warp != 0, by the smooth periodic
        deformation x_i -> x_i + warp * length * sin(k x_j) sin(k x_l) (k = 2 pi / length,
        (i, j, l) cyclic), which curves every element and keeps the box periodic."""
        x = hex8(c, X, Y, Z)
        g = grad_hex8(c, X, Y, Z)
        if self.warp == 0.0:
            return x, g
        a, k = self.warp * self.length, 2.0 * np.pi / self.length
        s_, c_ = np.sin(k * x), np.cos(k * x)
        W = np.zeros(x.shape + (3,))
        xw = x.copy()
        for i in range(3):
            j, l = (i + 1) % 3, (i + 2) % 3
            xw[..., i] += a * s_[..., j] * s_[..., l]
            W[..., i, i] = 1.0
            W[..., i, j] = a * k * c_[..., j] * s_[..., l]
            W[..., i, l] = a * k * s_[..., j] * c_[..., l]
        return xw, np.einsum("...ij,...jk->...ik", W, g)

    def _geometry(self):
        ne, ldx = self.nel, self.ldx
        L3 = ldx ** 3
        self.jacob = np.zeros((ne, L3))
        self.gmetg = np.zeros((ne, L3, 9))
        self.gmet = np.zeros((ne, L3, 9))
        self.xg = np.zeros((ne, L3, 3))
        for G in np.unique(self.G):
            G = int(G)
            L = G + 1
            ids = np.where(self.G == G)[0]
            c = self.corner[ids][:, None, None, None, :, :]
            cxg, cx = gauss_points(G), lobatto_points(L)
            # Gauss points: index (l, m, n) -> arrays broadcast as [l][m][n]
            X = cxg[None, None, :]
            Y = cxg[None, :, None]
            Z = cxg[:, None, None]
            xg, gx = self._map(c, X, Y, Z)
            gc, J = invert_metric(gx)
            q = (np.arange(G)[None, None, :] + ldx * (np.arange(G)[None, :, None] + ldx * np.arange(G)[:, None, None]))
            q = np.broadcast_to(q, (G, G, G)).ravel()
            self.jacob[np.ix_(ids, q)] = (1.0 / J).reshape(len(ids), -1)
            # gmetg(i,j) at i + 3j
            self.gmetg[ids[:, None], q[None, :], :] = np.swapaxes(gc, -1, -2).reshape(len(ids), G ** 3, 9)
            self.xg[ids[:, None], q[None, :], :] = xg.reshape(len(ids), G ** 3, 3)
            for d in range(3):
                ext = [G, G, G]
                ext[d] = L
                pts = [cxg, cxg, cxg]
                pts[d] = cx
                X = pts[0][None, None, :]
                Y = pts[1][None, :, None]
                Z = pts[2][:, None, None]
                gx = self._map(c, X, Y, Z)[1]
                gc, J = invert_metric(gx)
                row = J[..., None] * gc[..., d, :]  # [ids, l, m, n, 3]
                nn = np.arange(ext[0])[None, None, :]
                mm = np.arange(ext[1])[None, :, None]
                ll = np.arange(ext[2])[:, None, None]
                q = np.broadcast_to(nn + ldx * (mm + ldx * ll), (ext[2], ext[1], ext[0])).ravel()
                for b in range(3):
                    self.gmet[ids[:, None], q[None, :], d + 3 * b] = row[..., b].reshape(len(ids), -1)
        # mortars (their geometry is evaluated per group of equal master face and size, the
        # face normals per face and order, with the same elementwise arithmetic per point)
        nm = len(self.mort_raw)
        self.nmort = nm
        self.mortar = np.zeros((nm, 17), dtype=np.int32)
        self.n_hat = np.zeros((nm, ldx, ldx, 3))
        self.norm = np.zeros((nm, ldx, ldx))
        jobs = {}  # (master face, lenmortar) -> ([mortar], [master element])
        normals = {}
        for j, (id1, id2, f1, f2, orient, sign) in enumerate(self.mort_raw):
            if id2 < 0:  # boundary mortar: master face only, nsign = 1 (set_mortars.f90:361)
                Gm = int(self.G[id1])
                self.mortar[j] = [id1 + 1, 0, f1, 0, Gm, Gm, Gm, Gm, Gm, Gm, 0, 1, 1, 1, 1, 1, 1]
                job = jobs.setdefault((f1, Gm, Gm), ([], []))
                job[0].append(j)
                job[1].append(id1)
                continue
            Gm, Gs = int(self.G[id1]), int(self.G[id2])
            j1, j2 = (1, 0) if orient >= 4 else (0, 1)
            lens = [[Gm, Gs], [Gm, Gs]]
            lm = [max(lens[0][0], lens[j1][1]), max(lens[1][0], lens[j2][1])]
            conf = [lm[0] == lens[0][0], lm[1] == lens[1][0], lm[0] == lens[j1][1], lm[1] == lens[j2][1]]
            for f in (f1, f2):
                if f not in normals:
                    normals[f] = self._face_normals(f)
            n1, n2 = normals[f1][id1], normals[f2][id2]
            nsign = 1 if float(np.dot(n1, n2)) >= 0 else -1
            self.mortar[j] = [id1 + 1, id2 + 1, f1, f2, Gm, Gm, Gs, Gs, lm[0], lm[1], orient, sign, nsign] + \
                [int(x) for x in conf]
            job = jobs.setdefault((f1, lm[0], lm[1]), ([], []))
            job[0].append(j)
            job[1].append(id1)
        for (f1, l0, l1), (js, es) in jobs.items():
            self._mortar_geometry(np.array(js), np.array(es), f1, [l0, l1])

    def _face_normals(self, face):
        """Unit normal J grad X_d of face `face` of every element [nel][3], at the face's
        first Gauss point pair (the Lobatto end along d); its sign against the other side's
        gives nsign."""
        out = np.zeros((self.nel, 3))
        d = FACE_DIR[face]
        for G in np.unique(self.G):
            G = int(G)
            ids = np.where(self.G == G)[0]
            cx = lobatto_points(G + 1)
            cxg = gauss_points(G)
            pt = [cxg[0], cxg[0], cxg[0]]
            pt[d] = cx[-1] if face in (2, 4, 5) else cx[0]
            gx = self._map(self.corner[ids], np.float64(pt[0]), np.float64(pt[1]), np.float64(pt[2]))[1]
            gc, J = invert_metric(gx)
            g = J[:, None] * gc[:, d, :]
            out[ids] = g / np.sqrt(g[:, 0] * g[:, 0] + g[:, 1] * g[:, 1] + g[:, 2] * g[:, 2])[:, None]
        return out

    def _mortar_geometry(self, js, es, face, lm):
        """n_hat and norm of the mortars js, whose master faces `face` of elements es have
        lenmortar lm."""
        d = FACE_DIR[face]
        c1, c2 = gauss_points(lm[0]), gauss_points(lm[1])
        A = c1[None, :]
        B = c2[:, None]
        end = END_VALS[face - 1]
        if d == 1:
            X, Y, Z = A, np.full_like(A * B, end), B
        elif d == 2:
            X, Y, Z = A, B, np.full_like(A * B, end)
        else:
            X, Y, Z = np.full_like(A * B, end), A, B
        gx = self._map(self.corner[es][:, None, None, :, :], X + 0 * B, Y + 0 * A, Z + 0 * A)[1]
        gc, J = invert_metric(gx)
        r = gc[..., d, :]
        sqr = np.sqrt(r[..., 0] * r[..., 0] + r[..., 1] * r[..., 1] + r[..., 2] * r[..., 2])
        self.n_hat[js, :lm[1], :lm[0], :] = r / sqr[..., None]
        self.norm[js, :lm[1], :lm[0]] = J * sqr

    # ------------------------------------------------------------ exports
    def desc(self):
        return dict(ngrid=self.nel, nmort=self.nmort, ldx=self.ldx,
                    ncg=np.ascontiguousarray(np.repeat(self.G, 3).astype(np.int32)),
                    jacob=np.ascontiguousarray(self.jacob.ravel()),
                    gmetg=np.ascontiguousarray(self.gmetg.ravel()),
                    gmet=np.ascontiguousarray(self.gmet.ravel()),
                    mortar=np.ascontiguousarray(self.mortar.ravel()),
                    n_hat=np.ascontiguousarray(self.n_hat.ravel()),
                    norm=np.ascontiguousarray(self.norm.ravel()),
                    bcond=np.ascontiguousarray(self.bcond.ravel()) if self.bc else None)

    def boundary_mortars(self):
        """Indices of the boundary mortars (id(2) = 0)."""
        return np.where(self.mortar[:, 1] == 0)[0]

    def mortar_xyz(self):
        """Physical coordinates of the mortar Gauss points [nmort][ldx][ldx][3]
        (j, i order as mrtr%xg; zero in the padding)."""
        out = np.zeros((self.nmort, self.ldx, self.ldx, 3))
        for j in range(self.nmort):
            e, face, G = int(self.mortar[j, 0]) - 1, int(self.mortar[j, 2]), int(self.mortar[j, 8])
            d = FACE_DIR[face]
            c1 = gauss_points(G)
            A, B = c1[None, :], c1[:, None]
            end = np.full_like(A * B, END_VALS[face - 1])
            X, Y, Z = {1: (A + 0 * B, end, B + 0 * A), 2: (A + 0 * B, B + 0 * A, end), 0: (end, A + 0 * B, B + 0 * A)}[d]
            out[j, :G, :G] = self._map(self.corner[e], X, Y, Z)[0]
        return out

    def gauss_xyz(self):
        """Physical Gauss-point coordinates [nel][ldx^3][3] (zero in the padding)."""
        return self.xg

    def qshape(self):
        return (self.nel, NV, self.ldx, self.ldx, self.ldx)


def taylor_green(box, gamma=1.4, twall=100.0, v0=1.0):
    """J*Q of the Taylor-Green initial condition (exactsol,
    caseFiles/tgv/BackstepProblem-stoch.f90:1533-1570), stored as Q/jacob."""
    x, y, z = (box.xg[..., k] for k in range(3))
    uu = v0 * np.sin(x) * np.cos(y) * np.cos(z)
    vv = -v0 * np.cos(x) * np.sin(y) * np.cos(z)
    ww = np.zeros_like(uu)
    rho = np.ones_like(uu)
    p = twall * 1.0 / gamma + (np.cos(2.0 * x) + np.cos(2.0 * y)) * (np.cos(2.0 * z) + 2.0) / 16.0
    q = [rho, rho * uu, rho * vv, rho * ww, p / (gamma - 1.0) + 0.5 * rho * (uu * uu + vv * vv + ww * ww)]
    jq = np.zeros((box.nel, NV, box.ldx ** 3))
    mask = box.jacob != 0
    for v in range(NV):
        jq[:, v][mask] = q[v][mask] / box.jacob[mask]
    return jq.reshape(box.qshape())


def _modes_separable(box, K, kmax, amp, a, phase):
    """sum_m amp_m a_m cos(k_m.x + phase_m) at every point of box.xg, evaluated
    as three 1-D sums per element when each element's Gauss points form a
    tensor grid (x from n, y from m, z from l, to 1e-12); None otherwise."""
    ldx = box.ldx
    xg = box.xg.reshape(box.nel, ldx, ldx, ldx, 3)
    nk = 2 * kmax + 1
    C = np.zeros((nk, nk, nk, 3), dtype=complex)
    idx = K.astype(int) + kmax
    np.add.at(C, (idx[:, 0], idx[:, 1], idx[:, 2]), (amp * np.exp(1j * phase))[:, None] * a)
    ks = np.arange(-kmax, kmax + 1, dtype=float)
    u = np.zeros((box.nel, ldx, ldx, ldx, 3))
    for G in np.unique(box.G):
        G = int(G)
        ids = np.where(box.G == G)[0]
        x = xg[ids][:, :G, :G, :G]  # [e][l][m][n][c]
        xe, ye, ze = x[:, 0, 0, :, 0], x[:, 0, :, 0, 1], x[:, :, 0, 0, 2]
        tol = 1e-12 * max(1.0, float(np.abs(x).max()))
        if not (np.abs(x[..., 0] - xe[:, None, None, :]).max() <= tol and
                np.abs(x[..., 1] - ye[:, None, :, None]).max() <= tol and
                np.abs(x[..., 2] - ze[:, :, None, None]).max() <= tol):
            return None
        Ex = np.exp(1j * xe[:, :, None] * ks)  # [e][n][kx]
        Ey = np.exp(1j * ye[:, :, None] * ks)
        Ez = np.exp(1j * ze[:, :, None] * ks)
        t = np.einsum("abcv,elc->eablv", C, Ez, optimize=True)
        t = np.einsum("eablv,emb->eamlv", t, Ey, optimize=True)
        t = np.einsum("eamlv,ena->elmnv", t, Ex, optimize=True)
        u[ids, :G, :G, :G] = t.real
    return u.reshape(-1, 3)


def _isotropic_velocity(box, seed, k0):
    """Seeded divergence-free random-phase velocity with E(k) ~ k^4 exp(-2 (k/k0)^2)
    at every point of box.xg ([nel * ldx^3][3]) and its rms per component."""
    rng = np.random.default_rng(seed)
    kmax = int(3 * k0)
    ks = np.arange(-kmax, kmax + 1)
    KX, KY, KZ = np.meshgrid(ks, ks, ks, indexing="ij")
    K = np.stack([KX, KY, KZ], -1).reshape(-1, 3).astype(float)
    kk = np.linalg.norm(K, axis=1)
    sel = (kk > 0) & (kk <= kmax)
    K, kk = K[sel], kk[sel]
    amp = np.sqrt(kk ** 4 * np.exp(-2.0 * (kk / k0) ** 2) / (4 * np.pi * kk ** 2))
    a = rng.standard_normal((len(K), 3))
    a -= (np.sum(a * K, axis=1) / kk ** 2)[:, None] * K  # divergence free
    a /= np.linalg.norm(a, axis=1)[:, None] + 1e-300
    phase = rng.uniform(0, 2 * np.pi, len(K))
    u = _modes_separable(box, K, kmax, amp, a, phase)
    if u is None:  # rotated elements: direct sum over points and modes
        X = box.xg.reshape(-1, 3)
        u = np.zeros((X.shape[0], 3))
        for i in range(0, len(K), 256):
            arg = X @ K[i:i + 256].T + phase[i:i + 256]
            u += np.cos(arg) @ (amp[i:i + 256, None] * a[i:i + 256])
    mask = (box.jacob != 0).reshape(-1)
    urms = math.sqrt(np.mean(np.sum(u[mask] ** 2, axis=1)) / 3.0)
    return u, urms


def _jq(box, rho, u, p, gamma):
    jq = np.zeros((box.nel, NV, box.ldx ** 3))
    m2 = box.jacob != 0
    q = [rho, rho * u[..., 0], rho * u[..., 1], rho * u[..., 2],
         p / (gamma - 1.0) + 0.5 * rho * np.sum(u * u, axis=-1)]
    for v in range(NV):
        jq[:, v][m2] = q[v][m2] / box.jacob[m2]
    return jq.reshape(box.qshape())


def random_isotropic(box, seed, k0=4.0, mach_t=0.3, gamma=1.4, twall=100.0):
    """Seeded divergence-free random-phase velocity with E(k) ~ k^4 exp(-2 (k/k0)^2),
    scaled to turbulent Mach number mach_t (u_rms = M_t c0 / sqrt(3)), uniform
    density and pressure; evaluated at the Gauss points, returned as J*Q."""
    u, urms = _isotropic_velocity(box, seed, k0)
    p0 = twall / gamma
    c0 = math.sqrt(gamma * p0 / 1.0)
    u = (u * ((mach_t * c0 / math.sqrt(3.0)) / urms)).reshape(box.nel, -1, 3)
    return _jq(box, np.ones(u.shape[:2]), u, np.full(u.shape[:2], p0), gamma)


def perturbed_taylor_green(box, seed, amp=0.05, k0=2.0, gamma=1.4, twall=100.0):
    """Taylor-Green initial condition plus a seeded isotropic velocity of rms
    amp (same density and pressure).  The perturbation removes the exact
    symmetries of the Taylor-Green field (w = 0, zero normal velocity on
    symmetry planes) at which the Roe flux's branches meet, so derivatives of
    the flow with respect to its initial state are smooth."""
    x, y, z = (box.xg[..., k] for k in range(3))
    ut, urms = _isotropic_velocity(box, seed, k0)
    ut = ut.reshape(box.nel, -1, 3) * (amp / urms)
    u = np.stack([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z), np.zeros_like(x)], -1) + ut
    p = twall * 1.0 / gamma + (np.cos(2.0 * x) + np.cos(2.0 * y)) * (np.cos(2.0 * z) + 2.0) / 16.0
    return _jq(box, np.ones_like(x), u, p, gamma)


def boundary_state(box, rho, vel, p, gamma=1.4, seed=None, amp=0.0):
    """External states of the boundary mortars ([nmort][5][ldx][ldx], the
    mrtr%Q(:,:,:,2) that initc / inflow_time_bc fill): a uniform stream of
    density rho, velocity vel and pressure p, optionally with a seeded relative
    perturbation of size amp on every conserved variable."""
    out = np.zeros((box.nmort, NV, box.ldx, box.ldx))
    u, v, w = (float(x) for x in vel)
    q = np.array([rho, rho * u, rho * v, rho * w, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)])
    rng = np.random.default_rng(seed) if seed is not None else None
    for j in box.boundary_mortars():
        G = int(box.mortar[j, 8])
        blk = np.broadcast_to(q[:, None, None], (NV, G, G)).copy()
        if rng is not None and amp:
            blk *= 1.0 + amp * rng.standard_normal(blk.shape)
        out[j, :, :G, :G] = blk
    return out


def dtcalc(box, JQ, gamma=1.4):
    """Inviscid time-step limit (Parabolic3D/NS/NS/stac3m/dtcalc.f90:9-58),
    minimum over elements, before the CFL factor."""
    dt = np.inf
    ldx = box.ldx
    gm = box.gmet.reshape(box.nel, ldx, ldx, ldx, 3, 3)  # [e][l][m][n][j][i]
    for G in np.unique(box.G):
        G = int(G)
        ids = np.where(box.G == G)[0]
        cx = lobatto_points(G + 1)
        dc = cx[1:G + 1] - cx[:G]
        q = JQ[ids][:, :, :G, :G, :G]  # [e][v][l][m][n]
        jac = box.jacob[ids].reshape(len(ids), ldx, ldx, ldx)[:, :G, :G, :G]
        q1 = q[:, 0]
        u0 = np.abs(q[:, 1] / q1)
        v0 = np.abs(q[:, 2] / q1)
        w0 = np.abs(q[:, 3] / q1)
        p = (gamma - 1.0) * (q[:, 4] - 0.5 * q1 * (u0 * u0 + v0 * v0 + w0 * w0))
        a = np.sqrt(gamma * p / q1)
        g = gm[ids][:, :G, :G, :G]
        lam = []
        for d in range(3):
            r = (u0 + a) * g[..., 0, d] + (v0 + a) * g[..., 1, d] + (w0 + a) * g[..., 2, d]
            lam.append(np.abs(r * jac))
        dti = (lam[0] / dc[None, None, None, :] + lam[1] / dc[None, None, :, None] + lam[2] / dc[None, :, None, None]
               + 1.0e-14)
        dt = min(dt, float(np.min(1.0 / dti)))
    return dt
