"""Synthetic tetrahedral meshes, models and surveys shaped like EMFEM inputs.

TetGen is not available to this package, so meshes come from a graded tensor
grid whose hexahedra are split into six Kuhn tetrahedra.  The generator emits
exactly the arrays the reference keeps in its ``tetgenio`` (``em_mesh.h:81-96``):

* ``pointlist``            (V, 3) float64
* ``tetrahedronlist``      (T, 4) int32, positively oriented (det J > 0, the
  orientation ``TetAccessor::contains_point`` assumes, ``em_mesh.h:208-230``)
* ``tetrahedronattributelist`` (T,) int32 region ids
* ``edgelist``             (E, 2) int32 with endpoints sorted ascending
  (``Mesh::build_edge_info``, ``em_mesh.cc:448-461``)
* ``tet2edgelist``         (T, 6) int32
* ``neighborlist``         (T, 4) int32, face f is opposite vertex f, -1 on
  the boundary (TetGen convention used by ``em_fwd.cc:1059`` and
  ``em_fe.cc:254``)
* ``tet_non``              (T, 4) int32, the neighbour's local index of the
  shared face (``Mesh::build_neighbor_info``, ``em_mesh.cc:463-481``)
* ``edge_bdr_marker``      (E,) uint8, edges of boundary faces
  (``Mesh::build_boundary_info``, ``em_mesh.cc:483-502``)

Coordinates follow the reference: z grows downwards (depth), the air is at
negative z.  Sizes are in metres.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np

# Kuhn split of a unit cube; corner c = ix + 2*iy + 4*iz.
_KUHN = np.array([[0, 1, 3, 7], [0, 1, 5, 7], [0, 2, 3, 7],
                  [0, 2, 6, 7], [0, 4, 5, 7], [0, 4, 6, 7]], dtype=np.int64)
# Local edges of a tet as vertex pairs.
LOCAL_EDGES = np.array([[0, 1], [0, 2], [0, 3], [1, 2], [1, 3], [2, 3]],
                       dtype=np.int64)

ISOTROPIC, VERTICAL, TRIAXIAL, ARBITRARY = 0, 1, 2, 3
XY_POLAR, YX_POLAR = -1, -2


@dataclasses.dataclass
class TetMesh:
    points: np.ndarray        # (V,3) f64
    tets: np.ndarray          # (T,4) i32
    attr: np.ndarray          # (T,)  i32
    edges: np.ndarray         # (E,2) i32
    tet2edge: np.ndarray      # (T,6) i32
    neighbors: np.ndarray     # (T,4) i32
    tet_non: np.ndarray       # (T,4) i32
    edge_bdr: np.ndarray      # (E,)  u8
    vertex_bdr: np.ndarray    # (V,)  u8

    @property
    def n_vertices(self) -> int:
        return int(self.points.shape[0])

    @property
    def n_tets(self) -> int:
        return int(self.tets.shape[0])

    @property
    def n_edges(self) -> int:
        return int(self.edges.shape[0])


@dataclasses.dataclass
class Model:
    aniso_form: int
    rho: np.ndarray           # (n_rho, ncol) f64 as read by read_rho (em_io.cc:9-86)


@dataclasses.dataclass
class Survey:
    freqs: np.ndarray         # (nf,)
    tx: np.ndarray            # (ntx, 7): x y z azimuth dip current length (TX_SIZE)
    rx: np.ndarray            # (nrx, 3)
    kind: str                 # "mt" or "csem"


@dataclasses.dataclass
class Problem:
    name: str
    mesh: TetMesh
    model: Model
    survey: Survey


# ----------------------------------------------------------------------------
# grid axes
# ----------------------------------------------------------------------------
def graded_axis(lo, hi, core_lo, core_hi, h, growth, extra=()):
    """Uniform spacing ``h`` on [core_lo, core_hi], geometric growth outside."""
    n = max(1, int(round((core_hi - core_lo) / h)))
    core = np.linspace(core_lo, core_hi, n + 1)
    left, right = [], []
    x, d = core_lo, h
    while x > lo:
        d *= growth
        x -= d
        if x - lo < 0.5 * d:
            x = lo
        left.append(x)
    x, d = core_hi, h
    while x < hi:
        d *= growth
        x += d
        if hi - x < 0.5 * d:
            x = hi
        right.append(x)
    nodes = np.concatenate([np.array(left[::-1]), core, np.array(right)])
    # interface planes become nodes; grid nodes closer than 0.4 of the local
    # spacing to an interface are dropped so that no sliver layer appears
    extra = np.unique(np.asarray(extra, dtype=np.float64))
    keep = np.ones(nodes.size, dtype=bool)
    for e in extra:
        k = int(np.searchsorted(nodes, e))
        lo_i, hi_i = max(k - 1, 0), min(k, nodes.size - 1)
        hloc = max(nodes[min(k + 1, nodes.size - 1)] - nodes[max(k - 2, 0)], 1e-9) / 3.0
        for j in (lo_i, hi_i):
            if abs(nodes[j] - e) < 0.4 * hloc and nodes[j] not in (lo, hi):
                keep[j] = False
    nodes = np.unique(np.concatenate([nodes[keep], extra[(extra > lo) & (extra < hi)]]))
    return nodes


# ----------------------------------------------------------------------------
# topology (what TetGen's -nnef switches return)
# ----------------------------------------------------------------------------
def build_topology(points: np.ndarray, tets: np.ndarray, attr: np.ndarray) -> TetMesh:
    points = np.ascontiguousarray(points, dtype=np.float64)
    tets = np.ascontiguousarray(tets, dtype=np.int64)
    nt = tets.shape[0]
    nv = points.shape[0]
    # edges
    a = tets[:, LOCAL_EDGES[:, 0]]
    b = tets[:, LOCAL_EDGES[:, 1]]
    lo = np.minimum(a, b)
    hi = np.maximum(a, b)
    key = (lo * nv + hi).ravel()
    ukey, inv = np.unique(key, return_inverse=True)
    edges = np.stack([ukey // nv, ukey % nv], axis=1).astype(np.int32)
    tet2edge = inv.reshape(nt, 6).astype(np.int32)
    # faces: face f opposite vertex f
    fv = np.stack([tets[:, [1, 2, 3]], tets[:, [2, 3, 0]],
                   tets[:, [3, 0, 1]], tets[:, [0, 1, 2]]], axis=1)  # (T,4,3)
    fs = np.sort(fv, axis=2).reshape(-1, 3)
    fkey = (fs[:, 0] * nv + fs[:, 1]) * nv + fs[:, 2]
    order = np.argsort(fkey, kind="stable")
    sk = fkey[order]
    same = np.nonzero(sk[1:] == sk[:-1])[0]
    neighbors = np.full(nt * 4, -1, dtype=np.int64)
    tet_non = np.full(nt * 4, -1, dtype=np.int64)
    f1 = order[same]
    f2 = order[same + 1]
    neighbors[f1] = f2 // 4
    neighbors[f2] = f1 // 4
    tet_non[f1] = f2 % 4
    tet_non[f2] = f1 % 4
    neighbors = neighbors.reshape(nt, 4)
    tet_non = tet_non.reshape(nt, 4)
    # boundary markers: the three edges/vertices of every boundary face
    edge_bdr = np.zeros(edges.shape[0], dtype=np.uint8)
    vertex_bdr = np.zeros(nv, dtype=np.uint8)
    bt, bf = np.nonzero(neighbors < 0)
    if bt.size:
        # local edges that do not touch vertex f
        face_edges = np.array([[3, 4, 5], [1, 2, 5], [0, 2, 4], [0, 1, 3]])
        edge_bdr[tet2edge[bt[:, None], face_edges[bf]].ravel()] = 1
        face_verts = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]])
        vertex_bdr[tets[bt[:, None], face_verts[bf]].ravel()] = 1
    return TetMesh(points=points, tets=tets.astype(np.int32),
                   attr=np.ascontiguousarray(attr, dtype=np.int32),
                   edges=edges, tet2edge=tet2edge,
                   neighbors=neighbors.astype(np.int32), tet_non=tet_non.astype(np.int32),
                   edge_bdr=edge_bdr, vertex_bdr=vertex_bdr)


def tet_dets(points, tets):
    p = points[tets]
    a = p[:, 1] - p[:, 0]
    b = p[:, 2] - p[:, 0]
    c = p[:, 3] - p[:, 0]
    return np.einsum("ij,ij->i", a, np.cross(b, c))


def hex_grid_tets(xs, ys, zs):
    """Kuhn split of the tensor grid; returns points, tets (positively oriented)
    and the hexahedron index of every tet."""
    nx, ny, nz = len(xs), len(ys), len(zs)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    # vertex id = i + nx*(j + ny*k)
    pts = np.stack([X.transpose(2, 1, 0).ravel(), Y.transpose(2, 1, 0).ravel(),
                    Z.transpose(2, 1, 0).ravel()], axis=1)
    i, j, k = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), np.arange(nz - 1), indexing="ij")
    i = i.transpose(2, 1, 0).ravel()
    j = j.transpose(2, 1, 0).ravel()
    k = k.transpose(2, 1, 0).ravel()
    base = i + nx * (j + ny * k)
    corner = np.array([0, 1, nx, nx + 1, nx * ny, nx * ny + 1, nx * ny + nx, nx * ny + nx + 1])
    hexv = base[:, None] + corner[None, :]                    # (H,8)
    tets = hexv[:, _KUHN].reshape(-1, 4)                      # (6H,4)
    hexid = np.repeat(np.arange(base.size), 6)
    return pts, tets, hexid


def orient_positive(points, tets):
    d = tet_dets(points, tets)
    neg = d < 0
    tets = tets.copy()
    tets[neg, 2], tets[neg, 3] = tets[neg, 3].copy(), tets[neg, 2].copy()
    return tets


# ----------------------------------------------------------------------------
# problem builders
# ----------------------------------------------------------------------------
def _scaled_grid(target_tets, make_axes):
    """Pick the core spacing scale s so that the grid has ~target_tets tets."""
    lo, hi = 0.2, 20.0
    best = None
    for _ in range(40):
        s = math.sqrt(lo * hi)
        xs, ys, zs = make_axes(s)
        nt = 6 * (len(xs) - 1) * (len(ys) - 1) * (len(zs) - 1)
        if best is None or abs(nt - target_tets) < abs(best[0] - target_tets):
            best = (nt, xs, ys, zs)
        if nt > target_tets:
            lo = s
        else:
            hi = s
        if abs(nt - target_tets) < 0.03 * target_tets:
            break
    return best[1], best[2], best[3]


def mt_halfspace_block(target_tets=50_000, rho_half=100.0, rho_block=1.0,
                       rho_air=1e8, freqs=(0.1, 1.0, 10.0), with_block=True,
                       topo_height=0.0, topo_sigma=5e3, n_bodies=0, seed=0,
                       name="mt"):
    """MT model: 200 km box, 100 km of air over a halfspace, optional 2x2x1 km
    conductive block whose top is at 1 km, optional Gaussian hill and random
    anisotropic bodies (full SPD tensors, ``Arbitrary`` form)."""
    rng = np.random.default_rng(seed)
    L = 100e3

    def axes(s):
        hxy = 500.0 * s
        hz = 250.0 * s
        xs = graded_axis(-L, L, -4e3, 4e3, hxy, 1.5, extra=(-1e3, 1e3))
        ys = graded_axis(-L, L, -4e3, 4e3, hxy, 1.5, extra=(-1e3, 1e3))
        zs = graded_axis(-L, L, -1e3, 3e3, hz, 1.6, extra=(0.0, 1e3, 2e3))
        return xs, ys, zs

    xs, ys, zs = _scaled_grid(target_tets, axes)
    pts, tets, _ = hex_grid_tets(xs, ys, zs)
    ref = pts.copy()
    if topo_height != 0.0:
        r2 = pts[:, 0] ** 2 + pts[:, 1] ** 2
        zs_surf = -topo_height * np.exp(-r2 / (2 * topo_sigma ** 2))
        w = np.where(pts[:, 2] <= 0, 1 - pts[:, 2] / -L, 1 - pts[:, 2] / L)
        w = np.clip(w, 0.0, 1.0)
        pts = pts.copy()
        pts[:, 2] = pts[:, 2] + zs_surf * w
    tets = orient_positive(pts, tets)
    cen = ref[tets].mean(axis=1)
    attr = np.where(cen[:, 2] < 0, 0, 1).astype(np.int32)
    rho_rows = [[rho_air], [rho_half]]
    aniso = ISOTROPIC
    if with_block:
        inb = ((np.abs(cen[:, 0]) < 1e3) & (np.abs(cen[:, 1]) < 1e3) &
               (cen[:, 2] > 1e3) & (cen[:, 2] < 2e3))
        attr[inb] = len(rho_rows)
        rho_rows.append([rho_block])
    if n_bodies > 0:
        aniso = ARBITRARY
        rows = [[r[0], r[0], r[0], 0.0, 0.0, 0.0] for r in rho_rows]
        for _ in range(n_bodies):
            c = rng.uniform([-5e3, -5e3, 0.5e3], [5e3, 5e3, 3e3])
            size = rng.uniform([1e3, 1e3, 0.5e3], [4e3, 4e3, 2e3])
            rho = 10 ** rng.uniform(0, 3)
            aa, bb = rng.uniform(1, 5, size=2)
            ang = rng.uniform(-90, 90, size=3)
            inb = np.all(np.abs(cen - c) < size / 2, axis=1) & (cen[:, 2] > 0)
            attr[inb] = len(rows)
            rows.append([rho, rho * aa, rho * bb, ang[0], ang[1], ang[2]])
        rho_rows = rows
    mesh = build_topology(pts, tets, attr)
    g = np.arange(-10e3, 10e3 + 1, 1e3)
    rx = np.array([[x, y, 0.0] for y in g for x in g])
    if topo_height != 0.0:
        r2 = rx[:, 0] ** 2 + rx[:, 1] ** 2
        rx[:, 2] = -topo_height * np.exp(-r2 / (2 * topo_sigma ** 2))
        # receivers on the mapped surface: evaluate at the mesh surface by
        # linear interpolation is not needed for synthetic runs; nudge them
        # just below the true surface so that they lie in the earth.
        rx[:, 2] += 1.0
    survey = Survey(freqs=np.asarray(freqs, dtype=np.float64),
                    tx=np.zeros((0, 7)), rx=rx, kind="mt")
    model = Model(aniso_form=aniso, rho=np.asarray(rho_rows, dtype=np.float64))
    return Problem(name=name, mesh=mesh, model=model, survey=survey)


def marine_csem(target_tets=80_000, freqs=(0.25, 0.75, 1.25), n_reservoirs=0,
                n_tx=1, seed=1, name="csem"):
    """Marine CSEM: 1 km of 0.3 ohm-m sea over a VTI sediment (rho_h=1,
    rho_v=2), a 100 ohm-m reservoir 4x4 km x 100 m at 1 km below the seafloor,
    an x-directed HED 50 m above the seafloor and 41 in-line seafloor receivers."""
    rng = np.random.default_rng(seed)
    L = 50e3
    zsf = 1000.0

    def axes(s):
        h = 500.0 * s
        hz = 250.0 * s
        xs = graded_axis(-L, L, -10.5e3, 10.5e3, h, 1.5, extra=(-2e3, 2e3))
        ys = graded_axis(-L, L, -3e3, 3e3, h, 1.5, extra=(-2e3, 2e3))
        zs = graded_axis(-L, L, 0.0, 2.5e3, hz, 1.6,
                         extra=(0.0, zsf, zsf - 50.0, 2e3, 2.1e3))
        return xs, ys, zs

    xs, ys, zs = _scaled_grid(target_tets, axes)
    pts, tets, _ = hex_grid_tets(xs, ys, zs)
    tets = orient_positive(pts, tets)
    cen = pts[tets].mean(axis=1)
    attr = np.full(tets.shape[0], 2, dtype=np.int32)      # sediment
    attr[cen[:, 2] < zsf] = 1                             # sea
    attr[cen[:, 2] < 0] = 0                               # air
    rows = [[1e8, 1e8], [0.3, 0.3], [1.0, 2.0]]
    inr = ((np.abs(cen[:, 0]) < 2e3) & (np.abs(cen[:, 1]) < 2e3) &
           (cen[:, 2] > 2e3) & (cen[:, 2] < 2.1e3))
    attr[inr] = len(rows)
    rows.append([100.0, 100.0])
    for _ in range(n_reservoirs):
        c = rng.uniform([-8e3, -2e3, 1.5e3], [8e3, 2e3, 2.5e3])
        th = rng.uniform(50, 300)
        w = rng.uniform(2e3, 5e3, size=2)
        rho = rng.uniform(10, 200)
        inr = ((np.abs(cen[:, 0] - c[0]) < w[0] / 2) & (np.abs(cen[:, 1] - c[1]) < w[1] / 2) &
               (np.abs(cen[:, 2] - c[2]) < max(th, 250.0) / 2) & (cen[:, 2] > zsf))
        attr[inr] = len(rows)
        rows.append([rho, rho])
    mesh = build_topology(pts, tets, attr)
    rx = np.array([[x, 0.0, zsf] for x in np.arange(-10e3, 10e3 + 1, 500.0)])
    txs = []
    for i in range(n_tx):
        x0 = (i - (n_tx - 1) / 2.0) * 1e3
        txs.append([x0 + 1.0, 1.0, zsf - 50.0 + 1.0, 0.0, 0.0, 1.0, 0.0])
    survey = Survey(freqs=np.asarray(freqs, dtype=np.float64), tx=np.array(txs),
                    rx=rx, kind="csem")
    model = Model(aniso_form=VERTICAL, rho=np.asarray(rows, dtype=np.float64))
    return Problem(name=name, mesh=mesh, model=model, survey=survey)


def config(idx: int, scale: float = 1.0) -> Problem:
    """Seeded synthetic stand-ins for the five benchmark configurations.
    ``scale`` multiplies the tet count (tests use small scales)."""
    if idx == 0:
        return mt_halfspace_block(int(50_000 * scale), freqs=(0.1, 1.0, 10.0), seed=0,
                                  name="cfg0-mt-small")
    if idx == 1:
        return marine_csem(int(80_000 * scale), seed=1, name="cfg1-csem-aniso")
    if idx == 2:
        return mt_halfspace_block(int(1_500_000 * scale), with_block=False,
                                  topo_height=1e3, topo_sigma=5e3, n_bodies=10,
                                  freqs=tuple(np.logspace(-3, 2, 8)), seed=2,
                                  name="cfg2-mt-topo-batched")
    if idx == 3:
        return marine_csem(int(800_000 * scale), n_reservoirs=3, n_tx=16,
                           freqs=tuple(np.logspace(-1, 1, 24)), seed=3,
                           name="cfg3-csem-sweep")
    if idx == 4:
        return mt_halfspace_block(int(4_000_000 * scale), with_block=True,
                                  topo_height=1e3, n_bodies=10,
                                  freqs=tuple(np.logspace(-3, 2, 64)), seed=4,
                                  name="cfg4-full")
    raise ValueError(idx)


# ----------------------------------------------------------------------------
# host point location and layered background columns (host mesh work that the
# reference does with its KD-tree and TetAccessor, src/em_mesh.cc:504-566 and
# src/em_fwd.cc:74-159)
# ----------------------------------------------------------------------------
def _orient3d(a, b, c, d):
    ad, bd, cd = a - d, b - d, c - d
    return (ad[0] * (bd[1] * cd[2] - bd[2] * cd[1]) + bd[0] * (cd[1] * ad[2] - cd[2] * ad[1]) +
            cd[0] * (ad[1] * bd[2] - ad[2] * bd[1]))


def contains_point(mesh: TetMesh, t: int, p) -> bool:
    """TetAccessor::contains_point (src/em_mesh.h:208-230)."""
    v = mesh.points[mesh.tets[t]]
    p = np.asarray(p, dtype=np.float64)
    d = (_orient3d(v[0], v[1], v[3], p), _orient3d(v[1], v[2], v[3], p),
         _orient3d(v[1], v[0], v[2], p), _orient3d(v[0], v[3], v[2], p))
    return all(x >= 0.0 for x in d)


class PointLocator:
    """find_cell_around_point: breadth-first walk over face neighbours starting
    at the last tet that holds the vertex closest to the point (ties: lowest
    vertex index)."""

    def __init__(self, mesh: TetMesh):
        self.mesh = mesh
        v2t = np.full(mesh.n_vertices, -1, dtype=np.int64)
        np.maximum.at(v2t, mesh.tets.ravel().astype(np.int64), np.repeat(np.arange(mesh.n_tets), 4))
        self.v2t = v2t

    def closest_vertex(self, p):
        d = np.einsum("ij,ij->i", self.mesh.points - p, self.mesh.points - p)
        return int(np.argmin(d))

    def locate(self, p) -> int:
        p = np.asarray(p, dtype=np.float64)
        start = int(self.v2t[self.closest_vertex(p)])
        seen = {start}
        queue = [start]
        head = 0
        nbr = self.mesh.neighbors
        while head < len(queue):
            t = queue[head]
            head += 1
            if contains_point(self.mesh, t, p):
                return t
            for n in nbr[t]:
                n = int(n)
                if n >= 0 and n not in seen:
                    seen.add(n)
                    queue.append(n)
        return -1

    def locate_all(self, pts):
        return np.array([self.locate(p) for p in np.asarray(pts, dtype=np.float64).reshape(-1, 3)],
                        dtype=np.int32)


def sigma_mean(model: Model, attr: int) -> float:
    """Mean of the diagonal of the conductivity tensor (the trace is rotation
    invariant, so every anisotropy form reduces to the mean of 1/rho)."""
    r = model.rho[attr]
    f = model.aniso_form
    if f == ISOTROPIC:
        return 1.0 / r[0]
    if f == VERTICAL:
        return (2.0 / r[0] + 1.0 / r[1]) / 3.0
    return (1.0 / r[0] + 1.0 / r[1] + 1.0 / r[2]) / 3.0


def background_model(mesh: TetMesh, model: Model, maxl: int = 64):
    """update_background_model (src/em_fwd.cc:135-159): layered columns under
    the four top corners.  Returns (corners (4,3), nlay (4,), ztop (4,maxl),
    lsig (4,maxl))."""
    loc = PointLocator(mesh)
    pts = mesh.points
    tl = pts[loc.closest_vertex(np.array([-1e15, -1e15, -1e15]))]
    br = pts[loc.closest_vertex(np.array([1e15, 1e15, 1e15]))]
    corners = np.array([[tl[0], tl[1], tl[2]], [br[0], tl[1], tl[2]], [br[0], br[1], tl[2]],
                        [tl[0], br[1], tl[2]]])
    nlay = np.zeros(4, dtype=np.int32)
    ztop = np.zeros((4, maxl))
    lsig = np.zeros((4, maxl))
    for c in range(4):
        fp = corners[c].copy()
        z, sg = [], []
        while fp[2] < br[2]:
            v = loc.closest_vertex(fp)
            t = loc.locate(fp + np.array([0.0, 0.0, 1e-6]))
            if t < 0:
                raise RuntimeError("layered column left the mesh")
            z.append(fp[2])
            sg.append(sigma_mean(model, int(mesh.attr[t])))
            nxt = None
            for i in range(4):
                vi = int(mesh.tets[t, i])
                cv = pts[vi]
                if vi != v and abs(cv[0] - corners[c][0]) < 1e-6 and abs(cv[1] - corners[c][1]) < 1e-6:
                    nxt = cv.copy()
                    break
            if nxt is None:
                raise RuntimeError("no vertical edge below a corner vertex")
            fp = nxt
        zt, ls = [z[0]], [sg[0]]
        for i in range(len(z) - 1):
            if sg[i] != sg[i + 1]:
                zt.append(z[i + 1])
                ls.append(sg[i + 1])
        nlay[c] = len(zt)
        ztop[c, :len(zt)] = zt
        lsig[c, :len(ls)] = ls
    return corners, nlay, ztop, lsig
