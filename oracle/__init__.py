"""ctypes binding of the CPU oracle -- test infrastructure only.

The oracle (``oracle.cpp``) restates the reference's forward-solve path on the
CPU in FP64.  Only the test-suite, ``__graft_entry__.smoke()`` and the CPU
baseline legs of ``bench.py`` may use it, and only as the checker or the timed
CPU baseline; the emfem_b200 package never imports it.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class OrcMesh(C.Structure):
    _fields_ = [("nv", C.c_int), ("nt", C.c_int), ("ne", C.c_int),
                ("pts", C.c_void_p), ("tets", C.c_void_p), ("attr", C.c_void_p),
                ("edges", C.c_void_p), ("tet2edge", C.c_void_p), ("nbr", C.c_void_p),
                ("non", C.c_void_p), ("ebdr", C.c_void_p)]


class OrcModel(C.Structure):
    _fields_ = [("aniso_form", C.c_int), ("nrho", C.c_int), ("ncol", C.c_int),
                ("rho", C.c_void_p)]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        _LIB.orc_sparsity.restype = C.c_long
        _LIB.orc_solve.restype = C.c_int
    return _LIB


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Mesh:
    """Holds contiguous arrays alive for the C struct."""

    def __init__(self, m):
        self.pts = np.ascontiguousarray(m.points, dtype=np.float64)
        self.tets = np.ascontiguousarray(m.tets, dtype=np.int32)
        self.attr = np.ascontiguousarray(m.attr, dtype=np.int32)
        self.edges = np.ascontiguousarray(m.edges, dtype=np.int32)
        self.tet2edge = np.ascontiguousarray(m.tet2edge, dtype=np.int32)
        self.nbr = np.ascontiguousarray(m.neighbors, dtype=np.int32)
        self.non = np.ascontiguousarray(m.tet_non, dtype=np.int32)
        self.ebdr = np.ascontiguousarray(m.edge_bdr, dtype=np.uint8)
        self.nv, self.nt, self.ne = self.pts.shape[0], self.tets.shape[0], self.edges.shape[0]
        self.s = OrcMesh(self.nv, self.nt, self.ne, _p(self.pts), _p(self.tets), _p(self.attr),
                         _p(self.edges), _p(self.tet2edge), _p(self.nbr), _p(self.non),
                         _p(self.ebdr))

    @property
    def ref(self):
        return C.byref(self.s)


class Model:
    def __init__(self, md):
        self.rho = np.ascontiguousarray(md.rho, dtype=np.float64)
        self.s = OrcModel(int(md.aniso_form), self.rho.shape[0], self.rho.shape[1], _p(self.rho))

    @property
    def ref(self):
        return C.byref(self.s)


def num_threads(n=0):
    return lib().orc_num_threads(C.c_int(n))


def cell_sigma(model, idx):
    out = np.zeros(9)
    lib().orc_cell_sigma(Model(model).ref, C.c_int(idx), _p(out))
    return out.reshape(3, 3)


def fe_coefs(mesh: Mesh, t):
    abcd = np.zeros(16)
    ev = np.zeros(12, dtype=np.int32)
    lib().orc_fe_coefs(mesh.ref, C.c_int(t), _p(abcd), _p(ev))
    return abcd.reshape(4, 4), ev.reshape(6, 2)


def cell_quadrature(mesh: Mesh, t):
    q = np.zeros(12)
    w = np.zeros(4)
    lib().orc_cell_quadrature(mesh.ref, C.c_int(t), _p(q), _p(w))
    return q.reshape(4, 3), w


def face_quadrature(mesh: Mesh, t, f):
    q = np.zeros(9)
    w = np.zeros(3)
    lib().orc_face_quadrature(mesh.ref, C.c_int(t), C.c_int(f), _p(q), _p(w))
    return q.reshape(3, 3), w


def element_matrices(mesh: Mesh, model, t, omega):
    c = np.zeros(36)
    m = np.zeros(36)
    lib().orc_element_matrices(mesh.ref, Model(model).ref, C.c_int(t), C.c_double(omega), _p(c), _p(m))
    return c.reshape(6, 6), m.reshape(6, 6)


def tet_geometry(mesh: Mesh, t):
    v = C.c_double()
    d = C.c_double()
    fd = np.zeros(4)
    lib().orc_tet_geometry(mesh.ref, C.c_int(t), C.byref(v), C.byref(d), _p(fd))
    return v.value, d.value, fd


def sparsity(mesh: Mesh):
    rp = np.zeros(mesh.ne + 1, dtype=np.int32)
    cap = 40 * mesh.ne
    ci = np.zeros(cap, dtype=np.int32)
    nnz = lib().orc_sparsity(mesh.ref, _p(rp), _p(ci), C.c_long(cap))
    if nnz < 0:
        cap = -nnz
        ci = np.zeros(cap, dtype=np.int32)
        nnz = lib().orc_sparsity(mesh.ref, _p(rp), _p(ci), C.c_long(cap))
    return rp, ci[:nnz].copy()


def assemble(mesh: Mesh, model, freq, rp, ci):
    nnz = int(rp[-1])
    Cv = np.zeros(nnz)
    Mv = np.zeros(nnz)
    bdr = np.zeros(mesh.nt, dtype=np.uint8)
    lib().orc_assemble(mesh.ref, Model(model).ref, C.c_double(freq), _p(rp), _p(ci), _p(Cv), _p(Mv), _p(bdr))
    return Cv, Mv, bdr


def matshell_mult(rp, ci, Cv, Mv, x):
    n = rp.shape[0] - 1
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(2 * n)
    lib().orc_matshell_mult(C.c_int(n), _p(rp), _p(ci), _p(Cv), _p(Mv), _p(x), _p(y))
    return y


def plane_wave(ztop, lsig, freq, z):
    ztop = np.ascontiguousarray(ztop, dtype=np.float64)
    lsig = np.ascontiguousarray(lsig, dtype=np.float64)
    z = np.ascontiguousarray(np.atleast_1d(z), dtype=np.float64)
    out = np.zeros(z.size * 8)
    lib().orc_plane_wave(C.c_int(ztop.size), _p(ztop), _p(lsig), C.c_double(freq), C.c_int(z.size),
                         _p(z), _p(out))
    o = out.reshape(z.size, 4, 2)
    return o[..., 0] + 1j * o[..., 1]


def find_cell(mesh: Mesh, pts):
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(pts.shape[0], dtype=np.int32)
    lib().orc_find_cell(mesh.ref, C.c_int(pts.shape[0]), _p(pts), _p(out))
    return out


MAXL = 64


def background_model(mesh: Mesh, model):
    corners = np.zeros(12)
    nlay = np.zeros(4, dtype=np.int32)
    zt = np.zeros(4 * MAXL)
    ls = np.zeros(4 * MAXL)
    rc = lib().orc_background_model(mesh.ref, Model(model).ref, C.c_int(MAXL), _p(corners), _p(nlay),
                                    _p(zt), _p(ls))
    if rc != 0:
        raise RuntimeError("background model failed (%d)" % rc)
    return corners, nlay, zt, ls


def rhs_mt(mesh: Mesh, model, freq, mode, bg, bdr):
    corners, nlay, zt, ls = bg
    sr = np.zeros(mesh.ne)
    si = np.zeros(mesh.ne)
    lib().orc_rhs_mt(mesh.ref, Model(model).ref, C.c_double(freq), C.c_int(mode), _p(corners), _p(nlay),
                     _p(zt), _p(ls), C.c_int(MAXL), _p(bdr), _p(sr), _p(si))
    return sr, si


def rhs_csem(mesh: Mesh, freq, tx, n_div=20):
    tx = np.ascontiguousarray(tx, dtype=np.float64)
    sr = np.zeros(mesh.ne)
    si = np.zeros(mesh.ne)
    rc = lib().orc_rhs_csem(mesh.ref, C.c_double(freq), _p(tx), C.c_int(n_div), _p(sr), _p(si))
    if rc != 0:
        raise RuntimeError("Transmitter is not found in mesh.")
    return sr, si


def rhs_dual(mesh: Mesh, rx):
    rx = np.ascontiguousarray(rx, dtype=np.float64)
    sr = np.zeros(mesh.ne)
    si = np.zeros(mesh.ne)
    rc = lib().orc_rhs_dual(mesh.ref, C.c_int(rx.shape[0]), _p(rx), _p(sr), _p(si))
    if rc != 0:
        raise RuntimeError("Receiver %d is not found in mesh." % (-rc - 1))
    return sr, si


def solve(mesh: Mesh, rp, ci, Cv, Mv, sr, si, rtol=1e-8, maxit=100):
    n = rp.shape[0] - 1
    er = np.zeros(n)
    ei = np.zeros(n)
    stats = np.zeros(4)
    its = lib().orc_solve(mesh.ref, C.c_int(n), _p(rp), _p(ci), _p(Cv), _p(Mv),
                          _p(np.ascontiguousarray(sr)), _p(np.ascontiguousarray(si)),
                          C.c_double(rtol), C.c_int(maxit), _p(er), _p(ei), _p(stats))
    return er, ei, its, stats


def estimate(mesh: Mesh, model, freq, sols):
    """Per-solution per-tet indicators before the primal*dual combination."""
    nsol = len(sols)
    res = [np.ascontiguousarray(s[0], dtype=np.float64) for s in sols]
    ims = [np.ascontiguousarray(s[1], dtype=np.float64) for s in sols]
    pre = (C.c_void_p * nsol)(*[r.ctypes.data for r in res])
    pim = (C.c_void_p * nsol)(*[i.ctypes.data for i in ims])
    eta = np.zeros(nsol * mesh.nt)
    lib().orc_estimate(mesh.ref, Model(model).ref, C.c_double(freq), C.c_int(nsol), pre, pim, _p(eta))
    return eta.reshape(nsol, mesh.nt)


def refine_fixed_fraction(err, fraction, flag=None):
    err = np.ascontiguousarray(err, dtype=np.float64)
    flag = np.zeros(err.size, dtype=np.uint8) if flag is None else flag
    lib().orc_refine_fixed_fraction(C.c_int(err.size), _p(err), C.c_double(fraction), _p(flag))
    return flag


def refine_fixed_number(err, fraction, flag=None):
    err = np.ascontiguousarray(err, dtype=np.float64)
    flag = np.zeros(err.size, dtype=np.uint8) if flag is None else flag
    lib().orc_refine_fixed_number(C.c_int(err.size), _p(err), C.c_double(fraction), _p(flag))
    return flag


def interpolate_fields(mesh: Mesh, t, p, freq, er, ei):
    p = np.ascontiguousarray(p, dtype=np.float64)
    out = np.zeros(12)
    lib().orc_interpolate_fields(mesh.ref, C.c_int(t), _p(p), C.c_double(freq),
                                 _p(np.ascontiguousarray(er)), _p(np.ascontiguousarray(ei)), _p(out))
    o = out.reshape(6, 2)
    z = o[:, 0] + 1j * o[:, 1]
    return z[:3], z[3:]


def response_mt(freq, fields, otype):
    """calculate_response_mt for one receiver; fields (4, 3) complex (E_xy, H_xy,
    E_yx, H_yx).  Returns the complex value or None for a refused type."""
    f = np.ascontiguousarray(np.asarray(fields, dtype=np.complex128).reshape(4, 3)).view(np.float64)
    out = np.zeros(2)
    lib().orc_response_mt.restype = C.c_int
    rc = lib().orc_response_mt(C.c_double(freq), _p(f), C.c_int(otype), _p(out))
    return None if rc != 0 else out[0] + 1j * out[1]


def response_csem(fields, otype):
    """calculate_response_csem for one receiver; fields (2, 3) complex (E, H)."""
    f = np.ascontiguousarray(np.asarray(fields, dtype=np.complex128).reshape(2, 3)).view(np.float64)
    out = np.zeros(2)
    lib().orc_response_csem.restype = C.c_int
    rc = lib().orc_response_csem(_p(f), C.c_int(otype), _p(out))
    return None if rc != 0 else out[0] + 1j * out[1]
