"""Python mirror of the reference's forward-solve entry points over the C ABI.

Method names follow ``src/em_fwd.h`` and ``src/em_la.h`` of the reference
(create_linear_system, assemble_matrix, create_pc, solve_linear_system,
estimate_error, ...); errors surface as :class:`EMGError` carrying the C-ABI
status (``EMG_ERR_USER`` = the reference's ``EM_ERR_USER`` = -1).
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

EMG_OK = 0
EMG_ERR_USER = -1
EMG_ERR_ARG = -2
EMG_ERR_STATE = -3
EMG_ERR_CUDA = -4
EMG_ERR_NOMEM = -5
EMG_DIVERGED_ITS = -6
EMG_DIVERGED_NANORINF = -7
EMG_ERR_OPTION = -8
EMG_STOPPED_AT_FLOOR = 1         # block column at the FP64 rounding floor of its residual

XY_POLAR, YX_POLAR = -1, -2      # src/em_defs.h:39
SOL_CSEM, SOL_DUAL = 0, 1


class EMGError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("emfem_b200 error %d: %s" % (code, msg))
        self.code = code


class SolveInfo(C.Structure):
    _fields_ = [("outer_its", C.c_int), ("inner_its", C.c_int), ("reason", C.c_int),
                ("true_rel_res", C.c_double), ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BlockOpts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("max_it", C.c_int), ("use_guess", C.c_int),
                ("inner_fp32", C.c_int), ("restart", C.c_int)]


class WarmOpts(C.Structure):
    _fields_ = [("steps", C.c_int), ("batch", C.c_long), ("lr", C.c_float), ("seed", C.c_uint)]


def library_path() -> str:
    return os.path.join(_HERE, "libemfem_b200.so")


_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_SIGS = {
    "emg_last_error": ([], C.c_char_p),
    "emg_version": ([], C.c_char_p),
    "emg_create_context": ([C.POINTER(_P), _I], _I),
    "emg_destroy_context": ([_P], _I),
    "emg_process_options": ([_P, C.c_char_p], _I),
    "emg_get_option": ([_P, C.c_char_p, C.POINTER(_D)], _I),
    "emg_set_mesh": ([_P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _P, _P], _I),
    "emg_set_model": ([_P, _I, _I, _I, _P], _I),
    "emg_set_frequencies": ([_P, _I, _P], _I),
    "emg_create_linear_system": ([_P, _I], _I),
    "emg_destroy_linear_system": ([_P], _I),
    "emg_get_sparsity": ([_P, C.POINTER(C.c_long), _P, _P], _I),
    "emg_assemble_matrix": ([_P, _I], _I),
    "emg_get_matrices": ([_P, _P, _P, _P], _I),
    "emg_create_pc": ([_P], _I),
    "emg_destroy_pc": ([_P], _I),
    "emg_matshell_mult_a": ([_P, _P, _P], _I),
    "emg_pc_apply_b": ([_P, _P, _P], _I),
    "emg_solve_linear_system": ([_P, _I, _P, _P, _I, _D, C.POINTER(SolveInfo)], _I),
    "emg_get_solution": ([_P, _I, _P, _P], _I),
    "emg_set_solution": ([_P, _I, _P, _P], _I),
    "emg_set_background": ([_P, _P, _P, _P, _P, _I], _I),
    "emg_assemble_rhs_mt": ([_P, _I, _I, _P, _P], _I),
    "emg_assemble_rhs_csem": ([_P, _I, _P, _P, _P, _P], _I),
    "emg_assemble_rhs_dual": ([_P, _I, _P, _P, _P, _P], _I),
    "emg_estimate_error": ([_P, _I, _I, _P, _P], _I),
    "emg_refine_fixed_fraction": ([_I, _P, _D, _P], _I),
    "emg_refine_fixed_number": ([_I, _P, _D, _P], _I),
    "emg_interpolate_fields": ([_P, _I, _I, _I, _P, _P, _P], _I),
    "emg_solve_block": ([_P, _I, _P, _P, _P, C.POINTER(BlockOpts), _P], _I),
    "emg_solve_block_dev": ([_P, _I, _P, _P, _P, C.POINTER(BlockOpts), _P], _I),
    "emg_spmv_complex_dev": ([_P, _I, _P, _P, _P, _I], _I),
    "emg_spmm_layout_dev": ([_P, _I, _I, _I, _I, _P, _P, _P, _P], _I),
    "emg_orient3d_sign": ([_P, _P, _P, _P, C.POINTER(_I)], _I),
    "emg_last_kernel_ms": ([_P, C.c_char_p, C.POINTER(_D)], _I),
    "emg_stream_synchronize": ([_P], _I),
    "emg_launch_count": ([C.POINTER(C.c_long)], _I),
    "emg_profile_enable": ([_I], _I),
    "emg_profile_get": ([C.c_char_p, C.POINTER(C.c_long), C.POINTER(_D), C.POINTER(_D)], _I),
    "emg_spmm_layouts": ([C.c_char_p, C.c_long], _I),
    "emg_divergence_correct_dev": ([_P, _I, _P, _P, _P, _I, C.POINTER(C.c_long)], _I),
    "emg_assemble_rhs_mt_block": ([_P, _I, _P, _P, _P], _I),
    "emg_assemble_rhs_mt_block_dev": ([_P, _I, _P, _P, _P], _I),
    "emg_estimate_error_noalloc": ([_P, _I, _I, _P, _P], _I),
    "emg_calculate_response_mt": ([_D, _I, _P, _I, _P, _P, _P], _I),
    "emg_calculate_response_csem": ([_I, _P, _I, _P, _P, _P], _I),
    "emg_point_index_create": ([_I, _P, _I, _P, _P], _P),
    "emg_point_index_find": ([_P, _I, _P, _P], _I),
    "emg_point_index_destroy": ([_P], None),
    "emg_find_cell_around_point": ([_P, _I, _P, _P], _I),
    "emg_interpolate_fields_host": ([_P, _I, _I, _P, _P, _P, _P, _P], _I),
    "emg_save_vtk": ([_P, C.c_char_p, _I, _P, _P], _I),
    "emg_interpolate_fields_block_dev": ([_P, _I, _P, _P, _I, _P, _P, _P], _I),
    "emg_last_initial_residuals": ([_P, _I, _P], _I),
    "emg_last_residual_floors": ([_P, _I, _P], _I),
    "emg_amg_levels": ([_P, _I, _I, _D, _I, C.POINTER(_I), _P], _I),
    "emg_warm_start_train": ([_P, _I, _P, _P, _P, _P, C.POINTER(WarmOpts), C.POINTER(_D)], _I),
    "emg_warm_start_predict": ([_P, _I, _P, _P, _P, _P, _I, _P, _P, _P, _I, _P], _I),
    "emg_warm_start_params": ([_P, _P, _P, C.POINTER(_I)], _I),
    "emg_warm_start_gradients": ([_P, _I, _P, _P, _P, _P, C.c_long, _I, _P, C.POINTER(_D)], _I),
    "emg_warm_start_reset": ([_P], _I),
    "emg_warm_start_losses": ([_P, C.POINTER(_D), C.POINTER(_D)], _I),
    "emg_assemble_rhs_csem_block_dev": ([_P, _I, _P, _P, _P], _I),
    "emg_assemble_rhs_dual_block_dev": ([_P, _I, _I, _P, _P], _I),
    "emg_survey_read_emd": ([C.c_char_p], _P),
    "emg_survey_sizes": ([_P, _P, _P, _P, _P], _I),
    "emg_survey_get": ([_P, _P, _P, _P, _P, _P, _P, _P, _P, _P], _I),
    "emg_survey_write_rsp": ([_P, C.c_char_p, _P], _I),
    "emg_survey_destroy": ([_P], None),
}


def lib():
    """Loads libemfem_b200.so; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        path = library_path()
        if not os.path.exists(path):
            raise EMGError(EMG_ERR_STATE, "%s is not built (run __graft_entry__.build())" % path)
        L = C.CDLL(path)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _LIB = L
    return _LIB


def _check(rc):
    if rc != EMG_OK:
        raise EMGError(rc, lib().emg_last_error().decode())
    return rc


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def launch_count() -> int:
    n = C.c_long()
    _check(lib().emg_launch_count(C.byref(n)))
    return n.value


def orient3d_sign(a, b, c, d) -> int:
    """exact sign of det[a-d; b-d; c-d] (the point-location predicate)"""
    pts = [_f64(np.asarray(v, dtype=np.float64).reshape(3)) for v in (a, b, c, d)]
    out = _I()
    _check(lib().emg_orient3d_sign(_ptr(pts[0]), _ptr(pts[1]), _ptr(pts[2]), _ptr(pts[3]), C.byref(out)))
    return out.value


def spmm_layouts() -> str:
    """The SpMM lane layouts the autotuner chose so far (text)."""
    buf = C.create_string_buffer(4096)
    _check(lib().emg_spmm_layouts(buf, 4096))
    return buf.value.decode()


def profile_enable(on=True):
    _check(lib().emg_profile_enable(int(on)))


def profile_get(bin_name):
    """(launches, device ms, algorithmic bytes) accumulated in a profiler bin."""
    n, ms, by = C.c_long(), C.c_double(), C.c_double()
    _check(lib().emg_profile_get(bin_name.encode(), C.byref(n), C.byref(ms), C.byref(by)))
    return n.value, ms.value, by.value


def refine_fixed_fraction(err, fraction, flag=None):
    """refine_fixed_fraction (src/em_fwd.cc:1182-1215); ORs into flag."""
    err = _f64(err)
    flag = np.zeros(err.size, dtype=np.uint8) if flag is None else flag
    _check(lib().emg_refine_fixed_fraction(err.size, _ptr(err), float(fraction), _ptr(flag)))
    return flag


def refine_fixed_number(err, fraction, flag=None):
    """refine_fixed_number (src/em_fwd.cc:1217-1240); ORs into flag."""
    err = _f64(err)
    flag = np.zeros(err.size, dtype=np.uint8) if flag is None else flag
    _check(lib().emg_refine_fixed_number(err.size, _ptr(err), float(fraction), _ptr(flag)))
    return flag


class PointIndex:
    """find_cell_around_point (src/em_mesh.cc:527-566) over a mesh's
    pointlist / tetrahedronlist / neighborlist, reusable across queries."""

    def __init__(self, mesh):
        self._arrs = (_f64(mesh.points), _i32(mesh.tets), _i32(mesh.neighbors))
        self._h = lib().emg_point_index_create(mesh.n_vertices, _ptr(self._arrs[0]), mesh.n_tets,
                                               _ptr(self._arrs[1]), _ptr(self._arrs[2]))
        if not self._h:
            raise EMGError(EMG_ERR_ARG, lib().emg_last_error().decode())

    def find(self, pts):
        p = _f64(np.asarray(pts).reshape(-1, 3))
        out = np.zeros(p.shape[0], dtype=np.int32)
        _check(lib().emg_point_index_find(self._h, p.shape[0], _ptr(p), _ptr(out)))
        return out

    def close(self):
        if self._h:
            lib().emg_point_index_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Survey:
    """A survey file in the reference's .emd layout (read_emd,
    src/em_io.cc:202-287): freqs, tx (n, 7), rx (n, 3) and the observations
    (otype, fidx, tidx, ridx, obs, obserr; AP types as log amplitude and
    phase in radians).  write_rsp writes save_rsp's layout."""

    def __init__(self, path):
        self._h = lib().emg_survey_read_emd(os.fsencode(path))
        if not self._h:
            raise EMGError(EMG_ERR_USER, lib().emg_last_error().decode())
        n = [C.c_int() for _ in range(4)]
        _check(lib().emg_survey_sizes(self._h, *[C.byref(x) for x in n]))
        nf, ntx, nrx, nobs = [x.value for x in n]
        self.freqs = np.zeros(nf)
        self.tx = np.zeros((ntx, 7))
        self.rx = np.zeros((nrx, 3))
        self.otype, self.fidx, self.tidx, self.ridx = (np.zeros(nobs, dtype=np.int32) for _ in range(4))
        self.obs = np.zeros(nobs, dtype=np.complex128)
        self.obserr = np.zeros(nobs, dtype=np.complex128)
        _check(lib().emg_survey_get(self._h, _ptr(self.freqs), _ptr(self.tx), _ptr(self.rx), _ptr(self.otype),
                                    _ptr(self.fidx), _ptr(self.tidx), _ptr(self.ridx),
                                    _ptr(self.obs.view(np.float64)), _ptr(self.obserr.view(np.float64))))

    def write_rsp(self, path, rsp):
        r = np.ascontiguousarray(np.asarray(rsp, dtype=np.complex128).reshape(-1))
        if r.size != self.obs.size:
            raise EMGError(EMG_ERR_ARG, "one response per observation")
        _check(lib().emg_survey_write_rsp(self._h, os.fsencode(path), _ptr(r.view(np.float64))))

    def close(self):
        if self._h:
            lib().emg_survey_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# observation types (ObsType, src/em_defs.h:50-73)
F_EX_RI, F_EY_RI, F_EZ_RI, F_HX_RI, F_HY_RI, F_HZ_RI = 111, 121, 131, 141, 151, 161
F_EX_AP, F_EY_AP, F_EZ_AP, F_HX_AP, F_HY_AP, F_HZ_AP = 112, 122, 132, 142, 152, 162
R_XY_AP, R_YX_AP = 212, 222
Z_XX_RI, Z_XY_RI, Z_YX_RI, Z_YY_RI, T_ZX_RI, T_ZY_RI = 311, 321, 331, 341, 351, 361


def calculate_response_mt(freq, fields, otype, ridx):
    """calculate_response_mt (src/em_fwd.cc:747-800).  fields: (nrx, 4, 3)
    complex -- E_xy, H_xy, E_yx, H_yx per receiver; returns one complex value
    per observation (R_XY_AP / R_YX_AP: log(rho_a) + 1j * phase in radians,
    the reference's AP pair)."""
    f = np.ascontiguousarray(np.asarray(fields, dtype=np.complex128).reshape(-1, 4, 3))
    ot, ri = _i32(otype), _i32(ridx)
    out = np.zeros(ot.size, dtype=np.complex128)
    _check(lib().emg_calculate_response_mt(float(freq), f.shape[0], _ptr(f.view(np.float64)), ot.size,
                                           _ptr(ot), _ptr(ri), _ptr(out.view(np.float64))))
    return out


def calculate_response_csem(fields, otype, ridx):
    """calculate_response_csem (src/em_fwd.cc:802-871).  fields: (nrx, 2, 3)
    complex -- E, H per receiver."""
    f = np.ascontiguousarray(np.asarray(fields, dtype=np.complex128).reshape(-1, 2, 3))
    ot, ri = _i32(otype), _i32(ridx)
    out = np.zeros(ot.size, dtype=np.complex128)
    _check(lib().emg_calculate_response_csem(f.shape[0], _ptr(f.view(np.float64)), ot.size, _ptr(ot), _ptr(ri),
                                             _ptr(out.view(np.float64))))
    return out


class EMContext:
    """Device-resident counterpart of the reference's EMContext (src/em_ctx.h:15-64).

    ``device=-1`` gives a host-only context (options and host helpers only)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().emg_create_context(C.byref(h), int(device)))
        self._h = h
        self.device = device
        self.ne = self.nt = self.nv = 0
        self.freqs = np.zeros(0)

    def close(self):
        if getattr(self, "_h", None):
            lib().emg_destroy_context(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- configuration ---------------------------------------------------------------
    def process_options(self, text: str):
        _check(lib().emg_process_options(self._h, text.encode()))

    def get_option(self, key: str) -> float:
        v = C.c_double()
        _check(lib().emg_get_option(self._h, key.encode(), C.byref(v)))
        return v.value

    def set_mesh(self, m):
        self._mesh = m
        arrs = dict(pts=_f64(m.points), tets=_i32(m.tets), attr=_i32(m.attr), edges=_i32(m.edges),
                    t2e=_i32(m.tet2edge), nbr=_i32(m.neighbors), non=_i32(m.tet_non),
                    ebdr=np.ascontiguousarray(m.edge_bdr, dtype=np.uint8))
        _check(lib().emg_set_mesh(self._h, m.n_vertices, _ptr(arrs["pts"]), m.n_tets, _ptr(arrs["tets"]),
                                  _ptr(arrs["attr"]), m.n_edges, _ptr(arrs["edges"]), _ptr(arrs["t2e"]),
                                  _ptr(arrs["nbr"]), _ptr(arrs["non"]), _ptr(arrs["ebdr"])))
        self.nv, self.nt, self.ne = m.n_vertices, m.n_tets, m.n_edges

    def set_model(self, model):
        rho = _f64(model.rho)
        _check(lib().emg_set_model(self._h, int(model.aniso_form), rho.shape[0], rho.shape[1], _ptr(rho)))

    def set_frequencies(self, freqs):
        self.freqs = _f64(freqs)
        _check(lib().emg_set_frequencies(self._h, self.freqs.size, _ptr(self.freqs)))

    # -- em_fwd.h / em_la.h ---------------------------------------------------------------
    def create_linear_system(self, tidx: int):
        _check(lib().emg_create_linear_system(self._h, int(tidx)))

    def destroy_linear_system(self):
        _check(lib().emg_destroy_linear_system(self._h))

    def make_sparsity_patterns(self):
        nnz = C.c_long()
        _check(lib().emg_get_sparsity(self._h, C.byref(nnz), None, None))
        rp = np.zeros(self.ne + 1, dtype=np.int32)
        ci = np.zeros(nnz.value, dtype=np.int32)
        _check(lib().emg_get_sparsity(self._h, C.byref(nnz), _ptr(rp), _ptr(ci)))
        return rp, ci

    def assemble_matrix(self, fidx: int):
        _check(lib().emg_assemble_matrix(self._h, int(fidx)))

    def get_matrices(self):
        nnz = C.c_long()
        _check(lib().emg_get_sparsity(self._h, C.byref(nnz), None, None))
        Cv = np.zeros(nnz.value)
        Mv = np.zeros(nnz.value)
        bdr = np.zeros(self.nt, dtype=np.uint8)
        _check(lib().emg_get_matrices(self._h, _ptr(Cv), _ptr(Mv), _ptr(bdr)))
        return Cv, Mv, bdr

    def create_pc(self):
        _check(lib().emg_create_pc(self._h))

    def destroy_pc(self):
        _check(lib().emg_destroy_pc(self._h))

    def matshell_mult_a(self, x):
        x = _f64(x)
        y = np.zeros(2 * self.ne)
        _check(lib().emg_matshell_mult_a(self._h, _ptr(x), _ptr(y)))
        return y

    def pc_apply_b(self, b):
        b = _f64(b)
        x = np.zeros(2 * self.ne)
        _check(lib().emg_pc_apply_b(self._h, _ptr(b), _ptr(x)))
        return x

    def solve_linear_system(self, target, s_re, s_im, max_it=100, rtol=1e-8, raise_on_diverge=True):
        info = SolveInfo()
        rc = lib().emg_solve_linear_system(self._h, int(target), _ptr(_f64(s_re)), _ptr(_f64(s_im)), int(max_it),
                                           float(rtol), C.byref(info))
        if rc != EMG_OK and (raise_on_diverge or rc != EMG_DIVERGED_ITS):
            _check(rc)
        return info

    def get_solution(self, target):
        re = np.zeros(self.ne)
        im = np.zeros(self.ne)
        _check(lib().emg_get_solution(self._h, int(target), _ptr(re), _ptr(im)))
        return re, im

    def set_solution(self, target, re, im):
        _check(lib().emg_set_solution(self._h, int(target), _ptr(_f64(re)), _ptr(_f64(im))))

    def set_background(self, corners, nlay, ztop, lsig, maxl=None):
        """Layered columns under the four top corners (update_background_model);
        ztop/lsig are (4, maxl)."""
        ztop = _f64(ztop).reshape(4, -1)
        lsig = _f64(lsig).reshape(4, -1)
        maxl = ztop.shape[1] if maxl is None else int(maxl)
        _check(lib().emg_set_background(self._h, _ptr(_f64(corners)), _ptr(_i32(nlay)), _ptr(ztop),
                                        _ptr(lsig), maxl))

    def assemble_rhs_mt(self, fidx, mode):
        sr = np.zeros(self.ne)
        si = np.zeros(self.ne)
        _check(lib().emg_assemble_rhs_mt(self._h, int(fidx), int(mode), _ptr(sr), _ptr(si)))
        return sr, si

    def assemble_rhs_csem(self, fidx, tx, dipole_tets):
        sr = np.zeros(self.ne)
        si = np.zeros(self.ne)
        _check(lib().emg_assemble_rhs_csem(self._h, int(fidx), _ptr(_f64(tx)), _ptr(_i32(dipole_tets)),
                                           _ptr(sr), _ptr(si)))
        return sr, si

    def assemble_rhs_dual(self, rx, rx_tets):
        rx = _f64(rx).reshape(-1, 3)
        sr = np.zeros(self.ne)
        si = np.zeros(self.ne)
        _check(lib().emg_assemble_rhs_dual(self._h, rx.shape[0], _ptr(rx), _ptr(_i32(rx_tets)), _ptr(sr),
                                           _ptr(si)))
        return sr, si

    def estimate_error(self, fidx, tidx):
        nsol = 3 if tidx < 0 else 2
        err = np.zeros((nsol - 1) * self.nt)
        eta = np.zeros(nsol * self.nt)
        _check(lib().emg_estimate_error(self._h, int(fidx), int(tidx), _ptr(err), _ptr(eta)))
        return err.reshape(nsol - 1, self.nt), eta.reshape(nsol, self.nt)

    def estimate_error_noalloc_dev(self, fidx, tidx, err_ptr, eta_ptr):
        """estimate_error into caller-owned device buffers (err: n_err x T,
        eta: n_sol x T, float64) without any device allocation by the library."""
        _check(lib().emg_estimate_error_noalloc(self._h, int(fidx), int(tidx), C.c_void_p(err_ptr),
                                                C.c_void_p(eta_ptr)))

    def interpolate_fields(self, target, fidx, pts, tets):
        pts = _f64(pts).reshape(-1, 3)
        out = np.zeros(pts.shape[0] * 12)
        _check(lib().emg_interpolate_fields(self._h, int(target), int(fidx), pts.shape[0], _ptr(pts),
                                            _ptr(_i32(tets)), _ptr(out)))
        o = out.reshape(-1, 6, 2)
        z = o[..., 0] + 1j * o[..., 1]
        return z[:, :3], z[:, 3:]

    def assemble_rhs_mt_block(self, freqs, modes):
        """k MT right-hand sides at once: returns (n, k) complex."""
        freqs = _f64(freqs)
        modes = _i32(modes)
        out = np.zeros((self.ne, freqs.size), dtype=np.complex128)
        _check(lib().emg_assemble_rhs_mt_block(self._h, freqs.size, _ptr(freqs), _ptr(modes),
                                               _ptr(out.view(np.float64))))
        return out

    def assemble_rhs_mt_block_dev(self, freqs, modes, s_ptr):
        freqs = _f64(freqs)
        modes = _i32(modes)
        _check(lib().emg_assemble_rhs_mt_block_dev(self._h, freqs.size, _ptr(freqs), _ptr(modes),
                                                   C.c_void_p(s_ptr)))

    # -- batched fast path ----------------------------------------------------------------
    @staticmethod
    def _opts(rtol, max_it, use_guess, inner_fp32, restart):
        return BlockOpts(float(rtol), int(max_it), int(use_guess), int(inner_fp32), int(restart))

    def solve_block(self, freqs, rhs, x0=None, rtol=1e-8, max_it=100, inner_fp32=True, restart=30):
        """rhs: (n, k) complex -- the reference's s = s_re + i s_im per column.
        Returns (x (n, k) complex = e_re + i e_im, list of SolveInfo)."""
        freqs = _f64(freqs)
        k = freqs.size
        r = np.ascontiguousarray(np.asarray(rhs, dtype=np.complex128).reshape(self.ne, k))
        x = np.zeros((self.ne, k), dtype=np.complex128) if x0 is None else np.ascontiguousarray(
            np.asarray(x0, dtype=np.complex128).reshape(self.ne, k))
        infos = (SolveInfo * k)()
        o = self._opts(rtol, max_it, x0 is not None, inner_fp32, restart)
        rc = lib().emg_solve_block(self._h, k, _ptr(freqs), _ptr(r.view(np.float64)), _ptr(x.view(np.float64)),
                                   C.byref(o), C.cast(infos, C.c_void_p))
        _check(rc)
        return x, list(infos)

    def solve_block_dev(self, freqs, rhs_ptr, x_ptr, rtol=1e-8, max_it=100, use_guess=False, inner_fp32=True,
                        restart=30):
        freqs = _f64(freqs)
        k = freqs.size
        infos = (SolveInfo * k)()
        o = self._opts(rtol, max_it, use_guess, inner_fp32, restart)
        _check(lib().emg_solve_block_dev(self._h, k, _ptr(freqs), C.c_void_p(rhs_ptr), C.c_void_p(x_ptr),
                                         C.byref(o), C.cast(infos, C.c_void_p)))
        return list(infos)

    def divergence_correct_dev(self, freqs, rhs_ptr, x_ptr, fp32=True):
        """x += G phi (see emg_divergence_correct_dev); returns the FCG iterations."""
        freqs = _f64(freqs)
        its = C.c_long()
        _check(lib().emg_divergence_correct_dev(self._h, freqs.size, _ptr(freqs), C.c_void_p(rhs_ptr),
                                                C.c_void_p(x_ptr), int(bool(fp32)), C.byref(its)))
        return its.value

    def interpolate_fields_block_dev(self, freqs, x_ptr, pts, tets):
        """E and H of every column of a device block (n_edges x k complex) at
        receivers with known cells; returns E, H as (n_rx, k, 3) complex."""
        freqs = _f64(freqs)
        k = freqs.size
        p = _f64(np.asarray(pts).reshape(-1, 3))
        eh = np.zeros((p.shape[0], k, 2, 3), dtype=np.complex128)
        _check(lib().emg_interpolate_fields_block_dev(self._h, k, _ptr(freqs), C.c_void_p(x_ptr), p.shape[0],
                                                      _ptr(p), _ptr(_i32(tets)), _ptr(eh.view(np.float64))))
        return eh[:, :, 0, :], eh[:, :, 1, :]

    def assemble_rhs_csem_block_dev(self, freqs, tx, s_ptr):
        """CSEM right-hand sides for k (transmitter, frequency) columns into a
        device block; tx: (k, 7)."""
        freqs = _f64(freqs)
        t = _f64(np.asarray(tx).reshape(freqs.size, 7))
        _check(lib().emg_assemble_rhs_csem_block_dev(self._h, freqs.size, _ptr(freqs), _ptr(t), C.c_void_p(s_ptr)))

    def assemble_rhs_dual_block_dev(self, k, rx, s_ptr):
        """The dual right-hand side in all k columns of a device block."""
        r = _f64(np.asarray(rx).reshape(-1, 3))
        _check(lib().emg_assemble_rhs_dual_block_dev(self._h, int(k), r.shape[0], _ptr(r), C.c_void_p(s_ptr)))

    def amg_levels(self, sp, gpu, w_ref):
        """(rows, nnz A, nnz P, sum |A|, sum |P|) per level of a nodal hierarchy"""
        out = np.zeros(5 * 64)
        nl = C.c_int()
        _check(lib().emg_amg_levels(self._h, int(sp), int(bool(gpu)), float(w_ref), 64, C.byref(nl), _ptr(out)))
        return out[:5 * nl.value].reshape(nl.value, 5)

    def last_initial_residuals(self, k):
        out = np.zeros(int(k))
        _check(lib().emg_last_initial_residuals(self._h, int(k), _ptr(out)))
        return out

    def last_residual_floors(self, k):
        """per column of the last block solve: u || |b| + |A||x| || / ||b||, the
        relative residual below which the FP64 residual is rounding noise"""
        out = np.zeros(int(k))
        _check(lib().emg_last_residual_floors(self._h, int(k), _ptr(out)))
        return out

    # -- learned warm start ----------------------------------------------------------------
    @staticmethod
    def _cols(freqs, src, pos):
        f = _f64(freqs)
        s = _i32(src if src is not None else np.zeros(f.size, dtype=np.int32))
        p = None if pos is None else _f64(np.asarray(pos).reshape(f.size, 3))
        return f, s, p

    def warm_start_train(self, freqs, src, x_ptr, src_pos=None, steps=300, batch=65536, lr=2e-3, seed=1):
        """Trains the warm-start network on a solved device block; returns
        the last minibatch loss."""
        f, s, p = self._cols(freqs, src, src_pos)
        o = WarmOpts(int(steps), int(batch), float(lr), int(seed))
        loss = C.c_double()
        _check(lib().emg_warm_start_train(self._h, f.size, _ptr(f), _ptr(s), None if p is None else _ptr(p),
                                          C.c_void_p(x_ptr), C.byref(o), C.byref(loss)))
        return loss.value

    def warm_start_predict(self, freqs, src, x_ptr, tfreqs, tsrc, guess_ptr, src_pos=None, tsrc_pos=None,
                           network=True):
        f, s, p = self._cols(freqs, src, src_pos)
        tf, ts, tp = self._cols(tfreqs, tsrc, tsrc_pos)
        _check(lib().emg_warm_start_predict(self._h, f.size, _ptr(f), _ptr(s), None if p is None else _ptr(p),
                                            C.c_void_p(x_ptr), tf.size, _ptr(tf), _ptr(ts),
                                            None if tp is None else _ptr(tp),
                                            network if network in (0, 1, 2, 3) else int(bool(network)),
                                            C.c_void_p(guess_ptr)))

    def warm_start_params(self, set_to=None):
        n = C.c_int()
        _check(lib().emg_warm_start_params(self._h, None, None, C.byref(n)))
        out = np.zeros(n.value, dtype=np.float32)
        st = None if set_to is None else np.ascontiguousarray(set_to, dtype=np.float32)
        _check(lib().emg_warm_start_params(self._h, _ptr(out), None if st is None else _ptr(st), None))
        return out

    def warm_start_gradients(self, freqs, src, x_ptr, batch, step, src_pos=None):
        f, s, p = self._cols(freqs, src, src_pos)
        n = C.c_int()
        _check(lib().emg_warm_start_params(self._h, None, None, C.byref(n)))
        g = np.zeros(n.value, dtype=np.float32)
        loss = C.c_double()
        _check(lib().emg_warm_start_gradients(self._h, f.size, _ptr(f), _ptr(s), None if p is None else _ptr(p),
                                              C.c_void_p(x_ptr), int(batch), int(step), _ptr(g), C.byref(loss)))
        return g, loss.value

    def warm_start_reset(self):
        _check(lib().emg_warm_start_reset(self._h))

    def warm_start_losses(self):
        """(network loss, interpolation loss) of the last training step; -1 before training."""
        a, b = C.c_double(), C.c_double()
        _check(lib().emg_warm_start_losses(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def spmv_complex_dev(self, omegas, x_ptr, y_ptr, conj_out=False):
        om = _f64(omegas)
        _check(lib().emg_spmv_complex_dev(self._h, om.size, _ptr(om), C.c_void_p(x_ptr), C.c_void_p(y_ptr),
                                          int(conj_out)))

    def spmm_layout_dev(self, fp32, omegas, x_ptr, b_ptr, y_ptr, v, variant):
        """y = b - (C + w_c Ms) x on len(omegas) real columns with the lane
        layout (v, variant) forced; False when the layout is not built for
        that block width."""
        om = _f64(omegas)
        rc = lib().emg_spmm_layout_dev(self._h, int(bool(fp32)), om.size, int(v), int(variant), _ptr(om),
                                       C.c_void_p(x_ptr), C.c_void_p(b_ptr), C.c_void_p(y_ptr))
        if rc == EMG_ERR_ARG:
            return False
        _check(rc)
        return True

    def interpolate_fields_host(self, fidx, pts, tets, e_re, e_im):
        """interpolate_fields (src/em_fwd.cc:719-744) from a host solution;
        returns E, H as (n, 3) complex arrays."""
        p = _f64(np.asarray(pts).reshape(-1, 3))
        eh = np.zeros((p.shape[0], 2, 3), dtype=np.complex128)
        _check(lib().emg_interpolate_fields_host(self._h, int(fidx), p.shape[0], _ptr(p), _ptr(_i32(tets)),
                                                 _ptr(_f64(e_re)), _ptr(_f64(e_im)), _ptr(eh.view(np.float64))))
        return eh[:, 0, :], eh[:, 1, :]

    def save_vtk(self, path, arrays=None):
        """Mesh::save_vtk (src/em_mesh.cc:183-248): the mesh with tet_attr and
        the given per-tet arrays ({name: values}) as legacy ASCII VTK."""
        arrays = arrays or {}
        names = (C.c_char_p * max(1, len(arrays)))(*[k.encode() for k in arrays])
        vals = [_f64(v) for v in arrays.values()]
        for v in vals:
            if v.size != self.nt:
                raise EMGError(EMG_ERR_ARG, "one value per tet")
        ptrs = (C.c_void_p * max(1, len(vals)))(*[v.ctypes.data for v in vals])
        _check(lib().emg_save_vtk(self._h, os.fsencode(path), len(vals), C.cast(names, C.c_void_p),
                                  C.cast(ptrs, C.c_void_p)))

    def find_cell_around_point(self, pts):
        """find_cell_around_point (src/em_mesh.cc:527-566) on the context's mesh."""
        p = _f64(np.asarray(pts).reshape(-1, 3))
        out = np.zeros(p.shape[0], dtype=np.int32)
        _check(lib().emg_find_cell_around_point(self._h, p.shape[0], _ptr(p), _ptr(out)))
        return out

    def last_kernel_ms(self, name):
        v = C.c_double()
        _check(lib().emg_last_kernel_ms(self._h, name.encode(), C.byref(v)))
        return v.value

    def synchronize(self):
        _check(lib().emg_stream_synchronize(self._h))
