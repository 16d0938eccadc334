"""The allocation-free error estimator (emg_estimate_error_noalloc).

Callers whose device memory is owned by their own memory manager, or who may
not stall on cudaMalloc/cudaFree during a run, use this entry point: its
scratch is a fixed array inside the library and its results go to device
buffers the caller already owns.  It must give the same indicators as
emg_estimate_error (the estimator tolerance of the parity tests, 1e-10 of
the largest value) on consecutive calls, and refuse meshes larger than the
fixed scratch with a clear error.  This file is collected last so that a
failure here does not hide any other result.
"""

import numpy as np
import pytest

import emfem_b200 as E
from emfem_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _context(prob):
    c = E.EMContext(0)
    c.set_mesh(prob.mesh)
    c.set_model(prob.model)
    c.set_frequencies(prob.survey.freqs)
    c.create_linear_system(-3)
    return c


def test_noalloc_estimate_matches_allocating_entry_point():
    import torch
    prob = mg.mt_halfspace_block(4000, freqs=(0.1, 1.0, 10.0), name="noalloc")
    rx = prob.survey.rx
    tets = mg.PointLocator(prob.mesh).locate_all(rx)
    with _context(prob) as c:
        c.set_background(*mg.background_model(prob.mesh, prob.model))
        c.assemble_matrix(1)
        c.create_pc()
        for mode in (E.XY_POLAR, E.YX_POLAR):
            sr, si = c.assemble_rhs_mt(1, mode)
            c.solve_linear_system(mode, sr, si, 100, 1e-8)
        sr, si = c.assemble_rhs_dual(rx, tets)
        c.solve_linear_system(E.SOL_DUAL, sr, si, 100, 1e-6)
        nt = prob.mesh.n_tets
        err_d = torch.empty(2 * nt, dtype=torch.float64, device="cuda")
        eta_d = torch.empty(3 * nt, dtype=torch.float64, device="cuda")
        # two calls in a row at one frequency, then another frequency and back:
        # what an earlier call leaves in the shared scratch must not matter
        for fidx in (1, 1, 2, 1):
            err_ref, eta_ref = c.estimate_error(fidx, -3)
            err_d.fill_(float("nan"))
            eta_d.fill_(float("nan"))
            # the entry point runs on the context's stream, which is not
            # ordered after torch's: the fills must be finished first
            torch.cuda.synchronize()
            c.estimate_error_noalloc_dev(fidx, -3, err_d.data_ptr(), eta_d.data_ptr())
            err = err_d.cpu().numpy().reshape(2, nt)
            eta = eta_d.cpu().numpy().reshape(3, nt)
            assert np.isfinite(err).all() and np.isfinite(eta).all()
            assert np.abs(eta - eta_ref).max() <= 1e-10 * np.abs(eta_ref).max()
            assert np.abs(err - err_ref).max() <= 1e-10 * np.abs(err_ref).max()


def test_noalloc_estimate_csem_matches_allocating_entry_point():
    """CSEM form: two solutions (source and dual), one indicator per tet."""
    import torch
    prob = mg.marine_csem(5000, freqs=(0.25, 1.25), name="noalloc-csem")
    loc = mg.PointLocator(prob.mesh)
    tx = prob.survey.tx[0]
    rx = prob.survey.rx
    with E.EMContext(0) as c:
        c.set_mesh(prob.mesh)
        c.set_model(prob.model)
        c.set_frequencies(prob.survey.freqs)
        c.create_linear_system(0)
        nt = prob.mesh.n_tets
        err_d = torch.empty(nt, dtype=torch.float64, device="cuda")
        eta_d = torch.empty(2 * nt, dtype=torch.float64, device="cuda")
        for fidx in (0, 1):
            c.assemble_matrix(fidx)
            c.create_pc()
            sr, si = c.assemble_rhs_csem(fidx, tx, loc.locate_all(tx[None, :3]))
            c.solve_linear_system(E.SOL_CSEM, sr, si, 100, 1e-8)
            sr, si = c.assemble_rhs_dual(rx, loc.locate_all(rx))
            c.solve_linear_system(E.SOL_DUAL, sr, si, 100, 1e-6)
            for _ in range(2):
                err_ref, eta_ref = c.estimate_error(fidx, 0)
                err_d.fill_(float("nan"))
                eta_d.fill_(float("nan"))
                torch.cuda.synchronize()
                c.estimate_error_noalloc_dev(fidx, 0, err_d.data_ptr(), eta_d.data_ptr())
                err = err_d.cpu().numpy().reshape(1, nt)
                eta = eta_d.cpu().numpy().reshape(2, nt)
                assert np.isfinite(err).all() and np.isfinite(eta).all()
                assert np.abs(eta - eta_ref).max() <= 1e-10 * np.abs(eta_ref).max()
                assert np.abs(err - err_ref).max() <= 1e-10 * np.abs(err_ref).max()


def test_noalloc_estimate_rejects_meshes_beyond_its_scratch():
    import torch
    prob = mg.mt_halfspace_block(160_000, freqs=(1.0,), name="noalloc-big")
    assert prob.mesh.n_tets > 131072
    with _context(prob) as c:
        nt = prob.mesh.n_tets
        err_d = torch.empty(2 * nt, dtype=torch.float64, device="cuda")
        eta_d = torch.empty(3 * nt, dtype=torch.float64, device="cuda")
        with pytest.raises(E.EMGError) as ei:
            c.estimate_error_noalloc_dev(0, -3, err_d.data_ptr(), eta_d.data_ptr())
        assert ei.value.code == E.api.EMG_ERR_ARG
        assert "131072" in str(ei.value)
