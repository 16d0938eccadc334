"""AMS variants against the configuration the parity tests pin.

1. The fused nodal V-cycle (one cooperative launch per AMS subspace
correction, emg_fused.cu) against the step-by-step V-cycle it replays.

Both run the same recorded steps; only the SpMM lane layout, and with it the
order of the FP32/FP64 sums, differs.  So with the fused launch on and off:
  * the batched mixed-precision solve and the reference-facing FP64 solve
    converge in the same number of outer iterations (+-1) to the same
    tolerance;
  * their solutions agree to 1e-6 of the largest entry at rtol 1e-10 (the
    bound the solves are held to against the exact discrete solution).
A hierarchy coarsened to 16 rows (emg_amg_max_coarse) gives every nodal
subspace several levels even on this small mesh.

2. The vector Pi space (cycle character '2': Pi^T B Pi with its x/y/z
couplings and systems AMG with the unknown approach as hypre's cycle types
1/3/5/7 use it, or its three diagonal blocks side by side), in the FP32 block
cycle and the FP64 reference-facing solve, and the component cycle "034501"
with the inner iteration cap of the reference: every variant converges to
rtol 1e-10 and agrees with the exact discrete solution (sparse direct solve)
to 1e-6 of its largest entry.

3. The same bar with the edge-column SpMMs tiled (x rows of each row tile
staged once in shared memory), with the default 64 KB and with small tiles
(16 KB: more, shorter tiles).

4. The same bar with Chebyshev smoothers of degree 3 to 5 (the three-term
recurrence's middle steps) on the edges of both solvers and on the nodal
levels, stepwise and in the fused V-cycle; and with each nodal restriction
taking the fed level's first smoothing step (the default) or leaving it to
its own launch, for Chebyshev and l1-Jacobi smoothing; and with nodal V(0, m)
cycles (no pre-smoothing), stepwise and fused.
"""

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla

import emfem_b200 as E
from emfem_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _run(prob, fused, coarse, extra=""):
    bg = mg.background_model(prob.mesh, prob.model)
    with E.EMContext(0) as c:
        c.process_options("-emg_fused_vcycle %d -emg_amg_max_coarse %d %s" % (fused, coarse, extra))
        assert c.get_option("emg_fused_vcycle") == fused
        c.set_mesh(prob.mesh)
        c.set_model(prob.model)
        c.set_frequencies(prob.survey.freqs)
        c.create_linear_system(-3)
        c.set_background(*bg)
        cols, freqs = [], []
        for fidx in (0, 2):
            c.assemble_matrix(fidx)
            for mode in (E.XY_POLAR, E.YX_POLAR):
                sr, si = c.assemble_rhs_mt(fidx, mode)
                cols.append(sr + 1j * si)
                freqs.append(prob.survey.freqs[fidx])
        x, infos = c.solve_block(freqs, np.stack(cols, axis=1), rtol=1e-10, max_it=300, inner_fp32=True)
        blk = (x, [i.outer_its for i in infos], [i.true_rel_res for i in infos], [i.reason for i in infos])
        c.assemble_matrix(1)
        c.create_pc()
        sr, si = c.assemble_rhs_mt(1, E.XY_POLAR)
        info = c.solve_linear_system(E.XY_POLAR, sr, si, 300, 1e-10)
        er, ei = c.get_solution(E.XY_POLAR)
        plain = (er + 1j * ei, info.outer_its, info.true_rel_res, info.reason)
    return blk, plain


@pytest.mark.parametrize("coarse", [200, 16])
def test_fused_vcycle_matches_stepwise(mt_small, coarse):
    b0, p0 = _run(mt_small, 0, coarse)
    b1, p1 = _run(mt_small, 1, coarse)
    for blk in (b0, b1):
        assert all(r == 0 for r in blk[3]) and max(blk[2]) <= 1e-10
    for pl in (p0, p1):
        assert pl[3] == 0 and pl[2] <= 1e-10
    for j in range(len(b0[1])):
        assert abs(b0[1][j] - b1[1][j]) <= 1
        ref = b0[0][:, j]
        assert np.abs(b1[0][:, j] - ref).max() <= 1e-6 * np.abs(ref).max()
    assert abs(p0[1] - p1[1]) <= 1
    assert np.abs(p1[0] - p0[0]).max() <= 1e-6 * np.abs(p0[0]).max()


def _direct(rp, ci, Cv, Mv, sr, si):
    A = sp.csr_matrix((Cv + 1j * Mv, ci, rp)).tocsc()
    return sla.spsolve(A, sr - 1j * si)


@pytest.mark.parametrize("extra", ["-emg_fp32_cycle 0201 -B_pc_hypre_ams_cycle_type 1 -emg_pi_coupled 1",
                                   "-emg_fp32_cycle 0201 -B_pc_hypre_ams_cycle_type 3 -emg_pi_coupled 0",
                                   "-emg_fp32_cycle 034501 -emg_block_inner_max_it 100",
                                   "-emg_spmm_tiled 1",
                                   "-emg_spmm_tiled 1 -emg_tiled_smem_kb 16",
                                   "-emg_fp32_cycle 0201 -B_pc_hypre_ams_cycle_type 7 -emg_fused_vcycle 1 "
                                   "-emg_fused_rows 400",
                                   "-emg_block_cheb_degree 3 -emg_block_relax_times 1 -emg_cheb_degree 4 "
                                   "-emg_amg_cheb_degree 3",
                                   "-emg_block_cheb_degree 5 -emg_amg_cheb_degree 4 -emg_fused_vcycle 1 "
                                   "-emg_fused_rows 400",
                                   "-emg_restrict_smooth 0",
                                   "-emg_restrict_smooth 0 -emg_smoother l1jacobi",
                                   "-emg_smoother l1jacobi",
                                   "-emg_amg_pre_smooth 0",
                                   "-emg_amg_pre_smooth 0 -emg_amg_relax_times 2 -emg_fused_vcycle 1 -emg_fused_rows 400"])
def test_pi_vector_space_cycles(mt_small, extra):
    prob = mt_small
    bg = mg.background_model(prob.mesh, prob.model)
    with E.EMContext(0) as c:
        c.process_options(extra)
        c.set_mesh(prob.mesh)
        c.set_model(prob.model)
        c.set_frequencies(prob.survey.freqs)
        c.create_linear_system(-3)
        c.set_background(*bg)
        rp, ci = c.make_sparsity_patterns()
        cols, freqs, ref = [], [], []
        for fidx in (0, 2):
            c.assemble_matrix(fidx)
            Cv, Mv, _ = c.get_matrices()
            for mode in (E.XY_POLAR, E.YX_POLAR):
                sr, si = c.assemble_rhs_mt(fidx, mode)
                cols.append(sr + 1j * si)
                freqs.append(prob.survey.freqs[fidx])
                ref.append(_direct(rp, ci, Cv, Mv, sr, si))
        x, infos = c.solve_block(freqs, np.stack(cols, axis=1), rtol=1e-10, max_it=300, inner_fp32=True)
        for j in range(len(freqs)):
            assert infos[j].reason == 0 and infos[j].true_rel_res <= 1e-10
            assert np.abs(x[:, j] - ref[j]).max() <= 1e-6 * np.abs(ref[j]).max()
        c.assemble_matrix(1)
        Cv, Mv, _ = c.get_matrices()
        c.create_pc()
        sr, si = c.assemble_rhs_mt(1, E.XY_POLAR)
        info = c.solve_linear_system(E.XY_POLAR, sr, si, 300, 1e-10)
        assert info.reason == 0 and info.true_rel_res <= 1e-10
        er, ei = c.get_solution(E.XY_POLAR)
        z = _direct(rp, ci, Cv, Mv, sr, si)
        assert np.abs((er + 1j * ei) - z).max() <= 1e-6 * np.abs(z).max()


def test_fused_barrier_wait_runs_out_and_reports(mt_small):
    """The fused V-cycle's grid-barrier waits are bounded: with the test-only
    option that withholds the first barrier's release (the waiting blocks
    wait for a flag that nothing sets) and a 1 ms bound, every waiter gives
    up, the kernel ends, the error word is set and the solve returns
    EMG_ERR_CUDA; a fresh context then solves normally."""
    prob = mt_small
    bg = mg.background_model(prob.mesh, prob.model)
    freqs = [prob.survey.freqs[0], prob.survey.freqs[0]]
    modes = [E.XY_POLAR, E.YX_POLAR]
    for withhold in (1, 0):
        with E.EMContext(0) as c:
            c.process_options("-emg_fused_vcycle 1 -emg_fused_wait_ms 1 -emg_fused_test_withhold %d" % withhold)
            c.set_mesh(prob.mesh)
            c.set_model(prob.model)
            c.set_frequencies(prob.survey.freqs)
            c.create_linear_system(-3)
            c.set_background(*bg)
            c.assemble_matrix(0)
            rhs = c.assemble_rhs_mt_block(freqs, modes)
            if withhold:
                with pytest.raises(E.EMGError) as ei:
                    c.solve_block(freqs, rhs, rtol=1e-8, max_it=100, inner_fp32=True)
                assert ei.value.code == E.api.EMG_ERR_CUDA
                assert "timed out" in str(ei.value)
            else:
                x, infos = c.solve_block(freqs, rhs, rtol=1e-8, max_it=100, inner_fp32=True)
                assert all(i.reason == 0 and i.true_rel_res <= 1e-8 for i in infos)
