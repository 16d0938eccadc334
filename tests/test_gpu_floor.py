"""Block FGMRES stops a column at the rounding floor of its own residual.

A residual b - A x computed in FP64 carries rounding errors of order
u || |b| + |A||x| || (u = 2^-53); below that no iteration can lower it.  The
reference's KSP runs on to max_it there; the block path stops such a column
and reports EMG_STOPPED_AT_FLOOR with the floor (emg_last_residual_floors).

The test asks for a tolerance no FP64 residual can meet (rtol 1e-18):
  * floor stop on: every column stops at the floor -- reason
    EMG_STOPPED_AT_FLOOR, true residual within twice the reported floor, in
    fewer than max_it iterations;
  * floor stop off: the same solve runs to max_it and reports
    EMG_DIVERGED_ITS, ending no lower than the floor allows (the answers
    agree to 1e-8 of the largest entry: both sit at the rounding floor, and
    the operator's conditioning magnifies that floor in the solution).
"""

import numpy as np
import pytest

import emfem_b200 as E
from emfem_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _solve(prob, floor_stop, max_it):
    import torch
    with E.EMContext(0) as c:
        c.process_options("-emg_block_floor_stop %d" % int(floor_stop))
        c.set_mesh(prob.mesh)
        c.set_model(prob.model)
        c.set_frequencies(prob.survey.freqs)
        c.create_linear_system(-3)
        c.set_background(*mg.background_model(prob.mesh, prob.model))
        c.assemble_matrix(0)
        freqs = np.repeat(np.asarray(prob.survey.freqs, dtype=np.float64), 2)
        modes = np.tile(np.array([-1, -2], dtype=np.int32), len(prob.survey.freqs))
        ne = prob.mesh.n_edges
        rhs = torch.zeros((ne, freqs.size), dtype=torch.complex128, device="cuda")
        x = torch.zeros_like(rhs)
        c.assemble_rhs_mt_block_dev(freqs, modes, rhs.data_ptr())
        infos = c.solve_block_dev(freqs, rhs.data_ptr(), x.data_ptr(), rtol=1e-18, max_it=max_it,
                                  inner_fp32=False)
        floors = c.last_residual_floors(freqs.size)
        return x.cpu().numpy(), infos, floors


def test_columns_stop_at_the_rounding_floor(mt_small):
    max_it = 60
    x1, inf1, fl1 = _solve(mt_small, True, max_it)
    for i, f in zip(inf1, fl1):
        assert f > 0
        assert i.reason == E.api.EMG_STOPPED_AT_FLOOR, (i.as_dict(), f)
        assert i.true_rel_res <= 2.0 * f
        assert i.outer_its < max_it
    x0, inf0, fl0 = _solve(mt_small, False, max_it)
    assert np.all(fl0 == 0)
    for i, f in zip(inf0, fl1):
        assert i.reason == E.api.EMG_DIVERGED_ITS
        assert i.true_rel_res >= 0.1 * f
    assert np.abs(x1 - x0).max() <= 1e-8 * np.abs(x0).max()
