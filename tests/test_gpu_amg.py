"""The nodal AMG setup on the device (emg_amg_gpu.cu) against the host build
(emg_amg.cpp) on the same assembled operators: the same algorithms in the
same order, so every level has the same number of rows and nonzeros in A
and P, and the level operators agree to rounding (sums of |values| to 1e-10
relative; the Galerkin products sum in a different order).  Then a block
solve with the device-built hierarchy (the default) against one with the
host-built hierarchy: both converge to the same solution."""

import numpy as np
import pytest

import emfem_b200 as E
from emfem_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _ctx(prob, opts=""):
    c = E.EMContext(0)
    if opts:
        c.process_options(opts)
    c.set_mesh(prob.mesh)
    c.set_model(prob.model)
    c.set_frequencies(prob.survey.freqs)
    c.create_linear_system(-3)
    return c


@pytest.mark.parametrize("sp", [0, 1, 4])
def test_device_hierarchy_matches_host_build(mt_aniso, sp):
    w_ref = 2 * np.pi * 0.1
    with _ctx(mt_aniso) as c:
        c.assemble_matrix(0)
        g = c.amg_levels(sp, True, w_ref)
        h = c.amg_levels(sp, False, w_ref)
    print("subspace %d levels (rows, nnzA, nnzP):\n device %s\n host   %s" % (sp, g[:, :3].astype(int).tolist(),
                                                                         h[:, :3].astype(int).tolist()))
    assert g.shape == h.shape
    assert np.array_equal(g[:, :3], h[:, :3])
    assert np.allclose(g[:, 3:], h[:, 3:], rtol=1e-10, atol=0)


def test_block_solve_with_device_hierarchy(mt_small):
    prob = mt_small
    bg = mg.background_model(prob.mesh, prob.model)
    freqs = [prob.survey.freqs[0], prob.survey.freqs[0], prob.survey.freqs[2], prob.survey.freqs[2]]
    modes = [E.XY_POLAR, E.YX_POLAR] * 2
    xs = []
    for opts in ("-emg_gpu_amg 1", "-emg_gpu_amg 0"):
        with _ctx(prob, opts) as c:
            c.set_background(*bg)
            c.assemble_matrix(0)
            rhs = c.assemble_rhs_mt_block(freqs, modes)
            x, infos = c.solve_block(freqs, rhs, rtol=1e-10, max_it=300, inner_fp32=True)
            assert all(i.reason == 0 and i.true_rel_res <= 1e-10 for i in infos)
            xs.append(x)
    for j in range(len(freqs)):
        assert np.abs(xs[0][:, j] - xs[1][:, j]).max() <= 1e-6 * np.abs(xs[1][:, j]).max()
