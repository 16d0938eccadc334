"""The nodal AMG setup on the device (emg_amg_gpu.cu) against the host build
(emg_amg.cpp) on the same assembled operators: the same algorithms in the
same order: the finest level is identical (rows, nonzeros, values to
rounding); the coarser levels keep the same coarse points, with nonzeros and
values within the slack that rounding-level differences of the Galerkin sums
leave to the interpolation's truncation ties.  Then a block
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
    # the finest level is built from identical operators: identical
    # coarsening, interpolation and Galerkin pattern, values to rounding
    assert np.array_equal(g[0, :3], h[0, :3])
    assert np.allclose(g[0, 3:], h[0, 3:], rtol=1e-12, atol=0)
    # coarser levels start from Galerkin operators that differ in the last
    # bits (summation order), which can move a near-tie of the truncation:
    # the same coarse points, nonzeros within 0.5 %, values within 1e-3
    assert np.array_equal(g[:, 0], h[:, 0])
    assert np.all(np.abs(g[:, 1:3] - h[:, 1:3]) <= 0.005 * h[:, 1:3] + 2)
    assert np.allclose(g[:, 3:], h[:, 3:], rtol=1e-3, atol=0)


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
