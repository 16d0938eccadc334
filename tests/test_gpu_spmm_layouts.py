"""Every SpMM lane layout the autotuner can pick, against a float64 product.

The block solver times all legal layouts of its SpMM (row-split, row-group,
packed-record, software-pipelined, register-capped and chunked kernels, 1/2/4
columns per vector load)
on the first large operator it meets and keeps the fastest; the test meshes
are too small to trigger that tuning, so this test forces each layout through
emg_spmm_layout_dev on the assembled edge operator B = C + w_c Ms and checks
y = b - B x column by column.

Tolerances: FP64 layouts 1e-13 and FP32 layouts 1e-5 of the row scale
|b| + |B| |x| (the FP32 kernels round the operator, x and b to FP32 and
accumulate in FP32 over ~16 nonzeros per row).
"""

import numpy as np
import pytest
import scipy.sparse as sp

import emfem_b200 as E

pytestmark = pytest.mark.gpu

VARIANTS = [1, 2, 4, 8, 16, 32, -4, -8, 101, 102, 104, 204, 208, 304, 308, 401, 402, 501, 502, 601, 604]


@pytest.fixture(scope="module")
def edge_operator(mt_aniso):
    prob = mt_aniso
    c = E.EMContext(0)
    c.set_mesh(prob.mesh)
    c.set_model(prob.model)
    c.set_frequencies(prob.survey.freqs)
    c.create_linear_system(-3)
    c.assemble_matrix(0)
    rp, ci = c.make_sparsity_patterns()
    Cv, Mv, _ = c.get_matrices()
    w0 = 2 * np.pi * float(prob.survey.freqs[0])
    n = rp.size - 1
    Cm = sp.csr_matrix((Cv, ci, rp), shape=(n, n))
    Msm = sp.csr_matrix((Mv / w0, ci, rp), shape=(n, n))
    yield c, Cm, Msm
    c.close()


@pytest.mark.parametrize("fp32", [True, False])
@pytest.mark.parametrize("K", [8, 32])
def test_every_layout_matches_float64(edge_operator, fp32, K):
    import torch
    c, Cm, Msm = edge_operator
    n = Cm.shape[0]
    rng = np.random.default_rng(7 + K)
    omegas = 2 * np.pi * np.logspace(-3, 2, K)
    dt = torch.float32 if fp32 else torch.float64
    x = torch.from_numpy(rng.standard_normal((n, K))).to(dt).cuda()
    b = torch.from_numpy(rng.standard_normal((n, K))).to(dt).cuda()
    xh = x.double().cpu().numpy()
    bh = b.double().cpu().numpy()
    ref = np.empty((n, K))
    scale = np.empty((n, K))
    Ca, Ma = abs(Cm), abs(Msm)
    for j in range(K):
        A = Cm + omegas[j] * Msm
        ref[:, j] = bh[:, j] - A @ xh[:, j]
        scale[:, j] = np.abs(bh[:, j]) + (Ca + omegas[j] * Ma) @ np.abs(xh[:, j])
    tol = 1e-5 if fp32 else 1e-13
    ran = []
    for v in (1, 2, 4):
        for var in VARIANTS:
            y = torch.full_like(x, float("nan"))
            if not c.spmm_layout_dev(fp32, omegas, x.data_ptr(), b.data_ptr(), y.data_ptr(), v, var):
                continue
            torch.cuda.synchronize()
            err = (np.abs(y.double().cpu().numpy() - ref) / scale).max()
            assert err <= tol, (v, var, err)
            ran.append((v, var))
    # the pipelined and (FP32) packed and register-capped kernels are among
    # the layouts checked
    assert any(var in (204, 208) for _, var in ran)
    if fp32:
        assert any(var in (304, 308) for _, var in ran)
    if fp32 and K >= 16:
        assert any(var in (401, 402) for _, var in ran) and any(var in (501, 502) for _, var in ran)
    if fp32:
        assert any(var in (601, 604) for _, var in ran)
    assert len(ran) >= 8
