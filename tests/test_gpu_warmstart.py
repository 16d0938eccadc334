"""Learned warm start: the tensor-core network against its CPU restatement
(oracle/wsnet.py), and what it gains on a real solve.

Tolerances: the device and the CPU round the same operands to BF16 and
accumulate in FP32 in different orders, and a product rounded to BF16 can land
on the other side of a rounding boundary; gradients and outputs therefore
agree to 2e-3 of the largest value of each parameter group (an error in a
layout or a transposition gives errors of order 1).  The interpolation-only
guess has no BF16 step and agrees to 1e-6.
"""

import numpy as np
import pytest

import emfem_b200 as E
from emfem_b200 import meshgen as mg
import oracle.wsnet as W

pytestmark = pytest.mark.gpu

GROUPS = (("W1", 0, 1024), ("W2", 1024, 5120), ("W3", 5120, 9216), ("W4", 9216, 9344), ("b1", 9344, 9408),
          ("b2", 9408, 9472), ("b3", 9472, 9536), ("b4", 9536, 9538))


@pytest.fixture(scope="module")
def small():
    import torch
    prob = mg.mt_halfspace_block(3000, freqs=(0.1, 1.0, 10.0), name="ws-small")
    ne = prob.mesh.n_edges
    rng = np.random.default_rng(7)
    # smooth-ish complex columns: a few random modes of the edge midpoints
    mid = 0.5 * (prob.mesh.points[prob.mesh.edges[:, 0]] + prob.mesh.points[prob.mesh.edges[:, 1]]) / 1e4
    xs = np.zeros((ne, 6), dtype=np.complex128)
    for j in range(6):
        k = rng.normal(size=(3, 3))
        xs[:, j] = (np.sin(mid @ k[0]) + 1j * np.cos(mid @ k[1])) * np.exp(0.1 * (mid @ k[2])) * 10.0 ** rng.uniform(-3, 3)
    xs[rng.integers(0, ne, 20), :] = 0  # zero fields (homogeneous Dirichlet edges)
    freqs = np.array([0.1, 1.0, 10.0, 0.1, 1.0, 10.0])
    src = np.array([0, 0, 0, 1, 1, 1], dtype=np.int32)
    c = E.EMContext(0)
    c.set_mesh(prob.mesh)
    c.set_model(prob.model)
    c.set_frequencies(prob.survey.freqs)
    c.create_linear_system(-3)
    xd = torch.from_numpy(xs).to("cuda")
    yield dict(prob=prob, ctx=c, xs=xs, xd=xd, freqs=freqs, src=src, rng=rng)
    c.close()


def _random_params(rng):
    p = rng.normal(size=W.NPARAM).astype(np.float32) * 0.3
    return p


def test_gradients_match_cpu(small):
    c, rng = small["ctx"], small["rng"]
    params = _random_params(rng)
    c.warm_start_params(set_to=params)
    assert np.array_equal(c.warm_start_params(), params)
    batch, step = 5000, 3  # a partial last tile
    g, loss = c.warm_start_gradients(small["freqs"], small["src"], small["xd"].data_ptr(), batch, step)
    specs = W.training_specs(list(small["freqs"]), list(small["src"]))
    stat = W.edge_statics(small["prob"].mesh, small["prob"].model)
    sp_idx, e_idx = W.batch_samples(len(specs), small["prob"].mesh.n_edges, batch, step)
    X = np.zeros((batch, 16), dtype=np.float32)
    T = np.zeros((batch, 2), dtype=np.float32)
    for i, sp in enumerate(specs):
        sel = np.nonzero(sp_idx == i)[0]
        f, _, _, t = W.features(stat, small["xs"], sp, e_idx[sel], True)
        X[sel], T[sel] = f, t
    loss_c, g_c = W.gradients(params, X, T, np.float32(1.0 / batch))
    assert abs(loss - loss_c) <= 1e-3 * abs(loss_c)
    for name, a, b in GROUPS:
        err = np.abs(g[a:b] - g_c[a:b]).max() / max(np.abs(g_c[a:b]).max(), 1e-30)
        print("gradient %s: max %.3e rel err %.2e" % (name, np.abs(g_c[a:b]).max(), err))
        assert err <= 2e-3, name


def test_predictions_match_cpu(small):
    import torch
    c, rng = small["ctx"], small["rng"]
    params = _random_params(rng)
    c.warm_start_params(set_to=params)
    ne = small["prob"].mesh.n_edges
    # targets between the solved frequencies of each source
    tf = np.array([0.3, 3.0, 0.05, 30.0])
    ts = np.array([0, 1, 1, 0], dtype=np.int32)
    stat = W.edge_statics(small["prob"].mesh, small["prob"].model)
    for network in (False, True):
        gd = torch.zeros((ne, tf.size), dtype=torch.complex128, device="cuda")
        c.warm_start_predict(small["freqs"], small["src"], small["xd"].data_ptr(), tf, ts, gd.data_ptr(),
                             network=network)
        g = gd.cpu().numpy()
        for j in range(tf.size):
            cols = list(small["freqs"]) + [tf[j]]
            srcs = list(small["src"]) + [ts[j]]
            sp = [s for s in W.training_specs(cols, srcs) if s["tcol"] == len(cols) - 1][0]
            f, base, sc, _ = W.features(stat, small["xs"], sp, np.arange(ne), False)
            out = W.forward(params, f)[0] if network else np.zeros((ne, 2), np.float32)
            q = sp["q"]
            ref = ((base[:, 0] + q * out[:, 0]).astype(np.float64) + 1j * (base[:, 1] + q * out[:, 1])) * sc
            tol = 2e-3 if network else 1e-6
            assert np.abs(g[:, j] - ref).max() <= tol * np.abs(ref).max(), (network, j)


def test_quadratic_guess_matches_lagrange(small):
    """Mode 3: three-point Lagrange interpolation in log f where the three
    nearest solved columns of the source bracket the target (0.3 Hz, 3 Hz:
    bracketed by 0.1, 1, 10 Hz), the log-f interpolation elsewhere (0.05 Hz,
    30 Hz); FP64 arithmetic, 1e-12."""
    import torch
    c = small["ctx"]
    ne = small["prob"].mesh.n_edges
    tf = np.array([0.3, 3.0, 0.05, 30.0])
    ts = np.array([0, 1, 1, 0], dtype=np.int32)
    gd = torch.zeros((ne, tf.size), dtype=torch.complex128, device="cuda")
    c.warm_start_predict(small["freqs"], small["src"], small["xd"].data_ptr(), tf, ts, gd.data_ptr(), network=3)
    g = gd.cpu().numpy()
    lin = torch.zeros_like(gd)
    c.warm_start_predict(small["freqs"], small["src"], small["xd"].data_ptr(), tf, ts, lin.data_ptr(), network=0)
    lin = lin.cpu().numpy()
    xs, freqs, src = small["xs"], small["freqs"], small["src"]
    for j in range(2):
        cols = [i for i in range(freqs.size) if src[i] == ts[j]]
        u = np.log(freqs[cols])
        ut = np.log(tf[j])
        ref = np.zeros(ne, dtype=np.complex128)
        for a in range(3):
            w = np.prod([(ut - u[b]) / (u[a] - u[b]) for b in range(3) if b != a])
            ref += w * xs[:, cols[a]]
        assert np.abs(g[:, j] - ref).max() <= 1e-12 * np.abs(ref).max(), j
        assert np.abs(g[:, j] - lin[:, j]).max() > 1e-6 * np.abs(ref).max()  # not the linear guess
    for j in range(2, 4):  # outside the solved range: the linear interpolation
        assert np.abs(g[:, j] - lin[:, j]).max() <= 1e-12 * np.abs(lin[:, j]).max(), j


@pytest.fixture(scope="module")
def ab_runs():
    """Anchors (every other frequency, both polarisations) solved from zero;
    the network trained on them; the other frequencies solved from zero,
    from the log-f interpolation and from the network's guess."""
    import torch
    freqs = np.logspace(-2, 2, 7)
    prob = mg.mt_halfspace_block(12000, with_block=False, n_bodies=4, topo_height=500.0, freqs=tuple(freqs),
                                 seed=3, name="ws-ab")
    ne = prob.mesh.n_edges
    anchors = freqs[::2]
    targets = freqs[1::2]
    af, asrc = np.repeat(anchors, 2), np.tile(np.array([0, 1], np.int32), anchors.size)
    tf, tsrc = np.repeat(targets, 2), np.tile(np.array([0, 1], np.int32), targets.size)
    modes = lambda s: np.where(s == 0, E.XY_POLAR, E.YX_POLAR).astype(np.int32)
    out = {}
    with E.EMContext(0) as c:
        c.set_mesh(prob.mesh)
        c.set_model(prob.model)
        c.set_frequencies(freqs)
        c.create_linear_system(-3)
        c.set_background(*mg.background_model(prob.mesh, prob.model))
        c.assemble_matrix(0)
        sa = torch.zeros((ne, af.size), dtype=torch.complex128, device="cuda")
        xa = torch.zeros_like(sa)
        c.assemble_rhs_mt_block_dev(af, modes(asrc), sa.data_ptr())
        c.solve_block_dev(af, sa.data_ptr(), xa.data_ptr(), rtol=1e-8, max_it=200, inner_fp32=True)
        out["loss"] = c.warm_start_train(af, asrc, xa.data_ptr(), steps=200, batch=32768, lr=2e-3, seed=5)
        out["losses"] = c.warm_start_losses()
        st = torch.zeros((ne, tf.size), dtype=torch.complex128, device="cuda")
        c.assemble_rhs_mt_block_dev(tf, modes(tsrc), st.data_ptr())
        for arm in ("zero", "interp", "network", "auto"):
            x = torch.zeros_like(st)
            if arm != "zero":
                c.warm_start_predict(af, asrc, xa.data_ptr(), tf, tsrc, x.data_ptr(),
                                     network={"interp": 0, "network": 1, "auto": 2}[arm])
            infos = c.solve_block_dev(tf, st.data_ptr(), x.data_ptr(), rtol=1e-8, max_it=200, inner_fp32=True,
                                      use_guess=(arm != "zero"))
            out[arm] = dict(its=[i.outer_its for i in infos], res=[i.true_rel_res for i in infos],
                            ok=all(i.reason == 0 for i in infos), r0=c.last_initial_residuals(tf.size),
                            x=x.cpu().numpy())
    return out


def test_warm_start_converges_to_the_same_fields(ab_runs):
    z = ab_runs["zero"]["x"]
    for arm in ("zero", "interp", "network", "auto"):
        r = ab_runs[arm]
        assert r["ok"] and max(r["res"]) <= 1e-8
        for j in range(z.shape[1]):
            assert np.abs(r["x"][:, j] - z[:, j]).max() <= 1e-6 * np.abs(z[:, j]).max()


def test_warm_start_ab_iterations(ab_runs):
    """A/B: outer iterations of the target columns from zero, from the log-f
    interpolation, from the trained network's guess, and from the gated
    choice (the network only where its training loss is a quarter of the
    interpolation's).  Guesses are judged by their residual column by column,
    so no arm starts worse than zero; the gated arm does not iterate more
    than the zero start."""
    for arm in ("zero", "interp", "network", "auto"):
        r = ab_runs[arm]
        print("%-8s outer its %s (total %d), initial residual %s" % (arm, r["its"], sum(r["its"]),
                                                                   np.array2string(r["r0"], precision=2)))
    print("training loss %.3e (network) vs %.3e (interpolation alone)" % ab_runs["losses"])
    for arm in ("interp", "network", "auto"):
        assert np.all(ab_runs[arm]["r0"] <= 1.0)
    assert sum(ab_runs["auto"]["its"]) <= sum(ab_runs["zero"]["its"])
