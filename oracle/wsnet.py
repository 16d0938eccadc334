"""CPU restatement of the warm-start network (test infrastructure).

The network has no counterpart in the reference (which starts every FGMRES
from zero, src/em_la.cc:49); this module is the checker of the device
kernels in emfem_b200/csrc/emg_mlp.cu and emg_warmstart.cu: the same sample
selection, features, BF16 roundings (inputs, weights, activations and
back-propagated errors are BF16 operands of FP32-accumulated products) and
the same gradients, in numpy.  Only tests import it.
"""

import math

import numpy as np

NPARAM = 64 * 16 + 64 * 64 + 64 * 64 + 2 * 64 + 64 * 3 + 2


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p):
    p = np.asarray(p)
    o = 0
    out = {}
    for name, shape in (("W1", (64, 16)), ("W2", (64, 64)), ("W3", (64, 64)), ("W4", (2, 64)),
                        ("b1", (64,)), ("b2", (64,)), ("b3", (64,)), ("b4", (2,))):
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([d[k].ravel() for k in ("W1", "W2", "W3", "W4", "b1", "b2", "b3", "b4")]).astype(np.float32)


def _mix32(x):
    x = np.asarray(x, dtype=np.uint64) & 0xFFFFFFFF
    x ^= x >> 16
    x = (x * 0x7FEB352D) & 0xFFFFFFFF
    x ^= x >> 15
    x = (x * 0x846CA68B) & 0xFFFFFFFF
    x ^= x >> 16
    return x


def edge_statics(mesh, model):
    """Per-edge static features (3 x float4 per edge)."""
    rho = np.asarray(model.rho, dtype=np.float64)
    form = model.aniso_form
    rh, rv = rho[:, 0].copy(), rho[:, 0].copy()
    if form == 1:
        rv = rho[:, 1]
    elif form in (2, 3):
        rh = np.sqrt(rho[:, 0] * rho[:, 1])
        rv = rho[:, 2]
    lr = np.stack([np.log10(rh), np.log10(rv)], axis=1).astype(np.float32)
    ne = mesh.n_edges
    acc = np.zeros((ne, 3))
    t2e = mesh.tet2edge.astype(np.int64)
    a = lr[mesh.attr]
    for i in range(6):
        np.add.at(acc[:, 0], t2e[:, i], a[:, 0])
        np.add.at(acc[:, 1], t2e[:, i], a[:, 1])
        np.add.at(acc[:, 2], t2e[:, i], 1.0)
    acc = acc.astype(np.float32)
    n = np.maximum(acc[:, 2], np.float32(1))
    p = mesh.points
    d = p[mesh.edges[:, 1]] - p[mesh.edges[:, 0]]
    m = 0.5 * (p[mesh.edges[:, 1]] + p[mesh.edges[:, 0]])
    ln = np.sqrt((d * d).sum(axis=1))
    st = np.zeros((ne, 12), dtype=np.float32)
    st[:, 0] = (acc[:, 0] / n - np.float32(2)) / np.float32(3)
    st[:, 1] = (acc[:, 1] / n - np.float32(2)) / np.float32(3)
    st[:, 2] = np.log10(np.maximum(ln, 1e-3)).astype(np.float32) - np.float32(2.5)
    st[:, 3] = (d[:, 0] / ln).astype(np.float32)
    st[:, 4] = (d[:, 1] / ln).astype(np.float32)
    st[:, 5] = (d[:, 2] / ln).astype(np.float32)
    st[:, 8:11] = m.astype(np.float32)
    return st


def training_specs(freqs, src, pos=None):
    """(a, b, tcol, tau, logf, q, point, srcpos) per target, as the device builds them;
    q = (log10 f - log10 f_a)(log10 f - log10 f_b) scales the network's
    output (a curvature in log f) into the correction."""
    specs = []
    for j in range(len(freqs)):
        cand = sorted((abs(math.log(freqs[i] / freqs[j])), i) for i in range(len(freqs))
                      if i != j and src[i] == src[j])
        if not cand:
            continue
        a = cand[0][1]
        b = cand[1][1] if len(cand) > 1 else a
        fa, fb = freqs[a], freqs[b]
        tau = 0.0 if fa == fb else math.log(freqs[j] / fa) / math.log(fb / fa)
        lt = math.log10(freqs[j])
        q = (lt - math.log10(fa)) * (lt - math.log10(fb))
        specs.append(dict(a=a, b=b, tcol=j, tau=np.float32(tau), logf=np.float32(0.5 * lt), q=np.float32(q),
                          point=pos is not None, pos=None if pos is None else np.asarray(pos[j], np.float32)))
    return specs


def features(stat, xs, spec, edges, with_target):
    """Features (n x 16), base (n x 2), scale (n,), target curvature (n x 2):
    the guess is (base + q * output) * scale."""
    ea, eb = xs[edges, spec["a"]], xs[edges, spec["b"]]
    sc = np.maximum(np.abs(ea), np.abs(eb))
    ok = sc > 1e-300
    inv = np.where(ok, 1.0 / np.where(ok, sc, 1.0), 0.0)
    n = edges.size
    f = np.zeros((n, 16), dtype=np.float32)
    f[:, 0] = (ea.real * inv).astype(np.float32)
    f[:, 1] = (ea.imag * inv).astype(np.float32)
    f[:, 2] = (eb.real * inv).astype(np.float32)
    f[:, 3] = (eb.imag * inv).astype(np.float32)
    s = stat[edges]
    f[:, 4:10] = s[:, 0:6]
    if spec["point"]:
        dd = s[:, 8:11] - spec["pos"]
        dist = np.sqrt((dd * dd).sum(axis=1)).astype(np.float32)
    else:
        dist = s[:, 10]
    f[:, 10] = np.copysign(np.log10(np.float32(1) + np.abs(dist) * np.float32(0.01)), dist).astype(np.float32) * \
        np.float32(0.5)
    f[:, 11] = spec["logf"]
    f[:, 12] = spec["tau"]
    f[~ok] = 0
    tau = spec["tau"]
    base = np.stack([(np.float32(1) - tau) * f[:, 0] + tau * f[:, 2],
                     (np.float32(1) - tau) * f[:, 1] + tau * f[:, 3]], axis=1).astype(np.float32)
    tgt = np.zeros((n, 2), dtype=np.float32)
    q = spec["q"]
    if with_target and abs(q) >= np.float32(1e-4):
        et = xs[edges, spec["tcol"]]
        iq = np.float32(1) / q
        tgt[:, 0] = np.clip(((et.real * inv).astype(np.float32) - base[:, 0]) * iq, -4.0, 4.0)
        tgt[:, 1] = np.clip(((et.imag * inv).astype(np.float32) - base[:, 1]) * iq, -4.0, 4.0)
        tgt[~ok] = 0
    return f, base, np.where(ok, sc, 0.0), tgt


def _gelu(z, dtype=np.float32):
    z64 = z.astype(np.float64)
    e = np.vectorize(math.erf)(z64 / math.sqrt(2.0))
    g = 0.5 * z64 * (1 + e)
    gd = 0.5 * (1 + e) + z64 * np.exp(-0.5 * z64 * z64) / math.sqrt(2 * math.pi)
    return g.astype(dtype), gd.astype(dtype)


def forward(params, X, exact=False):
    """exact=False: the device's arithmetic (BF16 operands, FP32 sums);
    exact=True: float64 without rounding (for finite-difference checks)."""
    dt = np.float64 if exact else np.float32
    rnd = (lambda a: np.asarray(a, dtype=np.float64)) if exact else bf16
    P = unpack(params)
    P = {k: v.astype(dt) for k, v in P.items()}
    Wr = {k: rnd(P[k]) for k in ("W1", "W2", "W3", "W4")}
    H, G = [rnd(X)], []
    for w, b in ((Wr["W1"], P["b1"]), (Wr["W2"], P["b2"]), (Wr["W3"], P["b3"])):
        z = (H[-1] @ w.T + b).astype(dt)
        g, gd = _gelu(z, dt)
        H.append(rnd(g))
        G.append(rnd(gd))
    out = H[-1] @ Wr["W4"].T + P["b4"]
    return out.astype(dt), H, G, Wr


def gradients(params, X, tgt, inv_batch, exact=False):
    """Loss and parameter gradients (the device's parameter layout)."""
    rnd = (lambda a: np.asarray(a, dtype=np.float64)) if exact else bf16
    out, H, G, Wr = forward(params, X, exact)
    d = out - tgt
    loss = float(0.5 * (d.astype(np.float64) ** 2).sum() * inv_batch)
    dz4 = rnd(d * inv_batch)
    dz3 = rnd((dz4 @ Wr["W4"]) * G[2])
    dz2 = rnd((dz3 @ Wr["W3"]) * G[1])
    dz1 = rnd((dz2 @ Wr["W2"]) * G[0])
    g = dict(W1=dz1.T @ H[0], W2=dz2.T @ H[1], W3=dz3.T @ H[2], W4=dz4.T @ H[3],
             b1=dz1.sum(0), b2=dz2.sum(0), b3=dz3.sum(0), b4=dz4.sum(0))
    return loss, np.concatenate([g[k].ravel() for k in ("W1", "W2", "W3", "W4", "b1", "b2", "b3", "b4")])


def batch_samples(nspec, ne, batch, step):
    s = np.arange(batch, dtype=np.uint64)
    seed = (0x51ED2705 + 7919 * step) & 0xFFFFFFFF
    e = (_mix32((s * 0x9E3779B9 + seed) & 0xFFFFFFFF) % ne).astype(np.int64)
    return (s % nspec).astype(np.int64), e
