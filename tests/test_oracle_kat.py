"""Pins the CPU oracle against known answers (the reference ships no tests or
golden vectors; see tests/golden/make_golden.py for the independent
derivations).  CPU only."""

import json
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla

import oracle as O
from emfem_b200 import meshgen as mg

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MU = 4e-7 * np.pi


@pytest.fixture(scope="module")
def small():
    return mg.mt_halfspace_block(1500, freqs=(1.0,), name="kat")


def one_tet(verts, ids):
    ids = np.asarray(ids)
    order = np.argsort(ids)
    pts = np.zeros((int(ids.max()) + 1, 3))
    for v, i in zip(verts, ids):
        pts[i] = v
    tets = ids[order][None, :]
    return mg.build_topology(pts, tets, np.zeros(1, dtype=np.int32))


def test_whitney_element_matrices_match_closed_form():
    gold = json.load(open(os.path.join(GOLD, "whitney_elements.json")))
    for el in gold["elements"]:
        m = one_tet(np.array(el["verts"]), el["ids"])
        model = mg.Model(mg.ARBITRARY, np.array([el["rho"] + el["angles"]]))
        assert np.allclose(O.cell_sigma(model, 0), np.array(el["sigma"]), rtol=1e-12, atol=1e-15)
        C, M = O.element_matrices(O.Mesh(m), model, 0, 1.0)
        Cg, Mg = np.array(el["C"]), np.array(el["Ms"])
        assert np.abs(C - Cg).max() <= 1e-10 * np.abs(Cg).max()
        assert np.abs(M - Mg).max() <= 1e-10 * np.abs(Mg).max()


def test_quadrature_weights(small):
    om = O.Mesh(small.mesh)
    rng = np.random.default_rng(0)
    for t in rng.choice(om.nt, 20, replace=False):
        vol, diam, fd = O.tet_geometry(om, int(t))
        q, w = O.cell_quadrature(om, int(t))
        assert abs(w.sum() - vol) <= 1e-12 * vol
        p = small.mesh.points[small.mesh.tets[t]]
        assert np.allclose(q.mean(axis=0), p.mean(axis=0), rtol=0, atol=1e-9 * np.abs(p).max())
        for f in range(4):
            a, b, c = p[[(f + 1) % 4, (f + 2) % 4, (f + 3) % 4]]
            area = 0.5 * np.linalg.norm(np.cross(b - a, c - a))
            qf, wf = O.face_quadrature(om, int(t), f)
            assert abs(wf.sum() - 6 * area) <= 1e-10 * area      # the reference's rule sums to 6x the area
        # circumradius of the tet
        A = 2 * (p[1:] - p[0])
        rhs = (p[1:] ** 2).sum(1) - (p[0] ** 2).sum()
        cc = np.linalg.solve(A, rhs)
        assert abs(diam - np.linalg.norm(cc - p[0])) <= 1e-9 * diam


def test_sparsity_pattern_independent(small):
    m = small.mesh
    rp, ci = O.sparsity(O.Mesh(m))
    rows = np.repeat(m.tet2edge, 6, axis=1).ravel()
    cols = np.tile(m.tet2edge, (1, 6)).ravel()
    A = sp.csr_matrix((np.ones(rows.size), (rows, cols)), shape=(m.n_edges, m.n_edges))
    A.sum_duplicates()
    A.sort_indices()
    assert np.array_equal(rp, A.indptr) and np.array_equal(ci, A.indices)


def test_operators_symmetric_spd_and_curl_grad(small):
    m = small.mesh
    om = O.Mesh(m)
    rp, ci = O.sparsity(om)
    Cv, Mv, bdr = O.assemble(om, small.model, 1.0, rp, ci)
    C = sp.csr_matrix((Cv, ci, rp))
    M = sp.csr_matrix((Mv, ci, rp))
    assert abs(C - C.T).max() == 0 and abs(M - M.T).max() == 0
    B = (C + M).toarray()
    assert np.linalg.eigvalsh(B).min() > 0
    G = sp.csr_matrix((np.tile([-1.0, 1.0], m.n_edges), m.edges.ravel(), np.arange(0, 2 * m.n_edges + 1, 2)),
                      shape=(m.n_edges, m.n_vertices))
    CG = (C @ G).toarray()
    # rows whose couplings were not zeroed by the Dirichlet treatment
    touched = np.zeros(m.n_edges, bool)
    for t in range(m.n_tets):
        if m.edge_bdr[m.tet2edge[t]].any():
            touched[m.tet2edge[t]] = True
    inner = ~touched
    assert inner.any()
    assert np.abs(CG[inner]).max() <= 1e-10 * np.abs(C).max()
    # boundary cells are exactly the tets with a boundary edge
    assert np.array_equal(bdr.astype(bool), m.edge_bdr[m.tet2edge].any(axis=1))


def test_plane_wave_matches_layered_impedance():
    gold = json.load(open(os.path.join(GOLD, "plane_wave_layered.json")))
    for c in gold["cases"]:
        # the reference's column: 100 km of air above the earth
        ztop = [-100e3, 0.0] + list(np.cumsum(c["thickness"]))
        lsig = [1e-8] + c["sigma"]
        eh = O.plane_wave(ztop, lsig, c["freq"], [0.0])[0]
        Z = eh[0] / eh[1]
        w = 2 * np.pi * c["freq"]
        assert abs(abs(Z) ** 2 / (w * MU) - c["rho_a"]) <= 1e-6 * c["rho_a"]
        assert abs(abs(np.degrees(np.angle(Z))) - abs(c["phase_deg"])) <= 1e-6


def test_plane_wave_continuity_and_ode():
    ztop = np.array([-100e3, 0.0, 800.0, 3000.0])
    lsig = np.array([1e-8, 0.02, 0.5, 0.002])
    f = 1.0
    w = 2 * np.pi * f
    for zi in ztop[1:]:
        a = O.plane_wave(ztop, lsig, f, [zi - 1e-6])[0]
        b = O.plane_wave(ztop, lsig, f, [zi + 1e-6])[0]
        assert abs(a[0] - b[0]) <= 1e-6 * abs(a[0])     # E continuous
        assert abs(a[1] - b[1]) <= 1e-6 * abs(a[1])     # H continuous
    # d2E/dz2 = -i w mu sigma E inside a layer
    z0, h = 1500.0, 0.5
    e = O.plane_wave(ztop, lsig, f, [z0 - h, z0, z0 + h])[:, 0]
    d2 = (e[0] - 2 * e[1] + e[2]) / h ** 2
    assert abs(d2 - (-1j * w * MU * 0.5) * e[1]) <= 1e-4 * abs(w * MU * 0.5 * e[1])


def test_refine_marking_known_answers():
    err = np.array([5.0, 4.0, 3.0, 2.0, 1.0])
    assert O.refine_fixed_fraction(err, 0.5).tolist() == [1, 1, 0, 0, 0]
    assert O.refine_fixed_number(err, 0.4).tolist() == [1, 1, 0, 0, 0]
    assert O.refine_fixed_fraction(err, 0.9).tolist() == [1, 1, 1, 1, 0]
    flag = O.refine_fixed_fraction(np.array([1.0, 9.0, 1.0]), 0.5)
    O.refine_fixed_fraction(np.array([9.0, 1.0, 1.0]), 0.5, flag)   # ORs like the MT XY/YX pair
    assert flag.tolist() == [1, 1, 0]


def test_oracle_solve_matches_direct_solution(small):
    m = small.mesh
    om = O.Mesh(m)
    rp, ci = O.sparsity(om)
    Cv, Mv, bdr = O.assemble(om, small.model, 1.0, rp, ci)
    bg = O.background_model(om, small.model)
    sr, si = O.rhs_mt(om, small.model, 1.0, -1, bg, bdr)
    er, ei, its, st = O.solve(om, rp, ci, Cv, Mv, sr, si, 1e-10, 200)
    A = sp.csr_matrix((Cv + 1j * Mv, ci, rp)).tocsc()
    z = sla.spsolve(A, sr - 1j * si)
    assert st[0] <= 1e-10
    assert np.abs((er + 1j * ei) - z).max() <= 1e-6 * np.abs(z).max()
    # Dirichlet rows hold the prescribed boundary values
    bd = m.edge_bdr.astype(bool)
    C = sp.csr_matrix((Cv, ci, rp))
    vals = (sr - 1j * si)[bd] / C.diagonal()[bd]
    assert np.allclose(z[bd], vals, rtol=1e-10, atol=1e-14 * np.abs(vals).max())


def _halfspace_response(n_tets):
    prob = mg.mt_halfspace_block(n_tets, with_block=False, freqs=(1.0,), name="hs")
    m = prob.mesh
    om = O.Mesh(m)
    rp, ci = O.sparsity(om)
    Cv, Mv, bdr = O.assemble(om, prob.model, 1.0, rp, ci)
    bg = O.background_model(om, prob.model)
    sr, si = O.rhs_mt(om, prob.model, 1.0, -1, bg, bdr)
    z = sla.spsolve(sp.csr_matrix((Cv + 1j * Mv, ci, rp)).tocsc(), sr - 1j * si)
    r = np.array([0.0, 0.0, 0.0])
    t = O.find_cell(om, r[None, :])[0]
    E, H = O.interpolate_fields(om, int(t), r, 1.0, z.real, z.imag)
    Z = E[0] / H[1]
    return abs(Z) ** 2 / (2 * np.pi * MU), abs(np.degrees(np.angle(Z)))


def test_halfspace_mt_response_converges_to_plane_wave():
    """100 ohm-m halfspace at 1 Hz: the FE apparent resistivity and phase at
    the surface approach 100 ohm-m and 45 degrees as the mesh is refined."""
    rho_c, ph_c = _halfspace_response(5000)
    rho_f, ph_f = _halfspace_response(60000)
    assert abs(rho_f - 100.0) < abs(rho_c - 100.0) and abs(ph_f - 45.0) < abs(ph_c - 45.0)
    assert abs(rho_f - 100.0) < 6.0 and abs(ph_f - 45.0) < 2.0


def test_estimator_properties(small):
    m = small.mesh
    om = O.Mesh(m)
    z = np.zeros(m.n_edges)
    eta = O.estimate(om, small.model, 1.0, [(z, z), (z, z)])
    assert np.all(eta == 0)
    rng = np.random.default_rng(3)
    u = (rng.standard_normal(m.n_edges), rng.standard_normal(m.n_edges))
    e1 = O.estimate(om, small.model, 1.0, [u, u])
    e2 = O.estimate(om, small.model, 1.0, [(2 * u[0], 2 * u[1]), u])
    assert np.all(e1 >= 0)
    assert np.allclose(e2[0], 4 * e1[0], rtol=1e-12)     # quadratic in the solution
    assert np.allclose(e2[1], e1[1], rtol=0, atol=0)
