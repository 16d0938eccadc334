"""Receiver responses (calculate_response_mt / calculate_response_csem,
src/em_fwd.cc:747-871) through the C ABI against the oracle's restatement,
and apparent resistivity / phase against the exact layered-earth plane wave.

Tolerances: the response formulas are a handful of complex products and one
division; library and oracle evaluate the same expressions in the same order,
so they agree to 1e-14 relative.  Against the analytic 1-D solution the
derived rho_a and phase (the reference's AP pair: log amplitude, radians)
agree to 1e-9 relative / 1e-9 degrees (the plane-wave fields carry no
discretisation error).
"""

import numpy as np
import pytest

import emfem_b200 as E
import oracle as O

MU = 4e-7 * np.pi
MT_TYPES = [E.api.Z_XX_RI, E.api.Z_XY_RI, E.api.Z_YX_RI, E.api.Z_YY_RI, E.api.T_ZX_RI, E.api.T_ZY_RI,
            E.api.R_XY_AP, E.api.R_YX_AP]
CSEM_TYPES = [111, 121, 131, 141, 151, 161, 112, 122, 132, 142, 152, 162]


def _cplx(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def test_mt_responses_match_oracle():
    rng = np.random.default_rng(7)
    nrx = 9
    fields = _cplx(rng, (nrx, 4, 3))
    ot = np.array([t for t in MT_TYPES for _ in range(nrx)], dtype=np.int32)
    ri = np.array([r for _ in MT_TYPES for r in range(nrx)], dtype=np.int32)
    got = E.calculate_response_mt(0.37, fields, ot, ri)
    for o in range(ot.size):
        ref = O.response_mt(0.37, fields[ri[o]], int(ot[o]))
        assert abs(got[o] - ref) <= 1e-14 * max(abs(ref), 1.0)


def test_csem_responses_match_oracle():
    rng = np.random.default_rng(8)
    nrx = 5
    fields = _cplx(rng, (nrx, 2, 3))
    ot = np.array([t for t in CSEM_TYPES for _ in range(nrx)], dtype=np.int32)
    ri = np.array([r for _ in CSEM_TYPES for r in range(nrx)], dtype=np.int32)
    got = E.calculate_response_csem(fields, ot, ri)
    for o in range(ot.size):
        ref = O.response_csem(fields[ri[o]], int(ot[o]))
        assert abs(got[o] - ref) <= 1e-14 * max(abs(ref), 1.0)


def test_refused_types_and_bad_indices():
    f = np.ones((1, 4, 3), dtype=np.complex128)
    for t in (312, 322, 111, 999):  # Z_*_AP and CSEM types are refused by the MT path, as in the reference
        with pytest.raises(E.EMGError) as ei:
            E.calculate_response_mt(1.0, f, [t], [0])
        assert ei.value.code == E.api.EMG_ERR_USER
        assert O.response_mt(1.0, f[0], t) is None
    with pytest.raises(E.EMGError) as ei:
        E.calculate_response_mt(1.0, f, [E.api.Z_XY_RI], [1])
    assert ei.value.code == E.api.EMG_ERR_ARG
    with pytest.raises(E.EMGError) as ei:
        E.calculate_response_csem(np.ones((1, 2, 3)), [321], [0])
    assert ei.value.code == E.api.EMG_ERR_USER


@pytest.mark.parametrize("rho,freq", [(100.0, 1.0), (10.0, 0.01), (1000.0, 30.0)])
def test_halfspace_apparent_resistivity_and_phase(rho, freq):
    # the reference's 1-D column: 100 km of air over a homogeneous earth
    eh = O.plane_wave([-100e3, 0.0], [1e-8, 1.0 / rho], freq, [0.0])[0]
    # fields at a surface receiver: XY polarisation E = (Ex, 0, 0), H = (0, Hy, 0);
    # YX polarisation E = (0, Ey, 0), H = (Hx, 0, 0)
    f = np.zeros((1, 4, 3), dtype=np.complex128)
    f[0, 0, 0], f[0, 1, 1], f[0, 2, 1], f[0, 3, 0] = eh[0], eh[1], eh[2], eh[3]
    r = E.calculate_response_mt(freq, f, [E.api.R_XY_AP, E.api.R_YX_AP, E.api.Z_XY_RI], [0, 0, 0])
    # the reference's AP pair: log(rho_a) and the phase in radians
    assert abs(np.exp(r[0].real) - rho) <= 1e-9 * rho and abs(np.exp(r[1].real) - rho) <= 1e-9 * rho
    assert abs(np.degrees(r[0].imag) - 45.0) <= 1e-9 and abs(np.degrees(r[1].imag) + 135.0) <= 1e-9
    assert abs(r[2] - eh[0] / eh[1]) <= 1e-14 * abs(r[2])


# ---------------------------------------------------------------------------
# point location (find_cell_around_point, src/em_mesh.cc:527-566)
# ---------------------------------------------------------------------------
def test_point_location_matches_oracle_walk():
    """The indexed walk returns the oracle's tet for every point: random
    interior points, receivers on the surface (z = 0 lies on mesh faces, where
    two tets contain the point and the walk order decides) and mesh vertices
    (shared by many tets); points outside the mesh give -1."""
    from emfem_b200 import meshgen as mg
    prob = mg.mt_halfspace_block(4000, freqs=(1.0,), name="loc")
    m = prob.mesh
    om = O.Mesh(m)
    rng = np.random.default_rng(11)
    lo, hi = m.points.min(axis=0), m.points.max(axis=0)
    inner = lo + (hi - lo) * rng.uniform(0.02, 0.98, (400, 3))
    surf = np.column_stack([rng.uniform(lo[0] * 0.5, hi[0] * 0.5, 60), rng.uniform(lo[1] * 0.5, hi[1] * 0.5, 60),
                            np.zeros(60)])
    verts = m.points[rng.choice(m.n_vertices, 60, replace=False)]
    pts = np.vstack([inner, surf, verts, prob.survey.rx])
    ix = E.PointIndex(m)
    got = ix.find(pts)
    ref = O.find_cell(om, pts)
    assert (ref >= 0).all()
    assert np.array_equal(got, ref)
    outside = np.array([[hi[0] * 2, 0.0, 0.0], [0.0, lo[1] * 3, 0.0]])
    assert (ix.find(outside) == -1).all()
    ix.close()


def test_host_chain_fields_and_mt_responses():
    """The receiver chain on a host-only context: fields at the receivers
    from a solution held on the host (emg_interpolate_fields_host) match the
    oracle's interpolate_fields to 1e-12, and the MT responses built from
    them match the oracle's response restatement applied to the oracle's
    fields to 1e-10.  (How close rho_a and phase come to the plane wave is a
    property of the mesh, pinned by the halfspace convergence test of the
    oracle.)"""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    from emfem_b200 import meshgen as mg
    prob = mg.mt_halfspace_block(8000, with_block=False, freqs=(1.0,), name="chain")
    m = prob.mesh
    om = O.Mesh(m)
    rp, ci = O.sparsity(om)
    Cv, Mv, bdr = O.assemble(om, prob.model, 1.0, rp, ci)
    A = sp.csr_matrix((Cv + 1j * Mv, ci, rp)).tocsc()
    obg = O.background_model(om, prob.model)
    sols = []
    for mode in (E.XY_POLAR, E.YX_POLAR):
        sr, si = O.rhs_mt(om, prob.model, 1.0, mode, obg, bdr)
        sols.append(sla.spsolve(A, sr - 1j * si))
    rx = np.array([[0.0, 0.0, 0.0], [500.0, -300.0, 0.0]])
    with E.EMContext(-1) as c:
        c.set_mesh(m)
        c.set_model(prob.model)
        c.set_frequencies([1.0])
        tets = c.find_cell_around_point(rx)
        fields = np.zeros((len(rx), 4, 3), dtype=np.complex128)
        for p, z in enumerate(sols):
            Eh, Hh = c.interpolate_fields_host(0, rx, tets, z.real, z.imag)
            for r in range(len(rx)):
                Eo, Ho = O.interpolate_fields(om, int(tets[r]), rx[r], 1.0, z.real, z.imag)
                assert np.abs(Eh[r] - Eo).max() <= 1e-12 * np.abs(Eo).max()
                assert np.abs(Hh[r] - Ho).max() <= 1e-12 * np.abs(Ho).max()
            fields[:, 2 * p, :], fields[:, 2 * p + 1, :] = Eh, Hh
    ofields = np.zeros_like(fields)
    for p, z in enumerate(sols):
        for r in range(len(rx)):
            ofields[r, 2 * p], ofields[r, 2 * p + 1] = O.interpolate_fields(om, int(tets[r]), rx[r], 1.0,
                                                                            z.real, z.imag)
    ot = [t for t in MT_TYPES for _ in range(len(rx))]
    ri = [r for _ in MT_TYPES for r in range(len(rx))]
    rsp = E.calculate_response_mt(1.0, fields, ot, ri)
    for o in range(len(ot)):
        ref = O.response_mt(1.0, ofields[ri[o]], ot[o])
        assert abs(rsp[o] - ref) <= 1e-10 * max(abs(ref), 1.0)
