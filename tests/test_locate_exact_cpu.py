"""The point-location predicate's sign is exact.

TetAccessor::contains_point (src/em_mesh.h:208-230) reads only the signs of
TetGen's robust orient3d, which are exact.  emg_orient3d_sign (and the
oracle's restatement, through its walk) must give the same sign as the exact
rational determinant det[a-d; b-d; c-d] of the double inputs (Python
fractions), bit for bit:
  * general random quadruples;
  * exactly coplanar quadruples whose products need ~100 bits (coordinates
    2^20 + k 2^-30, d = b + c - a): the sign is 0, where an evaluation in
    80-bit long double rounds to a nonzero value for some of them;
  * the same with d moved by one ulp in one coordinate: a determinant of the
    order of 1e-25 of its terms, sign +1 or -1;
and the point walks of the library and the oracle find the same tets for
points exactly on shared faces of a mesh.
"""

from fractions import Fraction

import numpy as np

import emfem_b200 as E
from emfem_b200 import meshgen as mg
import oracle as O


def _exact(a, b, c, d):
    F = [[Fraction(float(v)) for v in p] for p in (a, b, c, d)]
    r = [[F[i][k] - F[3][k] for k in range(3)] for i in range(3)]
    det = (r[0][0] * (r[1][1] * r[2][2] - r[1][2] * r[2][1]) - r[0][1] * (r[1][0] * r[2][2] - r[1][2] * r[2][0]) +
           r[0][2] * (r[1][0] * r[2][1] - r[1][1] * r[2][0]))
    return (det > 0) - (det < 0)


def _long_double(a, b, c, d):
    L = np.longdouble
    A, B, Cc, D = (np.array(p, dtype=L) for p in (a, b, c, d))
    ad, bd, cd = A - D, B - D, Cc - D
    det = (ad[0] * (bd[1] * cd[2] - bd[2] * cd[1]) + bd[0] * (cd[1] * ad[2] - cd[2] * ad[1]) +
           cd[0] * (ad[1] * bd[2] - ad[2] * bd[1]))
    return int(det > 0) - int(det < 0)


def test_random_quadruples():
    rng = np.random.default_rng(3)
    for _ in range(300):
        a, b, c, d = (rng.normal(size=3) * 10.0 ** rng.uniform(-2, 5) for _ in range(4))
        assert E.api.orient3d_sign(a, b, c, d) == _exact(a, b, c, d)


def test_coplanar_and_one_ulp_away():
    rng = np.random.default_rng(11)
    base = 2.0 ** 20
    ld_wrong = 0
    for _ in range(400):
        a, b, c = (base + rng.integers(-2 ** 22, 2 ** 22, size=3) * 2.0 ** -30 for _ in range(3))
        d = b + c - a  # exact: every value is a multiple of 2^-30 below 2^21
        assert np.all(d == (b - a) + c)
        assert _exact(a, b, c, d) == 0
        assert E.api.orient3d_sign(a, b, c, d) == 0
        ld_wrong += _long_double(a, b, c, d) != 0
        for k in range(3):
            for direction in (np.inf, -np.inf):
                e = d.copy()
                e[k] = np.nextafter(e[k], direction)
                s = _exact(a, b, c, e)
                assert s != 0 or np.all(b - a == 0)
                assert E.api.orient3d_sign(a, b, c, e) == s
    print("long double gave a nonzero sign for %d of 400 coplanar quadruples" % ld_wrong)


def test_walks_agree_on_face_points():
    prob = mg.mt_halfspace_block(900, freqs=(1.0,), name="loc-exact")
    m = prob.mesh
    rng = np.random.default_rng(5)
    pts = []
    # points on the faces of random tets: barycentric combinations with
    # dyadic weights (on the plane up to the rounding of the combination)
    # and the face vertices and edge midpoints themselves
    for t in rng.integers(0, m.n_tets, 60):
        v = m.points[m.tets[t]]
        for f in range(4):
            w = v[[i for i in range(4) if i != f]]
            pts.append(w[0])
            pts.append(0.5 * (w[0] + w[1]))
            pts.append(0.25 * w[0] + 0.25 * w[1] + 0.5 * w[2])
    pts = np.asarray(pts, dtype=np.float64)
    with E.EMContext(-1) as c:
        c.set_mesh(m)
        got = c.find_cell_around_point(pts)
    ref = O.find_cell(O.Mesh(m), pts)
    assert np.array_equal(got, ref)
    assert np.all(got >= 0)
