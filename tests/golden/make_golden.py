"""Generates the golden fixtures of tests/golden from independent derivations.

* whitney_elements.json -- curl-curl and mass element matrices of lowest-order
  Nedelec (Whitney) elements on a few tetrahedra, derived here from the
  barycentric integration rule  int_T l_a l_b = |T| (1 + delta_ab) / 20  and
  curl(l_a grad l_b - l_b grad l_a) = 2 grad l_a x grad l_b, with the edge
  orientation lower -> higher vertex id.  No quadrature is involved.
* plane_wave_layered.json -- surface impedance of layered earths (apparent
  resistivity and phase) from propagating (E, H) upward with the exact
  matrix exponential of dE/dz = i w mu H, dH/dz = -sigma E, starting from the
  decaying eigenvector of the basement.  This is a different route from the
  reflection-coefficient recursion of the plane-wave code under test.

    python tests/golden/make_golden.py
"""

import json
import os

import numpy as np
import scipy.linalg as sla
from scipy.spatial.transform import Rotation

HERE = os.path.dirname(os.path.abspath(__file__))
MU = 4e-7 * np.pi
EDGES = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]


def whitney(verts, ids, sigma):
    """Element matrices in the local edge order EDGES of the vertex ids sorted
    ascending; returns (C, Ms) with Ms the mass matrix without omega."""
    order = np.argsort(ids)
    x = np.asarray(verts, dtype=float)[order]
    J = np.vstack([np.ones(4), x.T])            # columns (1, x_i)
    Ji = np.linalg.inv(J)                      # rows: l_i = a + b x + c y + d z
    grad = Ji[:, 1:]
    vol = abs(np.linalg.det(J)) / 6.0
    S = grad @ sigma @ grad.T
    L = vol / 20.0 * (np.ones((4, 4)) + np.eye(4))
    C = np.zeros((6, 6))
    M = np.zeros((6, 6))
    for i, (a, b) in enumerate(EDGES):
        ci = 2 * np.cross(grad[a], grad[b])
        for j, (c, d) in enumerate(EDGES):
            cj = 2 * np.cross(grad[c], grad[d])
            C[i, j] = vol / MU * ci @ cj
            M[i, j] = L[a, c] * S[b, d] - L[a, d] * S[b, c] - L[b, c] * S[a, d] + L[b, d] * S[a, c]
    return C, M, [int(ids[o]) for o in order]


def surface_impedance(thick, sig, freq):
    """Z = E/H at the top of a stack of layers over a basement (sig[-1])."""
    w = 2 * np.pi * freq
    lam = -np.sqrt(-1j * w * MU * sig[-1])
    u = np.array([1.0 + 0j, lam / (1j * w * MU)])
    for h, s in zip(thick[::-1], sig[-2::-1]):
        A = np.array([[0, 1j * w * MU], [-s, 0]], dtype=complex)
        u = sla.expm(-A * h) @ u
    return u[0] / u[1]


def main():
    rng = np.random.default_rng(7)
    elems = []
    for k in range(4):
        verts = rng.uniform(-1e3, 1e3, size=(4, 3))
        ids = rng.choice(100, size=4, replace=False)
        if k == 0:
            verts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)
            ids = np.array([3, 7, 11, 20])
        # positive orientation in the order of ascending vertex id
        order = np.argsort(ids)
        xs = verts[order]
        if np.linalg.det(np.vstack([np.ones(4), xs.T])) < 0:
            verts[[order[2], order[3]]] = verts[[order[3], order[2]]]
        # conductivity of the Arbitrary anisotropy form: principal resistivities
        # rotated by Euler angles (degrees); R = Rz(-g) Ry(-b) Rx(-a) as active
        # rotations composed by scipy
        rho = rng.uniform(1, 100, size=3)
        ang = rng.uniform(-90, 90, size=3)
        R = Rotation.from_euler("ZYX", [-ang[2], -ang[1], -ang[0]], degrees=True).as_matrix()
        sigma = R @ np.diag(1 / rho) @ R.T
        C, M, sorted_ids = whitney(verts, ids, sigma)
        elems.append(dict(verts=verts.tolist(), ids=[int(i) for i in ids], rho=rho.tolist(), angles=ang.tolist(),
                          sigma=sigma.tolist(), sorted_ids=sorted_ids, C=C.tolist(), Ms=M.tolist()))
    with open(os.path.join(HERE, "whitney_elements.json"), "w") as f:
        json.dump(dict(edge_order=EDGES, elements=elems), f, indent=1)

    cases = []
    models = [([], [0.01]),                        # 100 ohm-m halfspace
              ([1000.0], [0.01, 1.0]),             # conductive basement
              ([500.0, 2000.0], [0.1, 0.001, 0.05])]
    for thick, sig in models:
        for freq in (0.001, 0.1, 10.0, 100.0):
            Z = surface_impedance(np.array(thick), np.array(sig), freq)
            w = 2 * np.pi * freq
            cases.append(dict(thickness=thick, sigma=sig, freq=freq, rho_a=abs(Z) ** 2 / (w * MU),
                              phase_deg=float(np.degrees(np.angle(Z)))))
    with open(os.path.join(HERE, "plane_wave_layered.json"), "w") as f:
        json.dump(dict(cases=cases), f, indent=1)


if __name__ == "__main__":
    main()
