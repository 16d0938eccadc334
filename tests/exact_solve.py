"""Exact discrete solutions for the accuracy tests: a sparse direct solve of
(C + i M) e = s_re - i s_im in FP64 (the system solve_linear_system solves in
its real form, src/em_la.cc:35-87), one factorisation per frequency, run one
after another in this process (about 25 s each on configuration 0).
"""

import numpy as np


def _factor_solve(rp, ci, cv, mv, rhs):
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    A = sp.csr_matrix((cv + 1j * mv, ci, rp)).tocsc()
    lu = sla.splu(A, permc_spec="MMD_AT_PLUS_A", options=dict(SymmetricMode=True))
    return np.stack([lu.solve(np.ascontiguousarray(rhs[:, j])) for j in range(rhs.shape[1])], axis=1)


def exact_solutions(jobs):
    """jobs: list of (rp, ci, C, M, rhs (n, m) complex = s_re - i s_im); returns
    the solutions (n, m) per job."""
    return [_factor_solve(*job) for job in jobs]
