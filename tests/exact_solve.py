"""Exact discrete solutions for the accuracy tests: a sparse direct solve of
(C + i M) e = s_re - i s_im in FP64 (the system solve_linear_system solves in
its real form, src/em_la.cc:35-87), one factorisation per frequency.

The factorisations run in worker processes started with the 'spawn' method
(they hold the GIL and take tens of seconds on config-sized meshes).
"""

import multiprocessing as mp
from concurrent.futures import ProcessPoolExecutor

import numpy as np


def _factor_solve(args):
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    rp, ci, cv, mv, rhs = args
    A = sp.csr_matrix((cv + 1j * mv, ci, rp)).tocsc()
    lu = sla.splu(A, permc_spec="MMD_AT_PLUS_A", options=dict(SymmetricMode=True))
    return np.stack([lu.solve(np.ascontiguousarray(rhs[:, j])) for j in range(rhs.shape[1])], axis=1)


def exact_solutions(jobs):
    """jobs: list of (rp, ci, C, M, rhs (n, m) complex = s_re - i s_im); returns
    the solutions (n, m) per job."""
    ctx = mp.get_context("spawn")
    with ProcessPoolExecutor(max_workers=min(len(jobs), 4), mp_context=ctx) as ex:
        return list(ex.map(_factor_solve, jobs))
