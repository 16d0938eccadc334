"""The reference-facing drop-in: the replacement bodies of em_la.cc/em_fwd.cc
(tests/dropin/em_dropin.cc, the reference's own signatures over PETSc
Mat/Vec/PC handles) compiled with g++ against a PETSc stand-in
(tests/dropin/petsc.h) and the C ABI header, linked with libemfem_b200.so and
driven the way forward_csem calls them (tests/dropin/main.cc).

CPU: a host-only context -- CSEM and dual right-hand sides and marking through
the PETSc-shaped bodies equal the C ABI's own results exactly, and every
device entry point fails through SETERRQ with EM_ERR_USER.
GPU: the whole sequence -- system, assembly, preconditioner, primal and dual
solves, MatShell and PCShell callbacks on VecNest blocks, error estimate --
checked against the residual bar and the library's direct results.
"""

import os
import subprocess

import numpy as np
import pytest

import emfem_b200 as E
from emfem_b200 import meshgen as mg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "tests", "dropin")


def _build(tmp):
    exe = os.path.join(tmp, "dropin")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", DROPIN, "-I", os.path.join(ROOT, "include"),
           os.path.join(DROPIN, "em_dropin.cc"), os.path.join(DROPIN, "main.cc"),
           "-L", os.path.join(ROOT, "emfem_b200"), "-lemfem_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "emfem_b200"), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def _write(tmp, prob):
    m = prob.mesh
    rho = np.ascontiguousarray(prob.model.rho, dtype=np.float64)
    with open(os.path.join(tmp, "meta.txt"), "w") as f:
        f.write("%d %d %d %d %d %d %d %d\n" % (m.n_vertices, m.n_tets, m.n_edges, rho.shape[0], rho.shape[1],
                                               prob.model.aniso_form, len(prob.survey.freqs), len(prob.survey.rx)))
    for name, a, dt in (("pts", m.points, np.float64), ("tets", m.tets, np.int32), ("attr", m.attr, np.int32),
                        ("edges", m.edges, np.int32), ("t2e", m.tet2edge, np.int32), ("nbr", m.neighbors, np.int32),
                        ("non", m.tet_non, np.int32), ("ebdr", m.edge_bdr, np.uint8), ("rho", rho, np.float64),
                        ("freqs", prob.survey.freqs, np.float64), ("tx", prob.survey.tx[0], np.float64),
                        ("rx", prob.survey.rx, np.float64)):
        np.ascontiguousarray(a, dtype=dt).tofile(os.path.join(tmp, name))


def _read(tmp, name, dt=np.float64):
    return np.fromfile(os.path.join(tmp, name), dtype=dt)


def _host_ref(prob, ctx):
    loc = mg.PointLocator(prob.mesh)
    tx = prob.survey.tx[0]
    sr, si = ctx.assemble_rhs_csem(0, tx, loc.locate_all(tx[None, :3]))
    dr, di = ctx.assemble_rhs_dual(prob.survey.rx, loc.locate_all(prob.survey.rx))
    return np.concatenate([sr, si]), np.concatenate([dr, di])


@pytest.fixture(scope="module")
def problem():
    return mg.marine_csem(3000, freqs=(0.5,), name="dropin")


def test_dropin_host_only(problem, tmp_path):
    tmp = str(tmp_path)
    exe = _build(tmp)
    _write(tmp, problem)
    r = subprocess.run([exe, tmp, "-1"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "host-only: -1 -1 -1" in r.stdout
    with E.EMContext(-1) as c:
        c.set_mesh(problem.mesh)
        c.set_model(problem.model)
        c.set_frequencies(problem.survey.freqs)
        csem, dual = _host_ref(problem, c)
    assert np.array_equal(_read(tmp, "out_csem_rhs"), csem)
    assert np.array_equal(_read(tmp, "out_dual_rhs"), dual)
    nt = problem.mesh.n_tets
    flags = _read(tmp, "out_flags", np.uint8).reshape(2, nt)
    t = np.arange(nt)
    err = np.abs(np.sin(0.37 * t)) + 1e-3 * (t % 7)
    assert np.array_equal(flags[0], E.refine_fixed_fraction(err, 0.2))
    assert np.array_equal(flags[1], E.refine_fixed_number(err, 0.2))


@pytest.mark.gpu
def test_dropin_device_sequence(problem, tmp_path):
    tmp = str(tmp_path)
    exe = _build(tmp)
    _write(tmp, problem)
    r = subprocess.run([exe, tmp, "0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    ne, nt = problem.mesh.n_edges, problem.mesh.n_tets
    e = _read(tmp, "out_csem_e")
    s = _read(tmp, "out_csem_rhs")
    Ae = _read(tmp, "out_Ae")
    # MatShell callback on the solution reproduces the right-hand side to the solve tolerance
    assert np.linalg.norm(Ae - s) <= 1e-8 * np.linalg.norm(s) * (1 + 1e-6)
    # the same sequence through the library directly gives the same solution and indicators
    with E.EMContext(0) as c:
        c.set_mesh(problem.mesh)
        c.set_model(problem.model)
        c.set_frequencies(problem.survey.freqs)
        c.create_linear_system(0)
        c.assemble_matrix(0)
        c.create_pc()
        csem, dual = _host_ref(problem, c)
        c.solve_linear_system(E.SOL_CSEM, csem[:ne], csem[ne:], 100, 1e-8)
        er, ei = c.get_solution(E.SOL_CSEM)
        c.solve_linear_system(E.SOL_DUAL, dual[:ne], dual[ne:], 100, 1e-6)
        err, _ = c.estimate_error(0, 0)
        x = c.pc_apply_b(csem)
    z = er + 1j * ei
    zd = e[:ne] + 1j * e[ne:]
    # two processes: the Krylov reductions use atomics, so the solves agree to
    # the solve accuracy, not bit for bit
    assert np.abs(zd - z).max() <= 1e-6 * np.abs(z).max()
    assert np.abs(_read(tmp, "out_csem_error") - err[0]).max() <= 1e-6 * np.abs(err[0]).max()
    # pc_apply_b is an FCG solve stopped at 1e-2: rounding differences of the
    # two processes' reductions move its iterate by more than the outer solve's
    assert np.abs(_read(tmp, "out_pc_s") - x).max() <= 1e-4 * np.abs(x).max()
