"""C ABI checks that need no GPU: every declared symbol is exported, options
parsing (process_options, src/em_ctx.cc:100-175), host-side marking and
argument/state errors."""

import os
import re

import numpy as np
import pytest

import emfem_b200 as E
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "emfem_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(emg_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = E.lib()
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_options_parsing():
    with E.EMContext(-1) as c:
        c.process_options("""
            -iprefix model -oprefix out   # file prefixes
            -K_max_it 50 -e_rtol 1e-9 -dual_rtol 1e-7
            -inner_pc_type ams -pc_threshold 1000 -refine_strategy fixed_number
            -A_ksp_gmres_restart 20 -B_ksp_rtol 0.05 -B_ksp_max_it 40
            -B_pc_hypre_ams_cycle_type 11 -A_ksp_monitor_true_residual
            -emg_inner_precision fp32 -save_mesh 0
        """)
        assert c.get_option("K_max_it") == 50
        assert c.get_option("e_rtol") == 1e-9
        assert c.get_option("dual_rtol") == 1e-7
        assert c.get_option("inner_pc_type") == 1
        assert c.get_option("refine_strategy") == 0
        assert c.get_option("A_ksp_gmres_restart") == 20
        assert c.get_option("B_ksp_rtol") == 0.05
        assert c.get_option("emg_inner_precision") == 1
        assert c.get_option("save_mesh") == 0
        for bad in ("-bogus 1", "-K_max_it abc", "-inner_pc_type lu", "-A_ksp_gmres_restart 999",
                    "-B_pc_hypre_ams_cycle_type 2", "stray"):
            with pytest.raises(E.EMGError) as ei:
                c.process_options(bad)
            assert ei.value.code == E.api.EMG_ERR_OPTION
        # defaults of process_options are kept for untouched keys
        assert c.get_option("refine_fraction") == 0.1


def test_solver_extension_options():
    """emg_* keys of the batched path and the AMS variants: defaults, round
    trip, and rejection of out-of-range values."""
    with E.EMContext(-1) as c:
        defaults = {"emg_block_inner_max_it": 30, "emg_block_inner_rtol": 1e-2, "emg_block_fcg_mmax": 2,
                    "emg_pi_coupled": 0, "emg_fused_vcycle": 0, "emg_spmm_tiled": 0, "emg_tiled_smem_kb": 64,
                    "emg_graphs": 1, "emg_inner_precision": 0}
        for k, v in defaults.items():
            assert c.get_option(k) == v, k
        c.process_options("-emg_block_inner_max_it 45 -emg_block_inner_rtol 0.05 -emg_block_fcg_mmax 3 "
                          "-emg_pi_coupled 1 -emg_fused_vcycle -emg_fused_rows 5000 -emg_fused_blocks_per_sm 2 "
                          "-emg_spmm_tiled 1 -emg_tiled_smem_kb 32 -B_pc_hypre_ams_cycle_type 7")
        got = {k: c.get_option(k) for k in ("emg_block_inner_max_it", "emg_block_inner_rtol", "emg_block_fcg_mmax",
                                            "emg_pi_coupled", "emg_fused_vcycle", "emg_fused_rows",
                                            "emg_fused_blocks_per_sm", "emg_spmm_tiled", "emg_tiled_smem_kb")}
        assert got == {"emg_block_inner_max_it": 45, "emg_block_inner_rtol": 0.05, "emg_block_fcg_mmax": 3,
                       "emg_pi_coupled": 1, "emg_fused_vcycle": 1, "emg_fused_rows": 5000,
                       "emg_fused_blocks_per_sm": 2, "emg_spmm_tiled": 1, "emg_tiled_smem_kb": 32}
        for ct in (1, 3, 5, 7, 11, 13):
            c.process_options("-B_pc_hypre_ams_cycle_type %d" % ct)
        assert c.get_option("emg_restrict_smooth") == 1
        c.process_options("-emg_restrict_smooth 0")
        assert c.get_option("emg_restrict_smooth") == 0
        c.process_options("-emg_cheb_degree 3 -emg_block_cheb_degree 4 -emg_amg_cheb_degree 6")
        assert [c.get_option(k) for k in ("emg_cheb_degree", "emg_block_cheb_degree", "emg_amg_cheb_degree")] == \
            [3, 4, 6]
        for bad in ("-emg_block_inner_max_it 0", "-emg_block_inner_rtol 0", "-emg_block_fcg_mmax 31",
                    "-emg_tiled_smem_kb 300", "-B_pc_hypre_ams_cycle_type 14", "-emg_cheb_degree 1",
                    "-emg_block_cheb_degree 7", "-emg_amg_cheb_degree 0"):
            with pytest.raises(E.EMGError) as ei:
                c.process_options(bad)
            assert ei.value.code == E.api.EMG_ERR_OPTION


def test_host_only_context_refuses_device_work():
    with E.EMContext(-1) as c:
        from emfem_b200 import meshgen as mg
        prob = mg.mt_halfspace_block(800, freqs=(1.0,))
        c.set_mesh(prob.mesh)      # host arrays only
        for call in (lambda: c.create_linear_system(-3), lambda: c.assemble_matrix(0)):
            with pytest.raises(E.EMGError) as ei:
                call()
            assert ei.value.code == E.api.EMG_ERR_STATE


def test_host_only_context_rhs_and_location():
    """A context without a GPU (device -1) holds the mesh on the host and
    serves the host-side entry points: CSEM and dual right-hand sides
    (assemble_rhs_csem / assemble_rhs_dual, src/em_fwd.cc:582-717) against
    the oracle to 1e-12 of the largest entry, and point location on the
    context's mesh against the oracle's walk (identical tets)."""
    from emfem_b200 import meshgen as mg
    prob = mg.marine_csem(3000, freqs=(0.25, 1.25), name="csem-host")
    om = O.Mesh(prob.mesh)
    with E.EMContext(-1) as c:
        c.set_mesh(prob.mesh)
        c.set_model(prob.model)
        c.set_frequencies(prob.survey.freqs)
        rx = prob.survey.rx
        tets = c.find_cell_around_point(rx)
        assert np.array_equal(tets, O.find_cell(om, rx)) and (tets >= 0).all()
        sr, si = c.assemble_rhs_dual(rx, tets)
        osr, osi = O.rhs_dual(om, rx)
        assert np.abs(sr - osr).max() <= 1e-12 * np.abs(osr).max()
        assert np.abs(si - osi).max() <= 1e-12 * np.abs(osi).max()
        point = np.array(prob.survey.tx[0], dtype=np.float64)
        line = point.copy()
        line[3], line[6] = 30.0, 250.0  # a 250 m line source at azimuth 30 degrees
        for tx, (fidx, f) in ((point, (0, prob.survey.freqs[0])), (line, (1, prob.survey.freqs[1]))):
            if abs(tx[6]) <= 0.1:
                pts = tx[None, :3]
            else:  # the line source split into n_tx_divisions dipoles (default 20)
                d = np.array([np.cos(np.radians(tx[3])) * np.cos(np.radians(tx[4])),
                              np.sin(np.radians(tx[3])) * np.cos(np.radians(tx[4])), np.sin(np.radians(tx[4]))])
                a = tx[:3] - d * tx[6] / 2
                pts = np.array([a + d * tx[6] / 20 * (i + 0.5) for i in range(20)])
            dt = c.find_cell_around_point(pts)
            sr, si = c.assemble_rhs_csem(fidx, tx, dt)
            osr, osi = O.rhs_csem(om, f, tx)
            assert np.abs(sr).max() == 0.0
            assert np.abs(si - osi).max() <= 1e-12 * np.abs(osi).max()


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_refine_marking_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    err = rng.lognormal(size=5000)
    err[rng.integers(0, 5000, 50)] = err[0]            # ties
    for frac in (0.05, 0.1, 0.3):
        assert np.array_equal(E.refine_fixed_fraction(err, frac), O.refine_fixed_fraction(err, frac))
        assert np.array_equal(E.refine_fixed_number(err, frac), O.refine_fixed_number(err, frac))
    with pytest.raises(E.EMGError):
        E.refine_fixed_number(err, 1.5)


C_CLIENT = r"""
#include <stdio.h>
#include "emfem_b200.h"
/* two tets sharing the face (1,2,3): (0,1,2,3) and (4,1,3,2) */
static const double pts[15] = {0,0,0, 1,0,0, 0,1,0, 0,0,1, 1,1,1};
static const int tets[8] = {0,1,2,3, 4,1,3,2};
static const int nbr[8] = {-1,-1,-1,1, -1,-1,-1,0};
int main(int argc, char **argv) {
  const double q[9] = {0.1,0.1,0.1, 0.6,0.6,0.6, 5,5,5};
  int t[3] = {-9,-9,-9};
  emg_point_index *ix = emg_point_index_create(5, pts, 2, tets, nbr);
  if (!ix || emg_point_index_find(ix, 3, q, t) != EMG_OK) return 1;
  emg_point_index_destroy(ix);
  emg_survey *s = emg_survey_read_emd(argv[1]);
  if (!s) { printf("%s\n", emg_last_error()); return 2; }
  int nf, ntx, nrx, nobs;
  emg_survey_sizes(s, &nf, &ntx, &nrx, &nobs);
  int ot[4], ri[4];
  emg_survey_get(s, 0, 0, 0, ot, 0, 0, ri, 0, 0);
  double f[24] = {0}, rsp[8];
  f[0] = 1.0; f[8] = 1.0; f[14] = 2.0; f[18] = -1.0;  /* Ex, Hy (XY), Ey, Hx (YX) */
  if (emg_calculate_response_mt(1.0, nrx, f, nobs, ot, ri, rsp) != EMG_OK) return 3;
  if (emg_survey_write_rsp(s, argv[2], rsp) != EMG_OK) return 4;
  emg_survey_destroy(s);
  printf("%d %d %d %d %d %.6f %.6f\n", t[0], t[1], t[2], nobs, ot[0], rsp[0], rsp[2]);
  return 0;
}
"""


def test_c_client_uses_the_abi(tmp_path):
    """A plain C99 program compiled against include/emfem_b200.h and linked to
    the library uses the host-only entry points (point location, survey files,
    responses) without a GPU."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "client.c"
    src.write_text(C_CLIENT)
    exe = tmp_path / "client"
    libdir = os.path.dirname(E.library_path())
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(root, "include"), str(src),
                    "-L", libdir, "-lemfem_b200", "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    emd = tmp_path / "s.emd"
    emd.write_text("1\n1.0\n0\n1\n0 0 0\n2\n321 0 -3 0 1 0 0.1 0.1\n331 0 -3 0 1 0 0.1 0.1\n")
    out = subprocess.run([str(exe), str(emd), str(tmp_path / "s.rsp")], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    t0, t1, t2, nobs, ot0, z_xy, z_yx = out.stdout.split()
    assert (int(t0), int(t1), int(t2)) == (0, 1, -1)
    assert int(nobs) == 2 and int(ot0) == 321
    # 1-D fields: Z_XY = Ex / Hy = 1, Z_YX = Ey / Hx = -2
    assert float(z_xy) == 1.0 and float(z_yx) == -2.0
    assert (tmp_path / "s.rsp").read_text().startswith("# frequencies\n1\n")
