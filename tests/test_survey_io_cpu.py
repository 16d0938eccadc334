"""Survey files in the reference's layout: the .emd reader (read_emd,
src/em_io.cc:202-287) and the .rsp writer (save_rsp, src/em_io.cc:316-399).

The expected values restate the reference's rules in Python: '#' starts a
comment, lines are trimmed, tokens are whitespace separated; AP observations
are kept as (log amplitude, phase in radians) with errors ((err/100)^2,
(err in radians)^2); RI observations as (re, im) with squared errors.  The
.rsp text is compared character for character with the reference's printf
formats applied in Python (C and Python share the % conversions used).
"""

import math

import numpy as np
import pytest

import emfem_b200 as E

EMD = """# frequencies
2
 0.1   # low
10.0
# transmitters: x y z azimuth dip current length
1
\t0 0 -50   0  0 1 250
# receivers
3
 -1000 0 0
 0 0 0   # centre
 1000.5 0 -0.25

# observations
5
# otype fidx tidx ridx re im err_re err_im
 212 0 -3 0   100.0   45.0   5.0  1.5
 222 1 -3 2   12.5  -135.0  10.0  2.0
 321 0 -3 1   1e-3  -2e-3   1e-5  2e-5
 111 1  0 2   3.5e-9 -1.25e-9 1e-10 1e-10
 142 0  0 0   7.5e-7  30.0   2.0  1.0
"""


def _fmt_rows(rsp, otype, fidx, tidx, ridx, obs):
    ap = {212, 222, 112, 122, 132, 142, 152, 162}
    out = []
    for i in range(len(otype)):
        if otype[i] in ap:
            o = (math.exp(obs[i].real), obs[i].imag * 180.0 / math.pi)
            r = (math.exp(rsp[i].real), rsp[i].imag * 180.0 / math.pi)
            out.append("% 7d % 6d % 5d % 7d % 13.6E % 13.3f % 13.6E % 13.3f\n" % (otype[i], fidx[i], tidx[i], ridx[i],
                                                                              o[0], o[1], r[0], r[1]))
        else:
            out.append("% 7d % 6d % 5d % 7d % 13.6E % 13.6E % 13.6E % 13.6E\n" % (
                otype[i], fidx[i], tidx[i], ridx[i], obs[i].real, obs[i].imag, rsp[i].real, rsp[i].imag))
    return out


def test_read_emd_and_write_rsp(tmp_path):
    p = tmp_path / "survey.emd"
    p.write_text(EMD)
    s = E.Survey(str(p))
    assert np.array_equal(s.freqs, [0.1, 10.0])
    assert np.array_equal(s.tx, [[0, 0, -50, 0, 0, 1, 250]])
    assert np.array_equal(s.rx, [[-1000, 0, 0], [0, 0, 0], [1000.5, 0, -0.25]])
    assert list(s.otype) == [212, 222, 321, 111, 142]
    assert list(s.fidx) == [0, 1, 0, 1, 0] and list(s.tidx) == [-3, -3, -3, 0, 0]
    assert list(s.ridx) == [0, 2, 1, 2, 0]
    d = math.pi / 180.0
    want_obs = [complex(math.log(100.0), 45.0 * d), complex(math.log(12.5), -135.0 * d), complex(1e-3, -2e-3),
                complex(3.5e-9, -1.25e-9), complex(math.log(7.5e-7), 30.0 * d)]
    want_err = [complex((5.0 / 100) ** 2, (1.5 * d) ** 2), complex((10.0 / 100) ** 2, (2.0 * d) ** 2),
                complex(1e-5 ** 2, 2e-5 ** 2), complex(1e-10 ** 2, 1e-10 ** 2),
                complex((2.0 / 100) ** 2, (1.0 * d) ** 2)]
    assert np.array_equal(s.obs, np.array(want_obs))
    assert np.allclose(s.obserr, np.array(want_err), rtol=1e-15, atol=0)

    rsp = s.obs * (1.0 + 0.01j)
    out = tmp_path / "survey.rsp"
    s.write_rsp(str(out), rsp)
    text = out.read_text().splitlines(keepends=True)
    want = ["# frequencies\n", "2\n", "%.4E\n" % 0.1, "%.4E\n" % 10.0, "# transmiters\n", "1\n",
            "".join("% .4E " % v for v in s.tx[0]) + "\n", "# recievers\n", "3\n"]
    want += ["% .4E % .4E % .4E\n" % tuple(r) for r in s.rx]
    want += ["# observations\n", "5\n",
             "#%6s %6s %5s %7s %13s %13s %13s %13s\n" % ("otype", "fidx", "tidx", "ridx", "amp", "phase", "amp`",
                                                        "phase`")]
    want += _fmt_rows(rsp, s.otype, s.fidx, s.tidx, s.ridx, s.obs)
    assert text == want
    s.close()


def test_emd_errors(tmp_path):
    with pytest.raises(E.EMGError) as ei:
        E.Survey(str(tmp_path / "missing.emd"))
    assert ei.value.code == E.api.EMG_ERR_USER and "Unable to open" in str(ei.value)
    p = tmp_path / "short.emd"
    p.write_text("2\n0.1 1.0\n1\n0 0 0 0 0 1\n")  # six of the seven transmitter values
    with pytest.raises(E.EMGError) as ei:
        E.Survey(str(p))
    assert ei.value.code == E.api.EMG_ERR_USER and "transmitters" in str(ei.value)


def test_survey_responses_round_trip(tmp_path):
    """MT responses of a halfspace written against their own observations:
    the .rsp amplitude and phase columns carry rho_a and degrees."""
    import oracle as O
    p = tmp_path / "hs.emd"
    p.write_text("1\n1.0\n0\n1\n0 0 0\n2\n212 0 -3 0 100 45 5 1\n222 0 -3 0 100 -135 5 1\n")
    s = E.Survey(str(p))
    eh = O.plane_wave([-100e3, 0.0], [1e-8, 0.01], 1.0, [0.0])[0]
    f = np.zeros((1, 4, 3), dtype=np.complex128)
    f[0, 0, 0], f[0, 1, 1], f[0, 2, 1], f[0, 3, 0] = eh[0], eh[1], eh[2], eh[3]
    rsp = E.calculate_response_mt(1.0, f, s.otype, s.ridx)
    assert np.allclose(rsp, s.obs, rtol=0, atol=1e-12)
    out = tmp_path / "hs.rsp"
    s.write_rsp(str(out), rsp)
    rows = [l.split() for l in out.read_text().splitlines()[-2:]]
    assert [float(v) for v in rows[0][4:]] == [100.0, 45.0, 100.0, 45.0]
    assert [float(v) for v in rows[1][4:]] == [100.0, -135.0, 100.0, -135.0]


def test_save_vtk_layout(tmp_path):
    """Mesh::save_vtk (src/em_mesh.cc:183-248) on a host-only context: the
    text equals the reference's printf formats applied in Python, with the
    caller's arrays after subdomain and tet_attr in name order."""
    from emfem_b200 import meshgen as mg
    prob = mg.mt_halfspace_block(300, freqs=(1.0,), name="vtk")
    m = prob.mesh
    rng = np.random.default_rng(4)
    err_xy, rho = rng.random(m.n_tets), rng.random(m.n_tets) * 100
    out = tmp_path / "m.vtk"
    with E.EMContext(-1) as c:
        c.set_mesh(m)
        c.save_vtk(str(out), {"rho": rho, "error_xy": err_xy})
    want = ["# vtk DataFile Version 2.0\n", "Unstructured Grid\n", "ASCII\n", "DATASET UNSTRUCTURED_GRID\n",
            "POINTS %d double\n" % m.n_vertices]
    want += ["%.17g %.17g %.17g\n" % tuple(p) for p in m.points]
    want += ["\n", "CELLS %d %d\n" % (m.n_tets, 5 * m.n_tets)]
    want += ["%d" % 4 + "".join(" %4d" % v for v in t) + "\n" for t in m.tets]
    want += ["\n", "CELL_TYPES %d\n" % m.n_tets] + ["10\n"] * m.n_tets + ["\n", "CELL_DATA %d\n" % m.n_tets]
    for name, vals in (("subdomain", np.zeros(m.n_tets)), ("tet_attr", np.asarray(m.attr, dtype=float)),
                       ("error_xy", err_xy), ("rho", rho)):
        want += ["SCALARS %s double 1\n" % name, "LOOKUP_TABLE default\n"]
        want += ["%.15g\n" % v for v in vals] + ["\n"]
    assert out.read_text().splitlines(keepends=True) == want


def test_edge_cases_of_the_host_entry_points(tmp_path):
    """Empty and malformed inputs: zero observations and zero receivers are
    valid; bad array names, wrong lengths, unwritable paths and calls before
    a mesh fail with the documented status instead of writing garbage."""
    p = tmp_path / "empty.emd"
    p.write_text("0\n0\n0\n0\n")
    s = E.Survey(str(p))
    assert s.freqs.size == 0 and s.tx.shape == (0, 7) and s.rx.shape == (0, 3) and s.obs.size == 0
    s.write_rsp(str(tmp_path / "empty.rsp"), np.zeros(0, dtype=np.complex128))
    assert (tmp_path / "empty.rsp").read_text().splitlines()[-2:] == ["0", "#%6s %6s %5s %7s %13s %13s %13s %13s" % (
        "otype", "fidx", "tidx", "ridx", "amp", "phase", "amp`", "phase`")]
    with pytest.raises(E.EMGError) as ei:
        s.write_rsp(str(tmp_path / "no_such_dir" / "x.rsp"), np.zeros(0, dtype=np.complex128))
    assert ei.value.code == E.api.EMG_ERR_USER
    assert E.calculate_response_mt(1.0, np.zeros((0, 4, 3)), [], []).size == 0
    with pytest.raises(E.EMGError) as ei:
        E.calculate_response_mt(0.0, np.ones((1, 4, 3)), [E.api.Z_XY_RI], [0])
    assert ei.value.code == E.api.EMG_ERR_ARG
    from emfem_b200 import meshgen as mg
    prob = mg.mt_halfspace_block(300, freqs=(1.0,), name="edge")
    with E.EMContext(-1) as c:
        with pytest.raises(E.EMGError) as ei:
            c.save_vtk(str(tmp_path / "a.vtk"))
        assert ei.value.code == E.api.EMG_ERR_STATE
        with pytest.raises(E.EMGError) as ei:
            c.find_cell_around_point(np.zeros((1, 3)))
        assert ei.value.code == E.api.EMG_ERR_STATE
        c.set_mesh(prob.mesh)
        with pytest.raises(E.EMGError) as ei:
            c.save_vtk(str(tmp_path / "a.vtk"), {"two words": np.zeros(prob.mesh.n_tets)})
        assert ei.value.code == E.api.EMG_ERR_ARG
        with pytest.raises(E.EMGError):
            c.save_vtk(str(tmp_path / "a.vtk"), {"short": np.zeros(3)})
        c.save_vtk(str(tmp_path / "a.vtk"))  # mesh only: subdomain and tet_attr
        text = (tmp_path / "a.vtk").read_text()
        assert "SCALARS tet_attr double 1" in text and text.count("SCALARS") == 2
