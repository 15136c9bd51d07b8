"""The reference program's file formats (csrc/mfcfd_io.cpp through the C ABI).

Readers: 3d_input_data (point_preprocessor.f90:25-36) and stored-solution.dat
(initial_conditions.f90:18-29) under Fortran list-directed input rules.
Writers: residue.dat (q_lskum.f90:31) and the files of print_primal_output
(post_processor.f90:13-44) in gfortran's list-directed layout, whose 17
significant digits read back exactly.
"""
import os

import numpy as np
import pytest

FIELDS = ("status", "x", "y", "z", "tan1", "tan2", "nor", "nbhs", "conn", "min_dist")


def _same_cloud(a, b):
    for f in FIELDS:
        x, y = np.asarray(getattr(a, f)), np.asarray(getattr(b, f))
        assert np.array_equal(x, y.astype(x.dtype)), f


def test_read_input_point_data_round_trip(mfcfd_lib, small_cloud, tmp_path):
    from mfcfd import io
    from oracle import ref_translated
    p = tmp_path / "3d_input_data"
    p.write_text(ref_translated.input_text(small_cloud))
    assert io.count_input_points(str(p)) == small_cloud.n
    _same_cloud(io.read_input_point_data(str(p)), small_cloud)
    part = io.read_input_point_data(str(p), 100)       # max_points below the file's count
    assert part.n == 100 and np.array_equal(part.x, small_cloud.x[:100])


def test_list_directed_forms(mfcfd_lib, tmp_path):
    """Records spanning lines, commas, D and bare-signed exponents, repeat
    counts, CRLF, and values past the item list (discarded)."""
    from mfcfd import io
    text = ("1 1, 0.5D0 -1.0 +2.5e0 3*0.0\r\n"
            "1.0 0.0 0.0   0.0 1.0 0.0\r\n"
            " 2 2 1 1.5-3 trailing junk ignored\n"
            "2 0 1.0 2.0 3.0 1 0 0 0 1 0 0 0 1 3 1 2 1 0.25 99 98\n")
    p = tmp_path / "3d_input_data"
    p.write_text(text)
    assert io.count_input_points(str(p)) == 2
    c = io.read_input_point_data(str(p))
    assert list(c.status) == [1, 0]
    assert c.x[0] == 0.5 and c.y[0] == -1.0 and c.z[0] == 2.5
    assert list(c.tan1[0]) == [0.0, 0.0, 0.0] and list(c.tan2[0]) == [1.0, 0.0, 0.0]
    assert list(c.nor[0]) == [0.0, 1.0, 0.0]
    assert c.nbhs[0] == 2 and list(c.conn[0, :3]) == [2, 1, 0]
    assert c.min_dist[0] == 1.5e-3
    assert list(c.conn[1, :4]) == [1, 2, 1, 0] and c.min_dist[1] == 0.25


@pytest.mark.parametrize("text,what", [
    ("1 1 0.5 0.5\n", "end of file"),
    ("1 1.5 0 0 0 1 0 0 0 1 0 0 0 1 0 0.1\n", "bad integer"),
    ("1 1 0 0 0 1 0 0 0 1 0 0 0 1 28 0.1\n", "nbhs"),
    ("1 1 0 0 0 1 0 0 0 1 0 0 0 1 ,, 0.1\n", "null value"),
    ("1 1 0 0 0 1 0 0 0 1 0 0 0 1 0 x1\n", "bad real"),
])
def test_malformed_input_reports_io_error(mfcfd_lib, tmp_path, text, what):
    from mfcfd import io
    from mfcfd._lib import MfcfdError
    p = tmp_path / "3d_input_data"
    p.write_text(text)
    with pytest.raises(MfcfdError) as e:
        io.read_input_point_data(str(p), 1)
    assert e.value.code == 9 and what in str(e.value)


def test_missing_file(mfcfd_lib, tmp_path):
    from mfcfd import io
    from mfcfd._lib import MfcfdError
    with pytest.raises(MfcfdError) as e:
        io.read_stored_solution(str(tmp_path / "stored-solution.dat"), 3)
    assert e.value.code == 9 and "cannot open" in str(e.value)


def test_stored_solution_round_trip(mfcfd_lib, small_cloud, tmp_path):
    from mfcfd import cloud, io
    from oracle import ref_translated
    prim = cloud.initial_state(small_cloud, 0.8, 2.0)
    p = tmp_path / "stored-solution.dat"
    p.write_text(ref_translated.solution_text(small_cloud, prim))
    assert np.array_equal(io.read_stored_solution(str(p), small_cloud.n), prim)


def test_residue_layout_and_exact_read_back(mfcfd_lib, tmp_path):
    from mfcfd import io
    vals = np.array([[1.0, 0.1], [1e-5, -2.5], [0.0, 1e20], [123456.0, -0.0],
                     [0.099999999999999999, 9.87654321e16], [1e17, -3.25e-300]])
    p = tmp_path / "residue.dat"
    io.write_residue(str(p), 7, vals)
    lines = p.read_text().splitlines()
    assert lines[0] == "           7   1.0000000000000000       0.10000000000000001     "
    assert lines[1] == "           8   1.0000000000000001E-005  -2.5000000000000000     "
    assert lines[2] == "           9   0.0000000000000000        1.0000000000000000E+020"
    assert lines[3] == "          10   123456.00000000000       -0.0000000000000000     "
    assert lines[4].split()[1:] == ["0.10000000000000001", "98765432100000000."]
    assert lines[5].split()[1] == "1.0000000000000000E+017"
    back = np.array([[float(v.replace("E", "e")) for v in ln.split()[1:]] for ln in lines])
    assert np.array_equal(back, vals)
    assert [int(ln.split()[0]) for ln in lines] == list(range(7, 13))
    io.write_residue(str(p), 13, vals[:1], append=True)
    assert len(p.read_text().splitlines()) == 7


def _table(path):
    return np.array([[float(v.replace("E", "e")) for v in ln.split()] for ln in open(path)])


@pytest.mark.gpu
def test_print_primal_output_matches_fields(mfcfd_lib, small_cloud, tmp_path):
    from mfcfd import _lib
    from mfcfd.solver import Solver
    s = Solver(small_cloud, 0.8, 2.0)
    s.initial_conditions()
    s.q_lskum(2)
    s.print_primal_output(str(tmp_path))
    prim, flux, dq = s.get(_lib.FIELD_PRIM), s.get(_lib.FIELD_FLUX_RES), s.get(_lib.FIELD_DQ)
    a = _table(tmp_path / "primal-solution.dat")
    assert np.array_equal(a[:, :3], np.stack([small_cloud.x, small_cloud.y, small_cloud.z], 1))
    assert np.array_equal(a[:, 3:], prim)
    f = _table(tmp_path / "flux-residual.dat")
    assert np.array_equal(f[:, 0], np.arange(1, small_cloud.n + 1))
    assert np.array_equal(f[:, 1], small_cloud.status)
    assert np.array_equal(f[:, 2:], flux)
    q = _table(tmp_path / "qderivatives.dat")
    assert np.array_equal(q[:, 2:], dq.reshape(-1, 5, 3)[:, :, 2])   # dq(3, 1:5, k)
    assert os.path.getsize(tmp_path / "normals.dat") == 0
    s.close()


@pytest.mark.gpu
def test_program_end_to_end(mfcfd_lib, oracle_lib, small_cloud, tmp_path):
    """meshfree_solver.f90 as a run directory: files in, residue.dat and the
    post-processing files out.  residue.dat holds the run's own residuals, and
    the written state equals the CPU oracle's (solver libm) bit for bit."""
    from mfcfd import cloud, io, program
    from oracle import ref_translated
    prim0 = cloud.initial_state(small_cloud, 0.4, 0.0)
    (tmp_path / "3d_input_data").write_text(ref_translated.input_text(small_cloud))
    (tmp_path / "stored-solution.dat").write_text(ref_translated.solution_text(small_cloud, prim0))
    s = program.run(str(tmp_path), 0.4, 0.0, 5, chunk=2, echo=False)
    res = _table(tmp_path / "residue.dat")
    assert np.array_equal(res[:, 0], np.arange(1, 6))
    hist = np.array([[r, q] for _, r, q in s.history])
    assert np.array_equal(res[:, 1:], hist)
    o = oracle_lib.Oracle(small_cloud, 0.4, 0.0, libm=oracle_lib.LIBM_MFMATH)
    o.set_prim(prim0)
    for t in range(1, 6):
        o.step(t)
    a = _table(tmp_path / "primal-solution.dat")
    assert np.array_equal(a[:, 3:], o.get(oracle_lib.FIELD_PRIM))
    s.close()
