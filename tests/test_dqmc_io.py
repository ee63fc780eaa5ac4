"""Result writers, field files and the command line (no GPU): the text formats are checked
line by line against the reference's own example output (tests/golden/example_format.json,
written by make_golden.py from the reference's example/ folder)."""
import io
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def fmt():
    with open(os.path.join(HERE, "golden", "example_format.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def dio(hq):
    from hubbard_b200 import dqmc_io
    return dqmc_io


def render(fn, *args, **kw):
    buf = io.StringIO()
    fn(buf, *args, **kw)
    return buf.getvalue().splitlines()


def test_momentum_list_and_time_grids_match_the_reference_files(dio, fmt):
    # the reference's example: L = 4, AllKstars; beta = 8, nt = 160, dt = 0.05
    assert render(dio.print_momentum_list, 4, list(range(9))) == fmt["momenta.out"]
    assert render(dio.print_imaginary_time_grids, 160, 8.0, 0.05) == fmt["tgrids.out"]


def test_field_file_matches_the_reference_file(dio, fmt, tmp_path):
    from conftest import example_fields
    fields = example_fields()
    path = tmp_path / "ising.fields"
    dio.save_ising_fields(str(path), fields)
    lines = path.read_text().splitlines()
    assert lines[:len(fmt["ising.fields"])] == fmt["ising.fields"]
    back = dio.load_ising_fields(str(path), *fields.shape)
    assert np.array_equal(back, fields)
    with pytest.raises(ValueError):
        dio.load_ising_fields(str(path), fields.shape[0] + 1, fields.shape[1])


def test_binned_rows_match_the_reference_files(dio, fmt):
    # the reference's example files carry no header line (written by an older build); the rows
    # re-rendered from their own numbers must be identical
    def rows(name, ndim):
        vals = [ln.split() for ln in fmt[name]]
        idx = [tuple(int(x) for x in v[:ndim]) for v in vals]
        return idx, [float(v[ndim]) for v in vals]
    for name, ndim in (("filling.bins.out", 1), ("spin_corr.bins.out", 2), ("gf.bins.out", 3)):
        idx, val = rows(name, ndim)
        shape = tuple(max(i[d] for i in idx) + 1 for d in range(ndim))
        data = np.zeros(shape)
        for i, v in zip(idx, val):
            data[i] = v
        out = render(dio.print_observable_data, data, show_header=False)
        assert out[:len(idx)] == fmt[name], name
    vals = [ln.split() for ln in fmt["gf.out"]]
    mean = np.array([[float(v[2]) for v in vals]])
    std = np.array([[float(v[3]) for v in vals]])
    err = np.array([[float(v[4]) for v in vals]])
    assert render(dio.print_observable, mean, std, err, show_header=False) == fmt["gf.out"]


def test_headers_and_scalar_observables(dio):
    lines = render(dio.print_observable, np.float64(0.5), np.float64(0.25), np.float64(0.125))
    assert lines == ["{: 15d}".format(1), "{: 15d}{: 30.15f}{: 30.15f}{: 30.15f}".format(0, 0.5, 0.25, 0.125)]
    lines = render(dio.print_observable_data, np.zeros((3, 2)))
    assert lines[0] == "{: 15d}{: 15d}".format(3, 2) and len(lines) == 7


def test_command_line_help(hq):
    from hubbard_b200 import cli
    with pytest.raises(SystemExit) as ex:
        cli.main(["--help"])
    assert ex.value.code == 0
