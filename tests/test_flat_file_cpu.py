"""Real-data flat-file readers (readLocsFile, readLocsFile3d, readObsFile,
readTimeFile, countlines) through the C ABI, against numpy's reading of the
same files (no GPU).  Values are written with 17 significant digits, so the
round trip is exact."""
import numpy as np
import pytest


def _write(path, rows):
    path.write_text("".join(",".join("%.17g" % v for v in r) + "\n" for r in rows))
    return str(path)


def test_countlines_counts_newlines(xg, tmp_path):
    p = tmp_path / "a.csv"
    p.write_text("1,2\n3,4\n5,6")  # last line without a newline is not counted (MLE_misc.c:976-981)
    assert xg.countlines(str(p)) == 2
    assert xg.countlines(str(tmp_path / "missing.csv")) == 0


def test_locations_and_observations_round_trip(xg, tmp_path):
    rng = np.random.default_rng(0)
    n = 257
    x, y, z = rng.random(n), rng.random(n), rng.standard_normal(n)
    locs = _write(tmp_path / "locs.csv", zip(x, y))
    obs = _write(tmp_path / "obs.csv", ((v,) for v in z))
    rx, ry = xg.read_locs_file(locs)
    assert np.array_equal(rx, x) and np.array_equal(ry, y)
    assert np.array_equal(xg.read_obs_file(obs), z)
    assert np.array_equal(xg.read_obs_file(obs, time=True), z)
    ref = np.loadtxt(locs, delimiter=",")
    assert np.array_equal(ref[:, 0], rx)
    # a prefix: reading stops after n rows
    px, py = xg.read_locs_file(locs, n=100)
    assert np.array_equal(px, x[:100]) and np.array_equal(py, y[:100])


def test_three_column_locations_and_formats(xg, tmp_path):
    p = tmp_path / "l3.csv"
    p.write_text("0.5, 0.25 ,3\n\n1e-3,-2.5E2,7\r\n")  # spaces, a blank line, CRLF, exponents
    x, y, t = xg.read_locs_file(str(p), n=2, dims=3)
    assert np.array_equal(x, [0.5, 1e-3]) and np.array_equal(y, [0.25, -250.0]) and np.array_equal(t, [3, 7])


@pytest.mark.parametrize("text,n", [("1,2\n3\n", 2), ("1,2\nfoo,3\n", 2), ("1,2\n", 2), ("", 1)])
def test_short_or_malformed_files_are_errors(xg, tmp_path, text, n):
    p = tmp_path / "bad.csv"
    p.write_text(text)
    with pytest.raises(xg.XgError):
        xg.read_locs_file(str(p), n=n)


def test_missing_file_is_an_error(xg, tmp_path):
    with pytest.raises(xg.XgError):
        xg.read_obs_file(str(tmp_path / "none.csv"), n=3)
