"""Point files against the reference's own writers and readers
(ot::writePtsToFile / readPtsFromFile / writeDataPtsToFile /
readDataPtsFromFile, src/oct/OctFunctions.C:313-401): byte-identical files,
equal values read back.  Host code only: runs without a GPU."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["corner_points_d5", "uniform600_d7", "gauss1k_d8"]


def fixture(name):
    return np.load(os.path.join(GOLDEN, f"io_{name}.npz"))


@pytest.mark.parametrize("name", CASES)
def test_point_files_match_reference(tmp_path, name):
    import dendro_b200 as dg
    z = fixture(name)
    p = tmp_path / "p.pts"
    dg.writePtsToFile(p, z["pts"])
    assert np.array_equal(np.fromfile(p, np.uint8), z["pts_file"])
    ref = tmp_path / "ref.pts"
    z["pts_file"].tofile(ref)
    assert np.array_equal(dg.readPtsFromFile(ref), z["pts"])


@pytest.mark.parametrize("name", CASES)
def test_data_point_files_match_reference(tmp_path, name):
    import dendro_b200 as dg
    z = fixture(name)
    p = tmp_path / "d.pts"
    dg.writeDataPtsToFile(p, z["pts"], z["vals"])
    assert np.array_equal(np.fromfile(p, np.uint8), z["data_file"])
    ref = tmp_path / "ref.pts"
    z["data_file"].tofile(ref)
    pts, vals = dg.readDataPtsFromFile(ref)
    assert np.array_equal(pts, z["pts"]) and np.array_equal(vals, z["vals"])


def test_point_file_edge_cases(tmp_path):
    import dendro_b200 as dg
    # the reference's writer leaves an empty file for no points; it reads back as none
    e = tmp_path / "e.pts"
    dg.writePtsToFile(e, np.zeros((0, 3)))
    assert os.path.getsize(e) == 0 and dg.readPtsFromFile(e).shape == (0, 3)
    # with values the header is always written
    dg.writeDataPtsToFile(tmp_path / "ed.pts", np.zeros((0, 3)), np.zeros(0))
    assert os.path.getsize(tmp_path / "ed.pts") == 4
    pts, vals = dg.readDataPtsFromFile(tmp_path / "ed.pts")
    assert pts.shape == (0, 3) and vals.shape == (0,)
    # a truncated file and a missing file are errors, not garbage
    t = tmp_path / "t.pts"
    np.array([3], np.uint32).tofile(t)
    with pytest.raises(dg.DendroError):
        dg.readPtsFromFile(t)
    with pytest.raises(dg.DendroError):
        dg.readPtsFromFile(tmp_path / "missing.pts")
    with pytest.raises(ValueError):
        dg.writeDataPtsToFile(tmp_path / "x.pts", np.zeros((2, 3)), np.zeros(3))
