"""Octree files and mesh dumps against the reference's own code: .ot files
as ot::writeNodesToFile writes them and as ot::readNodesFromFile reads them
(src/oct/OctFunctions.C:403-439), and the three files of
examples/src/drivers/dumpMesh.C (one rank) from the GPU-built mesh, byte for
byte."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["corner_points_d5", "uniform600_d7", "gauss1k_d8"]


def fixture(name):
    return np.load(os.path.join(GOLDEN, f"io_{name}.npz"))


def as_octants(bal):
    from dendro_b200._lib import OCT_DTYPE
    o = np.zeros(len(bal), OCT_DTYPE)
    for i, f in enumerate(OCT_DTYPE.names):
        o[f] = bal[:, i]
    return o


def octant_rows(t):
    a = t.to_numpy()
    names = a.dtype.names
    return np.stack([a[names[0]], a[names[1]], a[names[2]], a[names[3]] & 31], 1).astype(np.uint32)


@pytest.mark.parametrize("name", CASES)
def test_octree_files_match_reference(gpu, tmp_path, name):
    z = fixture(name)
    t = gpu.Octree.from_octants(as_octants(z["bal"]), int(z["depth"]))
    p = tmp_path / "o.ot"
    gpu.writeNodesToFile(p, t)
    assert np.array_equal(np.fromfile(p, np.uint8), z["ot"])
    ref = tmp_path / "ref.ot"
    z["ot"].tofile(ref)
    r = gpu.readNodesFromFile(ref)
    assert r.maxDepth == int(z["depth"]) and np.array_equal(octant_rows(r), z["bal"])


@pytest.mark.parametrize("name", CASES)
def test_mesh_dump_matches_reference(gpu, tmp_path, name):
    z = fixture(name)
    ref = tmp_path / "ref.ot"
    z["ot"].tofile(ref)
    da = gpu.DA(gpu.readNodesFromFile(ref))
    da.dumpMesh(str(tmp_path / "m"))
    for key, suffix in (("nl", "_NL_0_1.out"), ("el", "_EL_0_1.out"), ("m", "_M_0_1.out")):
        assert np.array_equal(np.fromfile(tmp_path / f"m{suffix}", np.uint8), z[key]), key


def test_octree_file_errors(gpu, tmp_path):
    z = fixture("gauss1k_d8")
    lines = bytes(z["ot"]).decode().splitlines()
    # octants out of Morton order are not a linear octree
    bad = tmp_path / "bad.ot"
    bad.write_text("\n".join(lines[:2] + [lines[3], lines[2]] + lines[4:]) + "\n")
    with pytest.raises(gpu.DendroError):
        gpu.readNodesFromFile(bad)
    trunc = tmp_path / "trunc.ot"
    trunc.write_text("\n".join(lines[:10]) + "\n")
    with pytest.raises(gpu.DendroError):
        gpu.readNodesFromFile(trunc)
