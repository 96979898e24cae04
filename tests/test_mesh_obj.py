"""OBJ meshes (rbr_mesh_*: host code of the library, no GPU needed) against the reference's own
ObjImporter + TriangleMesh::toPrimitives on identical text: the same triangles, bit for bit,
with the same (normalised) vertex normals, and the same failures."""
import numpy as np
import pytest

from oracle import reference_dir
from rbr_b200 import load_obj, parse_obj

ASSETS = reference_dir() / "assets"

CASES = {
    "triangles": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nf 1 2 3\nf 1 3 4\n",
    "quad fan": b"v 0 0 0\nv 2 0 0\nv 2 2 0\nv 0 2 0\nv 1 3 0.5\nf 1 2 3 4 5\n",
    "negative indices": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0.25\nf -4 -3 -2\nf -3 -1 -2\n",
    "normals and uvs": (b"v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 0 1\nvn 0 0 2\nvn 0 0.5 1\nvn 1 1 1\n"
                        b"f 1/1/1 2/2/2 3/3/3\n"),
    "v//vn": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 1\nf 1//1 2//1 3//1\n",
    "normals missing on a corner": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nvn 0 0 1\nf 1//1 2//1 3//1\nf 2 4 3\n",
    "comments and blanks": b"# a mesh\n\nv 0 0 0\nv 1 0 0  # trailing\nv 0 1 0\no obj\ng grp\nusemtl m\nf 1 2 3\n",
    "shared corners": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1 2 3\nf 3 2 4\nf 1 2 4\n",
    "scientific": b"v 1e-3 -2.5E+2 3.25\nv 0.1 0.2 0.3\nv -7 8e1 9\nf 1 2 3\n",
}

BAD = {
    "index out of range": b"v 0 0 0\nv 1 0 0\nf 1 2 3\n",
    "zero index": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n",
    "no faces": b"v 0 0 0\nv 1 0 0\nv 0 1 0\n",
    "empty": b"",
}


def same(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("name", list(CASES))
def test_parse_matches_reference_importer(reference, name):
    text = CASES[name]
    v, n = parse_obj(text)
    rv, rn = reference.obj_triangles(text)
    assert same(v, rv)
    assert (n is None) == (rn is None)
    if n is not None:
        assert same(n, rn)


@pytest.mark.parametrize("name", list(BAD))
def test_malformed_files_fail_like_the_reference(reference, name):
    assert reference.obj_triangles(BAD[name]) is None
    with pytest.raises(ValueError):
        parse_obj(BAD[name])


@pytest.mark.parametrize("asset", ["barrel.obj", "motocompo.obj"])
def test_reference_assets(reference, asset):
    path = ASSETS / asset
    if not path.exists():
        pytest.skip("the reference's assets are not present")
    v, n = load_obj(path)
    rv, rn = reference.obj_triangles(path.read_bytes())
    assert len(v) > 1000 and same(v, rv)
    assert (n is None) == (rn is None)
    if n is not None:
        assert same(n, rn)


def test_missing_file():
    with pytest.raises(ValueError, match="could not open"):
        load_obj("/nonexistent/mesh.obj")
