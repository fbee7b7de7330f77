"""The host OBJ loader (rumi_b200.obj) against the reference's own Model(file, transform)
loader, on OBJ texts that exercise its parsing rules: vertices and normals bit-exact
(live reference build when present, else the committed fixture)."""
import os

import numpy as np
import pytest

import refimpl
from obj_cases import BAD_FACE, CASES, TRANSFORMS, canonical
from rumi_b200 import obj


@pytest.mark.parametrize("tname", sorted(TRANSFORMS))
@pytest.mark.parametrize("case", sorted(CASES))
def test_obj_loader_matches_reference_fixture(golden, tmp_path, case, tname):
    g = golden("obj_loader.npz")
    v, n = canonical(*obj.load_obj_bytes(CASES[case].encode(), TRANSFORMS[tname]))
    rv, rn = canonical(g[f"{case}__{tname}__v"], g[f"{case}__{tname}__n"])
    np.testing.assert_array_equal(v, rv)
    np.testing.assert_array_equal(n, rn)


@pytest.mark.skipif(not refimpl.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("case", sorted(CASES))
def test_obj_loader_matches_live_reference(tmp_path, case):
    path = os.path.join(str(tmp_path), case + ".obj")
    with open(path, "wb") as f:
        f.write(CASES[case].encode())
    for m in TRANSFORMS.values():
        rv, rn = canonical(*refimpl.load_obj(path, m))
        v, n = canonical(*obj.load_obj(path, m))
        np.testing.assert_array_equal(v, rv)
        np.testing.assert_array_equal(n, rn)


def test_obj_face_outside_the_vertex_list_is_rejected():
    with pytest.raises(ValueError):
        obj.load_obj_bytes(BAD_FACE.encode())


def test_obj_mesh_through_the_scene_api(tmp_path):
    from rumi_b200.scene import Model
    path = str(tmp_path / "mesh.obj")
    with open(path, "w") as f:
        f.write(CASES["mesh"])
    m = Model.from_obj(path, TRANSFORMS["translate_scale"])
    v, n = obj.load_obj(path, TRANSFORMS["translate_scale"])
    assert m.vertices.shape == (4 * 4 ** 4, 3, 3)
    np.testing.assert_array_equal(m.vertices, v)
    np.testing.assert_array_equal(m.normals, n)
