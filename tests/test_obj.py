"""The OBJ / MTL reader (mlbvh_obj_load; CPU only): faces of every corner
form, negative indices, quads split along the shorter diagonal, fans,
materials and their defaults; and, where the reference checkout is present,
the path tracer's oracle pinned to the reference's own pt on the scene the
reference renders (bin/assets/cornelbox.obj)."""
import os

import numpy as np
import pytest

import _objscene
import _oracle as O
import minimumlbvh_b200 as mb

# the reference checkout, named by MLBVH_REFERENCE_DIR (the test that needs it
# is skipped when the variable is unset)
REF_DIR = os.environ.get("MLBVH_REFERENCE_DIR", "")
REF_OBJ = os.path.join(REF_DIR, "bin", "assets", "cornelbox.obj") if REF_DIR else ""


def test_obj_face_forms_and_materials(tmp_path):
    (tmp_path / "m.mtl").write_text("newmtl a\nKd 0.1 0.2 0.3\nKe 4 5 6\nnewmtl grey\nKd 0.25\n")
    (tmp_path / "t.obj").write_text(
        "mtllib m.mtl\n"
        "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 3 0 0\nv 2 0 0\nv 3 1 0\n"
        "vt 0 0\nvt 1 0\nvn 0 0 1\nvn 0 1 0\n"
        "f 1 2 3\n"                       # no material: Kd 0.5, no emission, no normals
        "usemtl a\n"
        "f 1/1/1 2/2/1 3/1/2\n"           # v/vt/vn
        "usemtl nosuch\n"
        "f -7//-2 -6//-2 -5//-1\n"        # negative indices, unknown material: default
        "usemtl grey\n"
        "f 1/1 2/2 3/1 4/2\n"             # quad, diagonals equal: split (0,1,2), (0,2,3)
        "f 1 5 3 4\n"                     # |v2 - v0| shorter: (0,1,2), (0,2,3)
        "f 1 6 7 4\n"                     # |v3 - v1| shorter: (0,1,3), (1,2,3)
        "f 1 2 5 3 4\n")                  # pentagon: fan
    tris, at = mb.load_obj(str(tmp_path / "t.obj"))
    V = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [3, 0, 0], [2, 0, 0], [3, 1, 0]], np.float32)
    want = [(0, 1, 2), (0, 1, 2), (0, 1, 2), (0, 1, 2), (0, 2, 3), (0, 4, 2), (0, 2, 3), (0, 5, 3), (5, 6, 3),
            (0, 1, 4), (0, 4, 2), (0, 2, 3)]
    np.testing.assert_array_equal(tris, V[np.array(want)].reshape(-1, 9))
    np.testing.assert_array_equal(at[0, 9:15], [0.5, 0.5, 0.5, 0, 0, 0])
    np.testing.assert_array_equal(at[0, 0:9], 0)
    np.testing.assert_array_equal(at[1, 0:9], [0, 0, 1, 0, 0, 1, 0, 1, 0])
    np.testing.assert_allclose(at[1, 9:15], [0.1, 0.2, 0.3, 4, 5, 6])
    np.testing.assert_array_equal(at[2, 0:9], [0, 0, 1, 0, 0, 1, 0, 1, 0])
    np.testing.assert_array_equal(at[2, 9:15], [0.5, 0.5, 0.5, 0, 0, 0])
    np.testing.assert_array_equal(at[3:, 9:12], 0.25)


def test_obj_errors(tmp_path):
    with pytest.raises(mb.MlbvhError):
        mb.load_obj(str(tmp_path / "missing.obj"))
    (tmp_path / "bad.obj").write_text("v 0 0 0\nf 1 2 3\n")
    with pytest.raises(mb.MlbvhError) as e:
        mb.load_obj(str(tmp_path / "bad.obj"))
    assert "line 2" in str(e.value)


def test_generated_box_loads(tmp_path):
    tris, at = mb.load_obj(_objscene.write_cornell(str(tmp_path)))
    assert tris.shape == (32, 9) and at.shape == (32, 15)
    assert (at[:, 12:15].sum(1) > 0).sum() == 2  # the lamp's two triangles


@pytest.mark.skipif(not (REF_OBJ and os.path.exists(REF_OBJ) and O.ref_available()),
                    reason="needs MLBVH_REFERENCE_DIR (the reference checkout) and its host build")
def test_reference_cornell_box_pt_matches_reference_pt():
    """Path tracing of the reference's own scene: the oracle's pt (libm trig,
    the reference's sample order) equals the reference's pt compiled for the
    host, accumulator for accumulator, over the tree of the reference's
    stable-order build. Camera as the reference's viewer opens (eye (0, 1, 4),
    looking at (0, 1, 0)); fovy 45 degrees (the viewer library's default is
    not in the checkout)."""
    tris, at = mb.load_obj(REF_OBJ)
    assert len(tris) == 17716
    b = O.build(tris)
    w, h = 40, 30
    cam = O.lookat((0, 1, 4), (0, 1, 0), (0, 1, 0), np.float32(np.deg2rad(45.0)), w, h)
    ours = np.zeros((w * h, 4), np.float32)
    ref = np.zeros((w * h, 4), np.float32)
    for _ in range(2):
        O.render_pt(ours, cam, b["root"], b["nodes"], tris, at, w, h, 1, trig=0)
        O.ref_pt(ref, cam, b["root"], b["nodes"], tris, at, w, h, 1)
    np.testing.assert_array_equal(ours, ref)
    assert (ours[:, :3].sum(1) > 0).sum() > 0  # some paths reach the light
