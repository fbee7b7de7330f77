"""OBJ texts exercising the reference loader's rules (written here, not taken from the
reference's assets): plain faces, v//vn and v/vt/vn forms, negative indices, polygons
(only the first three vertices are kept), zero normals, comments and long lines, a
missing final newline, and a seeded 1,024-triangle mesh."""
import numpy as np

from rumi_b200 import scenes


def _mesh_text(seed=3, levels=4):
    tris = scenes.displaced_sphere(levels, (0.1, 0.2, 0.3), 0.5, 0.05, seed)
    verts, idx = np.unique(tris.reshape(-1, 3), axis=0, return_inverse=True)
    idx = idx.reshape(-1, 3)
    rng = np.random.default_rng(seed)
    nrm = rng.standard_normal((verts.shape[0], 3)).astype(np.float32)
    lines = ["# seeded mesh", "o sphere"]
    lines += ["v %.7g %.7g %.7g" % tuple(p) for p in verts]
    lines += ["vt %.4f %.4f" % tuple(rng.random(2)) for _ in range(verts.shape[0])]
    lines += ["vn %.6f %.6f %.6f" % tuple(n) for n in nrm]
    lines += ["f %d/%d/%d %d/%d/%d %d/%d/%d" % (a + 1, a + 1, a + 1, b + 1, b + 1, b + 1, c + 1, c + 1, c + 1)
              for a, b, c in idx]
    return "\n".join(lines) + "\n"


CASES = {
    "plain": "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0.5\nf 1 2 3\nf 2 4 3\n",
    "normals": "v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 1\nvn 0 0.6 0.8\nvn 0 0 0\nf 1//1 2//2 3//3\n",
    "uv_normals": ("v 0.5 0.25 -1\nv 1.5 0.0 -1\nv 0.5 2.0 -1.25\nvt 0 0\nvt 1 0\nvt 0 1\n"
                   "vn 1 2 3\nvn -1 0 0\nvn 0 1 1\nf 1/1/1 2/2/2 3/3/3\n"),
    "negative": "v 0 0 0\nv 2 0 0\nv 0 2 0\nv 2 2 1\nf -4 -3 -2\nf -3 -1 -2\n",
    "quad": "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n",
    "comments": ("# a comment line that is longer than four characters\nv 0 0 0\n# v 9 9 9\n"
                 "v 3 0 0\nv 0 3 0\ng group\nusemtl none\ns off\nf 1 2 3\n"),
    "no_final_newline": "v 0 0 1\nv 1 0 1\nv 0 1 1\nf 1 2 3",
    "exponents": "v 1e-3 2.5E+1 -3.25\nv -1.0e2 0.125 7\nv 3 -4.5e-2 0.0\nf 1 2 3\n",
    "mesh": _mesh_text(),
}

# row-major Mat4x4 transforms (Translation * Scaling, a rotation about y, identity)
TRANSFORMS = {
    "identity": np.eye(4, dtype=np.float32).reshape(16),
    "translate_scale": np.array([2, 0, 0, 0.5, 0, 3, 0, -1, 0, 0, 0.5, 2, 0, 0, 0, 1], np.float32),
    "rotate_y": np.array([0.8, 0, 0.6, 0.25, 0, 1, 0, 0, -0.6, 0, 0.8, 0.5, 0, 0, 0, 1], np.float32),
}


# a doubled separator closes an empty vertex (index 0 - 1): a face that points outside
# the vertex list
BAD_FACE = "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 4 4 4\nf 1 2  3\n"


def canonical(v, n):
    """Triangles sorted by their vertex and normal floats (the reference's Model returns
    them in its BVH order)."""
    key = np.concatenate([v.reshape(-1, 9), n.reshape(-1, 9)], 1)
    order = np.lexsort(key.T[::-1])
    return v[order], n[order]
