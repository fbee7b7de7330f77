"""Wavefront OBJ meshes as the reference's ``Model(file, transform)`` reads them.

Restates ``Model::LoadObjectFile`` (src/Shape/model.cpp:76-343) and the transform set-up
of ``Shape::Shape(const Mat4x4&)`` (src/Shape/shape.cpp:29-37) so that a mesh loaded here
is the mesh the reference renders, float for float:

* two passes over the file: the first counts ``v``/``vt``/``vn``/``f`` records (a line
  of more than 255 characters is read as several records), the second reads record
  tags of up to four characters ending at a space or newline, ``v``/``vt``/``vn``
  numbers with ``%f`` conversions and each face's rest of line -- so a comment such as
  ``# v 1 2 3`` is read as a vertex record by the second pass;
* a face keeps its first three vertices (no triangulation of polygons); indices are read
  digit by digit, ``/`` advances to the next field, ``-`` makes the index relative to the
  end of its list, and every separator -- a second space included -- closes a vertex;
* vertices are transformed by ``transform`` (translation included), normals by the
  transposed inverse (``Inverse`` by the reference's Gauss-Jordan elimination,
  src/Kernel/matrix.cpp:59-128) and normalised; a zero normal is replaced by the face
  normal of the transformed triangle; without ``vn`` records every vertex gets the face
  normal ``Normalize(Cross(v1 - v0, v2 - v0))``.

All arithmetic is float32 in the reference's operation order.  Triangles come out in file
order (the reference's Model then reorders its array while building its own BVH).  A face
that refers to a vertex or normal that does not exist raises ValueError (the reference
reads outside its arrays).
"""
from __future__ import annotations

import re

import numpy as np

F32 = np.float32
_FLOAT_RE = re.compile(rb"[+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan)", re.I)


def identity16() -> np.ndarray:
    return np.eye(4, dtype=F32).reshape(16)


def _mat_point(m, p):
    """Mat4x4 * Point3 / Vector3 (src/Kernel/matrix.cpp:44-64): the fourth column is added."""
    m = m.astype(F32)
    x, y, z = (F32(p[..., k]) for k in range(3))
    out = np.empty(p.shape, F32)
    for r in range(3):
        out[..., r] = ((m[4 * r] * x + m[4 * r + 1] * y) + m[4 * r + 2] * z) + m[4 * r + 3]
    return out


def inverse16(m) -> np.ndarray:
    """Inverse(const Mat4x4&): elimination below, then above the diagonal, then row scaling."""
    src = np.asarray(m, F32).copy()
    inv = identity16()
    for col in range(4):
        piv = col * 4 + col
        for row in range(col + 1, 4):
            ux = F32(-src[row * 4 + col] / src[piv])
            for k in range(4):
                src[row * 4 + k] = F32(src[row * 4 + k] + src[col * 4 + k] * ux)
                inv[row * 4 + k] = F32(inv[row * 4 + k] + inv[col * 4 + k] * ux)
    for col in range(4):
        piv = col * 4 + col
        for row in range(col - 1, -1, -1):
            ux = F32(-src[row * 4 + col] / src[piv])
            for k in range(4):
                src[row * 4 + k] = F32(src[row * 4 + k] + src[col * 4 + k] * ux)
                inv[row * 4 + k] = F32(inv[row * 4 + k] + inv[col * 4 + k] * ux)
    for i in range(4):
        ip = F32(F32(1.0) / src[i * 4 + i])
        for k in range(4):
            inv[i * 4 + k] = F32(inv[i * 4 + k] * ip)
    return inv


def transpose16(m) -> np.ndarray:
    return np.asarray(m, F32).reshape(4, 4).T.reshape(16).copy()


def _normalize(v):
    v = v.astype(F32)
    s = (v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1]) + v[..., 2] * v[..., 2]
    with np.errstate(divide="ignore", invalid="ignore"):  # degenerate triangles: NaN, as in the reference
        inv = (F32(1.0) / np.sqrt(s.astype(F32))).astype(F32)
        return (v * inv[..., None]).astype(F32)


def _cross(u, v):
    cx = u[..., 1] * v[..., 2] - v[..., 1] * u[..., 2]
    cy = u[..., 2] * v[..., 0] - v[..., 2] * u[..., 0]
    cz = u[..., 0] * v[..., 1] - v[..., 0] * u[..., 1]
    return np.stack([cx, cy, cz], -1).astype(F32)


def _records(data: bytes):
    """fgets(buffer, 256, file): records of at most 255 bytes, each ending after a newline."""
    pos = 0
    while pos < len(data):
        nl = data.find(b"\n", pos, pos + 255)
        end = nl + 1 if nl >= 0 else min(pos + 255, len(data))
        yield data[pos:end]
        pos = end


class _Stream:
    """The second pass's view of the file: fgetc, fscanf("%f"), fgets."""

    def __init__(self, data: bytes):
        self.d = data
        self.p = 0

    def getc(self):
        if self.p >= len(self.d):
            return None  # EOF
        c = self.d[self.p:self.p + 1]
        self.p += 1
        return c

    def scan_floats(self, n):
        """fscanf(file, "%f %f ...") with n conversions; unparsed values stay 0."""
        out = [F32(0.0)] * n
        for k in range(n):
            while self.p < len(self.d) and self.d[self.p:self.p + 1] in b" \t\n\r\v\f":
                self.p += 1
            m = _FLOAT_RE.match(self.d, self.p)
            if not m:
                break
            out[k] = F32(float(m.group(0)))
            self.p = m.end()
        return out

    def gets(self):
        if self.p >= len(self.d):
            return None
        nl = self.d.find(b"\n", self.p, self.p + 255)
        end = nl + 1 if nl >= 0 else min(self.p + 255, len(self.d))
        s = self.d[self.p:end]
        self.p = end
        return s


def _face_indices(buf: bytes, v_count, vt_count, vn_count):
    """The digit state machine of the face parser over a zero-padded 256-byte buffer."""
    b = buf + b"\0" * (256 - len(buf))
    idx_v, idx_vt, idx_vn = [0, 0, 0], [0, 0, 0], [0, 0, 0]
    n_in = 0
    neg = False
    field = 0
    data = [F32(0.0)] * 3
    for i in range(256):
        c = b[i:i + 1]
        if c == b"-":
            neg = True
        elif c.isdigit():
            data[field] = F32(data[field] * F32(10.0) + F32(ord(c) - 0x30))
        elif c == b"/":
            field += 1
            neg = False
        elif c in (b" ", b"\n", b"\0"):
            if not neg:
                idx_v[n_in], idx_vt[n_in], idx_vn[n_in] = (int(data[0] - F32(1)), int(data[1] - F32(1)),
                                                             int(data[2] - F32(1)))
            else:
                idx_v[n_in] = int(-data[0] + F32(v_count))
                idx_vt[n_in] = int(-data[1] + F32(vt_count))
                idx_vn[n_in] = int(-data[2] + F32(vn_count))
            n_in += 1
            field = 0
            data = [F32(0.0)] * 3
            neg = False
        if n_in == 3:
            break
    return idx_v, idx_vt, idx_vn


def load_obj_bytes(data: bytes, transform=None):
    """Triangles of an OBJ file's contents: (vertices (F,3,3), normals (F,3,3)) float32."""
    m = identity16() if transform is None else np.asarray(transform, F32).reshape(16)
    m_nrm = transpose16(inverse16(m))
    v_count = vt_count = vn_count = f_count = 0
    for rec in _records(data):
        if rec[:2] == b"v ":
            v_count += 1
        if rec[:2] == b"vt":
            vt_count += 1
        if rec[:2] == b"vn":
            vn_count += 1
        if rec[:2] == b"f ":
            f_count += 3
    v = np.zeros((v_count, 3), F32)
    vn = np.zeros((vn_count, 3), F32)
    v_idx_list = np.zeros(f_count, np.int64)
    vn_idx_list = np.zeros(f_count, np.int64)
    s = _Stream(data)
    vi = vni = fi = 0
    while True:
        tag = b""
        at_eof = False
        for k in range(4):
            c = s.getc()
            if c is None:
                if k == 0:
                    at_eof = True
                break
            tag += c
            if c in (b"\n", b" "):
                break
        if at_eof:
            break
        # a tag is read wherever the previous record stopped, so "# v 1 2 3" yields a
        # vertex; records beyond the first pass's counts are read and dropped (the
        # reference writes them past its arrays)
        if tag == b"v ":
            vals = s.scan_floats(3)
            if vi < v_count:
                v[vi] = vals
            vi += 1
        elif tag == b"vt ":
            s.scan_floats(2)
        elif tag == b"vn ":
            vals = s.scan_floats(3)
            if vni < vn_count:
                vn[vni] = vals
            vni += 1
        elif tag == b"f ":
            buf = s.gets()
            if buf is not None:
                iv, _, ivn = _face_indices(buf, v_count, vt_count, vn_count)
                if fi + 3 > f_count:
                    raise ValueError("OBJ face records differ between the two passes")
                v_idx_list[fi:fi + 3] = iv
                if vn_count > 0:
                    vn_idx_list[fi:fi + 3] = ivn
                fi += 3
    if (v_idx_list < 0).any() or (v_idx_list >= max(v_count, 1)).any():
        raise ValueError("OBJ face refers to a vertex that does not exist")
    tris = v[v_idx_list].reshape(-1, 3, 3)
    tv = _mat_point(m, tris)
    face = _normalize(_cross(tv[:, 1] - tv[:, 0], tv[:, 2] - tv[:, 0]))
    if vn_count > 0:
        if (vn_idx_list < 0).any() or (vn_idx_list >= vn_count).any():
            raise ValueError("OBJ face refers to a normal that does not exist")
        n = vn[vn_idx_list].reshape(-1, 3, 3).copy()
        zero = (n == 0).all(-1)
        n[zero] = np.repeat(face[:, None, :], 3, 1)[zero]
        n = _normalize(_mat_point(m_nrm, n))
    else:
        n = np.repeat(face[:, None, :], 3, 1)
    return np.ascontiguousarray(tv, F32), np.ascontiguousarray(n, F32)


def load_obj(path: str, transform=None):
    """``Model(path, transform)``'s triangles: (vertices (F,3,3), normals (F,3,3)) float32."""
    with open(path, "rb") as f:
        return load_obj_bytes(f.read(), transform)
