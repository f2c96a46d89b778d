"""Scene ingestion and film output (no GPU): OBJ meshes, Radiance .hdr and PFM
images, through the C ABI (cl_obj_*, cl_image_*).  The files are written by
the tests themselves (the reference's sample assets are not in its tree)."""
import numpy as np
import pytest

import colvillea_b200 as cb

OBJ = """# two groups: a textured quad and pentagon with normals, a box without normals
mtllib none.mtl
o plate
v 0 0 0
v 2 0 0
v 2 0 1
v 0 0 1
v 1 0 1.5
vt 0 0
vt 1 0
vt 1 0.5
vt 0 0.5
vt 0.5 0.75
vn 0 1 0
f 1/1/1 2/2/1 3/3/1 4/4/1
f -5/-5/-1 -2/-2/-1 \\
  -1/-1/-1
o box
v -1 -1 -1
v 1 -1 -1
v 1 1 -1
v -1 1 -1
v -1 -1 1
v 1 -1 1
v 1 1 1
v -1 1 1
f 6 9 8 7
f 10 11 12 13
f 6 7 11 10
f 8 9 13 12
f 6 10 13 9
f 7 8 12 11
"""


def test_obj(tmp_path):
    p = tmp_path / "scene.obj"
    p.write_text(OBJ)
    meshes = cb.load_obj(p)
    assert len(meshes) == 2
    plate, box = meshes
    # quad -> 2 triangles (fan), triangle -> 1
    assert plate.indices.shape == (3, 3)
    assert len(plate.positions) == 5
    np.testing.assert_array_equal(plate.indices[0], [0, 1, 2])
    np.testing.assert_array_equal(plate.indices[1], [0, 2, 3])
    np.testing.assert_allclose(plate.normals, np.tile([0, 1, 0], (5, 1)))
    # v flipped
    np.testing.assert_allclose(plate.uvs[:, 1], 1 - np.array([0, 0, 0.5, 0.5, 0.75]))
    # u runs along +x: tangent = dP/du = +x
    np.testing.assert_allclose(plate.tangents, np.tile([1, 0, 0], (5, 1)), atol=1e-6)
    # box: 6 quads, no normals or uvs: smooth normals along the corner diagonals
    assert box.indices.shape == (12, 3) and box.uvs is None and len(box.positions) == 8
    # expected: normalised sum of the (area-weighted) normals of the triangles at each vertex
    P, I = box.positions.astype(np.float64), box.indices
    fn = np.cross(P[I[:, 1]] - P[I[:, 0]], P[I[:, 2]] - P[I[:, 0]])
    acc = np.zeros_like(P)
    for k in range(3):
        np.add.at(acc, I[:, k], fn)
    acc /= np.linalg.norm(acc, axis=1, keepdims=True)
    np.testing.assert_allclose(box.normals, acc, atol=1e-6)
    assert np.all(np.sum(box.normals * box.positions, 1) > 0)       # outward
    assert np.all(np.abs(np.sum(box.normals * box.tangents, 1)) < 1e-6)
    np.testing.assert_allclose(np.linalg.norm(box.tangents, axis=1), 1, atol=1e-6)


@pytest.mark.parametrize("text,where", [("v 0 0 0\nf 1 2 3\n", "line 2"), ("v 0 0\n", "line 1"),
                                        ("v 0 0 0\nv 1 0 0\nf 1 2\n", "line 3"), ("# empty\n", "no faces")])
def test_obj_errors(tmp_path, text, where):
    p = tmp_path / "bad.obj"
    p.write_text(text)
    with pytest.raises(cb.ClError) as e:
        cb.load_obj(p)
    assert where in str(e.value) and e.value.status == 5


def rgbe_encode(rgb):
    """Own encoder: e = frexp exponent + 128, mantissa bytes floor(c * 256 / 2^e')."""
    m = rgb.max(-1)
    out = np.zeros(rgb.shape[:-1] + (4,), np.uint8)
    nz = m > 1e-32
    f, e = np.frexp(m[nz])
    scale = 256.0 / np.ldexp(1.0, e)
    out[nz, :3] = np.floor(rgb[nz] * scale[:, None]).astype(np.uint8)
    out[nz, 3] = (e + 128).astype(np.uint8)
    return out


def rgbe_decode(q):
    f = np.where(q[..., 3:4] > 0, np.ldexp(1.0, q[..., 3:4].astype(int) - 136), 0.0)
    rgb = q[..., :3] * f
    return np.concatenate([rgb, np.ones(q.shape[:-1] + (1,))], -1).astype(np.float32)


def rle_channel(v):
    out, i, n = bytearray(), 0, len(v)
    while i < n:
        j = i
        while j < n and j - i < 127 and v[j] == v[i]:
            j += 1
        if j - i >= 3:
            out += bytes([128 + j - i, v[i]])
            i = j
        else:
            k = i
            while k < n and k - i < 128 and not (k + 2 < n and v[k] == v[k + 1] == v[k + 2]):
                k += 1
            out += bytes([k - i]) + bytes(v[i:k])
            i = k
    return out


def write_hdr(path, q, rle):
    h, w = q.shape[:2]
    data = bytearray(b"#?RADIANCE\n# written by the test\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {h} +X {w}\n".encode())
    for y in range(h):
        if rle:
            data += bytes([2, 2, w >> 8, w & 255])
            for c in range(4):
                data += rle_channel(q[y, :, c].tolist())
        else:
            data += q[y].tobytes()
    path.write_bytes(bytes(data))


@pytest.mark.parametrize("rle", [True, False])
def test_hdr(tmp_path, rle):
    rng = np.random.default_rng(0)
    img = np.exp(rng.normal(0, 3, (37, 67, 3)))
    img[5:9, 10:40] = 2.5                      # runs
    img[0, :] = 0.0
    q = rgbe_encode(img)
    p = tmp_path / "dome.hdr"
    write_hdr(p, q, rle)
    got = cb.load_hdr(p)
    assert got.shape == (37, 67, 4) and got.dtype == np.float32
    np.testing.assert_array_equal(got, rgbe_decode(q))
    assert np.all(np.abs(got[..., :3] - img) <= img.max(-1, keepdims=True) / 128 + 1e-30)


def test_hdr_errors(tmp_path):
    p = tmp_path / "x.hdr"
    p.write_bytes(b"P6\n1 1\n255\n\x00\x00\x00")
    with pytest.raises(cb.ClError):
        cb.load_hdr(p)
    p.write_bytes(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 2 +X 2\n\x01\x01\x01\x80")
    with pytest.raises(cb.ClError) as e:
        cb.load_hdr(p)
    assert "truncated" in str(e.value)


def test_pfm_roundtrip(tmp_path):
    rng = np.random.default_rng(1)
    img = rng.normal(size=(13, 21, 4)).astype(np.float32)
    p = tmp_path / "film.pfm"
    cb.write_pfm(p, img)
    raw = p.read_bytes()
    hdr = b"PF\n21 13\n-1\n"
    assert raw.startswith(hdr)
    rows = np.frombuffer(raw[len(hdr):], np.float32).reshape(13, 21, 3)
    np.testing.assert_array_equal(rows[::-1], img[..., :3])     # stored bottom up
    back = cb.read_pfm(p)
    np.testing.assert_array_equal(back[..., :3], img[..., :3])
    assert np.all(back[..., 3] == 1)
