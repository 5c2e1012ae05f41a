"""Design output files through the C ABI (host only): DesignVolume.nii (TOP3D_XL.m:564-570) and
the closed 0.5 isosurface DesignVolume.stl (TOP3D_XL.m:206-222, 572-577)."""
import ctypes as C
import struct
from collections import Counter

import numpy as np
import pytest


def _lib():
    from top3d_xl_b200 import _lib as L
    return L.load(), L


def _write_stl(tmp_path, vol, iso=0.5):
    lib, L = _lib()
    ny, nx, nz = vol.shape
    v = np.ascontiguousarray(vol.reshape(-1, order="F"), dtype=np.float64)
    n = C.c_int64(-1)
    path = str(tmp_path / "d.stl")
    st = lib.topx_write_design_stl(v.ctypes.data_as(C.POINTER(C.c_double)), ny, nx, nz, iso, path.encode(),
                                   C.byref(n))
    assert st == L.TOPX_OK
    raw = open(path, "rb").read()
    (count,) = struct.unpack_from("<I", raw, 80)
    assert count == n.value and len(raw) == 84 + 50 * count
    rec = np.frombuffer(raw, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]), offset=84)
    return rec


def _closed_and_oriented(tris):
    """every directed edge once, and its reverse once: a closed, consistently oriented surface"""
    keys = [tuple(map(tuple, t)) for t in tris]
    directed = Counter()
    for a, b, c in keys:
        for e in ((a, b), (b, c), (c, a)):
            directed[e] += 1
    assert max(directed.values()) == 1
    assert all(directed[(b, a)] == 1 for (a, b) in directed)


def _volume(tris):
    t = tris.astype(np.float64)
    return float(np.sum(np.einsum("ij,ij->i", t[:, 0], np.cross(t[:, 1], t[:, 2]))) / 6.0)


def test_nifti_header_and_data(tmp_path):
    lib, L = _lib()
    vol = np.random.default_rng(0).uniform(0, 1, (6, 9, 4))
    v = np.ascontiguousarray(vol.reshape(-1, order="F"))
    path = str(tmp_path / "d.nii")
    assert lib.topx_write_design_nii(v.ctypes.data_as(C.POINTER(C.c_double)), 6, 9, 4, path.encode()) == L.TOPX_OK
    raw = open(path, "rb").read()
    assert struct.unpack_from("<i", raw, 0)[0] == 348
    assert struct.unpack_from("<8h", raw, 40) == (3, 6, 9, 4, 1, 1, 1, 1)
    assert struct.unpack_from("<2h", raw, 70) == (64, 64)  # FLOAT64, 64 bits
    assert struct.unpack_from("<f", raw, 108)[0] == 352.0
    assert raw[344:348] == b"n+1\0"
    data = np.frombuffer(raw, dtype="<f8", offset=352)
    assert np.array_equal(data, v)
    assert lib.topx_write_design_nii(None, 6, 9, 4, path.encode()) == -1


def test_solid_box_is_the_capped_lattice_box(tmp_path):
    # all ones: no interior surface, the caps alone close the box [1, nx] x [1, ny] x [1, nz]
    ny, nx, nz = 5, 7, 4
    rec = _write_stl(tmp_path, np.ones((ny, nx, nz)))
    tris = rec["v"]
    _closed_and_oriented(tris)
    assert abs(_volume(tris) - (nx - 1) * (ny - 1) * (nz - 1)) < 1e-9
    assert tris[..., 0].min() == 1 and tris[..., 0].max() == nx
    assert tris[..., 1].min() == 1 and tris[..., 1].max() == ny
    assert tris[..., 2].min() == 1 and tris[..., 2].max() == nz
    n = rec["n"].astype(np.float64)
    c = tris.astype(np.float64).mean(axis=1) - np.array([(nx + 1) / 2, (ny + 1) / 2, (nz + 1) / 2])
    assert np.all(np.einsum("ij,ij->i", n, c) > 0)  # normals point out of the box


@pytest.mark.parametrize("center", [(10.3, 9.7, 10.1), (3.2, 9.5, 8.8)])
def test_sphere_closed_with_caps_and_volume(tmp_path, center):
    # a smooth field whose 0.5 level set is a sphere of radius 6; the second one is cut by the
    # volume boundary, so caps close it
    ny, nx, nz = 20, 21, 19
    y, x, z = np.meshgrid(np.arange(1, ny + 1), np.arange(1, nx + 1), np.arange(1, nz + 1), indexing="ij")
    cx, cy, cz = center
    # the file flips y: the sample in row i sits at MATLAB y = ny - i
    d = np.sqrt((x - cx) ** 2 + ((ny + 1 - y) - cy) ** 2 + (z - cz) ** 2)
    vol = 1.0 / (1.0 + np.exp(d - 6.0)) + 1e-9
    rec = _write_stl(tmp_path, vol)
    tris = rec["v"]
    _closed_and_oriented(tris)
    V = _volume(tris)
    if center[0] > 6.5:
        assert abs(V - 4.0 / 3.0 * np.pi * 6.0 ** 3) < 0.03 * 4.0 / 3.0 * np.pi * 6.0 ** 3
    else:  # cut by the plane x = 1
        h = 6.0 - (center[0] - 1.0)
        cap = np.pi * h * h * (3 * 6.0 - h) / 3.0
        assert abs(V - (4.0 / 3.0 * np.pi * 6.0 ** 3 - cap)) < 0.04 * 4.0 / 3.0 * np.pi * 6.0 ** 3
    mid = tris.astype(np.float64).mean(axis=(0, 1))
    assert np.allclose(mid, center, atol=0.5 if center[0] > 6.5 else 2.5)


def test_empty_and_bad_arguments(tmp_path):
    lib, L = _lib()
    rec = _write_stl(tmp_path, np.zeros((4, 4, 4)))
    assert len(rec) == 0
    v = np.zeros(8)
    assert lib.topx_write_design_stl(v.ctypes.data_as(C.POINTER(C.c_double)), 1, 2, 4, 0.5, b"/tmp/x.stl",
                                     None) == -1
    assert lib.topx_write_design_stl(v.ctypes.data_as(C.POINTER(C.c_double)), 2, 2, 2, 0.5,
                                     str(tmp_path / "no" / "dir.stl").encode(), None) == -1
