"""Rasteriser oracle (or_raster_matrix / or_rasterize) pinned to the reference's
own code: CUDACamera::update + the float4x4 helpers, and
kernel_rasterizeMeshTree run as the reference launches it (2 x 2 blocks of
8 x 4 threads on host threads). Depth and (u, v) bit for bit; the face id is
the face's index here, the first index of its 192-face cache block in the
reference (it writes its cache-loop counter `k`,
kernels/CUDA_rasterizeMeshTree.cu:212)."""
import numpy as np
import pytest

from cudart_b200 import scenes

_ref = pytest.mark.skipif(not __import__("oracle.api", fromlist=["x"]).ref_available(), reason="reference tree not present")


def _camera(oracle, center, target, fov, ratio, roll=0.0):
    ang = oracle.camera_look_at(center, target)
    return oracle.look_dir(center, target), np.array([ang[0], ang[1], roll], np.float32)


CASES = {
    "terrain": lambda: (scenes.terrain(128, 0), (0.0, 1.5, -2.5), (0.0, 0.0, 0.0), 160, 120),
    "terrain_roll": lambda: (scenes.terrain(64, 3), (0.3, 1.2, -2.0), (0.1, 0.0, 0.2), 128, 96),
    "soup": lambda: (scenes.soup(20000, 5), (0.62, 0.71, -0.45), (0.5, 0.5, 0.5), 144, 96),
    "close": lambda: (scenes.terrain(32, 4), (0.2, 0.35, -0.6), (0.0, 0.0, 0.3), 136, 100),
}


@_ref
@pytest.mark.parametrize("case", sorted(CASES))
def test_raster_matches_reference_code(oracle, case):
    mesh, center, target, w, h = CASES[case]()
    fov = float(np.float32(np.pi / 3))
    ratio = float(np.float32(w) / np.float32(h))
    d, angle = _camera(oracle, center, target, fov, ratio, roll=0.3 if case == "terrain_roll" else 0.0)
    m = oracle.raster_matrix(center, d, angle, fov, ratio)
    assert np.array_equal(m.view(np.uint32), oracle.ref_raster_matrix(center, d, angle, fov, ratio).view(np.uint32))
    fo, uo, do = oracle.rasterize(mesh.vertices, mesh.faces, m, w, h)
    fr, ur, dr = oracle.ref_rasterize(mesh.vertices, mesh.faces, m, w, h)
    hit = do != oracle.HUGE
    assert hit.sum() > 0.05 * hit.size
    assert np.array_equal(do.view(np.uint32), dr.view(np.uint32))
    assert np.array_equal(uo.view(np.uint32), ur.view(np.uint32))
    assert np.array_equal(np.where(hit, fo // 192 * 192, 0), fr)


@_ref
def test_camera_along_z_has_no_up_axis(oracle):
    """A camera looking exactly along z: the reference's roll axis (dir.x, 0,
    dir.y) is zero, its normalisation NaN, so the view matrix is NaN and
    nothing is drawn (CUDACamera.cpp:248-251). The oracle agrees."""
    d, angle = _camera(oracle, (0.5, 0.5, -0.4), (0.5, 0.5, 0.5), 1.0, 1.0)
    m = oracle.raster_matrix((0.5, 0.5, -0.4), d, angle, 1.0, 1.0)
    mr = oracle.ref_raster_matrix((0.5, 0.5, -0.4), d, angle, 1.0, 1.0)
    assert np.isnan(m).any() and np.array_equal(np.isnan(m), np.isnan(mr))


def test_raster_depth_order(oracle):
    """Two overlapping quads: the nearer wins regardless of face order, and on
    an exact depth tie the earlier face wins."""
    v = np.array([[-1, -1, 2, 0], [1, -1, 2, 0], [-1, 1, 2, 0], [1, 1, 2, 0],
                  [-1, -1, 3, 0], [1, -1, 3, 0], [-1, 1, 3, 0], [1, 1, 3, 0]], np.float32)
    far = [[4, 5, 6, 0], [5, 7, 6, 0]]
    near = [[0, 1, 2, 0], [1, 3, 2, 0]]
    d, angle = _camera(oracle, (0.01, 0.02, -2.0), (0.0, 0.0, 0.0), 1.2, 1.0)
    m = oracle.raster_matrix((0.01, 0.02, -2.0), d, angle, 1.2, 1.0)
    for faces, near_ids in ((np.array(far + near, np.uint32), {2, 3}), (np.array(near + far, np.uint32), {0, 1})):
        fid, uv, dep = oracle.rasterize(v, faces, m, 64, 64)
        hit = dep != oracle.HUGE
        assert hit.sum() > 100 and set(np.unique(fid[hit])) <= near_ids
    dup = np.array(near + near, np.uint32)
    fid, _, dep = oracle.rasterize(v, dup, m, 64, 64)
    assert set(np.unique(fid[dep != oracle.HUGE])) <= {0, 1}


@pytest.mark.parametrize("case", sorted(CASES))
def test_host_raster_matrix_matches_oracle(oracle, case):
    """rt_raster_matrix (host code of the C ABI, no device needed) equals the oracle bit for bit."""
    from cudart_b200 import core
    mesh, center, target, w, h = CASES[case]()
    fov = float(np.float32(np.pi / 3))
    ratio = float(np.float32(w) / np.float32(h))
    roll = 0.3 if case == "terrain_roll" else 0.0
    d, angle = _camera(oracle, center, target, fov, ratio, roll=roll)
    cam = core.make_camera(center, target, fov=fov, ratio=ratio)
    cam.angle[2] = roll
    m = np.array(core.raster_matrix(cam, target), np.float32)
    assert np.array_equal(m.view(np.uint32), oracle.raster_matrix(center, d, angle, fov, ratio).view(np.uint32))
