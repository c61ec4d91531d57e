"""GPU rasteriser (include/rt_raster.h) against the oracle, which is pinned to
the reference's rasteriser kernel (tests/test_oracle_raster.py): face id,
(u, v) and depth bit for bit, for face-index ids and for the reference's
block-start ids; pre-filled depth surfaces; a scene whose pairs need several
chunks; faces drawn twice (exact depth ties); and a 1920 x 1080 frame of the
2^20-face soup."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup(oracle, mesh, center, target, w, h, roll=0.0):
    from cudart_b200 import core
    fov = float(np.float32(np.pi / 3))
    ratio = float(np.float32(w) / np.float32(h))
    cam = core.make_camera(center, target, fov=fov, ratio=ratio)
    cam.angle[2] = roll
    m = core.raster_matrix(cam, target)
    v = torch.from_numpy(mesh.vertices).cuda()
    f = torch.from_numpy(mesh.faces.view(np.int32)).cuda()
    return np.array(m, np.float32), v, f


def _compare(oracle, mesh, m, v, f, w, h, id_mode=0, depth0=None, pair_capacity=0):
    from cudart_b200 import core
    out = None
    if depth0 is not None:
        P = w * h
        out = dict(id=torch.zeros(P, dtype=torch.int32, device="cuda"), uv=torch.zeros((P, 2), dtype=torch.float32, device="cuda"),
                   depth=torch.from_numpy(depth0).cuda(), err=torch.zeros(1, dtype=torch.int32, device="cuda"))
    got = core.rasterize(v, f, m, w, h, id_mode=id_mode, out=out, pair_capacity=pair_capacity)
    torch.cuda.synchronize()
    assert int(got["err"].item()) == 0
    fo, uo, do = oracle.rasterize(mesh.vertices, mesh.faces, m, w, h, depths=depth0)
    hit = do != oracle.HUGE
    want_id = np.where(hit, fo // 192 * 192 if id_mode == 1 else fo, 0) if depth0 is None else (fo // 192 * 192 if id_mode else fo)
    assert np.array_equal(got["depth"].cpu().numpy().view(np.uint32), do.view(np.uint32))
    assert np.array_equal(got["uv"].cpu().numpy().view(np.uint32), uo.view(np.uint32))
    assert np.array_equal(got["id"].cpu().numpy().view(np.uint32), want_id.astype(np.uint32))
    return hit


@pytest.mark.parametrize("id_mode", [0, 1])
@pytest.mark.parametrize("case", ["terrain", "terrain_roll", "soup", "close"])
def test_raster_matches_oracle(oracle, case, id_mode):
    from cudart_b200 import scenes
    cases = {
        "terrain": (scenes.terrain(128, 0), (0.0, 1.5, -2.5), (0.0, 0.0, 0.0), 512, 384, 0.0),
        "terrain_roll": (scenes.terrain(64, 3), (0.3, 1.2, -2.0), (0.1, 0.0, 0.2), 333, 250, 0.3),
        "soup": (scenes.soup(100000, 5), (0.62, 0.71, -0.45), (0.5, 0.5, 0.5), 640, 360, 0.0),
        "close": (scenes.terrain(32, 4), (0.2, 0.35, -0.6), (0.0, 0.0, 0.3), 257, 131, 0.0),
    }
    mesh, center, target, w, h, roll = cases[case]
    m, v, f = _setup(oracle, mesh, center, target, w, h, roll)
    hit = _compare(oracle, mesh, m, v, f, w, h, id_mode)
    assert hit.mean() > 0.05


def test_raster_prefilled_depth(oracle):
    from cudart_b200 import scenes
    mesh = scenes.terrain(128, 0)
    w, h = 320, 240
    m, v, f = _setup(oracle, mesh, (0.0, 1.5, -2.5), (0.0, 0.0, 0.0), w, h)
    depth0 = np.random.default_rng(1).uniform(0.0, 1.2, w * h).astype(np.float32)
    _compare(oracle, mesh, m, v, f, w, h, depth0=depth0)


def test_raster_many_chunks(oracle):
    """600 screen-filling triangles at shuffled depths (with repeats): every
    face covers every zone, so at the smallest pair budget (128 faces' worth)
    the faces go through 5 chunks and the depth test carries across them."""
    from cudart_b200 import scenes
    rng = np.random.default_rng(4)
    k = 600
    z = rng.choice(np.linspace(2.0, 6.0, 300), k).astype(np.float32)
    jit = rng.uniform(-0.3, 0.3, (k, 3, 2)).astype(np.float32)
    v = np.zeros((3 * k, 4), np.float32)
    base = np.array([[-40.0, -40.0], [40.0, -40.0], [0.0, 40.0]], np.float32)
    v[:, :2] = (base[None] + jit).reshape(-1, 2)
    v[:, 2] = np.repeat(z, 3)
    faces = np.zeros((k, 4), np.uint32)
    faces[:, :3] = np.arange(3 * k, dtype=np.uint32).reshape(k, 3)
    mesh = scenes.Mesh(v, faces)
    w, h = 256, 128
    m, vv, ff = _setup(oracle, mesh, (0.01, 0.02, -1.0), (0.0, 0.0, 0.0), w, h)
    hit = _compare(oracle, mesh, m, vv, ff, w, h, pair_capacity=1)
    assert hit.mean() > 0.9


@pytest.mark.parametrize("pair_capacity", [0, 1])
def test_raster_exact_depth_ties(oracle, pair_capacity):
    """Every face drawn twice (the face list followed by itself, in reverse
    order in the copy): each covered pixel sees two faces at exactly the same
    depth, and the earlier index must win however the zone lists order them;
    at the smallest pair budget the two copies fall in different chunks."""
    from cudart_b200 import scenes
    src = scenes.soup(20000, 9)
    faces = np.concatenate([src.faces, src.faces[::-1]]).copy()
    mesh = scenes.Mesh(src.vertices, faces)
    w, h = 160, 96
    m, v, f = _setup(oracle, mesh, (0.62, 0.71, -0.45), (0.5, 0.5, 0.5), w, h)
    hit = _compare(oracle, mesh, m, v, f, w, h, pair_capacity=pair_capacity)
    assert hit.mean() > 0.05


def test_raster_full_frame_soup(oracle):
    from cudart_b200 import scenes
    mesh = scenes.soup(1 << 20, 1)
    m, v, f = _setup(oracle, mesh, (0.55, 0.6, -0.4), (0.5, 0.5, 0.5), 1920, 1080)
    _compare(oracle, mesh, m, v, f, 1920, 1080)
