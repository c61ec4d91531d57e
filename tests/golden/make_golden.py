"""Generates the golden fixtures in tests/golden/ from the reference's own code.

The reference ships no golden vectors or known-answer tests for this path (its
only self-check, samples/09_how_to_use_a_sorter.cpp, asserts sortedness of
time-seeded keys). These fixtures are therefore produced by running the
reference's own functions, compiled from its sources by oracle/build_ref.sh
(oracle/_ref/libref_cudart.so), on seeded synthetic scenes:

  terrain_c0.npz  128 x 128 terrain (32,258 triangles), 512 x 512 camera rays:
                  sorted codes, indices, nodes (bvnode words), reordered faces,
                  and per-ray hits (face position, t, u, v) for every 61st ray.
  soup_small.npz  soups of N in {1, 16, 17, 224, 225, 513, 5000} triangles:
                  nodes and indices per N.
  flatz.npz       a flat z = 0.5 plane (the node-box quirk).
  sah.npz         the reference's SAH kernels (kernels/CUDA_buildMeshTreeSAH.cu,
                  emulated blocks in serial order): nodes and indices of a full
                  SAH build of a 64 x 64 terrain and of a 5000-triangle soup, and
                  of the Hybrid build (LBVH depth 4, then SAH) of the terrain.
                  Internal nodes keep only bits 0-2 of their first word (the
                  reference leaves the rest unset).

Run:  CUDART_REFERENCE=<reference tree> make -C oracle   (builds oracle/_ref from the reference's sources)
      python tests/golden/make_golden.py [sah]           ("sah" writes sah.npz only)
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cudart_b200 import scenes  # noqa: E402
from oracle import api as O  # noqa: E402

RAY_STRIDE = 61
SOUP_SIZES = (1, 16, 17, 224, 225, 513, 5000)


def ref_build(mesh, tree_depth=12):
    hit = O.hitbox(mesh.vertices)
    boxes, _ = O.ref_mesh_boxes(mesh.vertices, mesh.faces)
    r = O.ref_lbvh_build(boxes, hit, tree_depth=tree_depth)
    faces = O.ref_reorder_faces(mesh.faces, r["indices"])
    return hit, boxes, r, faces


def main():
    if not O.ref_available():
        O.build()
    mesh, cam = scenes.terrain_small_scene()
    hit, boxes, r, faces = ref_build(mesh)
    o, d, basis, ang = O.ref_camera_rays(cam)
    tr = O.ref_trace(r["nodes"], mesh.vertices, faces, o, d, cam.width, cam.height)
    sel = np.arange(0, cam.width * cam.height, RAY_STRIDE)
    hit_mask = tr["t"][sel] != O.HUGE
    ids = np.where(hit_mask, tr["id"][sel].astype(np.int64), -1).astype(np.int32)
    uv = np.where(hit_mask[:, None], tr["uv"][sel], 0.0).astype(np.float32)
    np.savez_compressed(
        os.path.join(HERE, "terrain_c0.npz"),
        hitbox=hit, codes=r["codes"], indices=r["indices"], nodes=r["nodes"].view(np.uint32), faces=faces,
        basis=basis, angle=ang, ray_sel=sel.astype(np.int64), hit_id=ids, hit_t=tr["t"][sel], hit_uv=uv,
        boxes_sha256=np.frombuffer(hashlib.sha256(boxes.tobytes()).digest(), np.uint8),
        dirs_sha256=np.frombuffer(hashlib.sha256(d.tobytes()).digest(), np.uint8),
        real_depth=np.uint32(r["real_depth"]), split_count=np.uint32(r["split_count"]))
    out = {}
    for n in SOUP_SIZES:
        m = scenes.soup(n, seed=n)
        _, _, rr, _ = ref_build(m)
        out[f"nodes_{n}"] = rr["nodes"].view(np.uint32)
        out[f"indices_{n}"] = rr["indices"]
    np.savez_compressed(os.path.join(HERE, "soup_small.npz"), **out)
    m = flat_z_mesh()
    _, _, rr, _ = ref_build(m)
    np.savez_compressed(os.path.join(HERE, "flatz.npz"), nodes=rr["nodes"].view(np.uint32), indices=rr["indices"])
    print("golden fixtures written to", HERE)


def _mask_internal(nodes):
    w = nodes.view(np.uint32).copy()
    internal = (w[:, 0] & 1) == 0
    w[internal, 0] &= 7
    return w


def sah_fixtures():
    out = {}
    cases = {"terrain": (scenes.terrain(64, 2), None), "soup": (scenes.soup(5000, 4), None), "hybrid": (scenes.terrain(64, 2), 4)}
    for name, (m, depth) in cases.items():
        hit = O.hitbox(m.vertices)
        boxes, idx = O.ref_mesh_boxes(m.vertices, m.faces)
        if depth is None:
            st, nodes, ridx = O.ref_sah_build(boxes, hit, idx)
        else:
            lb = O.ref_lbvh_build(boxes, hit, tree_depth=depth, tree_complete=False)
            st, nodes, ridx = O.ref_sah_build(boxes, hit, lb["indices"], nodes_in=lb["nodes"])
        assert st == 0
        out[f"nodes_{name}"] = _mask_internal(nodes)
        out[f"indices_{name}"] = ridx
    np.savez_compressed(os.path.join(HERE, "sah.npz"), **out)


def flat_z_mesh():
    m = scenes.terrain(32, 3)
    v = m.vertices.copy()
    v[:, [1, 2]] = v[:, [2, 1]]
    v[:, 2] = 0.5
    return scenes.Mesh(v, m.faces)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "sah":
        sah_fixtures()
        print("sah.npz written to", HERE)
    else:
        main()
        sah_fixtures()
