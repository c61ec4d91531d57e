"""C-ABI library checks that need no GPU: it loads, exports every function
include/rt_core.h declares, refuses compute without a device (no CPU
fallback), and its host-side camera math equals the oracle's bit for bit."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from tests.conftest import cuda_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"^\s*(?:rt_status|const char\*|uint32_t|uint64_t)\s+(rt_\w+)\s*\(", text, re.M)))


def test_header_declarations_are_exported():
    from cudart_b200 import _abi
    lib = _abi.lib()
    declared = _declared("rt_core.h")
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) <= set(_abi.EXPORTS)
    proposal = _declared("rt_propose.h")
    assert len(proposal) >= 10
    for name in proposal:
        assert hasattr(lib, name), name
    assert set(proposal) == set(_abi.PROPOSE_EXPORTS)
    raster = _declared("rt_raster.h")
    assert set(raster) == set(_abi.RASTER_EXPORTS)
    for name in raster:
        assert hasattr(lib, name), name
    sah = _declared("rt_sah.h")
    assert set(sah) == set(_abi.SAH_EXPORTS)
    for name in sah:
        assert hasattr(lib, name), name


def test_status_strings_and_version():
    from cudart_b200 import _abi
    lib = _abi.lib()
    assert lib.rt_status_string(0) == b"ok"
    assert lib.rt_status_string(2) == b"no CUDA device"
    assert lib.rt_version() >= 100


@pytest.mark.skipif(cuda_available(), reason="checks the no-device path")
def test_no_cpu_fallback():
    from cudart_b200 import _abi
    lib = _abi.lib()
    assert lib.rt_device_check() == 2
    assert lib.rt_radix_sort_pairs(None, None, 0, 32, 0, None, 0, None) == 2
    desc = _abi.TraceDesc()
    desc.nodes = desc.orig = desc.dir = desc.hit_id = desc.hit_t = desc.hit_uv = desc.tris = 16  # never dereferenced
    assert lib.rt_trace_closest(C.byref(desc), None) == 2


def test_invalid_arguments_rejected():
    from cudart_b200 import _abi
    lib = _abi.lib()
    assert lib.rt_lbvh_build(None, None) == 1
    nb = C.c_size_t(0)
    assert lib.rt_lbvh_scratch_bytes(0, None, C.byref(nb), None) == 1
    assert lib.rt_reorder_faces(C.c_void_p(4096), C.c_void_p(64), 100, C.c_void_p(4096 + 16), None) == 1  # overlap


def test_ray_count_above_limit_refused():
    """More than RT_MAX_RAYS rays is refused before the device check (single and batched traces); the limit itself
    passes the argument checks, so only the missing device stops it. So are bounce outputs given in part, or with
    face ids (id_mode 1) as hit ids."""
    from cudart_b200 import _abi
    lib = _abi.lib()
    desc = _abi.TraceDesc()
    desc.nodes = desc.orig = desc.dir = desc.hit_id = desc.hit_t = desc.hit_uv = desc.tris = 16  # never dereferenced
    desc.ray_count = _abi.MAX_RAYS + 1
    assert lib.rt_trace_closest(C.byref(desc), None) == 1
    desc.ray_count = _abi.MAX_RAYS
    assert lib.rt_trace_closest(C.byref(desc), None) == 2
    b = _abi.BatchTraceDesc()
    b.mesh_count, b.face_count = 2, 8
    b.face_offsets = b.ray_offsets = b.accel = b.tris = b.orig = b.dir = b.hit_id = b.hit_t = b.hit_uv = 16
    b.ray_count = 0xFFFFFFFF
    assert lib.rt_batch_trace(C.byref(b), None) == 1
    b.ray_count = _abi.MAX_RAYS
    assert lib.rt_batch_trace(C.byref(b), None) == 2
    # bounce outputs: all three or none, and only with positions as hit ids
    b.ray_count = 64
    b.bounce_orig = 16
    assert lib.rt_batch_trace(C.byref(b), None) == 1
    b.bounce_dir = b.bounce_tmax = 16  # all three given, but sharing bytes with each other and the rays
    assert lib.rt_batch_trace(C.byref(b), None) == 1
    base = 1 << 20  # separate, never dereferenced ranges of 64 rays
    b.orig, b.dir, b.tmax, b.hit_id, b.hit_t, b.hit_uv = (base + k * 4096 for k in range(6))
    b.bounce_orig, b.bounce_dir, b.bounce_tmax = (base + k * 4096 for k in range(6, 9))
    assert lib.rt_batch_trace(C.byref(b), None) == 2
    b.bounce_dir = b.orig + 512  # overlaps the origins
    assert lib.rt_batch_trace(C.byref(b), None) == 1
    b.bounce_dir = base + 9 * 4096
    b.id_mode, b.indices = 1, 16
    assert lib.rt_batch_trace(C.byref(b), None) == 1


def test_pack_hits_refusals():
    """rt_pack_hits: scratch sized by its query, null outputs and too small a scratch refused before the device
    check; a well-formed call stops only at the missing device."""
    from cudart_b200 import _abi
    lib = _abi.lib()
    nb = C.c_size_t(0)
    assert lib.rt_pack_hits_scratch_bytes(100000, C.byref(nb)) == 0 and nb.value >= 4 * (100000 // 2048)
    F = 1 << 20
    assert lib.rt_pack_hits(F, F, F, 100000, F, None, F, nb.value, None) == 1  # no count word
    assert lib.rt_pack_hits(F, F, None, 100000, F, F, F, nb.value, None) == 1  # no uv
    assert lib.rt_pack_hits(F, F, F, 100000, F, F, F, nb.value - 1, None) == 4  # RT_ERR_SCRATCH_TOO_SMALL
    assert lib.rt_pack_hits(F, F, F, _abi.MAX_RAYS + 1, F, F, F, 1 << 40, None) == 1
    assert lib.rt_pack_hits(F, F, F, 100000, F, F, F, nb.value, None) == 2


def test_scratch_queries():
    from cudart_b200 import core
    nb, mx = core.lbvh_scratch_bytes(1 << 20)
    assert mx == 2 * (1 << 20) - 1
    assert nb > 8 * (1 << 20)


@pytest.mark.parametrize("scene", ["terrain", "soup"])
def test_camera_host_math_matches_oracle(oracle, scene):
    from cudart_b200 import core, scenes
    cam = scenes.terrain_small_scene()[1] if scene == "terrain" else scenes.soup_1m_scene()[1]
    c = core.make_camera(cam.center, cam.target, fov=cam.fov, ratio=cam.ratio)
    ang = np.array(list(c.angle), np.float32)
    assert np.array_equal(ang.view(np.uint32), oracle.camera_look_at(cam.center, cam.target).view(np.uint32))
    basis = np.array(core.camera_basis(c, cam.width, cam.height), np.float32)
    ob = oracle.camera_basis(cam.center, ang, cam.fov, cam.ratio, cam.width, cam.height)
    assert np.array_equal(basis.view(np.uint32), ob.view(np.uint32))


_STRUCTS = {  # C typedef -> ctypes mirror in cudart_b200._abi
    "rt_build_params": "BuildParams", "rt_build_info": "BuildInfo", "rt_build_desc": "BuildDesc", "rt_trace_desc": "TraceDesc",
    "rt_interp_desc": "InterpDesc", "rt_mesh_file": "MeshFile", "rt_tree_file": "TreeFile", "rt_batch_build_desc": "BatchBuildDesc",
    "rt_batch_trace_desc": "BatchTraceDesc", "rt_sah_desc": "SahDesc", "rt_raster_desc": "RasterDesc", "rt_gemm_desc": "GemmDesc",
    "rt_gemm_argmax_desc": "GemmArgmaxDesc", "rt_feature_desc": "FeatureDesc", "rt_adam_desc": "AdamDesc", "rt_slot_desc": "SlotDesc",
    "rt_seed_desc": "SeedDesc", "rt_batch_gather_desc": "BatchGatherDesc", "rt_batch_slot_desc": "BatchSlotDesc", "rt_camera": "Camera",
    "rt_mlp_propose_desc": "MlpProposeDesc", "rt_gemm_xent_desc": "GemmXentDesc",
}


def test_struct_layouts_match_headers(tmp_path):
    """Every ctypes mirror has the C struct's size and each field's offset
    (a C probe compiled with gcc against include/*.h prints them)."""
    import shutil
    import subprocess

    from cudart_b200 import _abi
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "rt_core.h"', '#include "rt_sah.h"', '#include "rt_raster.h"',
             '#include "rt_propose.h"', "int main(void) {"]
    for cname, pyname in _STRUCTS.items():
        st = getattr(_abi, pyname)
        lines.append(f'  printf("{pyname} size %zu\\n", sizeof({cname}));')
        for f in st._fields_:
            lines.append(f'  printf("{pyname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    inc = os.path.join(ROOT, "include")
    r = subprocess.run(["gcc", "-std=c11", "-I", inc, str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            py, field, val = ln.split()
            got[(py, field)] = int(val)
    for pyname in _STRUCTS.values():
        st = getattr(_abi, pyname)
        assert got[(pyname, "size")] == C.sizeof(st), pyname
        for f in st._fields_:
            assert got[(pyname, f[0])] == getattr(st, f[0]).offset, (pyname, f[0])
