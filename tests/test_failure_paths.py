"""Failure paths, made without a GPU fault.

Host side (any machine; the checks run before the device check, so no buffer
is touched): a build whose node array is smaller than 2N - 1 nodes is refused
with RT_ERR_CAPACITY, a build / batched build / sort whose scratch or blob is
too small with RT_ERR_SCRATCH_TOO_SMALL, all before the first launch.

Device side (-m gpu): the bounded wait that every tensor-core kernel uses runs
out on a barrier nothing arrives at (a 1 ms limit), reports
RT_DEVERR_WAIT_TIMEOUT and returns; the kernel releases its tensor memory, so
the context stays usable and a GEMM afterwards is exact against torch.
"""
import ctypes as C

import pytest

from tests.conftest import cuda_available

RT_ERR_SCRATCH_TOO_SMALL = 4
RT_ERR_CAPACITY = 5
FAKE = 1 << 40  # a non-null pointer value that no check reaches far enough to use


def _build_desc(n, max_nodes, scratch_bytes, accel_bytes=0):
    from cudart_b200 import _abi
    d = _abi.BuildDesc()
    d.vertices = d.faces_in = d.faces_out = d.boxes = d.indices = d.nodes = d.tris = FAKE
    d.vertex_count, d.face_count = 3 * n, n
    d.params = _abi.BuildParams(12, 1, 0, 0, 32)
    d.max_nodes = max_nodes
    d.scratch, d.scratch_bytes = FAKE, scratch_bytes
    if accel_bytes:
        d.accel, d.accel_bytes = FAKE, accel_bytes
    return d


@pytest.mark.skipif(cuda_available(), reason="host-side refusals, checked where no buffer can be touched")
def test_build_refusals_before_launch():
    from cudart_b200 import _abi, core
    lib = _abi.lib()
    n = 100000
    need, max_nodes = core.lbvh_scratch_bytes(n)
    assert max_nodes == 2 * n - 1
    acc = core.accel_bytes(n)
    # node array one short of 2N - 1: refused whatever else is wrong
    assert lib.rt_lbvh_build(C.byref(_build_desc(n, max_nodes - 1, need)), None) == RT_ERR_CAPACITY
    assert lib.rt_lbvh_build(C.byref(_build_desc(n, 1, 0)), None) == RT_ERR_CAPACITY
    # scratch or traversal blob too small (the queried sizes carry a little slack, so halve them)
    assert lib.rt_lbvh_build(C.byref(_build_desc(n, max_nodes, need // 2)), None) == RT_ERR_SCRATCH_TOO_SMALL
    assert lib.rt_lbvh_build(C.byref(_build_desc(n, max_nodes, need, acc // 2)), None) == RT_ERR_SCRATCH_TOO_SMALL
    # everything large enough: only the missing device stops it
    assert lib.rt_lbvh_build(C.byref(_build_desc(n, max_nodes, need, acc)), None) == 2


@pytest.mark.skipif(cuda_available(), reason="host-side refusals, checked where no buffer can be touched")
def test_batch_build_and_sort_refusals_before_launch():
    from cudart_b200 import _abi
    lib = _abi.lib()
    M, N = 4, 40000
    params = _abi.BuildParams(12, 1, 0, 0, 32)
    sb, ab = C.c_size_t(0), C.c_size_t(0)
    assert lib.rt_batch_sizes(M, N, C.byref(params), C.byref(sb), C.byref(ab)) == 0
    d = _abi.BatchBuildDesc()
    d.mesh_count, d.face_count, d.vertex_count = M, N, 3 * N
    d.face_offsets = d.vertex_offsets = d.vertices = d.faces_in = d.boxes = d.indices = d.codes = d.nodes = d.tris = FAKE
    d.faces_out = FAKE + 4096
    d.accel, d.info, d.scratch = FAKE, FAKE, FAKE
    d.params = params
    d.accel_bytes, d.scratch_bytes = ab.value, sb.value // 2
    assert lib.rt_batch_build(C.byref(d), None) == RT_ERR_SCRATCH_TOO_SMALL
    d.accel_bytes, d.scratch_bytes = ab.value // 2, sb.value
    assert lib.rt_batch_build(C.byref(d), None) == RT_ERR_SCRATCH_TOO_SMALL
    d.accel_bytes = ab.value
    assert lib.rt_batch_build(C.byref(d), None) == 2
    n = 5000  # above one 4096-key tile: the sort needs scratch
    nb = C.c_size_t(0)
    assert lib.rt_sort_scratch_bytes(n, C.byref(nb)) == 0
    assert lib.rt_radix_sort_pairs(C.c_void_p(FAKE), C.c_void_p(FAKE), n, 32, 0, C.c_void_p(FAKE), nb.value - 1, None) == \
        RT_ERR_SCRATCH_TOO_SMALL
    assert lib.rt_radix_sort_pairs(C.c_void_p(FAKE), C.c_void_p(FAKE), n, 32, 0, None, nb.value, None) == RT_ERR_SCRATCH_TOO_SMALL
    assert lib.rt_radix_sort_keys(C.c_void_p(FAKE), n, 32, C.c_void_p(FAKE), 16, None) == RT_ERR_SCRATCH_TOO_SMALL
    assert lib.rt_radix_sort_pairs(C.c_void_p(FAKE), C.c_void_p(FAKE), n, 32, 0, C.c_void_p(FAKE), nb.value, None) == 2


@pytest.mark.skipif(cuda_available(), reason="host-side refusals, checked where no buffer can be touched")
def test_cluster_tree_and_batched_rays_refusals_before_launch():
    """A cluster tree with leaves of more than 8 positions is refused (RT_ERR_UNSUPPORTED) before any launch, single
    and batched; the scratch of a build with the cluster tree is larger than without; rt_batch_primary_rays refuses
    a null pointer or an empty image before the device check, and more than 2^32 rays in all."""
    from cudart_b200 import _abi, core
    lib = _abi.lib()
    n = 100000
    plain, max_nodes = core.lbvh_scratch_bytes(n)
    with_clusters, _ = core.lbvh_scratch_bytes(n, clusters=True)
    assert with_clusters > plain + 60 * n  # arrival words, child pairs, child boxes and ranges per face
    acc = core.accel_bytes(n)
    d = _build_desc(n, max_nodes, with_clusters, acc)
    d.params = _abi.BuildParams(12, 1, 0, 0, 32, _abi.ACCEL_CLUSTERS, 9)
    assert lib.rt_lbvh_build(C.byref(d), None) == 6  # RT_ERR_UNSUPPORTED
    d.params = _abi.BuildParams(12, 1, 0, 0, 32, _abi.ACCEL_CLUSTERS, 3)
    assert lib.rt_lbvh_build(C.byref(d), None) == 2  # everything else in order: only the missing device stops it
    M, N = 4, 40000
    params = _abi.BuildParams(12, 1, 0, 0, 32, _abi.ACCEL_CLUSTERS, 9)
    sb, ab = C.c_size_t(0), C.c_size_t(0)
    assert lib.rt_batch_sizes(M, N, C.byref(params), C.byref(sb), C.byref(ab)) == 0
    b = _abi.BatchBuildDesc()
    b.mesh_count, b.face_count, b.vertex_count = M, N, 3 * N
    b.face_offsets = b.vertex_offsets = b.vertices = b.faces_in = b.boxes = b.indices = b.codes = b.nodes = b.tris = FAKE
    b.faces_out = FAKE + 4096
    b.accel, b.info, b.scratch = FAKE, FAKE, FAKE
    b.params = params
    b.accel_bytes, b.scratch_bytes = ab.value, sb.value
    assert lib.rt_batch_build(C.byref(b), None) == 6
    assert lib.rt_batch_primary_rays(None, 4, 8, 8, C.c_void_p(FAKE), C.c_void_p(FAKE), None) == 1
    assert lib.rt_batch_primary_rays(C.c_void_p(FAKE), 4, 0, 8, C.c_void_p(FAKE), C.c_void_p(FAKE), None) == 1
    assert lib.rt_batch_primary_rays(C.c_void_p(FAKE), 1 << 12, 1 << 10, 1 << 10, C.c_void_p(FAKE), C.c_void_p(FAKE), None) == 1
    assert lib.rt_batch_primary_rays(C.c_void_p(FAKE), 0, 8, 8, None, None, None) == 0  # nothing to make


@pytest.mark.gpu
def test_bounded_wait_runs_out_and_returns():
    import torch

    from cudart_b200 import _abi, proposal
    lib = _abi.lib()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    res = torch.full((2,), 7, dtype=torch.int32, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.rt_tc_wait_selftest(0, C.c_void_p(err.data_ptr()), C.c_void_p(res.data_ptr()), st) == 1
    for _ in range(2):  # twice: the first run released its tensor memory
        err.zero_()
        assert lib.rt_tc_wait_selftest(1000, C.c_void_p(err.data_ptr()), C.c_void_p(res.data_ptr()), st) == 0
        torch.cuda.synchronize()
        assert int(err.item()) & _abi.DEVERR_WAIT_TIMEOUT
        r = res.cpu().tolist()
        assert r[0] == 0  # the wait did not complete
        assert 1000 <= r[1] < 1_000_000, r  # it gave up after the limit, not at once and not never
    # the context is usable: a tensor-core GEMM afterwards runs clean and matches torch
    g = torch.Generator().manual_seed(1)
    a = torch.randn((256, 128), generator=g).to(torch.bfloat16).cuda()
    b = (torch.randn((128, 128), generator=g) * 0.1).to(torch.bfloat16).cuda()
    out = torch.empty((256, 128), device="cuda")
    err.zero_()
    proposal.gemm(a, b, out_f32=out, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = a.float() @ b.float().T
    assert float((out - ref).abs().max()) <= 1e-3 * float(ref.abs().max())
