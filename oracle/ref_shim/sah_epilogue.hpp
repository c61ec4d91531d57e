// sah_epilogue.hpp -- host driver around the reference's SAH kernels
// (kernels/CUDA_buildMeshTreeSAH.cu:224-666), restating the control flow of
// CUDA_buildMeshTreeSAH (:672-789) on host memory: push the root (or, for a
// tree that already has nodes, every leaf through kernel_initStack), then
// launch as many blocks as the stack holds until it is empty. Blocks run one
// after another (ShimBlockPool). The face boxes and the final face reorder are
// the callers' (ref_mesh_boxes / ref_reorder_faces). TEST INFRASTRUCTURE ONLY.
//
// Returns 0, 1 when the stack would overflow STACK_SIZE, 2 when the node count
// would pass `capacity` (the reference writes past its node buffer then: it
// never terminates on a node of >= MAX_LEAF_SIZE faces whose centroids share one bin).
REF_API int ref_sah_build(const float* boxes, const float* root_box, uint* indices, uint n, const bvnode* nodes_in,
                          uint node_count_in, bvnode* nodes_out, uint capacity, uint* node_count_out) {
  tex_boxes.ptr = (const float4*)boxes;
  std::vector<uint> indices_buffer(n + 1);
  std::vector<bvnode> nodes_buffer((size_t)capacity + 64);
  sp = 0;
  if (node_count_in == 0) {
    item it;
    it.node_id = 0;
    it.node_box.min = make_float4(root_box[0], root_box[1], root_box[2], root_box[3]);
    it.node_box.max = make_float4(root_box[4], root_box[5], root_box[6], root_box[7]);
    it.obj_id = 0;
    it.obj_bound = (int)n;
    stack[sp++] = it;
    node_count = 1;
  } else {
    for (uint k = 0; k < node_count_in; ++k) nodes_buffer[k] = nodes_in[k];
    node_count = node_count_in;
    blockDim.x = 32;
    for (uint k = 0; k < node_count_in; ++k) {
      blockIdx.x = k / 32;
      threadIdx.x = k % 32;
      kernel_initStack(nodes_buffer.data(), node_count_in);
    }
  }
  int status = 0;
  {
    ShimBlockPool pool;
    blockDim.x = 32;
    while (status == 0 && sp > 0) {
      if (sp >= STACK_SIZE) { status = 1; break; }
      const int blocks = sp;
      for (int b = 0; b < blocks; ++b) {
        blockIdx.x = (unsigned)b;
        pool.run([&] { kernel_buildMeshTree(indices, indices_buffer.data(), nodes_buffer.data()); });
        if (node_count + 2 > capacity) { status = 2; break; }
        if (sp >= STACK_SIZE) { status = 1; break; }
      }
    }
  }
  const uint count = node_count < capacity ? node_count : capacity;
  for (uint k = 0; k < count; ++k) nodes_out[k] = nodes_buffer[k];
  *node_count_out = node_count;
  return status;
}
