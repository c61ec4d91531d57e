// lbvh_epilogue.hpp -- drives the reference's own Morton, split, topology and
// bounding-box code (compiled from kernels/CUDA_buildMeshTreeLBVH.cu) in the
// order of CUDA_buildMeshTreeLBVH (:457-681), one simulated thread at a time.
// The GPU sorts of the reference are replaced by a stable sort (code, index),
// which is the tie rule of this build; the per-level split lists come out of
// the sequential split finder in position order, so every level is sorted.
// TEST INFRASTRUCTURE ONLY.

template <typename F>
static void shim_launch1d(uint count, uint block, F&& body) {
  uint grid = (count + block - 1) / block;
  blockDim = {block, 1, 1};
  for (uint b = 0; b < grid; ++b)
    for (uint t = 0; t < block; ++t) { blockIdx = {b, 0, 0}; threadIdx = {t, 0, 0}; body(); }
}

// info_out: node_count, real_depth, split_count
REF_API uint ref_lbvh_build(const float* boxes, uint n, const float* hitbox8, uint tree_depth, int tree_complete,
                            uint* codes_out, uint* indices_out, float* nodes_out, uint node_cap, uint* info_out) {
  std::vector<uint> codes(n);
  tex_boxes.ptr = (const float4*)boxes;
  float4 hmin = make_float4(hitbox8[0], hitbox8[1], hitbox8[2], hitbox8[3]);
  float4 hmax = make_float4(hitbox8[4], hitbox8[5], hitbox8[6], hitbox8[7]);
  shim_launch1d(n, BLOCK_SIZE, [&] { kernel_calcMortonCodes(codes.data(), hmin, hmax, n); });

  std::vector<uint> idx(n);
  std::iota(idx.begin(), idx.end(), 0u);
  std::stable_sort(idx.begin(), idx.end(), [&](uint a, uint b) { return codes[a] < codes[b]; });
  std::vector<uint> sorted(n);
  for (uint i = 0; i < n; ++i) sorted[i] = codes[idx[i]];

  split_count = 0;
  memset(level_split_count, 0, sizeof(level_split_count));
  std::vector<uint> s_idx(n + 1), s_lvl(n + 1);
  tex_codes.ptr = sorted.data();
  if (n > 1) shim_launch1d(n, BLOCK_SIZE, [&] { kernel_findSplits(s_idx.data(), s_lvl.data(), n); });
  std::vector<uint> order(split_count);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint a, uint b) { return s_lvl[a] < s_lvl[b]; });
  std::vector<uint> splits(split_count + 1);
  for (uint i = 0; i < split_count; ++i) splits[i] = s_idx[order[i]];
  uint host_level_split_count[32];
  memcpy(host_level_split_count, level_split_count, sizeof(host_level_split_count));

  std::vector<bvnode> nodes((size_t)2 * n + 64);
  memset(nodes.data(), 0, nodes.size() * sizeof(bvnode));
  uint node_count = 0, real_depth = 0;
  buildMeshTree(host_level_split_count, nodes.data(), node_count, splits.data(), n, tree_complete != 0, tree_depth, real_depth);

  tex_indices.ptr = idx.data();
  tex_boxes.ptr = (const float4*)boxes;
  for (uint k = 0; k < real_depth; ++k)
    shim_launch1d(node_count, BLOCK_SIZE, [&] { kernel_calcBoundingBoxes(nodes.data(), node_count, k); });

  memcpy(codes_out, sorted.data(), n * 4);
  memcpy(indices_out, idx.data(), n * 4);
  uint* w = (uint*)nodes_out;
  for (uint k = 0; k < node_count && k < node_cap; ++k) {
    const bvnode& b = nodes[k];
    uint w0 = isLeaf(b) ? (1u | ((uint)b.leaf.obj_count << 1)) : ((uint)b.node.axis << 1);
    uint w1 = isLeaf(b) ? b.leaf.obj_id : b.node.child_id;
    w[8 * k + 0] = w0; w[8 * k + 1] = w1;
    memcpy(&w[8 * k + 2], &b.box_min, 12);
    memcpy(&w[8 * k + 5], &b.box_max, 12);
  }
  info_out[0] = node_count; info_out[1] = real_depth; info_out[2] = split_count;
  return node_count;
}
