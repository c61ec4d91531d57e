// file_epilogue.hpp -- drivers for the reference's quickSave / quickLoad.
// TEST INFRASTRUCTURE ONLY.
template <typename T>
static CUDAArray<T>* shim_array(const void* p, uint n) {
  if (!p) return nullptr;
  CUDAArray<T>* a = new CUDAArray<T>(n);
  a->copyDataFromHost((const T*)p);
  return a;
}
REF_API void ref_mesh_quick_save(const char* path, const float* hitbox8, const float* v, uint nv, const float* nrm, uint nn,
                                 const float* col, uint nc, const float* tex, uint nt, const uint* faces, uint nf) {
  CUDAMesh m;
  memcpy(&m.hitbox, hitbox8, 32);
  m.vertices = shim_array<float4>(v, nv);
  m.normals = shim_array<float4>(nrm, nn);
  m.colors = shim_array<float4>(col, nc);
  m.texcoords = shim_array<float2>(tex, nt);
  m.faces = shim_array<uint4>(faces, nf);
  m.quickSave((char*)path, true);
}
// counts_out: vertices, normals, colors, texcoords, faces; arrays filled when non-null and large enough
REF_API void ref_mesh_quick_load(const char* path, float* hitbox8, uint* counts_out, float* v, float* nrm, float* col, float* tex, uint* faces) {
  CUDAMesh m;
  m.quickLoad((char*)path);
  memcpy(hitbox8, &m.hitbox, 32);
  counts_out[0] = m.vertices ? m.vertices->getUnitCount() : 0;
  counts_out[1] = m.normals ? m.normals->getUnitCount() : 0;
  counts_out[2] = m.colors ? m.colors->getUnitCount() : 0;
  counts_out[3] = m.texcoords ? m.texcoords->getUnitCount() : 0;
  counts_out[4] = m.faces ? m.faces->getUnitCount() : 0;
  if (v && m.vertices) m.vertices->copyDataToHost((float4*)v);
  if (nrm && m.normals) m.normals->copyDataToHost((float4*)nrm);
  if (col && m.colors) m.colors->copyDataToHost((float4*)col);
  if (tex && m.texcoords) m.texcoords->copyDataToHost((float2*)tex);
  if (faces && m.faces) m.faces->copyDataToHost((uint4*)faces);
}
REF_API void ref_tree_quick_save(const char* path, const uint* nodes, uint nn, const uint* indices, uint ni, const float* boxes, uint nb) {
  CUDAMeshTree t;
  t.nodes = shim_array<bvnode>(nodes, nn);
  t.indices = shim_array<uint>(indices, ni);
  t.boxes = shim_array<aabox>(boxes, nb);
  t.quickSave((char*)path, true);
}
