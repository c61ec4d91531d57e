// rt_file.cpp -- the reference's mesh / tree chunk files (quickSave / quickLoad).
//
// Format (CUDAMesh.cpp:134-400, CUDAMeshTree.cpp:114-289): a sequence of
// chunks, each `int magic, int chunk_length (bytes, header included)`, then,
// for array chunks, `uint count` and count records; the hit-box chunk holds one
// aabox without a count. Readers skip unknown chunks by their length, so mesh
// and tree chunks can share one file. Files written here are byte-identical to
// the reference's quickSave(path, overwrite = true).
//
// Two reference defects are not reproduced:
//  * its tree loader asserts that the stored index / box counts DIFFER from the
//    tree's (CUDAMeshTree.cpp:166,182), so a valid file aborts; here the counts
//    must be equal;
//  * with overwrite = false it opens the file in append mode and then seeks
//    back to patch each chunk length, which append mode ignores; here each
//    chunk is written whole with its length known up front.
// Arrays move between the file and the caller's buffers, device or host memory
// (cudaPointerGetAttributes decides; without a device every pointer is host
// memory); the calls are synchronous (file I/O).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/rt_core.h"

namespace {

const int32_t kHitboxMagic = 0x3027AD79;
const int32_t kVerticesMagic = (int32_t)0xBA5C1CC7;
const int32_t kNormalsMagic = 0x1DD14C48;
const int32_t kColorsMagic = 0x757B31AB;
const int32_t kTexcoordsMagic = 0x2B77D260;
const int32_t kFacesMagic = (int32_t)0x8E934163;
const int32_t kNodesMagic = (int32_t)0x9077086B;
const int32_t kIndicesMagic = 0x2CC8BD7D;
const int32_t kBoxesMagic = (int32_t)0xE54B7842;

bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

bool copy_out(void* host, const void* src, size_t bytes) {
  if (!bytes) return true;
  if (on_device(src)) return cudaMemcpy(host, src, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
  std::memcpy(host, src, bytes);
  return true;
}

bool copy_in(void* dst, const void* host, size_t bytes) {
  if (!bytes) return true;
  if (on_device(dst)) return cudaMemcpy(dst, host, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  std::memcpy(dst, host, bytes);
  return true;
}

struct File {
  FILE* f = nullptr;
  explicit File(FILE* p) : f(p) {}
  ~File() { if (f) fclose(f); }
};

// One array chunk: magic, length, count, records (copied from the device).
bool write_array(FILE* f, int32_t magic, const void* dev, uint32_t count, size_t unit) {
  std::vector<unsigned char> host((size_t)count * unit);
  if (!copy_out(host.data(), dev, host.size())) return false;
  const int64_t len = 8 + 4 + (int64_t)host.size();
  if (len > 0x7FFFFFFF) return false;  // the format's length field is an int
  const int32_t len32 = (int32_t)len;
  return fwrite(&magic, 4, 1, f) == 1 && fwrite(&len32, 4, 1, f) == 1 && fwrite(&count, 4, 1, f) == 1 &&
         (host.empty() || fwrite(host.data(), 1, host.size(), f) == host.size());
}

struct Chunk {
  int32_t magic;
  long payload;  // file offset after the 8-byte header
  int32_t length;
  uint32_t count;
};

bool scan(FILE* f, std::vector<Chunk>& out) {
  if (fseek(f, 0, SEEK_END) != 0) return false;
  const long end = ftell(f);
  long off = 0;
  while (off + 8 <= end) {
    if (fseek(f, off, SEEK_SET) != 0) return false;
    int32_t hdr[2];
    if (fread(hdr, 4, 2, f) != 2) return false;
    if (hdr[1] < 8 || off + hdr[1] > end) return false;  // corrupt length
    Chunk c{hdr[0], off + 8, hdr[1], 0};
    if (hdr[0] != kHitboxMagic && hdr[1] >= 12 && fread(&c.count, 4, 1, f) != 1) return false;
    out.push_back(c);
    off += hdr[1];
  }
  return off == end;
}

const Chunk* find(const std::vector<Chunk>& cs, int32_t magic) {
  const Chunk* hit = nullptr;
  for (const Chunk& c : cs)
    if (c.magic == magic) hit = &c;  // the last chunk wins, as in the reference's sequential reader
  return hit;
}

rt_status read_array(FILE* f, const Chunk* c, void* dev, uint32_t capacity, size_t unit) {
  if (!c || !dev) return RT_OK;
  if (c->count != capacity) return RT_ERR_CAPACITY;
  if ((int64_t)c->length != 12 + (int64_t)c->count * (int64_t)unit) return RT_ERR_INVALID_ARGUMENT;
  std::vector<unsigned char> host((size_t)c->count * unit);
  if (fseek(f, c->payload + 4, SEEK_SET) != 0 || (host.size() && fread(host.data(), 1, host.size(), f) != host.size()))
    return RT_ERR_INVALID_ARGUMENT;
  if (!copy_in(dev, host.data(), host.size())) return RT_ERR_CUDA;
  return RT_OK;
}

}  // namespace

extern "C" rt_status rt_mesh_file_save(const char* path, int overwrite, const rt_mesh_file* m) {
  if (!path || !m) return RT_ERR_INVALID_ARGUMENT;
  File file(fopen(path, overwrite ? "wb" : "ab"));
  if (!file.f) return RT_ERR_INVALID_ARGUMENT;
  const int32_t hb_len = 8 + 32;
  if (fwrite(&kHitboxMagic, 4, 1, file.f) != 1 || fwrite(&hb_len, 4, 1, file.f) != 1 || fwrite(m->hitbox, 4, 8, file.f) != 8)
    return RT_ERR_INVALID_ARGUMENT;
  if (m->vertices && !write_array(file.f, kVerticesMagic, m->vertices, m->vertex_count, 16)) return RT_ERR_CUDA;
  if (m->normals && !write_array(file.f, kNormalsMagic, m->normals, m->normal_count, 16)) return RT_ERR_CUDA;
  if (m->colors && !write_array(file.f, kColorsMagic, m->colors, m->color_count, 16)) return RT_ERR_CUDA;
  if (m->texcoords && !write_array(file.f, kTexcoordsMagic, m->texcoords, m->texcoord_count, 8)) return RT_ERR_CUDA;
  if (m->faces && !write_array(file.f, kFacesMagic, m->faces, m->face_count, 16)) return RT_ERR_CUDA;
  return RT_OK;
}

extern "C" rt_status rt_mesh_file_info(const char* path, rt_mesh_file* m) {
  if (!path || !m) return RT_ERR_INVALID_ARGUMENT;
  File file(fopen(path, "rb"));
  if (!file.f) return RT_ERR_INVALID_ARGUMENT;
  std::vector<Chunk> cs;
  if (!scan(file.f, cs)) return RT_ERR_INVALID_ARGUMENT;
  std::memset(m, 0, sizeof(*m));
  if (const Chunk* c = find(cs, kHitboxMagic)) {
    if (c->length != 40 || fseek(file.f, c->payload, SEEK_SET) != 0 || fread(m->hitbox, 4, 8, file.f) != 8) return RT_ERR_INVALID_ARGUMENT;
    m->has_hitbox = 1;
  }
  if (const Chunk* c = find(cs, kVerticesMagic)) m->vertex_count = c->count;
  if (const Chunk* c = find(cs, kNormalsMagic)) m->normal_count = c->count;
  if (const Chunk* c = find(cs, kColorsMagic)) m->color_count = c->count;
  if (const Chunk* c = find(cs, kTexcoordsMagic)) m->texcoord_count = c->count;
  if (const Chunk* c = find(cs, kFacesMagic)) m->face_count = c->count;
  return RT_OK;
}

extern "C" rt_status rt_mesh_file_load(const char* path, rt_mesh_file* m) {
  if (!path || !m) return RT_ERR_INVALID_ARGUMENT;
  File file(fopen(path, "rb"));
  if (!file.f) return RT_ERR_INVALID_ARGUMENT;
  std::vector<Chunk> cs;
  if (!scan(file.f, cs)) return RT_ERR_INVALID_ARGUMENT;
  if (const Chunk* c = find(cs, kHitboxMagic)) {
    if (c->length != 40 || fseek(file.f, c->payload, SEEK_SET) != 0 || fread(m->hitbox, 4, 8, file.f) != 8) return RT_ERR_INVALID_ARGUMENT;
    m->has_hitbox = 1;
  }
  rt_status s;
  if ((s = read_array(file.f, find(cs, kVerticesMagic), m->vertices, m->vertex_count, 16)) != RT_OK) return s;
  if ((s = read_array(file.f, find(cs, kNormalsMagic), m->normals, m->normal_count, 16)) != RT_OK) return s;
  if ((s = read_array(file.f, find(cs, kColorsMagic), m->colors, m->color_count, 16)) != RT_OK) return s;
  if ((s = read_array(file.f, find(cs, kTexcoordsMagic), m->texcoords, m->texcoord_count, 8)) != RT_OK) return s;
  if ((s = read_array(file.f, find(cs, kFacesMagic), m->faces, m->face_count, 16)) != RT_OK) return s;
  return RT_OK;
}

extern "C" rt_status rt_tree_file_save(const char* path, int overwrite, const rt_tree_file* t) {
  if (!path || !t) return RT_ERR_INVALID_ARGUMENT;
  File file(fopen(path, overwrite ? "wb" : "ab"));
  if (!file.f) return RT_ERR_INVALID_ARGUMENT;
  if (t->nodes && !write_array(file.f, kNodesMagic, t->nodes, t->node_count, 32)) return RT_ERR_CUDA;
  if (t->indices && !write_array(file.f, kIndicesMagic, t->indices, t->index_count, 4)) return RT_ERR_CUDA;
  if (t->boxes && !write_array(file.f, kBoxesMagic, t->boxes, t->box_count, 32)) return RT_ERR_CUDA;
  return RT_OK;
}

extern "C" rt_status rt_tree_file_info(const char* path, rt_tree_file* t) {
  if (!path || !t) return RT_ERR_INVALID_ARGUMENT;
  File file(fopen(path, "rb"));
  if (!file.f) return RT_ERR_INVALID_ARGUMENT;
  std::vector<Chunk> cs;
  if (!scan(file.f, cs)) return RT_ERR_INVALID_ARGUMENT;
  std::memset(t, 0, sizeof(*t));
  if (const Chunk* c = find(cs, kNodesMagic)) t->node_count = c->count;
  if (const Chunk* c = find(cs, kIndicesMagic)) t->index_count = c->count;
  if (const Chunk* c = find(cs, kBoxesMagic)) t->box_count = c->count;
  return RT_OK;
}

extern "C" rt_status rt_tree_file_load(const char* path, rt_tree_file* t) {
  if (!path || !t) return RT_ERR_INVALID_ARGUMENT;
  File file(fopen(path, "rb"));
  if (!file.f) return RT_ERR_INVALID_ARGUMENT;
  std::vector<Chunk> cs;
  if (!scan(file.f, cs)) return RT_ERR_INVALID_ARGUMENT;
  rt_status s;
  if ((s = read_array(file.f, find(cs, kNodesMagic), t->nodes, t->node_count, 32)) != RT_OK) return s;
  if ((s = read_array(file.f, find(cs, kIndicesMagic), t->indices, t->index_count, 4)) != RT_OK) return s;
  if ((s = read_array(file.f, find(cs, kBoxesMagic), t->boxes, t->box_count, 32)) != RT_OK) return s;
  return RT_OK;
}
