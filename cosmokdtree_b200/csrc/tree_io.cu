// tree_io.cu -- save a built tree (or forest) to a file and load it back.
//
// The file holds the handle's scalars and every device array as a raw copy, so a
// loaded tree is bit-for-bit the tree that was saved and returns identical
// results without rebuilding.  Layout (little-endian): magic "CKDTREE2", a header
// of fixed-size scalars, the tree offsets (n_trees + 1 int64), then each array as
// (int64 byte count, bytes) in a fixed order.  No counterpart in the reference,
// which rebuilds its tree on every run.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ckd_common.cuh"

namespace ckd {
void release_tree_handle(ckd_tree* t);
}

using namespace ckd;

namespace {

struct Header {
  int64_t n, n_trees;
  int32_t d, leaf, periodic, input_dtype, n_nodes, n_leaves, depth, screen_ok;
  double L[CKD_MAX_D];
  float slack[CKD_MAX_D];
};

struct Arr {
  void** dev;
  size_t bytes;
};

std::vector<Arr> arrays(ckd_tree* t) {
  const size_t n = (size_t)t->n, m = (size_t)t->n_nodes, d = (size_t)t->d, nv = (d + 3) / 4;
  return {{(void**)&t->meta, sizeof(NodeMeta) * m},
          {(void**)&t->box, sizeof(double) * 2 * d * m},
          {(void**)&t->cell, sizeof(double) * 2 * d * m},
          {(void**)&t->pts, sizeof(double) * d * n},
          {(void**)&t->ids, sizeof(int32_t) * n},
          {(void**)&t->box32, sizeof(float) * 2 * d * m},
          {(void**)&t->pts32, sizeof(float4) * nv * n},
          {(void**)&t->pts64, sizeof(double4) * nv * n},
          {(void**)&t->pair, sizeof(float4) * pair_f4((int)d) * m},
          {(void**)&t->cell32, sizeof(float) * 2 * d * m},
          {(void**)&t->centre, sizeof(double) * d * m}};
}

struct File {
  FILE* f;
  explicit File(FILE* p) : f(p) {}
  ~File() {
    if (f) fclose(f);
  }
};

}  // namespace

extern "C" {

ckd_status ckd_tree_save(const ckd_tree* tree, const char* path) {
  if (!tree || !path) return fail(CKD_ERR_BAD_ARG, "null tree or path");
  int cur = 0;
  CKD_CUDA(cudaGetDevice(&cur));
  if (cur != tree->device) return fail(CKD_ERR_BAD_ARG, "the current device is not the tree's device");
  File fh(fopen(path, "wb"));
  if (!fh.f) return fail(CKD_ERR_BAD_ARG, std::string("cannot open ") + path + " for writing");
  ckd_tree* t = const_cast<ckd_tree*>(tree);
  Header h;
  std::memset(&h, 0, sizeof(h));
  h.n = t->n;
  h.n_trees = t->n_trees;
  h.d = t->d;
  h.leaf = t->leaf;
  h.periodic = t->periodic;
  h.input_dtype = t->input_dtype;
  h.n_nodes = t->n_nodes;
  h.n_leaves = t->n_leaves;
  h.depth = t->depth;
  h.screen_ok = t->screen_ok ? 1 : 0;
  std::memcpy(h.L, t->L, sizeof(h.L));
  std::memcpy(h.slack, t->slack, sizeof(h.slack));
  bool ok = fwrite("CKDTREE2", 1, 8, fh.f) == 8 && fwrite(&h, sizeof(h), 1, fh.f) == 1 &&
            fwrite(t->tree_off.data(), sizeof(int64_t), t->tree_off.size(), fh.f) ==
                t->tree_off.size();
  std::vector<unsigned char> buf;
  for (const Arr& a : arrays(t)) {
    if (!ok) break;
    int64_t bytes = (int64_t)a.bytes;
    buf.resize(a.bytes);
    CKD_CUDA(cudaMemcpy(buf.data(), *a.dev, a.bytes, cudaMemcpyDeviceToHost));
    ok = fwrite(&bytes, sizeof(bytes), 1, fh.f) == 1 && fwrite(buf.data(), 1, a.bytes, fh.f) == a.bytes;
  }
  if (!ok) return fail(CKD_ERR_BAD_ARG, std::string("write error on ") + path);
  return CKD_OK;
}

ckd_status ckd_tree_load(const char* path, ckd_tree** out) {
  if (!path || !out) return fail(CKD_ERR_BAD_ARG, "null path or output handle");
  *out = nullptr;
  File fh(fopen(path, "rb"));
  if (!fh.f) return fail(CKD_ERR_BAD_ARG, std::string("cannot open ") + path);
  char magic[8];
  Header h;
  if (fread(magic, 1, 8, fh.f) != 8 || std::memcmp(magic, "CKDTREE2", 8) != 0 ||
      fread(&h, sizeof(h), 1, fh.f) != 1)
    return fail(CKD_ERR_BAD_ARG, std::string(path) + " is not a saved tree");
  if (h.d < 1 || h.d > CKD_MAX_D || h.n < 1 || h.n_trees < 1 || h.n_nodes < 1 || h.n_trees > h.n)
    return fail(CKD_ERR_BAD_ARG, std::string(path) + ": corrupt header");
  int dev = 0;
  CKD_CUDA(cudaGetDevice(&dev));
  int major = 0;
  CKD_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  if (major != 10) return fail(CKD_ERR_NO_DEVICE, "libckd is built for sm_100a (B200) devices only");
  ckd_tree* t = new ckd_tree();
  t->device = dev;
  t->n = h.n;
  t->n_trees = h.n_trees;
  t->d = h.d;
  t->leaf = h.leaf;
  t->periodic = h.periodic;
  t->input_dtype = h.input_dtype;
  t->n_nodes = h.n_nodes;
  t->n_leaves = h.n_leaves;
  t->depth = h.depth;
  t->screen_ok = h.screen_ok != 0;
  std::memcpy(t->L, h.L, sizeof(h.L));
  std::memcpy(t->slack, h.slack, sizeof(h.slack));
  t->tree_off.resize((size_t)h.n_trees + 1);
  ckd_status st = CKD_OK;
  if (fread(t->tree_off.data(), sizeof(int64_t), t->tree_off.size(), fh.f) != t->tree_off.size())
    st = fail(CKD_ERR_BAD_ARG, std::string(path) + ": truncated");
  std::vector<unsigned char> buf;
  for (const Arr& a : arrays(t)) {
    if (st != CKD_OK) break;
    int64_t bytes = 0;
    if (fread(&bytes, sizeof(bytes), 1, fh.f) != 1 || bytes != (int64_t)a.bytes) {
      st = fail(CKD_ERR_BAD_ARG, std::string(path) + ": array size mismatch");
      break;
    }
    buf.resize(a.bytes);
    if (fread(buf.data(), 1, a.bytes, fh.f) != a.bytes) {
      st = fail(CKD_ERR_BAD_ARG, std::string(path) + ": truncated");
      break;
    }
    cudaError_t e = dev_alloc(a.dev, a.bytes, 0);  // legacy stream: ordered before the copy
    if (e == cudaSuccess) e = cudaMemcpy(*a.dev, buf.data(), a.bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) st = cuda_fail(e, "uploading a saved tree");
  }
  if (st != CKD_OK) {
    release_tree_handle(t);
    return st;
  }
  *out = t;
  return CKD_OK;
}

}  // extern "C"
