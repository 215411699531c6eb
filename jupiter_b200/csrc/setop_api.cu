// jgpm_setop / jgpm_setop_batch: the sorted-set operations as library calls.
//
// One warp per operand pair (warp-cooperative primitives of setops.cuh).  Host arrays are
// staged to the device and results copied back; device arrays are used in place.
#include <cuda_runtime.h>

#include <vector>

#include "jgpm_internal.h"
#include "setops.cuh"

namespace jgpm {
namespace {

__global__ void k_setop_batch(int op, const int32_t* a, const int64_t* a_off, const int32_t* b,
                              const int64_t* b_off, int64_t nops, const int32_t* upper,
                              const int32_t* exclude, int32_t* counts, int32_t* out,
                              const int64_t* out_off) {
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nops;
       i += warps) {
    const int32_t* A = a + a_off[i];
    const int na = (int)(a_off[i + 1] - a_off[i]);
    const int32_t* B = b + b_off[i];
    const int nb = (int)(b_off[i + 1] - b_off[i]);
    const int32_t up = upper ? upper[i] : INT32_MAX;
    const int32_t ex = exclude ? exclude[i] : -1;
    int c = 0;
    switch (op) {
      case JGPM_OP_INTERSECT:
        c = warp_intersect(A, na, B, nb, up, out + out_off[i]);
        break;
      case JGPM_OP_INTERSECT_COUNT:
        c = warp_intersect_count(A, na, B, nb, up, ex, -1);
        break;
      case JGPM_OP_DIFFERENCE:
        c = warp_difference(A, na, B, nb, up, ex, out + out_off[i]);
        break;
      case JGPM_OP_DIFFERENCE_COUNT:
        c = warp_difference(A, na, B, nb, up, ex, nullptr);
        break;
    }
    if ((threadIdx.x & 31) == 0) counts[i] = c;
  }
}

// Fused splits, one warp per pair; pair i's outputs sit at the offsets of its operands
// (c and d at a_off[i], e at b_off[i]).
__global__ void k_split_batch(int kind, const int32_t* a, const int64_t* a_off, const int32_t* b,
                              const int64_t* b_off, int64_t nops, const int32_t* upper,
                              int32_t* counts, int32_t* c, int32_t* d, int32_t* e) {
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nops;
       i += warps) {
    const int64_t a0 = a_off[i], b0 = b_off[i];
    const int32_t* A = a + a0;
    const int na = (int)(a_off[i + 1] - a0);
    const int32_t* B = b + b0;
    const int nb = (int)(b_off[i + 1] - b0);
    int r;
    if (kind == JGPM_SPLIT_FUSE) {
      r = na - warp_split_by(A, na, B, nb, INT32_MAX, c + a0, d + a0);  // |A & B|
      warp_split_by(B, nb, A, na, INT32_MAX, e + b0, nullptr);
    } else {
      r = warp_split_by(A, na, B, nb, upper ? upper[i] : INT32_MAX, c + a0, d + a0);
    }
    if ((threadIdx.x & 31) == 0) counts[i] = r;
  }
}

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

// Device copy of a caller array (host or device) of `count` elements.
template <typename T>
struct Staged {
  T* d = nullptr;
  bool owned = false;
  cudaError_t init(const T* src, size_t count, cudaStream_t s) {
    if (!src) return cudaSuccess;
    if (is_device_ptr(src)) {
      d = const_cast<T*>(src);
      return cudaSuccess;
    }
    owned = true;
    cudaError_t e = cudaMalloc((void**)&d, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return e;
    if (count) return cudaMemcpyAsync(d, src, count * sizeof(T), cudaMemcpyHostToDevice, s);
    return cudaSuccess;
  }
  ~Staged() {
    if (owned && d) cudaFree(d);
  }
};

// A caller's output array on the device: used in place when it is device memory, else a
// device copy of its current contents (so entries the kernel does not write keep their
// values either way) that back() returns to the caller.
struct OutArray {
  int32_t* user = nullptr;
  int32_t* d = nullptr;
  size_t n = 0;
  bool staged = false;
  cudaError_t init(int32_t* p, size_t count, cudaStream_t s) {
    user = p;
    n = count;
    if (!p) return cudaSuccess;
    if (is_device_ptr(p)) {
      d = p;
      return cudaSuccess;
    }
    staged = true;
    cudaError_t e = cudaMalloc((void**)&d, std::max<size_t>(count, 1) * sizeof(int32_t));
    if (e != cudaSuccess) return e;
    if (count) return cudaMemcpyAsync(d, p, count * sizeof(int32_t), cudaMemcpyHostToDevice, s);
    return cudaSuccess;
  }
  cudaError_t back(cudaStream_t s) {
    if (!staged || !n) return cudaSuccess;
    return cudaMemcpyAsync(user, d, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  }
  ~OutArray() {
    if (staged && d) cudaFree(d);
  }
};

}  // namespace
}  // namespace jgpm

using namespace jgpm;

extern "C" {

int jgpm_setop_batch(int op, const int32_t* a, const int64_t* a_off, const int32_t* b,
                     const int64_t* b_off, int64_t nops, const int32_t* upper,
                     const int32_t* exclude, int32_t* counts, int32_t* out,
                     const int64_t* out_off) {
  if (op < JGPM_OP_INTERSECT || op > JGPM_OP_DIFFERENCE_COUNT || nops < 0 || !a_off || !b_off ||
      !counts) {
    jgpm_set_error_("jgpm_setop_batch: bad arguments");
    return JGPM_EINVAL;
  }
  const bool mat = (op == JGPM_OP_INTERSECT || op == JGPM_OP_DIFFERENCE);
  if (mat && (!out || !out_off)) {
    jgpm_set_error_("jgpm_setop_batch: materialising ops need out and out_off");
    return JGPM_EINVAL;
  }
  if (nops == 0) return JGPM_OK;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    jgpm_set_error_("no CUDA device");
    return JGPM_ENODEV;
  }
  // offsets are needed on the host to size the staged lists and to check capacities
  std::vector<int64_t> ha(nops + 1), hb(nops + 1), ho;
  const bool offs_dev = is_device_ptr(a_off);
  JGPM_CUDA_TRY(cudaMemcpy(ha.data(), a_off, (nops + 1) * 8, cudaMemcpyDefault));
  JGPM_CUDA_TRY(cudaMemcpy(hb.data(), b_off, (nops + 1) * 8, cudaMemcpyDefault));
  (void)offs_dev;
  if (mat) {
    ho.resize(nops + 1);
    JGPM_CUDA_TRY(cudaMemcpy(ho.data(), out_off, (nops + 1) * 8, cudaMemcpyDefault));
  }
  if (ha[0] < 0 || hb[0] < 0 || (ha[nops] > 0 && !a) || (hb[nops] > 0 && !b)) {
    jgpm_set_error_("jgpm_setop_batch: bad offsets or missing operand array");
    return JGPM_EINVAL;
  }
  for (int64_t i = 0; i < nops; ++i) {
    const int64_t na = ha[i + 1] - ha[i], nb = hb[i + 1] - hb[i];
    if (na < 0 || nb < 0 || na > INT32_MAX || nb > INT32_MAX) {
      jgpm_set_error_("jgpm_setop_batch: bad offsets");
      return JGPM_EINVAL;
    }
    if (mat) {
      const int64_t need = op == JGPM_OP_INTERSECT ? std::min(na, nb) : na;
      if (ho[i + 1] - ho[i] < need) {
        jgpm_set_error_("jgpm_setop_batch: output capacity too small");
        return JGPM_ECAPACITY;
      }
    }
  }
  cudaStream_t s = nullptr;
  JGPM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{s};
  Staged<int32_t> da, db, dup, dex;
  Staged<int64_t> dao, dbo, doo;
  JGPM_CUDA_TRY(da.init(a, (size_t)ha[nops], s));
  JGPM_CUDA_TRY(db.init(b, (size_t)hb[nops], s));
  JGPM_CUDA_TRY(dao.init(a_off, (size_t)nops + 1, s));
  JGPM_CUDA_TRY(dbo.init(b_off, (size_t)nops + 1, s));
  JGPM_CUDA_TRY(dup.init(upper, (size_t)nops, s));
  JGPM_CUDA_TRY(dex.init(exclude, (size_t)nops, s));
  // device buffers for host result arrays, freed on every return path
  struct DeviceBuf {
    int32_t* p = nullptr;
    ~DeviceBuf() {
      if (p) cudaFree(p);
    }
  } tmp_counts, tmp_out;
  int32_t* dcounts = counts;
  int32_t* dout = out;
  bool counts_host = !is_device_ptr(counts);
  bool out_host = mat && !is_device_ptr(out);
  if (counts_host) {
    JGPM_CUDA_TRY(cudaMalloc(&tmp_counts.p, nops * sizeof(int32_t)));
    dcounts = tmp_counts.p;
  }
  if (mat) {
    JGPM_CUDA_TRY(doo.init(out_off, (size_t)nops + 1, s));
    if (out_host) {
      JGPM_CUDA_TRY(cudaMalloc(&tmp_out.p, std::max<int64_t>(1, ho[nops]) * 4));
      dout = tmp_out.p;
    }
  }
  const int64_t blocks = std::min<int64_t>((nops + 7) / 8, 148 * 16);
  k_setop_batch<<<(int)std::max<int64_t>(1, blocks), 256, 0, s>>>(
      op, da.d, dao.d, db.d, dbo.d, nops, dup.d, dex.d, dcounts, mat ? dout : nullptr,
      mat ? doo.d : nullptr);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && counts_host)
    e = cudaMemcpyAsync(counts, dcounts, nops * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && out_host && ho[nops] > 0)
    e = cudaMemcpyAsync(out, dout, ho[nops] * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    jgpm_set_error_(std::string("jgpm_setop_batch: ") + cudaGetErrorString(e));
    return JGPM_ECUDA;
  }
  return JGPM_OK;
}

int jgpm_setop_split_batch(int kind, const int32_t* a, const int64_t* a_off, const int32_t* b,
                           const int64_t* b_off, int64_t nops, const int32_t* upper,
                           int32_t* counts, int32_t* c, int32_t* d, int32_t* e) {
  const bool fuse = kind == JGPM_SPLIT_FUSE;
  if ((!fuse && kind != JGPM_SPLIT_DIF_INT) || nops < 0 || !a_off || !b_off || !counts) {
    jgpm_set_error_("jgpm_setop_split_batch: bad arguments");
    return JGPM_EINVAL;
  }
  if (nops == 0) return JGPM_OK;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    jgpm_set_error_("no CUDA device");
    return JGPM_ENODEV;
  }
  std::vector<int64_t> ha(nops + 1), hb(nops + 1);
  JGPM_CUDA_TRY(cudaMemcpy(ha.data(), a_off, (nops + 1) * 8, cudaMemcpyDefault));
  JGPM_CUDA_TRY(cudaMemcpy(hb.data(), b_off, (nops + 1) * 8, cudaMemcpyDefault));
  if (ha[0] < 0 || hb[0] < 0) {
    jgpm_set_error_("jgpm_setop_split_batch: bad offsets");
    return JGPM_EINVAL;
  }
  if ((ha[nops] > 0 && (!a || !c || !d)) || (hb[nops] > 0 && !b) ||
      (fuse && hb[nops] > 0 && !e)) {
    jgpm_set_error_("jgpm_setop_split_batch: missing operand or output array");
    return JGPM_EINVAL;
  }
  for (int64_t i = 0; i < nops; ++i) {
    const int64_t na = ha[i + 1] - ha[i], nb = hb[i + 1] - hb[i];
    if (na < 0 || nb < 0 || na > INT32_MAX || nb > INT32_MAX) {
      jgpm_set_error_("jgpm_setop_split_batch: bad offsets");
      return JGPM_EINVAL;
    }
  }
  cudaStream_t s = nullptr;
  JGPM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{s};
  Staged<int32_t> da, db, dup;
  Staged<int64_t> dao, dbo;
  JGPM_CUDA_TRY(da.init(a, (size_t)ha[nops], s));
  JGPM_CUDA_TRY(db.init(b, (size_t)hb[nops], s));
  JGPM_CUDA_TRY(dao.init(a_off, (size_t)nops + 1, s));
  JGPM_CUDA_TRY(dbo.init(b_off, (size_t)nops + 1, s));
  if (!fuse) JGPM_CUDA_TRY(dup.init(upper, (size_t)nops, s));
  OutArray oc, od, oe, on;
  JGPM_CUDA_TRY(oc.init(c, (size_t)ha[nops], s));
  JGPM_CUDA_TRY(od.init(d, (size_t)ha[nops], s));
  if (fuse) JGPM_CUDA_TRY(oe.init(e, (size_t)hb[nops], s));
  JGPM_CUDA_TRY(on.init(counts, (size_t)nops, s));
  const int64_t blocks = std::min<int64_t>((nops + 7) / 8, 148 * 16);
  k_split_batch<<<(int)std::max<int64_t>(1, blocks), 256, 0, s>>>(
      kind, da.d, dao.d, db.d, dbo.d, nops, dup.d, on.d, oc.d, od.d, oe.d);
  cudaError_t err = cudaGetLastError();
  if (err == cudaSuccess) err = on.back(s);
  if (err == cudaSuccess) err = oc.back(s);
  if (err == cudaSuccess) err = od.back(s);
  if (err == cudaSuccess) err = oe.back(s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) {
    jgpm_set_error_(std::string("jgpm_setop_split_batch: ") + cudaGetErrorString(err));
    return JGPM_ECUDA;
  }
  return JGPM_OK;
}

int jgpm_setop_split(int kind, const int32_t* a, int32_t na, const int32_t* b, int32_t nb,
                     int32_t upper, int32_t* c, int32_t* d, int32_t* e, int32_t* count) {
  if (na < 0 || nb < 0 || !count || (na > 0 && !a) || (nb > 0 && !b)) {
    jgpm_set_error_("jgpm_setop_split: bad arguments");
    return JGPM_EINVAL;
  }
  const int64_t aoff[2] = {0, na}, boff[2] = {0, nb};
  const int32_t up[1] = {upper};
  int32_t cnt = 0;
  const int rc = jgpm_setop_split_batch(kind, a, aoff, b, boff, 1, up, &cnt, c, d, e);
  if (rc) return rc;
  *count = cnt;
  return JGPM_OK;
}

int jgpm_setop(int op, const int32_t* a, int32_t na, const int32_t* b, int32_t nb,
               int32_t upper, int32_t exclude, int32_t* out, int32_t* out_n) {
  if (na < 0 || nb < 0 || !out_n || (na > 0 && !a) || (nb > 0 && !b)) {
    jgpm_set_error_("jgpm_setop: bad arguments");
    return JGPM_EINVAL;
  }
  const int64_t aoff[2] = {0, na}, boff[2] = {0, nb};
  const bool mat = (op == JGPM_OP_INTERSECT || op == JGPM_OP_DIFFERENCE);
  const int64_t cap = op == JGPM_OP_INTERSECT ? std::min(na, nb) : na;
  const int64_t ooff[2] = {0, cap};
  int32_t cnt = 0;
  const int32_t up[1] = {upper};
  const int32_t ex[1] = {exclude};
  int rc = jgpm_setop_batch(op, a, aoff, b, boff, 1, up, ex, &cnt, mat ? out : nullptr,
                            mat ? ooff : nullptr);
  if (rc) return rc;
  *out_n = cnt;
  return JGPM_OK;
}

}  // extern "C"
