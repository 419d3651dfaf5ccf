// Row sharding of the ALS iteration across GPUs, one process per GPU, as host
// code over the engine's C ABI.
//
// Given the fixed opposite factor every row's solve is independent, so each
// rank solves an nnz-balanced contiguous range of each side's rows
// (als_model_set_row_range) with the whole CSR/CSC and both factor matrices
// resident, and after each half-step the ranges are exchanged by one NCCL
// all-gather: the ranges hold different row counts, so every rank sends a
// block of `span` rows (the largest range) that starts at its range, moved
// back inside the matrix for the last ranges, and afterwards copies the other
// ranks' ranges out of the gathered blocks. The low-precision copy of the
// side is then rebuilt from the FP32 rows (als_model_sync_lp). Test RMSE: each
// rank sums the squared errors of its share of the test entries, and the sums
// are added by an NCCL all-reduce of one double.
//
// NCCL is loaded when the first shard is created (the copy already in the
// process, such as PyTorch's, if there is one), so the library itself does not
// depend on it.
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/als_b200.h"
#include "als_internal.h"

using namespace als;

namespace {

struct NcclApi {
  ncclResult_t (*get_unique_id)(ncclUniqueId *) = nullptr;
  ncclResult_t (*comm_init_rank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*all_gather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t,
                             cudaStream_t) = nullptr;
  ncclResult_t (*all_reduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                             cudaStream_t) = nullptr;
  ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
  const char *(*error_string)(ncclResult_t) = nullptr;
  bool ok = false;
};

const NcclApi &nccl() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!h) return;
    api.get_unique_id = reinterpret_cast<decltype(api.get_unique_id)>(dlsym(h, "ncclGetUniqueId"));
    api.comm_init_rank = reinterpret_cast<decltype(api.comm_init_rank)>(dlsym(h, "ncclCommInitRank"));
    api.all_gather = reinterpret_cast<decltype(api.all_gather)>(dlsym(h, "ncclAllGather"));
    api.all_reduce = reinterpret_cast<decltype(api.all_reduce)>(dlsym(h, "ncclAllReduce"));
    api.comm_destroy = reinterpret_cast<decltype(api.comm_destroy)>(dlsym(h, "ncclCommDestroy"));
    api.error_string = reinterpret_cast<decltype(api.error_string)>(dlsym(h, "ncclGetErrorString"));
    api.ok = api.get_unique_id && api.comm_init_rank && api.all_gather && api.all_reduce &&
             api.comm_destroy && api.error_string;
  });
  return api;
}

int nccl_fail(ncclResult_t r, const char *where) {
  return api_fail(ALS_ERR_CUDA, std::string(where) + ": " + nccl().error_string(r));
}

#define SHARD_CUDA(call, where)                                                    \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) return api_fail(ALS_ERR_CUDA, std::string(where) + ": " + \
                                                             cudaGetErrorString(e_)); \
  } while (0)
#define SHARD_NCCL(call, where)                    \
  do {                                             \
    ncclResult_t r_ = (call);                      \
    if (r_ != ncclSuccess) return nccl_fail(r_, where); \
  } while (0)
#define SHARD_ALS(call)          \
  do {                           \
    int rc_ = (call);            \
    if (rc_ != ALS_OK) return rc_; \
  } while (0)

}  // namespace

struct als_shard {
  als_model *model = nullptr;
  int world = 1, rank = 0, f = 0;
  int64_t rows[2] = {0, 0};
  ncclComm_t comm = nullptr;
  std::vector<int64_t> bounds[2], start[2];
  int64_t span[2] = {0, 0};
  float *stage[2] = {nullptr, nullptr};  // world * span rows of f floats per side
  double *sums = nullptr;                // the RMSE partial sum (device)
  void *rmse_work = nullptr;             // the RMSE kernels' block sums (device)
  bool ranged[2] = {false, false};       // the model's row range of a side was set
};

extern "C" {

int als_shard_unique_id(void *id128) {
  if (!id128) return api_fail(ALS_ERR_INVALID, "als_shard_unique_id: null buffer");
  static_assert(sizeof(ncclUniqueId) == 128, "NCCL unique id is 128 bytes");
  if (!nccl().ok) return api_fail(ALS_ERR_UNSUPPORTED, "als_shard_unique_id: libnccl.so.2 not found");
  ncclUniqueId id;
  SHARD_NCCL(nccl().get_unique_id(&id), "ncclGetUniqueId");
  std::memcpy(id128, &id, sizeof(id));
  return ALS_OK;
}

int als_shard_partition(const int64_t *h_ptr, int64_t rows, int32_t world, int32_t f,
                        int64_t *h_bounds) {
  if (!h_ptr || !h_bounds || rows < 0 || world < 1 || f < 1)
    return api_fail(ALS_ERR_INVALID, "als_shard_partition: bad arguments");
  // cum[r] = cost of rows [0, r); a row costs nnz * f^2 (hermitian) + f^3 / 3
  // (solve); cut k is the first r with cum[r] >= total * k / world
  std::vector<double> cum((size_t)rows + 1, 0.0);
  const double ff = (double)f * (double)f, f3 = (double)f * ff / 3.0;
  for (int64_t r = 0; r < rows; ++r) {
    const int64_t d = h_ptr[r + 1] - h_ptr[r];
    cum[(size_t)r + 1] = cum[(size_t)r] + ((double)(d > 0 ? d : 0) * ff + f3);
  }
  h_bounds[0] = 0;
  for (int k = 1; k < world; ++k) {
    const double target = cum[(size_t)rows] * k / world;
    const int64_t cut = std::lower_bound(cum.begin(), cum.end(), target) - cum.begin();
    h_bounds[k] = std::max(h_bounds[k - 1], std::min(cut, rows));
  }
  h_bounds[world] = rows;
  return ALS_OK;
}

int als_shard_blocks(const int64_t *h_bounds, int32_t world, int64_t *h_span, int64_t *h_start) {
  if (!h_bounds || !h_span || !h_start || world < 1)
    return api_fail(ALS_ERR_INVALID, "als_shard_blocks: bad arguments");
  const int64_t rows = h_bounds[world];
  int64_t span = 0;
  for (int r = 0; r < world; ++r) span = std::max(span, h_bounds[r + 1] - h_bounds[r]);
  for (int r = 0; r < world; ++r) h_start[r] = std::min(h_bounds[r], rows - span);
  *h_span = span;
  return ALS_OK;
}

int als_shard_create(als_shard **out, als_model *model, const int64_t *h_csr_ptr,
                     const int64_t *h_csc_ptr, int64_t m, int64_t n, int32_t f, int32_t world,
                     int32_t rank, const void *id128, cudaStream_t stream) {
  if (!out || !model || !h_csr_ptr || !h_csc_ptr || m < 1 || n < 1 || f < 1 || world < 1 ||
      rank < 0 || rank >= world || !id128)
    return api_fail(ALS_ERR_INVALID, "als_shard_create: bad arguments");
  *out = nullptr;
  {
    int64_t mm = 0, nn = 0;
    int32_t ff = 0;
    model_dims(model, &mm, &nn, &ff);
    if (mm != m || nn != n || ff != f)
      return api_fail(ALS_ERR_INVALID, "als_shard_create: m, n, f differ from the model's");
  }
  if (!nccl().ok) return api_fail(ALS_ERR_UNSUPPORTED, "als_shard_create: libnccl.so.2 not found");
  auto *s = new als_shard();
  s->model = model;
  s->world = world;
  s->rank = rank;
  s->f = f;
  s->rows[ALS_SIDE_USERS] = m;
  s->rows[ALS_SIDE_ITEMS] = n;
  auto undo = [&](int rc) {
    als_shard_destroy(s);
    return rc;
  };
  for (int side = 0; side < 2; ++side) {
    s->bounds[side].assign((size_t)world + 1, 0);
    s->start[side].assign((size_t)world, 0);
    int rc = als_shard_partition(side == ALS_SIDE_USERS ? h_csr_ptr : h_csc_ptr, s->rows[side],
                                 world, f, s->bounds[side].data());
    if (rc == ALS_OK)
      rc = als_shard_blocks(s->bounds[side].data(), world, &s->span[side], s->start[side].data());
    if (rc != ALS_OK) return undo(rc);
    cudaError_t e = cudaMalloc(&s->stage[side], sizeof(float) * (size_t)world *
                                                    (size_t)std::max<int64_t>(s->span[side], 1) * f);
    if (e != cudaSuccess) return undo(api_fail(ALS_ERR_CUDA, std::string("als_shard_create: ") +
                                                                 cudaGetErrorString(e)));
    rc = als_model_set_row_range(model, side, s->bounds[side][rank], s->bounds[side][rank + 1],
                                 stream);
    if (rc != ALS_OK) return undo(rc);
    s->ranged[side] = true;
  }
  cudaError_t e = cudaMalloc(&s->sums, sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&s->rmse_work, als_rmse_work_bytes());
  if (e != cudaSuccess)
    return undo(api_fail(ALS_ERR_CUDA, std::string("als_shard_create: ") + cudaGetErrorString(e)));
  ncclUniqueId id;
  std::memcpy(&id, id128, sizeof(id));
  ncclResult_t r = nccl().comm_init_rank(&s->comm, world, id, rank);
  if (r != ncclSuccess) {
    s->comm = nullptr;
    return undo(nccl_fail(r, "ncclCommInitRank"));
  }
  *out = s;
  return ALS_OK;
}

int als_shard_bounds(const als_shard *s, int32_t side, int64_t *h_bounds) {
  if (!s || (side != ALS_SIDE_USERS && side != ALS_SIDE_ITEMS) || !h_bounds)
    return api_fail(ALS_ERR_INVALID, "als_shard_bounds: bad arguments");
  std::copy(s->bounds[side].begin(), s->bounds[side].end(), h_bounds);
  return ALS_OK;
}

int als_shard_exchange(als_shard *s, int32_t side, cudaStream_t stream) {
  if (!s || (side != ALS_SIDE_USERS && side != ALS_SIDE_ITEMS))
    return api_fail(ALS_ERR_INVALID, "als_shard_exchange: bad arguments");
  float *x = nullptr, *t = nullptr;
  SHARD_ALS(als_model_factors(s->model, &x, &t));
  float *target = side == ALS_SIDE_USERS ? x : t;
  const int64_t span = s->span[side];
  const size_t f = (size_t)s->f;
  if (span > 0) {
    const int64_t s0 = s->start[side][s->rank];
    SHARD_NCCL(nccl().all_gather(target + (size_t)s0 * f, s->stage[side], (size_t)span * f,
                                 ncclFloat, s->comm, stream),
               "ncclAllGather");
    for (int r = 0; r < s->world; ++r) {
      const int64_t lo = s->bounds[side][r], hi = s->bounds[side][r + 1];
      if (r == s->rank || hi == lo) continue;
      const size_t off = (size_t)r * span + (size_t)(lo - s->start[side][r]);
      SHARD_CUDA(cudaMemcpyAsync(target + (size_t)lo * f, s->stage[side] + off * f,
                                 sizeof(float) * (size_t)(hi - lo) * f, cudaMemcpyDeviceToDevice,
                                 stream),
                 "als_shard_exchange: copy");
    }
  }
  return als_model_sync_lp(s->model, side, stream);
}

int als_shard_half_step(als_shard *s, int32_t side, float lambda, cudaStream_t stream) {
  if (!s) return api_fail(ALS_ERR_INVALID, "als_shard_half_step: null shard");
  SHARD_ALS(als_model_half_step(s->model, side, lambda, stream));
  return als_shard_exchange(s, side, stream);
}

int als_shard_iterate(als_shard *s, float lambda, int32_t iters, cudaStream_t stream) {
  if (!s || iters < 0) return api_fail(ALS_ERR_INVALID, "als_shard_iterate: bad arguments");
  for (int it = 0; it < iters; ++it) {
    SHARD_ALS(als_shard_half_step(s, ALS_SIDE_USERS, lambda, stream));
    SHARD_ALS(als_shard_half_step(s, ALS_SIDE_ITEMS, lambda, stream));
  }
  return ALS_OK;
}

int als_shard_rmse(als_shard *s, int64_t nt, const int32_t *d_u, const int32_t *d_i,
                   const float *d_r, double *out, cudaStream_t stream) {
  if (!s || nt < 0 || !out || (nt > 0 && (!d_u || !d_i || !d_r)))
    return api_fail(ALS_ERR_INVALID, "als_shard_rmse: bad arguments");
  float *x = nullptr, *t = nullptr;
  SHARD_ALS(als_model_factors(s->model, &x, &t));
  // this rank's share of the entries: [nt * rank / world, nt * (rank + 1) / world)
  const int64_t lo = nt * s->rank / s->world, hi = nt * (s->rank + 1) / s->world;
  SHARD_CUDA(launch_rmse_sum(hi - lo, d_u + lo, d_i + lo, d_r + lo, x, s->f, t, s->f, s->f,
                             s->sums, s->rmse_work, stream),
             "als_shard_rmse");
  SHARD_NCCL(nccl().all_reduce(s->sums, s->sums, 1, ncclDouble, ncclSum, s->comm, stream),
             "ncclAllReduce");
  double sum = 0.0;
  SHARD_CUDA(cudaMemcpyAsync(&sum, s->sums, sizeof(double), cudaMemcpyDeviceToHost, stream),
             "als_shard_rmse: copy");
  SHARD_CUDA(cudaStreamSynchronize(stream), "als_shard_rmse: sync");
  *out = nt > 0 ? std::sqrt(sum / (double)nt) : 0.0;
  return ALS_OK;
}

void als_shard_destroy(als_shard *s) {
  if (!s) return;
  if (s->comm) nccl().comm_destroy(s->comm);
  // the model solves all its rows again
  for (int side = 0; side < 2; ++side)
    if (s->ranged[side]) als_model_set_row_range(s->model, side, 0, s->rows[side], nullptr);
  for (float *p : s->stage)
    if (p) cudaFree(p);
  if (s->sums) cudaFree(s->sums);
  if (s->rmse_work) cudaFree(s->rmse_work);
  delete s;
}

}  // extern "C"
