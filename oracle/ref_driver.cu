// ref_driver.cu -- test and baseline infrastructure, never linked by the product.
//
// A C ABI over the reference's own search path (cuRPLSH src/internal/{norm,
// search,select,broadcast,matrix_ops}.cu, compiled from its sources by
// oracle/Makefile into oracle/_ref/libcurplsh_ref.so).  It drives that code
// exactly as IndexBF would:
//   add    (src/index_bf.cpp:26-44): rows copied into a DeviceTensor, squared
//          norms by computeL2Norm on the resources' default stream;
//   search (src/index_bf.cpp:46-74): queries copied into a DeviceTensor,
//          searchL2Distance(resources, data, &norms, queries, k, indices,
//          distances, computeExactDistances = true), results copied back.
// IndexBF itself does not compile (it calls helpers that do not exist), so
// this file stands in for its two methods.
//
// Shapes the reference code handles in bounds, and which this driver
// therefore accepts (anything else is rejected before a kernel runs):
//   * d == 128.  computeL2Norm casts rows to float4 and, for 32 float4 per
//     row, runs its 32x8 special case; for d = 64, 96, 256 or 512 its
//     shared-memory index (idx * numWarps + y * numWarpsPerVec + warp)
//     exceeds the buffer it sizes (norm.cu:58/93 vs :143/152), and d = 96 also
//     shuffles over a partial warp.  Callers pad smaller d with zero columns
//     (distances are unchanged).
//   * rows (queries, and database rows when their norms are computed here) a
//     multiple of 8: the special case reads and writes 8 rows per block with
//     no row check unless fewer than BatchSize (= 1) rows remain (norm.cu:31).
//   * 2 <= k <= 1024 and k <= N: k = 1 takes kernelL2Select1, whose block
//     reduction and last-block predicate are wrong (select.cu:119-120).
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "device_resources.h"
#include "device_tensor.h"
#include "internal/norm.h"
#include "internal/search.h"

namespace {

thread_local std::string g_err;

int fail(const char* msg) {
  g_err = msg;
  return 1;
}

int cuda_fail(const char* what, cudaError_t e) {
  char buf[256];
  snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  g_err = buf;
  return 2;
}

// Never destroyed: the reference's destructor checks CUDA calls and exits the
// process on an error, and at process exit the CUDA runtime is already
// unloading (cudaErrorCudartUnloading).  The process's end releases it.
curplsh::DeviceResources* g_res = nullptr;
int g_dev = -1;

struct RefDatabase {
  int device;
  int dim;
  int num;
  curplsh::DeviceTensor<float, 2> data;
  curplsh::DeviceTensor<float, 1> norms;
};

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

extern "C" {

const char* curplsh_ref_last_error(void) { return g_err.c_str(); }

// Creates the reference's DeviceResources for `device` (once per process).
int curplsh_ref_open(int device) {
  if (g_res) return g_dev == device ? 0 : fail("curplsh_ref_open: already open on another device");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail("cudaSetDevice", e);
  g_res = new curplsh::DeviceResources();
  g_res->initializeForDevice(device);
  g_dev = device;
  return 0;
}

// IndexBF::add: copies `num` host rows of `dim` floats to the device and
// computes their squared norms with the reference's computeL2Norm, or takes
// them from `host_norms` when it is non-null (then num need not be a multiple of 8).
int curplsh_ref_add(const float* rows, int64_t num, int dim, const float* host_norms, void** out) {
  if (!g_res) return fail("curplsh_ref_add: call curplsh_ref_open first");
  if (!rows || !out || num <= 0 || num > (1LL << 30)) return fail("curplsh_ref_add: bad arguments");
  if (dim != 128) return fail("curplsh_ref_add: only d = 128 runs in bounds in the reference (pad with zeros)");
  if (!host_norms && num % 8) return fail("curplsh_ref_add: num must be a multiple of 8 when norms are computed");
  curplsh::DeviceScope scope(g_dev);
  auto* db = new RefDatabase{g_dev, dim, (int)num, curplsh::DeviceTensor<float, 2>({(int)num, dim}),
                             curplsh::DeviceTensor<float, 1>({(int)num})};
  cudaError_t e = cudaMemcpy(db->data.data(), rows, (size_t)num * dim * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    delete db;
    return cuda_fail("copy rows", e);
  }
  if (host_norms) {
    e = cudaMemcpy(db->norms.data(), host_norms, (size_t)num * sizeof(float), cudaMemcpyHostToDevice);
  } else {
    curplsh::computeL2Norm(db->data, db->norms, true, g_res->getDefaultStream(g_dev));
    e = cudaStreamSynchronize(g_res->getDefaultStream(g_dev));
  }
  if (e != cudaSuccess) {
    delete db;
    return cuda_fail("norms", e);
  }
  *out = db;
  return 0;
}

int curplsh_ref_free(void* h) {
  delete static_cast<RefDatabase*>(h);
  return 0;
}

// IndexBF::search of `nq` host queries: results to host arrays [nq x k].
// `reps` >= 1 searches run; ms_e2e gets the mean host time of one search
// including the query upload and result download (as IndexBF::search with
// host pointers), ms_resident the mean time of searchL2Distance alone with
// queries and results already on the device (the reference allocates its
// tile buffers inside every call; that is part of its time).
int curplsh_ref_search(void* h, const float* queries, int64_t nq, int k, int* indices, float* distances, int reps,
                       double* ms_e2e, double* ms_resident) {
  auto* db = static_cast<RefDatabase*>(h);
  if (!db || !queries || !indices || !distances) return fail("curplsh_ref_search: null argument");
  if (nq <= 0 || nq % 8 || nq > (1LL << 30)) return fail("curplsh_ref_search: nq must be a positive multiple of 8");
  if (k < 2 || k > 1024 || k > db->num) return fail("curplsh_ref_search: k must be in [2, min(1024, N)]");
  if (reps < 1) reps = 1;
  curplsh::DeviceScope scope(db->device);
  cudaStream_t st = g_res->getDefaultStream(db->device);
  double e2e = 0.0, resident = 0.0;
  for (int r = 0; r < reps; ++r) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail("sync", e);
    const double t0 = now_ms();
    curplsh::DeviceTensor<float, 2> q({(int)nq, db->dim});
    e = cudaMemcpyAsync(q.data(), queries, (size_t)nq * db->dim * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail("copy queries", e);
    curplsh::DeviceTensor<int, 2> idx({(int)nq, k});
    curplsh::DeviceTensor<float, 2> dist({(int)nq, k});
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail("sync", e);
    const double t1 = now_ms();
    curplsh::searchL2Distance(g_res, db->data, &db->norms, q, k, idx, dist, true);
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail("searchL2Distance", e);
    const double t2 = now_ms();
    e = cudaMemcpyAsync(indices, idx.data(), (size_t)nq * k * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(distances, dist.data(), (size_t)nq * k * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail("copy results", e);
    const double t3 = now_ms();
    e2e += t3 - t0;
    resident += t2 - t1;
  }
  if (ms_e2e) *ms_e2e = e2e / reps;
  if (ms_resident) *ms_resident = resident / reps;
  return 0;
}

}  // extern "C"
