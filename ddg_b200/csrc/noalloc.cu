// Allocation-free dot product.
//
// Some callers cannot allocate device memory at all: code running while a
// CUDA stream is being captured into a graph (cudaMalloc is not a capturable
// operation), code that must keep a fixed, pre-planned device-memory
// footprint (a solver embedded in a host application that owns its memory
// pool), or hosts that forbid allocation after start-up.  For them,
// ddg_dot_noalloc computes x.y like ddg_dot but keeps its scratch (one
// float64 partial sum per block and a completion counter) in a file-scope
// device array that exists for as long as the library is loaded; it never
// calls cudaMalloc, cudaFree or any allocating routine.
//
// Limits and rules:
//  * n <= DDG_DOT_NOALLOC_MAX_N (one partial per 8192-element chunk, at most
//    65536 chunks: 512 KiB of scratch per GPU that has used the entry point);
//    larger n is rejected with DDG_ERR_INVALID.
//  * The first call on each device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current).  Make that first call
//    before any stream capture; later calls only launch work and can be
//    captured.
//  * All calls share the one array and it keeps the previous call's
//    contents: each call clears the completion counter first (an async
//    memset on the given stream), and calls that overlap on the GPU (other
//    streams, concurrent graphs) race on the array and give wrong results.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "../../include/ddg_sipg.h"
#include "sipg_device.cuh"
#include "status.h"

namespace {

constexpr int kChunk = 8192;              // elements per block
constexpr int kMaxChunks = 65536;         // partials held by the scratch array
constexpr int kBlock = 256;

// [0, kMaxChunks) doubles: per-block partials; then one unsigned counter.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kMaxChunks * sizeof(double) + 256];

template <typename T>
__global__ void __launch_bounds__(kBlock) k_dot_chunks(int64_t n, const T* __restrict__ x, const T* __restrict__ y,
                                                       unsigned char* scratch, double* out) {
  __shared__ double s_red[64];
  double* part = reinterpret_cast<double*>(scratch);
  unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch + kMaxChunks * sizeof(double));
  const int64_t base = (int64_t)blockIdx.x * kChunk;
  const int64_t end = base + kChunk < n ? base + kChunk : n;
  double s = 0.0, d = 0.0;
  for (int64_t i = base + threadIdx.x; i < end; i += kBlock) s += (double)x[i] * (double)y[i];
  ddg::block_sum2<kBlock>(s, d, s_red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
  if (!ddg::is_last_block(ticket)) return;
  double t, u;
  ddg::reduce_partials2<kBlock>(part, nullptr, gridDim.x, t, u, s_red);
  if (threadIdx.x == 0) {
    *out = t;
    *ticket = 0u;
  }
}

std::mutex g_mu;
void* g_addr[64] = {nullptr};   // device address of the array, per device ordinal

}  // namespace

extern "C" int ddg_dot_noalloc(int64_t n, int precision, const void* x, const void* y, double* out, void* stream) {
  if (n < 0 || !out || (n > 0 && (!x || !y))) return ddg::fail(DDG_ERR_INVALID, "ddg_dot_noalloc: bad argument");
  if (precision != DDG_FP64 && precision != DDG_FP32)
    return ddg::fail(DDG_ERR_INVALID, "ddg_dot_noalloc: bad precision");
  if (n > (int64_t)DDG_DOT_NOALLOC_MAX_N)
    return ddg::fail(DDG_ERR_INVALID, "ddg_dot_noalloc: n = " + std::to_string(n) + " exceeds the maximum " +
                                          std::to_string((long long)DDG_DOT_NOALLOC_MAX_N) +
                                          " of its static scratch; use ddg_dot");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64)
    return ddg::fail(DDG_ERR_CUDA, std::string("ddg_dot_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {   // once per device, with that device current
      e = cudaGetSymbolAddress(&g_addr[dev], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_addr[dev] = nullptr;
        return ddg::fail(DDG_ERR_CUDA, std::string("ddg_dot_noalloc: cudaGetSymbolAddress: ") +
                                           cudaGetErrorString(e));
      }
    }
    scratch = g_addr[dev];
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) {
    e = cudaMemsetAsync(out, 0, sizeof(double), s);
    return e == cudaSuccess ? DDG_OK : ddg::fail(DDG_ERR_CUDA, "ddg_dot_noalloc: memset");
  }
  // the completion counter must start at zero
  e = cudaMemsetAsync(static_cast<unsigned char*>(scratch) + kMaxChunks * sizeof(double), 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return ddg::fail(DDG_ERR_CUDA, std::string("ddg_dot_noalloc: ") + cudaGetErrorString(e));
  const int grid = (int)((n + kChunk - 1) / kChunk);
  if (precision == DDG_FP64)
    k_dot_chunks<double><<<grid, kBlock, 0, s>>>(n, (const double*)x, (const double*)y, (unsigned char*)scratch, out);
  else
    k_dot_chunks<float><<<grid, kBlock, 0, s>>>(n, (const float*)x, (const float*)y, (unsigned char*)scratch, out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return ddg::fail(DDG_ERR_CUDA, std::string("ddg_dot_noalloc: ") + cudaGetErrorString(e));
  return DDG_OK;
}
