// Shared definitions for the bzip2gpu-b200 kernels and host engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

namespace bz2g {

// bzip2 format constants (src/compression/huffman.cu:10-11, include/compression.h:65-66
// of the reference).
constexpr int kMaxGroups = 6;
constexpr int kMaxAlpha = 258;
constexpr int kGroupSize = 50;
constexpr int kMaxCodeLen = 17;
constexpr int kIters = 4;

// Element tiles: every per-block array in the slab layout starts at a multiple
// of kTile elements, so a tile never straddles two blocks.
constexpr int kTile = 4096;
constexpr int kTileThreads = 256;
constexpr int kTileItems = kTile / kTileThreads;  // 16

// Raw-input tiles for RLE1 and CRC.
constexpr int kRawTile = 4096;

// Upper bound on the RLE1 output of n raw bytes (a run of exactly 4 becomes 5
// bytes, so the output is at most 5/4 of the input).
inline int64_t rle1_bound(int64_t n) { return n + n / 4 + 8; }
inline int64_t align_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// Status codes returned through the C-ABI (include/bz2g.h).
enum Status {
  kOk = 0,
  kErrCuda = 1,
  kErrArg = 2,
  kErrAlloc = 3,
  kErrInternal = 4,
  kErrTooLarge = 5,
  kErrTimeout = 6,  // a bounded wait inside a kernel ran out
};

[[noreturn]] void throw_cuda(cudaError_t e, const char *expr, const char *file, int line);

}  // namespace bz2g

#define BZ_CUDA(expr)                                                           \
  do {                                                                          \
    cudaError_t e__ = (expr);                                                   \
    if (e__ != cudaSuccess) ::bz2g::throw_cuda(e__, #expr, __FILE__, __LINE__); \
  } while (0)

namespace bz2g {
// Kernel launches issued by this library (all launch sites end with
// BZ_LAUNCH_CHECK), for the benchmark's launch count.
void count_launch();
}  // namespace bz2g
#define BZ_LAUNCH_CHECK()         \
  do {                            \
    ::bz2g::count_launch();       \
    BZ_CUDA(cudaGetLastError());  \
  } while (0)

#define BZ_REQUIRE(cond, code, msg)                 \
  do {                                              \
    if (!(cond)) throw ::bz2g::Error((code), (msg)); \
  } while (0)

// ----------------------------------------------------------- device helpers
#ifdef __CUDACC__
namespace bz2g {

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned warp_id() { return threadIdx.x >> 5; }

template <typename T>
__device__ __forceinline__ T warp_incl_sum(T v) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T o = __shfl_up_sync(0xffffffffu, v, d);
    if ((int)lane_id() >= d) v += o;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_incl_max(T v) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T o = __shfl_up_sync(0xffffffffu, v, d);
    if ((int)lane_id() >= d) v = o > v ? o : v;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_incl_min_rev(T v) {
  // suffix (from the highest lane down) inclusive minimum
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T o = __shfl_down_sync(0xffffffffu, v, d);
    if ((int)lane_id() + d < 32) v = o < v ? o : v;
  }
  return v;
}

// Block-wide exclusive sum; `scratch` holds blockDim.x/32 + 1 values.
// Returns the exclusive prefix; *total gets the block total.
template <typename T>
__device__ __forceinline__ T block_excl_sum(T v, T *scratch, T *total) {
  const int nw = blockDim.x >> 5;
  T inc = warp_incl_sum(v);
  if (lane_id() == 31) scratch[warp_id()] = inc;
  __syncthreads();
  if (warp_id() == 0) {
    T w = (int)lane_id() < nw ? scratch[lane_id()] : T(0);
    T wi = warp_incl_sum(w);
    if ((int)lane_id() < nw) scratch[lane_id()] = wi - w;
    if ((int)lane_id() == nw - 1) scratch[nw] = wi;
  }
  __syncthreads();
  T r = scratch[warp_id()] + inc - v;
  if (total) *total = scratch[nw];
  __syncthreads();
  return r;
}

// Block-wide inclusive max.
template <typename T>
__device__ __forceinline__ T block_incl_max(T v, T *scratch, T identity) {
  const int nw = blockDim.x >> 5;
  T inc = warp_incl_max(v);
  if (lane_id() == 31) scratch[warp_id()] = inc;
  __syncthreads();
  if (warp_id() == 0) {
    T w = (int)lane_id() < nw ? scratch[lane_id()] : identity;
    T wi = warp_incl_max(w);
    // exclusive max for each warp
    T ex = __shfl_up_sync(0xffffffffu, wi, 1);
    if (lane_id() == 0) ex = identity;
    if ((int)lane_id() < nw) scratch[lane_id()] = ex;
  }
  __syncthreads();
  T p = scratch[warp_id()];
  T r = p > inc ? p : inc;
  __syncthreads();
  return r;
}

// Block-wide suffix inclusive min (element i gets min over j >= i).
template <typename T>
__device__ __forceinline__ T block_suffix_min(T v, T *scratch, T identity) {
  const int nw = blockDim.x >> 5;
  T inc = warp_incl_min_rev(v);
  if (lane_id() == 0) scratch[warp_id()] = inc;
  __syncthreads();
  if (warp_id() == 0) {
    T w = (int)lane_id() < nw ? scratch[lane_id()] : identity;
    T wi = warp_incl_min_rev(w);
    T ex = __shfl_down_sync(0xffffffffu, wi, 1);
    if ((int)lane_id() >= nw - 1) ex = identity;
    if ((int)lane_id() < nw) scratch[lane_id()] = ex;
  }
  __syncthreads();
  T p = scratch[warp_id()];
  T r = p < inc ? p : inc;
  __syncthreads();
  return r;
}

}  // namespace bz2g
#endif
