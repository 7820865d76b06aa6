// bzip2 1.0.8's block split, on the GPU (no counterpart in the reference, whose
// blocks are 900,000 raw bytes for every level, src/main.cpp:26,36, and whose
// TODO.md:38-40 lists the split as missing).
//
// bzip2 1.0.8 (bzlib.c: ADD_CHAR_TO_BLOCK, add_pair_to_block,
// copy_input_until_stop, handle_compress) feeds input bytes into a pending
// run of at most 255 equal bytes; a run is written to the block when a
// different byte arrives or it is 255 long, as L bytes (L <= 3) or 4 bytes
// and a count (L >= 4).  Before each input byte, a block holding
// MAX = 100000 * level - 19 or more written bytes is closed, and the pending
// run (one byte long at that moment) stays pending: it begins the next block.
// So every block starts at a chunk start (the start of a run, or 255, 510, ...
// bytes into one), chunks are those of the whole input, and with
//   cnt(i) = 1, 1, 1, 2, 0, 0, ... for positions 0, 1, 2, 3, 4, ... of a chunk
//   G(x)   = sum of cnt(i) for i < x   (the RLE1 bytes before x)
// block k ends at the smallest chunk start x > start with
// G(x) >= G(start) + MAX (or at the end of the input).
//
// Device work: per 4096-byte tile, the first and last run start; scans give
// each tile the last run start before it and the first one at or after it;
// per tile the sum of cnt, and its exclusive prefix P.  One thread block then
// walks the blocks: a 256-way search of P for the tile where G reaches the
// target, one pass over that tile for the exact position, and the next chunk
// start from the run start and the following run start.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "split.h"

namespace bz2g {
namespace {

constexpr int kSplitTile = 4096;
constexpr int kSplitThreads = 256;  // 16 bytes per thread
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kCut = 255;

template <typename T, typename Op>
__device__ __forceinline__ T warp_scan(T v, Op op) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T o = __shfl_up_sync(0xffffffffu, v, d);
    if ((int)lane_id() >= d) v = op(o, v);
  }
  return v;
}

// Block-wide inclusive scan (sh: 32 values).
template <typename T, typename Op>
__device__ __forceinline__ T block_scan(T v, T *sh, Op op) {
  v = warp_scan(v, op);
  if (lane_id() == 31) sh[warp_id()] = v;
  __syncthreads();
  if (warp_id() == 0) {
    const int nw = blockDim.x >> 5;
    T w = (int)lane_id() < nw ? sh[lane_id()] : sh[0];
    w = warp_scan(w, op);
    if ((int)lane_id() < nw) sh[lane_id()] = w;
  }
  __syncthreads();
  if (warp_id() > 0) v = op(sh[warp_id() - 1], v);
  __syncthreads();
  return v;
}

struct MaxOp {
  __device__ int64_t operator()(int64_t a, int64_t b) const { return a > b ? a : b; }
};
struct MinOp {
  __device__ int64_t operator()(int64_t a, int64_t b) const { return a < b ? a : b; }
};
struct SumOp {
  __device__ int64_t operator()(int64_t a, int64_t b) const { return a + b; }
};

// RLE1 bytes charged to position q of a chunk, and their sum over q < Q.
__device__ __forceinline__ int cnt_of(int q) { return q < 3 ? 1 : (q == 3 ? 2 : 0); }
__device__ __forceinline__ int64_t cnt_below(int64_t q) { return q <= 3 ? q : 5; }

// The thread's 16 bytes at p0 (nv of them inside the input) and the mask of
// run starts among them (a byte that differs from the one before it, or
// byte 0 of the input).
__device__ __forceinline__ uint32_t load16(const uint8_t *in, int64_t n, int64_t p0,
                                           uint8_t (&c)[16], int &nv) {
  const int64_t left = n - p0;
  nv = left <= 0 ? 0 : (left >= 16 ? 16 : (int)left);
  if (nv == 16 && (reinterpret_cast<uintptr_t>(in + p0) & 15u) == 0) {
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(in + p0));
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 16; k++) c[k] = (uint8_t)(w[k >> 2] >> (8 * (k & 3)));
  } else {
#pragma unroll
    for (int k = 0; k < 16; k++) c[k] = k < nv ? in[p0 + k] : 0;
  }
  int pv = (p0 > 0 && nv > 0) ? (int)in[p0 - 1] : -1;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < 16; k++) {
    if (k < nv && (int)c[k] != pv) s |= 1u << k;
    pv = c[k];
  }
  return s;
}

// Per-tile kernels: one warp per 4096-byte tile, lane l on bytes
// 128 l .. 128 l + 127 (eight 16-byte pieces), warp shuffles only.
constexpr int kLaneBytes = kSplitTile / 32;

// fa[t] / la[t]: first / last run start in tile t (INT64_MAX / -1 if none).
__global__ void __launch_bounds__(kSplitThreads)
    k_split_runs(const uint8_t *__restrict__ in, int64_t n, int64_t T, int64_t *fa,
                 int64_t *la) {
  const int64_t nwarps = (int64_t)gridDim.x * (kSplitThreads / 32);
  for (int64_t t = (int64_t)blockIdx.x * (kSplitThreads / 32) + warp_id(); t < T; t += nwarps) {
    const int64_t base = t * kSplitTile + (int64_t)lane_id() * kLaneBytes;
    int64_t f = INT64_MAX, l = -1;
#pragma unroll
    for (int piece = 0; piece < kLaneBytes / 16; piece++) {
      const int64_t p0 = base + piece * 16;
      uint8_t c[16];
      int nv;
      const uint32_t sm = load16(in, n, p0, c, nv);
      if (sm) {
        f = min(f, p0 + __ffs(sm) - 1);
        l = max(l, p0 + 31 - __clz(sm));
      }
    }
    for (int o = 16; o; o >>= 1) {
      f = min(f, (int64_t)__shfl_xor_sync(0xffffffffu, (long long)f, o));
      l = max(l, (int64_t)__shfl_xor_sync(0xffffffffu, (long long)l, o));
    }
    if (lane_id() == 0) {
      fa[t] = f;
      la[t] = l;
    }
  }
}

// lb[t] = last run start before tile t (exclusive max of la);
// nf[t] = first run start at or after tile t (inclusive suffix min of fa),
// nf[T] = n.  One thread block.
__global__ void __launch_bounds__(kScanThreads)
    k_split_scan_runs(int64_t T, int64_t n, const int64_t *la, const int64_t *fa, int64_t *lb,
                      int64_t *nf) {
  __shared__ int64_t sh[32];
  constexpr int64_t kChunk = (int64_t)kScanThreads * kScanItems;
  int64_t carry = -1;
  for (int64_t base = 0; base < T; base += kChunk) {
    const int64_t i0 = base + (int64_t)threadIdx.x * kScanItems;
    int64_t v[kScanItems], m = -1;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      v[k] = i0 + k < T ? la[i0 + k] : -1;
      m = max(m, v[k]);
    }
    const int64_t inc = block_scan(m, sh, MaxOp());
    // exclusive: this thread's items start after the previous threads'
    int64_t ex = __shfl_up_sync(0xffffffffu, (long long)inc, 1);
    if (lane_id() == 0) ex = warp_id() == 0 ? -1 : sh[warp_id() - 1];
    ex = max(carry, ex);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      if (i0 + k < T) lb[i0 + k] = ex;
      ex = max(ex, v[k]);
    }
    carry = max(carry, sh[(kScanThreads / 32) - 1]);
    __syncthreads();
  }
  if (threadIdx.x == 0) nf[T] = n;
  carry = n;
  for (int64_t base = 0; base < T; base += kChunk) {
    // thread j takes the items T-1-(base + j*I + k), k = 0..I-1 (descending)
    const int64_t i0 = T - 1 - (base + (int64_t)threadIdx.x * kScanItems);
    int64_t v[kScanItems], m = INT64_MAX;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      v[k] = i0 - k >= 0 ? min(fa[i0 - k], n) : INT64_MAX;
      m = min(m, v[k]);
    }
    const int64_t inc = block_scan(m, sh, MinOp());
    int64_t ex = __shfl_up_sync(0xffffffffu, (long long)inc, 1);
    if (lane_id() == 0) ex = warp_id() == 0 ? INT64_MAX : sh[warp_id() - 1];
    ex = min(carry, ex);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      ex = min(ex, v[k]);
      if (i0 - k >= 0) nf[i0 - k] = ex;
    }
    carry = min(carry, sh[(kScanThreads / 32) - 1]);
    __syncthreads();
  }
}

// Per position of the thread's 16 bytes: the run start before p0 is rs_in;
// calls f(position, run start, position in its chunk) for each byte inside
// the input.
template <typename F>
__device__ __forceinline__ void walk16(int64_t p0, int nv, uint32_t s, int64_t rs_in, F f) {
  int64_t rs = rs_in;
  int q = (int)((p0 - rs_in) % kCut);  // chunk position of p0 if it continues the run
#pragma unroll
  for (int k = 0; k < 16; k++) {
    if (k < nv) {
      if ((s >> k) & 1u) {
        rs = p0 + k;
        q = 0;
      }
      f(p0 + k, rs, q);
      q = q + 1 == kCut ? 0 : q + 1;
    }
  }
}

// The run start before each thread's first byte in tile t (block-wide
// exclusive max of the threads' last run starts, from lb[t]).
__device__ __forceinline__ int64_t run_start_in(int64_t p0, uint32_t s, int64_t lbt,
                                                int64_t *sh) {
  const int64_t last = s ? p0 + 31 - __clz(s) : -1;
  const int64_t inc = block_scan(last, sh, MaxOp());
  int64_t ex = __shfl_up_sync(0xffffffffu, (long long)inc, 1);
  if (lane_id() == 0) ex = warp_id() == 0 ? -1 : sh[warp_id() - 1];
  __syncthreads();
  return max(ex, lbt);
}

// c[t] = sum of cnt over tile t.
__global__ void __launch_bounds__(kSplitThreads)
    k_split_count(const uint8_t *__restrict__ in, int64_t n, int64_t T, const int64_t *lb,
                  int32_t *c) {
  const int64_t nwarps = (int64_t)gridDim.x * (kSplitThreads / 32);
  for (int64_t t = (int64_t)blockIdx.x * (kSplitThreads / 32) + warp_id(); t < T; t += nwarps) {
    const int64_t base = t * kSplitTile + (int64_t)lane_id() * kLaneBytes;
    uint8_t b[kLaneBytes / 16][16];
    uint32_t sm[kLaneBytes / 16];
    int nv[kLaneBytes / 16];
    int64_t last = -1;
#pragma unroll
    for (int piece = 0; piece < kLaneBytes / 16; piece++) {
      sm[piece] = load16(in, n, base + piece * 16, b[piece], nv[piece]);
      if (sm[piece]) last = base + piece * 16 + 31 - __clz(sm[piece]);
    }
    // the run start before this lane's bytes: exclusive max over earlier lanes
    int64_t inc = last;
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t v = __shfl_up_sync(0xffffffffu, (long long)inc, o);
      if ((int)lane_id() >= o) inc = max(inc, v);
    }
    int64_t rs = __shfl_up_sync(0xffffffffu, (long long)inc, 1);
    if (lane_id() == 0) rs = -1;
    rs = max(rs, lb[t]);
    int sum = 0;
#pragma unroll
    for (int piece = 0; piece < kLaneBytes / 16; piece++) {
      const int64_t p0 = base + piece * 16;
      walk16(p0, nv[piece], sm[piece], rs, [&](int64_t, int64_t, int q) { sum += cnt_of(q); });
      if (sm[piece]) rs = p0 + 31 - __clz(sm[piece]);
    }
    for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane_id() == 0) c[t] = sum;
  }
}

// P[t] = exclusive prefix of c, P[T] = total.  One thread block.
__global__ void __launch_bounds__(kScanThreads)
    k_split_prefix(int64_t T, const int32_t *c, int64_t *P) {
  __shared__ int64_t sh[32];
  constexpr int64_t kChunk = (int64_t)kScanThreads * kScanItems;
  int64_t carry = 0;
  for (int64_t base = 0; base < T; base += kChunk) {
    const int64_t i0 = base + (int64_t)threadIdx.x * kScanItems;
    int64_t v[kScanItems], m = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      v[k] = i0 + k < T ? c[i0 + k] : 0;
      m += v[k];
    }
    const int64_t inc = block_scan(m, sh, SumOp());
    int64_t ex = carry + inc - m;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      if (i0 + k < T) P[i0 + k] = ex;
      ex += v[k];
    }
    carry += sh[(kScanThreads / 32) - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) P[T] = carry;
}

// The walk over the blocks (one thread block).  ends[k] = end of block k;
// *count = blocks; *err != 0 if cap was too small.
__global__ void __launch_bounds__(kSplitThreads)
    k_split_chain(const uint8_t *__restrict__ in, int64_t n, int64_t T, const int64_t *P,
                  const int64_t *lb, const int64_t *nf, int64_t maxw, int64_t *ends, int cap,
                  int *count, int *err) {
  __shared__ int64_t sh[32];
  __shared__ int64_t s_start, s_G, s_x0, s_Gx0, s_rs0, s_re0, s_last_rs, s_span;
  __shared__ int s_nb;
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_start = 0;
    s_G = 0;
    s_nb = 0;
    s_span = 0;
  }
  __syncthreads();
  const int64_t PT = P[T];
  for (;;) {
    const int64_t s = s_start, Gs = s_G;
    if (s >= n) break;
    if (s_nb >= cap) {
      if (tid == 0) *err = 1;
      break;
    }
    const int64_t target = Gs + maxw;
    int64_t xend = n, Gx = PT;
    if (PT >= target) {
      // t* = the last tile with P[t*] < target (P[s's tile] <= Gs < target)
      const int64_t lo0 = s / kSplitTile;
      int64_t lo = lo0, hi = T;
      if (s_span > 0) {
        // first probes: 256 consecutive tiles around the tile the previous
        // block's span predicts (block sizes change slowly)
        const int64_t fv = max(lo + 1, lo + s_span - kSplitThreads / 2);
        const int64_t lv = min(hi - 1, fv + kSplitThreads - 1);
        if (fv <= lv) {
          const int64_t q = fv + tid;
          const int k = __syncthreads_count(q <= lv && P[q] < target);
          if (k == 0) {
            hi = fv;
          } else if (k == lv - fv + 1) {
            lo = lv;
          } else {
            lo = fv + k - 1;
            hi = fv + k;
          }
        }
      }
      while (hi - lo > 1) {
        const int64_t step = (hi - lo + kSplitThreads - 1) / kSplitThreads;
        const int64_t q = lo + (int64_t)(tid + 1) * step;
        const int k = __syncthreads_count(q < hi && P[q] < target);
        const int64_t nlo = lo + (int64_t)k * step;
        hi = min(hi, nlo + step);
        lo = nlo;
      }
      const int64_t t = lo;
      const int64_t p0 = t * kSplitTile + tid * 16;
      uint8_t b[16];
      int nv;
      const uint32_t sm = load16(in, n, p0, b, nv);
      const int64_t rs_in = run_start_in(p0, sm, lb[t], sh);
      int64_t sum = 0;
      walk16(p0, nv, sm, rs_in, [&](int64_t, int64_t, int q) { sum += cnt_of(q); });
      const int64_t inc = block_scan(sum, sh, SumOp());
      // x0: the first position of the tile with G(x0) >= target
      int64_t g = P[t] + inc - sum, my_x0 = INT64_MAX, my_rs = -1, my_g = 0, last_rs = -1;
      walk16(p0, nv, sm, rs_in, [&](int64_t p, int64_t rs, int q) {
        if (my_x0 == INT64_MAX && g >= target) {
          my_x0 = p;
          my_rs = rs;
          my_g = g;
        }
        g += cnt_of(q);
        last_rs = rs;
      });
      const int64_t x0m = block_scan(my_x0, sh, MinOp());
      if (tid == kSplitThreads - 1) s_x0 = x0m;
      __syncthreads();
      if (my_x0 != INT64_MAX && my_x0 == s_x0) {
        s_rs0 = my_rs;
        s_Gx0 = my_g;
      }
      // the tile's last byte: its run start (for x0 at the next tile)
      if (nv > 0 && p0 + nv == min(n, (t + 1) * kSplitTile)) s_last_rs = last_rs;
      // the first run start after x0 inside the tile
      const int64_t x0 = s_x0;
      int64_t my_re = INT64_MAX;
      if (x0 != INT64_MAX) {
        for (uint32_t r = sm; r; r &= r - 1) {
          const int64_t p = p0 + __ffs(r) - 1;
          if (p > x0) {
            my_re = p;
            break;
          }
        }
      }
      const int64_t rem = block_scan(my_re, sh, MinOp());
      if (tid == kSplitThreads - 1) s_re0 = rem;
      __syncthreads();
      if (tid == 0) {
        int64_t ax0 = s_x0, rs0, gx0, re0 = s_re0;
        if (ax0 == INT64_MAX) {
          // G reaches the target exactly at the next tile's first byte
          ax0 = min(n, (t + 1) * kSplitTile);
          gx0 = P[t + 1];
          rs0 = (ax0 < n && in[ax0] != in[ax0 - 1]) ? ax0 : s_last_rs;
          re0 = INT64_MAX;
        } else {
          rs0 = s_rs0;
          gx0 = s_Gx0;
        }
        if (re0 == INT64_MAX) re0 = t + 1 < T ? nf[t + 1] : n;
        if (ax0 >= n) {
          s_x0 = n;
          s_Gx0 = PT;
        } else {
          const int64_t q0 = (ax0 - rs0) % kCut;
          int64_t x = ax0, gx = gx0;
          if (q0 != 0) {
            x = min(ax0 + (kCut - q0), max(re0, ax0 + 1));
            x = min(x, n);
            gx = gx0 + cnt_below(q0 + (x - ax0)) - cnt_below(q0);
          }
          s_x0 = x;
          s_Gx0 = gx;
        }
      }
      __syncthreads();
      xend = s_x0;
      Gx = s_Gx0;
      if (xend >= n) {
        xend = n;
        Gx = PT;
      }
    }
    if (tid == 0) {
      ends[s_nb] = xend;
      s_nb++;
      s_span = xend / kSplitTile - s / kSplitTile;
      s_start = xend;
      s_G = Gx;
    }
    __syncthreads();
  }
  if (tid == 0) *count = s_nb;
}

}  // namespace

int64_t bzip2_split_max_blocks(int64_t n, int level) {
  const int64_t maxw = 100000LL * level - 19;
  // a block holds >= maxw RLE1 bytes and RLE1 writes at most 5 bytes per 4
  return n * 5 / 4 / maxw + 2;
}

std::vector<int64_t> bzip2_split(const uint8_t *d_in, int64_t n, int level, cudaStream_t st) {
  std::vector<int64_t> ends;
  if (n <= 0) return ends;
  level = std::min(std::max(level, 1), 9);
  const int64_t T = (n + kSplitTile - 1) / kSplitTile;
  const int64_t cap = bzip2_split_max_blocks(n, level);
  BZ_REQUIRE(cap < (int64_t)1 << 30, kErrTooLarge, "input too large for the bzip2 split");
  BZ_REQUIRE(T < (int64_t)1 << 31, kErrTooLarge, "input too large for the bzip2 split");
  // one scratch region per device, kept between calls (grown when too small):
  // fa, la, lb, nf, P (T + 1 each), c, ends, counters
  const size_t words = 5 * (size_t)(T + 1) + (size_t)(T + 1) / 2 + 1 + (size_t)cap + 2;
  struct Scratch {
    std::mutex mu;
    int64_t *p = nullptr;
    size_t words = 0;
  };
  static std::mutex table_mu;
  static std::vector<Scratch *> per_device;  // kept for the process lifetime
  int dev0 = 0;
  BZ_CUDA(cudaGetDevice(&dev0));
  Scratch *sc;
  {
    std::lock_guard<std::mutex> g(table_mu);
    if ((int)per_device.size() <= dev0) per_device.resize(dev0 + 1, nullptr);
    if (!per_device[dev0]) per_device[dev0] = new Scratch();
    sc = per_device[dev0];
  }
  std::lock_guard<std::mutex> hold(sc->mu);  // calls on one device take turns
  if (sc->words < words) {
    if (sc->p) BZ_CUDA(cudaFree(sc->p));
    sc->p = nullptr;
    sc->words = 0;
    BZ_CUDA(cudaMalloc((void **)&sc->p, words * 8));
    sc->words = words;
  }
  int64_t *buf = sc->p;
  int64_t *fa = buf, *la = fa + (T + 1), *lb = la + (T + 1), *nf = lb + (T + 1),
          *P = nf + (T + 1);
  int32_t *c = reinterpret_cast<int32_t *>(P + (T + 1));
  int64_t *dends = P + (T + 1) + (T + 1) / 2 + 1;
  int *counters = reinterpret_cast<int *>(dends + cap);
  BZ_CUDA(cudaMemsetAsync(counters, 0, 8, st));
  int dev = 0, sms = 0;
  BZ_CUDA(cudaGetDevice(&dev));
  BZ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const unsigned grid =
      (unsigned)std::min<int64_t>((T + kSplitThreads / 32 - 1) / (kSplitThreads / 32), (int64_t)sms * 8);
  k_split_runs<<<grid, kSplitThreads, 0, st>>>(d_in, n, T, fa, la);
  BZ_LAUNCH_CHECK();
  k_split_scan_runs<<<1, kScanThreads, 0, st>>>(T, n, la, fa, lb, nf);
  BZ_LAUNCH_CHECK();
  k_split_count<<<grid, kSplitThreads, 0, st>>>(d_in, n, T, lb, c);
  BZ_LAUNCH_CHECK();
  k_split_prefix<<<1, kScanThreads, 0, st>>>(T, c, P);
  BZ_LAUNCH_CHECK();
  k_split_chain<<<1, kSplitThreads, 0, st>>>(d_in, n, T, P, lb, nf, 100000LL * level - 19,
                                             dends, (int)cap, counters, counters + 1);
  BZ_LAUNCH_CHECK();
  int h[2] = {0, 0};
  BZ_CUDA(cudaMemcpyAsync(h, counters, 8, cudaMemcpyDeviceToHost, st));
  BZ_CUDA(cudaStreamSynchronize(st));
  BZ_REQUIRE(h[1] == 0 && h[0] > 0, kErrInternal, "bzip2 split: block bound exceeded");
  ends.resize(h[0]);
  BZ_CUDA(cudaMemcpyAsync(ends.data(), dends, 8 * (size_t)h[0], cudaMemcpyDeviceToHost, st));
  BZ_CUDA(cudaStreamSynchronize(st));
  return ends;
}

}  // namespace bz2g
