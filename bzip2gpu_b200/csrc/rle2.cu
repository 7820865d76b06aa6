// RLE2: MTF values to bzip2 symbols, with the per-block symbol histogram.
//
// Reference: src/compression/rle2.cu:11-158 (and its oracle
// tests/compression/rle2.cu:9-33).  A value v > 0 becomes v + 1; a run of k
// zeros becomes the bijective base-2 digits of k, least significant first,
// RUNA (0) for digit 1 and RUNB (1) for digit 2 -- floor(log2(k+1)) symbols;
// EOB = nInUse + 1 ends the block.  Position q of a zero run emits digit q if
// q < floor(log2(k+1)), so output offsets are a scan of 0/1 counts and the
// run bounds are a max-scan / min-scan of non-zero positions.
#include "engine.h"

namespace bz2g {

namespace {

__device__ __forceinline__ int tile_len(const SlabDev &d, int t, int *b, int *lt, int64_t *off,
                                        int *m) {
  *b = d.tile_block[t];
  *off = d.off[*b];
  *lt = (int)((int64_t)t * kTile - *off);
  *m = d.m[*b];
  return min(kTile, *m - *lt);
}

__global__ void __launch_bounds__(256) k_rle2_scan_tiles(SlabDev d, const int32_t *list) {
  const int t = list ? list[blockIdx.x] : (int)blockIdx.x;
  __shared__ int red[2][8];
  int b, lt, m;
  int64_t off;
  int valid = tile_len(d, t, &b, &lt, &off, &m);
  if (valid <= 0) return;
  const uint8_t *V = d.mtf + off;
  int first = INT32_MAX, last = -1;
  for (int e = threadIdx.x; e < valid; e += blockDim.x) {
    if (V[lt + e] != 0) {
      first = min(first, lt + e);
      last = max(last, lt + e);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    first = min(first, __shfl_xor_sync(0xffffffffu, first, o));
    last = max(last, __shfl_xor_sync(0xffffffffu, last, o));
  }
  if (lane_id() == 0) {
    red[0][warp_id()] = first;
    red[1][warp_id()] = last;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int f = INT32_MAX, l = -1;
    for (int w = 0; w < 8; w++) {
      f = min(f, red[0][w]);
      l = max(l, red[1][w]);
    }
    d.tile_a[t] = f;
    d.tile_b[t] = l;
  }
}

// Per block: previous non-zero before each tile (tile_b) and next non-zero
// after each tile (tile_a, m if none).
__global__ void __launch_bounds__(256) k_rle2_block_carry(SlabDev d) {
  __shared__ int scratch[40];
  __shared__ int sx[256];
  const int b = blockIdx.x;
  const int m = d.m[b];
  if (m <= 0) return;
  const int nt = (m + kTile - 1) / kTile;
  const int t0 = (int)(d.off[b] / kTile);
  int carry = -1;
  for (int base = 0; base < nt; base += 256) {
    int k = base + threadIdx.x;
    int v = k < nt ? d.tile_b[t0 + k] : -1;
    int inc = block_incl_max(v, scratch, -1);
    sx[threadIdx.x] = inc;
    __syncthreads();
    int ex = threadIdx.x == 0 ? carry : max(carry, sx[threadIdx.x - 1]);
    if (k < nt) d.tile_b[t0 + k] = ex;
    int c2 = max(carry, sx[255]);
    __syncthreads();
    carry = c2;
  }
  int carry_min = m;
  for (int base = ((nt - 1) / 256) * 256; base >= 0; base -= 256) {
    int k = base + threadIdx.x;
    int v = k < nt ? d.tile_a[t0 + k] : INT32_MAX;
    int inc = block_suffix_min(v, scratch, INT32_MAX);
    sx[threadIdx.x] = inc;
    __syncthreads();
    int ex = threadIdx.x == 255 ? carry_min : min(carry_min, sx[threadIdx.x + 1]);
    if (k < nt) d.tile_a[t0 + k] = ex;
    int c2 = min(carry_min, sx[0]);
    __syncthreads();
    carry_min = c2;
  }
}

__device__ __forceinline__ int n_digits(int k) { return 31 - __clz(k + 1); }

// Thread-blocked view of a tile: each thread owns kTileItems consecutive
// positions and learns the previous / next non-zero around each of them.
struct ZeroRuns {
  int before, after;
};

__device__ __forceinline__ ZeroRuns zero_run_bounds(const SlabDev &d, const uint8_t *V, int t,
                                                    int lt, int valid, int p0, int *wl, int *wf) {
  int ls = -1, fs = INT32_MAX;
  for (int k = 0; k < kTileItems; k++) {
    int e = p0 + k;
    if (e >= valid) break;
    if (V[lt + e] != 0) {
      ls = lt + e;
      fs = min(fs, lt + e);
    }
  }
  int inc = warp_incl_max(ls);
  int exw = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane_id() == 31) wl[warp_id()] = inc;
  int incm = warp_incl_min_rev(fs);
  int exm = __shfl_down_sync(0xffffffffu, incm, 1);
  if (lane_id() == 0) wf[warp_id()] = incm;
  __syncthreads();
  int before = lane_id() == 0 ? -1 : exw;
  for (int w = 0; w < (int)warp_id(); w++) before = max(before, wl[w]);
  int after = lane_id() == 31 ? INT32_MAX : exm;
  for (int w = warp_id() + 1; w < (int)(blockDim.x >> 5); w++) after = min(after, wf[w]);
  ZeroRuns r;
  r.before = max(before, d.tile_b[t]);
  r.after = min(after, d.tile_a[t]);
  return r;
}

__global__ void __launch_bounds__(256) k_rle2_count(SlabDev d, const int32_t *list) {
  const int t = list ? list[blockIdx.x] : (int)blockIdx.x;
  __shared__ int scratch[40];
  __shared__ int wl[8], wf[8];
  int b, lt, m;
  int64_t off;
  int valid = tile_len(d, t, &b, &lt, &off, &m);
  if (valid <= 0) return;
  const uint8_t *V = d.mtf + off;
  const int p0 = threadIdx.x * kTileItems;
  ZeroRuns zr = zero_run_bounds(d, V, t, lt, valid, p0, wl, wf);
  int ends[kTileItems];
  {
    int cur = zr.after;
#pragma unroll
    for (int k = kTileItems - 1; k >= 0; k--) {
      int e = p0 + k;
      ends[k] = cur;
      if (e < valid && V[lt + e] != 0) cur = lt + e;
    }
  }
  int cnt = 0, prev_nz = zr.before;
#pragma unroll
  for (int k = 0; k < kTileItems; k++) {
    int e = p0 + k;
    if (e < valid) {
      if (V[lt + e] != 0) {
        cnt++;
        prev_nz = lt + e;
      } else {
        int zs = prev_nz + 1;
        int q = lt + e - zs;
        cnt += q < n_digits(ends[k] - zs) ? 1 : 0;
      }
    }
  }
  int tot;
  block_excl_sum(cnt, scratch, &tot);
  if (threadIdx.x == 0) d.tile_c[t] = tot;
}

__global__ void __launch_bounds__(256) k_rle2_block_offsets(SlabDev d) {
  __shared__ int scratch[40];
  const int b = blockIdx.x;
  const int m = d.m[b];
  const int nt = m > 0 ? (m + kTile - 1) / kTile : 0;
  const int t0 = (int)(d.off[b] / kTile);
  int carry = 0;
  for (int base = 0; base < nt; base += 256) {
    int k = base + threadIdx.x;
    int v = k < nt ? d.tile_c[t0 + k] : 0;
    int tot;
    int ex = block_excl_sum(v, scratch, &tot);
    if (k < nt) d.tile_c[t0 + k] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) {
    int eob = d.n_in_use[b] + 1;
    d.rle2[d.off[b] + carry] = (uint16_t)eob;
    d.s[b] = carry + 1;
    atomicAdd(&d.freq[b * kMaxAlpha + eob], 1);
  }
}

__global__ void __launch_bounds__(256) k_rle2_write(SlabDev d, const int32_t *list) {
  const int t = list ? list[blockIdx.x] : (int)blockIdx.x;
  __shared__ int scratch[40];
  __shared__ int wl[8], wf[8];
  __shared__ int hist[kMaxAlpha];
  int b, lt, m;
  int64_t off;
  int valid = tile_len(d, t, &b, &lt, &off, &m);
  if (valid <= 0) return;
  for (int i = threadIdx.x; i < kMaxAlpha; i += blockDim.x) hist[i] = 0;
  const uint8_t *V = d.mtf + off;
  const int p0 = threadIdx.x * kTileItems;
  ZeroRuns zr = zero_run_bounds(d, V, t, lt, valid, p0, wl, wf);
  int ends[kTileItems];
  {
    int cur = zr.after;
#pragma unroll
    for (int k = kTileItems - 1; k >= 0; k--) {
      int e = p0 + k;
      ends[k] = cur;
      if (e < valid && V[lt + e] != 0) cur = lt + e;
    }
  }
  int cnt = 0;
  {
    int prev_nz = zr.before;
#pragma unroll
    for (int k = 0; k < kTileItems; k++) {
      int e = p0 + k;
      if (e < valid) {
        if (V[lt + e] != 0) {
          cnt++;
          prev_nz = lt + e;
        } else {
          int zs = prev_nz + 1;
          cnt += (lt + e - zs) < n_digits(ends[k] - zs) ? 1 : 0;
        }
      }
    }
  }
  int tot;
  int o = block_excl_sum(cnt, scratch, &tot);
  uint16_t *out = d.rle2 + off + d.tile_c[t] + o;
  int prev_nz = zr.before;
  // RUNA, RUNB and symbol 2 (MTF index 1) are most of the symbols: counted
  // in registers, added to the tile's histogram once per thread
  int h0 = 0, h1 = 0, h2 = 0;
#pragma unroll
  for (int k = 0; k < kTileItems; k++) {
    int e = p0 + k;
    if (e < valid) {
      int v = V[lt + e];
      if (v != 0) {
        *out++ = (uint16_t)(v + 1);
        if (v == 1)
          h2++;
        else
          atomicAdd(&hist[v + 1], 1);
        prev_nz = lt + e;
      } else {
        int zs = prev_nz + 1;
        int q = lt + e - zs;
        int k2 = ends[k] - zs;
        if (q < n_digits(k2)) {
          int dgt = 0;
          for (int r = 0; r <= q; r++) {
            k2--;
            dgt = k2 & 1;
            k2 >>= 1;
          }
          *out++ = (uint16_t)dgt;
          h0 += dgt == 0;
          h1 += dgt == 1;
        }
      }
    }
  }
  if (h0) atomicAdd(&hist[0], h0);
  if (h1) atomicAdd(&hist[1], h1);
  if (h2) atomicAdd(&hist[2], h2);
  __syncthreads();
  for (int i = threadIdx.x; i < kMaxAlpha; i += blockDim.x)
    if (hist[i]) atomicAdd(&d.freq[b * kMaxAlpha + i], hist[i]);
}

}  // namespace

void stage_rle2(const SlabDev &d, cudaStream_t st) {
  BZ_CUDA(cudaMemsetAsync(d.freq, 0, sizeof(int32_t) * kMaxAlpha * d.nblocks, st));
  const int nlive = live_tiles(d, st);
  const int grid = nlive >= 0 ? nlive : d.ntiles;
  const int32_t *list = nlive >= 0 ? d.vt_list : nullptr;
  if (grid > 0) {
    k_rle2_scan_tiles<<<grid, 256, 0, st>>>(d, list);
    BZ_LAUNCH_CHECK();
  }
  k_rle2_block_carry<<<d.nblocks, 256, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
  if (grid > 0) {
    k_rle2_count<<<grid, 256, 0, st>>>(d, list);
    BZ_LAUNCH_CHECK();
  }
  k_rle2_block_offsets<<<d.nblocks, 256, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
  if (grid > 0) {
    k_rle2_write<<<grid, 256, 0, st>>>(d, list);
    BZ_LAUNCH_CHECK();
  }
}

}  // namespace bz2g
