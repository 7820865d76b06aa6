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

__device__ __forceinline__ int n_digits(int k) { return 31 - __clz(k + 1); }

// Thread-blocked view of a tile: each thread owns kTileItems consecutive
// positions and learns the previous / next non-zero around each of them.
struct ZeroRuns {
  int before, after;
};

// The thread's 16 MTF values (one 16-byte load; the buffer has slack past
// a block's end, and values at or past `valid` are not used).
struct Values16 {
  uint32_t w[4];
  __device__ __forceinline__ int operator[](int k) const { return (w[k >> 2] >> (8 * (k & 3))) & 0xff; }
};
__device__ __forceinline__ void load_values(const uint8_t *V, int lt, int p0, int valid,
                                            Values16 &v) {
  uint4 w = make_uint4(0, 0, 0, 0);
  if (p0 < valid) w = *reinterpret_cast<const uint4 *>(V + lt + p0);
  v.w[0] = w.x;
  v.w[1] = w.y;
  v.w[2] = w.z;
  v.w[3] = w.w;
}

// carry: include the non-zeros of the other tiles (tile_b / tile_a after the
// per-block kernel); without it, -1 / INT32_MAX when the tile has none.
__device__ __forceinline__ ZeroRuns zero_run_bounds(const SlabDev &d, const Values16 &v,
                                                    int t, int lt, int valid, int p0, int *wl,
                                                    int *wf, bool carry = true) {
  int ls = -1, fs = INT32_MAX;
#pragma unroll
  for (int k = kTileItems - 1; k >= 0; k--) {
    if (p0 + k < valid && v[k] != 0) {
      ls = max(ls, lt + p0 + k);
      fs = lt + p0 + k;
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
  r.before = carry ? max(before, d.tile_b[t]) : before;
  r.after = carry ? min(after, d.tile_a[t]) : after;
  return r;
}

// Per tile: first and last non-zero (tile_a, tile_b, and the first again in
// tile_d), and the output symbols of its non-zeros and of the zero runs
// between two of its non-zeros (tile_c); the zero runs at its ends are
// counted by the per-block kernel, which knows where they start and end.
__global__ void __launch_bounds__(256) k_rle2_scan_tiles(SlabDev d, const int32_t *list) {
  const int t = list ? list[blockIdx.x] : (int)blockIdx.x;
  __shared__ int scratch[40];
  __shared__ int wl[8], wf[8];
  __shared__ int red[2][8];
  int b, lt, m;
  int64_t off;
  int valid = tile_len(d, t, &b, &lt, &off, &m);
  if (valid <= 0) return;
  const int p0 = threadIdx.x * kTileItems;
  Values16 v;
  load_values(d.mtf + off, lt, p0, valid, v);
  ZeroRuns zr = zero_run_bounds(d, v, t, lt, valid, p0, wl, wf, false);
  uint32_t nzm = 0;
#pragma unroll
  for (int k = 0; k < kTileItems; k++) nzm |= (p0 + k < valid && v[k] != 0) ? 1u << k : 0u;
  int cnt = __popc(nzm);
  int prev_nz = zr.before;
#pragma unroll
  for (int k = 0; k < kTileItems; k++) {
    if (p0 + k < valid) {
      if ((nzm >> k) & 1u) {
        prev_nz = lt + p0 + k;
      } else if (prev_nz >= 0) {
        const uint32_t rest = k + 1 < kTileItems ? nzm >> (k + 1) : 0u;
        const int end = rest ? lt + p0 + k + __ffs(rest) : zr.after;
        if (end != INT32_MAX) {
          const int zs = prev_nz + 1;
          cnt += (lt + p0 + k - zs) < n_digits(end - zs) ? 1 : 0;
        }
      }
    }
  }
  int tot;
  block_excl_sum(cnt, scratch, &tot);
  int first = nzm ? lt + p0 + __ffs(nzm) - 1 : INT32_MAX;
  int last = nzm ? lt + p0 + 31 - __clz(nzm) : -1;
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
    d.tile_d[t] = f;
    d.tile_c[t] = tot;
  }
}

// Per block: previous non-zero before each tile (tile_b) and next non-zero
// after each tile (tile_a, m if none); tile output offsets (tile_c), the
// symbol count s with the EOB written and counted.
__global__ void __launch_bounds__(256) k_rle2_block_carry(SlabDev d) {
  __shared__ int scratch[40];
  __shared__ int sx[256];
  const int b = blockIdx.x;
  const int m = d.m[b];
  if (m <= 0) {
    if (threadIdx.x == 0) {
      const int eob = d.n_in_use[b] + 1;
      d.rle2[d.off[b]] = (uint16_t)eob;
      d.s[b] = 1;
      atomicAdd(&d.freq[b * kMaxAlpha + eob], 1);
    }
    return;
  }
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
  // Each tile's output: its own count plus the digits of the zero runs at
  // its ends that fall inside it (a zero run of length n starting at zs
  // emits its digits at positions zs .. zs + n_digits(n) - 1), then the
  // tile offsets, the block's symbol count and its EOB.
  int out_carry = 0;
  for (int base = 0; base < nt; base += 256) {
    const int k = base + threadIdx.x;
    int cnt = 0;
    if (k < nt) {
      const int t = t0 + k;
      const int lt = k * kTile;
      const int te = min(lt + kTile, m);
      const int first = d.tile_d[t];  // first non-zero in the tile
      const int prev = d.tile_b[t];   // last non-zero before the tile
      const int next = d.tile_a[t];   // first non-zero after the tile, or m
      auto digits_in = [](int zs, int end, int a, int b) {  // of run [zs, end), at [a, b)
        if (end <= zs || b <= a) return 0;
        const int nd = n_digits(end - zs);
        return min(b - zs, nd) - min(a - zs, nd);
      };
      cnt = d.tile_c[t];
      if (first == INT32_MAX) {
        cnt += digits_in(prev + 1, next, lt, te);
      } else {
        cnt += digits_in(prev + 1, first, lt, first);
        // the last non-zero of this tile is the last one before the next
        const int last = k + 1 < nt ? d.tile_b[t + 1] : carry;
        cnt += digits_in(last + 1, next, last + 1, te);
      }
    }
    int tot;
    const int o = block_excl_sum(cnt, scratch, &tot);
    if (k < nt) d.tile_c[t0 + k] = out_carry + o;
    out_carry += tot;
  }
  if (threadIdx.x == 0) {
    const int eob = d.n_in_use[b] + 1;
    d.rle2[d.off[b] + out_carry] = (uint16_t)eob;
    d.s[b] = out_carry + 1;
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
  Values16 v;
  load_values(V, lt, p0, valid, v);
  ZeroRuns zr = zero_run_bounds(d, v, t, lt, valid, p0, wl, wf);
  // non-zero values as a mask; the end of the zero run holding value k is
  // the next non-zero after it
  uint32_t nzm = 0;
#pragma unroll
  for (int k = 0; k < kTileItems; k++) nzm |= (p0 + k < valid && v[k] != 0) ? 1u << k : 0u;
  auto run_end = [&](int k) {
    const uint32_t rest = k + 1 < kTileItems ? nzm >> (k + 1) : 0u;
    return rest ? lt + p0 + k + __ffs(rest) : zr.after;
  };
  int cnt = 0;
  {
    int prev_nz = zr.before;
#pragma unroll
    for (int k = 0; k < kTileItems; k++) {
      int e = p0 + k;
      if (e < valid) {
        if (v[k] != 0) {
          cnt++;
          prev_nz = lt + e;
        } else {
          int zs = prev_nz + 1;
          cnt += (lt + e - zs) < n_digits(run_end(k) - zs) ? 1 : 0;
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
      const int x = v[k];
      if (x != 0) {
        *out++ = (uint16_t)(x + 1);
        if (x == 1)
          h2++;
        else
          atomicAdd(&hist[x + 1], 1);
        prev_nz = lt + e;
      } else {
        int zs = prev_nz + 1;
        int q = lt + e - zs;
        int k2 = run_end(k) - zs;
        if (q < n_digits(k2)) {
          // digit q of the run length in bijective base 2 (RUNA = 0 for 1,
          // RUNB = 1 for 2) is bit q of length + 1
          const int dgt = ((k2 + 1) >> q) & 1;
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
    k_rle2_write<<<grid, 256, 0, st>>>(d, list);
    BZ_LAUNCH_CHECK();
  }
}

}  // namespace bz2g
