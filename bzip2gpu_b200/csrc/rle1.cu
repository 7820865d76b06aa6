// RLE1 (runs cut at C = 259, or 255 for bzip2 1.0.8's format) and the block
// CRC-32, over every block of a slab.
//
// Reference: src/compression/rle1.cu:13-113 (RLE1), src/compression/crc32.cpp
// (CRC).  A maximal run of length L is emitted as floor(L/C) chunks
// "cccc (C-4)" followed by the remainder r = L mod C: r < 4 copies of c, or
// "cccc (r-4)".  Position j of a run (j = i - run_start) emits
//   1 byte (c)            if j mod C < 3,
//   2 bytes (c, len-4)    if j mod C == 3,  len = length of its C-chunk,
//   nothing               otherwise,
// so every output offset is an exclusive scan of a per-position count, and the
// run start / end of a position are a max-scan / min-scan of run-start flags.
//
// CRC: crc0(D) (zero init, no final complement) is linear over GF(2).  Per
// 4096-byte tile, thread l takes 16 bytes and multiplies their crc0 by
// x^(8*16*(255-l)) mod P (a compile-time table), and the XOR of the 256
// products is the tile's crc0; the per-block kernel shifts each tile's crc0
// by x^(8 * bytes after the tile) (one thread per tile) and XORs them; the
// init term ~0 * x^(8n) is added at the end.
#include "crc.cuh"
#include "engine.h"

namespace bz2g {

namespace {


// Stage one raw tile into shared memory: sb[0..len) = bytes, *prev = byte
// before the tile (or -1 at the block start).
__device__ __forceinline__ int load_raw_tile(const SlabDev &d, int t, uint8_t *sb, int *blk,
                                             int *start, int *n_out, int *prev) {
  int b = d.rt_block[t];
  int st = d.rt_start[t];
  int n = d.raw_len[b];
  int len = min(kRawTile, n - st);
  const uint8_t *base = d.raw + d.raw_off[b] + st;
  int nw = (len + 15) >> 4;
  for (int w = threadIdx.x; w < nw; w += blockDim.x)
    reinterpret_cast<uint4 *>(sb)[w] = reinterpret_cast<const uint4 *>(base)[w];
  *prev = st > 0 ? (int)base[-1] : -1;
  *blk = b;
  *start = st;
  *n_out = n;
  return len;
}

// The thread's 16 bytes of the staged tile (positions p0 .. p0 + 15, with
// p0 = 16 * thread, one 16-byte shared load) and the mask of run starts among
// them: bit k is set when byte k lies in the tile and differs from the byte
// before it (`prev` before the tile, -1 at a block start).
__device__ __forceinline__ uint32_t tile_bytes(const uint8_t *sb, int p0, int len, int prev,
                                               uint8_t (&c)[kTileItems]) {
  const uint4 v = *reinterpret_cast<const uint4 *>(sb + p0);
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int k = 0; k < kTileItems; k++) c[k] = (uint8_t)(w[k >> 2] >> (8 * (k & 3)));
  int pv = p0 == 0 ? prev : (int)sb[p0 - 1];
  uint32_t starts = 0;
#pragma unroll
  for (int k = 0; k < kTileItems; k++) {
    if (p0 + k < len && (int)c[k] != pv) starts |= 1u << k;
    pv = c[k];
  }
  return starts;
}

// Output bytes of the positions [0, n) of a run (the per-position counts
// summed: 5 per chunk of `cut`, and 1, 1, 1, 2 for its first four).
__device__ __forceinline__ int rle1_out_upto(int n, int cut) {
  const int f = n / cut, r = n - f * cut;
  return 5 * f + (r < 4 ? r : 5);
}

// Which of a thread's 16 bytes (bit k: byte k) emit output: positions 0..3
// of a run chunk emit their byte (e), position 3 also a length byte (e3).
// sm: the run starts among the bytes; nv: bytes in the tile.  With carry,
// byte 0 continues a run at position q0 of its chunk; the chunk starts are
// then the run starts, the carried chunk's start (byte -q0) and, while the
// carried run lasts, its next chunk start (byte cut - q0; a run beginning
// among these bytes reaches no chunk end within them, as cut > 16).
// Without carry the bytes before the first run start emit nothing here.
// A byte emits when a chunk starts within the 4 bytes up to it; it emits a
// length too when that start is exactly 3 before it.
__device__ __forceinline__ void rle1_emit_masks(uint32_t sm, int q0, int nv, int cut, bool carry,
                                                uint32_t *e, uint32_t *e3) {
  uint32_t s4 = sm << 4;  // bit k + 4: byte k
  if (carry) {
    if (q0 <= 3) {
      s4 |= 1u << (4 - q0);
    } else {
      const int pw = cut - q0;
      if (pw < kTileItems && (sm & ((1u << pw) - 1u)) == 0) s4 |= 1u << (pw + 4);
    }
  }
  const uint32_t nvm = (1u << nv) - 1u;
  uint32_t em = ((s4 | (s4 << 1) | (s4 << 2) | (s4 << 3)) >> 4) & nvm;
  uint32_t em3 = (((s4 << 3) & ~(s4 << 2) & ~(s4 << 1) & ~s4) >> 4) & nvm;
  if (!carry) {
    const uint32_t keep = sm ? ~((sm & (0u - sm)) - 1u) : 0u;
    em &= keep;
    em3 &= keep;
  }
  *e = em;
  *e3 = em3;
}

// Per raw tile: its first and last run start, its crc0, and its RLE1 output
// bytes from its first run start on (the bytes before it continue a run from
// an earlier tile; the per-block kernel adds their count in closed form).
__global__ void __launch_bounds__(256) k_rle1_scan_tiles(SlabDev d) {
  __shared__ __align__(16) uint8_t sb[kRawTile + 16];
  __shared__ uint32_t tbl[256];
  __shared__ uint32_t red4[16];
  __shared__ int red[2][9];
  __shared__ int scratch[40];
  __shared__ int wl[8];
  const int t = blockIdx.x;
  int b, st, n, prev;
  crc_table_fill(tbl);
  red4_fill(red4);
  int len = load_raw_tile(d, t, sb, &b, &st, &n, &prev);
  __syncthreads();

  // run starts: first and last in this tile (block-local indices)
  const int p0 = threadIdx.x * kTileItems;
  uint8_t c[kTileItems];
  const uint32_t sm = tile_bytes(sb, p0, len, prev, c);
  int first = sm ? st + p0 + __ffs(sm) - 1 : INT32_MAX;
  int last = sm ? st + p0 + 31 - __clz(sm) : -1;
  // block min / max
  for (int o = 16; o > 0; o >>= 1) {
    first = min(first, __shfl_xor_sync(0xffffffffu, first, o));
    last = max(last, __shfl_xor_sync(0xffffffffu, last, o));
  }
  if (lane_id() == 0) {
    red[0][warp_id()] = first;
    red[1][warp_id()] = last;
  }
  {
    // output bytes: each thread's bytes from the last run start before them
    // in this tile (positions in the run modulo the cut); bytes before the
    // tile's first run start are left to the per-block kernel
    const int nv = min(kTileItems, max(0, len - p0));
    const int ls = sm ? st + p0 + 31 - __clz(sm) : -1;
    const int inc = block_incl_max(ls, scratch, -1);
    int ex = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane_id() == 31) wl[warp_id()] = inc;
    __syncthreads();
    if (lane_id() == 0) ex = warp_id() == 0 ? -1 : wl[warp_id() - 1];
    const int cut = d.run_cut;
    uint32_t em, em3;
    rle1_emit_masks(sm, ex >= 0 ? (st + p0 - ex) % cut : 0, nv, cut, ex >= 0, &em, &em3);
    const int cnt = __popc(em) + __popc(em3);
    int total;
    block_excl_sum(cnt, scratch, &total);
    if (threadIdx.x == 0) d.tile_c[t] = total;
  }

  // crc0 of the tile, right-aligned into a virtual 4096-byte tile (leading
  // zeros leave a zero-init CRC unchanged): 16 bytes per thread, each
  // thread's crc0 moved to the tile's end by one multiplication, then XOR.
  __shared__ uint32_t wcrc[8];
  {
    const int pad = kRawTile - len;
    uint32_t r = 0;
    const int v0 = threadIdx.x * 16;
    if (pad == 0) {
#pragma unroll
      for (int k = 0; k < kTileItems; k++) r = (r << 8) ^ tbl[(r >> 24) ^ c[k]];
    } else {
      for (int v = max(v0, pad); v < v0 + 16; v++) {
        uint32_t byte = sb[v - pad];
        r = (r << 8) ^ tbl[(r >> 24) ^ byte];
      }
    }
    r = gf_mul_lane(r, threadIdx.x, red4);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r ^= __shfl_xor_sync(0xffffffffu, r, o);
    if (lane_id() == 0) wcrc[warp_id()] = r;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t r = 0;
    for (int w = 0; w < 8; w++) r ^= wcrc[w];
    d.tile_d[t] = (int32_t)r;  // the tile's crc0 (shifted per block)
  }
  if (threadIdx.x == 0) {
    int f = INT32_MAX, l = -1;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      f = min(f, red[0][w]);
      l = max(l, red[1][w]);
    }
    d.tile_a[t] = f;  // first run start in tile
    d.tile_b[t] = l;  // last run start in tile
  }
}

// Per block: exclusive max of last-starts (run start carried into a tile) and
// exclusive min of first-starts (next run start after a tile), and the CRC.
__global__ void __launch_bounds__(256) k_rle1_block_carry(SlabDev d, const int *rt_first) {
  __shared__ int scratch[40];
  __shared__ int sx[256];
  const int b = blockIdx.x;
  const int t0 = rt_first[b], nt = rt_first[b + 1] - t0;
  const int n = d.raw_len[b];
  int carry = -1, out_carry = 0;
  const int cut = d.run_cut;
  for (int base = 0; base < nt; base += 256) {
    int k = base + threadIdx.x;
    int v = k < nt ? d.tile_b[t0 + k] : -1;
    int inc = block_incl_max(v, scratch, -1);
    sx[threadIdx.x] = inc;
    __syncthreads();
    int ex = threadIdx.x == 0 ? carry : max(carry, sx[threadIdx.x - 1]);
    int cnt = 0;
    if (k < nt) {
      d.tile_b[t0 + k] = ex;
      // the tile's output: its own count plus that of its bytes before its
      // first run start, positions j0 .. j0 + pre - 1 of the run begun at ex
      const int st = d.rt_start[t0 + k];
      const int len = min(kRawTile, n - st);
      const int fs = d.tile_a[t0 + k];
      const int pre = (fs == INT32_MAX ? st + len : fs) - st;
      const int j0 = st - ex;
      cnt = d.tile_c[t0 + k] + (pre > 0 ? rle1_out_upto(j0 + pre, cut) - rle1_out_upto(j0, cut) : 0);
    }
    int c2 = max(carry, sx[255]);
    __syncthreads();
    carry = c2;
    int tot;
    const int o = block_excl_sum(cnt, scratch, &tot);
    if (k < nt) d.tile_c[t0 + k] = out_carry + o;
    out_carry += tot;
  }
  if (threadIdx.x == 0) d.m[b] = out_carry;
  int carry_min = n;
  // walk backwards for the suffix minimum
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
  // block CRC: each tile's crc0 shifted by x^(8 * bytes after it), XOR-ed
  uint32_t acc = 0;
  for (int k = threadIdx.x; k < nt; k += blockDim.x) {
    const int st = d.rt_start[t0 + k];
    const int len = min(kRawTile, n - st);
    const uint32_t c = (uint32_t)d.tile_d[t0 + k];
    if (c) acc ^= gf_mul(c, xpow8((uint64_t)(n - (st + len))));
  }
  for (int o = 16; o > 0; o >>= 1) acc ^= __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane_id() == 0) scratch[warp_id()] = (int)acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t a = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) a ^= (uint32_t)scratch[w];
    d.crc[b] = ~(gf_mul(0xFFFFFFFFu, xpow8((uint64_t)n)) ^ a);
  }
}

__global__ void __launch_bounds__(256) k_rle1_write(SlabDev d) {
  __shared__ __align__(16) uint8_t sb[kRawTile + 16];
  __shared__ __align__(16) uint8_t so[kRawTile + kRawTile / 4 + 16];  // the tile's output
  __shared__ int scratch[40];
  __shared__ int wl[8], wf[8];
  const int t = blockIdx.x;
  int b, st, n, prev;
  int len = load_raw_tile(d, t, sb, &b, &st, &n, &prev);
  __syncthreads();
  const int p0 = threadIdx.x * kTileItems;
  uint8_t c[kTileItems];
  const uint32_t sm = tile_bytes(sb, p0, len, prev, c);
  const int nv = min(kTileItems, max(0, len - p0));
  int ls = sm ? st + p0 + 31 - __clz(sm) : -1;
  int fs = sm ? st + p0 + __ffs(sm) - 1 : INT32_MAX;
  // exclusive max of last starts over earlier threads
  int inc = warp_incl_max(ls);
  int exw = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane_id() == 31) wl[warp_id()] = inc;
  // exclusive min of first starts over later threads
  int incm = warp_incl_min_rev(fs);
  int exm = __shfl_down_sync(0xffffffffu, incm, 1);
  if (lane_id() == 0) wf[warp_id()] = incm;
  __syncthreads();
  int before = lane_id() == 0 ? -1 : exw;
  for (int w = 0; w < (int)warp_id(); w++) before = max(before, wl[w]);
  int after = lane_id() == 31 ? INT32_MAX : exm;
  for (int w = warp_id() + 1; w < (int)(blockDim.x >> 5); w++) after = min(after, wf[w]);
  before = max(before, d.tile_b[t]);
  after = min(after, d.tile_a[t]);  // next start after the tile (or n)

  // each byte's emits: its position in its chunk from the run start before
  // the thread (one division per thread), then bit masks
  const int cut = d.run_cut;
  const int pbase = st + p0;  // block-local position of byte 0
  uint32_t em = 0, em3 = 0;
  if (nv > 0)
    rle1_emit_masks(sm, before >= 0 ? (pbase - before) % cut : 0, nv, cut, before >= 0, &em, &em3);
  int tot;
  const int o = block_excl_sum(__popc(em) + __popc(em3), scratch, &tot);
  uint8_t *out = so + o;
#pragma unroll
  for (int k = 0; k < kTileItems; k++) {
    if ((em >> k) & 1u) {
      const uint32_t below = (1u << k) - 1u;
      const int at = __popc(em & below) + __popc(em3 & below);
      out[at] = c[k];
      if ((em3 >> k) & 1u) {
        // the chunk's length: from its start (3 bytes back) to the run's end
        // or the cut, whichever comes first
        const uint32_t rest = k + 1 < kTileItems ? sm >> (k + 1) : 0u;
        const int run_end = rest ? pbase + k + __ffs(rest) : after;
        out[at + 1] = (uint8_t)(min(cut, run_end - (pbase + k - 3)) - 4);
      }
    }
  }
  __syncthreads();
  // coalesced copy of the tile's output to its place in the block
  uint8_t *dst = d.rle1 + d.off[b] + d.tile_c[t];
  for (int i = threadIdx.x; i < tot; i += blockDim.x) dst[i] = so[i];
}

}  // namespace

void stage_rle1_crc(const SlabDev &d, cudaStream_t st) {
  const int *rt_first = d.rt_first;
  if (d.n_raw_tiles > 0) {
    k_rle1_scan_tiles<<<d.n_raw_tiles, 256, 0, st>>>(d);
    BZ_LAUNCH_CHECK();
  }
  k_rle1_block_carry<<<d.nblocks, 256, 0, st>>>(d, rt_first);
  BZ_LAUNCH_CHECK();
  if (d.n_raw_tiles > 0) {
    k_rle1_write<<<d.n_raw_tiles, 256, 0, st>>>(d);
    BZ_LAUNCH_CHECK();
  }
}

void launch_crc_only(const SlabDev &d, cudaStream_t st) {
  const int *rt_first = d.rt_first;
  if (d.n_raw_tiles > 0) {
    k_rle1_scan_tiles<<<d.n_raw_tiles, 256, 0, st>>>(d);
    BZ_LAUNCH_CHECK();
  }
  k_rle1_block_carry<<<d.nblocks, 256, 0, st>>>(d, rt_first);
  BZ_LAUNCH_CHECK();
}

}  // namespace bz2g
