// Block headers, payload bit packing and stream placement, for a slab.
//
// Reference: src/compression/huffman_encode.cu:15-143 (per-symbol code from
// the group's table, exclusive scan of code lengths to bit offsets, MSB-first
// placement) and src/compression/compress.cu:119-137,284-375 (selector MTF
// and the block header fields).  Here the block header and payload are written
// straight to their final bit position in the .bz2 stream: the output is an
// array of big-endian 32-bit words (so memory order is stream byte order),
// zeroed first and OR-ed into, since neighbouring blocks share edge words.
#include "engine.h"

namespace bz2g {

namespace {

__device__ __forceinline__ uint32_t bswap32(uint32_t w) { return __byte_perm(w, 0, 0x0123); }

// MSB-first bit writer into zeroed big-endian words.
struct BitSink {
  uint32_t *out;
  int64_t word;
  uint64_t acc;
  int n;
  __device__ void init(uint32_t *o, int64_t bit) {
    out = o;
    word = bit >> 5;
    acc = 0;
    n = (int)(bit & 31);
  }
  __device__ __forceinline__ void put(uint32_t v, int nb) {
    acc = (acc << nb) | v;
    n += nb;
    if (n >= 32) {
      uint32_t w = (uint32_t)(acc >> (n - 32));
      atomicOr(out + word, bswap32(w));
      word++;
      n -= 32;
    }
  }
  __device__ void flush() {
    if (n > 0) atomicOr(out + word, bswap32((uint32_t)(acc << (32 - n))));
    n = 0;
  }
};

// Per block: selector MTF (src/compression/compress.cu:119-137) and the
// header size.  256 threads split the selectors into chunks; the MTF list at
// a chunk's start is the tables ordered by their last use before it (most
// recent first, unused ones in index order), read off a prefix max over the
// threads of each table's last position, so every chunk then runs its MTF on
// its own.
constexpr int kHdrThreads = 256;

__device__ __forceinline__ int sel_chunk(int nsel, int *a, int *e) {
  const int per = (nsel + kHdrThreads - 1) / kHdrThreads;
  *a = min(nsel, (int)threadIdx.x * per);
  *e = min(nsel, *a + per);
  return per;
}

__device__ int64_t table_bits(const uint8_t *len, int alpha) {
  int cur = len[0];
  int64_t tb = 5;
  for (int v = 0; v < alpha; v++) {
    int tg = len[v];
    tb += 2 * abs(tg - cur) + 1;
    cur = tg;
  }
  return tb;
}

__device__ int used_ranges(const uint32_t *pres) {
  int r = 0;
  for (int q = 0; q < 16; q++) r += ((pres[q >> 1] >> ((q & 1) * 16)) & 0xffffu) != 0;
  return r;
}

__global__ void __launch_bounds__(kHdrThreads) k_sel_mtf_hdr(SlabDev d) {
  __shared__ int scratch[40];
  __shared__ int64_t tbits[kMaxGroups];
  const int b = blockIdx.x;
  const int ngrp = d.n_groups[b];
  const int nsel = d.n_sel[b];
  const int alpha = d.n_in_use[b] + 2;
  const uint8_t *sel = d.sel + d.off[b] / 32;
  uint8_t *smtf = d.sel_mtf + d.off[b] / 32;
  int a, e;
  sel_chunk(nsel, &a, &e);
  int last[kMaxGroups];
#pragma unroll
  for (int t = 0; t < kMaxGroups; t++) last[t] = -1;
  for (int i = a; i < e; i++) {
    const int v = sel[i];
#pragma unroll
    for (int t = 0; t < kMaxGroups; t++)
      if (v == t) last[t] = i;
  }
  int prev[kMaxGroups];
#pragma unroll
  for (int t = 0; t < kMaxGroups; t++) {
    int inc = block_incl_max(last[t], scratch, -1);
    int ex = __shfl_up_sync(0xffffffffu, inc, 1);
    __shared__ int wl[kHdrThreads / 32];
    if (lane_id() == 31) wl[warp_id()] = inc;
    __syncthreads();
    if (lane_id() == 0) ex = warp_id() == 0 ? -1 : wl[warp_id() - 1];
    prev[t] = ex;
    __syncthreads();
  }
  // starting list: used tables by last use (latest first), then unused ones
  uint8_t pos[kMaxGroups];
  {
    int key[kMaxGroups];
    for (int t = 0; t < ngrp; t++) key[t] = prev[t] >= 0 ? prev[t] : -1 - t;
    for (int t = 0; t < ngrp; t++) {
      int r = 0;
      for (int u = 0; u < ngrp; u++) r += key[u] > key[t];
      pos[r] = (uint8_t)t;
    }
  }
  int unary = 0;
  for (int i = a; i < e; i++) {
    const uint8_t v = sel[i];
    int j = 0;
    uint8_t tmp = pos[0];
    while (v != tmp) {
      j++;
      uint8_t t2 = tmp;
      tmp = pos[j];
      pos[j] = t2;
    }
    pos[0] = tmp;
    smtf[i] = (uint8_t)j;
    unary += j + 1;
  }
  int total_unary;
  block_excl_sum(unary, scratch, &total_unary);
  if ((int)threadIdx.x < ngrp)
    tbits[threadIdx.x] =
        table_bits(d.len + ((size_t)b * kMaxGroups + threadIdx.x) * kMaxAlpha, alpha);
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t tb = 0;
    for (int t = 0; t < ngrp; t++) tb += tbits[t];
    const int ranges = used_ranges(d.present + b * 8);
    d.hdr_bits[b] = 48 + 32 + 1 + 24 + 16 + 16 * ranges + 3 + 15 + (int64_t)total_unary + tb;
  }
}

// Payload bits per 50-symbol group; exclusive offsets within the group tile.
__global__ void __launch_bounds__(kGroupTile) k_pay_bits(SlabDev d, const int32_t *list) {
  __shared__ uint32_t scratch[8];
  const int gt = list ? list[blockIdx.x] : (int)blockIdx.x;
  const int b = d.gt_block[gt];
  const int g0 = d.gt_first[gt];
  const int nsel = d.n_sel[b];
  if (g0 >= nsel) {
    if (threadIdx.x == 0) d.gt_bits[gt] = 0;
    return;
  }
  const int s = d.s[b];
  const int64_t off = d.off[b];
  const int g = g0 + threadIdx.x;
  uint32_t bits = 0;
  if (g < nsel) {
    const int t = d.sel[off / 32 + g];
    const uint8_t *len = d.len + ((size_t)b * kMaxGroups + t) * kMaxAlpha;
    const int a = g * kGroupSize, e = min(a + kGroupSize, s);
    for (int i = a; i < e; i++) bits += len[d.rle2[off + i]];
  }
  uint32_t tot;
  uint32_t ex = block_excl_sum(bits, scratch, &tot);
  if (g < nsel) d.grp_bits[off / 32 + g] = ex;
  if (threadIdx.x == 0) d.gt_bits[gt] = tot;
}

// Per block: exclusive sum over its group tiles; payload bits.
__global__ void __launch_bounds__(256) k_pay_block(SlabDev d) {
  __shared__ uint32_t scratch[40];
  const int b = blockIdx.x;
  // the group tiles that hold groups (the others are not run)
  const int nsel = d.n_sel[b];
  const int t0 = d.gt_begin[b];
  const int nt = min(d.gt_begin[b + 1] - t0, (nsel + kGroupTile - 1) / kGroupTile);
  int64_t carry = 0;
  for (int base = 0; base < nt; base += 256) {
    int k = base + threadIdx.x;
    uint32_t v = k < nt ? d.gt_bits[t0 + k] : 0;
    uint32_t tot;
    uint32_t ex = block_excl_sum(v, scratch, &tot);
    if (k < nt) d.gt_bits[t0 + k] = (uint32_t)(carry + ex);
    carry += tot;
  }
  if (threadIdx.x == 0) d.pay_bits[b] = carry;
}

__global__ void k_block_starts(SlabDev d, int64_t slab_start) {
  if (threadIdx.x != 0) return;
  int64_t run = slab_start;
  for (int b = 0; b < d.nblocks; b++) {
    d.blk_start[b] = run;
    run += d.hdr_bits[b] + d.pay_bits[b];
  }
}

// Block header at its stream position (src/compression/compress.cu:290-353).
// Thread 0 writes the fixed fields; every thread writes the unary selector
// codes of its chunk at an offset from a block scan; threads t < nGroups
// write table t's delta-coded lengths.
__global__ void __launch_bounds__(kHdrThreads) k_write_header(SlabDev d, int64_t w0) {
  __shared__ int scratch[40];
  __shared__ int64_t tbits[kMaxGroups];
  const int b = blockIdx.x;
  const int ngrp = d.n_groups[b];
  const int nsel = d.n_sel[b];
  const int alpha = d.n_in_use[b] + 2;
  const uint32_t *pres = d.present + b * 8;
  const uint8_t *smtf = d.sel_mtf + d.off[b] / 32;
  const int ranges = used_ranges(pres);
  const int64_t fixed = 48 + 32 + 1 + 24 + 16 + 16 * ranges + 3 + 15;
  const int64_t base = d.blk_start[b] - w0 * 32;
  if (threadIdx.x == 0) {
    BitSink w;
    w.init(d.out, base);
    w.put(0x314159u, 24);
    w.put(0x265359u, 24);
    w.put(d.crc[b], 32);
    w.put(0, 1);
    w.put((uint32_t)d.orig_ptr[b], 24);
    uint32_t l1 = 0;
    for (int r = 0; r < 16; r++)
      if ((pres[r >> 1] >> ((r & 1) * 16)) & 0xffffu) l1 |= 1u << (15 - r);
    w.put(l1, 16);
    for (int r = 0; r < 16; r++) {
      uint32_t half = (pres[r >> 1] >> ((r & 1) * 16)) & 0xffffu;
      if (!half) continue;
      uint32_t l2 = 0;
      for (int q = 0; q < 16; q++)
        if ((half >> q) & 1u) l2 |= 1u << (15 - q);
      w.put(l2, 16);
    }
    w.put((uint32_t)ngrp, 3);
    w.put((uint32_t)nsel, 15);
    w.flush();
  }
  int a, e;
  sel_chunk(nsel, &a, &e);
  int mine = 0;
  for (int i = a; i < e; i++) mine += smtf[i] + 1;
  int total;
  const int off = block_excl_sum(mine, scratch, &total);
  if (e > a) {
    BitSink w;
    w.init(d.out, base + fixed + off);
    for (int i = a; i < e; i++) {
      const int j = smtf[i];
      w.put(((1u << j) - 1u) << 1, j + 1);
    }
    w.flush();
  }
  if ((int)threadIdx.x < ngrp)
    tbits[threadIdx.x] =
        table_bits(d.len + ((size_t)b * kMaxGroups + threadIdx.x) * kMaxAlpha, alpha);
  __syncthreads();
  if ((int)threadIdx.x < ngrp) {
    const int t = threadIdx.x;
    int64_t at = base + fixed + total;
    for (int u = 0; u < t; u++) at += tbits[u];
    const uint8_t *len = d.len + ((size_t)b * kMaxGroups + t) * kMaxAlpha;
    BitSink w;
    w.init(d.out, at);
    int cur = len[0];
    w.put((uint32_t)cur, 5);
    for (int v = 0; v < alpha; v++) {
      const int tg = len[v];
      while (cur < tg) {
        w.put(2, 2);
        cur++;
      }
      while (cur > tg) {
        w.put(3, 2);
        cur--;
      }
      w.put(0, 1);
    }
    w.flush();
  }
}

// Payload: one thread per 50-symbol group.
__global__ void __launch_bounds__(kGroupTile) k_write_payload(SlabDev d, int64_t w0, const int32_t *list) {
  const int gt = list ? list[blockIdx.x] : (int)blockIdx.x;
  const int b = d.gt_block[gt];
  const int g0 = d.gt_first[gt];
  const int nsel = d.n_sel[b];
  const int g = g0 + threadIdx.x;
  if (g >= nsel) return;
  const int s = d.s[b];
  const int64_t off = d.off[b];
  const int t = d.sel[off / 32 + g];
  const uint8_t *len = d.len + ((size_t)b * kMaxGroups + t) * kMaxAlpha;
  const int32_t *code = d.code + ((size_t)b * kMaxGroups + t) * kMaxAlpha;
  int64_t bit = d.blk_start[b] + d.hdr_bits[b] + d.gt_bits[gt] + d.grp_bits[off / 32 + g];
  BitSink w;
  w.init(d.out, bit - w0 * 32);
  const int a = g * kGroupSize, e = min(a + kGroupSize, s);
  for (int i = a; i < e; i++) {
    int v = d.rle2[off + i];
    w.put((uint32_t)code[v], len[v]);
  }
  w.flush();
}

// Payload only, in the reference's word layout (word w = stream bits
// [32w, 32w+32), first bit in the MSB, host byte order), for one block.
__global__ void __launch_bounds__(kGroupTile) k_pack_words(SlabDev d, uint32_t *words, const int32_t *list) {
  const int gt = list ? list[blockIdx.x] : (int)blockIdx.x;
  const int b = d.gt_block[gt];
  const int g0 = d.gt_first[gt];
  const int nsel = d.n_sel[b];
  const int g = g0 + threadIdx.x;
  if (g >= nsel) return;
  const int s = d.s[b];
  const int64_t off = d.off[b];
  const int t = d.sel[off / 32 + g];
  const uint8_t *len = d.len + ((size_t)b * kMaxGroups + t) * kMaxAlpha;
  const int32_t *code = d.code + ((size_t)b * kMaxGroups + t) * kMaxAlpha;
  int64_t bit = (int64_t)d.gt_bits[gt] + d.grp_bits[off / 32 + g];
  int64_t word = bit >> 5;
  int n = (int)(bit & 31);
  uint64_t acc = 0;
  const int a = g * kGroupSize, e = min(a + kGroupSize, s);
  for (int i = a; i < e; i++) {
    int v = d.rle2[off + i];
    int nb = len[v];
    acc = (acc << nb) | (uint32_t)code[v];
    n += nb;
    if (n >= 32) {
      atomicOr(words + word, (uint32_t)(acc >> (n - 32)));
      word++;
      n -= 32;
    }
  }
  if (n > 0) atomicOr(words + word, (uint32_t)(acc << (32 - n)));
}

}  // namespace

// A group-tile kernel over the tiles that hold groups (every tile when the
// slab has no list).
template <typename F>
void launch_groups(const SlabDev &d, cudaStream_t st, F &&launch) {
  const int nlive = live_group_tiles(d, st);
  const int grid = nlive >= 0 ? nlive : d.n_group_tiles;
  if (grid <= 0) return;
  launch(grid, nlive >= 0 ? d.vg_list : nullptr);
}

void stage_sizes(const SlabDev &d, cudaStream_t st) {
  k_sel_mtf_hdr<<<d.nblocks, kHdrThreads, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
  launch_groups(d, st, [&](int grid, const int32_t *list) {
    k_pay_bits<<<grid, kGroupTile, 0, st>>>(d, list);
  });
  BZ_LAUNCH_CHECK();
  k_pay_block<<<d.nblocks, 256, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
}

void stage_sizes_payload_only(const SlabDev &d, cudaStream_t st) {
  launch_groups(d, st, [&](int grid, const int32_t *list) {
    k_pay_bits<<<grid, kGroupTile, 0, st>>>(d, list);
  });
  BZ_LAUNCH_CHECK();
  k_pay_block<<<d.nblocks, 256, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
}

void stage_place(const SlabDev &d, int64_t slab_start_bit, int64_t w0, int64_t nwords,
                 cudaStream_t st) {
  BZ_CUDA(cudaMemsetAsync(d.out, 0, sizeof(uint32_t) * nwords, st));
  k_block_starts<<<1, 32, 0, st>>>(d, slab_start_bit);
  BZ_LAUNCH_CHECK();
  k_write_header<<<d.nblocks, kHdrThreads, 0, st>>>(d, w0);
  BZ_LAUNCH_CHECK();
  launch_groups(d, st, [&](int grid, const int32_t *list) {
    k_write_payload<<<grid, kGroupTile, 0, st>>>(d, w0, list);
  });
  BZ_LAUNCH_CHECK();
}

// Blocks at word-aligned places of their own in `arena` (d.blk_start already
// holds each block's first bit); zeroes arena words [w0, w0 + nwords) first.
void stage_place_arena(const SlabDev &d, uint32_t *arena, int64_t w0, int64_t nwords,
                       cudaStream_t st) {
  BZ_CUDA(cudaMemsetAsync(arena + w0, 0, sizeof(uint32_t) * nwords, st));
  SlabDev a = d;
  a.out = arena;
  k_write_header<<<a.nblocks, kHdrThreads, 0, st>>>(a, 0);
  BZ_LAUNCH_CHECK();
  launch_groups(a, st, [&](int grid, const int32_t *list) {
    k_write_payload<<<grid, kGroupTile, 0, st>>>(a, 0, list);
  });
  BZ_LAUNCH_CHECK();
}

// Copy each block's bits (word-aligned in the arena) to its bit position in
// the output streams; the output is zeroed, and the first and last word of a
// block are OR-ed in because neighbours share them.
__global__ void __launch_bounds__(256) k_splice(const int64_t *src_addr, const int64_t *dst_bit,
                                                const int64_t *nbits, uint32_t *out) {
  const int b = blockIdx.x;
  const int64_t L = nbits[b];
  if (L <= 0) return;
  const int64_t D = dst_bit[b];
  const uint32_t *src = reinterpret_cast<const uint32_t *>(src_addr[b]);
  const int64_t srcw = (L + 31) >> 5;
  const int64_t w_first = D >> 5, w_last = (D + L - 1) >> 5;
  for (int64_t w = w_first + threadIdx.x; w <= w_last; w += blockDim.x) {
    const int64_t s = w * 32 - D;  // source bit of this word's first bit
    const int64_t a = s >= 0 ? s >> 5 : -1;
    const int sh = (int)(s - a * 32);
    const uint32_t x0 = (a >= 0 && a < srcw) ? bswap32(src[a]) : 0u;
    const uint32_t x1 = (a + 1 >= 0 && a + 1 < srcw) ? bswap32(src[a + 1]) : 0u;
    const uint32_t v = sh == 0 ? x0 : ((x0 << sh) | (x1 >> (32 - sh)));
    if (w == w_first || w == w_last) {
      if (v) atomicOr(out + w, bswap32(v));
    } else {
      out[w] = bswap32(v);
    }
  }
}

void launch_splice(const int64_t *src_addr, const int64_t *dst_bit, const int64_t *nbits,
                   int nblocks, uint32_t *out, cudaStream_t st) {
  if (nblocks <= 0) return;
  k_splice<<<nblocks, 256, 0, st>>>(src_addr, dst_bit, nbits, out);
  BZ_LAUNCH_CHECK();
}

void launch_pack_words(const SlabDev &d, uint32_t *words, cudaStream_t st) {
  launch_groups(d, st, [&](int grid, const int32_t *list) {
    k_pack_words<<<grid, kGroupTile, 0, st>>>(d, words, list);
  });
  BZ_LAUNCH_CHECK();
}

}  // namespace bz2g
