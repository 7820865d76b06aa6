// MTF over the BWT last column, for every block of a slab.
//
// Reference: src/compression/fmtf.cu:40-230.  L[j] = T[(SA[j]-1) mod m]; the
// list starts as the ascending in-use symbols of T; origPtr is the j with
// SA[j] == 0.  The reference stitches per-chunk partial lists with a scan.
// Here the list state at the start of a tile follows from one fact: the list
// is the in-use symbols ordered by their last occurrence before that point
// (most recent first), symbols not seen yet in ascending order.  So each tile
// records the last position of every symbol, a per-block prefix-max over
// tiles gives each tile's starting list, and one warp per tile then runs the
// sequential MTF with the 256-entry list spread over the lanes' registers.
#include "engine.h"

namespace bz2g {

namespace {

__global__ void __launch_bounds__(256) k_mtf_last(SlabDev d) {
  __shared__ int lastpos[256];
  __shared__ uint32_t pres[8];
  const int t = blockIdx.x;
  const int b = d.tile_block[t];
  const int64_t off = d.off[b];
  const int lt = (int)((int64_t)t * kTile - off);
  const int m = d.m[b];
  const int valid = min(kTile, m - lt);
  if (valid <= 0) return;
  lastpos[threadIdx.x] = -1;
  if (threadIdx.x < 8) pres[threadIdx.x] = 0;
  __syncthreads();
  const uint8_t *T = d.rle1 + off;
  const int32_t *SA = d.sa + off;
  uint8_t *L = d.last + off;
  for (int e = threadIdx.x; e < valid; e += blockDim.x) {
    int j = lt + e;
    int i = SA[j];
    if (i == 0) d.orig_ptr[b] = j;
    uint8_t c = T[i == 0 ? m - 1 : i - 1];
    L[j] = c;
    atomicMax(&lastpos[c], j);
    atomicOr(&pres[c >> 5], 1u << (c & 31));
  }
  __syncthreads();
  d.tile_last[(size_t)t * 256 + threadIdx.x] = lastpos[threadIdx.x];
  if (threadIdx.x < 8 && pres[threadIdx.x]) atomicOr(&d.present[b * 8 + threadIdx.x], pres[threadIdx.x]);
}

// Per block, per symbol: exclusive prefix max of last positions over tiles.
__global__ void __launch_bounds__(256) k_mtf_block_scan(SlabDev d) {
  const int b = blockIdx.x;
  const int m = d.m[b];
  if (m <= 0) return;
  const int nt = (m + kTile - 1) / kTile;
  const int t0 = (int)(d.off[b] / kTile);
  int carry = -1;
  for (int k = 0; k < nt; k++) {
    size_t idx = (size_t)(t0 + k) * 256 + threadIdx.x;
    int v = d.tile_last[idx];
    d.tile_last[idx] = carry;
    carry = max(carry, v);
  }
  if (threadIdx.x == 0) {
    int n = 0;
    for (int w = 0; w < 8; w++) n += __popc(d.present[b * 8 + w]);
    d.n_in_use[b] = n;
  }
}

// One warp per tile: starting list from the last-occurrence table, then the
// sequential move-to-front.  Lane l holds list entries 8l .. 8l+7.
__global__ void __launch_bounds__(32) k_mtf_apply(SlabDev d) {
  __shared__ int key[256];
  __shared__ int list[256];
  __shared__ uint8_t sL[kTile];
  __shared__ uint8_t sO[kTile];
  const int t = blockIdx.x;
  const int b = d.tile_block[t];
  const int64_t off = d.off[b];
  const int lt = (int)((int64_t)t * kTile - off);
  const int m = d.m[b];
  const int valid = min(kTile, m - lt);
  if (valid <= 0) return;
  const int ln = lane_id();
  uint32_t pw[8];
#pragma unroll
  for (int w = 0; w < 8; w++) pw[w] = d.present[b * 8 + w];
  // key: last position before this tile, or (-1 - c) for unseen symbols
  for (int c = ln; c < 256; c += 32) {
    int lp = d.tile_last[(size_t)t * 256 + c];
    bool use = (pw[c >> 5] >> (c & 31)) & 1u;
    key[c] = !use ? INT32_MIN : (lp >= 0 ? lp : -1 - c);
    list[c] = -1;
  }
  const uint4 *src = reinterpret_cast<const uint4 *>(d.last + off + lt);
  for (int w = ln; w < (valid + 15) / 16; w += 32) reinterpret_cast<uint4 *>(sL)[w] = src[w];
  __syncwarp();
  for (int c = ln; c < 256; c += 32) {
    int kc = key[c];
    if (kc == INT32_MIN) continue;
    int r = 0;
    for (int c2 = 0; c2 < 256; c2++) r += key[c2] > kc;
    list[r] = c;
  }
  __syncwarp();
  int e0 = list[ln * 8 + 0], e1 = list[ln * 8 + 1], e2 = list[ln * 8 + 2], e3 = list[ln * 8 + 3];
  int e4 = list[ln * 8 + 4], e5 = list[ln * 8 + 5], e6 = list[ln * 8 + 6], e7 = list[ln * 8 + 7];
  for (int e = 0; e < valid; e++) {
    const int c = sL[e];
    int slot = e0 == c ? 0 : e1 == c ? 1 : e2 == c ? 2 : e3 == c ? 3
             : e4 == c ? 4 : e5 == c ? 5 : e6 == c ? 6 : e7 == c ? 7 : -1;
    unsigned bal = __ballot_sync(0xffffffffu, slot >= 0);
    int owner = __ffs(bal) - 1;
    int os = __shfl_sync(0xffffffffu, slot, owner);
    if (ln == 0) sO[e] = (uint8_t)(owner * 8 + os);
    int carry = __shfl_up_sync(0xffffffffu, e7, 1);
    if (ln == 0) carry = c;
    if ((int)ln < owner) {
      e7 = e6; e6 = e5; e5 = e4; e4 = e3; e3 = e2; e2 = e1; e1 = e0; e0 = carry;
    } else if ((int)ln == owner) {
      if (os >= 7) e7 = e6;
      if (os >= 6) e6 = e5;
      if (os >= 5) e5 = e4;
      if (os >= 4) e4 = e3;
      if (os >= 3) e3 = e2;
      if (os >= 2) e2 = e1;
      if (os >= 1) e1 = e0;
      e0 = carry;
    }
  }
  __syncwarp();
  uint8_t *dst = d.mtf + off + lt;
  for (int e = ln; e < valid; e += 32) dst[e] = sO[e];
}

}  // namespace

void stage_mtf(const SlabDev &d, cudaStream_t st) {
  BZ_CUDA(cudaMemsetAsync(d.present, 0, sizeof(uint32_t) * 8 * d.nblocks, st));
  k_mtf_last<<<d.ntiles, 256, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
  k_mtf_block_scan<<<d.nblocks, 256, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
  k_mtf_apply<<<d.ntiles, 32, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
}

}  // namespace bz2g
