// MTF over the BWT last column, for every block of a slab.
//
// Reference: src/compression/fmtf.cu:40-230.  L[j] = T[(SA[j]-1) mod m]; the
// list starts as the ascending in-use symbols of T; origPtr is the j with
// SA[j] == 0.  The reference stitches per-chunk partial lists with a scan.
// Here the list state at the start of a tile follows from one fact: the list
// is the in-use symbols ordered by their last occurrence before that point
// (most recent first), symbols not seen yet in ascending order.  So each tile
// records the last position of every symbol, a per-block prefix-max over
// tiles gives each tile's starting list, and inside a tile the same fact,
// applied lane by lane, gives each lane its own starting list.
#include "engine.h"

namespace bz2g {

namespace {

// list: the tiles to run (blockIdx.x-th entry), or nullptr for every tile.
__global__ void __launch_bounds__(256) k_mtf_last(SlabDev d, const int32_t *list) {
  __shared__ int lastpos[256];
  const int t = list ? list[blockIdx.x] : (int)blockIdx.x;
  const int b = d.tile_block[t];
  const int64_t off = d.off[b];
  const int lt = (int)((int64_t)t * kTile - off);
  const int m = d.m[b];
  const int valid = min(kTile, m - lt);
  if (valid <= 0) return;
  lastpos[threadIdx.x] = -1;
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
  }
  __syncthreads();
  // thread k stands for symbol k: the symbols present in the tile are those
  // with a last position, one ballot per 32 symbols
  const int lp = lastpos[threadIdx.x];
  d.tile_last[(size_t)t * 256 + threadIdx.x] = lp;
  const unsigned pb = __ballot_sync(0xffffffffu, lp >= 0);
  if (lane_id() == 0 && pb) atomicOr(&d.present[b * 8 + warp_id()], pb);
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

// One warp per tile.  The tile's starting list comes from the
// last-occurrence table.  Lane k owns the 128 symbols [128k, 128k+128): it
// records their distinct values most recent first (its "partial list"); the
// warp then derives each lane's starting list in turn (list k = partial k-1
// followed by list k-1 without those symbols), and every lane runs the
// sequential move-to-front over its own symbols with its own list.
constexpr int kSub = kTile / 32;      // symbols per lane
constexpr int kListStride = 264;      // bytes per lane list (8-aligned, bank spread)
// The tile in shared memory: lane l's kSub bytes at l * (kSub + 4), so the 32
// lanes walking their own slices hit 32 different banks.
constexpr int kSLaneStride = kSub + 4;
__device__ __forceinline__ int sl_at(int i) { return i + (i / kSub) * 4; }

__global__ void __launch_bounds__(32) k_mtf_apply(SlabDev d, const int32_t *list) {
  // Lane k's list at lists[k]; lane k - 1 writes its partial list straight to
  // the front of list k, where the chain below wants it (13.5 KB of shared
  // memory in all: 15 single-warp blocks per SM).
  __shared__ __align__(16) uint8_t sL[32 * kSLaneStride];
  __shared__ __align__(16) uint8_t lists[32 * kListStride];
  __shared__ uint32_t pmask[32][9];  // padded row: no bank conflicts across lanes
  const int t = list ? list[blockIdx.x] : (int)blockIdx.x;
  const int b = d.tile_block[t];
  const int64_t off = d.off[b];
  const int lt = (int)((int64_t)t * kTile - off);
  const int m = d.m[b];
  const int valid = min(kTile, m - lt);
  if (valid <= 0) return;
  const int ln = lane_id();
  uint32_t pw[8];
  int nuse = 0;
#pragma unroll
  for (int w = 0; w < 8; w++) {
    pw[w] = d.present[b * 8 + w];
    nuse += __popc(pw[w]);
  }
  const uint4 *src = reinterpret_cast<const uint4 *>(d.last + off + lt);
  for (int w = ln; w < (valid + 15) / 16; w += 32) {
    const uint4 v = src[w];
    uint32_t *d4 = reinterpret_cast<uint32_t *>(sL + sl_at(16 * w));
    d4[0] = v.x;
    d4[1] = v.y;
    d4[2] = v.z;
    d4[3] = v.w;
  }
#pragma unroll
  for (int w = 0; w < 8; w++) pmask[ln][w] = 0;
  {
    // Lane 0's list: the in-use symbols by key, largest first, where a
    // symbol's key is its last position before this tile, or -1 - c for a
    // symbol not seen yet.  A bitonic sort of the 256 keys across the warp
    // (symbol 8k+q in register q of lane k; partners 8 or more apart sit in
    // other lanes and come by shuffle), each key packed with its symbol as
    // (key + 257) << 8 | symbol, 0 for symbols not in use.  Keys are distinct
    // and above -258, so the packing keeps their order.
    uint32_t v[8];
    {
      const int4 *k4 = reinterpret_cast<const int4 *>(d.tile_last + (size_t)t * 256) + 2 * ln;
      const int4 lo = k4[0], hi = k4[1];
      const int lp[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
      const uint32_t use = (pw[ln >> 2] >> (8 * (ln & 3))) & 0xffu;  // symbols 8 ln .. 8 ln + 7
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int c = 8 * ln + q;
        const int key = lp[q] >= 0 ? lp[q] : -1 - c;
        v[q] = ((use >> q) & 1u) ? ((uint32_t)(key + 257) << 8) | (uint32_t)c : 0u;
      }
    }
#pragma unroll
    for (int k = 2; k <= 256; k <<= 1) {
#pragma unroll
      for (int j = k >> 1; j > 0; j >>= 1) {
        if (j >= 8) {
          const int lj = j >> 3;
          const bool lower = (ln & lj) == 0;
#pragma unroll
          for (int q = 0; q < 8; q++) {
            const uint32_t o = __shfl_xor_sync(0xffffffffu, v[q], lj);
            const bool asc = ((8 * ln + q) & k) != 0;  // descending overall
            const bool keep_max = lower != asc;
            v[q] = keep_max ? max(v[q], o) : min(v[q], o);
          }
        } else {
#pragma unroll
          for (int q = 0; q < 8; q++) {
            if (q & j) continue;
            const int p = q | j;
            const bool asc = ((8 * ln + q) & k) != 0;
            const uint32_t a = v[q], b = v[p];
            const uint32_t mn = min(a, b), mx = max(a, b);
            v[q] = asc ? mn : mx;
            v[p] = asc ? mx : mn;
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 8; q++)
      if (8 * ln + q < nuse) lists[8 * ln + q] = (uint8_t)(v[q] & 0xffu);
  }
  // partial lists
  const int a0 = ln * kSub;
  const int a1 = min(valid, a0 + kSub);
  uint8_t *mySL = sL + 4 * ln;  // this lane's slice: mySL[i] for i in [a0, a1)
  __syncwarp();  // sL and pmask are in place
  int cnt = 0;  // this lane's partial-list length
  if (ln < 31) {  // lane 31's partial list starts no list
    uint8_t *pp = lists + (ln + 1) * kListStride;
    for (int i = a1 - 1; i >= a0; i--) {
      const int c = mySL[i];
      const uint32_t bit = 1u << (c & 31);
      const uint32_t mw = pmask[ln][c >> 5];
      if (!(mw & bit)) {
        pmask[ln][c >> 5] = mw | bit;
        pp[cnt++] = (uint8_t)c;
      }
    }
  }
  __syncwarp();
  // lane lists, in turn: list k = partial(k-1) ++ (list k-1 minus
  // partial(k-1)); partial(k-1) is already at the front of list k
  for (int k = 1; k < 32; k++) {
    const uint8_t *prevl = lists + (k - 1) * kListStride;
    uint8_t *cur = lists + k * kListStride;
    const int pc = __shfl_sync(0xffffffffu, cnt, k - 1);
    uint8_t keepv[8];
    int nk = 0;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int j = ln * 8 + q;
      uint8_t c = 0;
      bool keep = false;
      if (j < nuse) {
        c = prevl[j];
        keep = !((pmask[k - 1][c >> 5] >> (c & 31)) & 1u);
      }
      keepv[q] = c;
      nk += keep;
    }
    int inc = warp_incl_sum(nk);
    int o = pc + inc - nk;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int j = ln * 8 + q;
      if (j < nuse) {
        const uint8_t c = keepv[q];
        if (!((pmask[k - 1][c >> 5] >> (c & 31)) & 1u)) cur[o++] = c;
      }
    }
    __syncwarp();
  }
  // each lane: sequential move-to-front over its symbols, in place in sL.
  // The list is handled eight entries at a time: entry 8i+q is byte q of
  // little-endian word i.  A word without the symbol shifts up one byte (its
  // top byte carries into the next word); in the word holding it, the bytes
  // below it shift up and it leaves.
  {
    uint64_t *lw = reinterpret_cast<uint64_t *>(lists + ln * kListStride);
    const uint64_t ones = 0x0101010101010101ull, highs = 0x8080808080808080ull;
    for (int i = a0; i < a1; i++) {
      const uint32_t c = mySL[i];
      const uint64_t bc = ones * c;
      uint64_t carry = c;
      int q = 0;
      for (int wi = 0; wi < 32; wi++) {
        const uint64_t wv = lw[wi];
        const uint64_t x = wv ^ bc;
        const uint64_t z = (x - ones) & ~x & highs;  // lowest set bit marks the first match
        if (z) {
          const int j = (__ffsll((long long)z) - 1) >> 3;
          const uint64_t low = j == 7 ? ~0ull : ((1ull << (8 * (j + 1))) - 1);
          lw[wi] = (wv & ~low) | (((wv << 8) | carry) & low);
          q = wi * 8 + j;
          break;
        }
        lw[wi] = (wv << 8) | carry;
        carry = wv >> 56;
      }
      mySL[i] = (uint8_t)q;
    }
  }
  __syncwarp();
  uint4 *dst = reinterpret_cast<uint4 *>(d.mtf + off + lt);
  const int full = valid / 16;
  for (int w = ln; w < full; w += 32) {
    const uint32_t *s4 = reinterpret_cast<const uint32_t *>(sL + sl_at(16 * w));
    dst[w] = make_uint4(s4[0], s4[1], s4[2], s4[3]);
  }
  for (int i = full * 16 + ln; i < valid; i += 32) d.mtf[off + lt + i] = sL[sl_at(i)];
}

}  // namespace

void stage_mtf(const SlabDev &d, cudaStream_t st) {
  BZ_CUDA(cudaMemsetAsync(d.present, 0, sizeof(uint32_t) * 8 * d.nblocks, st));
  const int nlive = live_tiles(d, st);
  const int grid = nlive >= 0 ? nlive : d.ntiles;
  const int32_t *list = nlive >= 0 ? d.vt_list : nullptr;
  if (grid > 0) {
    k_mtf_last<<<grid, 256, 0, st>>>(d, list);
    BZ_LAUNCH_CHECK();
  }
  k_mtf_block_scan<<<d.nblocks, 256, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
  if (grid > 0) {
    k_mtf_apply<<<grid, 32, 0, st>>>(d, list);
    BZ_LAUNCH_CHECK();
  }
}

}  // namespace bz2g
