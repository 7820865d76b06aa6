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

// One warp per tile; lane l owns the kSub symbols [kSub*l, kSub*l + kSub)
// of the tile (its chunk).  Move-to-front is computed from occurrences, not
// by moving list entries: the index of symbol c at position i is
//   - if c occurred earlier in the chunk, last at p: the number of distinct
//     symbols in (p, i), i.e. of chunk positions in (p, i) that are the last
//     occurrence so far of their symbol (a 128-bit mask L, in registers);
//   - otherwise: the distinct symbols seen in the chunk so far, plus the
//     symbols ahead of c in the lane's starting list not seen yet: r - s,
//     r = c's rank in that list, s = seen symbols of lower rank (a 256-bit
//     mask S of their ranks, in registers).
// So each step is a fixed handful of bit operations, whatever the depth of
// the symbol in the list.  Lane l's starting list, as a rank per symbol,
// follows from lane l-1's: symbols seen in chunk l-1 come first, most
// recent first (their recency rank from a backward scan of the chunk), then
// the others in their previous order.  The tile's starting list (lane 0)
// comes from the last-occurrence table.
constexpr int kSub = kTile / 32;      // symbols per lane
constexpr int kRow = 260;             // bytes per lane row of a per-symbol table (bank spread)
// The tile in shared memory: lane l's kSub bytes at l * (kSub + 4), so the 32
// lanes walking their own slices hit 32 different banks.
constexpr int kSLaneStride = kSub + 4;
__device__ __forceinline__ int sl_at(int i) { return i + (i / kSub) * 4; }

// Set bits of the 128-bit mask (w0..w3) at positions 0..p.
__device__ __forceinline__ int popc_upto128(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3,
                                            int p) {
  const int w = p >> 5;
  const uint32_t m = (2u << (p & 31)) - 1u;
  const uint32_t ww = w == 0 ? w0 : w == 1 ? w1 : w == 2 ? w2 : w3;
  return (w > 0 ? __popc(w0) : 0) + (w > 1 ? __popc(w1) : 0) + (w > 2 ? __popc(w2) : 0) +
         __popc(ww & m);
}

// Set bits of the 256-bit mask s[0..7] below position r.
__device__ __forceinline__ int popc_below256(const uint32_t (&s)[8], int r) {
  const int w = r >> 5;
  const uint32_t m = (1u << (r & 31)) - 1u;
  int n = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) n += k < w ? __popc(s[k]) : (k == w ? __popc(s[k] & m) : 0);
  return n;
}

__global__ void __launch_bounds__(32) k_mtf_apply(SlabDev d, const int32_t *list) {
  __shared__ __align__(16) uint8_t sL[32 * kSLaneStride];
  __shared__ __align__(16) uint8_t rk[32 * kRow];   // lane l's starting list: rank of each symbol
  __shared__ __align__(16) uint8_t tab[32 * kRow];  // per lane: recency ranks, then last positions
  __shared__ __align__(16) uint8_t mark[256];       // chain: ranks held by seen symbols
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
  const uint32_t use = (pw[ln >> 2] >> (8 * (ln & 3))) & 0xffu;  // symbols 8 ln .. 8 ln + 7
  const uint4 *src = reinterpret_cast<const uint4 *>(d.last + off + lt);
  for (int w = ln; w < (valid + 15) / 16; w += 32) {
    const uint4 v = src[w];
    uint32_t *d4 = reinterpret_cast<uint32_t *>(sL + sl_at(16 * w));
    d4[0] = v.x;
    d4[1] = v.y;
    d4[2] = v.z;
    d4[3] = v.w;
  }
  uint32_t *myTw = reinterpret_cast<uint32_t *>(tab + ln * kRow);
#pragma unroll 8
  for (int w = 0; w < 64; w++) myTw[w] = ~0u;
  reinterpret_cast<uint64_t *>(mark)[ln] = 0;
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
    // position j of the sorted order (register q of lane j / 8) is rank j
#pragma unroll
    for (int q = 0; q < 8; q++)
      if (8 * ln + q < nuse) rk[v[q] & 0xffu] = (uint8_t)(8 * ln + q);
  }
  const int a0 = ln * kSub;
  const int a1 = min(valid, a0 + kSub);
  uint8_t *mySL = sL + 4 * ln;  // this lane's slice: mySL[i] for i in [a0, a1)
  uint8_t *myT = tab + ln * kRow;
  __syncwarp();  // sL, lane 0's ranks and the cleared tables are in place
  // recency ranks in this lane's chunk (0 = the symbol occurring last) and
  // the chunk's distinct symbol count
  int dist = 0;
  for (int i = a1 - 1; i >= a0; i--) {
    const int c = mySL[i];
    if (myT[c] == 0xffu) myT[c] = (uint8_t)dist++;
  }
  __syncwarp();
  // starting lists, lane by lane: rank in list k of symbol c =
  //   its recency rank in chunk k-1 if seen there, else
  //   dist(k-1) + its rank r in list k-1 - (seen symbols of rank below r);
  // the seen ranks are marked in `mark` and counted by a warp scan (lane j
  // holds ranks 8j .. 8j+7)
  for (int k = 1; k < 32; k++) {
    const uint8_t *rp = rk + (k - 1) * kRow;
    const uint8_t *tp = tab + (k - 1) * kRow;
    uint8_t *rn = rk + k * kRow;
    const int dk = __shfl_sync(0xffffffffu, dist, k - 1);
    int rq[8], sq[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int c = 8 * ln + q;
      const bool in = (use >> q) & 1u;
      sq[q] = in ? tp[c] : 0xff;
      rq[q] = in ? rp[c] : 0;
      if (in) mark[rq[q]] = sq[q] != 0xff;
    }
    __syncwarp();
    const uint2 mw = reinterpret_cast<const uint2 *>(mark)[ln];
    const uint32_t bits = (mw.x & 1u) | ((mw.x >> 7) & 2u) | ((mw.x >> 14) & 4u) |
                          ((mw.x >> 21) & 8u) | ((mw.y & 1u) << 4) | ((mw.y >> 3) & 0x20u) |
                          ((mw.y >> 10) & 0x40u) | ((mw.y >> 17) & 0x80u);
    const int cnt = __popc(bits);
    const int excl = warp_incl_sum(cnt) - cnt;
    const uint32_t packed = ((uint32_t)excl << 8) | bits;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const uint32_t x = __shfl_sync(0xffffffffu, packed, rq[q] >> 3);
      const int below = (int)(x >> 8) + __popc(x & ((1u << (rq[q] & 7)) - 1u));
      if ((use >> q) & 1u)
        rn[8 * ln + q] = (uint8_t)(sq[q] != 0xff ? sq[q] : dk + rq[q] - below);
    }
    __syncwarp();
  }
  // each lane: the move-to-front indices of its chunk, in place in sL;
  // myT now holds each symbol's last position in the chunk so far
#pragma unroll 8
  for (int w = 0; w < 64; w++) myTw[w] = ~0u;
  __syncwarp();
  {
    const uint8_t *myR = rk + ln * kRow;
    uint32_t L0 = 0, L1 = 0, L2 = 0, L3 = 0;  // last occurrences so far, by chunk position
    uint32_t S[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // starting-list ranks of the symbols seen
    int dc = 0;                                // distinct symbols seen (set bits of L)
    const int n = a1 - a0;
#pragma unroll
    for (int wq = 0; wq < 4; wq++) {
      const int e = min(n, 32 * wq + 32);
      for (int li = 32 * wq; li < e; li++) {
        const int c = mySL[a0 + li];
        const int pp = myT[c];
        myT[c] = (uint8_t)li;
        int idx;
        if (pp != 0xff) {
          idx = dc - popc_upto128(L0, L1, L2, L3, pp);
          const uint32_t bit = 1u << (pp & 31);
          const int w = pp >> 5;
          L0 ^= w == 0 ? bit : 0u;
          L1 ^= w == 1 ? bit : 0u;
          L2 ^= w == 2 ? bit : 0u;
          L3 ^= w == 3 ? bit : 0u;
        } else {
          const int r = myR[c];
          idx = dc + r - popc_below256(S, r);
#pragma unroll
          for (int k = 0; k < 8; k++) S[k] |= (r >> 5) == k ? 1u << (r & 31) : 0u;
          dc++;
        }
        const uint32_t me = 1u << (li & 31);
        if (wq == 0) L0 |= me;
        if (wq == 1) L1 |= me;
        if (wq == 2) L2 |= me;
        if (wq == 3) L3 |= me;
        mySL[a0 + li] = (uint8_t)idx;
      }
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
