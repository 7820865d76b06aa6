// BWT of every block of a slab: sorted cyclic rotations by prefix doubling.
//
// Reference: src/compression/fbwt.cu:47-106 (prefix doubling with a stable
// 64-bit key sort each round; ties, i.e. equal rotations, keep index order).
//
// Here:
//   1. One segmented LSD radix sort (segments = blocks) of every rotation by
//      its first P bytes (cyclic, big-endian), stable from index order, so
//      ties are index-ascending.
//   2. Ranks are group heads: head = first SA position of the group;
//      ISA[i] = head of rotation i.  Rotations in groups of size 1 are final.
//   3. The rotations still in groups of size >= 2 ("active") are compacted,
//      per block, with their SA position.  Round with shift h (prefix length
//      h -> 2h) keys them (head << kb) | ISA[(i + h) mod m] and re-sorts them
//      stably; the k-th of them in sorted order goes to the k-th active SA
//      position (groups are contiguous, so this sorts within each group).
//   4. A block stops when no rotation is active, when a round splits no group
//      (the rest are equal rotations, already index-ascending), or when the
//      prefix length reaches m.
// Block-local ranks fit kb = ceil(log2(max m + 1)) bits.  When 3*kb <= 64
// (m < 2^21, every bzip2 block) key and rotation share one 64-bit item and
// the sort moves items only: the first sort keys the first P = 4 bytes
// (item = prefix << 32 | i), rounds use item = head << 2kb | rank << kb | i.
// Larger m keeps separate 64-bit keys and 32-bit rotations, with P = 8.
#include <algorithm>
#include <cstring>

#include "engine.h"

namespace bz2g {

namespace {

constexpr int kSortWarps = kTileThreads / 32;  // 8
constexpr int kWarpSpan = kTile / kSortWarps;   // elements per warp in a tile (512)
// Digits of the doubling rounds' sorts may be 9 bits wide (fewer passes over
// the 2kb key bits); the tile and block digit tables (tile_hist, sort_base)
// are sized for kMaxRadix digits.  Shared memory of the scatter: the tile's
// keys (and values), per-warp digit counts, two digit tables.
template <int RB>
constexpr size_t scatter_smem_keys() {
  return (size_t)kTile * 8 + (size_t)kSortWarps * (1 << RB) * 4 + 2 * (1 << RB) * 4;
}
template <int RB>
constexpr size_t scatter_smem_vals() {
  return scatter_smem_keys<RB>() + (size_t)kTile * 4;
}

// How a sorted element is stored: packed (one item: key << low | rotation)
// or as separate keys[] and vals[].
struct Layout {
  int packed;
  int low;
};

__device__ __forceinline__ uint64_t key_of(const Layout L, uint64_t item) {
  return L.packed ? item >> L.low : item;
}

// Tile of this CTA: blockIdx.x, or the blockIdx.x-th entry of a list of the
// tiles that hold work (doubling rounds).
__device__ __forceinline__ int tile_id(const int32_t *list) {
  return list ? list[blockIdx.x] : (int)blockIdx.x;
}

__device__ __forceinline__ int tile_valid(const SlabDev &d, int t, const int32_t *lens, int *b_out,
                                          int *lt_out) {
  int b = d.tile_block[t];
  int lt = (int)((int64_t)t * kTile - d.off[b]);
  *b_out = b;
  *lt_out = lt;
  int v = lens[b] - lt;
  return v < 0 ? 0 : (v > kTile ? kTile : v);
}

// The valid lanes of the warp whose RB-bit digit equals this lane's: one
// ballot per digit bit (cheaper here than __match_any_sync).
template <int RB>
__device__ __forceinline__ unsigned digit_peers(int dg, bool ok) {
  unsigned peers = __ballot_sync(0xffffffffu, ok);
#pragma unroll
  for (int bit = 0; bit < RB; bit++) {
    const bool on = (dg >> bit) & 1;
    const unsigned bb = __ballot_sync(0xffffffffu, on);
    peers &= on ? bb : ~bb;
  }
  return peers;
}

// The first sort of the packed layout starts from index order, so its first
// pass builds each tile's items itself from the block's text (read in order:
// the item at element e of a tile is rotation lt + e) instead of reading
// them: item = (first 4 bytes of the rotation, big-endian) << 32 | rotation.
__device__ __forceinline__ uint64_t text_item(const uint8_t *T, int m, int i) {
  uint32_t k = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    int j = i + q;
    while (j >= m) j -= m;
    k = (k << 8) | T[j];
  }
  return ((uint64_t)k << 32) | (uint32_t)i;
}

template <int RB>
__device__ __forceinline__ void block_digit_scan(const SlabDev &d, int b, int force,
                                                 uint32_t *scratch);

// gen != 0: the generating first pass (items from the text, see text_item;
// 8-bit digits).  RB: digit width, tile_hist holds 2^RB counts per tile.
// The last tile of a block to finish its counts (a per-block counter, after
// a fence that publishes the counts) runs the block's scan over its tiles'
// counts, so the pass needs no scan launch of its own.
template <int RB>
__global__ void __launch_bounds__(256) k_radix_hist(SlabDev d, int shift, const int32_t *list,
                                                    int gen) {
  constexpr int kN = 1 << RB;
  __shared__ uint32_t cnt[kN];
  const int t = tile_id(list);
  int b, lt;
  int valid = tile_valid(d, t, d.sort_len, &b, &lt);
  if (valid == 0) return;
  for (int i = threadIdx.x; i < kN; i += blockDim.x) cnt[i] = 0;
  __syncthreads();
  const uint64_t *K = d.keys[d.sort_ctl[0]] + d.off[b] + lt;
  const uint8_t *T = d.rle1 + d.off[b];
  const int m = d.m[b];
  if (gen) {
    // digit bits [shift, shift + 8) of the item are byte 3 - (shift - 32) / 8
    // of the rotation's 4-byte prefix
    const int q = 3 - (shift - 32) / 8;
    for (int e = threadIdx.x; e < valid; e += blockDim.x) {
      int j = lt + e + q;
      while (j >= m) j -= m;
      atomicAdd(&cnt[T[j]], 1u);
    }
  } else {
    for (int e = threadIdx.x; e < valid; e += blockDim.x)
      atomicAdd(&cnt[(uint32_t)(K[e] >> shift) & (kN - 1)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kN; i += blockDim.x) d.tile_hist[(size_t)t * kN + i] = cnt[i];
  __threadfence();
  __syncthreads();
  __shared__ int s_last;
  __shared__ uint32_t scratch[40];
  if (threadIdx.x == 0) {
    const int nt = (d.sort_len[b] + kTile - 1) / kTile;
    s_last = atomicAdd(&d.blk_count[b], 1) == nt - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  block_digit_scan<RB>(d, b, gen, scratch);
  if (threadIdx.x == 0) d.blk_count[b] = 0;
}

// Per block: turn tile digit counts into each tile's count of the digit in
// the block's earlier tiles (one pass), and the digit's base in the block.
// force != 0 (the generating pass): the pass runs even if every tile holds one
// digit only, since it writes the items the later passes read.
// Thread i handles the kD = 2^RB / 256 consecutive digits kD*i .. kD*i+kD-1.
template <int RB>
__device__ __forceinline__ void block_digit_scan(const SlabDev &d, int b, int force,
                                                 uint32_t *scratch) {
  constexpr int kN = 1 << RB, kD = kN / 256;
  const int len = d.sort_len[b];
  const int nt = (len + kTile - 1) / kTile;
  const int t0 = (int)(d.off[b] / kTile);
  uint32_t *H = d.tile_hist + (size_t)t0 * kN + kD * threadIdx.x;
  // eight tiles' counts in flight at a time (the loads are independent)
  constexpr int kU = 8;
  uint32_t run[kD];
#pragma unroll
  for (int q = 0; q < kD; q++) run[q] = 0;
  for (int k0 = 0; k0 < nt; k0 += kU) {
#pragma unroll
    for (int q = 0; q < kD; q++) {
      uint32_t h[kU];
#pragma unroll
      for (int j = 0; j < kU; j++) h[j] = k0 + j < nt ? __ldcg(&H[(size_t)(k0 + j) * kN + q]) : 0u;
#pragma unroll
      for (int j = 0; j < kU; j++) {
        if (k0 + j < nt) H[(size_t)(k0 + j) * kN + q] = run[q];
        run[q] += h[j];
      }
    }
  }
  // the digit's base in the block (exclusive sum over digits of the block's
  // counts), added by the scatter to each tile's count before it
  uint32_t sum = 0;
  bool one = false;
#pragma unroll
  for (int q = 0; q < kD; q++) {
    sum += run[q];
    one |= run[q] == (uint32_t)len;
  }
  uint32_t tot;
  uint32_t base = block_excl_sum(sum, scratch, &tot);
  int trivial = __syncthreads_or(one);
  if ((!trivial || force) && threadIdx.x == 0) atomicOr(&d.sort_ctl[1], 1);
#pragma unroll
  for (int q = 0; q < kD; q++) {
    d.sort_base[(size_t)b * kN + kD * threadIdx.x + q] = (uint32_t)d.off[b] + base;
    base += run[q];
  }
}

// Stable scatter of one tile by one 8-bit digit.  Elements are warp-striped
// (lane l, item i <-> element w*512 + i*32 + l) so that ranking item by item
// over the lanes with equal digits keeps the original order; the tile is sorted locally
// in shared memory, then written so that equal digits go out contiguously.
// All of a thread's loads are issued before the ranking starts.
template <bool kVals, int RB>
__global__ void __launch_bounds__(256, kVals ? 2 : 3)
    k_radix_scatter(SlabDev d, int shift, int timed, const int32_t *list, int gen) {
  constexpr int kN = 1 << RB, kD = kN / 256;
  if (!d.sort_ctl[1]) return;
  const int t = tile_id(list);
  int b, lt;
  const int valid = tile_valid(d, t, d.sort_len, &b, &lt);
  if (valid == 0) return;
  if (timed >= 0 && threadIdx.x == 0)
    atomicAdd((unsigned long long *)&d.kt_elems[timed], (unsigned long long)valid);
  extern __shared__ __align__(16) uint8_t smem[];
  uint64_t *sk = reinterpret_cast<uint64_t *>(smem);
  uint32_t *sv = reinterpret_cast<uint32_t *>(sk + kTile);
  uint32_t *wcnt = kVals ? sv + kTile : reinterpret_cast<uint32_t *>(sk + kTile);  // [warp][digit]
  uint32_t *goff = wcnt + kSortWarps * kN + kN;  // global digit base for this tile
  const int cur = d.sort_ctl[0];
  const uint64_t *K = d.keys[cur] + d.off[b] + lt;
  const uint32_t *V = d.vals[cur] + d.off[b] + lt;
  const int w = warp_id(), ln = lane_id();

  uint64_t key[kTileItems];
  uint32_t val[kTileItems];
  if (!kVals && gen) {
    const uint8_t *T = d.rle1 + d.off[b];
    const int m = d.m[b];
#pragma unroll
    for (int i = 0; i < kTileItems; i++) {
      const int e = w * kWarpSpan + i * 32 + ln;
      key[i] = e < valid ? text_item(T, m, lt + e) : 0;
    }
  } else {
#pragma unroll
    for (int i = 0; i < kTileItems; i++) {
      const int e = w * kWarpSpan + i * 32 + ln;
      key[i] = e < valid ? K[e] : 0;
      if (kVals) val[i] = e < valid ? V[e] : 0;
    }
  }
#pragma unroll
  for (int q = 0; q < kSortWarps * kD; q++) wcnt[q * 256 + threadIdx.x] = 0;

  __syncthreads();

  uint32_t rank2[kTileItems / 2];  // two 16-bit ranks per register (ranks < 512)
  const unsigned lt_mask = (1u << ln) - 1u;
#pragma unroll
  for (int i = 0; i < kTileItems; i++) {
    const int e = w * kWarpSpan + i * 32 + ln;
    const bool ok = e < valid;
    const int dg = ok ? (int)((key[i] >> shift) & (kN - 1)) : 0;
    const unsigned peers = digit_peers<RB>(dg, ok);
    const uint32_t before = ok ? wcnt[w * kN + dg] : 0;
    const uint32_t r = before + __popc(peers & lt_mask);
    if (i & 1)
      rank2[i >> 1] |= r << 16;
    else
      rank2[i >> 1] = r;
    __syncwarp();
    if (ok && (peers & lt_mask) == 0) wcnt[w * kN + dg] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {
    // per digit: its local base (exclusive scan over digits of the tile's
    // counts); each warp's count becomes that warp's local start for the
    // digit, and the digit's global base becomes (global - local) base, so
    // the placement and the write below read one table entry each
    __shared__ uint32_t scratch[40];
    uint32_t tot;
    if constexpr (kD == 1) {
      const int dg = threadIdx.x;
      uint32_t run = 0;
      for (int ww = 0; ww < kSortWarps; ww++) run += wcnt[ww * kN + dg];
      const uint32_t lb = block_excl_sum(run, scratch, &tot);
      uint32_t at = lb;
      for (int ww = 0; ww < kSortWarps; ww++) {
        const uint32_t c = wcnt[ww * kN + dg];
        wcnt[ww * kN + dg] = at;
        at += c;
      }
      goff[dg] = d.tile_hist[(size_t)t * kN + dg] + d.sort_base[(size_t)b * kN + dg] - lb;
    } else {
      // thread i: the kD consecutive digits kD*i ..
      uint32_t run[kD], sum = 0;
#pragma unroll
      for (int q = 0; q < kD; q++) {
        const int dg = kD * threadIdx.x + q;
        run[q] = 0;
        for (int ww = 0; ww < kSortWarps; ww++) run[q] += wcnt[ww * kN + dg];
        sum += run[q];
      }
      uint32_t lb = block_excl_sum(sum, scratch, &tot);
#pragma unroll
      for (int q = 0; q < kD; q++) {
        const int dg = kD * threadIdx.x + q;
        uint32_t at = lb;
        for (int ww = 0; ww < kSortWarps; ww++) {
          const uint32_t c = wcnt[ww * kN + dg];
          wcnt[ww * kN + dg] = at;
          at += c;
        }
        goff[dg] = d.tile_hist[(size_t)t * kN + dg] + d.sort_base[(size_t)b * kN + dg] - lb;
        lb += run[q];
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kTileItems; i++) {
    const int e = w * kWarpSpan + i * 32 + ln;
    if (e < valid) {
      const int dg = (int)((key[i] >> shift) & (kN - 1));
      const uint32_t r = (i & 1) ? rank2[i >> 1] >> 16 : rank2[i >> 1] & 0xffffu;
      const uint32_t pos = wcnt[w * kN + dg] + r;
      sk[pos] = key[i];
      if (kVals) sv[pos] = val[i];
    }
  }
  __syncthreads();
  uint64_t *KO = d.keys[cur ^ 1];
  uint32_t *VO = d.vals[cur ^ 1];
  for (int k = threadIdx.x; k < valid; k += blockDim.x) {
    const uint64_t kk = sk[k];
    const int dg = (int)((kk >> shift) & (kN - 1));
    const uint32_t g = goff[dg] + (uint32_t)k;
    KO[g] = kk;
    if (kVals) VO[g] = sv[k];
  }
}

__global__ void k_radix_flip(SlabDev d) {
  if (d.sort_ctl[1]) d.sort_ctl[0] ^= 1;
  d.sort_ctl[1] = 0;
}

// Stable sort of each block's elements by key bits [lo, hi), over `grid`
// tiles (all tiles, or the listed ones).
// gen: the first pass generates the packed first-sort items from the text.
// RB: digit width (8; 9 for packed items of the doubling rounds where that
// takes fewer passes).
template <int RB>
void radix_passes(const SlabDev &d, int lo, int hi, int has_vals, cudaStream_t st, int grid,
                  const int32_t *list, bool gen) {
  BZ_REQUIRE(RB == 8 || (!has_vals && !gen), kErrInternal, "wide digits are for packed rounds");
  const size_t smem = has_vals ? scatter_smem_vals<RB>() : scatter_smem_keys<RB>();
  for (int shift = lo; shift < hi; shift += RB) {
    const int g = gen && shift == lo;
    k_radix_hist<RB><<<grid, 256, 0, st>>>(d, shift, list, g);
    BZ_LAUNCH_CHECK();
    int timed = -1;
    if (d.kt_on && *d.kt_n < kMaxTimedLaunches) {
      timed = (*d.kt_n)++;
      d.kt_bpe[timed] = has_vals ? 24 : g ? 9 : 16;  // the generating pass reads text bytes
      BZ_CUDA(cudaEventRecord(d.kt_ev[2 * timed], st));
    }
    if constexpr (RB == 8) {
      if (has_vals)
        k_radix_scatter<true, 8><<<grid, 256, smem, st>>>(d, shift, timed, list, 0);
      else
        k_radix_scatter<false, 8><<<grid, 256, smem, st>>>(d, shift, timed, list, g);
    } else {
      k_radix_scatter<false, RB><<<grid, 256, smem, st>>>(d, shift, timed, list, 0);
    }
    BZ_LAUNCH_CHECK();
    if (timed >= 0) BZ_CUDA(cudaEventRecord(d.kt_ev[2 * timed + 1], st));
    k_radix_flip<<<1, 1, 0, st>>>(d);
    BZ_LAUNCH_CHECK();
  }
}

void radix_sort(const SlabDev &d, int lo, int hi, int has_vals, cudaStream_t st, int grid,
                const int32_t *list, bool gen = false) {
  if (grid <= 0) return;
  // 9-bit digits where they take fewer passes than 8-bit ones (10-bit
  // digits also save a pass for 19- and 20-bit rank fields, but their
  // 4x digit tables made the deep rounds of long blocks slower)
  const int bits = hi - lo;
  if (!has_vals && !gen && (bits + 8) / 9 < (bits + 7) / 8)
    radix_passes<9>(d, lo, hi, has_vals, st, grid, list, gen);
  else
    radix_passes<8>(d, lo, hi, has_vals, st, grid, list, gen);
}

// ------------------------------------------------------------------- BWT
__global__ void k_bwt_init(SlabDev d) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b == 0)
    for (int k = 0; k < 10; k++) d.sort_ctl[k] = 0;
  if (b >= d.nblocks) return;
  int m = d.m[b];
  d.sort_len[b] = m > 1 ? m : 0;
  d.done[b] = m > 1 ? 0 : 1;
  d.ngroups[b] = -1;
  d.act_len[b] = 0;
  d.active_sum[b] = 0;
  d.blk_count[b] = 0;  // the histogram tile counter: each pass resets it, and so does this
  for (int k = 0; k < 8; k++) d.pstat[b * 8 + k] = 0;
  if (m == 1) d.sa[d.off[b]] = 0;
}

// The oracle's accounting of the rounds h = 1, 2, (4) that the first sort
// stands for (round h runs while the partition has a non-singleton group and
// the previous round split one), and the group count of the prefix before
// the first sort's as the fixed-point reference of the first ranking.
__global__ void k_bwt_prefix_account(SlabDev d, int nq) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nblocks) return;
  const int m = d.m[b];
  if (m <= 1) return;
  const int32_t *ps = d.pstat + b * 8;
  int64_t A = 0;
  bool stop = false;
  for (int q = 0; q < nq - 1 && !stop; q++) {
    const int G = ps[q], S = ps[4 + q];
    if (G == m) break;
    A += m - S;
    const int h = 1 << q;
    if (ps[q + 1] == G || 2 * h >= m) stop = true;
  }
  d.active_sum[b] = A;
  d.ngroups[b] = ps[nq - 2];
  if (A) atomicAdd(reinterpret_cast<unsigned long long *>(d.sort_ctl + 8), (unsigned long long)A);
}

// First keys: the first 4 (packed) or 8 bytes of each rotation.
__global__ void __launch_bounds__(256) k_bwt_keys0(SlabDev d, int packed) {
  __shared__ uint8_t sb[kTile + 8];
  int b, lt;
  int valid = tile_valid(d, blockIdx.x, d.sort_len, &b, &lt);
  if (valid == 0) return;
  const int m = d.m[b];
  const uint8_t *T = d.rle1 + d.off[b];
  for (int e = threadIdx.x; e < valid + 7; e += blockDim.x) {
    int i = lt + e;
    while (i >= m) i -= m;
    sb[e] = T[i];
  }
  __syncthreads();
  uint64_t *K = d.keys[0] + d.off[b] + lt;
  uint32_t *V = d.vals[0] + d.off[b] + lt;
  for (int e = threadIdx.x; e < valid; e += blockDim.x) {
    uint64_t k = 0;
    if (packed) {
#pragma unroll
      for (int q = 0; q < 4; q++) k = (k << 8) | sb[e + q];
      K[e] = (k << 32) | (uint32_t)(lt + e);
    } else {
#pragma unroll
      for (int q = 0; q < 8; q++) k = (k << 8) | sb[e + q];
      K[e] = k;
      V[e] = (uint32_t)(lt + e);
    }
  }
}

// ---------------------------------------------------------------- ranking
// After a sort, the sorted (key, rotation) pairs of a block sit at
// [off, off + len); element k belongs at SA position P[k] (k itself after the
// first sort; the k-th active position in later rounds).  A group starts
// where the key changes; its head is the SA position of its first element.
// Elements are read warp-striped (warp w owns [512w, 512w + 512), item i of
// lane l is element 512w + 32i + l) so every load is coalesced.
__device__ __forceinline__ uint64_t key_at(const uint64_t *K, int k) { return K[k]; }

// Per tile: last head (SA position), head count, singleton count, active
// (non-singleton) count.  After the first sort (nq > 0) it also counts, from
// the same reads, the group heads and singletons of the prefix-1, -2 (-4, -8)
// byte partitions (key_bits = 32 packed, 64 otherwise): pstat[b*8 + q] heads
// and pstat[b*8 + 4 + q] singletons of prefix 2^q bytes.
__global__ void __launch_bounds__(256) k_bwt_flags(SlabDev d, Layout L, int initial,
                                                   const int32_t *list, int key_bits, int nq) {
  __shared__ int red[4][kSortWarps];
  const int t = tile_id(list);
  int b, lt;
  const int valid = tile_valid(d, t, d.sort_len, &b, &lt);
  if (valid == 0) return;
  const int len = d.sort_len[b];
  const int64_t off = d.off[b];
  const uint64_t *K = d.keys[d.sort_ctl[0]] + off;
  const int32_t *P = d.kpos[d.sort_ctl[3]] + off;
  const int w = warp_id(), ln = lane_id();
  int last = -1, heads = 0, sing = 0;
  int pc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 4
  for (int i = 0; i < kTileItems; i++) {
    const int e = w * kWarpSpan + i * 32 + ln;
    if (e < valid) {
      const int k = lt + e;
      const uint64_t key = key_of(L, K[k]);
      const uint64_t kp = k > 0 ? key_of(L, K[k - 1]) : 0;
      const uint64_t kn = k + 1 < len ? key_of(L, K[k + 1]) : 0;
      const bool hd = k == 0 || key != kp;
      if (hd) {
        const bool tl = k + 1 == len || kn != key;
        last = max(last, initial ? k : P[k]);
        heads++;
        sing += tl;
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        if (q < nq) {
          const int sh = key_bits - 8 * (1 << q);
          const uint64_t a = sh > 0 ? key >> sh : key;
          const bool h2 = k == 0 || a != (sh > 0 ? kp >> sh : kp);
          const bool t2 = k + 1 == len || a != (sh > 0 ? kn >> sh : kn);
          pc[q] += h2;
          pc[4 + q] += h2 && t2;
        }
      }
    }
  }
  if (nq > 0) {
#pragma unroll
    for (int q = 0; q < 8; q++) {
      int v = pc[q];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (ln == 0 && v) atomicAdd(&d.pstat[b * 8 + q], v);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    last = max(last, __shfl_xor_sync(0xffffffffu, last, o));
    heads += __shfl_xor_sync(0xffffffffu, heads, o);
    sing += __shfl_xor_sync(0xffffffffu, sing, o);
  }
  if (ln == 0) {
    const int wvalid = min(max(valid - w * kWarpSpan, 0), kWarpSpan);
    d.warp_last[t * kSortWarps + w] = last;
    d.warp_act[t * kSortWarps + w] = wvalid - sing;  // elements in groups of size >= 2
    red[1][w] = heads;
    red[2][w] = sing;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int h = 0, sg = 0;
    for (int q = 0; q < kSortWarps; q++) {
      h += red[1][q];
      sg += red[2][q];
    }
    d.tile_b[t] = h;
    d.tile_c[t] = sg;
  }
}

// Per block: carry of the last head into each warp span (512 elements of a
// tile), compaction offsets of the active elements per warp span, and the
// stop test: no active element left, no group split by this round (the rest
// are equal rotations), or prefix >= m.
__global__ void __launch_bounds__(256) k_bwt_rank_block(SlabDev d, int64_t prefix_len) {
  __shared__ int scratch[40];
  __shared__ int sx[256];
  const int b = blockIdx.x;
  const int len = d.sort_len[b];
  if (len <= 0) return;
  const int nt = (len + kTile - 1) / kTile;
  const int t0 = (int)(d.off[b] / kTile);
  const int nw = nt * kSortWarps;
  int32_t *WL = d.warp_last + (int64_t)t0 * kSortWarps;
  int32_t *WA = d.warp_act + (int64_t)t0 * kSortWarps;
  int carry = -1, heads = 0, singles = 0, active = 0;
  for (int base = 0; base < nw; base += 256) {
    const int k = base + threadIdx.x;
    const int v = k < nw ? WL[k] : -1;
    const int ac = k < nw ? WA[k] : 0;
    const int inc = block_incl_max(v, scratch, -1);
    sx[threadIdx.x] = inc;
    __syncthreads();
    const int ex = threadIdx.x == 0 ? carry : max(carry, sx[threadIdx.x - 1]);
    if (k < nw) WL[k] = ex;
    const int c2 = max(carry, sx[255]);
    __syncthreads();
    carry = c2;
    int tot;
    const int ao = block_excl_sum(ac, scratch, &tot);
    if (k < nw) WA[k] = active + ao;
    active += tot;
  }
  for (int base = 0; base < nt; base += 256) {
    const int k = base + threadIdx.x;
    int tot;
    block_excl_sum(k < nt ? d.tile_b[t0 + k] : 0, scratch, &tot);
    heads += tot;
    block_excl_sum(k < nt ? d.tile_c[t0 + k] : 0, scratch, &tot);
    singles += tot;
  }
  if (threadIdx.x == 0) {
    const int m = d.m[b];
    const bool fin = active == 0 || heads == d.ngroups[b] || prefix_len >= m;
    d.ngroups[b] = heads - singles;  // groups among the rotations still active
    if (fin) {
      d.done[b] = 1;
      d.act_len[b] = 0;
    } else {
      d.act_len[b] = active;
      atomicAdd(&d.sort_ctl[2], 1);
      atomicAdd(&d.sort_ctl[6], active);
      atomicAdd(&d.sort_ctl[4], (active + kTile - 1) / kTile);
      d.active_sum[b] += active;  // rotations entering the next round
    }
  }
}

// Write SA and ISA for the sorted elements, and compact the elements of
// groups of size >= 2 (for blocks still sorting) into the other key/value/
// position buffers, keyed by their new head (rank of i+h added next round).
__global__ void __launch_bounds__(256) k_bwt_apply(SlabDev d, Layout L, int initial, int kb,
                                                   const int32_t *list) {
  const int t = tile_id(list);
  int b, lt;
  const int valid = tile_valid(d, t, d.sort_len, &b, &lt);
  if (valid == 0) return;
  const int len = d.sort_len[b];
  const int64_t off = d.off[b];
  const int cur = d.sort_ctl[0], pc = d.sort_ctl[3];
  const uint64_t *K = d.keys[cur] + off;
  const uint32_t *V = d.vals[cur] + off;
  const int32_t *P = d.kpos[pc] + off;
  const bool compact = d.done[b] == 0;
  const int w = warp_id(), ln = lane_id();
  // this warp span's head carry and compaction offset (k_bwt_rank_block)
  int carry = d.warp_last[t * kSortWarps + w];
  int aoff = d.warp_act[t * kSortWarps + w];
  uint64_t *KO = d.keys[cur ^ 1] + off;
  uint32_t *VO = d.vals[cur ^ 1] + off;
  int32_t *PO = d.kpos[pc ^ 1] + off;
  int32_t *SA = d.sa + off;
  int32_t *IS = d.isa + off;
  const unsigned lt_mask = (1u << ln) - 1u;
  // heads by a running max, writes, compaction
#pragma unroll 4
  for (int i = 0; i < kTileItems; i++) {
    const int e = w * kWarpSpan + i * 32 + ln;
    const bool ok = e < valid;
    int pos = 0, hdpos = -1;
    uint32_t val = 0;
    bool active = false;
    if (ok) {
      const int k = lt + e;
      const uint64_t item = K[k];
      const uint64_t key = key_of(L, item);
      const bool hd = k == 0 || key != key_of(L, K[k - 1]);
      const bool tl = k + 1 == len || key_of(L, K[k + 1]) != key;
      pos = initial ? k : P[k];
      val = L.packed ? (uint32_t)(item & ((1ull << L.low) - 1)) : V[k];
      if (hd) hdpos = pos;
      active = !(hd && tl);
    }
    const int head = max(carry, warp_incl_max(hdpos));
    carry = __shfl_sync(0xffffffffu, head, 31);
    const unsigned am = __ballot_sync(0xffffffffu, active);
    if (ok) {
      SA[pos] = (int32_t)val;
      IS[val] = head;
      if (compact && active) {
        const int r = aoff + __popc(am & lt_mask);
        if (L.packed) {
          KO[r] = ((uint64_t)(uint32_t)head << (2 * kb)) | val;
        } else {
          KO[r] = (uint64_t)(uint32_t)head << kb;
          VO[r] = val;
        }
        PO[r] = pos;
      }
    }
    aoff += __popc(am);
  }
}

// Next round: sort_len = active rotations; list the tiles that hold them.
__global__ void k_bwt_tile_list(SlabDev d) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nblocks) return;
  const int len = d.act_len[b];
  d.sort_len[b] = len;
  if (len <= 0) return;
  const int nt = (len + kTile - 1) / kTile;
  const int at = atomicAdd(&d.sort_ctl[5], nt);
  const int t0 = (int)(d.off[b] / kTile);
  for (int k = 0; k < nt; k++) d.tile_list[at + k] = t0 + k;
}

__global__ void k_bwt_flip(SlabDev d) {
  d.sort_ctl[0] ^= 1;
  d.sort_ctl[3] ^= 1;
}

// Round keys for the compacted active rotations: add the rank of i+h.
__global__ void __launch_bounds__(256) k_bwt_round_keys(SlabDev d, int h, int packed, int kb,
                                                        const int32_t *list) {
  const int t = tile_id(list);
  const int b = d.tile_block[t];
  const int64_t off = d.off[b];
  const int lt = (int)((int64_t)t * kTile - off);
  const int len = d.sort_len[b];
  const int valid = min(kTile, len - lt);
  if (valid <= 0) return;
  const int m = d.m[b];
  const int cur = d.sort_ctl[0];
  uint64_t *K = d.keys[cur] + off + lt;
  const uint32_t *V = d.vals[cur] + off + lt;
  const int32_t *IS = d.isa + off;
  const uint64_t mask = (1ull << kb) - 1;
  for (int e = threadIdx.x; e < valid; e += blockDim.x) {
    if (packed) {
      const uint64_t item = K[e];
      int i2 = (int)(item & mask) + h;
      if (i2 >= m) i2 -= m;
      K[e] = item | ((uint64_t)(uint32_t)IS[i2] << kb);
    } else {
      int i2 = (int)V[e] + h;
      if (i2 >= m) i2 -= m;
      K[e] |= (uint32_t)IS[i2];
    }
  }
}

bool smem_configured = false;

}  // namespace

void stage_bwt(const SlabDev &d, int max_m, cudaStream_t st) {
  if (!smem_configured) {
    BZ_CUDA(cudaFuncSetAttribute(k_radix_scatter<true, 8>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)scatter_smem_vals<8>()));
    BZ_CUDA(cudaFuncSetAttribute(k_radix_scatter<false, 8>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)scatter_smem_keys<8>()));
    BZ_CUDA(cudaFuncSetAttribute(k_radix_scatter<false, 9>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)scatter_smem_keys<9>()));
    smem_configured = true;
  }
  k_bwt_init<<<(d.nblocks + 127) / 128, 128, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
  if (max_m <= 1) return;
  // the tiles holding rotations (a block's workspace has room for its
  // worst-case RLE1 output, so most of its tiles are usually empty), and the
  // slab's largest m, which sets the width of the rank fields
  const int nlive = live_tiles(d, st);
  if (nlive == 0) return;
  if (nlive > 0 && d.live[2] >= 0) max_m = std::min(max_m, std::max(d.live[2], 1));
  if (max_m <= 1) return;
  int kb = 1;
  while ((1ll << kb) <= (int64_t)max_m) kb++;
  const int packed = 3 * kb <= 64;
  bool rounds_timed = d.kt_on && d.rt_ev != nullptr;
  if (rounds_timed) {
    d.rt_act[0] = 0;
    BZ_CUDA(cudaEventRecord(d.rt_ev[0], st));
  }
  const int grid0 = nlive > 0 ? nlive : d.ntiles;
  const int32_t *list0 = nlive > 0 ? d.vt_list : nullptr;
  // first sort: 4-byte prefixes in the high half of packed items, or 8-byte keys
  const Layout first = {packed, packed ? 32 : 0};
  const Layout round = {packed, packed ? kb : 0};
  if (packed) {
    radix_sort(d, 32, 64, 0, st, grid0, list0, true);
  } else {
    k_bwt_keys0<<<d.ntiles, 256, 0, st>>>(d, packed);
    BZ_LAUNCH_CHECK();
    radix_sort(d, 0, 64, 1, st, d.ntiles, nullptr);
  }
  const int nq = packed ? 3 : 4;  // prefixes 1,2,4 (,8) bytes
  int64_t prefix = packed ? 4 : 8;
  int grid = grid0;
  const int32_t *list = list0;
  int r = 0;  // round being run (0: the first sort)
  for (int initial = 1;; initial = 0) {
    const Layout L = initial ? first : round;
    BZ_CUDA(cudaMemsetAsync(d.sort_ctl + 2, 0, sizeof(int32_t), st));
    BZ_CUDA(cudaMemsetAsync(d.sort_ctl + 4, 0, 3 * sizeof(int32_t), st));
    k_bwt_flags<<<grid, 256, 0, st>>>(d, L, initial, list, packed ? 32 : 64, initial ? nq : 0);
    BZ_LAUNCH_CHECK();
    if (initial) {
      k_bwt_prefix_account<<<(d.nblocks + 127) / 128, 128, 0, st>>>(d, nq);
      BZ_LAUNCH_CHECK();
    }
    k_bwt_rank_block<<<d.nblocks, 256, 0, st>>>(d, prefix);
    BZ_LAUNCH_CHECK();
    k_bwt_apply<<<grid, 256, 0, st>>>(d, L, initial, kb, list);
    BZ_LAUNCH_CHECK();
    k_bwt_flip<<<1, 1, 0, st>>>(d);
    BZ_LAUNCH_CHECK();
    if (rounds_timed) {
      BZ_CUDA(cudaEventRecord(d.rt_ev[2 * r + 1], st));
      *d.rt_n = r + 1;
    }
    if (prefix >= max_m) break;
    k_bwt_tile_list<<<(d.nblocks + 127) / 128, 128, 0, st>>>(d);
    BZ_LAUNCH_CHECK();
    BZ_CUDA(cudaMemcpyAsync(d.h_flags, d.sort_ctl + 2, 8 * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            st));
    BZ_CUDA(cudaStreamSynchronize(st));
    if (rounds_timed && initial)
      std::memcpy(&d.rt_act[0], d.h_flags + 6, sizeof(int64_t));  // sort_ctl[8..9]
    if (d.h_flags[0] == 0) break;
    grid = d.h_flags[2];  // tiles holding active rotations
    list = d.tile_list;
    r++;
    if (rounds_timed && r >= kMaxRounds) rounds_timed = false;
    if (rounds_timed) {
      d.rt_act[r] = d.h_flags[4];  // rotations entering this round
      BZ_CUDA(cudaEventRecord(d.rt_ev[2 * r], st));
    }
    k_bwt_round_keys<<<grid, 256, 0, st>>>(d, (int)prefix, packed, kb, list);
    BZ_LAUNCH_CHECK();
    if (packed)
      radix_sort(d, kb, 3 * kb, 0, st, grid, list);
    else
      radix_sort(d, 0, 2 * kb, 1, st, grid, list);
    prefix *= 2;
  }
}

}  // namespace bz2g
