// BWT of every block of a slab: sorted cyclic rotations by prefix doubling.
//
// Reference: src/compression/fbwt.cu:47-106 (prefix doubling with a stable
// 64-bit key sort each round; ties, i.e. equal rotations, keep index order).
//
// Here:
//   1. One segmented LSD radix sort (segments = blocks) of every rotation by
//      its first 8 bytes (cyclic, big-endian 64-bit key), index as value.
//      The sort is stable from index order, so ties are index-ascending.
//   2. Ranks are group heads: head(j) = first sorted position of j's group.
//      ISA[i] = head of rotation i, HEAD[j] = head of sorted position j.
//   3. Round with shift h (prefix length h -> 2h): each position j of a block
//      still sorting gets key (HEAD[j] << kb) | ISA[(SA[j] + h) mod m]
//      (0 for singletons) and is re-sorted stably within its block.
//   4. A block stops when every group is a singleton, when a round splits no
//      group (the rest are equal rotations, already index-ascending), or when
//      the prefix length reaches m.
// Block-local ranks fit kb = ceil(log2(max m + 1)) bits, so keys are 2*kb bits.
#include <algorithm>

#include "engine.h"

namespace bz2g {

namespace {

constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kSortWarps = kTileThreads / 32;  // 8
constexpr size_t kScatterSmem =
    (size_t)kTile * 8 + (size_t)kTile * 4 + (size_t)kSortWarps * kRadix * 4 + 2 * kRadix * 4;

__device__ __forceinline__ int tile_valid(const SlabDev &d, int t, const int32_t *lens, int *b_out,
                                          int *lt_out) {
  int b = d.tile_block[t];
  int lt = (int)((int64_t)t * kTile - d.off[b]);
  *b_out = b;
  *lt_out = lt;
  int v = lens[b] - lt;
  return v < 0 ? 0 : (v > kTile ? kTile : v);
}

__global__ void __launch_bounds__(256) k_radix_hist(SlabDev d, int shift) {
  __shared__ uint32_t cnt[kRadix];
  int b, lt;
  int valid = tile_valid(d, blockIdx.x, d.sort_len, &b, &lt);
  if (valid == 0) return;
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t *K = d.keys[d.sort_ctl[0]] + d.off[b] + lt;
  for (int e = threadIdx.x; e < valid; e += blockDim.x)
    atomicAdd(&cnt[(uint32_t)(K[e] >> shift) & (kRadix - 1)], 1u);
  __syncthreads();
  d.tile_hist[(size_t)blockIdx.x * kRadix + threadIdx.x] = cnt[threadIdx.x];
}

// Per block: turn tile digit counts into global scatter bases.
__global__ void __launch_bounds__(256) k_radix_scan(SlabDev d) {
  __shared__ uint32_t scratch[40];
  const int b = blockIdx.x;
  const int len = d.sort_len[b];
  if (len <= 0) return;
  const int nt = (len + kTile - 1) / kTile;
  const int t0 = (int)(d.off[b] / kTile);
  const int dg = threadIdx.x;
  uint32_t run = 0;
  for (int k = 0; k < nt; k++) {
    size_t idx = (size_t)(t0 + k) * kRadix + dg;
    uint32_t h = d.tile_hist[idx];
    d.tile_hist[idx] = run;
    run += h;
  }
  uint32_t tot;
  uint32_t base = block_excl_sum(run, scratch, &tot);
  int trivial = __syncthreads_or(run == (uint32_t)len);
  if (!trivial && threadIdx.x == 0) atomicOr(&d.sort_ctl[1], 1);
  uint32_t add = (uint32_t)d.off[b] + base;
  for (int k = 0; k < nt; k++) d.tile_hist[(size_t)(t0 + k) * kRadix + dg] += add;
}

// Stable scatter of one tile by one 8-bit digit.  Elements are warp-striped
// (lane l, item i <-> element w*512 + i*32 + l) so that ranking item by item
// with __match_any_sync keeps the original order; the tile is sorted locally
// in shared memory, then written so that equal digits go out contiguously.
__global__ void __launch_bounds__(256) k_radix_scatter(SlabDev d, int shift) {
  if (!d.sort_ctl[1]) return;
  int b, lt;
  int valid = tile_valid(d, blockIdx.x, d.sort_len, &b, &lt);
  if (valid == 0) return;
  extern __shared__ __align__(16) uint8_t smem[];
  uint64_t *sk = reinterpret_cast<uint64_t *>(smem);
  uint32_t *sv = reinterpret_cast<uint32_t *>(sk + kTile);
  uint32_t *wcnt = sv + kTile;                 // [warp][digit]
  uint32_t *lbase = wcnt + kSortWarps * kRadix;  // local digit base
  uint32_t *goff = lbase + kRadix;             // global digit base for this tile
  const int cur = d.sort_ctl[0];
  const uint64_t *K = d.keys[cur] + d.off[b] + lt;
  const uint32_t *V = d.vals[cur] + d.off[b] + lt;
  const int w = warp_id(), ln = lane_id();
  for (int i = threadIdx.x; i < kSortWarps * kRadix; i += blockDim.x) wcnt[i] = 0;
  goff[threadIdx.x] = d.tile_hist[(size_t)blockIdx.x * kRadix + threadIdx.x];
  __syncthreads();

  uint64_t key[kTileItems];
  uint32_t val[kTileItems];
  uint32_t rank[kTileItems];
  const unsigned lt_mask = (1u << ln) - 1u;
#pragma unroll
  for (int i = 0; i < kTileItems; i++) {
    int e = w * 512 + i * 32 + ln;
    bool ok = e < valid;
    key[i] = ok ? K[e] : 0;
    val[i] = ok ? V[e] : 0;
    int dg = ok ? (int)((key[i] >> shift) & (kRadix - 1)) : kRadix + 1;
    unsigned peers = __match_any_sync(0xffffffffu, dg);
    uint32_t before = ok ? wcnt[w * kRadix + dg] : 0;
    rank[i] = before + __popc(peers & lt_mask);
    __syncwarp();
    if (ok && (peers & lt_mask) == 0) wcnt[w * kRadix + dg] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {
    // prefix over warps for each digit, then exclusive scan over digits
    const int dg = threadIdx.x;
    uint32_t run = 0;
    for (int ww = 0; ww < kSortWarps; ww++) {
      uint32_t c = wcnt[ww * kRadix + dg];
      wcnt[ww * kRadix + dg] = run;
      run += c;
    }
    __shared__ uint32_t scratch[40];
    uint32_t tot;
    uint32_t ex = block_excl_sum(run, scratch, &tot);
    lbase[dg] = ex;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kTileItems; i++) {
    int e = w * 512 + i * 32 + ln;
    if (e < valid) {
      int dg = (int)((key[i] >> shift) & (kRadix - 1));
      uint32_t pos = lbase[dg] + wcnt[w * kRadix + dg] + rank[i];
      sk[pos] = key[i];
      sv[pos] = val[i];
    }
  }
  __syncthreads();
  uint64_t *KO = d.keys[cur ^ 1];
  uint32_t *VO = d.vals[cur ^ 1];
  for (int k = threadIdx.x; k < valid; k += blockDim.x) {
    uint64_t kk = sk[k];
    int dg = (int)((kk >> shift) & (kRadix - 1));
    uint32_t g = goff[dg] + (uint32_t)k - lbase[dg];
    KO[g] = kk;
    VO[g] = sv[k];
  }
}

__global__ void k_radix_flip(SlabDev d) {
  if (d.sort_ctl[1]) d.sort_ctl[0] ^= 1;
  d.sort_ctl[1] = 0;
}

void radix_sort(const SlabDev &d, int nbits, cudaStream_t st) {
  for (int shift = 0; shift < nbits; shift += kRadixBits) {
    k_radix_hist<<<d.ntiles, 256, 0, st>>>(d, shift);
    BZ_LAUNCH_CHECK();
    k_radix_scan<<<d.nblocks, 256, 0, st>>>(d);
    BZ_LAUNCH_CHECK();
    k_radix_scatter<<<d.ntiles, 256, kScatterSmem, st>>>(d, shift);
    BZ_LAUNCH_CHECK();
    k_radix_flip<<<1, 1, 0, st>>>(d);
    BZ_LAUNCH_CHECK();
  }
}

// ------------------------------------------------------------------- BWT
__global__ void k_bwt_init(SlabDev d) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b == 0) {
    d.sort_ctl[0] = 0;
    d.sort_ctl[1] = 0;
    d.sort_ctl[2] = 0;
  }
  if (b >= d.nblocks) return;
  int m = d.m[b];
  d.sort_len[b] = m > 1 ? m : 0;
  d.done[b] = m > 1 ? 0 : 1;
  d.ngroups[b] = -1;
  d.active_sum[b] = 0;
  for (int k = 0; k < 8; k++) d.pstat[b * 8 + k] = 0;
  if (m == 1) d.sa[d.off[b]] = 0;
}

// Group heads and singletons of the prefix-1, -2, -4 and -8 partitions, read
// off the 8-byte sorted keys (pstat[b*8 + q] heads, [b*8 + 4 + q] singletons).
__global__ void __launch_bounds__(256) k_bwt_prefix_stats(SlabDev d) {
  int b, lt;
  int valid = tile_valid(d, blockIdx.x, d.sort_len, &b, &lt);
  if (valid == 0) return;
  const int m = d.m[b];
  const uint64_t *K = d.keys[d.sort_ctl[0]] + d.off[b];
  int cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int e = threadIdx.x; e < valid; e += blockDim.x) {
    const int j = lt + e;
    const uint64_t k = K[j];
    const uint64_t kp = j > 0 ? K[j - 1] : 0;
    const uint64_t kn = j + 1 < m ? K[j + 1] : 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int sh = 64 - 8 * (1 << q);
      const uint64_t a = sh > 0 ? k >> sh : k;
      const bool hd = j == 0 || a != (sh > 0 ? kp >> sh : kp);
      const bool tl = j + 1 == m || a != (sh > 0 ? kn >> sh : kn);
      cnt[q] += hd;
      cnt[4 + q] += hd && tl;
    }
  }
#pragma unroll
  for (int q = 0; q < 8; q++) {
    int v = cnt[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane_id() == 0 && v) atomicAdd(&d.pstat[b * 8 + q], v);
  }
}

// The oracle's accounting of rounds h = 1, 2, 4 (round h runs while the
// partition has a non-singleton group and the previous round split one), and
// the prefix-4 group count as the fixed-point reference of the first round.
__global__ void k_bwt_prefix_account(SlabDev d) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nblocks) return;
  const int m = d.m[b];
  if (m <= 1) return;
  const int32_t *ps = d.pstat + b * 8;
  int64_t A = 0;
  bool stop = false;
  for (int q = 0; q < 3 && !stop; q++) {
    const int G = ps[q], S = ps[4 + q];
    if (G == m) break;
    A += m - S;
    const int h = 1 << q;
    if (ps[q + 1] == G || 2 * h >= m) stop = true;
  }
  d.active_sum[b] = A;
  d.ngroups[b] = ps[2];
}

// Initial keys: the first 8 bytes of each rotation.
__global__ void __launch_bounds__(256) k_bwt_keys0(SlabDev d) {
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
#pragma unroll
    for (int q = 0; q < 8; q++) k = (k << 8) | sb[e + q];
    K[e] = k;
    V[e] = (uint32_t)(lt + e);
  }
}

// Group heads after a sort: per tile, the last head position and head count.
__global__ void __launch_bounds__(256) k_bwt_rank_tiles(SlabDev d) {
  __shared__ int red[3][8];
  int b, lt;
  int valid = tile_valid(d, blockIdx.x, d.sort_len, &b, &lt);
  if (valid == 0) return;
  const uint64_t *K = d.keys[d.sort_ctl[0]] + d.off[b];
  const int m = d.sort_len[b];
  int last = -1, cnt = 0, sing = 0;
  for (int e = threadIdx.x; e < valid; e += blockDim.x) {
    int j = lt + e;
    bool hd = j == 0 || K[j] != K[j - 1];
    if (hd) {
      last = max(last, j);
      cnt++;
      sing += j + 1 == m || K[j + 1] != K[j];
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    last = max(last, __shfl_xor_sync(0xffffffffu, last, o));
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    sing += __shfl_xor_sync(0xffffffffu, sing, o);
  }
  if (lane_id() == 0) {
    red[0][warp_id()] = last;
    red[1][warp_id()] = cnt;
    red[2][warp_id()] = sing;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int l = -1, c = 0, sg = 0;
    for (int w = 0; w < 8; w++) {
      l = max(l, red[0][w]);
      c += red[1][w];
      sg += red[2][w];
    }
    d.tile_a[blockIdx.x] = l;
    d.tile_b[blockIdx.x] = c;
    d.tile_c[blockIdx.x] = sg;
  }
}

// Per block: carry of the last head into each tile; group count; stop test.
__global__ void __launch_bounds__(256) k_bwt_rank_block(SlabDev d, int64_t prefix_len) {
  __shared__ int scratch[40];
  __shared__ int sx[256];
  const int b = blockIdx.x;
  const int len = d.sort_len[b];
  if (len <= 0) return;
  const int nt = (len + kTile - 1) / kTile;
  const int t0 = (int)(d.off[b] / kTile);
  int carry = -1, count = 0, singles = 0;
  for (int base = 0; base < nt; base += 256) {
    int k = base + threadIdx.x;
    int v = k < nt ? d.tile_a[t0 + k] : -1;
    int c = k < nt ? d.tile_b[t0 + k] : 0;
    int sg = k < nt ? d.tile_c[t0 + k] : 0;
    int inc = block_incl_max(v, scratch, -1);
    sx[threadIdx.x] = inc;
    __syncthreads();
    int ex = threadIdx.x == 0 ? carry : max(carry, sx[threadIdx.x - 1]);
    if (k < nt) d.tile_a[t0 + k] = ex;
    int c2 = max(carry, sx[255]);
    __syncthreads();
    carry = c2;
    int tot;
    block_excl_sum(c, scratch, &tot);
    count += tot;
    block_excl_sum(sg, scratch, &tot);
    singles += tot;
  }
  if (threadIdx.x == 0) {
    int m = d.m[b];
    bool fin = count == m || count == d.ngroups[b] || prefix_len >= m;
    d.ngroups[b] = count;
    if (fin) {
      d.done[b] = 1;
    } else {
      atomicAdd(&d.sort_ctl[2], 1);
      d.active_sum[b] += m - singles;  // rotations entering the next round
    }
  }
}

// Write SA, HEAD and ISA for the sorted positions of each block still sorting.
__global__ void __launch_bounds__(256) k_bwt_rank_apply(SlabDev d) {
  __shared__ int scratch[40];
  __shared__ int wl[8];
  int b, lt;
  int valid = tile_valid(d, blockIdx.x, d.sort_len, &b, &lt);
  if (valid == 0) return;
  const int cur = d.sort_ctl[0];
  const int64_t off = d.off[b];
  const uint64_t *K = d.keys[cur] + off;
  const uint32_t *V = d.vals[cur] + off;
  const int p0 = threadIdx.x * kTileItems;
  int ls = -1;
  for (int k = 0; k < kTileItems; k++) {
    int e = p0 + k;
    if (e >= valid) break;
    int j = lt + e;
    if (j == 0 || K[j] != K[j - 1]) ls = j;
  }
  int inc = block_incl_max(ls, scratch, -1);
  int ex = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane_id() == 31) wl[warp_id()] = inc;
  __syncthreads();
  if (lane_id() == 0) ex = warp_id() == 0 ? -1 : wl[warp_id() - 1];
  int cur_head = max(ex, d.tile_a[blockIdx.x]);
  for (int k = 0; k < kTileItems; k++) {
    int e = p0 + k;
    if (e >= valid) break;
    int j = lt + e;
    if (j == 0 || K[j] != K[j - 1]) cur_head = j;
    int i = (int)V[j];
    d.sa[off + j] = i;
    d.head[off + j] = cur_head;
    d.isa[off + i] = cur_head;
  }
}

// Round keys: (HEAD[j] << kb) | ISA[(SA[j] + h) mod m]; singletons get 0.
__global__ void __launch_bounds__(256) k_bwt_round_keys(SlabDev d, int h, int kb) {
  const int t = blockIdx.x;
  const int b = d.tile_block[t];
  const int64_t off = d.off[b];
  const int lt = (int)((int64_t)t * kTile - off);
  const int m = d.m[b];
  const bool dn = d.done[b] != 0;
  if (lt == 0 && threadIdx.x == 0) d.sort_len[b] = dn ? 0 : m;
  if (dn) return;
  int valid = min(kTile, m - lt);
  if (valid <= 0) return;
  const int cur = d.sort_ctl[0];
  uint64_t *K = d.keys[cur] + off;
  uint32_t *V = d.vals[cur] + off;
  const int32_t *SA = d.sa + off;
  const int32_t *HD = d.head + off;
  const int32_t *IS = d.isa + off;
  for (int e = threadIdx.x; e < valid; e += blockDim.x) {
    int j = lt + e;
    int i = SA[j];
    int hd = HD[j];
    bool single = hd == j && (j + 1 == m || HD[j + 1] == j + 1);
    uint32_t k2 = 0;
    if (!single) {
      int i2 = i + h;
      if (i2 >= m) i2 -= m;
      k2 = (uint32_t)IS[i2];
    }
    K[j] = ((uint64_t)(uint32_t)hd << kb) | k2;
    V[j] = (uint32_t)i;
  }
}

bool smem_configured = false;

}  // namespace

void stage_bwt(const SlabDev &d, int max_m, cudaStream_t st) {
  if (!smem_configured) {
    BZ_CUDA(cudaFuncSetAttribute(k_radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kScatterSmem));
    smem_configured = true;
  }
  int kb = 1;
  while ((1ll << kb) <= (int64_t)max_m) kb++;
  k_bwt_init<<<(d.nblocks + 127) / 128, 128, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
  if (max_m <= 1) return;
  k_bwt_keys0<<<d.ntiles, 256, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
  radix_sort(d, 64, st);
  k_bwt_prefix_stats<<<d.ntiles, 256, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
  k_bwt_prefix_account<<<(d.nblocks + 127) / 128, 128, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
  int64_t prefix = 8;
  for (int round = 0;; round++) {
    BZ_CUDA(cudaMemsetAsync(d.sort_ctl + 2, 0, sizeof(int32_t), st));
    k_bwt_rank_tiles<<<d.ntiles, 256, 0, st>>>(d);
    BZ_LAUNCH_CHECK();
    k_bwt_rank_block<<<d.nblocks, 256, 0, st>>>(d, prefix);
    BZ_LAUNCH_CHECK();
    k_bwt_rank_apply<<<d.ntiles, 256, 0, st>>>(d);
    BZ_LAUNCH_CHECK();
    if (prefix >= max_m) break;
    BZ_CUDA(cudaMemcpyAsync(d.h_flags, d.sort_ctl + 2, sizeof(int32_t), cudaMemcpyDeviceToHost,
                            st));
    BZ_CUDA(cudaStreamSynchronize(st));
    if (d.h_flags[0] == 0) break;
    int h = (int)prefix;
    k_bwt_round_keys<<<d.ntiles, 256, 0, st>>>(d, h, kb);
    BZ_LAUNCH_CHECK();
    radix_sort(d, 2 * kb, st);
    prefix *= 2;
  }
}

}  // namespace bz2g
