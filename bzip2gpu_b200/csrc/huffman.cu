// Huffman table selection and code lengths, for every block of a slab.
//
// Reference: src/compression/huffman.cu:126-364 (bzip2 1.0.8 sendMTFValues
// semantics): nGroups from the symbol count; initial tables from the symbol
// histogram; 4 passes of (per 50-symbol group: cost of every table, first
// minimum wins, per-table frequencies of the chosen groups) each followed by
// length-limited (17) Huffman code lengths per table; canonical codes.
// The histogram is defined as zeroed (the reference leaves it uninitialised).
#include "engine.h"
#include "selector.h"

namespace bz2g {

namespace {

// Which blocks a launch serves: every block, the plain-selector blocks, the
// learned-selector blocks, or (learned form, after the judge) the plain
// blocks that still have passes to run in this round.
enum Which { kAll = 0, kPlain = 1, kLearned = 2, kPlainRound = 3 };

__device__ __forceinline__ bool serves(const SlabDev &d, int b, int which, int round) {
  switch (which) {
    case kAll:
      return true;
    case kPlain:
      return d.learned[b] == 0;
    case kLearned:
      return d.learned[b] != 0;
    default:
      return d.learned[b] == 0 && round < d.plain_left[b];
  }
}

// bzip2's initial tables (src/compression/huffman.cu:148-185): every length
// 15, then table n_part - 1 gets length 0 over the next range of symbols
// holding about remaining / n_part of the symbol count.  One warp.
__device__ void init_tables(const SlabDev &d, int b) {
  const int s = d.s[b];
  const int ng = d.n_groups[b];
  const int alpha = d.n_in_use[b] + 2;
  uint8_t *len = d.len + (size_t)b * kMaxGroups * kMaxAlpha;
  for (int i = lane_id(); i < kMaxGroups * kMaxAlpha; i += 32) len[i] = 15;
  __syncwarp();
  if (lane_id() == 0) {
    const int32_t *freq = d.freq + (size_t)b * kMaxAlpha;
    int gs = 0, remaining = s;
    for (int n_part = ng; n_part > 0; n_part--) {
      int t_freq = remaining / n_part;
      int ge = gs - 1, a_freq = 0;
      while (a_freq < t_freq && ge < alpha) {
        ge++;
        a_freq += ge < kMaxAlpha ? freq[ge] : 0;
      }
      if (ge > gs && n_part != ng && n_part != 1 && ((ng - n_part) % 2 == 1)) {
        a_freq -= ge < kMaxAlpha ? freq[ge] : 0;
        ge--;
      }
      uint8_t *row = len + (n_part - 1) * kMaxAlpha;
      for (int v = 0; v < alpha; v++) row[v] = (v >= gs && v <= ge) ? 0 : 15;
      gs = ge + 1;
      remaining -= a_freq;
    }
  }
  __syncwarp();
}

// learned_mode: blocks with six tables take the learned selector; the plain
// blocks of the learned form have 2 passes left after the two shared ones.
__global__ void k_huff_init(SlabDev d, int learned_mode) {
  const int b = blockIdx.x;
  const int s = d.s[b];
  const int ng = s < 200 ? 2 : s < 600 ? 3 : s < 1200 ? 4 : s < 2400 ? 5 : 6;
  if (threadIdx.x == 0) {
    d.n_groups[b] = ng;
    d.n_sel[b] = (s + 49) / 50;
    d.learned[b] = (learned_mode && ng == kMaxGroups) ? 1 : 0;
    d.plain_left[b] = kIters - 2;
  }
  __syncwarp();
  init_tables(d, b);
}

// One thread per 50-symbol group.  Costs of all tables are packed in 10-bit
// fields of one 64-bit word per symbol (50 * 17 < 1024), so a group's six
// costs are one 64-bit sum.
// grid.y == 2 (the learned form's second passes): y = 1 runs, for the
// learned blocks, the plain selector's second pass over its first-pass
// tables (len2) into sel2 / rfreq2, beside y = 0's pass over len.
// list: the group tiles to run (blockIdx.x-th entry), or nullptr for all.
__global__ void __launch_bounds__(kGroupTile) k_huff_select(SlabDev d, int which, int round,
                                                            const int32_t *list) {
  __shared__ uint16_t sy[kGroupTile * kGroupSize];
  __shared__ uint64_t plen[kMaxAlpha];
  __shared__ int rf[kMaxGroups * kMaxAlpha];
  const int gt = list ? list[blockIdx.x] : (int)blockIdx.x;
  const int b = d.gt_block[gt];
  const int g0 = d.gt_first[gt];
  const int nsel = d.n_sel[b];
  const bool second = blockIdx.y == 1;
  if (g0 >= nsel) return;
  if (second ? !d.learned[b] : !serves(d, b, which, round)) return;
  const uint8_t *len_src = second ? d.len2 : d.len;
  uint8_t *sel_dst = second ? d.sel2 : d.sel;
  int32_t *rf_dst = second ? d.rfreq2 : d.rfreq;
  const int ng_here = min(kGroupTile, nsel - g0);
  const int s = d.s[b];
  const int ngrp = d.n_groups[b];
  const int alpha = d.n_in_use[b] + 2;
  const int64_t off = d.off[b];
  const int sym0 = g0 * kGroupSize;
  const int nsym = min(s, (g0 + ng_here) * kGroupSize) - sym0;
  const uint8_t *len = len_src + (size_t)b * kMaxGroups * kMaxAlpha;
  for (int i = threadIdx.x; i < nsym; i += blockDim.x) sy[i] = d.rle2[off + sym0 + i];
  for (int v = threadIdx.x; v < kMaxAlpha; v += blockDim.x) {
    uint64_t p = 0;
    if (v < alpha)
      for (int t = 0; t < ngrp; t++) p |= (uint64_t)len[t * kMaxAlpha + v] << (10 * t);
    plen[v] = p;
  }
  for (int i = threadIdx.x; i < kMaxGroups * kMaxAlpha; i += blockDim.x) rf[i] = 0;
  __syncthreads();
  const int g = threadIdx.x;
  if (g < ng_here) {
    const int a = g * kGroupSize;
    const int e = min(a + kGroupSize, nsym);
    uint64_t cost = 0;
    for (int i = a; i < e; i++) cost += plen[sy[i]];
    uint32_t bc = 0xFFFFFFFFu;
    int bt = -1;
    for (int t = 0; t < ngrp; t++) {
      uint32_t c = (uint32_t)(cost >> (10 * t)) & 1023u;
      if (c < bc) {
        bc = c;
        bt = t;
      }
    }
    sel_dst[off / 32 + g0 + g] = (uint8_t)bt;
    // RUNA, RUNB and MTF index 1 (symbols 0, 1, 2) make up most of a block's
    // symbols: count them in registers, so that the threads of a warp do not
    // all add to the same few counters one symbol at a time
    int c0 = 0, c1 = 0, c2 = 0;
    int *rft = rf + bt * kMaxAlpha;
    for (int i = a; i < e; i++) {
      const int v = sy[i];
      if (v < 3) {
        c0 += v == 0;
        c1 += v == 1;
        c2 += v == 2;
      } else {
        atomicAdd(&rft[v], 1);
      }
    }
    if (c0) atomicAdd(&rft[0], c0);
    if (c1) atomicAdd(&rft[1], c1);
    if (c2) atomicAdd(&rft[2], c2);
  }
  __syncthreads();
  int32_t *rfreq = rf_dst + (size_t)b * kMaxGroups * kMaxAlpha;
  for (int i = threadIdx.x; i < ngrp * kMaxAlpha; i += blockDim.x)
    if (rf[i]) atomicAdd(&rfreq[i], rf[i]);
}

// bzip2's length-limited Huffman lengths (src/compression/huffman.cu:13-124),
// one warp per block: lane t runs table t's heap (a block's tables share
// its alphabet size, so the lanes' heaps have equal sizes at every step and
// stay in step), so the warp issues about one heap's instructions for all
// six.  Heap entries carry their node's weight in the high half (weight << 32
// | node), so a sift step reads a sibling pair with one 16-byte shared load;
// comparisons use the weight half only, with the reference's strict '<', so
// ties resolve exactly as there.  All lanes then walk the parent links for
// the code lengths, table by table.
constexpr int kHeapN = kMaxAlpha + 2;
constexpr int kNodeN = kMaxAlpha * 2;

__device__ __forceinline__ uint32_t hw(uint64_t e) { return (uint32_t)(e >> 32); }

// split (the learned form, grid.y = 2): y = 0 builds every block's tables
// into len, y = 1 the learned blocks' plain-selector tables into len2.
// split == 1 (first build): y = 0 from the counts of the first pass (the
// MLP's counts for learned blocks), y = 1 from the first plain pass's counts.
// split == 2 (second build): y = 0 from rfreq, y = 1 from rfreq2.
__global__ void __launch_bounds__(32) k_huff_lengths(SlabDev d, int which, int round, int split) {
  __shared__ __align__(16) uint64_t heap_s[kMaxGroups][kHeapN + 2];
  __shared__ int32_t leafw_s[kMaxGroups][kMaxAlpha + 1];
  __shared__ int16_t parent_s[kMaxGroups][kNodeN];
  const int b = blockIdx.x;
  const int ln = lane_id();
  const int ngrp = d.n_groups[b];
  const int32_t *rf_base = d.rfreq;
  uint8_t *len_base = d.len;
  if (split) {
    if (blockIdx.y == 0) {
      if (split == 1 && d.learned[b]) rf_base = d.rfreq_m;
    } else {
      if (!d.learned[b]) return;
      len_base = d.len2;
      if (split == 2) rf_base = d.rfreq2;
    }
  } else if (!serves(d, b, which, round)) {
    return;
  }
  const int alpha = d.n_in_use[b] + 2;
  for (int t = 0; t < ngrp; t++) {
    const int32_t *freq = rf_base + ((size_t)b * kMaxGroups + t) * kMaxAlpha;
    for (int i = ln; i < alpha; i += 32) {
      const int f = freq[i];
      leafw_s[t][i + 1] = (f == 0 ? 1 : f) << 8;
    }
  }
  __syncwarp();
  unsigned pending = (1u << ngrp) - 1u;  // tables whose lengths are not final yet
  while (pending) {
    if ((pending >> ln) & 1u) {
      uint64_t *heap = heap_s[ln];
      const int32_t *leafw = leafw_s[ln];
      int16_t *parent = parent_s[ln];
      int n_nodes = alpha, n_heap = 0;
      heap[0] = 0;  // sentinel: weight 0
      for (int i = 1; i <= alpha; i++) {
        parent[i] = -1;
        n_heap++;
        const uint64_t e = ((uint64_t)(uint32_t)leafw[i] << 32) | (uint32_t)i;
        int zz = n_heap;
        uint64_t up = heap[zz >> 1];
        while (hw(e) < hw(up)) {
          heap[zz] = up;
          zz >>= 1;
          up = heap[zz >> 1];
        }
        heap[zz] = e;
      }
      while (n_heap > 1) {
        uint64_t pick[2];
        for (int q = 0; q < 2; q++) {
          pick[q] = heap[1];
          const uint64_t tmp = heap[n_heap];
          n_heap--;
          int zz = 1;
          for (;;) {
            int yy = zz << 1;
            if (yy > n_heap) break;
            const ulonglong2 pr = *reinterpret_cast<const ulonglong2 *>(&heap[yy]);
            uint64_t c = pr.x;
            if (yy < n_heap && hw(pr.y) < hw(pr.x)) {
              yy++;
              c = pr.y;
            }
            if (hw(tmp) < hw(c)) break;
            heap[zz] = c;
            zz = yy;
          }
          heap[zz] = tmp;
        }
        const uint32_t w1 = hw(pick[0]), w2 = hw(pick[1]);
        const int n1 = (int)(uint32_t)pick[0], n2 = (int)(uint32_t)pick[1];
        n_nodes++;
        parent[n1] = parent[n2] = (int16_t)n_nodes;
        const uint32_t d1 = w1 & 0xff, d2 = w2 & 0xff;
        const uint32_t wn = ((w1 & 0xffffff00u) + (w2 & 0xffffff00u)) | (1 + (d1 > d2 ? d1 : d2));
        parent[n_nodes] = -1;
        n_heap++;
        const uint64_t e = ((uint64_t)wn << 32) | (uint32_t)n_nodes;
        int zz = n_heap;
        uint64_t up = heap[zz >> 1];
        while (hw(e) < hw(up)) {
          heap[zz] = up;
          zz >>= 1;
          up = heap[zz >> 1];
        }
        heap[zz] = e;
      }
    }
    __syncwarp();
    unsigned redo = 0;
    for (int t = 0; t < ngrp; t++) {
      if (!((pending >> t) & 1u)) continue;
      const int16_t *parent = parent_s[t];
      uint8_t *len = len_base + ((size_t)b * kMaxGroups + t) * kMaxAlpha;
      bool too_long = false;
      for (int i = ln + 1; i <= alpha; i += 32) {
        int j = 0, k = i;
        while (parent[k] >= 0) {
          k = parent[k];
          j++;
        }
        len[i - 1] = (uint8_t)j;
        too_long |= j > kMaxCodeLen;
      }
      if (__any_sync(0xffffffffu, too_long)) {
        redo |= 1u << t;
        for (int i = ln + 1; i <= alpha; i += 32) {
          int j = leafw_s[t][i] >> 8;
          j = 1 + (j / 2);
          leafw_s[t][i] = j << 8;
        }
      }
    }
    __syncwarp();
    pending = redo;
  }
}

// Predicted coded size of a block's selection (bits): payload from the
// per-table counts and lengths, plus the table headers (5-bit start, 2 bits
// per unit of length change, 1 terminator bit per symbol).  One warp.
__device__ int64_t predicted_bits(const SlabDev &d, int b, const uint8_t *len_base,
                                  const int32_t *rf_base) {
  const int ng = d.n_groups[b];
  const int alpha = d.n_in_use[b] + 2;
  const int32_t *rf = rf_base + (size_t)b * kMaxGroups * kMaxAlpha;
  const uint8_t *len = len_base + (size_t)b * kMaxGroups * kMaxAlpha;
  int64_t e = 0;
  for (int t = 0; t < ng; t++)
    for (int v = lane_id(); v < alpha; v += 32) {
      const int l = len[t * kMaxAlpha + v];
      const int p = v ? len[t * kMaxAlpha + v - 1] : l;
      e += (int64_t)rf[t * kMaxAlpha + v] * l + 2 * abs(l - p) + 1;
    }
  for (int o = 16; o; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  return e + 5 * ng;
}

// Learned form, after the second passes: a learned block whose predicted
// size exceeds that of the plain selector's first two passes takes the
// plain two-pass selection (sel2, len2) instead.
__global__ void k_huff_judge(SlabDev d) {
  const int b = blockIdx.x;
  if (!d.learned[b]) return;
  const int64_t el = predicted_bits(d, b, d.len, d.rfreq);
  const int64_t ep = predicted_bits(d, b, d.len2, d.rfreq2);
  if (el <= ep) return;
  const size_t tb = (size_t)b * kMaxGroups * kMaxAlpha;
  for (int i = lane_id(); i < kMaxGroups * kMaxAlpha; i += 32) d.len[tb + i] = d.len2[tb + i];
  const int64_t s0 = d.off[b] / 32;
  const int nsel = d.n_sel[b];
  for (int g = lane_id(); g < nsel; g += 32) d.sel[s0 + g] = d.sel2[s0 + g];
  if (lane_id() == 0) {
    d.learned[b] = 0;
    d.plain_left[b] = 0;
  }
}

// Canonical codes (src/compression/huffman.cu:135-146,352-362): for each
// length from the shortest to the longest, the symbols of that length in
// symbol order take consecutive codes; the next length starts at twice the
// running code.  One warp per table: lane l holds symbols l, l + 32, ...; a
// ballot per 32 symbols gives each symbol its place among that length's.
constexpr int kCodeSlots = (kMaxAlpha + 31) / 32;  // 9

__global__ void __launch_bounds__(kMaxGroups * 32) k_huff_codes(SlabDev d) {
  const int b = blockIdx.x;
  const int t = warp_id();
  const int ln = lane_id();
  if (t >= d.n_groups[b]) return;
  const int alpha = d.n_in_use[b] + 2;
  const uint8_t *len = d.len + ((size_t)b * kMaxGroups + t) * kMaxAlpha;
  int32_t *code = d.code + ((size_t)b * kMaxGroups + t) * kMaxAlpha;
  int lv[kCodeSlots];
  int mn = 32, mx = 0;
#pragma unroll
  for (int q = 0; q < kCodeSlots; q++) {
    const int v = 32 * q + ln;
    lv[q] = v < alpha ? (int)len[v] : -1;
    if (v < alpha) {
      mn = min(mn, lv[q]);
      mx = max(mx, lv[q]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  const unsigned below = (1u << ln) - 1u;
  int vec = 0;
  for (int l = mn; l <= mx; l++) {
#pragma unroll
    for (int q = 0; q < kCodeSlots; q++) {
      const bool hit = lv[q] == l;
      const unsigned bal = __ballot_sync(0xffffffffu, hit);
      if (hit) code[32 * q + ln] = vec + __popc(bal & below);
      vec += __popc(bal);
    }
    vec <<= 1;
  }
}

}  // namespace

namespace {
void select_pass(const SlabDev &d, int which, int round, cudaStream_t st) {
  BZ_CUDA(cudaMemsetAsync(d.rfreq, 0, sizeof(int32_t) * kMaxGroups * kMaxAlpha * d.nblocks, st));
  const int nlive = live_group_tiles(d, st);
  const int grid = nlive >= 0 ? nlive : d.n_group_tiles;
  if (grid <= 0) return;
  k_huff_select<<<grid, kGroupTile, 0, st>>>(d, which, round, nlive >= 0 ? d.vg_list : nullptr);
  BZ_LAUNCH_CHECK();
}
void lengths_pass(const SlabDev &d, int which, int round, cudaStream_t st) {
  k_huff_lengths<<<d.nblocks, 32, 0, st>>>(d, which, round, 0);
  BZ_LAUNCH_CHECK();
}
}  // namespace

// Plain form (the reference's): initial tables, then 4 passes of selection
// and code lengths.
// Learned form, blocks with six tables: the MLP's choice gives the first
// tables, one exact selection pass and code lengths follow.  Beside them the
// plain selector runs its first two passes (initial tables, then its
// first-pass tables); that is the judge: a block whose learned tables predict
// a larger size takes the plain two-pass selection.  The judge thus costs no
// launch of its own, and the stage runs two rounds of selection and code
// lengths where the plain form runs four.  Blocks with fewer tables run the
// plain passes in the same launches (launches that serve none of a slab's
// blocks return at once).
void stage_huffman(const SlabDev &d, cudaStream_t st, const uint8_t *learned, int plain_passes,
                   uint8_t *mlp_sel_out, size_t mlp_sel_bytes) {
  k_huff_init<<<d.nblocks, 32, 0, st>>>(d, learned ? 1 : 0);
  BZ_LAUNCH_CHECK();
  if (!learned) {
    for (int it = 0; it < plain_passes; it++) {
      select_pass(d, kAll, 0, st);
      lengths_pass(d, kAll, 0, st);
    }
  } else {
    const size_t rf_bytes = sizeof(int32_t) * kMaxGroups * kMaxAlpha * d.nblocks;
    BZ_CUDA(cudaMemsetAsync(d.rfreq_m, 0, rf_bytes, st));
    select_pass(d, kAll, 0, st);  // the plain selector's first pass, every block
    mlp::launch_select(d, learned, nullptr, nullptr, d.rfreq_m, st);
    if (mlp_sel_out)
      BZ_CUDA(cudaMemcpyAsync(mlp_sel_out, d.sel, mlp_sel_bytes, cudaMemcpyDeviceToDevice, st));
    k_huff_lengths<<<dim3(d.nblocks, 2), 32, 0, st>>>(d, kAll, 0, 1);
    BZ_LAUNCH_CHECK();
    // second passes, side by side: every block over its tables (the plain
    // blocks' second pass, the learned tables' exact pass) and, for learned
    // blocks, the plain selector's second pass over its first-pass tables
    BZ_CUDA(cudaMemsetAsync(d.rfreq, 0, rf_bytes, st));
    BZ_CUDA(cudaMemsetAsync(d.rfreq2, 0, rf_bytes, st));
    {
      const int nlive = live_group_tiles(d, st);
      const int grid = nlive >= 0 ? nlive : d.n_group_tiles;
      if (grid > 0) {
        k_huff_select<<<dim3(grid, 2), kGroupTile, 0, st>>>(d, kAll, 0,
                                                          nlive >= 0 ? d.vg_list : nullptr);
        BZ_LAUNCH_CHECK();
      }
    }
    k_huff_lengths<<<dim3(d.nblocks, 2), 32, 0, st>>>(d, kAll, 0, 2);
    BZ_LAUNCH_CHECK();
    k_huff_judge<<<d.nblocks, 32, 0, st>>>(d);
    BZ_LAUNCH_CHECK();
    // plain blocks (fewer than six tables) finish their four passes
    for (int r = 0; r < kIters - 2; r++) {
      select_pass(d, kPlainRound, r, st);
      lengths_pass(d, kPlainRound, r, st);
    }
  }
  k_huff_codes<<<d.nblocks, kMaxGroups * 32, 0, st>>>(d);
  BZ_LAUNCH_CHECK();
}

}  // namespace bz2g
