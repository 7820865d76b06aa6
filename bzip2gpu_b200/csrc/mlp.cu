// Learned table selector on the 5th-generation tensor cores (tcgen05).
//
// Inference (k_mlp_select): one persistent CTA per SM walks the slab's group
// tiles (128 groups of 50 symbols each).  Per tile:
//   warps 0-3  build the 128 x 272 count matrix in shared memory (the MMA's A
//              operand), then run the epilogues: TMEM -> registers,
//              scale / bias / ReLU, bf16 back into shared memory as the next
//              layer's A operand; finally the masked argmax, the selector and
//              the chosen table's symbol counts;
//   warp 4     one thread issues tcgen05.mma (M=128, N=256, K=16 steps) for
//              the three layers into TMEM (layer 1 -> columns 0..255,
//              layer 2 -> 256..511, layer 3 -> 0..15);
//   warp 5     one thread streams the 8 KB weight chunks of layers 1 and 2
//              through an 8-stage shared-memory ring with bulk copies (the
//              weights are stored in global memory already in the operand
//              layout, so one chunk is one contiguous copy).
// mbarriers link the roles; every wait is bounded (tc::mbar_wait) and a
// time-out ends the kernel with an error word instead of a hang.
//
// Training (k_gemm): a general C = A * B^T with bf16 operands read through
// arbitrary strides (so transposed operands need no copies), staged by all
// threads into the K-major operand layout, two-stage double buffering, one
// thread issuing tcgen05.mma, fused epilogues (bias, row scale, ReLU, ReLU
// mask, split-K atomic accumulation).
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>

#include "engine.h"
#include "selector.h"
#include "tc.cuh"

namespace bz2g {
namespace mlp {

using bf16 = __nv_bfloat16;
using namespace tc;

namespace {

__device__ __forceinline__ float bf2f(bf16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float u2f(uint32_t v) { return __uint_as_float(v); }

// ------------------------------------------------------------ weight packing
__global__ void k_pack(const float *__restrict__ P, uint8_t *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  // W1: 256 x 272, W2: 256 x 256, W3: 16 x 256, then the biases
  if (i < kHid * kInPad) {
    const int n = i / kInPad, k = i % kInPad;
    const int j = k >> 4, kk = k & 15;
    *reinterpret_cast<bf16 *>(out + kPW1 + j * kChunkBytes + kmajor_off(n, kk, 16)) =
        __float2bfloat16(P[kW1 + i]);
  } else if (i < kHid * kInPad + kHid * kHid) {
    const int e = i - kHid * kInPad;
    const int n = e / kHid, k = e % kHid;
    const int j = k >> 4, kk = k & 15;
    *reinterpret_cast<bf16 *>(out + kPW2 + j * kChunkBytes + kmajor_off(n, kk, 16)) =
        __float2bfloat16(P[kW2 + e]);
  } else if (i < kHid * kInPad + kHid * kHid + kOutPad * kHid) {
    const int e = i - kHid * kInPad - kHid * kHid;
    const int n = e / kHid, k = e % kHid;
    const int j = k >> 4, kk = k & 15;
    *reinterpret_cast<bf16 *>(out + kPW3 + j * (kOutPad * 16 * 2) + kmajor_off(n, kk, 16)) =
        __float2bfloat16(P[kW3 + e]);
  } else {
    const int e = i - (kHid * kInPad + kHid * kHid + kOutPad * kHid);
    float *bias = reinterpret_cast<float *>(out + kPBias);
    if (e < kHid) bias[e] = P[kB1 + e];
    else if (e < 2 * kHid) bias[e] = P[kB2 + e - kHid];
    else if (e < 2 * kHid + kOutPad) bias[e] = P[kB3 + e - 2 * kHid];
  }
}

__global__ void k_to_bf16(const float *__restrict__ P, bf16 *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kParams) out[i] = __float2bfloat16(P[i]);
}

// ------------------------------------------------------- fused inference
constexpr int kStages = 8;
constexpr int kSelThreads = 192;
constexpr int kComputeThreads = 128;
constexpr int kL1Steps = kInPad / 16;  // 17
constexpr int kL2Steps = kHid / 16;    // 16
constexpr int kChunksPerTile = kL1Steps + kL2Steps;

constexpr int kSAct = 0;                                         // 128 x 272 bf16
constexpr int kSRing = kSAct + kGroupTile * kInPad * 2;          // 69,632
constexpr int kSW3 = kSRing + kStages * kChunkBytes;             // 135,168
constexpr int kSBias = kSW3 + kW3Bytes;                          // 143,360
constexpr int kSSym = kSBias + kBiasBytes;                       // 145,472
constexpr int kSRf = kSSym + kGroupTile * kGroupSize * 2;        // 158,272
constexpr int kSBar = kSRf + kMaxGroups * kMaxAlpha * 4;         // 164,464
constexpr int kNBars = 2 * kStages + 8;
constexpr int kSMisc = kSBar + kNBars * 8;
constexpr int kSelSmem = kSMisc + 16;
static_assert(kSRing % 16 == 0 && kSW3 % 16 == 0 && kSBias % 16 == 0 && kSSym % 16 == 0,
              "bulk copy destinations must be 16-byte aligned");
static_assert(kSBar % 8 == 0, "mbarriers are 8-byte aligned");
static_assert(kSelSmem <= 227 * 1024, "shared memory");

// The compute warps (0-3) agree on a flag; also a barrier among them.
__device__ __forceinline__ bool compute_any(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ bool tile_active(const SlabDev &d, int gt, int *b, int *g0, int *nh) {
  const int bb = d.gt_block[gt];
  const int first = d.gt_first[gt];
  const int nsel = d.n_sel[bb];
  if (first >= nsel || !d.learned[bb]) return false;
  *b = bb;
  *g0 = first;
  *nh = min(kGroupTile, nsel - first);
  return true;
}

// Bounded wait that ignores the abort flag (used to drain in-flight copies).
__device__ __forceinline__ void mbar_drain(uint64_t *bar, uint32_t parity) {
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > 1000000000ull) return;
}

// 32 accumulator columns of one row -> scale, bias, ReLU -> bf16 -> the
// row's slice of the next layer's A operand (kt = 256).
__device__ __forceinline__ void epilogue_chunk(const uint32_t (&r)[32], float scale,
                                               const float *bias, uint8_t *act, int row,
                                               int col0) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    uint32_t w[4];
#pragma unroll
    for (int h = 0; h < 4; h++) {
      const int c = q * 8 + h * 2;
      const float a = fmaxf(fmaf(u2f(r[c]), scale, bias[col0 + c]), 0.f);
      const float b = fmaxf(fmaf(u2f(r[c + 1]), scale, bias[col0 + c + 1]), 0.f);
      w[h] = pack_bf16x2(a, b);
    }
    *reinterpret_cast<uint4 *>(act + kmajor_off(row, col0 + q * 8, kHid)) =
        make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// wait_ns bounds every wait of the kernel.  withhold != 0 (the failure-path
// check, never the pipeline) makes the weight producer issue no copy and
// signal nothing, so the waits for the weights run out.
__global__ void __launch_bounds__(kSelThreads, 1)
    k_mlp_select(SlabDev d, const uint8_t *__restrict__ packed, float *logits,
                 int32_t *rfreq_out, uint64_t wait_ns, int withhold) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t *act = sm + kSAct;
  uint8_t *ring = sm + kSRing;
  uint8_t *w3 = sm + kSW3;
  const float *b1 = reinterpret_cast<const float *>(sm + kSBias);
  const float *b2 = b1 + kHid;
  const float *b3 = b2 + kHid;
  uint16_t *sym = reinterpret_cast<uint16_t *>(sm + kSSym);
  int *rf = reinterpret_cast<int *>(sm + kSRf);
  uint64_t *bars = reinterpret_cast<uint64_t *>(sm + kSBar);
  uint64_t *full = bars, *empty = bars + kStages;
  uint64_t *wbar = bars + 2 * kStages, *xbar = wbar + 1, *h1bar = wbar + 2, *h2bar = wbar + 3;
  uint64_t *d1bar = wbar + 4, *d2bar = wbar + 5, *d3bar = wbar + 6, *fbar = wbar + 7;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + kSMisc);
  volatile int *abort_s = reinterpret_cast<volatile int *>(sm + kSMisc + 4);
  int *err = d.err;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int i = 0; i < kStages; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(wbar, 1);
    mbar_init(xbar, kComputeThreads);
    mbar_init(h1bar, kComputeThreads);
    mbar_init(h2bar, kComputeThreads);
    mbar_init(d1bar, 1);
    mbar_init(d2bar, 1);
    mbar_init(d3bar, 1);
    mbar_init(fbar, 1);
    *abort_s = 0;
    mbar_fence_init();
  }
  if (warp == 0) tmem_alloc(tslot, 512);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tbase = *tslot;

  if (warp == 5) {
    // ---------------------------------------------------- weight producer
    if (lane == 0 && !withhold) {
      mbar_expect_tx(wbar, kW3Bytes + kBiasBytes);
      bulk_g2s(w3, packed + kPW3, kW3Bytes, wbar);
      bulk_g2s(sm + kSBias, packed + kPBias, kBiasBytes, wbar);
      uint32_t q = 0;
      bool ok = true;
      for (int gt = blockIdx.x; gt < d.n_group_tiles && ok; gt += gridDim.x) {
        int b, g0, nh;
        if (!tile_active(d, gt, &b, &g0, &nh)) continue;
        for (int c = 0; c < kChunksPerTile; c++, q++) {
          const uint32_t s = q % kStages, n = q / kStages;
          if (n > 0 && !mbar_wait(&empty[s], (n - 1) & 1, abort_s, err, 1, wait_ns)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&full[s], kChunkBytes);
          const uint8_t *src = c < kL1Steps ? packed + kPW1 + c * kChunkBytes
                                            : packed + kPW2 + (c - kL1Steps) * kChunkBytes;
          bulk_g2s(ring + s * kChunkBytes, src, kChunkBytes, &full[s]);
        }
      }
      // every copy issued has landed before the CTA may exit
      mbar_drain(wbar, 0);
      for (uint32_t r = q > kStages ? q - kStages : 0; r < q; r++)
        mbar_drain(&full[r % kStages], (r / kStages) & 1);
    }
    __syncwarp();
  } else if (warp == 4) {
    // ---------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const uint32_t id_h = idesc_bf16_f32(128, kHid), id_o = idesc_bf16_f32(128, kOutPad);
      const uint32_t a0 = smem_u32(act), r0 = smem_u32(ring), w30 = smem_u32(w3);
      bool ok = mbar_wait(wbar, 0, abort_s, err, 2, wait_ns);
      uint32_t q = 0, it = 0;
      for (int gt = blockIdx.x; gt < d.n_group_tiles && ok; gt += gridDim.x) {
        int b, g0, nh;
        if (!tile_active(d, gt, &b, &g0, &nh)) continue;
        const uint32_t ph = it & 1;
        if (!(ok = mbar_wait(xbar, ph, abort_s, err, 2, wait_ns))) break;
        fence_after_sync();
        for (int j = 0; j < kL1Steps && ok; j++, q++) {
          const uint32_t s = q % kStages;
          if (!(ok = mbar_wait(&full[s], (q / kStages) & 1, abort_s, err, 2, wait_ns))) break;
          mma_bf16(tbase, desc_noswizzle(a0 + j * 256, 128, kInPad * 16),
                   desc_noswizzle(r0 + s * kChunkBytes, 128, 256), id_h, j > 0);
          mma_commit(&empty[s]);
        }
        if (!ok) break;
        mma_commit(d1bar);
        if (!(ok = mbar_wait(h1bar, ph, abort_s, err, 2, wait_ns))) break;
        fence_after_sync();
        for (int j = 0; j < kL2Steps && ok; j++, q++) {
          const uint32_t s = q % kStages;
          if (!(ok = mbar_wait(&full[s], (q / kStages) & 1, abort_s, err, 2, wait_ns))) break;
          mma_bf16(tbase + kHid, desc_noswizzle(a0 + j * 256, 128, kHid * 16),
                   desc_noswizzle(r0 + s * kChunkBytes, 128, 256), id_h, j > 0);
          mma_commit(&empty[s]);
        }
        if (!ok) break;
        mma_commit(d2bar);
        if (!(ok = mbar_wait(h2bar, ph, abort_s, err, 2, wait_ns))) break;
        fence_after_sync();
        for (int j = 0; j < kL2Steps; j++)
          mma_bf16(tbase, desc_noswizzle(a0 + j * 256, 128, kHid * 16),
                   desc_noswizzle(w30 + j * (kOutPad * 32), 128, 256), id_o, j > 0);
        mma_commit(d3bar);
        it++;
      }
      // all MMAs issued by this thread complete before TMEM is released
      mma_commit(fbar);
      mbar_drain(fbar, 0);
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------ compute warps
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    bool stop = compute_any(!mbar_wait(wbar, 0, abort_s, err, 4, wait_ns));
    uint32_t it = 0;
    for (int gt = blockIdx.x; gt < d.n_group_tiles && !stop; gt += gridDim.x) {
      int b, g0, nh;
      if (!tile_active(d, gt, &b, &g0, &nh)) continue;
      const uint32_t ph = it & 1;
      const int64_t off = d.off[b];
      const int sym0 = g0 * kGroupSize;
      const int nsym = min(d.s[b], (g0 + nh) * kGroupSize) - sym0;
      const uint16_t *src = d.rle2 + off + sym0;
      for (int i = tid; i < nsym; i += kComputeThreads) sym[i] = src[i];
      const uint4 z = make_uint4(0, 0, 0, 0);
      for (int i = tid; i < kGroupTile * kInPad * 2 / 16; i += kComputeThreads)
        reinterpret_cast<uint4 *>(act)[i] = z;
      for (int i = tid; i < kMaxGroups * kMaxAlpha; i += kComputeThreads) rf[i] = 0;
      compute_any(false);
      // counts of this thread's group: row tid of the A operand
      const int ga = tid * kGroupSize, ge = min(ga + kGroupSize, nsym);
      float inv = 0.f;
      if (ga < ge) {
        for (int i = ga; i < ge; i++) {
          const int v = sym[i];
          if (v >= kIn) continue;  // symbols are < nInUse + 2 <= 258
          bf16 *p = reinterpret_cast<bf16 *>(act + kmajor_off(tid, v, kInPad));
          *p = __float2bfloat16(bf2f(*p) + 1.0f);
        }
        inv = 1.0f / (float)(ge - ga);
      }
      fence_async_smem();
      mbar_arrive(xbar);
      // layer 1: scale by 1/size, bias, ReLU -> H1 (kt = 256) over the counts
      if ((stop = compute_any(!mbar_wait(d1bar, ph, abort_s, err, 4, wait_ns)))) break;
      fence_after_sync();
#pragma unroll 1
      for (int c = 0; c < kHid / 32; c++) {
        uint32_t r[32];
        BZ_TMEM_LD32(tbase + lane_base + c * 32, r);
        tmem_wait_ld();
        epilogue_chunk(r, inv, b1, act, tid, c * 32);
      }
      fence_async_smem();
      fence_before_sync();
      mbar_arrive(h1bar);
      // layer 2: bias, ReLU -> H2
      if ((stop = compute_any(!mbar_wait(d2bar, ph, abort_s, err, 4, wait_ns)))) break;
      fence_after_sync();
#pragma unroll 1
      for (int c = 0; c < kHid / 32; c++) {
        uint32_t r[32];
        BZ_TMEM_LD32(tbase + kHid + lane_base + c * 32, r);
        tmem_wait_ld();
        epilogue_chunk(r, 1.0f, b2, act, tid, c * 32);
      }
      fence_async_smem();
      fence_before_sync();
      mbar_arrive(h2bar);
      // layer 3: logits, first maximum over the six tables
      if ((stop = compute_any(!mbar_wait(d3bar, ph, abort_s, err, 4, wait_ns)))) break;
      fence_after_sync();
      uint32_t r[16];
      BZ_TMEM_LD16(tbase + lane_base, r);
      tmem_wait_ld();
      fence_before_sync();
      float lg[kOut];
#pragma unroll
      for (int t = 0; t < kOut; t++) lg[t] = u2f(r[t]) + b3[t];
      int best = 0;
#pragma unroll
      for (int t = 1; t < kOut; t++)
        if (lg[t] > lg[best]) best = t;
      if (ga < ge) {
        d.sel[off / 32 + g0 + tid] = (uint8_t)best;
        for (int i = ga; i < ge; i++)
          if (sym[i] < kMaxAlpha) atomicAdd(&rf[best * kMaxAlpha + sym[i]], 1);
        if (logits) {
          float *o = logits + ((int64_t)gt * kGroupTile + tid) * 8;
#pragma unroll
          for (int t = 0; t < kOut; t++) o[t] = lg[t];
        }
      }
      compute_any(false);
      int32_t *rfreq = rfreq_out + (size_t)b * kMaxGroups * kMaxAlpha;
      for (int i = tid; i < kMaxGroups * kMaxAlpha; i += kComputeThreads)
        if (rf[i]) atomicAdd(&rfreq[i], rf[i]);
      compute_any(false);
      it++;
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(tbase, 512);
  }
}

// ------------------------------------------------------------- generic GEMM
enum Epi { kEpiF32 = 0, kEpiF32Atomic = 1, kEpiReluBf16 = 2, kEpiMaskBf16 = 3 };

struct GemmArgs {
  int M, N, K, kchunk;
  const bf16 *A;
  int64_t sam, sak;
  const float *a_kscale;  // optional per-k factor applied to A while staging
  const bf16 *B;
  int64_t sbn, sbk;
  int epi;
  float *Cf;
  bf16 *Cb;
  int64_t ldc;
  const float *bias;       // per column
  const float *row_scale;  // per row
  const bf16 *mask;        // ReLU mask source (value > 0 keeps), ld = ldm
  int64_t ldm;
  int *err;
};

constexpr int kGM = 128, kGN = 128, kGK = 64;
constexpr int kGTileBytes = kGM * kGK * 2;  // 16 KB (A and B tiles alike)
constexpr int kGSmem = 4 * kGTileBytes + 64;

// 128 rows x 64 k of a strided bf16 matrix -> K-major operand tile.
__device__ __forceinline__ void stage_tile(uint8_t *dst, const bf16 *src, int64_t s_row,
                                           int64_t s_k, const float *kscale, int row0,
                                           int nrows, int k0, int kend) {
  const int tid = threadIdx.x;
  const bool vec = s_k == 1 && (s_row % 8) == 0 && ((uintptr_t)src % 16) == 0 && !kscale;
  if (vec) {
    for (int idx = tid; idx < kGM * (kGK / 8); idx += blockDim.x) {
      const int r = idx >> 3, c = idx & 7;
      const int row = row0 + r, k = k0 + c * 8;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (row < nrows) {
        if (k + 8 <= kend) {
          v = *reinterpret_cast<const uint4 *>(src + (int64_t)row * s_row + k);
        } else if (k < kend) {
          uint16_t e[8];
          for (int i = 0; i < 8; i++)
            e[i] = k + i < kend
                       ? __bfloat16_as_ushort(src[(int64_t)row * s_row + k + i])
                       : (uint16_t)0;
          v = make_uint4(e[0] | (uint32_t)e[1] << 16, e[2] | (uint32_t)e[3] << 16,
                         e[4] | (uint32_t)e[5] << 16, e[6] | (uint32_t)e[7] << 16);
        }
      }
      *reinterpret_cast<uint4 *>(dst + kmajor_off(r, c * 8, kGK)) = v;
    }
  } else {
    // neighbouring threads take neighbouring rows (coalesced when s_row == 1)
    for (int idx = tid; idx < kGM * (kGK / 8); idx += blockDim.x) {
      const int r = idx % kGM, c = idx / kGM;
      const int row = row0 + r;
      float x[8];
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int k = k0 + c * 8 + i;
        float v = 0.f;
        if (row < nrows && k < kend) {
          v = bf2f(src[(int64_t)row * s_row + (int64_t)k * s_k]);
          if (kscale) v *= kscale[k];
        }
        x[i] = v;
      }
      *reinterpret_cast<uint4 *>(dst + kmajor_off(r, c * 8, kGK)) =
          make_uint4(pack_bf16x2(x[0], x[1]), pack_bf16x2(x[2], x[3]),
                     pack_bf16x2(x[4], x[5]), pack_bf16x2(x[6], x[7]));
    }
  }
}

__global__ void __launch_bounds__(128) k_gemm(GemmArgs g) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t *sa[2] = {sm, sm + kGTileBytes};
  uint8_t *sb[2] = {sm + 2 * kGTileBytes, sm + 3 * kGTileBytes};
  uint64_t *done = reinterpret_cast<uint64_t *>(sm + 4 * kGTileBytes);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + 4 * kGTileBytes + 16);
  volatile int *abort_s = reinterpret_cast<volatile int *>(sm + 4 * kGTileBytes + 20);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kGM, n0 = blockIdx.y * kGN;
  const int kb = blockIdx.z * g.kchunk;
  const int ke = min(g.K, kb + g.kchunk);
  const int nk = ke > kb ? (ke - kb + kGK - 1) / kGK : 0;
  if (tid == 0) {
    mbar_init(&done[0], 1);
    mbar_init(&done[1], 1);
    *abort_s = 0;
    mbar_fence_init();
  }
  if (warp == 0) tmem_alloc(tslot, 128);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tbase = *tslot;
  const uint32_t idesc = idesc_bf16_f32(kGM, kGN);
  bool failed = false;
  for (int kk = 0; kk < nk; kk++) {
    const int buf = kk & 1;
    if (kk >= 2) {
      const bool ok = mbar_wait(&done[buf], ((kk - 2) >> 1) & 1, abort_s, g.err, 8);
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
    }
    const int k0 = kb + kk * kGK;
    stage_tile(sa[buf], g.A, g.sam, g.sak, g.a_kscale, m0, g.M, k0, ke);
    stage_tile(sb[buf], g.B, g.sbn, g.sbk, nullptr, n0, g.N, k0, ke);
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
      const uint32_t a = smem_u32(sa[buf]), b = smem_u32(sb[buf]);
#pragma unroll
      for (int j = 0; j < kGK / 16; j++)
        mma_bf16(tbase, desc_noswizzle(a + j * 256, 128, kGK * 16),
                 desc_noswizzle(b + j * 256, 128, kGK * 16), idesc, (kk > 0 || j > 0) ? 1u : 0u);
      mma_commit(&done[buf]);
    }
  }
  if (nk > 0 && !failed) {
    const bool ok = mbar_wait(&done[(nk - 1) & 1], ((nk - 1) >> 1) & 1, abort_s, g.err, 8);
    failed = __syncthreads_or(!ok);
  }
  fence_after_sync();
  if (!failed && !(nk == 0 && g.epi == kEpiF32Atomic)) {
    const int row = warp * 32 + lane;
    const int m = m0 + row;
    const float rs = (g.row_scale && m < g.M) ? g.row_scale[m] : 1.0f;
#pragma unroll 1
    for (int c = 0; c < kGN / 32; c++) {
      uint32_t r[32];
      if (nk > 0) {
        BZ_TMEM_LD32(tbase + ((uint32_t)(warp * 32) << 16) + c * 32, r);
        tmem_wait_ld();
      } else {
#pragma unroll
        for (int i = 0; i < 32; i++) r[i] = 0;
      }
      if (m < g.M) {
#pragma unroll 4
        for (int i = 0; i < 32; i++) {
          const int n = n0 + c * 32 + i;
          if (n >= g.N) break;
          float x = u2f(r[i]);
          const int64_t o = (int64_t)m * g.ldc + n;
          switch (g.epi) {
            case kEpiF32:
              g.Cf[o] = x * rs + (g.bias ? g.bias[n] : 0.f);
              break;
            case kEpiF32Atomic:
              atomicAdd(&g.Cf[o], x);
              break;
            case kEpiReluBf16:
              g.Cb[o] = __float2bfloat16(fmaxf(x * rs + (g.bias ? g.bias[n] : 0.f), 0.f));
              break;
            default:
              if (!(bf2f(g.mask[(int64_t)m * g.ldm + n]) > 0.f)) x = 0.f;
              g.Cb[o] = __float2bfloat16(x);
              break;
          }
        }
      }
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(tbase, 128);
  }
}

// ------------------------------------------------------------- small kernels
// One warp per group: symbol counts -> bf16 row of X, 1/size.
__global__ void k_features(const uint16_t *__restrict__ gs, int64_t G, bf16 *__restrict__ X,
                           float *__restrict__ inv) {
  __shared__ int cnt[8][kInPad];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t g = (int64_t)blockIdx.x * 8 + w; g < G; g += (int64_t)gridDim.x * 8) {
    for (int i = lane; i < kInPad; i += 32) cnt[w][i] = 0;
    __syncwarp();
    int n = 0;
    for (int i0 = 0; i0 < kGroupSize; i0 += 32) {  // uniform trip count: the ballot is warp-wide
      const int i = i0 + lane;
      const int v = i < kGroupSize ? gs[g * kGroupSize + i] : kPadSym;
      const bool ok = v != kPadSym && v < kIn;
      if (ok) atomicAdd(&cnt[w][v], 1);
      n += __popc(__ballot_sync(0xffffffffu, ok));
    }
    __syncwarp();
    uint32_t *row = reinterpret_cast<uint32_t *>(X + g * kInPad);
    for (int i = lane; i < kInPad / 2; i += 32)
      row[i] = pack_bf16x2((float)cnt[w][2 * i], (float)cnt[w][2 * i + 1]);
    if (lane == 0) inv[g] = n ? 1.0f / (float)n : 0.f;
    __syncwarp();
  }
}

// Softmax cross-entropy over the 6 logits: dZ3 = (p - onehot) / B,
// stats[0] += loss, stats[1] += correct.
__global__ void k_ce(const float *__restrict__ Z3, const uint8_t *__restrict__ y, int B,
                     bf16 *__restrict__ dZ3, float *stats) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  float loss = 0.f, corr = 0.f;
  if (row < B) {
    float z[kOut], mx = -INFINITY;
    int am = 0;
    for (int t = 0; t < kOut; t++) {
      z[t] = Z3[(int64_t)row * kOutPad + t];
      if (z[t] > mx) {
        mx = z[t];
        am = t;
      }
    }
    float se = 0.f;
    for (int t = 0; t < kOut; t++) se += expf(z[t] - mx);
    const int lab = y[row];
    loss = -(z[lab] - mx - logf(se));
    corr = am == lab ? 1.f : 0.f;
    const float invB = 1.0f / (float)B;
    for (int t = 0; t < kOutPad; t++) {
      const float gr = t < kOut ? (expf(z[t] - mx) / se - (t == lab ? 1.f : 0.f)) * invB : 0.f;
      dZ3[(int64_t)row * kOutPad + t] = __float2bfloat16(gr);
    }
  }
  for (int o = 16; o; o >>= 1) {
    loss += __shfl_xor_sync(0xffffffffu, loss, o);
    corr += __shfl_xor_sync(0xffffffffu, corr, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&stats[0], loss);
    atomicAdd(&stats[1], corr);
  }
}

// Column sums of a bf16 [B x N] matrix into out[N] (pre-zeroed).
__global__ void k_colsum(const bf16 *__restrict__ Z, int B, int N, float *out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int r0 = blockIdx.y * 512, r1 = min(B, r0 + 512);
  float s = 0.f;
  for (int r = r0; r < r1; r++) s += bf2f(Z[(int64_t)r * N + n]);
  atomicAdd(&out[n], s);
}

__global__ void k_adam(float *P, const float *G, float *m, float *v, bf16 *p16, float lr,
                       float b1, float b2, float eps, float bc1, float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  const float g = G[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float p = P[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  P[i] = p;
  p16[i] = __float2bfloat16(p);
}

// ------------------------------------------------------------ training tap
__global__ void k_tap_offsets(SlabDev d, SelectorTap t) {
  int64_t base = *t.count;
  for (int b = 0; b < d.nblocks; b++) {
    t.blk_base[b] = base;
    if (d.n_groups[b] == kMaxGroups) base += d.n_sel[b];
  }
  *t.count = base;
}

__global__ void k_tap_export(SlabDev d, SelectorTap t) {
  const int gt = blockIdx.x;
  const int b = d.gt_block[gt];
  const int g = d.gt_first[gt] + threadIdx.x;
  if (d.n_groups[b] != kMaxGroups || g >= d.n_sel[b]) return;
  const int64_t idx = t.blk_base[b] + g;
  if (idx >= t.cap) return;
  const int64_t off = d.off[b];
  const int s = d.s[b];
  const int a = g * kGroupSize;
  for (int i = 0; i < kGroupSize; i++)
    t.syms[idx * kGroupSize + i] = a + i < s ? d.rle2[off + a + i] : kPadSym;
  t.labels[idx] = d.sel[off / 32 + g];
}

int num_sms() {
  int dev = 0, n = 0;
  BZ_CUDA(cudaGetDevice(&dev));
  BZ_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  return n;
}

// Large dynamic shared memory is opted into once per device.
template <typename Kernel>
void smem_attr(Kernel k, int bytes, std::atomic<uint64_t> &done) {
  int dev = 0;
  BZ_CUDA(cudaGetDevice(&dev));
  const uint64_t bit = uint64_t(1) << (dev & 63);
  if (done.load() & bit) return;
  BZ_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done.fetch_or(bit);
}
std::atomic<uint64_t> g_gemm_attr{0}, g_select_attr{0};

void gemm(const GemmArgs &a, int ksplit, cudaStream_t st) {
  smem_attr(k_gemm, kGSmem, g_gemm_attr);
  GemmArgs g = a;
  const int chunks = (g.K + kGK - 1) / kGK;
  ksplit = std::max(1, std::min(ksplit, chunks));
  g.kchunk = ((chunks + ksplit - 1) / ksplit) * kGK;
  ksplit = (g.K + g.kchunk - 1) / g.kchunk;
  if (ksplit > 1) BZ_REQUIRE(g.epi == kEpiF32Atomic, kErrInternal, "split-K needs atomic epilogue");
  dim3 grid((g.M + kGM - 1) / kGM, (g.N + kGN - 1) / kGN, std::max(ksplit, 1));
  k_gemm<<<grid, 128, kGSmem, st>>>(g);
  BZ_LAUNCH_CHECK();
}

GemmArgs args(int M, int N, int K, const bf16 *A, int64_t sam, int64_t sak, const bf16 *B,
              int64_t sbn, int64_t sbk, int *err) {
  GemmArgs g{};
  g.M = M;
  g.N = N;
  g.K = K;
  g.A = A;
  g.sam = sam;
  g.sak = sak;
  g.B = B;
  g.sbn = sbn;
  g.sbk = sbk;
  g.err = err;
  return g;
}

// Split factor for the weight-gradient GEMMs (K = batch): about two waves.
int ksplit_for(int tiles, int K) {
  const int want = std::max(1, 2 * num_sms() / std::max(tiles, 1));
  return std::min(want, std::max(1, K / 512));
}

}  // namespace

void pack(const float *params, uint8_t *packed, cudaStream_t st) {
  const int n = kHid * kInPad + kHid * kHid + kOutPad * kHid + 2 * kHid + kOutPad;
  k_pack<<<(n + 255) / 256, 256, 0, st>>>(params, packed);
  BZ_LAUNCH_CHECK();
}

void to_bf16(const float *params, bf16 *out, cudaStream_t st) {
  k_to_bf16<<<(kParams + 255) / 256, 256, 0, st>>>(params, out);
  BZ_LAUNCH_CHECK();
}

void launch_select(const SlabDev &d, const uint8_t *packed, float *logits, int *err,
                   int32_t *rfreq, cudaStream_t st, uint64_t wait_ns, int withhold) {
  smem_attr(k_mlp_select, kSelSmem, g_select_attr);
  if (d.n_group_tiles <= 0) return;
  SlabDev dd = d;
  if (err) dd.err = err;
  const int grid = std::min(d.n_group_tiles, num_sms());
  k_mlp_select<<<grid, kSelThreads, kSelSmem, st>>>(dd, packed, logits, rfreq ? rfreq : d.rfreq,
                                                    wait_ns, withhold);
  BZ_LAUNCH_CHECK();
}

void tap_groups(const SlabDev &d, const SelectorTap &t, cudaStream_t st) {
  k_tap_offsets<<<1, 1, 0, st>>>(d, t);
  BZ_LAUNCH_CHECK();
  if (d.n_group_tiles <= 0) return;
  k_tap_export<<<d.n_group_tiles, kGroupTile, 0, st>>>(d, t);
  BZ_LAUNCH_CHECK();
}

void features(const uint16_t *gsyms, int64_t G, bf16 *X, float *inv, cudaStream_t st) {
  if (G <= 0) return;
  const int64_t blocks = std::min<int64_t>((G + 7) / 8, 8 * num_sms());
  k_features<<<(int)blocks, 256, 0, st>>>(gsyms, G, X, inv);
  BZ_LAUNCH_CHECK();
}

void forward(const bf16 *p16, const float *P, const Batch &b, int *err, cudaStream_t st) {
  // H1 = relu((X W1^T) / size + b1)
  GemmArgs g = args(b.B, kHid, kInPad, b.X, kInPad, 1, p16 + kW1, kInPad, 1, err);
  g.epi = kEpiReluBf16;
  g.Cb = b.H1;
  g.ldc = kHid;
  g.bias = P + kB1;
  g.row_scale = b.inv;
  gemm(g, 1, st);
  // H2 = relu(H1 W2^T + b2)
  g = args(b.B, kHid, kHid, b.H1, kHid, 1, p16 + kW2, kHid, 1, err);
  g.epi = kEpiReluBf16;
  g.Cb = b.H2;
  g.ldc = kHid;
  g.bias = P + kB2;
  gemm(g, 1, st);
  // Z3 = H2 W3^T + b3
  g = args(b.B, kOutPad, kHid, b.H2, kHid, 1, p16 + kW3, kHid, 1, err);
  g.epi = kEpiF32;
  g.Cf = b.Z3;
  g.ldc = kOutPad;
  g.bias = P + kB3;
  gemm(g, 1, st);
}

void grads(const bf16 *p16, const float *P, const Batch &b, float *grad, int *err,
           cudaStream_t st) {
  BZ_REQUIRE(b.B > 0 && b.B % 128 == 0, kErrArg, "batch must be a positive multiple of 128");
  forward(p16, P, b, err, st);
  BZ_CUDA(cudaMemsetAsync(grad, 0, sizeof(float) * kParams, st));
  BZ_CUDA(cudaMemsetAsync(b.stats, 0, sizeof(float) * 2, st));
  k_ce<<<(b.B + 255) / 256, 256, 0, st>>>(b.Z3, b.labels, b.B, b.dZ3, b.stats);
  BZ_LAUNCH_CHECK();
  // dW3 = dZ3^T H2 (K = batch)
  GemmArgs g = args(kOutPad, kHid, b.B, b.dZ3, 1, kOutPad, b.H2, 1, kHid, err);
  g.epi = kEpiF32Atomic;
  g.Cf = grad + kW3;
  g.ldc = kHid;
  gemm(g, ksplit_for(2, b.B), st);
  // db3
  k_colsum<<<dim3(1, (b.B + 511) / 512), 128, 0, st>>>(b.dZ3, b.B, kOutPad, grad + kB3);
  BZ_LAUNCH_CHECK();
  // dZ2 = (dZ3 W3) * [H2 > 0]
  g = args(b.B, kHid, kOutPad, b.dZ3, kOutPad, 1, p16 + kW3, 1, kHid, err);
  g.epi = kEpiMaskBf16;
  g.Cb = b.dZ2;
  g.ldc = kHid;
  g.mask = b.H2;
  g.ldm = kHid;
  gemm(g, 1, st);
  // dW2 = dZ2^T H1
  g = args(kHid, kHid, b.B, b.dZ2, 1, kHid, b.H1, 1, kHid, err);
  g.epi = kEpiF32Atomic;
  g.Cf = grad + kW2;
  g.ldc = kHid;
  gemm(g, ksplit_for(4, b.B), st);
  k_colsum<<<dim3(kHid / 128, (b.B + 511) / 512), 128, 0, st>>>(b.dZ2, b.B, kHid, grad + kB2);
  BZ_LAUNCH_CHECK();
  // dZ1 = (dZ2 W2) * [H1 > 0]
  g = args(b.B, kHid, kHid, b.dZ2, kHid, 1, p16 + kW2, 1, kHid, err);
  g.epi = kEpiMaskBf16;
  g.Cb = b.dZ1;
  g.ldc = kHid;
  g.mask = b.H1;
  g.ldm = kHid;
  gemm(g, 1, st);
  // dW1 = (dZ1 / size)^T X
  g = args(kHid, kInPad, b.B, b.dZ1, 1, kHid, b.X, 1, kInPad, err);
  g.a_kscale = b.inv;
  g.epi = kEpiF32Atomic;
  g.Cf = grad + kW1;
  g.ldc = kInPad;
  gemm(g, ksplit_for(6, b.B), st);
  k_colsum<<<dim3(kHid / 128, (b.B + 511) / 512), 128, 0, st>>>(b.dZ1, b.B, kHid, grad + kB1);
  BZ_LAUNCH_CHECK();
}

void adam(float *P, const float *G, float *m, float *v, bf16 *p16, float lr, float beta1,
          float beta2, float eps, int step, cudaStream_t st) {
  const float bc1 = 1.f - powf(beta1, (float)step), bc2 = 1.f - powf(beta2, (float)step);
  k_adam<<<(kParams + 255) / 256, 256, 0, st>>>(P, G, m, v, p16, lr, beta1, beta2, eps, bc1,
                                                 bc2);
  BZ_LAUNCH_CHECK();
}

}  // namespace mlp
}  // namespace bz2g
