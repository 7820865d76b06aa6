// Learned table selector (no counterpart in the reference): an MLP
// 258 -> 256 -> 256 -> 6 (ReLU) over the symbol histogram of each 50-symbol
// group predicts the Huffman table that bzip2's iterative selector
// (src/compression/huffman.cu:188-243,304-323 of the reference) would assign.
// The learned form runs: MLP assignment -> code lengths -> one exact
// selection pass -> code lengths -> canonical codes.  Blocks with fewer than
// six tables keep the plain selector.
//
// Parameters, fp32, one flat array (row-major, zero padding):
//   W1 [256 x 272]  (inputs 258..271 are padding)   b1 [256]
//   W2 [256 x 256]                                   b2 [256]
//   W3 [16 x 256]   (outputs 6..15 are padding)      b3 [16]
// Layer 1 sees the group's symbol counts; its pre-activation is scaled by
// 1 / (symbols in the group), i.e. it sees the normalised histogram.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace bz2g {

struct SlabDev;

namespace mlp {

constexpr int kIn = 258, kInPad = 272, kHid = 256, kOut = 6, kOutPad = 16;
constexpr int kW1 = 0;
constexpr int kB1 = kW1 + kHid * kInPad;
constexpr int kW2 = kB1 + kHid;
constexpr int kB2 = kW2 + kHid * kHid;
constexpr int kW3 = kB2 + kHid;
constexpr int kB3 = kW3 + kOutPad * kHid;
constexpr int kParams = kB3 + kOutPad;  // 139,792

// Inference copy of the weights: bf16 in 16-column K-chunks laid out as the
// tensor-core operand (see tc.cuh), then the fp32 biases.
constexpr int kChunkBytes = kHid * 16 * 2;                 // 8192
constexpr int kW1Chunks = kInPad / 16;                      // 17
constexpr int kW2Chunks = kHid / 16;                        // 16
constexpr int kPW1 = 0;
constexpr int kPW2 = kPW1 + kW1Chunks * kChunkBytes;        // 139,264
constexpr int kPW3 = kPW2 + kW2Chunks * kChunkBytes;        // 270,336
constexpr int kW3Bytes = kOutPad * kHid * 2;                // 8192
constexpr int kPBias = kPW3 + kW3Bytes;                     // 278,528
constexpr int kBiasBytes = (kHid + kHid + kOutPad) * 4;     // 2112
constexpr int kPackedBytes = kPBias + kBiasBytes;           // 280,640

// Group symbols of the training set: kGroupSize uint16 per group, entries
// past the group's end are kPadSym.
constexpr uint16_t kPadSym = 0xFFFF;

// fp32 params -> packed inference copy (device, kPackedBytes).
void pack(const float *params, uint8_t *packed, cudaStream_t st);
// fp32 params -> bf16 copy (same flat layout).
void to_bf16(const float *params, __nv_bfloat16 *out, cudaStream_t st);

// Learned selection over the slab's blocks with d.learned[b] != 0: writes
// d.sel and adds the chosen tables' symbol counts into rfreq (nullptr:
// d.rfreq; same layout).  logits (optional, debugging and tests): per group
// tile, 128 rows x 8 floats.  err: device word (nullptr: d.err), nonzero if a
// wait inside the kernel timed out.  wait_ns bounds each wait; withhold != 0
// (failure-path check only) keeps the weight producer from issuing anything,
// so the waits for the weights run out and the kernel returns with err set.
void launch_select(const SlabDev &d, const uint8_t *packed, float *logits, int *err,
                   int32_t *rfreq, cudaStream_t st, uint64_t wait_ns = 2000000000ull,
                   int withhold = 0);

// ---------------------------------------------------------------- training
// Training-set tap of the compression pipeline: for every block with six
// tables, its groups' symbols (padded with kPadSym) and the plain selector's
// final choice, appended in slab order (blk_base: device scratch, one entry
// per slab block).  Groups past cap are counted but not written.
struct SelectorTap {
  uint16_t *syms;     // [cap x kGroupSize]
  uint8_t *labels;    // [cap]
  int64_t cap;
  int64_t *count;     // device counter
  int64_t *blk_base;  // device [max slab blocks]
};
void tap_groups(const SlabDev &d, const SelectorTap &t, cudaStream_t st);

// Features of G groups (G a multiple of 128): counts as bf16 [G x 272] and
// 1 / (symbols in the group) [G].
void features(const uint16_t *gsyms, int64_t G, __nv_bfloat16 *X, float *inv, cudaStream_t st);

// Work buffers of one training batch of B groups (B a multiple of 128).
struct Batch {
  int B;
  const __nv_bfloat16 *X;  // [B x 272]
  const float *inv;        // [B]
  const uint8_t *labels;   // [B]
  __nv_bfloat16 *H1, *H2;  // [B x 256]
  float *Z3;               // [B x 16]
  __nv_bfloat16 *dZ3;      // [B x 16]
  __nv_bfloat16 *dZ2, *dZ1;// [B x 256]
  float *stats;            // [2]: summed cross-entropy, correct predictions
};

// Loss and gradients (fp32 flat, kParams; overwritten) of the mean
// cross-entropy over the batch, from the bf16 copy of the parameters.
void grads(const __nv_bfloat16 *p16, const float *params, const Batch &b, float *grad,
           int *err, cudaStream_t st);
// Forward only: logits Z3 [B x 16] (and H1, H2).
void forward(const __nv_bfloat16 *p16, const float *params, const Batch &b, int *err,
             cudaStream_t st);
// Adam step on the fp32 parameters; refreshes the bf16 copy.
void adam(float *params, const float *grad, float *m, float *v, __nv_bfloat16 *p16, float lr,
          float beta1, float beta2, float eps, int step, cudaStream_t st);

}  // namespace mlp
}  // namespace bz2g
