/*
 * bz2g.h -- C-ABI of bzip2gpu-b200, the B200 (sm_100a) implementation of the
 * bzip2gpu compression path.
 *
 * Plain pointers and sizes only.  "d_" arguments are device pointers on the
 * current CUDA device; `stream` is a cudaStream_t (NULL = legacy default
 * stream).  Every function returns BZ2G_OK or an error code; the message of
 * the last error on the calling thread is bz2g_last_error().  Functions that
 * return host-visible results (lengths, origPtr, tables) synchronise `stream`
 * before returning, as the reference's do.
 *
 * Each declaration names the reference interface it replaces (paths are
 * within SebastianBoteroLeonik/bzip2gpu).
 */
#ifndef BZ2G_H
#define BZ2G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BZ2G_OK 0
#define BZ2G_ERR_CUDA 1
#define BZ2G_ERR_ARG 2
#define BZ2G_ERR_ALLOC 3
#define BZ2G_ERR_INTERNAL 4
#define BZ2G_ERR_TOO_LARGE 5
#define BZ2G_ERR_TIMEOUT 6 /* a bounded wait inside a kernel ran out */

#define BZ2G_MAX_GROUPS 6  /* include/compression.h:65 max_n_groups */
#define BZ2G_MAX_ALPHA 258 /* include/compression.h:66 max_alphabet_size */

const char *bz2g_last_error(void);
int bz2g_version(void);

/* ----------------------------------------------------------- whole stream */

/* block_bytes value selecting bzip2 1.0.8's block format instead of the
 * reference's: runs cut at 255 (not 259) and blocks cut where their RLE1
 * output reaches 100000 * level - 19 bytes, as libbz2 cuts them.  The stream
 * is then byte-identical to libbz2's at the same level, except that a block
 * whose RLE1 output is periodic (equal rotations) may carry another origPtr
 * among the equal rotations, which decodes the same.  The split walks the
 * whole input, so in this mode a host input is first copied to device memory
 * whole (it must fit there; the reference format streams slab by slab).
 * No counterpart in the
 * reference, whose TODO.md:38-40 lists the split as missing and which cuts
 * 900000 raw bytes for every level, src/main.cpp:26,36. */
#define BZ2G_BZIP2_BLOCKS (-1)

/* The block ends (raw offsets, ascending, the last one n) of bzip2 1.0.8's
 * split of n device bytes at `level`: *count blocks, the first min(count, cap)
 * ends stored in host array ends.  bz2g_bzip2_split_bound gives a sufficient
 * cap.  stream: a cudaStream_t (NULL: the legacy default stream). */
int bz2g_bzip2_split(const uint8_t *d_in, size_t n, int level, int64_t *ends, size_t cap,
                     size_t *count, void *stream);
size_t bz2g_bzip2_split_bound(size_t n, int level);

/* Compress n host bytes into a complete .bz2 stream: header "BZh" + level
 * digit, one block per block_bytes raw bytes (the reference always splits at
 * its input buffer size, 900000) or bzip2's blocks (BZ2G_BZIP2_BLOCKS),
 * end-of-stream marker and combined CRC.
 * *out is allocated here (release with bz2g_free).  Empty input gives the
 * 14-byte empty stream.
 * Replaces: bzip2_gpu_compress(BZFileInputStream&, int n, std::vector<uint8_t>&)
 *           include/compression.h:86-87, src/compression/compress.cu:184-378 */
int bz2g_compress(const uint8_t *in, size_t n, int level, int block_bytes, uint8_t **out,
                  size_t *out_len);

/* As bz2g_compress with the input already in device memory. */
int bz2g_compress_device(const uint8_t *d_in, size_t n, int level, int block_bytes,
                         uint8_t **out, size_t *out_len);

/* As bz2g_compress into a caller buffer of `cap` bytes (BZ2G_ERR_TOO_LARGE if
 * it does not fit; bz2g_compress_bound gives a sufficient size). */
int bz2g_compress_into(const uint8_t *in, size_t n, int level, int block_bytes, uint8_t *out,
                       size_t cap, size_t *out_len);
/* As bz2g_compress_device into a caller host buffer (page-locked memory
 * receives the device copies directly). */
int bz2g_compress_device_into(const uint8_t *d_in, size_t n, int level, int block_bytes,
                              uint8_t *out, size_t cap, size_t *out_len);
size_t bz2g_compress_bound(size_t n, int block_bytes);
void bz2g_free(void *p);

/* Batched form: `count` independent inputs, each compressed into its own
 * .bz2 stream (header digit levels[i], blocks of block_bytes[i] raw bytes,
 * or levels[i] * 100000 when block_bytes is NULL or the entry is 0).  All
 * blocks of all inputs share the GPU in one length-ordered queue; stream i is
 * written to out[offsets[i], offsets[i+1]) and equals bz2g_compress of input
 * i alone.  inputs are host pointers, or device pointers if on_device.
 * No counterpart in the reference (it compresses one stream per call,
 * include/compression.h:86-87). */
int bz2g_compress_batch(int count, const uint8_t *const *inputs, const size_t *sizes,
                        const int *levels, const int *block_bytes, int on_device, uint8_t *out,
                        size_t cap, size_t *offsets);
size_t bz2g_compress_batch_bound(int count, const size_t *sizes, const int *levels,
                                 const int *block_bytes);

/* Engine shape used by the whole-stream calls on this thread's device:
 * blocks per slab and worker streams (default 384 and 4).  0 keeps the
 * current value.  Each worker's workspace takes about 56 MB of device memory
 * per 900,000-byte block it holds (21.5 GB at 384 blocks) and is allocated when
 * a call first needs it: a call of k blocks takes room for min(k,
 * slab_blocks) blocks per worker, and a later, larger call grows it (at least
 * doubling, at most to slab_blocks); it is kept until the shape changes.
 * bz2g_get_engine: the current shape. */
int bz2g_set_engine(int slab_blocks, int workers);
int bz2g_get_engine(int *slab_blocks, int *workers);
/* Batched-form tuning (no counterpart in the reference; the table that
 * bzip2gpu_b200/autotune.py measures and commits): entry i says that a slab
 * whose longest block has at most max_block_len[i] raw bytes takes up to
 * slab_blocks[i] blocks (at most 1024, and within the engine's memory per
 * slab), and that a batch whose byte-weighted median block falls in entry i
 * runs on up to workers[i] worker streams.  n = 0 restores the engine's own
 * shape (bz2g_set_engine).  Outputs are identical whatever the tuning. */
int bz2g_set_batch_tuning(int n, const int *max_block_len, const int *slab_blocks,
                          const int *workers);

/* Measurement (no counterpart in the reference, which only prints wall-clock
 * Stopwatch lines, include/stopwatch.h:12-42).  bz2g_set_timing(1) records
 * CUDA events around every stage of the following whole-stream calls.
 * bz2g_last_stats fills out[0..n) with, for the last whole-stream call on
 * this thread: blocks, sum n, sum m, sum A, sum s, sum groups, payload bits,
 * then device ms of RLE1+CRC, BWT, MTF, RLE2, Huffman, sizes, placement,
 * then the radix-scatter kernel's timed launches, their summed device ms and
 * their algorithmic bytes (items read + written), then the blocks whose
 * tables came from the learned selector and the blocks with six tables;
 * returns the field count.
 * bz2g_launch_count: kernels launched by this library since it was loaded. */
int bz2g_set_timing(int on);
int bz2g_last_stats(double *out, int n);
/* Per BWT round of the last whole-stream call with timing on, summed over its
 * slabs: out[3r] = r, out[3r+1] = rotations the HBM byte model charges to the
 * round, out[3r+2] = device milliseconds.  Round 0 is the first sort by 4-byte
 * prefixes (it stands for the reference's doubling rounds with shift 1 and 2,
 * src/compression/fbwt.cu:66-95); round r >= 1 is the doubling round with
 * shift 4 * 2^(r-1), charged with the rotations still in groups of two or
 * more when it starts.  Returns the number of rounds. */
int bz2g_last_round_stats(double *out, int n);
int64_t bz2g_launch_count(void);

/* ------------------------------------------------------------- per stage */

/* Upper bound of the RLE1 output of n bytes (n + n/4 + 8). */
size_t bz2g_rle1_bound(size_t n);

/* RLE1 with runs cut at 259; d_out holds bz2g_rle1_bound(n) bytes; *m gets
 * the output length.
 * Replaces: int rle1_compress(const uint8_t*, int, uint8_t*&, cudaStream_t)
 *           include/compression.h:17-18, src/compression/rle1.cu:60-113 */
int bz2g_rle1(const uint8_t *d_in, int n, uint8_t *d_out, int *m, void *stream);

/* Same result as bz2g_rle1, allocating nothing: no counterpart in the
 * reference.  For callers that may not allocate device memory while they run
 * (a service that reserves its whole memory budget at start-up, or a hot path
 * that must not take cudaMalloc / cudaFree's implicit synchronisation).  Its
 * scratch is one static device array in the library (about 1 MiB, held by
 * every GPU that loads the library until the process exits), so n is at
 * most 1048576 bytes (BZ2G_ERR_TOO_LARGE beyond, with a message in
 * bz2g_last_error).  d_out holds bz2g_rle1_bound(n) bytes.  The first call on
 * a device (or on a device context created anew) looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture begins.  Each call waits for its stream to finish the work before
 * it returns, since *m is read back to the host.  Calls share the array:
 * calls that overlap on the GPU (for example from two host threads on two
 * streams) race, so serialise them. */
int bz2g_rle1_noalloc(const uint8_t *d_in, int n, uint8_t *d_out, int *m, void *stream);

/* bzip2 block CRC of n device bytes.
 * Replaces: uint32_t bzip2_crc32(const uint8_t*, size_t)
 *           src/compression/crc32.h:7-8, src/compression/crc32.cpp:22-29 */
int bz2g_crc32(const uint8_t *d_in, size_t n, uint32_t *crc, void *stream);

/* Suffix array of the cyclic rotations of d_in[0..m) (equal rotations in
 * index order) into d_sa[0..m).
 * Replaces: void fbwt(const uint8_t*, int, int*&, cudaStream_t)
 *           include/compression.h:81, src/compression/fbwt.cu:47-106 */
int bz2g_bwt(const uint8_t *d_in, int m, int32_t *d_sa, void *stream);

/* Move-to-front of L[i] = d_orig[(d_sa[i]-1) mod m] with the list starting as
 * the ascending in-use symbols; *orig_ptr = i with d_sa[i] == 0; present
 * (256 bytes, may be NULL) gets 0/1 per byte value; *n_in_use the count.
 * Replaces: int fmtf(const uint8_t*, const int*, int, uint8_t*&, int&, bool*,
 *           cudaStream_t) include/compression.h:53-55, src/compression/fmtf.cu:147-230 */
int bz2g_mtf(const uint8_t *d_orig, const int32_t *d_sa, int m, uint8_t *d_out, int *orig_ptr,
             uint8_t *present, int *n_in_use, void *stream);

/* Ascending byte values present in d_in[0..n) into table (256 bytes).
 * Replaces: int make_symbols_table(const uint8_t*, int, uint8_t*&, cudaStream_t)
 *           include/compression.h:43-44, src/compression/fmtf.cu:114-140 */
int bz2g_symbols_table(const uint8_t *d_in, int n, uint8_t *table, int *count, void *stream);

/* RUNA/RUNB coding of MTF values, EOB = table_size + 1.  d_out holds m + 1
 * symbols; *d_out_len (device) gets the count.  m == 0 writes 0 and no EOB.
 * Replaces: void rle2_compress(const uint8_t*, int, uint16_t*, uint32_t*, int,
 *           cudaStream_t) include/compression.h:30-31, src/compression/rle2.cu:99-158 */
int bz2g_rle2(const uint8_t *d_in, int m, int table_size, uint16_t *d_out, uint32_t *d_out_len,
              void *stream);

/* Table selection (4 refinement passes), code lengths (max 17) and canonical
 * codes for s symbols over nInUse + 2 values.  len / code are host arrays
 * [6][258] (rows >= *n_groups of code untouched); selectors is a host array
 * of ceil(s/50) bytes.
 * Replaces: int huffman_build_trees(uint16_t*, int, int, uint8_t[6][258],
 *           int32_t[6][258], uint8_t*&, int&, cudaStream_t)
 *           include/compression.h:67-72, src/compression/huffman.cu:256-364 */
int bz2g_huffman_build(const uint16_t *d_syms, int s, int n_in_use, uint8_t *len, int32_t *code,
                       uint8_t *selectors, int *n_selectors, int *n_groups, void *stream);

/* MSB-first packing of the codes into 32-bit words (word w = bits
 * [32w, 32w+32), first bit in the MSB).  d_words must hold
 * (17 * s + 31) / 32 words; *bits gets the bit count.
 * Replaces: int huffman_encode(uint16_t*, int, int, uint32_t*&, uint8_t[6][258],
 *           int32_t[6][258], uint8_t*, int32_t, int, cudaStream_t)
 *           include/compression.h:89-94, src/compression/huffman_encode.cu:75-143 */
int bz2g_huffman_encode(const uint16_t *d_syms, int s, const uint8_t *len, const int32_t *code,
                        const uint8_t *d_selectors, int n_selectors, int n_groups,
                        uint32_t *d_words, int64_t *bits, void *stream);

/* Symbol histogram over 258 values (freqs is a device array the caller has
 * zeroed, as the reference's own test does).
 * Replaces: __global__ count_frequencies(uint16_t*, int, int*)
 *           src/compression/huffman.cu:126-133 */
int bz2g_count_frequencies(const uint16_t *d_syms, int s, int32_t *d_freqs, void *stream);

/* ----------------------------------------------------------- decompression */
/* No counterpart in the reference (its TODO.md:28-34 lists it as missing).
 * Decodes a .bz2 stream (or concatenated streams) on the GPU, blocks in
 * parallel; every block CRC and the stream CRC are checked.  Accepts the
 * reference's streams whose blocks exceed the header digit's size.  *out is
 * malloc'ed (release with bz2g_free).  A malformed stream gives an error
 * status. */
int bz2g_decompress(const uint8_t *in, size_t n, uint8_t **out, size_t *out_len);
int bz2g_decompress_device(const uint8_t *d_in, size_t n, uint8_t **out, size_t *out_len);
/* As above into a caller buffer of `cap` bytes, host (pinned or pageable) or
 * device memory; *out_len = decoded bytes.  BZ2G_ERR_TOO_LARGE if they do not
 * fit (the buffer then holds a prefix of the output). */
int bz2g_decompress_into(const uint8_t *in, size_t n, uint8_t *out, size_t cap,
                         size_t *out_len);
int bz2g_decompress_device_into(const uint8_t *d_in, size_t n, uint8_t *d_out, size_t cap,
                                size_t *out_len);

/* ------------------------------------------------------------ file streams */
/* A file (NULL: standard input) compressed to a .bz2 file (NULL: standard
 * output) with bounded host memory: a reader thread keeps a ring of pinned
 * 900,000-byte chunks ahead, groups of group_blocks blocks (0: 384) compress
 * on the GPU while the next group is read, and each group's bytes are written
 * as it finishes.  Blocks are 900,000 raw bytes and the header digit is the
 * level, as in the reference's CLI (src/main.cpp:26-45).  A missing input
 * file is an error (the reference waits forever).
 * Replaces: main's loop over BZFileInputStream + bzip2_gpu_compress
 * (src/main.cpp:26-58). */
int bz2g_compress_file(const char *in_path, const char *out_path, int level, int group_blocks);

/* ------------------------------------------- one stream over several GPUs */
/* No counterpart in the reference (one GPU).  Blocks are independent, so a
 * stream is cut into parts of whole blocks, each compressed on its own GPU;
 * the only exchange is each part's bit count and CRC fold, then the parts are
 * spliced at their bit offsets.
 * bz2g_compress_part: the blocks of in[0..n) (block_bytes raw bytes each;
 * on_device != 0: in is device memory) compressed into a part starting at
 * bit 0 of d_part (device memory of the current device, cap bytes, at least
 * bz2g_part_bound(n, block_bytes)); no stream header, no end-of-stream
 * marker; the bytes after the part up to the next 4-byte boundary are zero.
 * *bits: the part's bit count; *crc_fold: its blocks' CRCs folded as the
 * stream CRC is (rotate left by 1, xor) starting from 0; *nblocks: its blocks.
 * A stream = header + parts in order + marker; its CRC folds the parts'
 * folds: crc = rotl(crc, nblocks_r) ^ crc_fold_r. */
size_t bz2g_part_bound(size_t n, int block_bytes);
int bz2g_compress_part(const uint8_t *in, size_t n, int block_bytes, int on_device,
                       uint8_t *d_part, size_t cap, int64_t *bits, uint32_t *crc_fold,
                       int *nblocks);
/* The parts (device memory of the current device, each 4-byte aligned) spliced
 * after 'BZh' + level into one .bz2 stream in host memory out[0..cap), with
 * the end-of-stream marker and the combined CRC; *out_len: its length. */
int bz2g_assemble(int nparts, const uint8_t *const *d_parts, const int64_t *bits,
                  const uint32_t *crc_folds, const int *nblocks, int level, uint8_t *out,
                  size_t cap, size_t *out_len);

/* ------------------------------------------------- learned table selector */
/* No counterpart in the reference.  An MLP 258 -> 256 -> 256 -> 6 (ReLU, bf16
 * weights, fp32 accumulation on the tensor cores) over each 50-symbol
 * group's symbol histogram predicts the table the reference's iterative
 * selector (src/compression/huffman.cu:188-243,304-323) would choose.  With
 * the learned selector on, a block with six tables takes: MLP assignment ->
 * code lengths -> one exact selection pass -> code lengths -> codes, unless
 * the plain selector's first two passes (run beside it as the judge) predict
 * a smaller block, in which case it takes those; blocks with fewer tables
 * keep the plain selector.  Streams stay valid bzip2; they are no longer
 * byte-identical to the reference's.
 *
 * Parameters: BZ2G_SELECTOR_PARAMS floats, one flat array, row-major with
 * zero padding: W1[256][272] b1[256] W2[256][256] b2[256] W3[16][256] b3[16]
 * (W1 columns 258..271 and W3 rows 6..15 are padding).  Layer 1's
 * pre-activation is (counts . W1) / (symbols in the group) + b1. */
#define BZ2G_SELECTOR_PARAMS 139792

/* Loads parameters (host fp32) for the current device. */
int bz2g_selector_load(const float *params, size_t count);
/* Selector of the whole-stream calls: 0 = plain (default, the reference's),
 * 1 = learned, 2 = plain with a single selection pass (the baseline the
 * learned form is measured against). */
int bz2g_set_selector(int mode);
int bz2g_get_selector(void);

/* The fused tensor-core selector over s symbols treated as one six-table
 * block: logits (device, ceil(s/50) x 6 floats) and choices (device,
 * ceil(s/50) bytes); d_params: device fp32 parameters. */
int bz2g_selector_logits(const uint16_t *d_syms, int s, const float *d_params, float *d_logits,
                         uint8_t *d_sel, void *stream);

/* Failure-path check of the tensor-core selector kernel (no counterpart in
 * the reference, which has no error path: include/utils.h:3-12).  Every wait
 * inside that kernel is bounded; a wait that runs out sets a device error
 * word, the kernel's threads leave their loops, free their tensor memory and
 * return, and the host turns the word into an error.  This runs the kernel
 * over s symbols as one six-table block with each wait limited to
 * wait_limit_ns.  withhold_weights != 0 keeps the kernel's weight producer
 * from issuing any copy, so the waits for the weights run out: the call then
 * returns BZ2G_ERR_TIMEOUT (the error word in bz2g_last_error) and the
 * device stays usable.  With withhold_weights == 0 it returns BZ2G_OK once
 * the kernel met all its waits. */
int bz2g_selector_wait_check(const uint16_t *d_syms, int s, const float *d_params,
                             uint64_t wait_limit_ns, int withhold_weights, void *stream);

/* bz2g_huffman_build with the learned selector (d_params: device fp32
 * parameters).  mlp_selectors (host, ceil(s/50) bytes, may be NULL) gets the
 * MLP's own choices before the exact pass. */
int bz2g_huffman_build_learned(const uint16_t *d_syms, int s, int n_in_use, const float *d_params,
                               uint8_t *len, int32_t *code, uint8_t *selectors,
                               uint8_t *mlp_selectors, int *n_selectors, int *n_groups,
                               void *stream);

/* Training set: the inputs (device memory) compressed as the batched form
 * does (block = 100000 * level), and for every block with six tables each
 * group's 50 symbols (0xFFFF past the group's end) and the plain selector's
 * choice, in a deterministic order.  At most cap groups are written;
 * *n_groups gets the number available. */
int bz2g_selector_dataset(int count, const uint8_t *const *d_inputs, const size_t *sizes,
                          const int *levels, uint16_t *d_group_syms, uint8_t *d_labels,
                          int64_t cap, int64_t *n_groups);

/* Training on the tensor cores.  d_X: bf16 [G][272] symbol counts, d_inv:
 * 1 / (symbols in the group); d_p16: bf16 copy of the parameters (same flat
 * layout).  Batches B are multiples of 128; d_work holds
 * bz2g_mlp_work_bytes(B) bytes. */
int bz2g_mlp_features(const uint16_t *d_group_syms, int64_t G, void *d_X, float *d_inv,
                      void *stream);
size_t bz2g_mlp_work_bytes(int B);
/* Mean cross-entropy gradients into d_grad (BZ2G_SELECTOR_PARAMS floats);
 * d_stats[0] += summed loss, d_stats[1] += correct predictions (zeroed
 * first). */
int bz2g_mlp_grads(const void *d_p16, const float *d_params, int B, const void *d_X,
                   const float *d_inv, const uint8_t *d_labels, void *d_work, float *d_grad,
                   float *d_stats, void *stream);
/* Logits (device, B x 16 floats; columns 6..15 are padding). */
int bz2g_mlp_forward(const void *d_p16, const float *d_params, int B, const void *d_X,
                     const float *d_inv, void *d_work, float *d_logits, void *stream);
int bz2g_mlp_adam(float *d_params, const float *d_grad, float *d_m, float *d_v, void *d_p16,
                  float lr, float beta1, float beta2, float eps, int step, void *stream);
int bz2g_mlp_to_bf16(const float *d_params, void *d_p16, void *stream);
/* Waits for the stream; reports a timed-out tensor-core wait of the training
 * kernels since the last call. */
int bz2g_mlp_status(void *stream);

/* ------------------------------------------------------ synthetic inputs */
/* Seeded workload generators (no counterpart in the reference, which has no
 * data generator): identical bytes on the host and the device.
 * bz2g_gen_markov: order-1 Markov source over alphabet[0..A) with
 * Dirichlet(alpha) transition rows and run starts of probability p_run and
 * length uniform in [run_min, run_max]; definition in
 * bzip2gpu_b200/csrc/gen.cu.  on_device != 0: out is a device pointer. */
int bz2g_gen_markov(uint64_t seed, const uint8_t *alphabet, int A, double alpha, double p_run,
                    int run_min, int run_max, uint8_t *out, int64_t n, int on_device,
                    void *stream);
int bz2g_gen_uniform(uint64_t seed, uint8_t *out, int64_t n, int on_device, void *stream);

#ifdef __cplusplus
}
#endif
#endif
