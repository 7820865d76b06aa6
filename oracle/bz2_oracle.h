/*
 * bz2_oracle.h -- CPU restatement of the bzip2gpu compression path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is
 * compared against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it; the product library never links or calls it.
 *
 * Every function restates one stage of the reference (SebastianBoteroLeonik/
 * bzip2gpu) and cites the file:line it follows.  Semantics are the reference's,
 * including its deviations from bzip2 1.0.8 (RLE1 runs split at 259, the block
 * split is the caller's chunk size, the header digit is the level only).
 *
 * Parity pin: the stage functions are checked against the reference's own CPU
 * test oracles compiled from the reference tree (oracle/Makefile, target
 * `ref`) on the reference tests' glibc rand() vectors, and the whole pipeline
 * against outputs of the reference GPU operators run on a B200
 * (tests/golden/, made by tests/golden/make_golden.py).
 */
#ifndef BZ2_ORACLE_H
#define BZ2_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_GROUPS 6
#define ORC_MAX_ALPHA 258
#define ORC_GROUP_SIZE 50

/* Non-reflected CRC-32 (poly 0x04C11DB7, init ~0, final ~).
 * src/compression/crc32.cpp:6-29 */
uint32_t orc_crc32(const uint8_t *data, size_t n);

/* RLE1 with runs split at 259.  out needs n + n/4 + 4 bytes.  Returns m.
 * src/compression/rle1.cu:13-58, tests/compression/rle1.cu:8-32 */
int orc_rle1(const uint8_t *in, int n, uint8_t *out);
/* The same with runs split at `cut` (255: bzip2 1.0.8). */
int orc_rle1_cut(const uint8_t *in, int n, uint8_t *out, int cut);

/* block_bytes value of orc_compress / orc_compress_bound selecting bzip2
 * 1.0.8's blocks (orc_bzip2_split) and runs split at 255.  Not a reference
 * mode: this restatement of libbz2's split is pinned to libbz2 itself. */
#define ORC_BZIP2_BLOCKS (-1)

/* bzip2 1.0.8's block split of in[0..n) at `level`: ends[k] = end offset of
 * block k (up to cap entries stored).  Returns the number of blocks. */
int64_t orc_bzip2_split(const uint8_t *in, int64_t n, int level, int64_t *ends,
                        int64_t cap);

/* Sorted cyclic rotations of in[0..m), equal rotations by index ascending.
 * src/compression/fbwt.cu:47-106, tests/compression/fbwt.cu:12-24 */
void orc_bwt(const uint8_t *in, int m, int32_t *sa);

/* Same as orc_bwt, and also returns A = sum over doubling rounds (h = 1, 2, 4 ..)
 * of the number of rotations in rank groups of size >= 2 at the start of the
 * round, and the number of rounds run before the partition became final. */
void orc_bwt_stats(const uint8_t *in, int m, int32_t *sa, int64_t *active_sum,
                   int *rounds);

/* Move-to-front over the BWT last column L[i] = orig[(sa[i]-1) mod m] with the
 * list initialised to the ascending in-use symbols of orig.  Writes origPtr
 * (first i with sa[i]==0) and present[256].  Returns nInUse.
 * src/compression/fmtf.cu:40-97,147-230, tests/compression/fmtf.cu:48-74 */
int orc_mtf(const uint8_t *orig, const int32_t *sa, int m, uint8_t *out,
            int *orig_ptr, uint8_t *present);

/* Symbol table: ascending present byte values.  Returns count.
 * src/compression/fmtf.cu:114-140 */
int orc_symbols_table(const uint8_t *in, int n, uint8_t *table);

/* RUNA/RUNB zero-run coding with v -> v+1 and EOB = table_size+1.
 * out needs m+1 entries.  Returns s.
 * src/compression/rle2.cu:11-77, tests/compression/rle2.cu:9-33 */
int orc_rle2(const uint8_t *in, int m, int table_size, uint16_t *out);

/* bzip2's length-limited Huffman code lengths (heap algorithm).
 * src/compression/huffman.cu:13-124 */
void orc_code_lengths(const int32_t *freq, uint8_t *len, int alpha_size,
                      int max_len);

/* Table selection with the reference's 4 refinement passes, code lengths and
 * canonical codes.  alphabet_size is nInUse (2 is added, as the reference
 * does).  selectors needs ceil(s/50) bytes.  Writes *n_groups.  Returns the
 * number of selectors.  Uses a zeroed symbol histogram.
 * src/compression/huffman.cu:126-364 */
/* The plain selector with `passes` selection passes (the reference's 4). */
int orc_huffman_build_passes(const uint16_t *syms, int s, int alphabet_size, int passes,
                             uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                             int32_t code[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                             uint8_t *selectors, int *n_groups_out);
int orc_huffman_build(const uint16_t *syms, int s, int alphabet_size,
                      uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                      int32_t code[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                      uint8_t *selectors, int *n_groups);

/* The learned form's passes after its first assignment sel_in (six tables):
 * code lengths from the chosen tables' counts, n_refine passes of exact
 * selection + code lengths, canonical codes.  Returns the selector count. */
int orc_huffman_refine(const uint16_t *syms, int s, int alphabet_size, const uint8_t *sel_in,
                       int n_refine, uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                       int32_t code[ORC_MAX_GROUPS][ORC_MAX_ALPHA], uint8_t *selectors);

/* The learned form given the MLP's choices, with the single-pass judge and
 * the plain fallback (*fell_back).  Returns the selector count. */
int orc_huffman_learned(const uint16_t *syms, int s, int alphabet_size, const uint8_t *sel_mlp,
                        uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                        int32_t code[ORC_MAX_GROUPS][ORC_MAX_ALPHA], uint8_t *selectors,
                        int *n_groups_out, int *fell_back);

/* Selection-dependent bits of a block: payload + unary selector MTF +
 * table deltas (src/compression/compress.cu:300-345). */
int64_t orc_coded_bits(const uint16_t *syms, int s, const uint8_t *selectors, int ng,
                       int alphabet_size, const uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA]);

/* Initial table assignment only (before refinement).
 * src/compression/huffman.cu:148-185 */
void orc_initial_assignment(int n_groups, int s, int alpha_size,
                            const int32_t *freqs,
                            uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA]);

/* MSB-first packing of the codes into 32-bit words (word w holds stream bits
 * [32w, 32w+32), first bit in the MSB).  words needs enough zeroed space.
 * Returns total bits.  src/compression/huffman_encode.cu:15-71 */
int64_t orc_encode(const uint16_t *syms, int s, const uint8_t *selectors,
                   const uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                   const int32_t code[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                   uint32_t *words);

/* Selector move-to-front over 0..n_groups-1.  src/compression/compress.cu:119-137 */
void orc_selector_mtf(const uint8_t *sel, int n_sel, int n_groups, uint8_t *out);

/* Per-block record of every stage, for stage-by-stage comparison. */
typedef struct {
  int n;             /* raw bytes */
  int m;             /* RLE1 bytes */
  int s;             /* RLE2 symbols incl. EOB */
  int n_in_use;
  int orig_ptr;
  int n_groups;
  int n_selectors;
  uint32_t crc;
  int64_t payload_bits;
  int64_t header_bits;
  int64_t active_sum; /* A, for the HBM byte model */
  uint8_t present[256];
  uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA];
  int32_t code[ORC_MAX_GROUPS][ORC_MAX_ALPHA];
} orc_block_info;

/* Run one block through every stage.  Any of the stage buffers may be NULL.
 * rle1 needs n+n/4+4, sa m ints, mtf m, rle2 m+1, selectors m/50+2. */
int orc_compress_block(const uint8_t *raw, int n, orc_block_info *info,
                       uint8_t *rle1, int32_t *sa, uint8_t *mtf, uint16_t *rle2,
                       uint8_t *selectors);

/* Whole .bz2 stream: 'BZh' + level digit, blocks of block_bytes raw bytes
 * (or bzip2's blocks: ORC_BZIP2_BLOCKS), end-of-stream marker and combined CRC.  Empty input gives the 14-byte empty
 * stream.  Returns the byte length, or -1 if cap is too small.
 * src/compression/compress.cu:184-378 */
int64_t orc_compress(const uint8_t *in, int64_t n, int level, int block_bytes,
                     uint8_t *out, int64_t cap, int threads);

/* A part of a stream (the blocks' bits from bit 0, no header, no marker) and
 * the assembly of parts into a stream; see bzip2gpu_b200/shard.py. */
int64_t orc_compress_part(const uint8_t *in, int64_t n, int block_bytes, uint8_t *out,
                          int64_t cap, int threads, int64_t *bits, uint32_t *fold);
int64_t orc_assemble(int nparts, const uint8_t *const *parts, const int64_t *bits,
                     const uint32_t *folds, const int *nblocks, int level, uint8_t *out,
                     int64_t cap);

/* Upper bound of orc_compress's output size. */
int64_t orc_compress_bound(int64_t n, int block_bytes);

#ifdef __cplusplus
}
#endif
#endif
