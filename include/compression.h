/*
 * compression.h -- drop-in C++ API of the bzip2gpu compression path,
 * implemented by libbz2gpu_b200.so on sm_100a.
 *
 * Same entry points, argument meanings, defaults and ownership as the
 * reference's include/compression.h (SebastianBoteroLeonik/bzip2gpu):
 * device outputs that the reference allocates with cudaMallocAsync /
 * cudaMalloc are allocated here the same way (release with cudaFree or
 * cudaFreeAsync); host outputs documented as new[] are new[]-allocated.
 * Errors print a message to stderr and exit(EXIT_FAILURE), like the
 * reference's CUDA_ERROR_CHECK.  Each function cites the reference
 * declaration it replaces.
 */
#ifndef BZ2GPU_B200_COMPRESSION_H
#define BZ2GPU_B200_COMPRESSION_H

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "io.h"

/* RLE1 (runs cut at 259) of in_len device bytes; *out gets a device buffer
 * holding the result; returns its length.  include/compression.h:17-18 */
int rle1_compress(const uint8_t *in, int in_len, uint8_t *&out, cudaStream_t stream = 0);

/* RLE2 of in_len MTF values into the caller's device buffer `out`
 * (capacity in_len + 1); *out_len (device) gets the symbol count; EOB is
 * table_size + 1.  include/compression.h:30-31 */
void rle2_compress(const uint8_t *in, int in_len, uint16_t *out, uint32_t *out_len,
                   int table_size, cudaStream_t stream = 0);

/* Ascending byte values present in d_in; symbols_table = new uint8_t[count].
 * Returns count.  include/compression.h:43-44 */
int make_symbols_table(const uint8_t *d_in, int d_in_len, uint8_t *&symbols_table,
                       cudaStream_t stream = 0);

/* MTF of the BWT last column of in_original under in_suffix_array; *out gets
 * a device buffer of in_len bytes; orig_ptr the row of rotation 0;
 * present_symbols (if given) 256 flags.  Returns the in-use symbol count.
 * include/compression.h:53-55 */
int fmtf(const uint8_t *in_original, const int *in_suffix_array, int in_len, uint8_t *&out,
         int &orig_ptr, bool *present_symbols = nullptr, cudaStream_t stream = 0);

constexpr int max_n_groups = 6;        /* include/compression.h:65 */
constexpr int max_alphabet_size = 258; /* include/compression.h:66 */

/* Huffman tables for data_in_len device symbols over alphabet_size in-use
 * symbols (+2 added internally); selectors = new uint8_t[returned count].
 * include/compression.h:67-72 */
int huffman_build_trees(uint16_t *device_data_in, int data_in_len, int alphabet_size,
                        uint8_t len[max_n_groups][max_alphabet_size],
                        int32_t code[max_n_groups][max_alphabet_size], uint8_t *&selectors,
                        int &n_groups, cudaStream_t stream);

/* Suffix array of the cyclic rotations of in[0..in_len); *out gets a device
 * buffer of in_len ints.  include/compression.h:81 */
void fbwt(const uint8_t *in, int in_len, int *&out, cudaStream_t stream = 0);

/* Whole .bz2 stream from the chunks of in_stream (one block per chunk),
 * header digit n; appended to out.  include/compression.h:86-87 */
void bzip2_gpu_compress(BZFileInputStream &in_stream, int n, std::vector<uint8_t> &out);

/* MSB-first packing of the codes; *dev_encoded_data gets a cudaMalloc'ed
 * word buffer; returns the bit count.  include/compression.h:89-94 */
int huffman_encode(uint16_t *dev_data_in, int data_in_len, int alphabet_size,
                   uint32_t *&dev_encoded_data, uint8_t len[max_n_groups][max_alphabet_size],
                   int32_t code[max_n_groups][max_alphabet_size], uint8_t *dev_selectors,
                   int32_t num_selectors, int n_groups, cudaStream_t stream);

/* Symbol histogram kernel, launched directly by the reference's tests
 * (tests/compression/huffman.cu:7,29); freqs must be zeroed by the caller.
 * src/compression/huffman.cu:126-133 */
__global__ void count_frequencies(uint16_t *data_in, int data_len, int *freqs);

#endif
