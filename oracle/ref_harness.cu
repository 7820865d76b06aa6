/* Driver for the reference's own GPU operators, used to make golden fixtures.
 *
 * TEST INFRASTRUCTURE ONLY.  Linked against the reference core built from the
 * reference tree by oracle/Makefile (target `ref`); runs on a GPU.
 *
 *   ref_harness stages <input> <block_bytes> <outdir>
 *       Per block of the input: the reference's rle1_compress, fbwt, fmtf,
 *       rle2_compress, huffman_build_trees and huffman_encode
 *       (include/compression.h:17-94), each stage's output written to
 *       <outdir>/b<k>.<stage>.  Before huffman_build_trees a 258-int buffer
 *       is allocated, zeroed and freed on the same stream, so the stream-
 *       ordered pool hands that zeroed memory to the reference's un-zeroed
 *       histogram (src/compression/huffman.cu:281-286); the scalars file
 *       records whether the histogram it used was the zeroed one.
 *   ref_harness stream <input> <level> <out.bz2>
 *       The reference's bzip2_gpu_compress (src/compression/compress.cu:184)
 *       over BZFileInputStream(10, 900000, input), as its CLI does
 *       (src/main.cpp:36-45).
 */
#include "compression.h"
#include "io.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

uint32_t bzip2_crc32(const uint8_t *data, size_t length);

#define CK(x)                                                                  \
  do {                                                                         \
    cudaError_t e_ = (x);                                                      \
    if (e_ != cudaSuccess) {                                                   \
      fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_));                 \
      exit(2);                                                                 \
    }                                                                          \
  } while (0)

static void dump(const std::string &path, const void *p, size_t n) {
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) { perror(path.c_str()); exit(3); }
  if (n) fwrite(p, 1, n, f);
  fclose(f);
}

static std::vector<uint8_t> slurp(const char *path) {
  FILE *f = fopen(path, "rb");
  if (!f) { perror(path); exit(3); }
  std::vector<uint8_t> v;
  uint8_t buf[1 << 16];
  size_t k;
  while ((k = fread(buf, 1, sizeof buf, f)) > 0) v.insert(v.end(), buf, buf + k);
  fclose(f);
  return v;
}

static int stages(const char *input, int block_bytes, const std::string &outdir) {
  std::vector<uint8_t> data = slurp(input);
  size_t nb = (data.size() + block_bytes - 1) / block_bytes;
  cudaStream_t st;
  CK(cudaStreamCreate(&st));
  FILE *sc = fopen((outdir + "/scalars.txt").c_str(), "w");
  for (size_t b = 0; b < nb; b++) {
    const uint8_t *raw = data.data() + b * (size_t)block_bytes;
    int n = (int)std::min<size_t>(block_bytes, data.size() - b * (size_t)block_bytes);
    std::string pre = outdir + "/b" + std::to_string(b);
    uint8_t *d_in;
    CK(cudaMalloc(&d_in, n));
    CK(cudaMemcpy(d_in, raw, n, cudaMemcpyHostToDevice));
    uint8_t *d_rle1 = nullptr;
    int m = rle1_compress(d_in, n, d_rle1, st);
    CK(cudaStreamSynchronize(st));
    std::vector<uint8_t> h_rle1(m);
    CK(cudaMemcpy(h_rle1.data(), d_rle1, m, cudaMemcpyDeviceToHost));
    dump(pre + ".rle1", h_rle1.data(), m);

    int *d_sa = nullptr;
    fbwt(d_rle1, m, d_sa, st);
    CK(cudaStreamSynchronize(st));
    std::vector<int> h_sa(m);
    CK(cudaMemcpy(h_sa.data(), d_sa, sizeof(int) * m, cudaMemcpyDeviceToHost));
    dump(pre + ".sa", h_sa.data(), sizeof(int) * m);

    uint8_t *d_mtf = nullptr;
    int orig_ptr = -1;
    bool present[256];
    int n_in_use = fmtf(d_rle1, d_sa, m, d_mtf, orig_ptr, present, st);
    CK(cudaStreamSynchronize(st));
    std::vector<uint8_t> h_mtf(m);
    CK(cudaMemcpy(h_mtf.data(), d_mtf, m, cudaMemcpyDeviceToHost));
    dump(pre + ".mtf", h_mtf.data(), m);
    uint8_t pres[256];
    for (int i = 0; i < 256; i++) pres[i] = present[i] ? 1 : 0;
    dump(pre + ".present", pres, 256);

    uint16_t *d_rle2;
    uint32_t *d_len;
    CK(cudaMalloc(&d_rle2, sizeof(uint16_t) * (2 * (size_t)m + 100)));
    CK(cudaMalloc(&d_len, sizeof(uint32_t)));
    rle2_compress(d_mtf, m, d_rle2, d_len, n_in_use, st);
    uint32_t s = 0;
    CK(cudaMemcpyAsync(&s, d_len, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<uint16_t> h_rle2(s);
    CK(cudaMemcpy(h_rle2.data(), d_rle2, sizeof(uint16_t) * s, cudaMemcpyDeviceToHost));
    dump(pre + ".rle2", h_rle2.data(), sizeof(uint16_t) * s);

    /* hand the histogram a zeroed block of the stream-ordered pool */
    int32_t *z;
    CK(cudaMallocAsync(&z, sizeof(int32_t) * max_alphabet_size, st));
    CK(cudaMemsetAsync(z, 0, sizeof(int32_t) * max_alphabet_size, st));
    CK(cudaFreeAsync(z, st));
    int32_t *probe;
    CK(cudaMallocAsync(&probe, sizeof(int32_t) * max_alphabet_size, st));
    int same_block = probe == z;
    CK(cudaFreeAsync(probe, st));

    uint8_t len[max_n_groups][max_alphabet_size];
    int32_t code[max_n_groups][max_alphabet_size];
    memset(len, 0, sizeof len);
    memset(code, 0, sizeof code);
    uint8_t *sel = nullptr;
    int n_groups = 0;
    int nsel = huffman_build_trees(d_rle2, (int)s, n_in_use, len, code, sel, n_groups, st);
    dump(pre + ".sel", sel, nsel);
    dump(pre + ".len", len, sizeof len);
    dump(pre + ".code", code, sizeof code);

    uint8_t *d_sel;
    CK(cudaMalloc(&d_sel, nsel));
    CK(cudaMemcpy(d_sel, sel, nsel, cudaMemcpyHostToDevice));
    uint32_t *d_enc = nullptr;
    int bits = huffman_encode(d_rle2, (int)s, n_in_use + 2, d_enc, len, code, d_sel, nsel,
                              n_groups, st);
    CK(cudaStreamSynchronize(st));
    int words = (bits + 31) / 32;
    std::vector<uint32_t> h_enc(words);
    CK(cudaMemcpy(h_enc.data(), d_enc, sizeof(uint32_t) * words, cudaMemcpyDeviceToHost));
    dump(pre + ".payload", h_enc.data(), sizeof(uint32_t) * words);

    uint32_t crc = bzip2_crc32(raw, n);
    fprintf(sc, "%zu n=%d m=%d crc=%u n_in_use=%d orig_ptr=%d s=%u n_groups=%d nsel=%d bits=%d zeroed_hist=%d\n",
            b, n, m, crc, n_in_use, orig_ptr, s, n_groups, nsel, bits, same_block);
    delete[] sel;
    CK(cudaFree(d_in));
    CK(cudaFree(d_rle1));
    CK(cudaFree(d_sa));
    CK(cudaFree(d_mtf));
    CK(cudaFree(d_rle2));
    CK(cudaFree(d_len));
    CK(cudaFree(d_sel));
    CK(cudaFree(d_enc));
  }
  fclose(sc);
  CK(cudaStreamDestroy(st));
  return 0;
}

static int stream(const char *input, int level, const char *out_path) {
  BZFileInputStream in(10, 900000, std::string(input));
  std::vector<uint8_t> out;
  bzip2_gpu_compress(in, level, out);
  dump(out_path, out.data(), out.size());
  return 0;
}

int main(int argc, char **argv) {
  if (argc == 5 && !strcmp(argv[1], "stages")) return stages(argv[2], atoi(argv[3]), argv[4]);
  if (argc == 5 && !strcmp(argv[1], "stream")) return stream(argv[2], atoi(argv[3]), argv[4]);
  fprintf(stderr, "usage: ref_harness stages <in> <block_bytes> <outdir> | stream <in> <level> <out>\n");
  return 1;
}
