/* C entry points over the reference's own CPU test oracles.
 *
 * TEST INFRASTRUCTURE ONLY.  The functions declared below are defined in the
 * reference's test sources (compiled unchanged from the reference tree by
 * oracle/Makefile, target `ref`); this file only exposes them to ctypes so
 * that tests can pin the oracle restatement against them.
 *   simple_rle1_compress  tests/compression/rle1.cu:8-32
 *   simple_fbwt           tests/compression/fbwt.cu:12-24
 *   simple_fmtf           tests/compression/fmtf.cu:48-74
 *   simple_rle2_compress  tests/compression/rle2.cu:9-33
 */
#include <cstdint>
#include <cstring>

int simple_rle1_compress(uint8_t *in, int in_len, uint8_t *&out);
void simple_fbwt(const uint8_t *in, int in_len, int *&out);
void simple_fmtf(const uint8_t *in, int in_len, uint8_t *&out);
void simple_rle2_compress(const uint8_t *in, int in_len, uint16_t *&out,
                          uint32_t &out_len, int table_size);

extern "C" {
int ref_rle1(uint8_t *in, int n, uint8_t *out) {
  uint8_t *o = nullptr;
  int m = simple_rle1_compress(in, n, o);
  std::memcpy(out, o, (size_t)m);
  delete[] o;
  return m;
}
void ref_bwt(const uint8_t *in, int n, int32_t *sa) {
  int *o = nullptr;
  simple_fbwt(in, n, o);
  std::memcpy(sa, o, sizeof(int) * (size_t)n);
  delete[] o;
}
void ref_mtf_plain(const uint8_t *in, int n, uint8_t *out) {
  uint8_t *o = nullptr;
  simple_fmtf(in, n, o);
  std::memcpy(out, o, (size_t)n);
  delete[] o;
}
int ref_rle2(const uint8_t *in, int n, int table_size, uint16_t *out) {
  uint16_t *o = nullptr;
  uint32_t len = 0;
  simple_rle2_compress(in, n, o, len, table_size);
  std::memcpy(out, o, sizeof(uint16_t) * len);
  delete[] o;
  return (int)len;
}
}
