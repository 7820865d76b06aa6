// Drives the drop-in C++ API the way the reference's main() does
// (reference src/main.cpp:20-60): a BZFileInputStream over a file, then
// bzip2_gpu_compress(stream, level, out); writes `out` to a file.  Also
// checks the CRC functions (crc32.h) against a bitwise CRC written here.
// Test infrastructure: built and run by tests/test_gpu_reference_suite.py.
//
//   dropin_harness <input> <level> <buffer_size> <output>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "compression.h"
#include "crc32.h"
#include "io.h"

// bzip2's CRC-32 (polynomial 0x04c11db7, MSB first, init and final ~0), bit
// by bit.
static uint32_t crc_bitwise(const uint8_t *p, size_t n) {
  uint32_t c = 0xffffffffu;
  for (size_t i = 0; i < n; i++) {
    c ^= (uint32_t)p[i] << 24;
    for (int k = 0; k < 8; k++) c = (c & 0x80000000u) ? (c << 1) ^ 0x04c11db7u : c << 1;
  }
  return ~c;
}

int main(int argc, char **argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s <input> <level> <buffer_size> <output>\n", argv[0]);
    return 2;
  }
  const int level = std::atoi(argv[2]);
  const int buffer_size = std::atoi(argv[3]);
  std::vector<uint8_t> out;
  {
    BZFileInputStream in(10, buffer_size, std::string(argv[1]));
    bzip2_gpu_compress(in, level, out);
  }
  FILE *f = std::fopen(argv[4], "wb");
  if (!f || std::fwrite(out.data(), 1, out.size(), f) != out.size()) return 3;
  std::fclose(f);

  crc32_init();
  std::vector<uint8_t> probe(100003);
  for (size_t i = 0; i < probe.size(); i++) probe[i] = (uint8_t)(i * 2654435761u >> 24);
  const uint32_t got = bzip2_crc32(probe.data(), probe.size());
  const uint32_t want = crc_bitwise(probe.data(), probe.size());
  if (got != want) {
    std::fprintf(stderr, "bzip2_crc32 %08x, expected %08x\n", got, want);
    return 4;
  }
  std::printf("ok %zu bytes\n", out.size());
  return 0;
}
