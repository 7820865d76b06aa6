// CRC-32 of the bzip2 format (polynomial 0x04C11DB7, bits taken most
// significant first; src/compression/crc32.cpp of the reference) and the
// GF(2) arithmetic that combines the CRCs of separately processed pieces.
//
// crc0(D) (zero initial value, no final complement) is linear over GF(2):
//   crc0(A || B) = crc0(A) * x^(8|B|) ^ crc0(B)        (mod P)
// and the format's CRC is ~(~0 * x^(8|D|) ^ crc0(D)).
#pragma once

#include <stdint.h>

namespace bz2g {
namespace {

constexpr uint32_t kPoly = 0x04C11DB7u;

constexpr uint32_t gf_mul_c(uint32_t a, uint32_t b) {
  uint32_t r = 0;
  for (int i = 31; i >= 0; --i) {
    r = (r << 1) ^ ((r & 0x80000000u) ? kPoly : 0u);
    if ((b >> i) & 1u) r ^= a;
  }
  return r;
}
constexpr uint32_t xpow8_pow2(int i) {
  uint32_t v = 0x100u;  // x^8
  for (int k = 0; k < i; ++k) v = gf_mul_c(v, v);
  return v;
}

#define BZ_XP4(i) xpow8_pow2(i), xpow8_pow2(i + 1), xpow8_pow2(i + 2), xpow8_pow2(i + 3)
// c_xpow[i] = x^(8 * 2^i) mod P
__constant__ uint32_t c_xpow[32] = {BZ_XP4(0),  BZ_XP4(4),  BZ_XP4(8),  BZ_XP4(12),
                                    BZ_XP4(16), BZ_XP4(20), BZ_XP4(24), BZ_XP4(28)};
#undef BZ_XP4

// c_klane.v[l] = x^(8 * 16 * (255 - l)) mod P: thread l's 16 bytes sit that
// far before the end of a 4096-byte tile.
struct LaneShift {
  uint32_t v[256];
  constexpr LaneShift() : v() {
    uint32_t k = 1u;
    const uint32_t step = xpow8_pow2(4);  // x^(8*16)
    for (int l = 255; l >= 0; --l) {
      v[l] = k;
      k = gf_mul_c(k, step);
    }
  }
};
__constant__ LaneShift c_klane{};

// c_lane_nib.v[l][t] = t(x) * c_klane.v[l] mod P for every 4-bit polynomial
// t, and c_red4.v[t] = t(x) * x^32 mod P: a product by a lane's shift then
// takes 4 bits of the other factor per step instead of 1.
struct LaneShiftNib {
  uint32_t v[256][16];
  constexpr LaneShiftNib() : v() {
    const LaneShift ls;
    for (int l = 0; l < 256; ++l) {
      uint32_t p[4] = {ls.v[l], 0u, 0u, 0u};
      for (int b = 1; b < 4; ++b) p[b] = (p[b - 1] << 1) ^ ((p[b - 1] & 0x80000000u) ? kPoly : 0u);
      for (int t = 0; t < 16; ++t) {
        uint32_t s = 0;
        for (int b = 0; b < 4; ++b)
          if ((t >> b) & 1) s ^= p[b];
        v[l][t] = s;
      }
    }
  }
};
__device__ const LaneShiftNib c_lane_nib{};

struct Reduce4 {
  uint32_t v[16];
  constexpr Reduce4() : v() {
    for (int t = 0; t < 16; ++t) {
      uint32_t r = (uint32_t)t << 28;
      for (int k = 0; k < 4; ++k) r = (r << 1) ^ ((r & 0x80000000u) ? kPoly : 0u);
      v[t] = r;
    }
  }
};
__constant__ Reduce4 c_red4{};

// Fills red4[0..16) (shared memory) from c_red4; the caller synchronises.
__device__ __forceinline__ void red4_fill(uint32_t *red4) {
  if (threadIdx.x < 16) red4[threadIdx.x] = c_red4.v[threadIdx.x];
}

// r * c_klane.v[lane] mod P: Horner over the nibbles of r, most significant
// first (acc * x^4 = acc << 4 ^ red4[top nibble of acc]).
__device__ __forceinline__ uint32_t gf_mul_lane(uint32_t r, int lane, const uint32_t *red4) {
  const uint32_t *kt = c_lane_nib.v[lane];
  uint32_t acc = 0;
#pragma unroll
  for (int i = 7; i >= 0; --i) acc = (acc << 4) ^ red4[acc >> 28] ^ kt[(r >> (4 * i)) & 15u];
  return acc;
}

__device__ __forceinline__ uint32_t gf_mul(uint32_t a, uint32_t b) {
  uint32_t r = 0;
#pragma unroll 8
  for (int i = 31; i >= 0; --i) {
    r = (r << 1) ^ ((r & 0x80000000u) ? kPoly : 0u);
    if ((b >> i) & 1u) r ^= a;
  }
  return r;
}

// x^(8j) mod P
__device__ __forceinline__ uint32_t xpow8(uint64_t j) {
  uint32_t r = 1u;
  for (int i = 0; j; ++i, j >>= 1)
    if (j & 1u) r = gf_mul(r, c_xpow[i]);
  return r;
}

// c_crc_byte.v[b] = crc0 of the single byte b
struct ByteCrcTable {
  uint32_t v[256];
  constexpr ByteCrcTable() : v() {
    for (int i = 0; i < 256; ++i) {
      uint32_t c = (uint32_t)i << 24;
      for (int k = 0; k < 8; k++) c = (c & 0x80000000u) ? (c << 1) ^ kPoly : (c << 1);
      v[i] = c;
    }
  }
};
__device__ const ByteCrcTable c_crc_byte{};

// tbl[b] = crc0 of the single byte b (shared memory; the caller synchronises)
__device__ __forceinline__ void crc_table_fill(uint32_t *tbl) {
  for (int i = threadIdx.x; i < 256; i += blockDim.x) tbl[i] = c_crc_byte.v[i];
}

__device__ __forceinline__ uint32_t crc_byte(uint32_t crc, uint32_t byte, const uint32_t *tbl) {
  return (crc << 8) ^ tbl[(crc >> 24) ^ byte];
}

}  // namespace
}  // namespace bz2g
