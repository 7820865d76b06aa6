// GPU decompressor for .bz2 streams (no counterpart in the reference, whose
// TODO.md:28-34 lists decompression as missing).
//
// Blocks are decoded in parallel:
//   1. k_dec_magic: every bit offset of the stream is tested for the 48-bit
//      block magic 0x314159265359 and the end-of-stream magic 0x177245385090;
//      the host then follows the chain (a block starts where the previous one
//      ended), so a magic that happens to appear inside a payload is ignored.
//   2. k_dec_block: one warp per candidate block.  All 32 lanes walk the bit
//      stream in lockstep (the same reads, so shared-memory tables are read as
//      broadcasts): header (CRC, origPtr, symbol map, tables, selectors),
//      Huffman symbols via an 8-bit lookup table with the canonical slow path
//      for longer codes, RUNA/RUNB zero runs, and the inverse move-to-front
//      32 MTF steps at a time across the warp.  Out: the BWT last column L.
//   3. k_dec_lf_hist / _scan / _rank: LF vector
//      tt[C[L[i]] + rank(i)] = i << 8 | L[i] by a stable counting sort.
//   4. k_dec_split / k_dec_walk / k_dec_chain: per block, the chain from
//      origPtr gives the RLE1 bytes, cut at up to 2048 splitters that are
//      walked in parallel.
//   5. k_dec_unrle1_count / _write: per block, one warp expands the RLE1 runs
//      (4 equal bytes then a count byte) from 32 segments at once; k_dec_crc
//      computes each block's CRC over its output (4096-byte chunks combined
//      over GF(2)), checked against the header.
// Batches of blocks go through steps 2-5 while the previous batch's bytes are
// copied out on a second stream; within a batch the largest compressed blocks
// start first, since a launch lasts as long as its slowest blocks.
// Every field read from the stream is range-checked and every loop is bounded,
// so a malformed stream gives an error status, not a fault.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bz2g.h"
#include "common.cuh"
#include "compressor.h"
#include "crc.cuh"

namespace bz2g {

void set_last_error(const std::string &msg);

namespace {

constexpr int kDecMaxGroups = 6;
constexpr int kDecMaxAlpha = 258;
constexpr int kDecMaxCode = 20;
constexpr int kDecMaxSel = 18002;
constexpr int kLutBits = 8;
// Per-block capacity of the last column (the reference's 900,000-byte raw
// blocks can exceed 900,000 RLE1 bytes by up to a quarter).
constexpr int kDecCap = 1200000;

enum DecStatus {
  kDecOk = 0,
  kDecBadHeader = 1,
  kDecBadTables = 2,
  kDecBadSymbol = 3,
  kDecTooLong = 4,
  kDecBadOrigPtr = 5,
  kDecBadCrc = 6,
};

__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

// Sequential big-endian bit reader over the stream's words (reads past the end
// return zeros).  A three-word window w0:w1:w2 (already byte-swapped) and the
// bit offset in w0: peek32 is one funnel shift, and the word after the
// window is loaded when the offset passes a word, well before it is needed.
struct BitReader {
  const uint32_t *w;
  int64_t nwords, wnext;  // wnext: index of the word after the window
  uint32_t w0, w1, w2;
  int bo;
  __device__ __forceinline__ uint32_t ld(int64_t i) const {
    return i < nwords ? bswap32(w[i]) : 0u;
  }
  __device__ void init(const uint32_t *words, int64_t nw, int64_t bitpos) {
    w = words;
    nwords = nw;
    const int64_t i = bitpos >> 5;
    w0 = ld(i);
    w1 = ld(i + 1);
    w2 = ld(i + 2);
    wnext = i + 3;
    bo = (int)(bitpos & 31);
  }
  // the 32 bits from the current position
  __device__ __forceinline__ uint32_t peek32() const { return __funnelshift_l(w1, w0, bo); }
  __device__ __forceinline__ uint32_t peek(int n) const { return peek32() >> (32 - n); }
  // n <= 32
  __device__ __forceinline__ void skip(int n) {
    bo += n;
    if (bo >= 32) {
      bo -= 32;
      w0 = w1;
      w1 = w2;
      w2 = ld(wnext++);
    }
  }
  __device__ __forceinline__ uint32_t get(int n) {
    if (n == 0) return 0;
    const uint32_t v = peek(n);
    skip(n);
    return v;
  }
  __device__ __forceinline__ int64_t pos() const { return (wnext - 3) * 32 + bo; }
};

__global__ void k_dec_magic(const uint32_t *words, int64_t nwords, int64_t nbits,
                            int64_t *blk, int *nblk, int64_t *eos, int *neos, int cap) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nwords) return;
  const uint64_t a = bswap32(words[i]);
  const uint64_t b = i + 1 < nwords ? bswap32(words[i + 1]) : 0u;
  const uint64_t c = i + 2 < nwords ? bswap32(words[i + 2]) : 0u;
  const uint64_t hi = (a << 32) | b;  // bits 32i .. 32i + 63
  for (int s = 0; s < 32; s++) {
    const int64_t p = i * 32 + s;
    if (p + 48 > nbits) break;
    const uint64_t v = ((hi << s) | (s ? (c >> (32 - s)) : 0)) >> 16;  // 48 bits at p
    if (v == 0x314159265359ull) {
      const int k = atomicAdd(nblk, 1);
      if (k < cap) blk[k] = p;
    } else if (v == 0x177245385090ull) {
      const int k = atomicAdd(neos, 1);
      if (k < cap) eos[k] = p;
    }
  }
}

// Per-block results of k_dec_block.
struct DecBlock {
  int64_t start;    // bit position of the block magic
  int64_t end;      // bit position after the payload
  int32_t m;        // last-column length
  int32_t orig_ptr;
  uint32_t crc;     // from the header
  int32_t status;
};

struct DecShared {
  uint16_t lut[kDecMaxGroups][1 << kLutBits];  // (len << 9) | symbol; 0 = longer code
  int32_t limit[kDecMaxGroups][kDecMaxCode + 2];
  int32_t base[kDecMaxGroups][kDecMaxCode + 2];
  uint16_t perm[kDecMaxGroups][kDecMaxAlpha];
  uint8_t minlen[kDecMaxGroups];
  uint8_t len[kDecMaxGroups][kDecMaxAlpha];
  uint8_t seq2unseq[256];
  uint8_t list[2][256];  // MTF list before / after a batch of steps
  uint32_t used[8];      // list positions a batch read
};

// c copies of byte v at d (word stores between unaligned ends).
__device__ __forceinline__ void fill_bytes(uint8_t *d, int c, uint8_t v) {
  while (c > 0 && (reinterpret_cast<uintptr_t>(d) & 3u)) {
    *d++ = v;
    c--;
  }
  const uint32_t wv = 0x01010101u * v;
  for (; c >= 4; c -= 4, d += 4) *reinterpret_cast<uint32_t *>(d) = wv;
  while (c-- > 0) *d++ = v;
}

// One warp per candidate.  sel: per-candidate selector scratch (kDecMaxSel).
__global__ void __launch_bounds__(32) k_dec_block(const uint32_t *words, int64_t nwords,
                                                  const int64_t *cand, int ncand,
                                                  DecBlock *out, uint8_t *Lbuf,
                                                  uint8_t *selbuf, int cap,
                                                  const int32_t *order) {
  __shared__ DecShared sh;
  if ((int)blockIdx.x >= ncand) return;
  const int bi = order[blockIdx.x];  // largest compressed blocks first
  const int ln = threadIdx.x;
  DecBlock r;
  r.start = cand[bi];
  r.end = r.start;
  r.m = 0;
  r.orig_ptr = -1;
  r.crc = 0;
  r.status = kDecOk;
  uint8_t *L = Lbuf + (size_t)bi * cap;
  uint8_t *sel = selbuf + (size_t)bi * kDecMaxSel;
  BitReader br;
  br.init(words, nwords, r.start + 48);
  r.crc = br.get(32);
  const uint32_t randomised = br.get(1);
  r.orig_ptr = (int32_t)br.get(24);
  // symbol map
  const uint32_t used16 = br.get(16);
  int nuse = 0;
  for (int i = 0; i < 16; i++) {
    if ((used16 >> (15 - i)) & 1u) {
      const uint32_t bits = br.get(16);
      for (int j = 0; j < 16; j++)
        if ((bits >> (15 - j)) & 1u) {
          if (ln == 0) sh.seq2unseq[nuse] = (uint8_t)(i * 16 + j);
          nuse++;
        }
    }
  }
  const int alpha = nuse + 2;
  const int ng = (int)br.get(3);
  const int nsel = (int)br.get(15);
  if (randomised || nuse == 0 || ng < 2 || ng > 6 || nsel < 1 || nsel > kDecMaxSel) {
    r.status = kDecBadHeader;
  }
  // selectors: unary-coded MTF indices over 0..ng-1
  if (r.status == kDecOk) {
    uint32_t lst = 0x543210u;  // nibble k = table at list position k
    for (int i = 0; i < nsel && r.status == kDecOk; i++) {
      int j = 0;
      while (br.get(1)) {
        if (++j >= ng) {
          r.status = kDecBadHeader;
          break;
        }
      }
      if (r.status != kDecOk) break;
      const uint32_t t = (lst >> (4 * j)) & 0xFu;
      // move to front: nibbles below j shift up one
      const uint32_t low = (1u << (4 * j)) - 1u;
      lst = (lst & ~((low << 4) | 0xFu)) | ((lst & low) << 4) | t;
      if (ln == 0) sel[i] = (uint8_t)t;
    }
  }
  // code lengths: 5-bit start, then per symbol 1x (x=0: +1, x=1: -1), 0 ends
  if (r.status == kDecOk) {
    for (int t = 0; t < ng && r.status == kDecOk; t++) {
      int cur = (int)br.get(5);
      for (int v = 0; v < alpha; v++) {
        int steps = 0;
        for (;;) {
          if (cur < 1 || cur > kDecMaxCode || ++steps > 64) {
            r.status = kDecBadTables;
            break;
          }
          if (!br.get(1)) break;
          cur += br.get(1) ? -1 : 1;
        }
        if (r.status != kDecOk) break;
        if (ln == 0) sh.len[t][v] = (uint8_t)cur;
      }
    }
  }
  __syncwarp();
  // canonical decoding tables: for each length, the symbols of that length in
  // symbol order get consecutive codes; limit[n] = largest code of length n,
  // base[n] turns a length-n code into an index into perm.
  if (r.status == kDecOk) {
    for (int t = 0; t < ng; t++) {
      int mn = 32, mx = 0;
      for (int v = 0; v < alpha; v++) {
        mn = min(mn, (int)sh.len[t][v]);
        mx = max(mx, (int)sh.len[t][v]);
      }
      if (ln == 0) {
        sh.minlen[t] = (uint8_t)mn;
        int pp = 0;
        for (int l = mn; l <= mx; l++)
          for (int v = 0; v < alpha; v++)
            if (sh.len[t][v] == l) sh.perm[t][pp++] = (uint16_t)v;
        int count[kDecMaxCode + 2];
        for (int l = 0; l <= kDecMaxCode + 1; l++) count[l] = 0;
        for (int v = 0; v < alpha; v++) count[sh.len[t][v]]++;
        int code = 0, idx = 0;
        for (int l = 0; l <= kDecMaxCode + 1; l++) {
          sh.limit[t][l] = -1;
          sh.base[t][l] = 0;
        }
        for (int l = mn; l <= mx; l++) {
          // codes of length l: [code, code + count[l]), perm index idx ..
          sh.base[t][l] = code - idx;
          sh.limit[t][l] = code + count[l] - 1;
          idx += count[l];
          code = (code + count[l]) << 1;
        }
      }
    }
  }
  __syncwarp();
  if (r.status == kDecOk) {
    // lookup tables: every kLutBits-bit prefix that starts a code of at most
    // kLutBits bits
    for (int t = 0; t < ng; t++) {
      for (int p = ln; p < (1 << kLutBits); p += 32) {
        uint16_t e = 0;
        for (int l = sh.minlen[t]; l <= kLutBits; l++) {
          const int code = p >> (kLutBits - l);
          if (code <= sh.limit[t][l] && sh.limit[t][l] >= 0) {
            const int idx = code - sh.base[t][l];
            if (idx >= 0 && idx < alpha) e = (uint16_t)((l << 9) | sh.perm[t][idx]);
            break;
          }
        }
        sh.lut[t][p] = e;
      }
    }
  }
  __syncwarp();
  // Huffman symbols -> RUNA/RUNB runs -> MTF steps, batched: lane q holds
  // step q of the batch (v = MTF index, 0 for a zero run; bytes = 1, or the
  // run length).  A full batch is resolved across the warp at once:
  //  * lane t walks its index back through the batch's earlier steps s: a
  //    step moved the entry at v_s to the front, so position p after it was
  //    p - 1 before it when 1 <= p <= v_s, and p == 0 is step s's own output;
  //  * lanes that reach position 0 point at that step's lane, the others read
  //    the list as it was before the batch; pointer jumping settles pointers;
  //  * the new list: the batch's distinct outputs, most recent first, then
  //    the untouched entries in their old order (equal outputs found by
  //    ballots).
  for (int p = ln; p < 256; p += 32) sh.list[0][p] = (uint8_t)p;
  __syncwarp();
  int cur = 0;
  int my_v = 0, my_n = 0, nst = 0;
  int m = 0;     // bytes written by resolved batches
  int pend = 0;  // bytes of the batch being filled
  int64_t zrun = 0;
  int zbit = 0;
  const int eob = nuse + 1;
  int gsel = 0, gleft = 0, tsel = 0;
  auto resolve_batch = [&]() {
    const unsigned full = 0xffffffffu;
    const bool act = ln < nst;
    int p = my_v, ptr = -1;
#pragma unroll
    for (int s = 30; s >= 0; --s) {
      const int vs = __shfl_sync(full, my_v, s);
      if (ln > s && ptr < 0) {
        if (p == 0) ptr = s;
        else if (p <= vs) p--;
      }
    }
    const uint8_t *lst = sh.list[cur];
    const bool from_list = act && ptr < 0;
    int val = from_list ? (int)lst[p] : -1;
#pragma unroll
    for (int r2 = 0; r2 < 5; r2++) {
      const int src = ptr >= 0 ? ptr : ln;
      const int tv = __shfl_sync(full, val, src);
      const int tp = __shfl_sync(full, ptr, src);
      if (val < 0 && ptr >= 0) {
        if (tv >= 0) val = tv;
        else ptr = tp;
      }
    }
    // active lanes with the same output: one ballot per bit of it
    unsigned peers = __ballot_sync(full, act);
#pragma unroll
    for (int bit = 0; bit < 8; bit++) {
      const bool on = act && ((val >> bit) & 1);
      const unsigned bb = __ballot_sync(full, on);
      peers &= on ? bb : ~bb;
    }
    const unsigned above = ~((2u << ln) - 1u);  // lanes after this one
    const bool last = act && (peers & above) == 0u;
    const unsigned lastm = __ballot_sync(full, last);
    const int D = __popc(lastm);
    if (ln < 8) sh.used[ln] = 0u;
    __syncwarp();
    if (from_list) atomicOr(&sh.used[p >> 5], 1u << (p & 31));
    __syncwarp();
    uint8_t *nx = sh.list[cur ^ 1];
    if (last) nx[__popc(lastm & above)] = (uint8_t)val;
    {
      const int q0 = 8 * ln;
      int below = 0;
      for (int x = 0; x < (q0 >> 5); x++) below += __popc(sh.used[x]);
      const uint32_t uw = sh.used[q0 >> 5];
      for (int j = 0; j < 8; j++) {
        const int q = q0 + j;
        if (q >= nuse) break;
        const uint32_t bit = 1u << (q & 31);
        if (!(uw & bit)) nx[D + q - below - __popc(uw & (bit - 1u))] = lst[q];
      }
    }
    // bytes: step t at m + (bytes of the earlier steps)
    const int nb = act ? my_n : 0;
    const int incl = warp_incl_sum(nb);
    if (act) {
      const uint8_t c = sh.seq2unseq[val];
      if (nb == 1) L[m + incl - 1] = c;
      else fill_bytes(L + m + incl - nb, nb, c);
    }
    m += __shfl_sync(full, incl, 31);
    cur ^= 1;
    nst = 0;
    pend = 0;
    __syncwarp();
  };
  // queue one step (the caller has checked the capacity)
  auto push_step = [&](int v, int bytes) {
    if (ln == nst) {
      my_v = v;
      my_n = bytes;
    }
    nst++;
    pend += bytes;
    if (nst == 32) resolve_batch();
  };
  // Every iteration takes one symbol of a 50-symbol group and the groups are
  // bounded by nsel, so the loop ends.
  if (r.status == kDecOk) {
    int tsel_next = sel[0];
    const uint16_t *lut = sh.lut[0];
    for (;;) {
      if (gleft == 0) {
        if (gsel >= nsel) {
          r.status = kDecBadSymbol;
          break;
        }
        tsel = tsel_next;
        lut = sh.lut[tsel];
        gsel++;
        tsel_next = gsel < nsel ? sel[gsel] : 0;  // next group's table, loaded early
        gleft = 50;
      }
      gleft--;
      // one symbol with table tsel
      int sym;
      const uint32_t win = br.peek32();
      const uint32_t e = lut[win >> (32 - kLutBits)];
      if (e) {
        br.skip((int)(e >> 9));
        sym = (int)(e & 511u);
      } else {
        // longer than the table: the canonical limits from kLutBits + 1 bits
        int n = max((int)sh.minlen[tsel], kLutBits + 1);
        int code = (int)(win >> (32 - n));
        while (n <= kDecMaxCode && code > sh.limit[tsel][n]) {
          n++;
          code = (int)(win >> (32 - n));
        }
        const int idx = n <= kDecMaxCode ? code - sh.base[tsel][n] : -1;
        if (idx < 0 || idx >= alpha) {
          r.status = kDecBadSymbol;
          break;
        }
        br.skip(n);
        sym = sh.perm[tsel][idx];
      }
      if (sym <= 1) {  // RUNA / RUNB: bijective base-2 digits, least significant first
        if (zbit > 40) {
          r.status = kDecTooLong;
          break;
        }
        zrun += (int64_t)(sym + 1) << zbit;
        zbit++;
        continue;
      }
      // a pending zero run: copies of the list's front entry (no move)
      if (zrun > 0) {
        if (zrun > (int64_t)(cap - m - pend)) {
          r.status = kDecTooLong;
          break;
        }
        push_step(0, (int)zrun);
        zrun = 0;
        zbit = 0;
      }
      if (sym == eob) break;
      // value v = sym - 1 >= 1: the entry at list position v moves to the front
      const int v = sym - 1;
      if (v >= nuse || m + pend >= cap) {
        r.status = v >= nuse ? kDecBadSymbol : kDecTooLong;
        break;
      }
      push_step(v, 1);
    }
    if (r.status == kDecOk && nst > 0) resolve_batch();
  }
  if (r.status == kDecOk && (r.orig_ptr < 0 || r.orig_ptr >= m)) r.status = kDecBadOrigPtr;
  r.m = m;
  r.end = br.pos();
  if (ln == 0) out[bi] = r;
}

// LF vector without serial ranks: T[C[L[i]] + rank(i)] = i << 8 | L[i], with
// rank(i) = #{j < i : L[j] == L[i]} (then for j = LF(i), psi(j) = i and
// F[j] = L[i]).  A stable counting sort by the byte: per 4096-entry chunk a
// histogram, per block a scan over chunks (each chunk's start per byte value,
// C included), then per chunk the ranks of 256 entries at a time: equal bytes
// in a warp by ballots, earlier warps by shared counts.
constexpr int kLfChunk = 4096;
constexpr int kLfChunks = (kDecCap + kLfChunk - 1) / kLfChunk;

__global__ void __launch_bounds__(256) k_dec_lf_hist(const int32_t *idx, const DecBlock *db,
                                                     const uint8_t *Lbuf, int32_t *H, int cap) {
  __shared__ int cnt[256];
  const int k = blockIdx.y, ch = blockIdx.x;
  const int bi = idx[k];
  const int m = db[bi].m;
  const int c0 = ch * kLfChunk;
  if (c0 >= m) return;
  const uint8_t *L = Lbuf + (size_t)bi * cap;
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const int c1 = min(m, c0 + kLfChunk);
  for (int i = c0 + threadIdx.x; i < c1; i += 256) atomicAdd(&cnt[L[i]], 1);
  __syncthreads();
  H[((size_t)k * kLfChunks + ch) * 256 + threadIdx.x] = cnt[threadIdx.x];
}

// Per block (thread = byte value): H[chunk][c] becomes the position of the
// chunk's first c in F order.
__global__ void __launch_bounds__(256) k_dec_lf_scan(const int32_t *idx, const DecBlock *db,
                                                     int32_t *H) {
  __shared__ int scratch[40];
  const int k = blockIdx.x;
  const int m = db[idx[k]].m;
  const int nch = (m + kLfChunk - 1) / kLfChunk;
  int32_t *h = H + (size_t)k * kLfChunks * 256 + threadIdx.x;
  int tot = 0;
  for (int ch = 0; ch < nch; ch++) tot += h[(size_t)ch * 256];
  int all;
  int run = block_excl_sum(tot, scratch, &all);  // C[c]
  for (int ch = 0; ch < nch; ch++) {
    const int v = h[(size_t)ch * 256];
    h[(size_t)ch * 256] = run;
    run += v;
  }
}

__global__ void __launch_bounds__(256) k_dec_lf_rank(const int32_t *idx, const DecBlock *db,
                                                     const uint8_t *Lbuf, const int32_t *H,
                                                     uint32_t *tt, int cap) {
  __shared__ int run[256];
  __shared__ int wc[8][256];
  const int k = blockIdx.y, ch = blockIdx.x;
  const int bi = idx[k];
  const int m = db[bi].m;
  const int c0 = ch * kLfChunk;
  if (c0 >= m) return;
  const uint8_t *L = Lbuf + (size_t)bi * cap;
  uint32_t *T = tt + (size_t)k * cap;
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
  run[threadIdx.x] = H[((size_t)k * kLfChunks + ch) * 256 + threadIdx.x];
  for (int sub = 0; sub < kLfChunk / 256; sub++) {
    const int i = c0 + sub * 256 + threadIdx.x;
    if (c0 + sub * 256 >= m) break;  // uniform
    const bool valid = i < m;
    const int c = valid ? (int)L[i] : 256 + ln;
    for (int q = threadIdx.x; q < 8 * 256; q += 256) (&wc[0][0])[q] = 0;
    __syncthreads();
    // lanes with the same byte: one ballot per bit (cheaper than match_any)
    unsigned peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
    for (int bit = 0; bit < 8; bit++) {
      const bool on = (c >> bit) & 1;
      const unsigned bb = __ballot_sync(0xffffffffu, on);
      peers &= on ? bb : ~bb;
    }
    const int wr = __popc(peers & ((1u << ln) - 1u));
    if (valid && wr == 0) wc[w][c] = __popc(peers);
    __syncthreads();
    if (valid) {
      int j = run[c] + wr;
      for (int q = 0; q < w; q++) j += wc[q][c];
      if (j >= 0 && j < m) T[j] = ((uint32_t)i << 8) | (uint32_t)c;
    }
    __syncthreads();
    if (valid && wr == 0) atomicAdd(&run[c], __popc(peers));
  }
}

// The RLE1 bytes of each block follow tt from origPtr:
// T[j] = psi(j) << 8 | F[j], psi = LF^-1, and the text is F[origPtr],
// F[psi(origPtr)], ...  One dependent load per byte, so the chain is cut at
// S splitters per block (origPtr and evenly spaced positions, marked in bit
// 31 of their T entry, which the walk loads anyway): every walker counts the
// steps to the next marked position, the segments are ordered along the chain
// from origPtr, and the walkers walk again writing their segment at its
// offset.  Segment lengths along the chain are close to exponential, so the
// longest is about ln(S) times the mean (m / S, about 512 here).  A periodic
// block (its cycle closes before m bytes) repeats that one cycle.
constexpr int kMaxWalkers = 2048;
constexpr int kWalkSpan = 512;
constexpr uint32_t kMark = 0x80000000u;
constexpr uint32_t kPsiMask = 0x7FFFFF00u;

struct WalkCtl {
  int32_t nw;        // splitters
  int32_t cycle;     // bytes of the chain from origPtr before it closes (m if it does not)
  int32_t pos[kMaxWalkers];   // sorted splitter positions
  int32_t len[kMaxWalkers];   // segment length (steps to the next splitter)
  int32_t next[kMaxWalkers];  // index of the splitter reached
  int32_t off[kMaxWalkers];   // output offset, -1 when off the chain
};

// Splitter positions (one thread) and their marks in T (all threads).
__global__ void k_dec_split(const int32_t *idx, const DecBlock *db, WalkCtl *ctl, uint32_t *tt,
                            int cap) {
  const int k = blockIdx.x;
  const DecBlock b = db[idx[k]];
  WalkCtl &c = ctl[k];
  uint32_t *T = tt + (size_t)k * cap;
  const int m = b.m;
  if (threadIdx.x == 0) {
    const int S = max(1, min(kMaxWalkers, m / kWalkSpan));
    int n = 0;
    bool placed = false;
    for (int t = 1; t <= S; t++) {
      const int j = t < S ? (int)((int64_t)t * m / S) : m;  // t == S: sentinel
      if (!placed && b.orig_ptr <= j) {
        c.pos[n++] = b.orig_ptr;
        placed = true;
      }
      if (t < S && j != b.orig_ptr && j < m) c.pos[n++] = j;
    }
    if (!placed) c.pos[n++] = b.orig_ptr;
    c.nw = n;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < c.nw; q += blockDim.x) {
    const int p = c.pos[q];
    if (p >= 0 && p < m) T[p] |= kMark;
  }
}

__device__ __forceinline__ int splitter_index(const WalkCtl &c, int p) {
  int lo = 0, hi = c.nw - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (c.pos[mid] < p) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// write == 0: segment lengths and successors; write != 0: the segment bytes.
__global__ void k_dec_walk(const int32_t *idx, const DecBlock *db, const uint32_t *tt,
                           WalkCtl *ctl, uint8_t *rle, int cap, int write) {
  const int k = blockIdx.y;
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  WalkCtl &c = ctl[k];
  if (w >= c.nw) return;
  const int m = db[idx[k]].m;
  const uint32_t *T = tt + (size_t)k * cap;
  uint8_t *R = rle + (size_t)idx[k] * cap;
  if (write && c.off[w] < 0) return;
  uint32_t p = (uint32_t)c.pos[w];
  int n = 0;
  const int o = write ? c.off[w] : 0;
  const int lim = write ? c.len[w] : m;
  bool at_mark = false;
  for (;;) {
    if (p >= (uint32_t)m || n >= lim || o + n >= m) break;
    const uint32_t e = T[p];
    if (n > 0 && (e & kMark)) {
      at_mark = true;
      break;
    }
    if (write) R[o + n] = (uint8_t)(e & 0xFFu);
    n++;
    p = (e & kPsiMask) >> 8;
  }
  if (!write) {
    c.len[w] = n;
    c.next[w] = at_mark ? splitter_index(c, (int)p) : -1;
  }
}

// Per block: segment offsets along the chain from origPtr (one thread walks
// the segments, held in shared memory).
__global__ void __launch_bounds__(256) k_dec_chain(const int32_t *idx, const DecBlock *db,
                                                   WalkCtl *ctl, int *bad) {
  __shared__ int32_t len[kMaxWalkers], nxt[kMaxWalkers], off[kMaxWalkers];
  const int k = blockIdx.x;
  const DecBlock b = db[idx[k]];
  WalkCtl &c = ctl[k];
  const int nw = c.nw;
  for (int q = threadIdx.x; q < nw; q += blockDim.x) {
    len[q] = c.len[q];
    nxt[q] = c.next[q];
    off[q] = -1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int w0 = splitter_index(c, b.orig_ptr);
    int w = w0, o = 0;
    for (int steps = 0; steps <= nw; steps++) {
      if (w < 0 || w >= nw || off[w] >= 0) break;
      off[w] = o;
      o += len[w];
      if (o >= b.m) break;
      w = nxt[w];
    }
    c.cycle = min(o, b.m);
    if (c.cycle <= 0 || b.m % c.cycle != 0) atomicOr(bad, 1);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nw; q += blockDim.x) c.off[q] = off[q];
}

// A periodic block: the first `cycle` bytes repeated to m.
__global__ void k_dec_repeat(const int32_t *idx, const DecBlock *db, const WalkCtl *ctl,
                             uint8_t *rle, int cap) {
  const int k = blockIdx.y;
  const int m = db[idx[k]].m;
  const int cyc = ctl[k].cycle;
  if (cyc <= 0 || cyc >= m) return;
  uint8_t *R = rle + (size_t)idx[k] * cap;
  for (int i = cyc + blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    R[i] = R[i % cyc];
}


// Inverse RLE1 (4 equal bytes are followed by a count of further copies), one
// warp per block.  The block's RLE1 bytes are cut into 32 lane segments.  What
// a segment produces depends only on the run state it starts in: 0 = no run
// (block start, or just after a count byte), 1..3 = the byte before the
// segment closes a run of that length, 4 = the next byte is a count.  The
// count pass follows each segment from all five states at once until they
// merge (typically within a few bytes: at a byte that differs from the one
// before it), chains the lanes' state maps from state 0 across the warp and
// keeps each lane's entry state and output offset; the write pass expands
// every segment at its offset (runs with word stores), and k_dec_crc computes
// the block CRCs over the output.
constexpr int kUnrleWarps = 8;

struct LaneStart {
  int32_t state;
  int32_t off;  // output offset of the segment within its block
};

__device__ __forceinline__ void rle1_step(int &r, int &n, int c, int p) {
  if (r == 4) {
    n += c;
    r = 0;
  } else if (r >= 1 && c == p) {
    r++;
    n++;
  } else {
    r = 1;
    n++;
  }
}

__device__ __forceinline__ int pick5(int x, int a0, int a1, int a2, int a3, int a4) {
  return x == 0 ? a0 : x == 1 ? a1 : x == 2 ? a2 : x == 3 ? a3 : a4;
}

__global__ void __launch_bounds__(32 * kUnrleWarps)
    k_dec_unrle1_count(const int32_t *idx, const DecBlock *db, const uint8_t *rle, int nacc,
                       int cap, LaneStart *lanes, int64_t *lens) {
  const int k = blockIdx.x * kUnrleWarps + (threadIdx.x >> 5);
  const int ln = threadIdx.x & 31;
  if (k >= nacc) return;  // the whole warp
  const int bi = idx[k];
  const int m = db[bi].m;
  const uint8_t *R = rle + (size_t)bi * cap;
  const int seg = (m + 31) / 32;
  const int s0 = min(ln * seg, m), e0 = min(s0 + seg, m);
  int p = s0 > 0 ? R[s0 - 1] : -1;
  int r0 = 0, r1 = 1, r2 = 2, r3 = 3, r4 = 4;
  int n0 = 0, n1 = 0, n2 = 0, n3 = 0, n4 = 0;
  int i = s0;
  bool merged = false;
  while (i < e0 && !merged) {
    const int c = R[i++];
    rle1_step(r0, n0, c, p);
    rle1_step(r1, n1, c, p);
    rle1_step(r2, n2, c, p);
    rle1_step(r3, n3, c, p);
    rle1_step(r4, n4, c, p);
    p = c;
    merged = r0 == r1 && r0 == r2 && r0 == r3 && r0 == r4;
  }
  int r = r0, nb = 0;
  while (i < e0) {
    const int c = R[i++];
    rle1_step(r, nb, c, p);
    p = c;
  }
  if (merged) {
    r0 = r1 = r2 = r3 = r4 = r;
    n0 += nb;
    n1 += nb;
    n2 += nb;
    n3 += nb;
    n4 += nb;
  }
  int state = 0, off = 0, my_state = 0, my_off = 0;
  for (int l = 0; l < 32; l++) {
    if (ln == l) {
      my_state = state;
      my_off = off;
    }
    const int ro = __shfl_sync(0xffffffffu, pick5(state, r0, r1, r2, r3, r4), l);
    const int no = __shfl_sync(0xffffffffu, pick5(state, n0, n1, n2, n3, n4), l);
    state = ro;
    off += no;
  }
  lanes[(size_t)k * 32 + ln] = LaneStart{my_state, my_off};
  if (ln == 0) lens[k] = off;
}

__global__ void __launch_bounds__(32 * kUnrleWarps)
    k_dec_unrle1_write(const int32_t *idx, const DecBlock *db, const uint8_t *rle, int nacc,
                       int cap, const LaneStart *lanes, const int64_t *off, uint8_t *out) {
  const int k = blockIdx.x * kUnrleWarps + (threadIdx.x >> 5);
  const int ln = threadIdx.x & 31;
  if (k >= nacc) return;
  const int bi = idx[k];
  const int m = db[bi].m;
  const uint8_t *R = rle + (size_t)bi * cap;
  const int seg = (m + 31) / 32;
  const int s0 = min(ln * seg, m), e0 = min(s0 + seg, m);
  int p = s0 > 0 ? R[s0 - 1] : -1;
  const LaneStart ls = lanes[(size_t)k * 32 + ln];
  int r = ls.state;
  uint8_t *O = out + off[k] + ls.off;
  for (int i = s0; i < e0; i++) {
    const int c = R[i];
    if (r == 4) {
      fill_bytes(O, c, (uint8_t)p);
      O += c;
      r = 0;
    } else {
      r = (r >= 1 && c == p) ? r + 1 : 1;
      *O++ = (uint8_t)c;
    }
    p = c;
  }
}

// Block CRCs of the expanded output, one thread block per block: 4096-byte
// chunks staged in shared memory, thread l's 16 bytes give crc0 * x^(8*16*(255-l))
// (the chunk right-aligned in 4096 bytes when shorter), the XOR is the
// chunk's crc0, and the block's crc0 accumulates chunk by chunk.
__global__ void __launch_bounds__(256) k_dec_crc(const int64_t *lens, const int64_t *off,
                                                 const uint8_t *out, uint32_t *crcs) {
  __shared__ uint32_t tbl[256];
  __shared__ uint32_t red4[16];
  __shared__ __align__(16) uint8_t chunk[4096];
  __shared__ uint32_t part[2][8];
  crc_table_fill(tbl);
  red4_fill(red4);
  const int k = blockIdx.x;
  const int64_t n = lens[k];
  const uint8_t *src = out + off[k];
  uint32_t acc = 0;  // thread 0
  int it = 0;
  for (int64_t base = 0; base < n; base += 4096, it++) {
    const int len = n - base < 4096 ? (int)(n - base) : 4096;
    const int pad = 4096 - len;
    __syncthreads();  // chunk free
    for (int i = threadIdx.x; i < 4096; i += 256) chunk[i] = i >= pad ? src[base + i - pad] : 0;
    __syncthreads();
    uint32_t r = 0;
    const uint4 v = *reinterpret_cast<const uint4 *>(chunk + 16 * threadIdx.x);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int q = 0; q < 16; q++) r = crc_byte(r, (w[q >> 2] >> (8 * (q & 3))) & 0xFFu, tbl);
    r = gf_mul_lane(r, threadIdx.x, red4);
    for (int o = 16; o; o >>= 1) r ^= __shfl_xor_sync(0xffffffffu, r, o);
    if ((threadIdx.x & 31) == 0) part[it & 1][threadIdx.x >> 5] = r;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t c = 0;
      for (int q = 0; q < 8; q++) c ^= part[it & 1][q];
      // acc * x^(8 len) ^ c
      acc = (acc ? gf_mul(acc, len == 4096 ? c_xpow[12] : xpow8((uint64_t)len)) : 0u) ^ c;
    }
  }
  if (threadIdx.x == 0) crcs[k] = ~(gf_mul(0xFFFFFFFFu, xpow8((uint64_t)n)) ^ acc);
}

// Device buffer that only grows (contents are not kept).
struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  template <typename T>
  T *get() const {
    return static_cast<T *>(p);
  }
  void reserve(size_t bytes) {
    bytes = std::max<size_t>(bytes, 16);
    if (bytes <= cap) return;
    if (p) BZ_CUDA(cudaFree(p));
    p = nullptr;
    cap = 0;
    BZ_CUDA(cudaMalloc(&p, bytes));
    cap = bytes;
  }
};

// Where decoded bytes go, batch by batch, in stream order.
struct DecSink {
  size_t size = 0;
  virtual ~DecSink() = default;
  // Queue the copy of n device bytes to the end of the output on stream cs.
  virtual void put(const uint8_t *d_src, size_t n, cudaStream_t cs) = 0;
};

// A caller's buffer of cap bytes (host or device memory).
struct BufferSink : DecSink {
  uint8_t *dst;
  size_t cap;
  BufferSink(uint8_t *d, size_t c) : dst(d), cap(c) {}
  void put(const uint8_t *d_src, size_t n, cudaStream_t cs) override {
    BZ_REQUIRE(n <= cap - size, kErrTooLarge,
               "decoded data larger than the output buffer (" + std::to_string(cap) + " bytes)");
    if (n) BZ_CUDA(cudaMemcpyAsync(dst + size, d_src, n, cudaMemcpyDefault, cs));
    size += n;
  }
};

// A malloc'ed host buffer grown by realloc (large blocks are remapped, not
// copied, and pages are touched only by the copies into them).
struct MallocSink : DecSink {
  uint8_t *buf = nullptr;
  size_t cap = 0;
  ~MallocSink() override { std::free(buf); }
  void put(const uint8_t *d_src, size_t n, cudaStream_t cs) override {
    if (n > cap - size) {
      BZ_CUDA(cudaStreamSynchronize(cs));  // no copy into the old buffer in flight
      const size_t nc = std::max(size + n, 2 * cap);
      void *q = std::realloc(buf, nc);
      BZ_REQUIRE(q != nullptr, kErrAlloc, "host allocation failed");
      buf = static_cast<uint8_t *>(q);
      cap = nc;
    }
    if (n) BZ_CUDA(cudaMemcpyAsync(buf + size, d_src, n, cudaMemcpyDefault, cs));
    size += n;
  }
  uint8_t *release() {
    uint8_t *p = buf;
    if (!p) p = static_cast<uint8_t *>(std::malloc(1));
    else if (size && size < cap) p = static_cast<uint8_t *>(std::realloc(buf, size));
    BZ_REQUIRE(p != nullptr, kErrAlloc, "host allocation failed");
    buf = nullptr;
    cap = 0;
    return p;
  }
};

// The decoder's device scratch, one per device, grown on demand and kept
// between calls.  Output batches alternate between two device buffers: the
// copy of one batch to the sink (stream cs) overlaps the decoding of the next
// (stream st).
struct DecWork {
  std::mutex mu;
  DevBuf words, blk, eos, cnt, cand, order, db, L, hist, sel, idx, tt, lens, off, crc, ctl, bad,
      lanes;
  DevBuf out[2];
  cudaStream_t st = nullptr, cs = nullptr;
  cudaEvent_t written[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr};
  bool used[2] = {false, false};
  uint32_t *h_crc = nullptr;  // pinned
  size_t h_crc_cap = 0;
  int resident = 0;  // k_dec_block warps resident on the whole device

  void init() {
    if (st) return;
    BZ_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    BZ_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    for (int q = 0; q < 2; q++) {
      BZ_CUDA(cudaEventCreateWithFlags(&written[q], cudaEventDisableTiming));
      BZ_CUDA(cudaEventCreateWithFlags(&copied[q], cudaEventDisableTiming));
    }
    int dev = 0, sms = 0, per_sm = 0;
    BZ_CUDA(cudaGetDevice(&dev));
    BZ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    BZ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dec_block, 32, 0));
    resident = std::max(1, sms * per_sm);
  }
  size_t held() const {
    size_t s = 0;
    for (const DevBuf *b : {&L, &hist, &tt, &sel, &ctl, &out[0], &out[1]}) s += b->cap;
    return s;
  }
};

DecWork &dec_work() {
  static std::mutex mu;
  static std::vector<DecWork *> per_device;  // kept for the process lifetime
  int dev = 0;
  BZ_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  if ((int)per_device.size() <= dev) per_device.resize(dev + 1, nullptr);
  if (!per_device[dev]) per_device[dev] = new DecWork();
  return *per_device[dev];
}

// Device bytes of one candidate slot: last column (later the RLE1 bytes), LF
// vector, chunk histograms, selectors, walk control.
constexpr size_t kSlotBytes = (size_t)kDecCap * 5 + (size_t)kLfChunks * 256 * 4 + kDecMaxSel +
                              sizeof(WalkCtl) + sizeof(DecBlock) + 32 * 8 + 64;
constexpr int kMaxBatch = 4096;

bool is_header(const uint8_t *h) {
  return h[0] == 'B' && h[1] == 'Z' && h[2] == 'h' && h[3] >= '1' && h[3] <= '9';
}

// The decoder proper.  w.words holds the n stream bytes, zero-padded to whole
// words plus two.
void decode_words(DecWork &w, size_t n, DecSink &sink) {
  cudaStream_t st = w.st, cs = w.cs;
  // on every exit no kernel or copy is left in flight (the sink's memory may
  // be released by the caller)
  struct Drain {
    cudaStream_t a, b;
    ~Drain() {
      cudaStreamSynchronize(a);
      cudaStreamSynchronize(b);
    }
  } drain{st, cs};
  const uint8_t *bytes = w.words.get<uint8_t>();
  const int64_t nwords = (int64_t)(n + 3) / 4 + 2;
  uint8_t head[4];
  BZ_CUDA(cudaMemcpyAsync(head, bytes, 4, cudaMemcpyDeviceToHost, st));
  BZ_CUDA(cudaStreamSynchronize(st));
  BZ_REQUIRE(is_header(head), kErrArg, "not a bzip2 stream (bad header)");
  const int64_t nbits = (int64_t)n * 8;
  // candidates
  const int ccap = (int)std::min<int64_t>((int64_t)n / 8 + 64, 1 << 26);
  w.blk.reserve(8 * (size_t)ccap);
  w.eos.reserve(8 * (size_t)ccap);
  w.cnt.reserve(8);
  BZ_CUDA(cudaMemsetAsync(w.cnt.p, 0, 8, st));
  k_dec_magic<<<(unsigned)((nwords + 255) / 256), 256, 0, st>>>(
      w.words.get<uint32_t>(), nwords, nbits, w.blk.get<int64_t>(), w.cnt.get<int>(),
      w.eos.get<int64_t>(), w.cnt.get<int>() + 1, ccap);
  BZ_LAUNCH_CHECK();
  int hcnt[2];
  BZ_CUDA(cudaMemcpyAsync(hcnt, w.cnt.p, 8, cudaMemcpyDeviceToHost, st));
  BZ_CUDA(cudaStreamSynchronize(st));
  BZ_REQUIRE(hcnt[0] <= ccap && hcnt[1] <= ccap, kErrTooLarge, "too many block candidates");
  std::vector<int64_t> cands(hcnt[0]), eoss(hcnt[1]);
  if (hcnt[0])
    BZ_CUDA(cudaMemcpyAsync(cands.data(), w.blk.p, 8 * hcnt[0], cudaMemcpyDeviceToHost, st));
  if (hcnt[1])
    BZ_CUDA(cudaMemcpyAsync(eoss.data(), w.eos.p, 8 * hcnt[1], cudaMemcpyDeviceToHost, st));
  BZ_CUDA(cudaStreamSynchronize(st));
  std::sort(cands.begin(), cands.end());
  std::sort(eoss.begin(), eoss.end());
  // batch: whole waves of resident k_dec_block warps where memory allows
  size_t freeb = 0, totb = 0;
  BZ_CUDA(cudaMemGetInfo(&freeb, &totb));
  int bmax = (int)std::min<size_t>(kMaxBatch, (freeb + w.held()) / 3 / kSlotBytes);
  bmax = std::max(bmax, 32);
  if (bmax >= w.resident) bmax = bmax / w.resident * w.resident;
  // BZ2G_DECODE_BATCH caps the blocks per batch (smaller batches, less memory)
  if (const char *e = std::getenv("BZ2G_DECODE_BATCH")) {
    const int v = std::atoi(e);
    if (v > 0) bmax = std::min(bmax, v);
  }
  const int batch = (int)std::min<size_t>(bmax, std::max<size_t>(cands.size(), 1));
  const int cap = kDecCap;
  w.cand.reserve(8 * (size_t)batch);
  w.order.reserve(4 * (size_t)batch);
  w.db.reserve(sizeof(DecBlock) * (size_t)batch);
  w.L.reserve((size_t)batch * cap);
  w.hist.reserve((size_t)batch * kLfChunks * 256 * 4);
  w.sel.reserve((size_t)batch * kDecMaxSel);
  w.idx.reserve(4 * (size_t)batch);
  w.tt.reserve((size_t)batch * cap * 4);
  w.lens.reserve(8 * (size_t)batch);
  w.off.reserve(8 * (size_t)batch);
  w.crc.reserve(4 * (size_t)batch);
  w.ctl.reserve(sizeof(WalkCtl) * (size_t)batch);
  w.bad.reserve(16);
  w.lanes.reserve(sizeof(LaneStart) * 32 * (size_t)batch);
  if (w.h_crc_cap < (size_t)batch) {
    if (w.h_crc) BZ_CUDA(cudaFreeHost(w.h_crc));
    w.h_crc = nullptr;
    w.h_crc_cap = 0;
    BZ_CUDA(cudaMallocHost((void **)&w.h_crc, 4 * (size_t)batch));
    w.h_crc_cap = batch;
  }
  uint8_t *L = w.L.get<uint8_t>();  // the RLE1 bytes overwrite the last column
  int64_t expect = 32;              // next block or end-of-stream marker
  uint32_t stream_crc = 0;
  bool stream_done = false;
  size_t ci = 0;
  int nbatch = 0;
  std::vector<DecBlock> hdb(batch);
  std::vector<int32_t> order;
  // block CRCs of the last batch, checked once st has caught up
  std::vector<uint32_t> want;
  auto settle = [&]() {
    if (want.empty()) return;
    BZ_CUDA(cudaStreamSynchronize(st));
    for (size_t q = 0; q < want.size(); q++) {
      BZ_REQUIRE(w.h_crc[q] == want[q], kErrArg, "bzip2 stream: block CRC mismatch");
      stream_crc = ((stream_crc << 1) | (stream_crc >> 31)) ^ w.h_crc[q];
    }
    want.clear();
  };
  for (;;) {
    if (stream_done) {
      // another stream may follow, from the next byte boundary
      const int64_t nb = (expect + 7) / 8;
      if (nb + 14 > (int64_t)n) break;
      uint8_t h[4];
      BZ_CUDA(cudaMemcpyAsync(h, bytes + nb, 4, cudaMemcpyDeviceToHost, st));
      BZ_CUDA(cudaStreamSynchronize(st));
      if (!is_header(h)) break;
      expect = nb * 8 + 32;
      stream_crc = 0;
      stream_done = false;
    }
    // the end-of-stream marker at `expect`?
    if (std::binary_search(eoss.begin(), eoss.end(), expect)) {
      settle();
      // combined CRC after the 48-bit marker
      const int64_t p = expect + 48;
      uint8_t tail[8] = {0};
      const int64_t b0 = p / 8;
      const size_t nb = (size_t)std::min<int64_t>(8, (int64_t)n - b0);
      BZ_CUDA(cudaMemcpyAsync(tail, bytes + b0, nb, cudaMemcpyDeviceToHost, st));
      BZ_CUDA(cudaStreamSynchronize(st));
      uint64_t win = 0;
      for (int q = 0; q < 8; q++) win = (win << 8) | tail[q];
      const uint32_t got = (uint32_t)((win << (p % 8)) >> 32);
      BZ_REQUIRE(got == stream_crc, kErrArg, "bzip2 stream CRC mismatch");
      expect = p + 32;
      stream_done = true;
      continue;
    }
    // next candidates from `expect` on
    while (ci < cands.size() && cands[ci] < expect) ci++;
    BZ_REQUIRE(ci < cands.size() && cands[ci] == expect, kErrArg,
               "bzip2 stream: no block or end-of-stream marker where one must start");
    const int nc = (int)std::min<size_t>(batch, cands.size() - ci);
    BZ_CUDA(cudaMemcpyAsync(w.cand.p, cands.data() + ci, 8 * nc, cudaMemcpyHostToDevice, st));
    // A launch lasts as long as its slowest blocks: start the largest ones
    // first (compressed size = distance to the next candidate).
    order.resize(nc);
    for (int q = 0; q < nc; q++) order[q] = q;
    auto csize = [&](int q) {
      const size_t k = ci + (size_t)q;
      return (k + 1 < cands.size() ? cands[k + 1] : nbits) - cands[k];
    };
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return csize(a) > csize(b); });
    BZ_CUDA(cudaMemcpyAsync(w.order.p, order.data(), 4 * nc, cudaMemcpyHostToDevice, st));
    k_dec_block<<<nc, 32, 0, st>>>(w.words.get<uint32_t>(), nwords, w.cand.get<int64_t>(), nc,
                                   w.db.get<DecBlock>(), L, w.sel.get<uint8_t>(), cap,
                                   w.order.get<int32_t>());
    BZ_LAUNCH_CHECK();
    BZ_CUDA(cudaMemcpyAsync(hdb.data(), w.db.p, sizeof(DecBlock) * nc, cudaMemcpyDeviceToHost,
                            st));
    BZ_CUDA(cudaStreamSynchronize(st));
    settle();
    // accept the chain within this batch
    std::vector<int32_t> acc;
    size_t used = 0;
    for (int q = 0; q < nc; q++) {
      if (hdb[q].start != expect) continue;
      BZ_REQUIRE(hdb[q].status == kDecOk, kErrArg,
                 "bzip2 stream: corrupt block (status " + std::to_string(hdb[q].status) + ")");
      acc.push_back(q);
      expect = hdb[q].end;
      used = q + 1;
      if (std::binary_search(eoss.begin(), eoss.end(), expect)) break;
    }
    ci += std::max<size_t>(used, 1);
    const int na = (int)acc.size();
    if (na == 0) continue;
    const int32_t *didx = w.idx.get<int32_t>();
    const DecBlock *ddb = w.db.get<DecBlock>();
    BZ_CUDA(cudaMemcpyAsync(w.idx.p, acc.data(), 4 * na, cudaMemcpyHostToDevice, st));
    const dim3 lgrid(kLfChunks, na);
    k_dec_lf_hist<<<lgrid, 256, 0, st>>>(didx, ddb, L, w.hist.get<int32_t>(), cap);
    BZ_LAUNCH_CHECK();
    k_dec_lf_scan<<<na, 256, 0, st>>>(didx, ddb, w.hist.get<int32_t>());
    BZ_LAUNCH_CHECK();
    k_dec_lf_rank<<<lgrid, 256, 0, st>>>(didx, ddb, L, w.hist.get<int32_t>(),
                                         w.tt.get<uint32_t>(), cap);
    BZ_LAUNCH_CHECK();
    k_dec_split<<<na, 256, 0, st>>>(didx, ddb, w.ctl.get<WalkCtl>(), w.tt.get<uint32_t>(), cap);
    BZ_LAUNCH_CHECK();
    const dim3 wgrid(kMaxWalkers / 64, na);
    k_dec_walk<<<wgrid, 64, 0, st>>>(didx, ddb, w.tt.get<uint32_t>(), w.ctl.get<WalkCtl>(), L,
                                     cap, 0);
    BZ_LAUNCH_CHECK();
    BZ_CUDA(cudaMemsetAsync(w.bad.p, 0, 4, st));
    k_dec_chain<<<na, 256, 0, st>>>(didx, ddb, w.ctl.get<WalkCtl>(), w.bad.get<int>());
    BZ_LAUNCH_CHECK();
    k_dec_walk<<<wgrid, 64, 0, st>>>(didx, ddb, w.tt.get<uint32_t>(), w.ctl.get<WalkCtl>(), L,
                                     cap, 1);
    BZ_LAUNCH_CHECK();
    k_dec_repeat<<<dim3(16, na), 256, 0, st>>>(didx, ddb, w.ctl.get<WalkCtl>(), L, cap);
    BZ_LAUNCH_CHECK();
    const unsigned ugrid = (unsigned)((na + kUnrleWarps - 1) / kUnrleWarps);
    k_dec_unrle1_count<<<ugrid, 32 * kUnrleWarps, 0, st>>>(
        didx, ddb, L, na, cap, w.lanes.get<LaneStart>(), w.lens.get<int64_t>());
    BZ_LAUNCH_CHECK();
    std::vector<int64_t> lens(na), offs(na);
    int hbad = 0;
    BZ_CUDA(cudaMemcpyAsync(lens.data(), w.lens.p, 8 * na, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaMemcpyAsync(&hbad, w.bad.p, 4, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    BZ_REQUIRE(hbad == 0, kErrArg, "bzip2 stream: inconsistent block (BWT chain)");
    int64_t tot = 0;
    for (int q = 0; q < na; q++) {
      offs[q] = tot;
      tot += lens[q];
    }
    const int slot = nbatch++ & 1;
    if (w.used[slot]) {
      if ((size_t)tot + 16 > w.out[slot].cap) BZ_CUDA(cudaEventSynchronize(w.copied[slot]));
      BZ_CUDA(cudaStreamWaitEvent(st, w.copied[slot], 0));
    }
    w.out[slot].reserve((size_t)tot + 16);
    BZ_CUDA(cudaMemcpyAsync(w.off.p, offs.data(), 8 * na, cudaMemcpyHostToDevice, st));
    k_dec_unrle1_write<<<ugrid, 32 * kUnrleWarps, 0, st>>>(
        didx, ddb, L, na, cap, w.lanes.get<LaneStart>(), w.off.get<int64_t>(),
        w.out[slot].get<uint8_t>());
    BZ_LAUNCH_CHECK();
    k_dec_crc<<<na, 256, 0, st>>>(w.lens.get<int64_t>(), w.off.get<int64_t>(),
                                  w.out[slot].get<uint8_t>(), w.crc.get<uint32_t>());
    BZ_LAUNCH_CHECK();
    BZ_CUDA(cudaMemcpyAsync(w.h_crc, w.crc.p, 4 * na, cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaEventRecord(w.written[slot], st));
    BZ_CUDA(cudaStreamWaitEvent(cs, w.written[slot], 0));
    sink.put(w.out[slot].get<uint8_t>(), (size_t)tot, cs);
    BZ_CUDA(cudaEventRecord(w.copied[slot], cs));
    w.used[slot] = true;
    want.resize(na);
    for (int q = 0; q < na; q++) want[q] = hdb[acc[q]].crc;
  }
  settle();
  BZ_REQUIRE(stream_done, kErrArg, "bzip2 stream: no end-of-stream marker");
  BZ_CUDA(cudaStreamSynchronize(cs));
}

// Stages the stream (host or device memory) in the workspace and decodes it.
void decode_into_sink(const uint8_t *in, size_t n, DecSink &sink) {
  BZ_REQUIRE(n >= 14, kErrArg, "not a bzip2 stream (shorter than 14 bytes)");
  DecWork &w = dec_work();
  std::lock_guard<std::mutex> g(w.mu);
  w.init();
  const size_t nwords = (n + 3) / 4 + 2;
  w.words.reserve(nwords * 4);
  const size_t body = n / 4 * 4;
  BZ_CUDA(cudaMemsetAsync(w.words.get<uint8_t>() + body, 0, nwords * 4 - body, w.st));
  BZ_CUDA(cudaMemcpyAsync(w.words.p, in, n, cudaMemcpyDefault, w.st));
  decode_words(w, n, sink);
}

template <typename F>
int guarded(F f) {
  try {
    f();
    set_last_error("");
    return BZ2G_OK;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return BZ2G_ERR_INTERNAL;
  }
}

int decompress_malloc(const uint8_t *in, size_t n, uint8_t **out, size_t *out_len) {
  return guarded([&] {
    BZ_REQUIRE(out && out_len && (n == 0 || in), kErrArg, "bad arguments");
    MallocSink sink;
    decode_into_sink(in, n, sink);
    *out_len = sink.size;
    *out = sink.release();
  });
}

int decompress_buffer(const uint8_t *in, size_t n, uint8_t *out, size_t cap,
                      size_t *out_len) {
  return guarded([&] {
    BZ_REQUIRE(out_len && (n == 0 || in) && (cap == 0 || out), kErrArg, "bad arguments");
    BufferSink sink(out, cap);
    decode_into_sink(in, n, sink);
    *out_len = sink.size;
  });
}

}  // namespace
}  // namespace bz2g

using namespace bz2g;

extern "C" int bz2g_decompress(const uint8_t *in, size_t n, uint8_t **out, size_t *out_len) {
  return decompress_malloc(in, n, out, out_len);
}

extern "C" int bz2g_decompress_device(const uint8_t *d_in, size_t n, uint8_t **out,
                                      size_t *out_len) {
  return decompress_malloc(d_in, n, out, out_len);
}

extern "C" int bz2g_decompress_into(const uint8_t *in, size_t n, uint8_t *out, size_t cap,
                                    size_t *out_len) {
  return decompress_buffer(in, n, out, cap, out_len);
}

extern "C" int bz2g_decompress_device_into(const uint8_t *d_in, size_t n, uint8_t *d_out,
                                           size_t cap, size_t *out_len) {
  return decompress_buffer(d_in, n, d_out, cap, out_len);
}
