/* Block boundaries of a .bz2 stream, and one block re-wrapped as a stream of
 * its own -- TEST INFRASTRUCTURE ONLY.
 *
 * A stream is "BZh" + level digit, then blocks that each start with the
 * 48-bit magic 0x314159265359 followed by the block CRC (32 bits), then the
 * 48-bit end-of-stream magic 0x177245385090, the combined CRC and padding to a
 * byte.  Blocks sit at arbitrary bit offsets.  Cutting a stream at its block
 * magics and giving each block its own header and end-of-stream marker (with
 * the block's CRC as the combined CRC, which is what a one-block stream has)
 * lets libbz2 decode the blocks of a long stream in parallel.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define BLOCK_MAGIC 0x314159265359ull
#define EOS_MAGIC 0x177245385090ull

static uint64_t bits_at(const uint8_t *s, int64_t nbytes, int64_t bit, int nb) {
  uint64_t v = 0;
  for (int k = 0; k < nb; k++) {
    const int64_t b = bit + k;
    const int64_t byte = b >> 3;
    const int on = byte < nbytes ? (s[byte] >> (7 - (b & 7))) & 1 : 0;
    v = (v << 1) | (uint64_t)on;
  }
  return v;
}

typedef struct {
  const uint8_t *s;
  int64_t nbytes, b0, b1;  /* byte range whose bit offsets this job tests */
  int64_t *hits;
  int64_t nhits, cap;
  int kind; /* 0 block magic, 1 end-of-stream magic */
} scan_job_t;

static void *scan_worker(void *arg) {
  scan_job_t *j = (scan_job_t *)arg;
  const uint64_t magic = j->kind ? EOS_MAGIC : BLOCK_MAGIC;
  const uint64_t mask = (1ull << 48) - 1;
  for (int64_t byte = j->b0; byte < j->b1; byte++) {
    /* 56 bits from this byte on: the 48-bit windows at its 8 bit offsets */
    uint64_t w = 0;
    for (int k = 0; k < 7; k++) w = (w << 8) | (byte + k < j->nbytes ? j->s[byte + k] : 0);
    for (int sh = 0; sh < 8; sh++) {
      if (((w >> (8 - sh)) & mask) == magic && (byte * 8 + sh + 48) <= j->nbytes * 8) {
        if (j->nhits == j->cap) {
          j->cap = j->cap ? 2 * j->cap : 1024;
          j->hits = (int64_t *)realloc(j->hits, sizeof(int64_t) * j->cap);
        }
        j->hits[j->nhits++] = byte * 8 + sh;
      }
    }
  }
  return NULL;
}

/* Bit offsets of every match of the block magic (kind 0) or of the
 * end-of-stream magic (kind 1), ascending.  Returns the number of matches;
 * at most cap are stored in out. */
int64_t orc_scan_magic(const uint8_t *s, int64_t nbytes, int kind, int64_t *out, int64_t cap,
                       int threads) {
  if (threads < 1) threads = 1;
  scan_job_t *jobs = (scan_job_t *)calloc((size_t)threads, sizeof(scan_job_t));
  pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * threads);
  const int64_t per = (nbytes + threads - 1) / threads;
  for (int t = 0; t < threads; t++) {
    jobs[t].s = s;
    jobs[t].nbytes = nbytes;
    jobs[t].b0 = per * t < nbytes ? per * t : nbytes;
    jobs[t].b1 = per * (t + 1) < nbytes ? per * (t + 1) : nbytes;
    jobs[t].kind = kind;
    pthread_create(&th[t], NULL, scan_worker, &jobs[t]);
  }
  int64_t n = 0;
  for (int t = 0; t < threads; t++) {
    pthread_join(th[t], NULL);
    for (int64_t k = 0; k < jobs[t].nhits; k++) {
      if (n < cap) out[n] = jobs[t].hits[k];
      n++;
    }
    free(jobs[t].hits);
  }
  free(jobs);
  free(th);
  return n;
}

/* The block at stream bits [b0, b1) (from its magic to the next block's
 * magic or the end-of-stream magic) as a stream of its own with header digit
 * `level`.  out needs (b1 - b0) / 8 + 32 bytes; returns the bytes written. */
int64_t orc_rewrap_block(const uint8_t *s, int64_t nbytes, int64_t b0, int64_t b1, int level,
                         uint8_t *out) {
  const int64_t nb = b1 - b0;
  const int64_t cap = nb / 8 + 32;
  memset(out, 0, (size_t)cap);
  out[0] = 'B';
  out[1] = 'Z';
  out[2] = 'h';
  out[3] = (uint8_t)('0' + level);
  int64_t o = 32; /* output bit */
  /* copy whole bytes of the source bit range at its phase */
  const int sh = (int)(b0 & 7);
  const int64_t byte0 = b0 >> 3;
  const int64_t full = nb / 8;
  for (int64_t i = 0; i < full; i++) {
    const uint32_t hi = s[byte0 + i];
    const uint32_t lo = byte0 + i + 1 < nbytes ? s[byte0 + i + 1] : 0;
    out[4 + i] = (uint8_t)(((hi << 8 | lo) >> (8 - sh)) & 0xff);
  }
  o += full * 8;
  for (int64_t b = b0 + full * 8; b < b1; b++, o++)
    if (bits_at(s, nbytes, b, 1)) out[o >> 3] |= (uint8_t)(0x80u >> (o & 7));
  const uint64_t crc = bits_at(s, nbytes, b0 + 48, 32);
  const uint64_t tail[2] = {EOS_MAGIC, crc};
  const int tl[2] = {48, 32};
  for (int q = 0; q < 2; q++)
    for (int k = tl[q] - 1; k >= 0; k--, o++)
      if ((tail[q] >> k) & 1) out[o >> 3] |= (uint8_t)(0x80u >> (o & 7));
  return (o + 7) >> 3;
}
