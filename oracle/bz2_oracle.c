/*
 * bz2_oracle.c -- CPU restatement of the bzip2gpu compression path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.
 * See bz2_oracle.h for the contract and for how the restatement is pinned.
 * Paths in comments are relative to the reference project root.
 */
#include "bz2_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ CRC32 */
/* src/compression/crc32.cpp:6-20: table of the MSB-first CRC-32. */
static uint32_t g_crc_table[256];

__attribute__((constructor)) static void crc_table_init(void) {
  for (uint32_t i = 0; i < 256; i++) {
    uint32_t c = i << 24;
    for (int j = 0; j < 8; j++) c = (c & 0x80000000u) ? (c << 1) ^ 0x04C11DB7u : (c << 1);
    g_crc_table[i] = c;
  }
}

/* src/compression/crc32.cpp:22-29 */
uint32_t orc_crc32(const uint8_t *data, size_t n) {
  uint32_t crc = 0xFFFFFFFFu;
  for (size_t i = 0; i < n; i++) crc = (crc << 8) ^ g_crc_table[(crc >> 24) ^ data[i]];
  return ~crc;
}

/* ------------------------------------------------------------------- RLE1 */
/* Runs are cut greedily at 259 = 4 + 255 (tests/compression/rle1.cu:15), a cut
 * of length < 4 is copied, otherwise 4 copies + (len - 4)
 * (src/compression/rle1.cu:34-57). */
int orc_rle1(const uint8_t *in, int n, uint8_t *out) { return orc_rle1_cut(in, n, out, 259); }

/* The same with runs cut at `cut` (bzip2 1.0.8 cuts at 255: its pending run
 * is written when it reaches 255, bzlib.c ADD_CHAR_TO_BLOCK). */
int orc_rle1_cut(const uint8_t *in, int n, uint8_t *out, int cut) {
  int o = 0, i = 0;
  while (i < n) {
    uint8_t c = in[i];
    int j = i + 1;
    while (j < n && in[j] == c && j - i < cut) j++;
    int run = j - i;
    if (run < 4) {
      for (int k = 0; k < run; k++) out[o++] = c;
    } else {
      out[o++] = c; out[o++] = c; out[o++] = c; out[o++] = c;
      out[o++] = (uint8_t)(run - 4);
    }
    i = j;
  }
  return o;
}

/* -------------------------------------------------------------------- BWT */
/* Prefix doubling over cyclic rotations (src/compression/fbwt.cu:47-95): round
 * h sorts by (rank_h[i], rank_h[(i+h) mod m]) stably, so equal rotations keep
 * index order, then re-ranks densely.  The reference runs every round while
 * h < m; rounds after the partition is all singletons or stops splitting
 * leave the order unchanged, so this loop stops there.  The counting sorts are
 * LSD over index order, which gives the same (key, index) order as the
 * reference's stable sort of the previous order. */
void orc_bwt_stats(const uint8_t *T, int n, int32_t *sa, int64_t *active_sum,
                   int *rounds_out) {
  int64_t A = 0;
  int rounds = 0;
  if (n <= 0) {
    if (active_sum) *active_sum = 0;
    if (rounds_out) *rounds_out = 0;
    return;
  }
  int cap = n > 256 ? n : 256;
  int32_t *rank = (int32_t *)malloc(sizeof(int32_t) * n);
  int32_t *nrank = (int32_t *)malloc(sizeof(int32_t) * n);
  int32_t *tmp = (int32_t *)malloc(sizeof(int32_t) * n);
  int32_t *cnt = (int32_t *)malloc(sizeof(int32_t) * (cap + 1));

  /* initial order: by first byte, index ascending */
  memset(cnt, 0, sizeof(int32_t) * 257);
  for (int i = 0; i < n; i++) cnt[T[i] + 1]++;
  for (int c = 0; c < 256; c++) cnt[c + 1] += cnt[c];
  for (int i = 0; i < n; i++) sa[cnt[T[i]]++] = i;
  int R = 0;
  rank[sa[0]] = 0;
  for (int j = 1; j < n; j++) {
    if (T[sa[j]] != T[sa[j - 1]]) R++;
    rank[sa[j]] = R;
  }
  R++;

  for (int64_t h = 1;; h *= 2) {
    if (R == n) break; /* all singletons */
    /* rotations in groups of size >= 2 at the start of this round */
    {
      int64_t a = 0;
      int j = 0;
      while (j < n) {
        int k = j + 1;
        while (k < n && rank[sa[k]] == rank[sa[j]]) k++;
        if (k - j >= 2) a += k - j;
        j = k;
      }
      A += a;
    }
    rounds++;
    int hh = (int)(h % n);
    /* stable by second key, from index order */
    memset(cnt, 0, sizeof(int32_t) * (R + 1));
    for (int i = 0; i < n; i++) {
      int i2 = i + hh; if (i2 >= n) i2 -= n;
      cnt[rank[i2] + 1]++;
    }
    for (int r = 0; r < R; r++) cnt[r + 1] += cnt[r];
    for (int i = 0; i < n; i++) {
      int i2 = i + hh; if (i2 >= n) i2 -= n;
      tmp[cnt[rank[i2]]++] = i;
    }
    /* stable by first key */
    memset(cnt, 0, sizeof(int32_t) * (R + 1));
    for (int j = 0; j < n; j++) cnt[rank[tmp[j]] + 1]++;
    for (int r = 0; r < R; r++) cnt[r + 1] += cnt[r];
    for (int j = 0; j < n; j++) sa[cnt[rank[tmp[j]]]++] = tmp[j];
    /* dense re-rank */
    int nr = 0;
    nrank[sa[0]] = 0;
    for (int j = 1; j < n; j++) {
      int a = sa[j], b = sa[j - 1];
      int a2 = a + hh; if (a2 >= n) a2 -= n;
      int b2 = b + hh; if (b2 >= n) b2 -= n;
      if (rank[a] != rank[b] || rank[a2] != rank[b2]) nr++;
      nrank[a] = nr;
    }
    nr++;
    int32_t *t = rank; rank = nrank; nrank = t;
    if (nr == R) break;       /* fixed point: remaining ties are equal rotations */
    R = nr;
    if (2 * h >= n) break;    /* whole rotations compared */
  }
  free(rank); free(nrank); free(tmp); free(cnt);
  if (active_sum) *active_sum = A;
  if (rounds_out) *rounds_out = rounds;
}

void orc_bwt(const uint8_t *in, int m, int32_t *sa) { orc_bwt_stats(in, m, sa, NULL, NULL); }

/* -------------------------------------------------------------------- MTF */
int orc_symbols_table(const uint8_t *in, int n, uint8_t *table) {
  uint8_t seen[256] = {0};
  for (int i = 0; i < n; i++) seen[in[i]] = 1;
  int c = 0;
  for (int i = 0; i < 256; i++) if (seen[i]) table[c++] = (uint8_t)i;
  return c;
}

/* src/compression/fmtf.cu:51-56,80-96: L[i] = orig[sa[i]-1], or orig[m-1]
 * when sa[i]==0; list starts as the ascending in-use symbols of orig
 * (fmtf.cu:176-210); origPtr = first i with sa[i]==0 (fmtf.cu:222-225). */
int orc_mtf(const uint8_t *orig, const int32_t *sa, int m, uint8_t *out,
            int *orig_ptr, uint8_t *present) {
  if (m <= 0) return 0;
  uint8_t seen[256] = {0};
  for (int i = 0; i < m; i++) seen[orig[i]] = 1;
  uint8_t list[256];
  int nuse = 0;
  for (int i = 0; i < 256; i++) {
    if (present) present[i] = seen[i];
    if (seen[i]) list[nuse++] = (uint8_t)i;
  }
  int op = m;
  for (int i = 0; i < m; i++) {
    int s = sa[i];
    if (s == 0 && op == m) op = i;
    uint8_t c = s == 0 ? orig[m - 1] : orig[s - 1];
    int pos = 0;
    while (list[pos] != c) pos++;
    out[i] = (uint8_t)pos;
    for (int k = pos; k > 0; k--) list[k] = list[k - 1];
    list[0] = c;
  }
  if (orig_ptr) *orig_ptr = op;
  return nuse;
}

/* ------------------------------------------------------------------- RLE2 */
/* tests/compression/rle2.cu:9-33 (== src/compression/rle2.cu:41-74): v>0 ->
 * v+1; a zero run of k -> bijective base-2 digits of k, least significant
 * first, RUNA=0 for digit 1 and RUNB=1 for digit 2; EOB = table_size+1. */
int orc_rle2(const uint8_t *in, int m, int table_size, uint16_t *out) {
  int o = 0, i = 0;
  while (i < m) {
    if (in[i] != 0) {
      out[o++] = (uint16_t)(in[i] + 1);
      i++;
    } else {
      int k = 0;
      while (i < m && in[i] == 0) { k++; i++; }
      while (k > 0) {
        k--;
        out[o++] = (k & 1) ? 1 : 0;
        k >>= 1;
      }
    }
  }
  out[o++] = (uint16_t)(table_size + 1);
  return o;
}

/* ---------------------------------------------------------------- Huffman */
/* src/compression/huffman.cu:13-124.  Weights are (freq or 1) << 8 with the
 * subtree depth in the low byte; a 1-based binary min-heap with strict '<'
 * comparisons (UPHEAP huffman.cu:38-48, DOWNHEAP huffman.cu:20-36); two
 * minima are merged per step; if a length exceeds max_len every weight w
 * becomes (1 + (w>>8)/2) << 8 and the build restarts (huffman.cu:116-122). */
void orc_code_lengths(const int32_t *freq, uint8_t *len, int alpha_size,
                      int max_len) {
  int32_t heap[ORC_MAX_ALPHA + 2];
  int32_t weight[ORC_MAX_ALPHA * 2];
  int32_t parent[ORC_MAX_ALPHA * 2];
  for (int i = 0; i < alpha_size; i++) weight[i + 1] = (freq[i] == 0 ? 1 : freq[i]) << 8;

  for (;;) {
    int n_nodes = alpha_size, n_heap = 0;
    heap[0] = 0; weight[0] = 0; parent[0] = -2;
    for (int i = 1; i <= alpha_size; i++) {
      parent[i] = -1;
      n_heap++;
      heap[n_heap] = i;
      /* sift up */
      int zz = n_heap, tmp = heap[zz];
      while (weight[tmp] < weight[heap[zz >> 1]]) { heap[zz] = heap[zz >> 1]; zz >>= 1; }
      heap[zz] = tmp;
    }
    while (n_heap > 1) {
      int n1, n2;
      for (int pick = 0; pick < 2; pick++) {
        int top = heap[1];
        heap[1] = heap[n_heap];
        n_heap--;
        /* sift down from the root */
        int zz = 1, tmp = heap[zz];
        for (;;) {
          int yy = zz << 1;
          if (yy > n_heap) break;
          if (yy < n_heap && weight[heap[yy + 1]] < weight[heap[yy]]) yy++;
          if (weight[tmp] < weight[heap[yy]]) break;
          heap[zz] = heap[yy];
          zz = yy;
        }
        heap[zz] = tmp;
        if (pick == 0) n1 = top; else n2 = top;
      }
      n_nodes++;
      parent[n1] = parent[n2] = n_nodes;
      int32_t w1 = weight[n1], w2 = weight[n2];
      int32_t d1 = w1 & 0xff, d2 = w2 & 0xff;
      weight[n_nodes] = (int32_t)(((uint32_t)(w1 & 0xffffff00) + (uint32_t)(w2 & 0xffffff00)) |
                                  (uint32_t)(1 + (d1 > d2 ? d1 : d2)));
      parent[n_nodes] = -1;
      n_heap++;
      heap[n_heap] = n_nodes;
      int zz = n_heap, tmp = heap[zz];
      while (weight[tmp] < weight[heap[zz >> 1]]) { heap[zz] = heap[zz >> 1]; zz >>= 1; }
      heap[zz] = tmp;
    }
    int too_long = 0;
    for (int i = 1; i <= alpha_size; i++) {
      int j = 0, k = i;
      while (parent[k] >= 0) { k = parent[k]; j++; }
      len[i - 1] = (uint8_t)j;
      if (j > max_len) too_long = 1;
    }
    if (!too_long) break;
    for (int i = 1; i <= alpha_size; i++) {
      int j = weight[i] >> 8;
      j = 1 + (j / 2);
      weight[i] = j << 8;
    }
  }
}

/* src/compression/huffman.cu:148-185 (bzip2's initial partition of the
 * alphabet by cumulative frequency, with the odd-part back-off). */
void orc_initial_assignment(int n_groups, int s, int alpha_size,
                            const int32_t *freqs_in,
                            uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA]) {
  int32_t freqs[ORC_MAX_ALPHA + 1];
  for (int i = 0; i <= ORC_MAX_ALPHA; i++) freqs[i] = i < alpha_size ? freqs_in[i] : 0;
  int gs = 0, remaining = s;
  for (int n_part = n_groups; n_part > 0; n_part--) {
    int t_freq = remaining / n_part;
    int ge = gs - 1, a_freq = 0;
    while (a_freq < t_freq && ge < alpha_size) {
      ge++;
      a_freq += freqs[ge];
    }
    if (ge > gs && n_part != n_groups && n_part != 1 && ((n_groups - n_part) % 2 == 1)) {
      a_freq -= freqs[ge];
      ge--;
    }
    for (int v = 0; v < alpha_size; v++) len[n_part - 1][v] = (v >= gs && v <= ge) ? 0 : 15;
    gs = ge + 1;
    remaining -= a_freq;
  }
}

/* One selection pass (src/compression/huffman.cu:188-243): per 50-symbol
 * group the cost of every table, the first minimum wins, and the chosen
 * table's symbol counts. */
static void select_pass(const uint16_t *syms, int s, int ng,
                        uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA], uint8_t *selectors,
                        int32_t rfreq[ORC_MAX_GROUPS][ORC_MAX_ALPHA]) {
  int nsel = (s + 49) / 50;
  memset(rfreq, 0, sizeof(int32_t) * ORC_MAX_GROUPS * ORC_MAX_ALPHA);
  for (int g = 0; g < nsel; g++) {
    int gs = g * 50, ge = gs + 49;
    if (ge >= s) ge = s - 1;
    uint32_t cost[ORC_MAX_GROUPS] = {0};
    for (int i = gs; i <= ge; i++)
      for (int t = 0; t < ng; t++) cost[t] += len[t][syms[i]];
    uint32_t bc = 0xFFFFFFFFu;
    int bt = -1;
    for (int t = 0; t < ng; t++)
      if (cost[t] < bc) { bc = cost[t]; bt = t; }
    selectors[g] = (uint8_t)bt;
    for (int i = gs; i <= ge; i++) rfreq[bt][syms[i]]++;
  }
}

/* canonical codes, src/compression/huffman.cu:135-146,352-362 */
static void canonical_codes(int ng, int alpha, uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                            int32_t code[ORC_MAX_GROUPS][ORC_MAX_ALPHA]) {
  for (int t = 0; t < ng; t++) {
    int mn = 32, mx = 0;
    for (int v = 0; v < alpha; v++) {
      if (len[t][v] > mx) mx = len[t][v];
      if (len[t][v] < mn) mn = len[t][v];
    }
    int vec = 0;
    for (int l = mn; l <= mx; l++) {
      for (int v = 0; v < alpha; v++)
        if (len[t][v] == l) code[t][v] = vec++;
      vec <<= 1;
    }
  }
}

/* src/compression/huffman.cu:256-364 with a zeroed histogram, with
 * `passes` selection passes (the reference's 4). */
int orc_huffman_build_passes(const uint16_t *syms, int s, int alphabet_size, int passes,
                             uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                             int32_t code[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                             uint8_t *selectors, int *n_groups_out) {
  int alpha = alphabet_size + 2;
  for (int g = 0; g < ORC_MAX_GROUPS; g++)
    for (int v = 0; v < alpha; v++) len[g][v] = 15;
  int ng = s < 200 ? 2 : s < 600 ? 3 : s < 1200 ? 4 : s < 2400 ? 5 : 6;
  int32_t freqs[ORC_MAX_ALPHA] = {0};
  for (int i = 0; i < s; i++) freqs[syms[i]]++;
  orc_initial_assignment(ng, s, alpha, freqs, len);
  int nsel = (s + 49) / 50;
  int32_t rfreq[ORC_MAX_GROUPS][ORC_MAX_ALPHA];
  for (int iter = 0; iter < passes; iter++) {
    select_pass(syms, s, ng, len, selectors, rfreq);
    for (int t = 0; t < ng; t++) orc_code_lengths(rfreq[t], len[t], alpha, 17);
  }
  canonical_codes(ng, alpha, len, code);
  *n_groups_out = ng;
  return nsel;
}

int orc_huffman_build(const uint16_t *syms, int s, int alphabet_size,
                      uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                      int32_t code[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                      uint8_t *selectors, int *n_groups_out) {
  return orc_huffman_build_passes(syms, s, alphabet_size, 4, len, code, selectors, n_groups_out);
}

/* The learned form's passes after its first assignment sel_in (six tables):
 * code lengths from the chosen tables' symbol counts, then n_refine passes
 * of exact selection and code lengths, then canonical codes.  Written from
 * bzip2gpu_b200/csrc/huffman.cu's learned schedule; the pass itself is the
 * reference's (src/compression/huffman.cu:188-243). */
int orc_huffman_refine(const uint16_t *syms, int s, int alphabet_size, const uint8_t *sel_in,
                       int n_refine, uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                       int32_t code[ORC_MAX_GROUPS][ORC_MAX_ALPHA], uint8_t *selectors) {
  const int alpha = alphabet_size + 2, ng = ORC_MAX_GROUPS;
  const int nsel = (s + 49) / 50;
  for (int g = 0; g < ORC_MAX_GROUPS; g++)
    for (int v = 0; v < alpha; v++) len[g][v] = 15;
  int32_t rfreq[ORC_MAX_GROUPS][ORC_MAX_ALPHA];
  memset(rfreq, 0, sizeof(rfreq));
  for (int g = 0; g < nsel; g++) {
    int gs = g * 50, ge = gs + 49;
    if (ge >= s) ge = s - 1;
    selectors[g] = sel_in[g];
    for (int i = gs; i <= ge; i++) rfreq[sel_in[g]][syms[i]]++;
  }
  for (int t = 0; t < ng; t++) orc_code_lengths(rfreq[t], len[t], alpha, 17);
  for (int r = 0; r < n_refine; r++) {
    select_pass(syms, s, ng, len, selectors, rfreq);
    for (int t = 0; t < ng; t++) orc_code_lengths(rfreq[t], len[t], alpha, 17);
  }
  canonical_codes(ng, alpha, len, code);
  return nsel;
}

/* Predicted coded size of a selection: payload from the per-table counts
 * and lengths plus the table headers (5-bit start, 2 bits per unit of
 * length change, 1 terminator bit per symbol); the selector codes are not
 * counted.  Written from bzip2gpu_b200/csrc/huffman.cu (predicted_bits). */
static int64_t predicted_bits(int ng, int alpha, int32_t rfreq[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                              uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA]) {
  int64_t e = 5 * ng;
  for (int t = 0; t < ng; t++)
    for (int v = 0; v < alpha; v++) {
      int l = len[t][v], p = v ? len[t][v - 1] : l;
      e += (int64_t)rfreq[t][v] * l + 2 * (l > p ? l - p : p - l) + 1;
    }
  return e;
}

/* The learned form for one block given the MLP's choices sel_mlp (written
 * from bzip2gpu_b200/csrc/huffman.cu's learned schedule): with six tables,
 * the learned tables come from the MLP's choice, one exact selection pass and
 * code lengths.  Beside them the plain selector runs its first two passes
 * (initial tables, then one pass over the first pass's tables).  If the
 * learned tables' predicted size exceeds the plain two-pass one, the block
 * is coded with the plain two-pass selection and *fell_back = 1.  Blocks with
 * fewer tables are plain (four passes).  Returns the selector count. */
int orc_huffman_learned(const uint16_t *syms, int s, int alphabet_size, const uint8_t *sel_mlp,
                        uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                        int32_t code[ORC_MAX_GROUPS][ORC_MAX_ALPHA], uint8_t *selectors,
                        int *n_groups_out, int *fell_back) {
  const int alpha = alphabet_size + 2;
  const int ng = s < 200 ? 2 : s < 600 ? 3 : s < 1200 ? 4 : s < 2400 ? 5 : 6;
  *fell_back = 0;
  if (ng != ORC_MAX_GROUPS)
    return orc_huffman_build(syms, s, alphabet_size, len, code, selectors, n_groups_out);
  static __thread int32_t rfreq[ORC_MAX_GROUPS][ORC_MAX_ALPHA];
  static __thread uint8_t lp[ORC_MAX_GROUPS][ORC_MAX_ALPHA];
  static __thread int32_t cp[ORC_MAX_GROUPS][ORC_MAX_ALPHA];
  const int nsel = (s + 49) / 50;
  uint8_t *sel_plain = (uint8_t *)malloc(nsel + 1);
  /* the plain selector's first two passes, and the counts of its selection */
  int ngp = 0;
  orc_huffman_build_passes(syms, s, alphabet_size, 2, lp, cp, sel_plain, &ngp);
  memset(rfreq, 0, sizeof(rfreq));
  for (int g = 0; g < nsel; g++) {
    const int gs = g * 50, ge = gs + 50 < s ? gs + 50 : s;
    for (int i = gs; i < ge; i++) rfreq[sel_plain[g]][syms[i]]++;
  }
  const int64_t est = predicted_bits(ng, alpha, rfreq, lp);
  /* learned: MLP choice -> tables -> exact pass -> tables */
  orc_huffman_refine(syms, s, alphabet_size, sel_mlp, 0, len, code, selectors);
  select_pass(syms, s, ng, len, selectors, rfreq);
  for (int t = 0; t < ng; t++) orc_code_lengths(rfreq[t], len[t], alpha, 17);
  if (predicted_bits(ng, alpha, rfreq, len) > est) {
    *fell_back = 1;
    memcpy(selectors, sel_plain, nsel);
    memcpy(len, lp, sizeof(lp));
  }
  free(sel_plain);
  canonical_codes(ng, alpha, len, code);
  *n_groups_out = ng;
  return nsel;
}

/* Bits of one block's coded part that depend on the table selection:
 * payload, the unary selector MTF codes, and the table deltas
 * (src/compression/compress.cu:300-345). */
int64_t orc_coded_bits(const uint16_t *syms, int s, const uint8_t *selectors, int ng,
                       int alphabet_size, const uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA]) {
  const int alpha = alphabet_size + 2, nsel = (s + 49) / 50;
  int64_t bits = 0;
  for (int i = 0; i < s; i++) bits += len[selectors[i / 50]][syms[i]];
  uint8_t *mtf = (uint8_t *)malloc(nsel > 0 ? nsel : 1);
  orc_selector_mtf(selectors, nsel, ng, mtf);
  for (int g = 0; g < nsel; g++) bits += mtf[g] + 1;
  free(mtf);
  for (int t = 0; t < ng; t++) {
    int cur = len[t][0];
    bits += 5;
    for (int v = 0; v < alpha; v++) {
      int d = (int)len[t][v] - cur;
      bits += 2 * (d < 0 ? -d : d) + 1;
      cur = len[t][v];
    }
  }
  return bits;
}

/* src/compression/huffman_encode.cu:30-71: code of symbol i from table
 * selectors[i/50], MSB-first at the running bit offset. */
int64_t orc_encode(const uint16_t *syms, int s, const uint8_t *selectors,
                   const uint8_t len[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                   const int32_t code[ORC_MAX_GROUPS][ORC_MAX_ALPHA],
                   uint32_t *words) {
  int64_t bit = 0;
  for (int i = 0; i < s; i++) {
    int t = selectors[i / 50];
    int l = len[t][syms[i]];
    uint32_t c = (uint32_t)code[t][syms[i]];
    for (int k = l - 1; k >= 0; k--) {
      if ((c >> k) & 1u) words[bit >> 5] |= 0x80000000u >> (bit & 31);
      bit++;
    }
  }
  return bit;
}

/* src/compression/compress.cu:120-137 */
void orc_selector_mtf(const uint8_t *sel, int n_sel, int n_groups, uint8_t *out) {
  uint8_t pos[ORC_MAX_GROUPS];
  for (int i = 0; i < n_groups; i++) pos[i] = (uint8_t)i;
  for (int i = 0; i < n_sel; i++) {
    uint8_t v = sel[i];
    int j = 0;
    uint8_t tmp = pos[j];
    while (v != tmp) {
      j++;
      uint8_t tmp2 = tmp;
      tmp = pos[j];
      pos[j] = tmp2;
    }
    pos[0] = tmp;
    out[i] = (uint8_t)j;
  }
}

/* -------------------------------------------------------------- container */
/* MSB-first bit writer (src/compression/compress.cu:26-58). */
typedef struct {
  uint8_t *buf;
  int64_t cap, pos;
  uint64_t acc;
  int nacc;
  int overflow;
} bitw;

static void bw_put(bitw *w, uint32_t v, int nbits) {
  if (nbits == 0) return;
  v &= (uint32_t)((1ull << nbits) - 1);
  w->acc = (w->acc << nbits) | v;
  w->nacc += nbits;
  while (w->nacc >= 8) {
    w->nacc -= 8;
    if (w->pos < w->cap) w->buf[w->pos] = (uint8_t)(w->acc >> w->nacc);
    else w->overflow = 1;
    w->pos++;
  }
}

static void bw_flush(bitw *w) {
  if (w->nacc > 0) {
    uint8_t b = (uint8_t)(w->acc << (8 - w->nacc));
    if (w->pos < w->cap) w->buf[w->pos] = b; else w->overflow = 1;
    w->pos++;
    w->nacc = 0;
    w->acc = 0;
  }
}

typedef struct {
  orc_block_info info;
  uint8_t *sel_mtf;
  uint32_t *payload;
} blk_out;

static int compress_block_cut(const uint8_t *raw, int n, int cut, orc_block_info *info,
                              uint8_t *rle1_out, int32_t *sa_out, uint8_t *mtf_out,
                              uint16_t *rle2_out, uint8_t *sel_out) {
  memset(info, 0, sizeof(*info));
  info->n = n;
  info->crc = orc_crc32(raw, (size_t)n);
  uint8_t *rle1 = rle1_out ? rle1_out : (uint8_t *)malloc((size_t)n + n / 4 + 8);
  int m = orc_rle1_cut(raw, n, rle1, cut);
  info->m = m;
  int32_t *sa = sa_out ? sa_out : (int32_t *)malloc(sizeof(int32_t) * (m > 0 ? m : 1));
  int rounds = 0;
  orc_bwt_stats(rle1, m, sa, &info->active_sum, &rounds);
  uint8_t *mtf = mtf_out ? mtf_out : (uint8_t *)malloc(m > 0 ? m : 1);
  info->n_in_use = orc_mtf(rle1, sa, m, mtf, &info->orig_ptr, info->present);
  uint16_t *rle2 = rle2_out ? rle2_out : (uint16_t *)malloc(sizeof(uint16_t) * (m + 2));
  int s = orc_rle2(mtf, m, info->n_in_use, rle2);
  info->s = s;
  uint8_t *sel = sel_out ? sel_out : (uint8_t *)malloc(s / 50 + 2);
  info->n_selectors = orc_huffman_build(rle2, s, info->n_in_use, info->len, info->code, sel,
                                        &info->n_groups);
  int64_t bits = 0;
  for (int i = 0; i < s; i++) bits += info->len[sel[i / 50]][rle2[i]];
  info->payload_bits = bits;
  if (!rle1_out) free(rle1);
  if (!sa_out) free(sa);
  if (!mtf_out) free(mtf);
  if (!rle2_out) free(rle2);
  if (!sel_out) free(sel);
  return 0;
}

int orc_compress_block(const uint8_t *raw, int n, orc_block_info *info,
                       uint8_t *rle1_out, int32_t *sa_out, uint8_t *mtf_out,
                       uint16_t *rle2_out, uint8_t *sel_out) {
  return compress_block_cut(raw, n, 259, info, rle1_out, sa_out, mtf_out, rle2_out, sel_out);
}

/* Whole block, keeping what the container needs. */
static void run_block(const uint8_t *raw, int n, int cut, blk_out *o) {
  uint8_t *rle1 = (uint8_t *)malloc((size_t)n + n / 4 + 8);
  int32_t *sa = (int32_t *)malloc(sizeof(int32_t) * ((size_t)n + n / 4 + 8));
  uint8_t *mtf = (uint8_t *)malloc((size_t)n + n / 4 + 8);
  uint16_t *rle2 = (uint16_t *)malloc(sizeof(uint16_t) * ((size_t)n + n / 4 + 8));
  uint8_t *sel = (uint8_t *)malloc((size_t)n / 40 + 64);
  compress_block_cut(raw, n, cut, &o->info, rle1, sa, mtf, rle2, sel);
  o->sel_mtf = (uint8_t *)malloc((size_t)o->info.n_selectors + 1);
  orc_selector_mtf(sel, o->info.n_selectors, o->info.n_groups, o->sel_mtf);
  size_t nw = (size_t)(o->info.payload_bits + 31) / 32 + 1;
  o->payload = (uint32_t *)calloc(nw, sizeof(uint32_t));
  orc_encode(rle2, o->info.s, sel, (const uint8_t(*)[ORC_MAX_ALPHA])o->info.len,
             (const int32_t(*)[ORC_MAX_ALPHA])o->info.code, o->payload);
  free(rle1); free(sa); free(mtf); free(rle2); free(sel);
}

typedef struct {
  const uint8_t *in;
  const int64_t *ends;  /* block b = [ends[b-1], ends[b]) */
  int cut;
  int nblocks;
  blk_out *blocks;
  int next;
  pthread_mutex_t mu;
} pool_ctx;

static void *pool_worker(void *arg) {
  pool_ctx *c = (pool_ctx *)arg;
  for (;;) {
    pthread_mutex_lock(&c->mu);
    int b = c->next++;
    pthread_mutex_unlock(&c->mu);
    if (b >= c->nblocks) return NULL;
    int64_t off = b ? c->ends[b - 1] : 0;
    run_block(c->in + off, (int)(c->ends[b] - off), c->cut, &c->blocks[b]);
  }
}

/* bzip2 1.0.8's block split (bzlib.c: ADD_CHAR_TO_BLOCK, add_pair_to_block,
 * copy_input_until_stop, handle_compress), restated as the state machine it
 * runs over the input: a pending run of at most 255 equal bytes is written
 * (L bytes for L <= 3, else 4 + a count byte) when a different byte arrives or
 * it is 255 long; before each byte, a block holding 100000 * level - 19 or
 * more written bytes is closed without the pending run, which begins the next
 * block; the last block takes what is left.  ends[k] = end of block k.
 * Returns the number of blocks (ends[] needs that many entries; entries past
 * cap are not stored). */
int64_t orc_bzip2_split(const uint8_t *in, int64_t n, int level, int64_t *ends,
                        int64_t cap) {
  if (level < 1) level = 1;
  if (level > 9) level = 9;
  const int64_t max_written = 100000LL * level - 19;
  int64_t nb = 0, written = 0;
  int ch = -1, len = 0;
  for (int64_t i = 0; i < n; i++) {
    if (written >= max_written) {
      if (nb < cap) ends[nb] = i - len;
      nb++;
      written = 0;
    }
    if (in[i] == ch && len < 255) {
      len++;
    } else {
      if (ch >= 0) written += len < 4 ? len : 5;
      ch = in[i];
      len = 1;
    }
  }
  if (n > 0) {
    if (nb < cap) ends[nb] = n;
    nb++;
  }
  return nb;
}

static int64_t split_bound(int64_t n) {
  /* blocks hold >= 99981 RLE1 bytes (level 1) and RLE1 writes <= 5 per 4 */
  return n * 5 / 4 / 99981 + 2;
}

int64_t orc_compress_bound(int64_t n, int block_bytes) {
  int64_t nb = block_bytes == ORC_BZIP2_BLOCKS ? split_bound(n)
                                               : (n + block_bytes - 1) / block_bytes;
  /* per block: header <= 1300 bytes; payload <= 17 bits per symbol, and
   * symbols <= 5/4 raw bytes + 2 */
  return 64 + nb * 1400 + (n / 4 + 4 * nb) * 17 / 8 + n * 17 / 8;
}

/* src/compression/compress.cu:184-378.  part != 0: no stream header and no
 * end-of-stream marker; *part_bits and *part_fold get the bit count and the
 * blocks' CRC fold. */
static int64_t compress_impl(const uint8_t *in, int64_t n, int level, int block_bytes,
                             uint8_t *out, int64_t cap, int threads, int part,
                             int64_t *part_bits, uint32_t *part_fold) {
  if (level < 1) level = 1;
  if (level > 9) level = 9;
  int cut = 259;
  int64_t *ends;
  int nblocks;
  if (block_bytes == ORC_BZIP2_BLOCKS) {
    cut = 255;
    int64_t nb = orc_bzip2_split(in, n, level, NULL, 0);
    ends = (int64_t *)malloc(sizeof(int64_t) * (nb > 0 ? nb : 1));
    orc_bzip2_split(in, n, level, ends, nb);
    nblocks = (int)nb;
  } else {
    if (block_bytes <= 0) block_bytes = 900000;
    nblocks = (int)((n + block_bytes - 1) / block_bytes);
    ends = (int64_t *)malloc(sizeof(int64_t) * (nblocks > 0 ? nblocks : 1));
    for (int b = 0; b < nblocks; b++)
      ends[b] = (int64_t)(b + 1) * block_bytes < n ? (int64_t)(b + 1) * block_bytes : n;
  }
  bitw w = {out, cap, 0, 0, 0, 0};
  if (!part) {
    bw_put(&w, 0x42, 8); bw_put(&w, 0x5A, 8); bw_put(&w, 0x68, 8); bw_put(&w, 0x30 + level, 8);
  }
  blk_out *blocks = (blk_out *)calloc(nblocks > 0 ? nblocks : 1, sizeof(blk_out));
  pool_ctx ctx;
  ctx.in = in; ctx.ends = ends; ctx.cut = cut; ctx.nblocks = nblocks;
  ctx.blocks = blocks; ctx.next = 0;
  pthread_mutex_init(&ctx.mu, NULL);
  if (threads < 1) threads = 1;
  if (threads > nblocks) threads = nblocks > 0 ? nblocks : 1;
  if (threads == 1) {
    pool_worker(&ctx);
  } else {
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    for (int t = 0; t < threads; t++) pthread_create(&th[t], NULL, pool_worker, &ctx);
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    free(th);
  }
  pthread_mutex_destroy(&ctx.mu);

  uint32_t stream_crc = 0;
  for (int b = 0; b < nblocks; b++) {
    blk_out *o = &blocks[b];
    orc_block_info *bi = &o->info;
    int64_t start = w.pos * 8 + w.nacc;
    stream_crc = (stream_crc << 1) | (stream_crc >> 31);
    stream_crc ^= bi->crc;
    bw_put(&w, 0x31, 8); bw_put(&w, 0x41, 8); bw_put(&w, 0x59, 8);
    bw_put(&w, 0x26, 8); bw_put(&w, 0x53, 8); bw_put(&w, 0x59, 8);
    bw_put(&w, bi->crc, 32);
    bw_put(&w, 0, 1);
    bw_put(&w, (uint32_t)bi->orig_ptr, 24);
    uint32_t l1 = 0;
    for (int r = 0; r < 16; r++) {
      int any = 0;
      for (int q = 0; q < 16; q++) any |= bi->present[r * 16 + q];
      if (any) l1 |= 1u << (15 - r);
    }
    bw_put(&w, l1, 16);
    for (int r = 0; r < 16; r++) {
      if ((l1 >> (15 - r)) & 1) {
        uint32_t l2 = 0;
        for (int q = 0; q < 16; q++)
          if (bi->present[r * 16 + q]) l2 |= 1u << (15 - q);
        bw_put(&w, l2, 16);
      }
    }
    bw_put(&w, (uint32_t)bi->n_groups, 3);
    bw_put(&w, (uint32_t)bi->n_selectors, 15);
    for (int i = 0; i < bi->n_selectors; i++) {
      for (int k = 0; k < o->sel_mtf[i]; k++) bw_put(&w, 1, 1);
      bw_put(&w, 0, 1);
    }
    int alpha = bi->n_in_use + 2;
    for (int t = 0; t < bi->n_groups; t++) {
      int cur = bi->len[t][0];
      bw_put(&w, (uint32_t)cur, 5);
      for (int v = 0; v < alpha; v++) {
        int tgt = bi->len[t][v];
        while (cur < tgt) { bw_put(&w, 2, 2); cur++; }
        while (cur > tgt) { bw_put(&w, 3, 2); cur--; }
        bw_put(&w, 0, 1);
      }
    }
    bi->header_bits = w.pos * 8 + w.nacc - start;
    int64_t rem = bi->payload_bits;
    for (int64_t i = 0; rem > 0; i++) {
      int k = rem < 32 ? (int)rem : 32;
      bw_put(&w, o->payload[i] >> (32 - k), k);
      rem -= k;
    }
    free(o->sel_mtf);
    free(o->payload);
  }
  free(blocks);
  free(ends);
  if (part) {
    *part_bits = w.pos * 8 + w.nacc;
    *part_fold = stream_crc;
    bw_flush(&w);
    return w.overflow ? -1 : w.pos;
  }
  bw_put(&w, 0x17, 8); bw_put(&w, 0x72, 8); bw_put(&w, 0x45, 8);
  bw_put(&w, 0x38, 8); bw_put(&w, 0x50, 8); bw_put(&w, 0x90, 8);
  bw_put(&w, stream_crc, 32);
  bw_flush(&w);
  return w.overflow ? -1 : w.pos;
}

int64_t orc_compress(const uint8_t *in, int64_t n, int level, int block_bytes,
                     uint8_t *out, int64_t cap, int threads) {
  return compress_impl(in, n, level, block_bytes, out, cap, threads, 0, NULL, NULL);
}

/* A part: the blocks' bits from bit 0, no header, no marker.  Returns the
 * bytes written (-1 if cap is too small). */
int64_t orc_compress_part(const uint8_t *in, int64_t n, int block_bytes, uint8_t *out,
                          int64_t cap, int threads, int64_t *bits, uint32_t *fold) {
  return compress_impl(in, n, 9, block_bytes, out, cap, threads, 1, bits, fold);
}

/* Header + parts in order + end-of-stream marker with the CRC combined from
 * the parts' folds (crc = rotl(crc, nblocks_r) ^ fold_r). */
int64_t orc_assemble(int nparts, const uint8_t *const *parts, const int64_t *bits,
                     const uint32_t *folds, const int *nblocks, int level, uint8_t *out,
                     int64_t cap) {
  if (level < 1) level = 1;
  if (level > 9) level = 9;
  bitw w = {out, cap, 0, 0, 0, 0};
  bw_put(&w, 0x42, 8); bw_put(&w, 0x5A, 8); bw_put(&w, 0x68, 8); bw_put(&w, 0x30 + level, 8);
  uint32_t crc = 0;
  for (int r = 0; r < nparts; r++) {
    int64_t full = bits[r] / 8;
    for (int64_t i = 0; i < full; i++) bw_put(&w, parts[r][i], 8);
    int rem = (int)(bits[r] % 8);
    if (rem) bw_put(&w, parts[r][full] >> (8 - rem), rem);
    int k = nblocks[r] % 32;
    crc = (k ? ((crc << k) | (crc >> (32 - k))) : crc) ^ folds[r];
  }
  bw_put(&w, 0x17, 8); bw_put(&w, 0x72, 8); bw_put(&w, 0x45, 8);
  bw_put(&w, 0x38, 8); bw_put(&w, 0x50, 8); bw_put(&w, 0x90, 8);
  bw_put(&w, crc, 32);
  bw_flush(&w);
  return w.overflow ? -1 : w.pos;
}
