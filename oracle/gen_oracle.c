/* Seeded workload bytes on the CPU -- TEST INFRASTRUCTURE ONLY.
 *
 * A C restatement of the workload definition that the product library's
 * generator implements (order-1 Markov bytes with run starts, and uniform
 * bytes).  The CPU reference timing and the tests build their inputs here, so
 * that nothing on the checker side needs the product library loaded.  A test
 * pins these bytes to the product generator's for several parameter sets.
 *
 * Definition:
 *   PRNG    xoshiro256** seeded through splitmix64.
 *   rows    P[a, .] ~ Dirichlet(alpha * 1_A): normalised Gamma(alpha) draws
 *           (Marsaglia-Tsang; for alpha < 1 the Gamma(alpha + 1) * U^(1/alpha)
 *           boost; normals by Box-Muller), from splitmix64(seed ^ 0x5EED), in
 *           row order, kept as 32-bit cumulative thresholds (the last one
 *           2^32 - 1).
 *   chains  the output is cut into chains of 65536 bytes; chain c runs its own
 *           xoshiro state seeded from seed + c * 0x9E3779B97F4A7C15 and starts
 *           at alphabet[next() % A].
 *   step    r = next(); if (uint32)r < p_run * 2^32 a run starts: the current
 *           byte repeats until the run holds L = run_min + (r >> 32) %
 *           (run_max - run_min + 1) bytes (cut at the chain end); otherwise
 *           the next symbol is the first j with (r >> 32) <= cdf[cur][j].
 *   uniform chain c: the bytes of successive next() values, little end first.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define CHAIN 65536

typedef struct {
  uint64_t s[4];
} xo_t;

static uint64_t splitmix(uint64_t *x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static void xo_seed(xo_t *g, uint64_t x) {
  for (int i = 0; i < 4; i++) g->s[i] = splitmix(&x);
}

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t xo_next(xo_t *g) {
  uint64_t *s = g->s;
  const uint64_t r = rotl64(s[1] * 5, 7) * 9;
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl64(s[3], 45);
  return r;
}

static double xo_uniform(xo_t *g) { return (xo_next(g) >> 11) * (1.0 / 9007199254740992.0); }

static double xo_normal(xo_t *g) {
  double u1 = xo_uniform(g), u2 = xo_uniform(g);
  if (u1 < 1e-300) u1 = 1e-300;
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

static double gamma_draw(xo_t *g, double a) {
  if (a < 1.0) {
    double u = xo_uniform(g);
    return gamma_draw(g, a + 1.0) * pow(u, 1.0 / a);
  }
  const double d = a - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
  for (;;) {
    double x, v;
    do {
      x = xo_normal(g);
      v = 1.0 + c * x;
    } while (v <= 0.0);
    v = v * v * v;
    double u = xo_uniform(g);
    if (u < 1.0 - 0.0331 * x * x * x * x) return d * v;
    if (log(u) < 0.5 * x * x + d * (1.0 - v + log(v))) return d * v;
  }
}

/* cdf[a * A + j]: the Dirichlet rows as 32-bit cumulative thresholds. */
static void build_cdf(uint64_t seed, int A, double alpha, uint32_t *cdf) {
  xo_t g;
  xo_seed(&g, seed ^ 0x5EEDull);
  double *w = (double *)malloc(sizeof(double) * A);
  for (int a = 0; a < A; a++) {
    double sum = 0;
    for (int j = 0; j < A; j++) {
      w[j] = gamma_draw(&g, alpha);
      sum += w[j];
    }
    if (!(sum > 0)) {
      for (int j = 0; j < A; j++) w[j] = 0;
      w[xo_next(&g) % (uint64_t)A] = 1.0;
      sum = 1.0;
    }
    double acc = 0;
    for (int j = 0; j < A; j++) {
      acc += w[j] / sum;
      double v = acc * 4294967296.0;
      cdf[(size_t)a * A + j] = v >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)v;
    }
    cdf[(size_t)a * A + A - 1] = 0xFFFFFFFFu;
  }
  free(w);
}

typedef struct {
  uint64_t seed;
  int A;
  const uint8_t *alphabet;
  const uint32_t *cdf;
  uint32_t p_run;
  int run_min, run_max;
  uint8_t *out;
  int64_t n;
  int uniform;
  int nthreads, t;
} gen_job_t;

static void markov_chain(const gen_job_t *p, int64_t c, uint8_t *out, int64_t len) {
  xo_t g;
  xo_seed(&g, p->seed + (uint64_t)c * 0x9E3779B97F4A7C15ull);
  int cur = (int)(xo_next(&g) % (uint64_t)p->A);
  int64_t pos = 0;
  out[pos++] = p->alphabet[cur];
  const uint32_t span = (uint32_t)(p->run_max - p->run_min + 1);
  while (pos < len) {
    const uint64_t r = xo_next(&g);
    const uint32_t hi = (uint32_t)(r >> 32);
    if ((uint32_t)r < p->p_run) {
      int64_t rep = p->run_min + (int64_t)(hi % span) - 1;
      if (rep > len - pos) rep = len - pos;
      memset(out + pos, p->alphabet[cur], (size_t)rep);
      pos += rep;
    } else {
      const uint32_t *row = p->cdf + (size_t)cur * p->A;
      int lo = 0, up = p->A - 1;
      while (lo < up) {
        const int mid = (lo + up) >> 1;
        if (hi <= row[mid]) up = mid;
        else lo = mid + 1;
      }
      cur = lo;
      out[pos++] = p->alphabet[cur];
    }
  }
}

static void uniform_chain(uint64_t seed, int64_t c, uint8_t *out, int64_t len) {
  xo_t g;
  xo_seed(&g, seed + (uint64_t)c * 0x9E3779B97F4A7C15ull);
  for (int64_t i = 0; i < len; i += 8) {
    const uint64_t r = xo_next(&g);
    for (int k = 0; k < 8 && i + k < len; k++) out[i + k] = (uint8_t)(r >> (8 * k));
  }
}

static void *gen_worker(void *arg) {
  const gen_job_t *p = (const gen_job_t *)arg;
  const int64_t nch = (p->n + CHAIN - 1) / CHAIN;
  for (int64_t c = p->t; c < nch; c += p->nthreads) {
    const int64_t len = p->n - c * CHAIN < CHAIN ? p->n - c * CHAIN : CHAIN;
    if (p->uniform) uniform_chain(p->seed, c, p->out + c * CHAIN, len);
    else markov_chain(p, c, p->out + c * CHAIN, len);
  }
  return NULL;
}

static void run_jobs(gen_job_t *base, int threads) {
  if (threads < 1) threads = 1;
  pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * threads);
  gen_job_t *jobs = (gen_job_t *)malloc(sizeof(gen_job_t) * threads);
  for (int t = 0; t < threads; t++) {
    jobs[t] = *base;
    jobs[t].nthreads = threads;
    jobs[t].t = t;
    pthread_create(&th[t], NULL, gen_worker, &jobs[t]);
  }
  for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
  free(jobs);
  free(th);
}

/* Order-1 Markov bytes.  Returns 0, or -1 on bad arguments. */
int orc_gen_markov(uint64_t seed, const uint8_t *alphabet, int A, double alpha, double p_run,
                   int run_min, int run_max, uint8_t *out, int64_t n, int threads) {
  if (A < 1 || A > 256 || !(alpha > 0) || run_min < 1 || run_max < run_min || n < 0) return -1;
  if (n == 0) return 0;
  uint32_t *cdf = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)A * A);
  build_cdf(seed, A, alpha, cdf);
  const double pr = p_run * 4294967296.0;
  gen_job_t job = {seed, A, alphabet, cdf,
                   pr >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)(pr < 0 ? 0 : pr),
                   run_min, run_max, out, n, 0, 1, 0};
  run_jobs(&job, threads);
  free(cdf);
  return 0;
}

/* Uniform bytes. */
int orc_gen_uniform(uint64_t seed, uint8_t *out, int64_t n, int threads) {
  if (n < 0) return -1;
  if (n == 0) return 0;
  gen_job_t job = {seed, 0, NULL, NULL, 0, 0, 0, out, n, 1, 1, 0};
  run_jobs(&job, threads);
  return 0;
}
