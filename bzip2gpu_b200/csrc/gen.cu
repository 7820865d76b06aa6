// Seeded synthetic inputs: order-1 Markov source over an alphabet, with run
// starts, and uniform bytes.  Byte generation is integer-only, so the host and
// device generators give identical bytes for the same arguments.
//
// Definition (the data of every workload in this project):
//   PRNG          xoshiro256** seeded through splitmix64.
//   rows          P[a, .] ~ Dirichlet(alpha * 1_A): normalised Gamma(alpha)
//                 draws (Marsaglia-Tsang 2000; for alpha < 1 the
//                 Gamma(alpha+1) * U^(1/alpha) boost), drawn on the host from
//                 splitmix64(seed ^ 0x5EED) in row order, stored as 32-bit
//                 cumulative thresholds (last forced to 2^32-1).
//   chains        the output is cut into chains of 65536 bytes; chain c uses
//                 its own xoshiro state from splitmix64(seed + c * 0x9E3779B97F4A7C15)
//                 and starts at alphabet[next() % A].
//   each step     r = next(); if (uint32)r < p_run * 2^32 a run starts: the
//                 current byte is repeated until the run has L bytes,
//                 L = run_min + (r >> 32) % (run_max - run_min + 1) (cut at the
//                 chain end), and the chain continues from that byte;
//                 otherwise the next symbol is the first j with
//                 (r >> 32) <= cdf[cur][j].
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "bz2g.h"
#include "common.cuh"

namespace bz2g {
namespace {

constexpr int64_t kChain = 65536;

struct Xoshiro {
  uint64_t s[4];
  __host__ __device__ static uint64_t splitmix(uint64_t &x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  __host__ __device__ void seed(uint64_t x) {
    for (int i = 0; i < 4; i++) s[i] = splitmix(x);
  }
  __host__ __device__ static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  __host__ __device__ uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
};

double normal(Xoshiro &g) {
  // Box-Muller
  double u1 = g.uniform(), u2 = g.uniform();
  if (u1 < 1e-300) u1 = 1e-300;
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

double gamma_draw(Xoshiro &g, double a) {
  if (a < 1.0) {
    double u = g.uniform();
    return gamma_draw(g, a + 1.0) * std::pow(u, 1.0 / a);
  }
  const double d = a - 1.0 / 3.0, c = 1.0 / std::sqrt(9.0 * d);
  for (;;) {
    double x, v;
    do {
      x = normal(g);
      v = 1.0 + c * x;
    } while (v <= 0.0);
    v = v * v * v;
    double u = g.uniform();
    if (u < 1.0 - 0.0331 * x * x * x * x) return d * v;
    if (std::log(u) < 0.5 * x * x + d * (1.0 - v + std::log(v))) return d * v;
  }
}

struct MarkovParams {
  uint64_t seed;
  int A;
  uint8_t alphabet[256];
  uint32_t p_run;
  int run_min, run_max;
};

void build_cdf(uint64_t seed, int A, double alpha, std::vector<uint32_t> &cdf) {
  Xoshiro g;
  g.seed(seed ^ 0x5EEDull);
  cdf.assign((size_t)A * A, 0);
  std::vector<double> w(A);
  for (int a = 0; a < A; a++) {
    double sum = 0;
    for (int j = 0; j < A; j++) {
      w[j] = gamma_draw(g, alpha);
      sum += w[j];
    }
    if (!(sum > 0)) {
      for (int j = 0; j < A; j++) w[j] = 0;
      w[g.next() % A] = 1.0;
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
}

__host__ __device__ inline void gen_chain(const MarkovParams &p, const uint32_t *cdf, int64_t c,
                                          uint8_t *out, int64_t len) {
  Xoshiro g;
  g.seed(p.seed + (uint64_t)c * 0x9E3779B97F4A7C15ull);
  int cur = (int)(g.next() % (uint64_t)p.A);
  int64_t pos = 0;
  out[pos++] = p.alphabet[cur];
  const uint32_t span = (uint32_t)(p.run_max - p.run_min + 1);
  while (pos < len) {
    uint64_t r = g.next();
    uint32_t hi = (uint32_t)(r >> 32);
    if ((uint32_t)r < p.p_run) {
      int64_t L = p.run_min + (int64_t)(hi % span);
      int64_t rep = L - 1;
      if (rep > len - pos) rep = len - pos;
      const uint8_t byte = p.alphabet[cur];
      for (int64_t k = 0; k < rep; k++) out[pos++] = byte;
    } else {
      const uint32_t *row = cdf + (size_t)cur * p.A;
      int lo = 0, hi_i = p.A - 1;
      while (lo < hi_i) {
        int mid = (lo + hi_i) >> 1;
        if (hi <= row[mid]) hi_i = mid;
        else lo = mid + 1;
      }
      cur = lo;
      out[pos++] = p.alphabet[cur];
    }
  }
}

__global__ void k_gen_markov(MarkovParams p, const uint32_t *cdf, uint8_t *out, int64_t n) {
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t nch = (n + kChain - 1) / kChain;
  if (c >= nch) return;
  int64_t len = n - c * kChain < kChain ? n - c * kChain : kChain;
  gen_chain(p, cdf, c, out + c * kChain, len);
}

__host__ __device__ inline void gen_uniform_chain(uint64_t seed, int64_t c, uint8_t *out,
                                                  int64_t len) {
  Xoshiro g;
  g.seed(seed + (uint64_t)c * 0x9E3779B97F4A7C15ull);
  for (int64_t i = 0; i < len; i += 8) {
    uint64_t r = g.next();
    for (int k = 0; k < 8 && i + k < len; k++) out[i + k] = (uint8_t)(r >> (8 * k));
  }
}

__global__ void k_gen_uniform(uint64_t seed, uint8_t *out, int64_t n) {
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t nch = (n + kChain - 1) / kChain;
  if (c >= nch) return;
  int64_t len = n - c * kChain < kChain ? n - c * kChain : kChain;
  gen_uniform_chain(seed, c, out + c * kChain, len);
}

template <typename F>
void host_chains(int64_t n, F &&f) {
  int64_t nch = (n + kChain - 1) / kChain;
  int nt = (int)std::min<int64_t>(std::max(1u, std::thread::hardware_concurrency()), nch);
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++)
    th.emplace_back([&, t] {
      for (int64_t c = t; c < nch; c += nt) f(c, std::min(kChain, n - c * kChain));
    });
  for (auto &x : th) x.join();
}

thread_local std::string g_gen_err;

}  // namespace
}  // namespace bz2g

using namespace bz2g;

extern "C" {

/* Order-1 Markov bytes (see the definition at the top of this file).
 * on_device: out is a device pointer, generated on the current device. */
int bz2g_gen_markov(uint64_t seed, const uint8_t *alphabet, int A, double alpha, double p_run,
                    int run_min, int run_max, uint8_t *out, int64_t n, int on_device,
                    void *stream) {
  try {
    if (A < 1 || A > 256 || alpha <= 0 || run_min < 1 || run_max < run_min || n < 0)
      return BZ2G_ERR_ARG;
    if (n == 0) return BZ2G_OK;
    MarkovParams p;
    p.seed = seed;
    p.A = A;
    std::memcpy(p.alphabet, alphabet, A);
    double pr = p_run * 4294967296.0;
    p.p_run = pr >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)(pr < 0 ? 0 : pr);
    p.run_min = run_min;
    p.run_max = run_max;
    std::vector<uint32_t> cdf;
    build_cdf(seed, A, alpha, cdf);
    if (on_device) {
      cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
      uint32_t *d_cdf = nullptr;
      BZ_CUDA(cudaMallocAsync((void **)&d_cdf, cdf.size() * 4, st));
      BZ_CUDA(cudaMemcpyAsync(d_cdf, cdf.data(), cdf.size() * 4, cudaMemcpyHostToDevice, st));
      int64_t nch = (n + kChain - 1) / kChain;
      k_gen_markov<<<(unsigned)((nch + 127) / 128), 128, 0, st>>>(p, d_cdf, out, n);
      BZ_LAUNCH_CHECK();
      BZ_CUDA(cudaFreeAsync(d_cdf, st));
      BZ_CUDA(cudaStreamSynchronize(st));
    } else {
      host_chains(n, [&](int64_t c, int64_t len) { gen_chain(p, cdf.data(), c, out + c * kChain, len); });
    }
    return BZ2G_OK;
  } catch (const std::exception &e) {
    g_gen_err = e.what();
    return BZ2G_ERR_CUDA;
  }
}

/* Uniform random bytes. */
int bz2g_gen_uniform(uint64_t seed, uint8_t *out, int64_t n, int on_device, void *stream) {
  try {
    if (n < 0) return BZ2G_ERR_ARG;
    if (n == 0) return BZ2G_OK;
    if (on_device) {
      cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
      int64_t nch = (n + kChain - 1) / kChain;
      k_gen_uniform<<<(unsigned)((nch + 127) / 128), 128, 0, st>>>(seed, out, n);
      BZ_LAUNCH_CHECK();
      BZ_CUDA(cudaStreamSynchronize(st));
    } else {
      host_chains(n, [&](int64_t c, int64_t len) { gen_uniform_chain(seed, c, out + c * kChain, len); });
    }
    return BZ2G_OK;
  } catch (const std::exception &e) {
    g_gen_err = e.what();
    return BZ2G_ERR_CUDA;
  }
}

}  // extern "C"
