// RLE1 entry point that allocates nothing (bz2g_rle1_noalloc, include/bz2g.h).
//
// For callers that cannot allocate device memory when they call in: services
// that reserve their whole device-memory budget up front and forbid later
// cudaMalloc, and code that must not pay cudaMalloc / cudaFree's implicit
// device synchronisation on its hot path.  The scratch that bz2g_rle1 takes
// from a per-call workspace lives here instead, in one file-scope device
// array sized for inputs of up to kNoAllocMaxInput bytes; every GPU that
// loads the library holds it until the process exits.  The RLE1 kernels are
// the same ones bz2g_rle1 runs.
#include <cstring>
#include <map>
#include <utility>
#include <mutex>
#include <string>

#include "bz2g.h"
#include "engine.h"

namespace bz2g {

void set_last_error(const std::string &msg);

namespace {

// Largest input accepted (1 MiB), and the scratch carved from one array.
constexpr int kNoAllocMaxInput = 1 << 20;
constexpr int kNoAllocTiles = kNoAllocMaxInput / kRawTile;  // raw tiles
// layout (byte offsets, each 256-aligned)
constexpr size_t kOffRaw = 0;                                        // input copy + slack
constexpr size_t kOffPlan64 = kOffRaw + kNoAllocMaxInput + 256;      // raw_off, off, cap
constexpr size_t kOffPlan32 = kOffPlan64 + 256;                      // raw_len, rt_first[2]
constexpr size_t kOffRtBlock = kOffPlan32 + 256;
constexpr size_t kOffRtStart = kOffRtBlock + 4 * kNoAllocTiles;
constexpr size_t kOffTileA = kOffRtStart + 4 * kNoAllocTiles;
constexpr size_t kOffTileB = kOffTileA + 4 * kNoAllocTiles;
constexpr size_t kOffTileC = kOffTileB + 4 * kNoAllocTiles;
constexpr size_t kOffTileD = kOffTileC + 4 * kNoAllocTiles;          // tile CRCs
constexpr size_t kOffScalars = kOffTileD + 4 * kNoAllocTiles;        // m, crc, crc_acc
constexpr size_t kNoAllocBytes = kOffScalars + 256;

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocBytes];

// Set-up, once per device context with that device current: the device
// address of the scratch (the host-side symbol is only a stand-in and must
// not be passed to a kernel).  The address is kept per (device, context), so
// a context that was torn down and created again (cudaDeviceReset) gets a
// fresh lookup instead of a stale address.  The current context comes from
// the driver's cuCtxGetCurrent, reached through the runtime's entry-point
// query so that the library needs no link to the driver library.
using CtxGetCurrentFn = int (*)(void **);

void *current_context() {
  static CtxGetCurrentFn fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      f = nullptr;
    }
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  void *ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

std::mutex g_mu;
std::map<std::pair<int, void *>, uint8_t *> g_addr;

uint8_t *lookup_scratch() {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess)
    throw Error(kErrCuda, std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") +
                              cudaGetErrorString(e));
  return static_cast<uint8_t *>(p);
}

uint8_t *scratch_address() {
  int dev = 0;
  BZ_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(g_mu);
  void *ctx = current_context();
  if (ctx) {
    auto it = g_addr.find({dev, ctx});
    if (it != g_addr.end()) return it->second;
  }
  // the lookup itself makes the device's context current if it was not yet
  uint8_t *p = lookup_scratch();
  ctx = current_context();
  if (ctx) g_addr[{dev, ctx}] = p;
  return p;
}

// One-block plan for n input bytes, written into the scratch.
__global__ void k_noalloc_plan(uint8_t *base, int n) {
  int64_t *p64 = reinterpret_cast<int64_t *>(base + kOffPlan64);
  int32_t *p32 = reinterpret_cast<int32_t *>(base + kOffPlan32);
  int32_t *rt_block = reinterpret_cast<int32_t *>(base + kOffRtBlock);
  int32_t *rt_start = reinterpret_cast<int32_t *>(base + kOffRtStart);
  const int nt = (n + kRawTile - 1) / kRawTile;
  for (int t = threadIdx.x; t < nt; t += blockDim.x) {
    rt_block[t] = 0;
    rt_start[t] = t * kRawTile;
  }
  if (threadIdx.x == 0) {
    p64[0] = 0;                                     // raw_off
    p64[1] = 0;                                     // off
    p64[2] = 0;                                     // cap (unused by RLE1)
    p32[0] = n;                                     // raw_len
    p32[1] = 0;                                     // rt_first[0]
    p32[2] = nt;                                    // rt_first[1]
  }
}

}  // namespace
}  // namespace bz2g

using namespace bz2g;

extern "C" int bz2g_rle1_noalloc(const uint8_t *d_in, int n, uint8_t *d_out, int *m,
                                 void *stream) {
  try {
    if (n < 0 || !m) throw Error(kErrArg, "bz2g_rle1_noalloc: bad arguments");
    if (n == 0) {
      *m = 0;
      set_last_error("");
      return BZ2G_OK;
    }
    if (!d_in || !d_out) throw Error(kErrArg, "bz2g_rle1_noalloc: null device pointer");
    if (n > kNoAllocMaxInput) {
      throw Error(kErrTooLarge, "bz2g_rle1_noalloc: input of " + std::to_string(n) +
                                    " bytes exceeds the " + std::to_string(kNoAllocMaxInput) +
                                    "-byte limit of its static scratch");
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    uint8_t *base = scratch_address();
    SlabDev d;
    std::memset(&d, 0, sizeof(d));
    d.nblocks = 1;
    d.run_cut = 259;
    d.n_raw_tiles = (n + kRawTile - 1) / kRawTile;
    d.raw = base + kOffRaw;
    d.raw_off = reinterpret_cast<const int64_t *>(base + kOffPlan64);
    d.off = d.raw_off + 1;
    d.cap = d.raw_off + 2;
    d.raw_len = reinterpret_cast<const int *>(base + kOffPlan32);
    d.rt_first = d.raw_len + 1;
    d.rt_block = reinterpret_cast<const int *>(base + kOffRtBlock);
    d.rt_start = reinterpret_cast<const int *>(base + kOffRtStart);
    d.tile_a = reinterpret_cast<int32_t *>(base + kOffTileA);
    d.tile_b = reinterpret_cast<int32_t *>(base + kOffTileB);
    d.tile_c = reinterpret_cast<int32_t *>(base + kOffTileC);
    d.tile_d = reinterpret_cast<int32_t *>(base + kOffTileD);
    d.m = reinterpret_cast<int32_t *>(base + kOffScalars);
    d.crc = reinterpret_cast<uint32_t *>(base + kOffScalars + 4);
    d.crc_acc = reinterpret_cast<uint32_t *>(base + kOffScalars + 8);
    d.rle1 = d_out;  // written in place: off[0] == 0
    BZ_CUDA(cudaMemcpyAsync(d.raw, d_in, (size_t)n, cudaMemcpyDeviceToDevice, st));
    k_noalloc_plan<<<1, 256, 0, st>>>(base, n);
    BZ_LAUNCH_CHECK();
    stage_rle1_crc(d, st);
    int h_m = 0;
    BZ_CUDA(cudaMemcpyAsync(&h_m, d.m, sizeof(int), cudaMemcpyDeviceToHost, st));
    BZ_CUDA(cudaStreamSynchronize(st));
    *m = h_m;
    set_last_error("");
    return BZ2G_OK;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    set_last_error(std::string("bz2g_rle1_noalloc: ") + e.what());
    return BZ2G_ERR_INTERNAL;
  }
}
