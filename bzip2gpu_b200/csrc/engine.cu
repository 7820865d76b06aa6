// Slab plan and workspace (device buffers of one slab context).
#include "engine.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <sstream>

namespace bz2g {

static std::atomic<int64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
int64_t launch_count() { return g_launches.load(); }

[[noreturn]] void throw_cuda(cudaError_t e, const char *expr, const char *file, int line) {
  std::ostringstream os;
  os << expr << " failed at " << file << ":" << line << ": " << cudaGetErrorName(e) << " ("
     << cudaGetErrorString(e) << ")";
  throw Error(kErrCuda, os.str());
}

static int64_t m_bound(int64_t raw_len, int64_t m_cap) {
  const int64_t b = rle1_bound(raw_len);
  return m_cap > 0 ? std::min(b, m_cap) : b;
}

static int64_t groups_bound(int64_t raw_len, int64_t m_cap = 0) {
  // symbols <= RLE1 bytes + 1 (EOB), 50 symbols per group
  return (m_bound(raw_len, m_cap) + 1 + kGroupSize - 1) / kGroupSize;
}

BlockNeeds block_needs(int64_t L, int64_t m_cap) {
  BlockNeeds r;
  r.raw = align_up(L, 16);
  r.raw_tiles = (int)((L + kRawTile - 1) / kRawTile);
  r.elems = align_up(std::max<int64_t>(m_bound(L, m_cap), 1), kTile);
  r.tiles = (int)(r.elems / kTile);
  r.group_tiles = (int)((groups_bound(L, m_cap) + kGroupTile - 1) / kGroupTile);
  return r;
}

void SlabPlan::build(const int *lens, int n, int cut, int64_t mcap) {
  nblocks = n;
  run_cut = cut;
  m_cap = mcap;
  raw_off.assign(n, 0);
  off.assign(n, 0);
  cap.assign(n, 0);
  raw_len.assign(lens, lens + n);
  rt_block.clear();
  rt_start.clear();
  rt_first.assign(n + 1, 0);
  tile_block.clear();
  gt_block.clear();
  gt_first.clear();
  gt_begin.assign(n + 1, 0);
  raw_total = 0;
  elem_total = 0;
  max_m_bound = 0;
  for (int b = 0; b < n; b++) {
    const int64_t L = lens[b];
    raw_off[b] = raw_total;
    raw_total += align_up(L, 16);
    rt_first[b] = (int)rt_block.size();
    for (int64_t st = 0; st < L; st += kRawTile) {
      rt_block.push_back(b);
      rt_start.push_back((int)st);
    }
    const int64_t c = align_up(std::max<int64_t>(m_bound(L, m_cap), 1), kTile);
    off[b] = elem_total;
    cap[b] = c;
    for (int64_t k = 0; k < c / kTile; k++) tile_block.push_back(b);
    elem_total += c;
    gt_begin[b] = (int)gt_block.size();
    const int64_t G = groups_bound(L, m_cap);
    for (int64_t g = 0; g < G; g += kGroupTile) {
      gt_block.push_back(b);
      gt_first.push_back((int)g);
    }
    max_m_bound = std::max<int>(max_m_bound, (int)m_bound(L, m_cap));
  }
  rt_first[n] = (int)rt_block.size();
  gt_begin[n] = (int)gt_block.size();
}

void *Workspace::alloc(size_t bytes) {
  void *p = nullptr;
  BZ_CUDA(cudaMalloc(&p, std::max<size_t>(bytes, 256)));
  allocs_.push_back(p);
  return p;
}

Workspace::Workspace(int mb, int64_t mr, int64_t me, int mt, int mrt, int mgt)
    : max_blocks(mb), max_raw(mr), max_elems(me), max_tiles(mt), max_raw_tiles(mrt),
      max_group_tiles(mgt) {
  std::memset(&dev, 0, sizeof(dev));
  try {
    const int64_t E = me + kTile;  // slack for vector loads past a block's end
    dev.raw = (uint8_t *)alloc(mr + 64);
    dev.rle1 = (uint8_t *)alloc(E);
    dev.last = (uint8_t *)alloc(E);
    dev.mtf = (uint8_t *)alloc(E);
    dev.sa = (int32_t *)alloc(E * 4);
    dev.isa = (int32_t *)alloc(E * 4);
    dev.kpos[0] = (int32_t *)alloc(E * 4);
    dev.kpos[1] = (int32_t *)alloc(E * 4);
    dev.keys[0] = (uint64_t *)alloc(E * 8);
    dev.keys[1] = (uint64_t *)alloc(E * 8);
    dev.vals[0] = (uint32_t *)alloc(E * 4);
    dev.vals[1] = (uint32_t *)alloc(E * 4);
    dev.rle2 = (uint16_t *)alloc(E * 2);
    dev.sel = (uint8_t *)alloc(E / 32 + 64);
    dev.sel_mtf = (uint8_t *)alloc(E / 32 + 64);
    dev.grp_bits = (uint32_t *)alloc((E / 32 + 64) * 4);
    // payload: <= 17 bits per symbol; header: <= 6 bits per selector + tables
    out_words = E * kMaxCodeLen / 32 + (int64_t)mb * 8192 + 64;
    dev.out = (uint32_t *)alloc(out_words * 4);
    const int64_t T = std::max<int64_t>(mt, mrt) + 1;
    dev.tile_a = (int32_t *)alloc(T * 4);
    dev.tile_b = (int32_t *)alloc(T * 4);
    dev.tile_c = (int32_t *)alloc(T * 4);
    dev.tile_d = (int32_t *)alloc(T * 4);
    dev.tile_list = (int32_t *)alloc(T * 4);
    dev.vt_list = (int32_t *)alloc(T * 4);
    dev.vg_list = (int32_t *)alloc(((int64_t)mgt + 1) * 4);
    dev.warp_last = (int32_t *)alloc(((int64_t)mt + 1) * (kTileThreads / 32) * 4);
    dev.warp_act = (int32_t *)alloc(((int64_t)mt + 1) * (kTileThreads / 32) * 4);
    dev.tile_hist = (uint32_t *)alloc((int64_t)mt * kMaxRadix * 4);
    dev.tile_last = (int32_t *)alloc((int64_t)mt * 256 * 4);
    dev.gt_bits = (uint32_t *)alloc(((int64_t)mgt + 1) * 4);
    const int64_t B = mb + 1;
    dev.m = (int32_t *)alloc(B * 4);
    dev.s = (int32_t *)alloc(B * 4);
    dev.n_in_use = (int32_t *)alloc(B * 4);
    dev.orig_ptr = (int32_t *)alloc(B * 4);
    dev.n_groups = (int32_t *)alloc(B * 4);
    dev.n_sel = (int32_t *)alloc(B * 4);
    dev.crc = (uint32_t *)alloc(B * 4);
    dev.crc_acc = (uint32_t *)alloc(B * 4);
    dev.present = (uint32_t *)alloc(B * 8 * 4);
    dev.freq = (int32_t *)alloc(B * kMaxAlpha * 4);
    dev.len = (uint8_t *)alloc(B * kMaxGroups * kMaxAlpha);
    dev.code = (int32_t *)alloc(B * kMaxGroups * kMaxAlpha * 4);
    dev.rfreq = (int32_t *)alloc(B * kMaxGroups * kMaxAlpha * 4);
    dev.learned = (int32_t *)alloc(B * 4);
    dev.rfreq_m = (int32_t *)alloc(B * kMaxGroups * kMaxAlpha * 4);
    dev.len2 = (uint8_t *)alloc(B * kMaxGroups * kMaxAlpha);
    dev.sel2 = (uint8_t *)alloc(E / 32 + 64);
    dev.rfreq2 = (int32_t *)alloc(B * kMaxGroups * kMaxAlpha * 4);
    dev.plain_left = (int32_t *)alloc(B * 4);
    dev.err = (int32_t *)alloc(64);
    BZ_CUDA(cudaMemset(dev.err, 0, 64));
    dev.sort_len = (int32_t *)alloc(B * 4);
    dev.done = (int32_t *)alloc(B * 4);
    dev.ngroups = (int32_t *)alloc(B * 4);
    dev.act_len = (int32_t *)alloc(B * 4);
    dev.active_sum = (int64_t *)alloc(B * 8);
    dev.pstat = (int32_t *)alloc(B * 8 * 4);
    dev.hdr_bits = (int64_t *)alloc(B * 8);
    dev.pay_bits = (int64_t *)alloc(B * 8);
    dev.blk_start = (int64_t *)alloc(B * 8);
    dev.sort_ctl = (int32_t *)alloc(64);
    dev.sort_base = (uint32_t *)alloc(B * kMaxRadix * 4);
    dev.blk_count = (int32_t *)alloc(B * 4);
    BZ_CUDA(cudaMemset(dev.blk_count, 0, B * 4));
    dev.stream = (uint64_t *)alloc(64);
    dev.kt_elems = (uint64_t *)alloc(8 * kMaxTimedLaunches);
    // plan arrays: 3 int64 per block + ints
    pinned_plan_bytes = (size_t)B * 3 * 8 + ((size_t)B * 4 + mrt * 2 + mt + mgt * 2) * 4 + 1024;
    plan_dev_ = alloc(pinned_plan_bytes);
    BZ_CUDA(cudaMallocHost(&pinned_plan, pinned_plan_bytes));
    BZ_CUDA(cudaMallocHost((void **)&dev.h_flags, 64));
    BZ_CUDA(cudaMallocHost((void **)&dev.live, 8 * sizeof(int)));
    dev.live[0] = dev.live[1] = dev.live[2] = -1;
  } catch (...) {
    for (void *p : allocs_) cudaFree(p);
    allocs_.clear();
    if (pinned_plan) cudaFreeHost(pinned_plan);
    if (dev.h_flags) cudaFreeHost(dev.h_flags);
    if (dev.live) cudaFreeHost(dev.live);
    throw;
  }
}

Workspace::~Workspace() {
  for (void *p : allocs_) cudaFree(p);
  if (pinned_plan) cudaFreeHost(pinned_plan);
  if (dev.h_flags) cudaFreeHost(dev.h_flags);
  if (dev.live) cudaFreeHost(dev.live);
}

void Workspace::upload_plan(const SlabPlan &p, cudaStream_t st) {
  dev.live[0] = dev.live[1] = dev.live[2] = -1;  // a new slab: its lists are built anew
  BZ_REQUIRE(p.nblocks <= max_blocks && p.raw_total <= max_raw && p.elem_total <= max_elems &&
                 (int)p.tile_block.size() <= max_tiles && (int)p.rt_block.size() <= max_raw_tiles &&
                 (int)p.gt_block.size() <= max_group_tiles,
             kErrInternal, "slab plan exceeds workspace");
  uint8_t *h = (uint8_t *)pinned_plan;
  uint8_t *dbase = (uint8_t *)plan_dev_;
  size_t pos = 0;
  auto put = [&](const void *src, size_t bytes) -> const void * {
    std::memcpy(h + pos, src, bytes);
    const void *dp = dbase + pos;
    pos += (bytes + 15) / 16 * 16;
    return dp;
  };
  const int n = p.nblocks;
  dev.raw_off = (const int64_t *)put(p.raw_off.data(), 8 * n);
  dev.off = (const int64_t *)put(p.off.data(), 8 * n);
  dev.cap = (const int64_t *)put(p.cap.data(), 8 * n);
  dev.raw_len = (const int *)put(p.raw_len.data(), 4 * n);
  dev.rt_block = (const int *)put(p.rt_block.data(), 4 * p.rt_block.size());
  dev.rt_start = (const int *)put(p.rt_start.data(), 4 * p.rt_start.size());
  dev.rt_first = (const int *)put(p.rt_first.data(), 4 * (n + 1));
  dev.tile_block = (const int *)put(p.tile_block.data(), 4 * p.tile_block.size());
  dev.gt_block = (const int *)put(p.gt_block.data(), 4 * p.gt_block.size());
  dev.gt_first = (const int *)put(p.gt_first.data(), 4 * p.gt_first.size());
  dev.gt_begin = (const int *)put(p.gt_begin.data(), 4 * (n + 1));
  BZ_REQUIRE(pos <= pinned_plan_bytes, kErrInternal, "plan staging overflow");
  BZ_CUDA(cudaMemcpyAsync(plan_dev_, pinned_plan, pos, cudaMemcpyHostToDevice, st));
  dev.nblocks = n;
  dev.run_cut = p.run_cut;
  dev.ntiles = (int)p.tile_block.size();
  dev.n_raw_tiles = (int)p.rt_block.size();
  dev.n_group_tiles = (int)p.gt_block.size();
}

Workspace *Workspace::create_for(int max_blocks, int64_t max_block_bytes, int block_slots) {
  const int64_t nb = std::max<int64_t>(max_block_bytes, 1);
  const int64_t cap = align_up(std::max<int64_t>(rle1_bound(nb), 1), kTile);
  const int64_t E = (int64_t)max_blocks * cap;
  const int64_t R = (int64_t)max_blocks * align_up(nb, 16);
  BZ_REQUIRE(E + kTile < (int64_t(1) << 32), kErrArg,
             "slab too large: its element offsets must fit 32 bits (use fewer slab blocks)");
  const int mt = (int)(E / kTile);
  const int mrt = (int)(max_blocks * ((nb + kRawTile - 1) / kRawTile));
  const int mgt = (int)(max_blocks * ((groups_bound(nb) + kGroupTile - 1) / kGroupTile));
  return new Workspace(std::max(max_blocks, block_slots), R, E, mt, mrt, mgt);
}

namespace {

// One block of threads lists, in block order, the tiles that hold data:
// element tiles (groups = 0) of the m[b] bytes from off[b], or group tiles
// (groups = 1) of the ceil(s[b] / 50) groups from gt_begin[b].  The count
// goes to sort_ctl[10 + groups].
__global__ void __launch_bounds__(256) k_live_tiles(SlabDev d, int groups) {
  __shared__ int scratch[40];
  int32_t *list = groups ? d.vg_list : d.vt_list;
  int base = 0, mmax = 0;
  for (int b0 = 0; b0 < d.nblocks; b0 += 256) {
    const int b = b0 + threadIdx.x;
    int cnt = 0, first = 0;
    if (b < d.nblocks) {
      if (groups) {
        const int s = d.s[b];
        const int nsel = s > 0 ? (s + kGroupSize - 1) / kGroupSize : 0;
        cnt = (nsel + kGroupTile - 1) / kGroupTile;
        first = d.gt_begin[b];
      } else {
        const int m = d.m[b];
        cnt = m > 0 ? (m + kTile - 1) / kTile : 0;
        first = (int)(d.off[b] / kTile);
        mmax = max(mmax, m);
      }
    }
    int tot;
    const int at = base + block_excl_sum(cnt, scratch, &tot);
    for (int k = 0; k < cnt; k++) list[at + k] = first + k;
    base += tot;
  }
  if (!groups) {
    for (int o = 16; o > 0; o >>= 1) mmax = max(mmax, __shfl_xor_sync(0xffffffffu, mmax, o));
    if (lane_id() == 0) atomicMax(&d.sort_ctl[12], mmax);
  }
  if (threadIdx.x == 0) d.sort_ctl[10 + groups] = base;
}

int live_list(const SlabDev &d, cudaStream_t st, int groups) {
  if (!d.live) return -1;
  if (d.live[groups] >= 0) return d.live[groups];
  if (!groups) BZ_CUDA(cudaMemsetAsync(d.sort_ctl + 12, 0, sizeof(int32_t), st));
  k_live_tiles<<<1, 256, 0, st>>>(d, groups);
  BZ_LAUNCH_CHECK();
  BZ_CUDA(cudaMemcpyAsync(d.live + 4, d.sort_ctl + 10, 3 * sizeof(int32_t),
                          cudaMemcpyDeviceToHost, st));
  BZ_CUDA(cudaStreamSynchronize(st));
  d.live[groups] = d.live[4 + groups];
  if (!groups) d.live[2] = d.live[6];  // the largest m of the slab
  return d.live[groups];
}

}  // namespace

int live_tiles(const SlabDev &d, cudaStream_t st) { return live_list(d, st, 0); }
int live_group_tiles(const SlabDev &d, cudaStream_t st) { return live_list(d, st, 1); }

}  // namespace bz2g
