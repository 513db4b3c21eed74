// Host runtime behind the C-ABI (include/glst_c.h): owns the plan, the device
// buffers and the launch sequence of one GLST system on one GPU.
#include <dlfcn.h>
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "glst_c.h"
#include "worklist.cuh"
#include "planner.hpp"

using glst::Plan;
using glst::PlanError;
using glst::TDesignStore;
namespace dev = glst::dev;

// ---------------------------------------------------------------- errors
static thread_local std::string g_last_error;

static glst_status fail(glst_status s, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

// For the other translation units of the library: C++ linkage and hidden
// visibility, so it is not part of the exported interface.
__attribute__((visibility("hidden"))) void glst_internal_set_last_error(const char *msg) {
  g_last_error = msg;
}

#define CUDA_TRY(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess)                                                      \
      return fail(e_ == cudaErrorMemoryAllocation ? GLST_ERR_OUT_OF_MEMORY      \
                                                  : GLST_ERR_CUDA,              \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),       \
                  __FILE__, __LINE__);                                          \
  } while (0)

#define GLST_TRY(expr)            \
  do {                            \
    glst_status s_ = (expr);      \
    if (s_ != GLST_OK) return s_; \
  } while (0)

// ---------------------------------------------------------------- t-designs
static std::mutex g_store_mu;
static std::string g_store_path;  // explicit override
static std::map<std::string, std::shared_ptr<TDesignStore>> g_stores;

static std::string library_dir() {
  Dl_info info;
  if (dladdr(reinterpret_cast<void *>(&library_dir), &info) && info.dli_fname) {
    std::string p = info.dli_fname;
    size_t s = p.rfind('/');
    if (s != std::string::npos) return p.substr(0, s);
  }
  return ".";
}

static bool path_exists(const std::string &p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0;
}

static std::string resolve_store_path() {
  if (!g_store_path.empty()) return g_store_path;
  if (const char *e = std::getenv("GLST_TDESIGN_PATH"))
    if (*e) return e;
  if (path_exists("SS31-Mar-2016/")) return "SS31-Mar-2016/";
  return library_dir() + "/data/tdesigns.bin";
}

static std::shared_ptr<TDesignStore> get_store() {
  std::lock_guard<std::mutex> lk(g_store_mu);
  const std::string p = resolve_store_path();
  auto it = g_stores.find(p);
  if (it != g_stores.end()) return it->second;
  auto s = TDesignStore::open(p);
  g_stores[p] = s;
  return s;
}

// ---------------------------------------------------------------- handle
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

struct glst_handle {
  Plan plan;
  int device = 0;
  dev::Grid grid{};
  uint32_t K = 0;
  uint32_t nsplit = 1;  // long-range chunks (rows of part)
  uint32_t shard = 0, nshards = 1;  // node split across devices (1 = whole system)
  uint32_t k_begin = 0;             // first node (internal order) of this shard
  uint32_t lr_waves = 8;            // long-range CTAs ~ lr_waves x resident slots
  uint32_t lr_variant = 0;          // gather's FMA-pipe sin/cos share (kLrPolyMasks)
  uint32_t sf_max_npt = dev::kSfMaxNpt;  // radial nodes per thread, at most, in the structure-factor units
  size_t part_cap = 0;              // rows the part buffer holds
  size_t sat_per_node = 0;          // shell-sum shared bytes per node
  size_t sat_budget = 0;            // shell-sum shared bytes per CTA, at most
  int nsm = 148;
  uint32_t sr_rows = dev::kSrRowsPlanes;  // near-field partial-sum rows
  size_t smem_sm = 0;  // shared memory per SM, less four CTAs' system reserve
  std::vector<uint32_t> g_node_base, g_dir_base, g_kappa_base;  // per group, internal order
  std::vector<uint32_t> g_quad_base;  // per group, first radial-scale quad in kquads
  dev::LrKappaQuads kquads{};         // the gather's radial scales (parameter space)
  uint32_t sat_nb = 1, sat_stride = 0;
  bool sat_xyz = true;  // shell-sum cell-coordinate table in shared memory
  uint32_t combine_blocks = 1;
  bool computed = false;
  bool assigned = false;  // packets of some positions are in place (far-field accessor)
  std::vector<DevBuf> bufs;
  struct PendingBuf {
    void **out;
    size_t bytes;
  };
  std::vector<PendingBuf> pending;  // requested, not yet carved (setup)
  uint64_t bytes = 0;
  // atoms
  uint32_t *atom_cell = nullptr, *atom_slot = nullptr, *perm = nullptr;
  uint32_t *sorted_idx = nullptr, *cell_count = nullptr, *cell_point = nullptr;
  uint32_t *flags = nullptr;
  float4 *pk = nullptr;
  double4 *pd = nullptr;
  // nodes, internal order: group -> direction -> radial
  double4 *node64 = nullptr;
  uint32_t *node_radii = nullptr;
  float4 *dirs = nullptr;       // unit directions, FP32
  float *kappa = nullptr;       // radial scales per group, FP32
  dev::LrChunk *chunks = nullptr;
  dev::SfUnit *sf_units = nullptr;  // structure-factor work units (whole directions)
  size_t chunk_cap = 0, unit_cap = 0;         // entries the tables hold
  bool chunks_owned = false, units_owned = false, part_owned = false;  // own cudaMalloc (else arena)
  std::vector<dev::LrChunk> host_chunks;      // set-up: uploaded after the arena is committed
  std::vector<dev::SfUnit> host_units;
  uint32_t n_sf_units = 0;
  // far field
  float2 *S = nullptr;
  float2 *R = nullptr;
  double4 *part = nullptr;
  double4 *sr = nullptr;
  // outputs
  double *cfx = nullptr, *cfy = nullptr, *cfz = nullptr, *cen = nullptr;
  double *ofx = nullptr, *ofy = nullptr, *ofz = nullptr, *oen = nullptr;
  double *block_energy = nullptr, *energy = nullptr;
  // host-visible staging for the end-to-end path
  double *in_host = nullptr;  // device copy of host inputs (4 x natom)
  // streams/events for the near-field fork and the far-field pipeline
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_done = nullptr;  // end of a compute, for glst_reduce_shards
  // Node stages: the far field runs stage by stage (structure factors, shell
  // sums, gather over a contiguous range of whole directions), so S and R
  // hold one stage's nodes; a large system needs a fraction of the C x K
  // operand the whole node set would take.
  struct FarRange {
    uint32_t kb, ke, c0, c1;  // nodes and long-range chunks of one stage
    uint32_t u0, u1;          // structure-factor units of the same nodes
  };
  std::vector<FarRange> ranges;
  uint32_t stage_kmax = 0;    // nodes of the largest stage (S and R hold this many)
  uint32_t part_rows = 1;     // rows of `part` (chunks of the largest stage)
  uint32_t part_zero_from = 0;  // rows from here on are zeroed before stage 0
  // shell sums in global memory (grids whose per-node table does not fit
  // in shared memory): FP64 tables of a batch of node blocks, twiddles
  bool gsat = false;
  uint32_t gsat_nblk = 1;     // node blocks per batch
  double2 *gsat_T = nullptr;  // gsat_nblk x C x kNodeBlock
  double2 *gsat_tw = nullptr; // stage_kmax x (nx + ny + nz)
};

// Buffers of a handle are requested first and then carved out of one
// allocation (commit_allocs): one cudaMalloc per system keeps set-up cheap
// for servers that create systems while others compute.
static glst_status dalloc(glst_handle *h, void **out, size_t bytes) {
  *out = nullptr;
  h->pending.push_back({out, std::max<size_t>(bytes, 16)});
  return GLST_OK;
}

// Handle memory comes from one stream-ordered pool per device that keeps
// freed blocks for later handles (release threshold: unlimited).  Plain
// cudaMalloc calls took ~25 ms each, and held up other threads' CUDA calls,
// while a server's requests kept the GPU busy; a pool that already holds
// the memory hands it out without touching the device's page tables.
static glst_status handle_pool(int device, cudaMemPool_t *pool) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lk(mu);
  auto it = pools.find(device);
  if (it != pools.end()) {
    *pool = it->second;
    return GLST_OK;
  }
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t p = nullptr;
  CUDA_TRY(cudaMemPoolCreate(&p, &props));
  uint64_t keep = ~0ull;
  CUDA_TRY(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep));
  pools[device] = p;
  *pool = p;
  return GLST_OK;
}

static glst_status commit_allocs(glst_handle *h) {
  auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
  size_t total = 0;
  for (const auto &p : h->pending) total += al(p.bytes);
  if (!total) return GLST_OK;
  void *base = nullptr;
  cudaMemPool_t pool = nullptr;
  GLST_TRY(handle_pool(h->device, &pool));
  // ordered on the handle's side stream; set-up synchronises it before
  // returning, after which any stream may use the memory
  const cudaError_t e = cudaMallocFromPoolAsync(&base, total, pool, h->side);
  if (e != cudaSuccess) {
    cudaGetLastError();
    h->pending.clear();
    return fail(GLST_ERR_OUT_OF_MEMORY, "device allocation of %zu bytes failed: %s", total, cudaGetErrorString(e));
  }
  h->bufs.push_back({base, total});
  h->bytes += total;
  size_t off = 0;
  for (const auto &p : h->pending) {
    *p.out = static_cast<char *>(base) + off;
    off += al(p.bytes);
  }
  h->pending.clear();
  return GLST_OK;
}

template <typename T>
static glst_status dalloc_n(glst_handle *h, T **out, size_t n) {
  return dalloc(h, reinterpret_cast<void **>(out), n * sizeof(T));
}

// `device_idle`: the caller knows no work on this handle's memory is in
// flight (a server's idle system); otherwise the device is synchronised
// first, as cudaFree would, before the memory goes back to the pool.
static void release(glst_handle *h, bool device_idle = false) {
  if (!h->bufs.empty() && !device_idle) cudaDeviceSynchronize();
  for (auto &b : h->bufs) cudaFreeAsync(b.p, h->side);
  h->bufs.clear();
  h->pending.clear();
  if (h->chunks_owned && h->chunks) cudaFree(h->chunks);
  if (h->units_owned && h->sf_units) cudaFree(h->sf_units);
  if (h->part_owned && h->part) cudaFree(h->part);
  h->chunks = nullptr;
  h->sf_units = nullptr;
  h->part = nullptr;
  h->chunks_owned = h->units_owned = h->part_owned = false;
  h->chunk_cap = h->unit_cap = h->part_cap = 0;
  h->bytes = 0;
  if (h->side) cudaStreamDestroy(h->side);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  if (h->ev_done) cudaEventDestroy(h->ev_done);
  h->side = nullptr;
  h->ev_fork = h->ev_join = h->ev_done = nullptr;
}

// ---------------------------------------------------------------- tuning
// Launch shapes picked by glst_autotune, remembered per (cells, nodes, atoms
// bucket) for every later handle of that shape in this process.
struct Tuning {
  uint32_t sat_nb = 0, lr_waves = 0;  // 0 = default
  uint32_t lr_variant = 0, sf_max_npt = 0;
};
static std::mutex g_tune_mu;
static std::map<std::tuple<uint32_t, uint32_t, uint32_t>, Tuning> g_tune;

static std::tuple<uint32_t, uint32_t, uint32_t> tune_key(const Plan &p, uint32_t K) {
  uint32_t nb = 0;
  for (uint32_t n = p.natom; n > 1; n >>= 1) nb++;  // atoms bucket: log2
  return std::make_tuple(p.ncell, K, nb);
}

static Tuning tuned(const Plan &p, uint32_t K) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(tune_key(p, K));
  return it == g_tune.end() ? Tuning{} : it->second;
}

// Bytes of S + R one node stage may hold (default 4 GiB; the environment
// variable GLST_STAGE_BYTES, read when a handle is set up, overrides it).
// Systems whose C x K operand is larger run in several stages.
static uint64_t stage_budget() {
  uint64_t b = 4ull << 30;
  if (const char *e = std::getenv("GLST_STAGE_BYTES")) {
    const unsigned long long x = std::strtoull(e, nullptr, 10);
    if (x >= (1ull << 20)) b = x;
  }
  return b;
}

// Nodes per gather chunk, at most (a CTA's work is 128 atoms x its chunk's
// nodes; water10k's chunks hold ~1,800 nodes) and at least: every chunk
// writes a partial row of 32 bytes per atom that the combine reads back, so
// 256 nodes or more keep that traffic at <= 0.25 byte per (atom, node) pair
// (the 3,000-atom, 4^3-cell system had 33-node chunks: 28 MB of partial
// rows, 2 bytes per pair, against 10 MB of S and R).
static constexpr size_t kMaxChunkNodes = 2048;
static constexpr size_t kMinChunkNodes = 256;

// Near-field rows (kernels.cuh): nine when three rows' CTAs (one per cell
// and x plane) would be fewer than six per SM (up to 6^3 cells on B200:
// 13,500-18,000 atoms on 6^3 solve 2 % faster with nine; on 7^3 grids nine
// rows gained nothing for 24,000 atoms and cost 0.2 % for 30,000).
static uint32_t sr_rows_for(size_t ncell, int nsm) {
  return 3 * ncell < 6 * (size_t)std::max(1, nsm) ? dev::kSrRowsLines : dev::kSrRowsPlanes;
}

static uint32_t pow2_floor(uint32_t v) {
  uint32_t p = 1;
  while (p * 2 <= v && p < 32) p *= 2;
  return p;
}

// Node stages and long-range chunks.  First this handle's node range: all
// nodes, or -- when the system is split over several devices -- a contiguous
// run of whole directions holding about K / nshards nodes (the reference
// splits its node list into contiguous per-GPU ranges,
// src/glst_force.cu:276-293).  Then stages: contiguous runs of whole
// directions of about equal node count, as many as the S + R budget needs.
// Then, per stage, long-range chunks (whole directions of one group) sized so
// that the gather's grid is about lr_waves waves of resident CTAs, and the
// structure-factor units.
static glst_status build_chunks(glst_handle *h, bool in_arena = false) {
  const Plan &p = h->plan;
  const size_t C = p.ncell, Kall = p.has_far ? p.K() : 0, N = p.natom;
  const size_t slots = (size_t)h->nsm * 16;
  const size_t want_chunks = std::max<size_t>(1, ((size_t)h->lr_waves * slots + C - 1) / C);
  struct Dir {
    uint32_t gi, j;  // group, direction within the group
    uint32_t k;      // first node (internal order) of the direction
  };
  std::vector<Dir> dirs_all;
  for (size_t gi = 0; gi < (Kall ? p.groups.size() : 0); gi++)
    for (uint32_t j = 0; j < p.groups[gi].n_dir; j++)
      dirs_all.push_back({(uint32_t)gi, j, h->g_node_base[gi] + j * p.groups[gi].n_radial});
  auto dir_nodes = [&](const Dir &d) { return p.groups[d.gi].n_radial; };
  // The whole system's stage count and chunk size.  A shard cuts its chunks
  // at the whole system's chunk size, so that its chunks are exactly the
  // whole system's chunks of its node range (the shards' sum then groups
  // every FP32 partial sum as the unsharded solve).
  const uint64_t kpad_sys = (Kall + dev::kNodeBlock - 1) / dev::kNodeBlock * dev::kNodeBlock;
  const uint64_t nst_sys = std::max<uint64_t>(1, (C * kpad_sys * 16 + stage_budget() - 1) / stage_budget());
  auto chunk_nodes = [&](size_t stage_nodes) {
    return std::max<size_t>(kMinChunkNodes, std::min<size_t>(kMaxChunkNodes, stage_nodes / want_chunks));
  };
  // this handle's directions [d0, d1)
  size_t d0 = 0, d1 = dirs_all.size();
  if (h->nshards > 1 && Kall) {
    // shard by provisional chunks of the whole system's chunk size, each
    // assigned to the shard its middle node falls in
    const size_t target = chunk_nodes(Kall / nst_sys);
    bool any = false;
    size_t i = 0;
    while (i < dirs_all.size()) {
      const uint32_t gi = dirs_all[i].gi;
      const uint32_t dpc = (uint32_t)std::max<size_t>(1, target / p.groups[gi].n_radial);
      size_t e = i;
      while (e < dirs_all.size() && dirs_all[e].gi == gi && e - i < dpc) e++;
      const uint64_t nodes = (uint64_t)(e - i) * p.groups[gi].n_radial;
      const uint64_t mid = (uint64_t)dirs_all[i].k + nodes / 2;
      if (mid * h->nshards / Kall == h->shard) {
        if (!any) d0 = i;
        d1 = e;
        any = true;
      }
      i = e;
    }
    if (!any) d0 = d1 = 0;
  }
  const uint32_t kb = d0 < d1 ? dirs_all[d0].k : 0;
  const uint32_t ke = d0 < d1 ? dirs_all[d1 - 1].k + dir_nodes(dirs_all[d1 - 1]) : 0;
  h->k_begin = kb;
  h->K = ke - kb;
  const uint64_t K = h->K;
  // stages
  const uint64_t kpad_all = (K + dev::kNodeBlock - 1) / dev::kNodeBlock * dev::kNodeBlock;
  uint64_t nst = std::max<uint64_t>(1, (C * kpad_all * 16 + stage_budget() - 1) / stage_budget());
  nst = std::min<uint64_t>(nst, std::max<size_t>(1, d1 - d0));
  std::vector<std::pair<size_t, size_t>> stage_dirs;  // [first, last) direction of each stage
  {
    // directions per structure-factor unit of group gi: a stage ends on a
    // unit boundary of its group (no partial unit inside a group's run but
    // at its end), or at the end of a group
    auto dpu = [&](uint32_t gi) {
      const uint32_t nr = p.groups[gi].n_radial;
      return (uint32_t)dev::kSfThreads / ((nr + h->sf_max_npt - 1) / h->sf_max_npt);
    };
    size_t i = d0;
    for (uint64_t st = 0; st < nst && i < d1; st++) {
      const uint64_t target_end = kb + K * (st + 1) / nst;  // node where this stage should end
      size_t e = i + 1;
      while (e < d1 && dirs_all[e].k < target_end) e++;
      while (e < d1 && dirs_all[e].gi == dirs_all[e - 1].gi && dirs_all[e].j % dpu(dirs_all[e].gi) != 0) e++;
      if (st + 1 == nst) e = d1;
      stage_dirs.push_back({i, e});
      i = e;
    }
  }
  // chunks and units per stage
  std::vector<dev::LrChunk> chunks;
  std::vector<dev::SfUnit> units;
  h->ranges.clear();
  h->stage_kmax = 0;
  h->part_rows = 1;
  for (const auto &sd : stage_dirs) {
    glst_handle::FarRange rg{};
    rg.kb = dirs_all[sd.first].k - kb;
    rg.ke = dirs_all[sd.second - 1].k + dir_nodes(dirs_all[sd.second - 1]) - kb;
    // ... and at most kMaxChunkNodes nodes, so that on large systems (few
    // chunks fill the GPU) the last wave of gather CTAs stays short; at least
    // kMinChunkNodes (partial-row traffic on small systems)
    const size_t target_nodes = chunk_nodes(h->nshards > 1 ? Kall / nst_sys : rg.ke - rg.kb);
    rg.c0 = (uint32_t)chunks.size();
    rg.u0 = (uint32_t)units.size();
    size_t i = sd.first;
    while (i < sd.second) {
      // this group's run of directions inside the stage
      const uint32_t gi = dirs_all[i].gi;
      const auto &g = p.groups[gi];
      size_t e = i;
      while (e < sd.second && dirs_all[e].gi == gi) e++;
      const uint32_t n_dir = (uint32_t)(e - i), j_first = dirs_all[i].j;
      const uint32_t dpc = (uint32_t)std::max<size_t>(1, target_nodes / g.n_radial);
      for (uint32_t j0 = 0; j0 < n_dir; j0 += dpc) {
        dev::LrChunk c{};
        c.n_dir = std::min(dpc, n_dir - j0);
        c.n_rad = g.n_radial;
        c.node_begin = dirs_all[i].k + j0 * g.n_radial - kb;
        c.dir_begin = h->g_dir_base[gi] + j_first + j0;
        c.kappa_begin = h->g_kappa_base[gi];
        c.pad[0] = h->g_quad_base[gi];
        chunks.push_back(c);
      }
      // Structure-factor units: the group's whole run cut into units of
      // kSfThreads / nb directions, nb threads per direction of npt <=
      // kSfMaxNpt radial nodes (cutting the whole run, not each chunk, keeps
      // the units full).
      const uint32_t nb = (g.n_radial + h->sf_max_npt - 1) / h->sf_max_npt;
      const uint32_t npt = (g.n_radial + nb - 1) / nb;
      const uint32_t dpu = dev::kSfThreads / nb;
      for (uint32_t j0 = 0; j0 < n_dir; j0 += dpu) {
        dev::SfUnit u{};
        u.node_begin = dirs_all[i].k + j0 * g.n_radial - kb;
        u.dir_begin = h->g_dir_base[gi] + j_first + j0;
        u.n_dir = std::min(dpu, n_dir - j0);
        u.n_rad = g.n_radial;
        u.nb = nb;
        u.npt = npt;
        u.kappa_begin = h->g_kappa_base[gi];
        units.push_back(u);
      }
      i = e;
    }
    rg.c1 = (uint32_t)chunks.size();
    rg.u1 = (uint32_t)units.size();
    if (rg.c1 - rg.c0 > 65535) return fail(GLST_ERR_SIZE, "too many long-range chunks in a node stage");
    h->stage_kmax = std::max(h->stage_kmax, rg.ke - rg.kb);
    h->part_rows = std::max(h->part_rows, rg.c1 - rg.c0);
    h->ranges.push_back(rg);
  }
  // rows a later stage writes beyond what stage 0 writes start at zero
  h->part_zero_from = h->ranges.empty() ? h->part_rows : h->ranges[0].c1 - h->ranges[0].c0;
  h->nsplit = (uint32_t)chunks.size();
  h->n_sf_units = (uint32_t)units.size();
  if (units.size() > 0x7FFFFFFFu) return fail(GLST_ERR_SIZE, "too many structure-factor units");
  const size_t part_rows = h->part_rows;
  if (in_arena) {
    // first build (set-up): carve the tables and partial rows out of the
    // handle's single allocation; uploaded once it is committed.  Separate
    // small cudaMalloc calls here took 25-270 ms while a server's other
    // requests kept the GPU busy.
    GLST_TRY(dalloc_n(h, &h->chunks, std::max<size_t>(1, chunks.size())));
    GLST_TRY(dalloc_n(h, &h->sf_units, std::max<size_t>(1, units.size())));
    GLST_TRY(dalloc_n(h, &h->part, part_rows * std::max<size_t>(1, N)));
    h->chunk_cap = std::max<size_t>(1, chunks.size());
    h->unit_cap = std::max<size_t>(1, units.size());
    h->part_cap = part_rows;
    h->host_chunks = std::move(chunks);
    h->host_units = std::move(units);
    return GLST_OK;
  }
  // rebuild (autotune): reuse the buffers when the new tables fit, else
  // allocate larger ones of their own
  auto regrow = [&](void **buf, bool &owned, size_t &cap, size_t need, size_t elem) -> glst_status {
    if (need <= cap) return GLST_OK;
    if (owned && *buf) {
      cudaFree(*buf);
      h->bytes -= cap * elem;
    }
    *buf = nullptr;
    cap = 0;
    owned = true;
    CUDA_TRY(cudaMalloc(buf, need * elem));
    cap = need;
    h->bytes += need * elem;
    return GLST_OK;
  };
  GLST_TRY(regrow(reinterpret_cast<void **>(&h->chunks), h->chunks_owned, h->chunk_cap,
                  std::max<size_t>(1, chunks.size()), sizeof(dev::LrChunk)));
  GLST_TRY(regrow(reinterpret_cast<void **>(&h->sf_units), h->units_owned, h->unit_cap,
                  std::max<size_t>(1, units.size()), sizeof(dev::SfUnit)));
  size_t part_cap_elems = h->part_cap * std::max<size_t>(1, N);
  GLST_TRY(regrow(reinterpret_cast<void **>(&h->part), h->part_owned, part_cap_elems,
                  part_rows * std::max<size_t>(1, N), sizeof(double4)));
  h->part_cap = part_cap_elems / std::max<size_t>(1, N);
  if (!chunks.empty())
    CUDA_TRY(cudaMemcpy(h->chunks, chunks.data(), chunks.size() * sizeof(dev::LrChunk), cudaMemcpyHostToDevice));
  if (!units.empty())
    CUDA_TRY(cudaMemcpy(h->sf_units, units.data(), units.size() * sizeof(dev::SfUnit), cudaMemcpyHostToDevice));
  return GLST_OK;
}

// Kernel attributes (the opt-in shared-memory maxima) are set once per
// device and process, with one process-wide value, so handles with different
// plans coexist.  Setting them for every new handle cost servers time: the
// call can wait while the same kernels run on other streams.
static glst_status set_kernel_attributes(int device, size_t shell_smem) {
  static std::mutex mu;
  static std::map<int, int> done;  // device -> bit 1: sort, bit 2: shell sums
  std::lock_guard<std::mutex> lk(mu);
  int &d = done[device];
  if (!(d & 1)) {
    CUDA_TRY(cudaFuncSetAttribute(dev::k_sort_pack, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(dev::kSortCap * sizeof(uint32_t))));
    d |= 1;
  }
  if (shell_smem && !(d & 2)) {
    CUDA_TRY(cudaFuncSetAttribute(dev::k_shell_sums<dev::kSatThreads, 3>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shell_smem));
    CUDA_TRY(cudaFuncSetAttribute(dev::k_shell_sums<dev::kSatThreadsSmall, 4>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shell_smem));
    CUDA_TRY(cudaFuncSetAttribute(dev::k_shell_sums<dev::kSatThreadsOne, 1>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shell_smem));
    d |= 2;
  }
  return GLST_OK;
}

static glst_status setup(glst_handle *h, uint32_t natom, double tol,
                         const double box[3], double rcut, int ct_float,
                         uint32_t shard = 0, uint32_t nshards = 1) {
  if (nshards == 0 || shard >= nshards) return fail(GLST_ERR_INVALID_ARG, "shard must be < nshards");
  h->shard = shard;
  h->nshards = nshards;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return fail(GLST_ERR_NO_DEVICE, "no CUDA capable device found");
  }
  CUDA_TRY(cudaGetDevice(&h->device));
  CUDA_TRY(cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->device));
  CUDA_TRY(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
  CUDA_TRY(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&h->ev_done, cudaEventDisableTiming));
  try {
    auto store = get_store();
    h->plan = glst::make_plan(natom, tol, box, rcut, ct_float, *store);
  } catch (const PlanError &e) {
    return fail(static_cast<glst_status>(e.status), "%s", e.msg.c_str());
  } catch (const std::exception &e) {
    return fail(GLST_ERR_TDESIGN, "planning failed: %s", e.what());
  }
  const Plan &p = h->plan;
  h->grid = dev::Grid{p.n[0], p.n[1], p.n[2], p.ncell, p.cell_dim, p.ct_float};
  h->K = p.has_far ? p.K() : 0;
  const size_t N = natom, C = p.ncell, K = h->K;

  // Node arrays, in the internal order group -> direction -> radial (the
  // reference's is group -> radial -> direction, src/cubature.cu:120-145).
  // Nodes and weights are rounded to CT first, as the reference stores them
  // (src/cubature.cu:138-141).
  std::vector<uint32_t> kappa_base, dir_base, node_base;
  std::vector<double4> n64(K);
  std::vector<uint32_t> radii(K);
  std::vector<float4> dirs;
  std::vector<float> kap;
  std::vector<uint32_t> quad_base;  // per group, the first of its radial-scale quads
  dev::LrKappaQuads kq{};
  uint32_t nquad = 0;
  {
    uint32_t ref_base = 0, ibase = 0;
    for (size_t gi = 0; gi < (K ? p.groups.size() : 0); gi++) {
      const auto &g = p.groups[gi];
      kappa_base.push_back((uint32_t)kap.size());
      dir_base.push_back((uint32_t)dirs.size());
      node_base.push_back(ibase);
      for (unsigned r = 0; r < g.n_radial; r++) kap.push_back((float)g.kappa[r]);
      quad_base.push_back(nquad);
      for (unsigned r0 = 0; r0 < g.n_radial; r0 += 4, nquad++) {
        if (nquad >= (uint32_t)dev::kLrKappaQuads)
          return fail(GLST_ERR_SIZE, "more than %d radial-scale quads", dev::kLrKappaQuads);
        float v[4];
        for (unsigned i = 0; i < 4; i++) v[i] = r0 + i < g.n_radial ? (float)g.kappa[r0 + i] : 0.f;
        kq.q[nquad] = make_float4(v[0], v[1], v[2], v[3]);
      }
      for (unsigned j = 0; j < g.n_dir; j++)
        dirs.push_back(make_float4((float)g.dirs[3 * j], (float)g.dirs[3 * j + 1], (float)g.dirs[3 * j + 2], 0.f));
      for (unsigned j = 0; j < g.n_dir; j++) {
        for (unsigned r = 0; r < g.n_radial; r++) {
          const size_t ref = ref_base + (size_t)r * g.n_dir + j;
          const size_t k = ibase + (size_t)j * g.n_radial + r;
          double kx = p.kx[ref], ky = p.ky[ref], kz = p.kz[ref], w = p.w[ref];
          if (p.ct_float) {
            kx = (double)(float)kx; ky = (double)(float)ky; kz = (double)(float)kz; w = (double)(float)w;
          }
          n64[k] = make_double4(kx, ky, kz, w);
          radii[k] = (g.r_in & 0xffffu) | (g.r_out << 16);
        }
      }
      ref_base += g.n_radial * g.n_dir;
      ibase += g.n_radial * g.n_dir;
      if (g.n_radial > (unsigned)dev::kLrfTileNodes)
        return fail(GLST_ERR_SIZE, "%u radial nodes exceed the tile of the long-range kernel", g.n_radial);
    }
    GLST_TRY(dalloc_n(h, &h->node64, K));
    GLST_TRY(dalloc_n(h, &h->node_radii, K));
    GLST_TRY(dalloc_n(h, &h->dirs, dirs.size()));
    GLST_TRY(dalloc_n(h, &h->kappa, kap.size()));
  }
  GLST_TRY(dalloc_n(h, &h->atom_cell, N));
  GLST_TRY(dalloc_n(h, &h->atom_slot, N));
  GLST_TRY(dalloc_n(h, &h->perm, N));
  GLST_TRY(dalloc_n(h, &h->sorted_idx, N));
  GLST_TRY(dalloc_n(h, &h->cell_count, C));
  GLST_TRY(dalloc_n(h, &h->cell_point, C));
  GLST_TRY(dalloc_n(h, &h->flags, 4));
  GLST_TRY(dalloc_n(h, &h->pk, N));
  GLST_TRY(dalloc_n(h, &h->pd, N));
  h->sr_rows = sr_rows_for(C, h->nsm);
  GLST_TRY(dalloc_n(h, &h->sr, (size_t)h->sr_rows * N));
  for (double **o : {&h->cfx, &h->cfy, &h->cfz, &h->cen, &h->ofx, &h->ofy, &h->ofz, &h->oen})
    GLST_TRY(dalloc_n(h, o, N));
  h->combine_blocks = (uint32_t)std::max<size_t>(1, (N + dev::kCombineAtoms - 1) / dev::kCombineAtoms);
  GLST_TRY(dalloc_n(h, &h->block_energy, h->combine_blocks));
  GLST_TRY(dalloc_n(h, &h->energy, 1));
  GLST_TRY(dalloc_n(h, &h->in_host, 4 * N));

  if (K) {
    // Shared-memory plan of the shell-sum kernel: per node a row of ncell+1
    // complex doubles plus its twiddle tables; a few nodes per CTA when the
    // grid is small (occupancy), one when it is large.  Grids whose row does
    // not fit take the global-memory form (k_gsat_*).
    int smem_optin = 0, nsm = 148;
    CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
    int smem_sm = 0, smem_reserved = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, h->device));
    CUDA_TRY(cudaDeviceGetAttribute(&smem_reserved, cudaDevAttrReservedSharedMemoryPerBlock, h->device));
    h->smem_sm = (size_t)std::max(0, smem_sm - 4 * smem_reserved);
    // row stride = 1 (mod 8) complex doubles: rows of consecutive nodes start
    // 16 bytes apart modulo 128, so the node-fastest accesses of the shell
    // pass spread over all shared-memory banks
    h->sat_stride = (uint32_t)(C + 1);
    while (h->sat_stride % 8 != 1) h->sat_stride++;
    const size_t per_node = ((size_t)h->sat_stride + p.n[0] + p.n[1] + p.n[2]) * sizeof(double2);
    // the cell-coordinate table (4 bytes per cell) comes off the budget when
    // a row and the table fit together; otherwise the kernel divides
    const size_t smem_total = (size_t)smem_optin;
    const size_t xyz_bytes = (C * 4 + 15) & ~size_t(15);
    h->sat_xyz = per_node + xyz_bytes <= smem_total;
    const size_t budget = h->sat_xyz ? smem_total - xyz_bytes : smem_total;
    const char *force_global = std::getenv("GLST_GLOBAL_SHELL_SUMS");
    h->gsat = p.n[0] >= 1024 || p.n[1] >= 1024 || p.n[2] >= 1024 || per_node > budget ||
              (force_global && force_global[0] == '1');
    h->sat_per_node = per_node;
    h->sat_budget = budget;
    GLST_TRY(set_kernel_attributes(h->device, smem_total));
    h->nsm = nsm;
    // Nodes per CTA: the most (<= 32) with which four CTAs still share an
    // SM, when that is 8 or more (4^3 cells: 32, 5^3: 16, 7^3: 8, as
    // glst_autotune picks them; a 3,000-atom 4^3 solve 0.484 -> 0.421 ms
    // against 8), else at most 8 within one CTA's shared memory.
    const size_t xyz_used = h->sat_xyz ? xyz_bytes : 0;
    const size_t four = h->smem_sm / 4 > xyz_used ? (h->smem_sm / 4 - xyz_used) / per_node : 0;
    h->sat_nb = four >= 8 ? pow2_floor((uint32_t)std::min<size_t>(32, four))
                          : pow2_floor((uint32_t)std::max<size_t>(1, std::min<size_t>(8, budget / per_node)));
    // ... but no fewer than four CTAs per SM's worth of node blocks (few nodes)
    while (h->sat_nb > 8 && (K + h->sat_nb - 1) / h->sat_nb < 4 * (size_t)nsm) h->sat_nb >>= 1;
    h->g_node_base = node_base;
    h->g_dir_base = dir_base;
    h->g_kappa_base = kappa_base;
    h->g_quad_base = quad_base;
    h->kquads = kq;
    {
      const Tuning t = tuned(p, h->K);
      if (t.sat_nb && !h->gsat)
        h->sat_nb = pow2_floor(std::min<uint32_t>(t.sat_nb, (uint32_t)std::max<size_t>(1, budget / per_node)));
      if (t.lr_waves) h->lr_waves = t.lr_waves;
      h->lr_variant = t.lr_variant;
      if (t.sf_max_npt) h->sf_max_npt = t.sf_max_npt;
    }
    GLST_TRY(build_chunks(h, /*in_arena=*/true));
    const size_t kpad = ((size_t)h->stage_kmax + dev::kNodeBlock - 1) / dev::kNodeBlock * dev::kNodeBlock;
    GLST_TRY(dalloc_n(h, &h->S, C * kpad));
    GLST_TRY(dalloc_n(h, &h->R, C * kpad));
    if (h->gsat) {
      // tables of a batch of node blocks: ~64 MB (L2-sized) or one block
      const size_t blk_bytes = C * dev::kNodeBlock * sizeof(double2);
      const size_t nblk_stage = kpad / dev::kNodeBlock;
      h->gsat_nblk = (uint32_t)std::max<size_t>(1, std::min<size_t>(nblk_stage, (64ull << 20) / blk_bytes));
      GLST_TRY(dalloc_n(h, &h->gsat_T, (size_t)h->gsat_nblk * C * dev::kNodeBlock));
      GLST_TRY(dalloc_n(h, &h->gsat_tw, kpad * (p.n[0] + p.n[1] + p.n[2])));
    }
  }
  GLST_TRY(commit_allocs(h));
  if (!h->host_chunks.empty()) {
    CUDA_TRY(cudaMemcpyAsync(h->chunks, h->host_chunks.data(), h->host_chunks.size() * sizeof(dev::LrChunk),
                             cudaMemcpyHostToDevice, h->side));
    CUDA_TRY(cudaMemcpyAsync(h->sf_units, h->host_units.data(), h->host_units.size() * sizeof(dev::SfUnit),
                             cudaMemcpyHostToDevice, h->side));
  }
  h->host_chunks.clear();
  h->host_units.clear();
  if (K) {
    CUDA_TRY(cudaMemcpyAsync(h->node64, n64.data(), K * sizeof(double4), cudaMemcpyHostToDevice, h->side));
    CUDA_TRY(cudaMemcpyAsync(h->node_radii, radii.data(), K * sizeof(uint32_t), cudaMemcpyHostToDevice, h->side));
    CUDA_TRY(cudaMemcpyAsync(h->dirs, dirs.data(), dirs.size() * sizeof(float4), cudaMemcpyHostToDevice, h->side));
    CUDA_TRY(cudaMemcpyAsync(h->kappa, kap.data(), kap.size() * sizeof(float), cudaMemcpyHostToDevice, h->side));
  }
  if (shard > 0) CUDA_TRY(cudaMemsetAsync(h->sr, 0, (size_t)h->sr_rows * N * sizeof(double4), h->side));
  GLST_TRY(set_kernel_attributes(h->device, 0));
  CUDA_TRY(cudaMemsetAsync(h->flags, 0, 4 * sizeof(uint32_t), h->side));
  CUDA_TRY(cudaStreamSynchronize(h->side));  // memory and tables ready for any stream
  h->computed = false;
  h->assigned = false;
  return GLST_OK;
}

// ---------------------------------------------------------------- phases
static inline cudaStream_t S_(void *s) { return reinterpret_cast<cudaStream_t>(s); }

static glst_status phase_assign(glst_handle *h, const double *rx, const double *ry,
                                const double *rz, const double *qc, cudaStream_t st) {
  const uint32_t N = h->plan.natom, C = h->plan.ncell;
  if (N && (!rx || !ry || !rz || !qc)) return fail(GLST_ERR_INVALID_ARG, "null input pointer");
  CUDA_TRY(cudaMemsetAsync(h->cell_count, 0, C * sizeof(uint32_t), st));
  if (N) {
    const uint32_t nb = (N + 255) / 256;
    dev::k_bin<<<nb, 256, 0, st>>>(rx, ry, rz, N, h->grid, h->atom_cell, h->atom_slot, h->cell_count);
    CUDA_TRY(cudaGetLastError());
  }
  dev::k_scan<<<1, 1024, 0, st>>>(h->cell_count, C, h->cell_point);
  CUDA_TRY(cudaGetLastError());
  if (N) {
    const uint32_t nb = (N + 255) / 256;
    dev::k_scatter<<<nb, 256, 0, st>>>(h->atom_cell, h->atom_slot, h->cell_point, N, h->perm);
    CUDA_TRY(cudaGetLastError());
    dev::k_sort_pack<<<C, 256, dev::kSortCap * sizeof(uint32_t), st>>>(
        h->perm, h->cell_count, h->cell_point, h->grid, h->atom_cell, N, rx, ry, rz, qc, h->sorted_idx, h->pk,
        h->pd);
    CUDA_TRY(cudaGetLastError());
  }
  h->assigned = true;
  return GLST_OK;
}

// Far-field phases of one node stage: structure-factor units [u0, u1),
// shell sums over nodes [kb, ke), long-range chunks [c0, c1).  S and R hold
// the stage's nodes (local index = node - rg.kb).
static glst_status sf_stage(glst_handle *h, const glst_handle::FarRange &rg, cudaStream_t st) {
  if (rg.u1 <= rg.u0 || !h->plan.natom) return GLST_OK;
  const uint32_t cg = (h->plan.ncell + dev::kSfCellsPerCta - 1) / dev::kSfCellsPerCta;
  for (uint32_t r0 = 0; r0 < cg; r0 += 65535u) {  // gridDim.y is at most 65,535
    dim3 grid(rg.u1 - rg.u0, std::min<uint32_t>(cg - r0, 65535u));
    dev::k_structure_factors<<<grid, dev::kSfThreads, 0, st>>>(h->pk, h->cell_count, h->cell_point, h->grid,
                                                                h->sf_units + rg.u0, h->dirs, h->kappa, rg.kb,
                                                                r0 * dev::kSfCellsPerCta, h->S, h->R);
    CUDA_TRY(cudaGetLastError());
  }
  return GLST_OK;
}

static glst_status shell_stage(glst_handle *h, const glst_handle::FarRange &rg, cudaStream_t st) {
  const uint32_t kb = rg.kb, ke = rg.ke;
  if (ke <= kb || !h->plan.natom) return GLST_OK;
  const double4 *n64 = h->node64 + h->k_begin + kb;
  const uint32_t *radii = h->node_radii + h->k_begin + kb;
  if (h->gsat) {
    const uint32_t K = ke - kb, C = h->plan.ncell;
    const uint32_t naxis = h->grid.nx + h->grid.ny + h->grid.nz;
    const uint64_t ntw = (uint64_t)K * naxis;
    dev::k_gsat_twiddles<<<(uint32_t)((ntw + 255) / 256), 256, 0, st>>>(h->grid, n64, K, h->gsat_tw);
    CUDA_TRY(cudaGetLastError());
    const uint32_t nblk_all = (K + dev::kNodeBlock - 1) / dev::kNodeBlock;
    for (uint32_t b0 = 0; b0 < nblk_all; b0 += h->gsat_nblk) {
      dev::GsatArgs a{h->S, n64, radii, h->gsat_tw, h->gsat_T, h->R, K, b0,
                      std::min(h->gsat_nblk, nblk_all - b0)};
      const uint64_t per_line = (uint64_t)a.nblk * dev::kNodeBlock;
      auto blocks = [](uint64_t threads) { return (uint32_t)((threads + 255) / 256); };
      dev::k_gsat_z<<<blocks((uint64_t)h->grid.nx * h->grid.ny * per_line), 256, 0, st>>>(h->grid, a);
      dev::k_gsat_prefix<<<blocks((uint64_t)h->grid.nx * h->grid.nz * per_line), 256, 0, st>>>(h->grid, a, 1);
      dev::k_gsat_prefix<<<blocks((uint64_t)h->grid.ny * h->grid.nz * per_line), 256, 0, st>>>(h->grid, a, 0);
      dev::k_gsat_shell<<<blocks((uint64_t)C * per_line), 256, 0, st>>>(h->grid, a);
      CUDA_TRY(cudaGetLastError());
    }
    return GLST_OK;
  }
  uint32_t lg = 0;
  while ((1u << lg) < h->sat_nb) lg++;
  // the cell-coordinate table serves the several-nodes form only (the
  // one-node form steps its cells' coordinates)
  const bool table = h->sat_xyz && h->sat_nb > 1;
  dev::SatArgs a{h->S, n64, radii, ke - kb, 0, h->sat_nb, lg, table ? 1u : 0u, h->sat_stride, h->R};
  const uint32_t nblk = (ke - kb + h->sat_nb - 1) / h->sat_nb;
  const size_t smem = h->sat_per_node * h->sat_nb + (table ? (((size_t)h->plan.ncell * 4 + 15) & ~size_t(15)) : 0);
  // several nodes per CTA: 256 threads, 4 CTAs per SM where four CTAs'
  // tables fit in shared memory, else 512 threads, 3 CTAs per SM; one node
  // per CTA (large grids, one CTA fills the shared memory): 512 threads
  if (h->sat_nb == 1)
    dev::k_shell_sums<dev::kSatThreadsOne, 1><<<nblk, dev::kSatThreadsOne, smem, st>>>(h->grid, a);
  else if (4 * smem <= h->smem_sm)
    dev::k_shell_sums<dev::kSatThreadsSmall, 4><<<nblk, dev::kSatThreadsSmall, smem, st>>>(h->grid, a);
  else
    dev::k_shell_sums<dev::kSatThreads, 3><<<nblk, dev::kSatThreads, smem, st>>>(h->grid, a);
  CUDA_TRY(cudaGetLastError());
  return GLST_OK;
}

static glst_status lr_stage(glst_handle *h, size_t stage, cudaStream_t st) {
  const auto &rg = h->ranges[stage];
  if (rg.c1 <= rg.c0 || !h->plan.natom) return GLST_OK;
  dim3 grid((h->plan.natom + dev::kLrThreads - 1) / dev::kLrThreads, rg.c1 - rg.c0);
  // stage 0 writes its rows, later stages add into the same rows
#define GLST_LR(v)                                                                                            \
  case v:                                                                                                     \
    dev::k_long_range_flat<v><<<grid, dev::kLrThreads, 0, st>>>(h->pk, h->cell_point, h->plan.ncell,          \
                                                                h->chunks + rg.c0, h->dirs, h->kappa, h->R,   \
                                                                rg.kb, h->plan.natom, stage > 0 ? 1 : 0,      \
                                                                h->part, h->kquads);                          \
    break;
  switch (h->lr_variant) {
    GLST_LR(0) GLST_LR(1) GLST_LR(2) GLST_LR(3)
    default: return fail(GLST_ERR_INVALID_ARG, "bad gather variant");
  }
#undef GLST_LR
  CUDA_TRY(cudaGetLastError());
  return GLST_OK;
}

// Rows that a later stage accumulates into but stage 0 does not write.
static glst_status zero_part_tail(glst_handle *h, cudaStream_t st) {
  if (h->part_zero_from < h->part_rows && h->plan.natom)
    CUDA_TRY(cudaMemsetAsync(h->part + (size_t)h->part_zero_from * h->plan.natom, 0,
                             (size_t)(h->part_rows - h->part_zero_from) * h->plan.natom * sizeof(double4), st));
  return GLST_OK;
}

// The far field of every stage, in order, on one stream.
static glst_status far_all(glst_handle *h, cudaStream_t st) {
  if (!h->K || !h->plan.natom) return GLST_OK;
  GLST_TRY(zero_part_tail(h, st));
  for (size_t r = 0; r < h->ranges.size(); r++) {
    GLST_TRY(sf_stage(h, h->ranges[r], st));
    GLST_TRY(shell_stage(h, h->ranges[r], st));
    GLST_TRY(lr_stage(h, r, st));
  }
  return GLST_OK;
}

// The reference's phase methods.  With one node stage each runs its own
// kernel; with several (S and R hold one stage at a time) calc_sf runs the
// whole far field stage by stage and sum_rmt_sf / calc_lr_ef have nothing
// left to do -- the results are the same as the fused call's.
static bool single_stage(const glst_handle *h) { return h->ranges.size() <= 1; }

static glst_status phase_sf(glst_handle *h, cudaStream_t st) {
  if (!h->K) return GLST_OK;
  if (!single_stage(h)) return far_all(h, st);
  return sf_stage(h, h->ranges[0], st);
}

static glst_status phase_shell(glst_handle *h, cudaStream_t st) {
  return (h->K && single_stage(h)) ? shell_stage(h, h->ranges[0], st) : GLST_OK;
}

static glst_status phase_lr(glst_handle *h, cudaStream_t st) {
  return (h->K && single_stage(h)) ? lr_stage(h, 0, st) : GLST_OK;
}

static glst_status phase_sr(glst_handle *h, cudaStream_t st) {
  if (!h->plan.natom || h->shard > 0) return GLST_OK;  // shard 0 owns the near field
  dim3 grid(h->plan.ncell, h->sr_rows);
  dev::k_short_range<<<grid, dev::kSrThreads, 0, st>>>(h->pd, h->cell_count, h->cell_point, h->grid,
                                                       h->plan.natom, h->sr, h->sr_rows);
  CUDA_TRY(cudaGetLastError());
  return GLST_OK;
}

// Where a solve's input-order outputs and total energy go: the handle's own
// buffers, or (a batch) slices of the batch's arrays.
struct OutDest {
  double *ofx = nullptr, *ofy = nullptr, *ofz = nullptr, *oen = nullptr, *energy = nullptr;
};

static glst_status phase_combine(glst_handle *h, cudaStream_t st, const OutDest *od = nullptr) {
  const uint32_t N = h->plan.natom;
  double *ofx = od && od->ofx ? od->ofx : h->ofx, *ofy = od && od->ofy ? od->ofy : h->ofy;
  double *ofz = od && od->ofz ? od->ofz : h->ofz, *oen = od && od->oen ? od->oen : h->oen;
  double *energy = od && od->energy ? od->energy : h->energy;
  if (N) {
    dev::k_combine<<<h->combine_blocks, dev::kCombineThreads, 0, st>>>(
        h->sr, h->sr_rows, h->part, h->part_rows, h->sorted_idx, N, h->K ? 1 : 0, h->cfx, h->cfy, h->cfz, h->cen,
        ofx, ofy, ofz, oen, h->block_energy);
    CUDA_TRY(cudaGetLastError());
    dev::k_energy_total<<<1, 256, 0, st>>>(h->block_energy, h->combine_blocks, energy);
    CUDA_TRY(cudaGetLastError());
  } else {
    CUDA_TRY(cudaMemsetAsync(energy, 0, sizeof(double), st));
  }
  h->computed = true;
  return GLST_OK;
}

static glst_status compute_all(glst_handle *h, const double *rx, const double *ry, const double *rz,
                               const double *qc, cudaStream_t st, const OutDest *od = nullptr) {
  GLST_TRY(phase_assign(h, rx, ry, rz, qc, st));
  // The near field (FP64 pipe) runs on a side stream, overlapping the far
  // field on the same SMs.  It is forked after the (first stage's) structure
  // factors, so it shares the SMs with the shell sums and the gather:
  // measured on water10k 3.336 ms per solve against 3.375 ms forked before
  // the structure factors (whose FMA and SFU pipes it slowed) and 3.52 ms
  // after the shell sums.  (Splitting one system's far field over two
  // streams measured no overlap: the structure-factor kernel fills every
  // SM's register file, so the other stream's blocks only start as it
  // drains; water10k 3.27-3.42 ms per solve at 2-8 node ranges against 3.14.)
  bool sr_forked = false;
  auto fork_sr = [&]() -> glst_status {
    CUDA_TRY(cudaEventRecord(h->ev_fork, st));
    CUDA_TRY(cudaStreamWaitEvent(h->side, h->ev_fork, 0));
    GLST_TRY(phase_sr(h, h->side));
    CUDA_TRY(cudaEventRecord(h->ev_join, h->side));
    sr_forked = true;
    return GLST_OK;
  };
  if (h->K && h->plan.natom && !h->ranges.empty()) {
    GLST_TRY(zero_part_tail(h, st));
    for (size_t r = 0; r < h->ranges.size(); r++) {
      GLST_TRY(sf_stage(h, h->ranges[r], st));
      if (!sr_forked) GLST_TRY(fork_sr());
      GLST_TRY(shell_stage(h, h->ranges[r], st));
      GLST_TRY(lr_stage(h, r, st));
    }
  }
  if (!sr_forked) GLST_TRY(fork_sr());
  CUDA_TRY(cudaStreamWaitEvent(st, h->ev_join, 0));
  return phase_combine(h, st, od);
}

// Entry points run on the handle's device whatever device is current, and
// leave the caller's current device as they found it.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(const glst_handle *h) {
    if (!h) return;
    if (cudaGetDevice(&prev) == cudaSuccess && prev != h->device) cudaSetDevice(h->device);
    else prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// ---------------------------------------------------------------- C-ABI
extern "C" {

const char *glst_last_error(void) { return g_last_error.c_str(); }

const char *glst_status_string(glst_status s) {
  switch (s) {
    case GLST_OK: return "ok";
    case GLST_ERR_INVALID_ARG: return "invalid argument";
    case GLST_ERR_CUDA: return "CUDA error";
    case GLST_ERR_NO_DEVICE: return "no CUDA device";
    case GLST_ERR_TDESIGN: return "spherical t-design unavailable";
    case GLST_ERR_NO_CONVERGENCE: return "no convergence";
    case GLST_ERR_OUT_OF_MEMORY: return "out of device memory";
    case GLST_ERR_SIZE: return "size limit exceeded";
    case GLST_ERR_STATE: return "invalid state";
  }
  return "unknown";
}

const char *glst_version(void) { return "glst-b200 0.1 (sm_100a)"; }

uint32_t glst_max_atoms_per_cell(void) { return dev::kSortCap; }

glst_status glst_set_tdesign_path(const char *path) {
  std::lock_guard<std::mutex> lk(g_store_mu);
  g_store_path = path ? path : "";
  return GLST_OK;
}

glst_status glst_create(glst_handle **out, uint32_t natom, double tol, double bx, double by,
                        double bz, double rcut, glst_ct ct) {
  if (!out) return fail(GLST_ERR_INVALID_ARG, "null handle pointer");
  *out = nullptr;
  if (ct != GLST_CT_DOUBLE && ct != GLST_CT_FLOAT) return fail(GLST_ERR_INVALID_ARG, "bad calculation type");
  auto h = std::make_unique<glst_handle>();
  const double box[3] = {bx, by, bz};
  glst_status s = setup(h.get(), natom, tol, box, rcut, ct == GLST_CT_FLOAT);
  if (s != GLST_OK) {
    release(h.get());
    return s;
  }
  *out = h.release();
  return GLST_OK;
}

glst_status glst_create_shard(glst_handle **out, uint32_t natom, double tol, double bx, double by,
                              double bz, double rcut, glst_ct ct, uint32_t shard, uint32_t nshards) {
  if (!out) return fail(GLST_ERR_INVALID_ARG, "null handle pointer");
  *out = nullptr;
  if (ct != GLST_CT_DOUBLE && ct != GLST_CT_FLOAT) return fail(GLST_ERR_INVALID_ARG, "bad calculation type");
  auto h = std::make_unique<glst_handle>();
  const double box[3] = {bx, by, bz};
  glst_status s = setup(h.get(), natom, tol, box, rcut, ct == GLST_CT_FLOAT, shard, nshards);
  if (s != GLST_OK) {
    release(h.get());
    return s;
  }
  *out = h.release();
  return GLST_OK;
}

glst_status glst_create_ncell(glst_handle **out, uint32_t natom, double tol, double bx, double by,
                              double bz, uint32_t ncx, uint32_t ncy, uint32_t ncz, glst_ct ct) {
  if (!ncx || !ncy || !ncz) return fail(GLST_ERR_INVALID_ARG, "cell counts must be > 0");
  const double box[3] = {bx, by, bz};
  const uint32_t nc[3] = {ncx, ncy, ncz};
  return glst_create(out, natom, tol, bx, by, bz, glst::rcut_from_ncell(box, nc), ct);
}

glst_status glst_init(glst_handle *h, uint32_t natom, double tol, double bx, double by, double bz,
                      double rcut) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  const int ct = h->plan.ct_float;
  const uint32_t shard = h->shard, nshards = h->nshards;
  CUDA_TRY(cudaDeviceSynchronize());
  release(h);
  const double box[3] = {bx, by, bz};
  return setup(h, natom, tol, box, rcut, ct, shard, nshards);
}

glst_status glst_destroy(glst_handle *h) {
  if (!h) return GLST_OK;
  DeviceGuard guard_(h);
  cudaDeviceSynchronize();
  release(h, /*device_idle=*/true);
  delete h;
  return GLST_OK;
}

glst_status glst_compute(glst_handle *h, const double *rx, const double *ry, const double *rz,
                         const double *qc, void *stream) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  return compute_all(h, rx, ry, rz, qc, S_(stream));
}

glst_status glst_assign_atoms(glst_handle *h, const double *rx, const double *ry, const double *rz,
                              const double *qc, void *stream) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  return phase_assign(h, rx, ry, rz, qc, S_(stream));
}
glst_status glst_calc_sf(glst_handle *h, void *stream) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  return phase_sf(h, S_(stream));
}
glst_status glst_sum_rmt_sf(glst_handle *h, void *stream) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  return phase_shell(h, S_(stream));
}
glst_status glst_calc_lr_ef(glst_handle *h, void *stream) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  return phase_lr(h, S_(stream));
}
glst_status glst_calc_sr_ef(glst_handle *h, void *stream) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  return phase_sr(h, S_(stream));
}
glst_status glst_comm_ef(glst_handle *h, void *stream) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  return phase_combine(h, S_(stream));
}

glst_status glst_get_ef(glst_handle *h, double *fx, double *fy, double *fz, double *en,
                        int on_device, void *stream) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  if (!h->computed) return fail(GLST_ERR_STATE, "get_ef called before a compute");
  const size_t bytes = (size_t)h->plan.natom * sizeof(double);
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  cudaStream_t st = S_(stream);
  double *dst[4] = {fx, fy, fz, en};
  double *src[4] = {h->ofx, h->ofy, h->ofz, h->oen};
  for (int i = 0; i < 4; i++)
    if (dst[i] && bytes) CUDA_TRY(cudaMemcpyAsync(dst[i], src[i], bytes, kind, st));
  if (!on_device) CUDA_TRY(cudaStreamSynchronize(st));
  return GLST_OK;
}

glst_status glst_cell_outputs(glst_handle *h, double **fx, double **fy, double **fz, double **en) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  if (fx) *fx = h->cfx;
  if (fy) *fy = h->cfy;
  if (fz) *fz = h->cfz;
  if (en) *en = h->cen;
  return GLST_OK;
}

glst_status glst_energy(glst_handle *h, double *e, void *stream) {
  if (!h || !e) return fail(GLST_ERR_INVALID_ARG, "null argument");
  DeviceGuard guard_(h);
  if (!h->computed) return fail(GLST_ERR_STATE, "energy requested before a compute");
  CUDA_TRY(cudaMemcpyAsync(e, h->energy, sizeof(double), cudaMemcpyDeviceToHost, S_(stream)));
  CUDA_TRY(cudaStreamSynchronize(S_(stream)));
  return GLST_OK;
}

glst_status glst_compute_host(glst_handle *h, const double *rx, const double *ry, const double *rz,
                              const double *qc, double *fx, double *fy, double *fz, double *en,
                              void *stream) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  const size_t N = h->plan.natom, bytes = N * sizeof(double);
  cudaStream_t st = S_(stream);
  if (N && (!rx || !ry || !rz || !qc)) return fail(GLST_ERR_INVALID_ARG, "null input pointer");
  const double *src[4] = {rx, ry, rz, qc};
  for (int i = 0; i < 4; i++)
    if (bytes) CUDA_TRY(cudaMemcpyAsync(h->in_host + i * N, src[i], bytes, cudaMemcpyHostToDevice, st));
  GLST_TRY(compute_all(h, h->in_host, h->in_host + N, h->in_host + 2 * N, h->in_host + 3 * N, st));
  return glst_get_ef(h, fx, fy, fz, en, 0, stream);
}

glst_status glst_get_assignment(glst_handle *h, uint32_t *sorted_idx, uint32_t *cell_count,
                                uint32_t *cell_point) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  CUDA_TRY(cudaDeviceSynchronize());
  if (sorted_idx && h->plan.natom)
    CUDA_TRY(cudaMemcpy(sorted_idx, h->sorted_idx, h->plan.natom * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (cell_count)
    CUDA_TRY(cudaMemcpy(cell_count, h->cell_count, h->plan.ncell * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (cell_point)
    CUDA_TRY(cudaMemcpy(cell_point, h->cell_point, h->plan.ncell * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  return GLST_OK;
}

static void fill_info(const Plan &p, glst_info *info) {
  std::memset(info, 0, sizeof *info);
  info->natom = p.natom;
  for (int a = 0; a < 3; a++) info->ncell[a] = p.n[a];
  info->ncell_total = p.ncell;
  info->cell_dim = p.cell_dim;
  info->ngroup = (uint32_t)p.groups.size();
  info->num_nodes = p.K();
  info->has_far_field = p.has_far ? 1u : 0u;
  for (size_t g = 0; g < p.groups.size() && g < 16; g++) {
    const auto &G = p.groups[g];
    info->group_nodes[g] = G.n_radial * G.n_dir;
    info->group_gl_degree[g] = G.gl_degree;
    info->group_t_degree[g] = G.t_degree;
    info->group_alpha[g] = G.alpha;
    info->group_zcut[g] = G.zcut;
    info->group_rmax[g] = G.rmax;
    info->group_r_in[g] = G.r_in;
    info->group_r_out[g] = G.r_out;
  }
}

glst_status glst_get_info(const glst_handle *h, glst_info *info) {
  if (!h || !info) return fail(GLST_ERR_INVALID_ARG, "null argument");
  DeviceGuard guard_(h);
  fill_info(h->plan, info);
  info->device_bytes = h->bytes;
  // assignment 4 (+0 without atoms), near field 1, far field per stage:
  // structure factors 1, shell sums 1 (global-memory form: twiddles 1 + 4
  // per node batch), gather 1; combine 2
  uint32_t far = 0;
  if (h->K && h->plan.natom)
    for (const auto &rg : h->ranges) {
      const uint32_t nblk = (rg.ke - rg.kb + dev::kNodeBlock - 1) / dev::kNodeBlock;
      far += 2u + (h->gsat ? 1u + 4u * ((nblk + h->gsat_nblk - 1) / h->gsat_nblk) : 1u);
    }
  info->kernels_per_compute = h->plan.natom ? 4u + (h->shard == 0 ? 1u : 0u) + far + 2u : 2u;
  info->node_stages = (uint32_t)h->ranges.size();
  info->shell_sums_form = h->gsat ? 1u : 0u;
  info->gather_variant = h->lr_variant;
  info->sf_max_npt = h->sf_max_npt;
  return GLST_OK;
}

glst_status glst_plan(uint32_t natom, double tol, double bx, double by, double bz, double rcut,
                      glst_ct ct, glst_info *info, double *kx, double *ky, double *kz, double *w,
                      uint32_t *group) {
  if (!info) return fail(GLST_ERR_INVALID_ARG, "null info");
  if (ct != GLST_CT_DOUBLE && ct != GLST_CT_FLOAT) return fail(GLST_ERR_INVALID_ARG, "bad calculation type");
  const double box[3] = {bx, by, bz};
  Plan p;
  try {
    auto store = get_store();
    p = glst::make_plan(natom, tol, box, rcut, ct == GLST_CT_FLOAT, *store);
  } catch (const PlanError &e) {
    return fail(static_cast<glst_status>(e.status), "%s", e.msg.c_str());
  } catch (const std::exception &e) {
    return fail(GLST_ERR_TDESIGN, "planning failed: %s", e.what());
  }
  fill_info(p, info);
  const size_t K = p.K();
  if (kx) std::memcpy(kx, p.kx.data(), K * sizeof(double));
  if (ky) std::memcpy(ky, p.ky.data(), K * sizeof(double));
  if (kz) std::memcpy(kz, p.kz.data(), K * sizeof(double));
  if (w) std::memcpy(w, p.w.data(), K * sizeof(double));
  if (group) std::memcpy(group, p.group.data(), K * sizeof(uint32_t));
  return GLST_OK;
}

glst_status glst_get_nodes(const glst_handle *h, double *kx, double *ky, double *kz, double *w,
                           uint32_t *group) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  const Plan &p = h->plan;
  const size_t K = p.K();
  if (kx) std::memcpy(kx, p.kx.data(), K * sizeof(double));
  if (ky) std::memcpy(ky, p.ky.data(), K * sizeof(double));
  if (kz) std::memcpy(kz, p.kz.data(), K * sizeof(double));
  if (w) std::memcpy(w, p.w.data(), K * sizeof(double));
  if (group) std::memcpy(group, p.group.data(), K * sizeof(uint32_t));
  return GLST_OK;
}

glst_status glst_autotune(glst_handle *h, const double *rx, const double *ry, const double *rz,
                          const double *qc, void *stream, uint32_t *sat_nb, uint32_t *lr_waves) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  cudaStream_t st = S_(stream);
  if (h->K && h->plan.natom && h->nshards == 1 && single_stage(h)) {
    GLST_TRY(phase_assign(h, rx, ry, rz, qc, st));
    GLST_TRY(phase_sf(h, st));
    cudaEvent_t a, b;
    CUDA_TRY(cudaEventCreate(&a));
    CUDA_TRY(cudaEventCreate(&b));
    auto timed = [&](glst_status (*ph)(glst_handle *, cudaStream_t), float *ms) -> glst_status {
      GLST_TRY(ph(h, st));  // warm
      CUDA_TRY(cudaEventRecord(a, st));
      for (int i = 0; i < 3; i++) GLST_TRY(ph(h, st));
      CUDA_TRY(cudaEventRecord(b, st));
      CUDA_TRY(cudaEventSynchronize(b));
      CUDA_TRY(cudaEventElapsedTime(ms, a, b));
      return GLST_OK;
    };
    // shell sums: nodes per CTA
    uint32_t best_nb = h->sat_nb;
    float best = 1e30f;
    for (uint32_t nb : {1u, 2u, 4u, 8u, 16u, 32u}) {
      if (h->gsat || h->sat_per_node * nb > h->sat_budget) break;
      h->sat_nb = nb;
      float ms = 0.f;
      GLST_TRY(timed(phase_shell, &ms));
      if (ms < best) best = ms, best_nb = nb;
    }
    h->sat_nb = best_nb;
    GLST_TRY(phase_shell(h, st));
    // long-range gather: waves of chunk CTAs
    uint32_t best_w = h->lr_waves;
    best = 1e30f;
    for (uint32_t w : {2u, 4u, 8u, 16u, 32u}) {
      h->lr_waves = w;
      GLST_TRY(build_chunks(h));
      float ms = 0.f;
      GLST_TRY(timed(phase_lr, &ms));
      if (ms < best) best = ms, best_w = w;
    }
    h->lr_waves = best_w;
    GLST_TRY(build_chunks(h));
    // long-range gather: FMA-pipe sine/cosine share (compiled variants)
    uint32_t best_v = h->lr_variant;
    best = 1e30f;
    for (uint32_t v = 0; v < (uint32_t)dev::kLrVariants; v++) {
      h->lr_variant = v;
      float ms = 0.f;
      GLST_TRY(timed(phase_lr, &ms));
      if (ms < best) best = ms, best_v = v;
    }
    h->lr_variant = best_v;
    // structure factors: radial nodes per thread, at most (units' shape)
    uint32_t best_npt = h->sf_max_npt;
    best = 1e30f;
    for (uint32_t npt : {12u, 8u, 6u}) {
      h->sf_max_npt = npt;
      GLST_TRY(build_chunks(h));
      float ms = 0.f;
      GLST_TRY(timed(phase_sf, &ms));
      if (ms < best) best = ms, best_npt = npt;
    }
    h->sf_max_npt = best_npt;
    GLST_TRY(build_chunks(h));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[tune_key(h->plan, h->K)] = Tuning{h->sat_nb, h->lr_waves, h->lr_variant, h->sf_max_npt};
  }
  if (sat_nb) *sat_nb = h->sat_nb;
  if (lr_waves) *lr_waves = h->lr_waves;
  return GLST_OK;
}

glst_status glst_direct_coulomb(uint32_t natom, const double *rx, const double *ry, const double *rz,
                                const double *qc, double *fx, double *fy, double *fz, double *en, void *stream) {
  if (natom && (!rx || !ry || !rz || !qc || !fx || !fy || !fz || !en))
    return fail(GLST_ERR_INVALID_ARG, "null pointer");
  if (!natom) return GLST_OK;
  const uint32_t nb = (natom + dev::kDirectThreads - 1) / dev::kDirectThreads;
  dev::k_direct_coulomb<<<nb, dev::kDirectThreads, 0, S_(stream)>>>(rx, ry, rz, qc, natom, fx, fy, fz, en);
  CUDA_TRY(cudaGetLastError());
  return GLST_OK;
}

glst_status glst_measure_pipe_peaks(double *sfu_per_s, double *fma_per_s) {
  int device = 0, nsm = 0;
  CUDA_TRY(cudaGetDevice(&device));
  CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  const int threads = 512, blocks = nsm * 4, iters = 4096;
  float *buf = nullptr;
  CUDA_TRY(cudaMalloc(&buf, sizeof(float) * threads * blocks));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float best_sfu = 1e30f, best_fma = 1e30f, ms = 0.f;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(a);
    dev::k_probe_sfu<<<blocks, threads>>>(buf, iters);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    if (rep) best_sfu = std::min(best_sfu, ms);
    cudaEventRecord(a);
    dev::k_probe_fma<<<blocks, threads>>>(buf, iters * 4);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    if (rep) best_fma = std::min(best_fma, ms);
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(buf);
  if (e != cudaSuccess) return fail(GLST_ERR_CUDA, "pipe probe failed: %s", cudaGetErrorString(e));
  const double n = (double)threads * blocks * 8.0;
  if (sfu_per_s) *sfu_per_s = n * iters * 2.0 / (best_sfu * 1e-3);
  if (fma_per_s) *fma_per_s = n * iters * 4.0 / (best_fma * 1e-3);
  return GLST_OK;
}

glst_status glst_check(glst_handle *h, void *stream) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  uint32_t flags[4] = {0, 0, 0, 0};
  CUDA_TRY(cudaMemcpyAsync(flags, h->flags, sizeof flags, cudaMemcpyDeviceToHost, S_(stream)));
  CUDA_TRY(cudaStreamSynchronize(S_(stream)));
  if (flags[0]) return fail(GLST_ERR_STATE, "device error flags 0x%x raised by the last compute", flags[0]);
  return GLST_OK;
}

glst_status glst_reduce_shards(glst_handle *const *shards, uint32_t n, void *const *streams) {
  if (!shards || !streams || n == 0) return fail(GLST_ERR_INVALID_ARG, "null argument or no shards");
  if (n > (uint32_t)dev::kMaxShards) return fail(GLST_ERR_SIZE, "at most %d shards", dev::kMaxShards);
  glst_handle *h0 = shards[0];
  for (uint32_t s = 0; s < n; s++) {
    const glst_handle *h = shards[s];
    if (!h) return fail(GLST_ERR_INVALID_ARG, "null shard handle");
    if (h->nshards != n || h->shard != s)
      return fail(GLST_ERR_INVALID_ARG, "shards[%u] is shard %u of %u, expected %u of %u", s, h->shard, h->nshards, s,
                  n);
    if (h->plan.natom != h0->plan.natom || h->plan.ncell != h0->plan.ncell)
      return fail(GLST_ERR_INVALID_ARG, "shards of different systems");
    if (!h->computed) return fail(GLST_ERR_STATE, "shard %u has not computed", s);
  }
  if (n == 1) return GLST_OK;
  const uint32_t N = h0->plan.natom;
  DeviceGuard guard_(h0);
  cudaStream_t st0 = S_(streams[0]);
  // shard 0's stream waits for every other shard's compute; peer access from
  // shard 0's device to theirs
  for (uint32_t s = 1; s < n; s++) {
    glst_handle *h = shards[s];
    if (h->device != h0->device) {
      int ok = 0;
      CUDA_TRY(cudaDeviceCanAccessPeer(&ok, h0->device, h->device));
      if (!ok) return fail(GLST_ERR_CUDA, "device %d cannot access device %d's memory", h0->device, h->device);
      const cudaError_t e = cudaDeviceEnablePeerAccess(h->device, 0);
      if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
      else if (e != cudaSuccess) return fail(GLST_ERR_CUDA, "peer access: %s", cudaGetErrorString(e));
      CUDA_TRY(cudaSetDevice(h->device));
    }
    // the shard's own event, recorded on its compute stream, on its device
    CUDA_TRY(cudaEventRecord(h->ev_done, S_(streams[s])));
    if (h->device != h0->device) CUDA_TRY(cudaSetDevice(h0->device));
    CUDA_TRY(cudaStreamWaitEvent(st0, h->ev_done, 0));
  }
  if (!N) return GLST_OK;
  dev::ShardSet ss{};
  ss.n = n;
  for (uint32_t s = 0; s < n; s++) {
    const glst_handle *h = shards[s];
    const double *a[8] = {h->ofx, h->ofy, h->ofz, h->oen, h->cfx, h->cfy, h->cfz, h->cen};
    for (int k = 0; k < 8; k++) ss.src[s][k] = a[k];
  }
  // the sums land in shard 0's outputs: every element is read from all
  // shards before it is written (one thread per element)
  double *d[8] = {h0->ofx, h0->ofy, h0->ofz, h0->oen, h0->cfx, h0->cfy, h0->cfz, h0->cen};
  for (int k = 0; k < 8; k++) ss.dst[k] = d[k];
  const uint32_t nb = (N + dev::kCombineThreads - 1) / dev::kCombineThreads;  // <= combine_blocks
  dev::k_reduce_shards<<<nb, dev::kCombineThreads, 0, st0>>>(ss, N, h0->block_energy);
  CUDA_TRY(cudaGetLastError());
  dev::k_energy_total<<<1, 256, 0, st0>>>(h0->block_energy, nb, h0->energy);
  CUDA_TRY(cudaGetLastError());
  return GLST_OK;
}

glst_status glst_get_far_field(glst_handle *h, double *sf_re, double *sf_im, double *rmt_re, double *rmt_im,
                               void *stream) {
  if (!h) return fail(GLST_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard_(h);
  if (h->nshards > 1) return fail(GLST_ERR_STATE, "far-field arrays are available for whole-system handles only");
  if (!h->assigned) return fail(GLST_ERR_STATE, "far-field arrays requested before positions were assigned");
  const Plan &p = h->plan;
  const size_t C = p.ncell, K = p.has_far ? p.K() : 0;
  double *outs[4] = {sf_re, sf_im, rmt_re, rmt_im};
  for (double *o : outs)
    if (o) std::fill(o, o + C * K, 0.0);
  if (!K || !p.natom) return GLST_OK;
  cudaStream_t st = S_(stream);
  // internal node (group -> direction -> radial) -> reference index (group ->
  // radial -> direction, src/cubature.cu:120-145), and the node vector as the
  // device holds it (rounded to CT)
  std::vector<uint32_t> ref_of(K);
  {
    size_t base = 0;
    for (const auto &g : p.groups) {
      for (uint32_t j = 0; j < g.n_dir; j++)
        for (uint32_t r = 0; r < g.n_radial; r++)
          ref_of[base + (size_t)j * g.n_radial + r] = (uint32_t)(base + (size_t)r * g.n_dir + j);
      base += (size_t)g.n_radial * g.n_dir;
    }
  }
  auto ct = [&](double v) { return p.ct_float ? (double)(float)v : v; };
  const double l = h->grid.l;
  std::vector<float2> hs, hr;
  for (const auto &rg : h->ranges) {
    const size_t nk = rg.ke - rg.kb;
    const size_t nel = C * ((nk + dev::kNodeBlock - 1) / dev::kNodeBlock * dev::kNodeBlock);
    hs.resize(nel);
    hr.resize(nel);
    GLST_TRY(sf_stage(h, rg, st));
    CUDA_TRY(cudaMemcpyAsync(hs.data(), h->S, nel * sizeof(float2), cudaMemcpyDeviceToHost, st));
    GLST_TRY(shell_stage(h, rg, st));
    CUDA_TRY(cudaMemcpyAsync(hr.data(), h->R, nel * sizeof(float2), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t kl = 0; kl < nk; kl++) {
      const size_t ref = ref_of[rg.kb + kl];
      const double kx = ct(p.kx[ref]), ky = ct(p.ky[ref]), kz = ct(p.kz[ref]);
      for (size_t c = 0; c < C; c++) {
        const uint32_t x = (uint32_t)(c / ((size_t)p.n[1] * p.n[2])), y = (uint32_t)((c / p.n[2]) % p.n[1]),
                       z = (uint32_t)(c % p.n[2]);
        const double ph = kx * ((x + 0.5) * l) + ky * ((y + 0.5) * l) + kz * ((z + 0.5) * l);
        const double cs = std::cos(ph), sn = -std::sin(ph);  // e^{-ik.c}
        const float2 a = hs[dev::sr_index((uint32_t)c, (uint32_t)kl, (uint32_t)C)];
        const float2 b = hr[dev::sr_index((uint32_t)c, (uint32_t)kl, (uint32_t)C)];
        const size_t o = c * K + ref;
        if (sf_re) sf_re[o] = a.x * cs - a.y * sn;
        if (sf_im) sf_im[o] = a.x * sn + a.y * cs;
        if (rmt_re) rmt_re[o] = b.x * cs - b.y * sn;
        if (rmt_im) rmt_im[o] = b.x * sn + b.y * cs;
      }
    }
  }
  return GLST_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- batches
struct glst_batch {
  int device = 0;
  std::vector<glst_handle *> sys;
  std::vector<uint64_t> off;            // atom offsets (prefix sums)
  std::vector<uint32_t> order;          // systems, largest estimated cost first
  std::vector<uint32_t> branch_of;      // branch of each system
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> branch_done;
  cudaStream_t own = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void *key[8] = {};
  int key_mode = -1;                    // mode the graph was captured in
  double *energies = nullptr;           // device, one per system
  // Work list: systems solved by one persistent launch per phase (the rest
  // keep their own launch sequences on the other branches).
  std::vector<uint32_t> wl;             // batch indices of the work-list systems (descriptor order)
  std::vector<uint8_t> in_wl;           // per system
  enum { kZero, kBin, kScan, kScatter, kSort, kSf, kShell, kLr, kSr, kCombine, kEnergy, kPhases };
  // The work-list systems form `groups` work lists, each launched on its own
  // graph branch, so that phases of different groups overlap (the SFU-bound
  // structure factors of one group beside the shared-memory-bound shell sums
  // of another).
  struct WlGroup {
    uint32_t ph_off[kPhases] = {}, ph_n[kPhases] = {}, ph_grid[kPhases] = {};
    size_t shell_smem = 0;              // dynamic shared memory of the shell-sum launch
    cudaStream_t side = nullptr;        // near field beside the far field
    cudaEvent_t fork = nullptr, join = nullptr;
  };
  std::vector<WlGroup> groups;
  dev::WorkItem *d_items = nullptr;
  dev::SysDesc *d_desc = nullptr;
};

static constexpr uint32_t kBatchLargeAtoms = 20000;  // fills the GPU by itself

static void batch_release(glst_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  if (!b->sys.empty()) cudaDeviceSynchronize();
  for (auto *h : b->sys) {
    if (h) {
      release(h, /*device_idle=*/true);
      delete h;
    }
  }
  b->sys.clear();
  for (auto s : b->branch) cudaStreamDestroy(s);
  for (auto e : b->branch_done) cudaEventDestroy(e);
  b->branch.clear();
  b->branch_done.clear();
  if (b->own) cudaStreamDestroy(b->own);
  if (b->ev_in) cudaEventDestroy(b->ev_in);
  if (b->ev_out) cudaEventDestroy(b->ev_out);
  if (b->energies) cudaFree(b->energies);
  if (b->d_items) cudaFree(b->d_items);
  if (b->d_desc) cudaFree(b->d_desc);
  for (auto &gr : b->groups) {
    if (gr.side) cudaStreamDestroy(gr.side);
    if (gr.fork) cudaEventDestroy(gr.fork);
    if (gr.join) cudaEventDestroy(gr.join);
  }
  b->groups.clear();
  b->own = nullptr;
  b->ev_in = b->ev_out = nullptr;
  b->energies = nullptr;
  b->d_items = nullptr;
  b->d_desc = nullptr;
}

// A system joins the work list when its solve is one launch of each kernel
// with the shapes the work-list kernels use: whole system, one node stage,
// shell sums in shared memory with several nodes per CTA (or no far field).
static bool worklist_ok(const glst_handle *h) {
  if (h->nshards != 1 || h->ranges.size() > 1 || h->gsat) return false;
  if (h->lr_variant != 0) return false;  // the work-list gather is the default variant
  if (h->K && h->sat_nb < 2) return false;
  if ((h->plan.ncell + dev::kSfCellsPerCta - 1) / dev::kSfCellsPerCta > 65535u) return false;
  return true;
}

// Work items of every phase for the work-list systems, split into groups
// (systems dealt largest first to the least loaded group), and each phase
// kernel's grid: one CTA per item, or -- GLST_WORKLIST_GRID=persistent when a
// batch is created -- resident CTAs on every SM taking the items in a
// stride.  GLST_WORKLIST_GROUPS sets the number of groups (default 4, at
// most the batch's branches).
static glst_status worklist_build(glst_batch *b, const std::vector<double> &cost) {
  b->wl.clear();
  b->in_wl.assign(b->sys.size(), 0);
  std::vector<uint32_t> cand;
  for (uint32_t i : b->order)  // largest estimated cost first
    if (worklist_ok(b->sys[i])) cand.push_back(i);
  if (cand.empty()) return GLST_OK;
  uint32_t ng = 4;
  if (const char *e = std::getenv("GLST_WORKLIST_GROUPS")) ng = (uint32_t)std::max(1, std::atoi(e));
  ng = std::max<uint32_t>(1, std::min<uint32_t>({ng, (uint32_t)b->branch.size(), (uint32_t)cand.size()}));
  const char *ge = std::getenv("GLST_WORKLIST_GRID");
  const bool persistent = ge && std::string(ge) == "persistent";
  std::vector<std::vector<uint32_t>> members(ng);
  {
    std::vector<double> load(ng, 0.0);
    for (uint32_t i : cand) {
      const uint32_t gsel = (uint32_t)(std::min_element(load.begin(), load.end()) - load.begin());
      members[gsel].push_back(i);
      load[gsel] += cost[i];
    }
  }
  for (auto &m : members)
    for (uint32_t i : m) {
      b->in_wl[i] = 1;
      b->wl.push_back(i);  // descriptor index = position in wl
    }
  b->groups.assign(ng, glst_batch::WlGroup{});
  std::vector<dev::WorkItem> items;
  int nsm = 148, smem_optin = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device));
  CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device));
  CUDA_TRY(cudaFuncSetAttribute(dev::k_shell_sums_multi, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin));
  CUDA_TRY(cudaFuncSetAttribute(dev::k_sort_pack_multi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(dev::kSortCap * sizeof(uint32_t))));
  uint32_t w0 = 0;
  for (uint32_t gi = 0; gi < ng; gi++) {
    glst_batch::WlGroup &gr = b->groups[gi];
    const uint32_t nw = (uint32_t)members[gi].size();
    auto each = [&](int ph, auto &&fn) {
      gr.ph_off[ph] = (uint32_t)items.size();
      for (uint32_t w = w0; w < w0 + nw; w++) fn(w, b->sys[b->wl[w]]);
      gr.ph_n[ph] = (uint32_t)items.size() - gr.ph_off[ph];
    };
    each(glst_batch::kZero, [&](uint32_t w, glst_handle *h) {
      for (uint32_t c = 0; c < (h->plan.ncell + 1023) / 1024; c++) items.push_back({w, c, 0, 0});
    });
    each(glst_batch::kBin, [&](uint32_t w, glst_handle *h) {
      for (uint32_t a = 0; a < (h->plan.natom + 255) / 256; a++) items.push_back({w, a, 0, 0});
    });
    each(glst_batch::kScan, [&](uint32_t w, glst_handle *) { items.push_back({w, 0, 0, 0}); });
    each(glst_batch::kScatter, [&](uint32_t w, glst_handle *h) {
      for (uint32_t a = 0; a < (h->plan.natom + 255) / 256; a++) items.push_back({w, a, 0, 0});
    });
    each(glst_batch::kSort, [&](uint32_t w, glst_handle *h) {
      if (h->plan.natom)
        for (uint32_t c = 0; c < h->plan.ncell; c++) items.push_back({w, c, 0, 0});
    });
    each(glst_batch::kSf, [&](uint32_t w, glst_handle *h) {
      if (!h->K || !h->plan.natom) return;
      const uint32_t rows = (h->plan.ncell + dev::kSfCellsPerCta - 1) / dev::kSfCellsPerCta;
      for (uint32_t r = 0; r < rows; r++)
        for (uint32_t u = 0; u < h->n_sf_units; u++) items.push_back({w, u, r, 0});
    });
    each(glst_batch::kShell, [&](uint32_t w, glst_handle *h) {
      if (!h->K || !h->plan.natom) return;
      for (uint32_t k = 0; k < (h->K + h->sat_nb - 1) / h->sat_nb; k++) items.push_back({w, k, 0, 0});
    });
    each(glst_batch::kLr, [&](uint32_t w, glst_handle *h) {
      if (!h->K || !h->plan.natom) return;
      const uint32_t ab = (h->plan.natom + dev::kLrThreads - 1) / dev::kLrThreads;
      for (uint32_t c = 0; c < h->nsplit; c++)
        for (uint32_t a = 0; a < ab; a++) items.push_back({w, a, c, 0});
    });
    each(glst_batch::kSr, [&](uint32_t w, glst_handle *h) {
      if (!h->plan.natom) return;
      for (uint32_t pl = 0; pl < h->sr_rows; pl++)
        for (uint32_t c = 0; c < h->plan.ncell; c++) items.push_back({w, c, pl, 0});
    });
    each(glst_batch::kCombine, [&](uint32_t w, glst_handle *h) {
      if (h->plan.natom)
        for (uint32_t a = 0; a < h->combine_blocks; a++) items.push_back({w, a, 0, 0});
    });
    each(glst_batch::kEnergy, [&](uint32_t w, glst_handle *) { items.push_back({w, 0, 0, 0}); });
    // shell sums: the group's largest shared-memory need
    for (uint32_t w = w0; w < w0 + nw; w++) {
      const glst_handle *h = b->sys[b->wl[w]];
      if (!h->K) continue;
      const bool table = h->sat_xyz && h->sat_nb > 1;
      gr.shell_smem = std::max(gr.shell_smem, h->sat_per_node * h->sat_nb +
                                                  (table ? (((size_t)h->plan.ncell * 4 + 15) & ~size_t(15)) : 0));
    }
    auto grid = [&](int ph, const void *fn, int threads, size_t smem) -> glst_status {
      uint32_t g = gr.ph_n[ph];
      if (persistent) {
        int per_sm = 0;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
        g = std::min<uint32_t>(g, (uint32_t)std::max(1, per_sm) * nsm);
      }
      gr.ph_grid[ph] = std::max<uint32_t>(1, g);
      return GLST_OK;
    };
    GLST_TRY(grid(glst_batch::kZero, (const void *)dev::k_zero_counts_multi, 1024, 0));
    GLST_TRY(grid(glst_batch::kBin, (const void *)dev::k_bin_multi, 256, 0));
    GLST_TRY(grid(glst_batch::kScan, (const void *)dev::k_scan_multi, 1024, 0));
    GLST_TRY(grid(glst_batch::kScatter, (const void *)dev::k_scatter_multi, 256, 0));
    GLST_TRY(grid(glst_batch::kSort, (const void *)dev::k_sort_pack_multi, 256, dev::kSortCap * sizeof(uint32_t)));
    GLST_TRY(grid(glst_batch::kSf, (const void *)dev::k_structure_factors_multi, dev::kSfThreads, 0));
    GLST_TRY(grid(glst_batch::kShell, (const void *)dev::k_shell_sums_multi, dev::kSatThreads, gr.shell_smem));
    GLST_TRY(grid(glst_batch::kLr, (const void *)dev::k_long_range_multi, dev::kLrThreads, 0));
    GLST_TRY(grid(glst_batch::kSr, (const void *)dev::k_short_range_multi, dev::kSrThreads, 0));
    GLST_TRY(grid(glst_batch::kCombine, (const void *)dev::k_combine_multi, dev::kCombineThreads, 0));
    GLST_TRY(grid(glst_batch::kEnergy, (const void *)dev::k_energy_multi, 256, 0));
    CUDA_TRY(cudaStreamCreateWithFlags(&gr.side, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&gr.fork, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&gr.join, cudaEventDisableTiming));
    w0 += nw;
  }
  CUDA_TRY(cudaMalloc(&b->d_items, std::max<size_t>(1, items.size()) * sizeof(dev::WorkItem)));
  CUDA_TRY(cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(dev::WorkItem), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMalloc(&b->d_desc, b->wl.size() * sizeof(dev::SysDesc)));
  return GLST_OK;
}

// Descriptors of the work-list systems for these inputs and outputs
// (uploaded before the graph is captured; the graph reads them).
static glst_status worklist_descriptors(glst_batch *b, const double *const in[4], double *const out[4]) {
  std::vector<dev::SysDesc> ds(b->wl.size());
  for (size_t w = 0; w < b->wl.size(); w++) {
    const uint32_t i = b->wl[w];
    const glst_handle *h = b->sys[i];
    const size_t o = b->off[i];
    dev::SysDesc &d = ds[w];
    std::memset(&d, 0, sizeof d);
    d.g = h->grid;
    d.natom = h->plan.natom;
    d.combine_blocks = h->combine_blocks;
    d.part_rows = h->part_rows;
    d.use_far = h->K ? 1u : 0u;
    if (h->K) {
      uint32_t lg = 0;
      while ((1u << lg) < h->sat_nb) lg++;
      const bool table = h->sat_xyz && h->sat_nb > 1;
      d.sat = dev::SatArgs{h->S, h->node64, h->node_radii, h->K, 0, h->sat_nb, lg, table ? 1u : 0u,
                           h->sat_stride, h->R};
    }
    d.rx = in[0] + o; d.ry = in[1] + o; d.rz = in[2] + o; d.qc = in[3] + o;
    d.atom_cell = h->atom_cell; d.atom_slot = h->atom_slot; d.perm = h->perm;
    d.sorted_idx = h->sorted_idx; d.cell_count = h->cell_count; d.cell_point = h->cell_point;
    d.pk = h->pk; d.pd = h->pd; d.dirs = h->dirs; d.kappa = h->kappa;
    d.chunks = h->chunks; d.sf_units = h->sf_units;
    d.S = h->S; d.R = h->R; d.part = h->part; d.sr = h->sr; d.sr_rows = h->sr_rows;
    d.cfx = h->cfx; d.cfy = h->cfy; d.cfz = h->cfz; d.cen = h->cen;
    // input-order outputs straight into the batch's arrays (or the
    // handle's own when the caller passes none)
    d.ofx = out[0] ? out[0] + o : h->ofx;
    d.ofy = out[1] ? out[1] + o : h->ofy;
    d.ofz = out[2] ? out[2] + o : h->ofz;
    d.oen = out[3] ? out[3] + o : h->oen;
    d.block_energy = h->block_energy;
    d.energy = b->energies + i;
  }
  if (!ds.empty()) CUDA_TRY(cudaMemcpy(b->d_desc, ds.data(), ds.size() * sizeof(dev::SysDesc), cudaMemcpyHostToDevice));
  return GLST_OK;
}

// One group's work-list solve on stream st: one launch per phase for all its
// systems; the near field on a side stream beside the far field.
static glst_status worklist_launch(glst_batch *b, glst_batch::WlGroup &gr, cudaStream_t st) {
  const dev::SysDesc *D = b->d_desc;
  auto go = [&](int ph, auto kern, int threads, size_t smem, cudaStream_t s) -> glst_status {
    if (!gr.ph_n[ph]) return GLST_OK;
    kern<<<gr.ph_grid[ph], threads, smem, s>>>(D, b->d_items + gr.ph_off[ph], gr.ph_n[ph]);
    CUDA_TRY(cudaGetLastError());
    return GLST_OK;
  };
  GLST_TRY(go(glst_batch::kZero, dev::k_zero_counts_multi, 1024, 0, st));
  GLST_TRY(go(glst_batch::kBin, dev::k_bin_multi, 256, 0, st));
  GLST_TRY(go(glst_batch::kScan, dev::k_scan_multi, 1024, 0, st));
  GLST_TRY(go(glst_batch::kScatter, dev::k_scatter_multi, 256, 0, st));
  GLST_TRY(go(glst_batch::kSort, dev::k_sort_pack_multi, 256, dev::kSortCap * sizeof(uint32_t), st));
  GLST_TRY(go(glst_batch::kSf, dev::k_structure_factors_multi, dev::kSfThreads, 0, st));
  // near field forked after the structure factors, as in a single solve
  CUDA_TRY(cudaEventRecord(gr.fork, st));
  CUDA_TRY(cudaStreamWaitEvent(gr.side, gr.fork, 0));
  GLST_TRY(go(glst_batch::kSr, dev::k_short_range_multi, dev::kSrThreads, 0, gr.side));
  CUDA_TRY(cudaEventRecord(gr.join, gr.side));
  GLST_TRY(go(glst_batch::kShell, dev::k_shell_sums_multi, dev::kSatThreads, gr.shell_smem, st));
  GLST_TRY(go(glst_batch::kLr, dev::k_long_range_multi, dev::kLrThreads, 0, st));
  CUDA_TRY(cudaStreamWaitEvent(st, gr.join, 0));
  GLST_TRY(go(glst_batch::kCombine, dev::k_combine_multi, dev::kCombineThreads, 0, st));
  GLST_TRY(go(glst_batch::kEnergy, dev::k_energy_multi, 256, 0, st));
  return GLST_OK;
}

// One system: its solve, the combine writing the input-order outputs and the
// total energy straight into the batch's arrays (no copies).
static glst_status batch_one(glst_batch *b, uint32_t i, const double *const in[4], double *const out[4],
                             cudaStream_t st) {
  glst_handle *h = b->sys[i];
  const size_t o = b->off[i];
  OutDest od;
  od.ofx = out[0] ? out[0] + o : nullptr;
  od.ofy = out[1] ? out[1] + o : nullptr;
  od.ofz = out[2] ? out[2] + o : nullptr;
  od.oen = out[3] ? out[3] + o : nullptr;
  od.energy = b->energies + i;
  return compute_all(h, in[0] + o, in[1] + o, in[2] + o, in[3] + o, st, &od);
}

// Graph of one batched solve.  mode 0: every system its own launch sequence
// on the branches (large systems on branch 0, the rest spread over the
// others); mode 2: the work-list systems by one launch per phase (in groups
// on the first branches), every other system its own launch sequence on the
// remaining branches.
static glst_status batch_capture(glst_batch *b, const double *const in[4], double *const out[4], int mode) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  const bool wl = mode == 2 && !b->wl.empty();
  if (wl) GLST_TRY(worklist_descriptors(b, in, out));
  CUDA_TRY(cudaStreamBeginCapture(b->own, cudaStreamCaptureModeThreadLocal));
  glst_status s = GLST_OK;
  cudaError_t e = cudaEventRecord(b->ev_in, b->own);
  for (size_t j = 0; e == cudaSuccess && j < b->branch.size(); j++) e = cudaStreamWaitEvent(b->branch[j], b->ev_in, 0);
  const size_t nbr = b->branch.size();
  const size_t ng = wl ? b->groups.size() : 0;  // groups on branches 0 .. ng-1
  for (size_t gi = 0; e == cudaSuccess && s == GLST_OK && gi < ng; gi++)
    s = worklist_launch(b, b->groups[gi], b->branch[gi]);
  size_t next = 0;  // round robin over the branches after the groups' for the others
  for (size_t t = 0; e == cudaSuccess && s == GLST_OK && t < b->order.size(); t++) {
    const uint32_t i = b->order[t];
    if (wl && b->in_wl[i]) continue;
    cudaStream_t st = b->branch[b->branch_of[i]];
    if (wl) st = b->branch[nbr > ng ? ng + (next++ % (nbr - ng)) : (next++ % nbr)];
    s = batch_one(b, i, in, out, st);
  }
  for (size_t j = 0; e == cudaSuccess && j < b->branch.size(); j++) {
    e = cudaEventRecord(b->branch_done[j], b->branch[j]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->own, b->branch_done[j], 0);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(b->own, &g);
  if (s != GLST_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(GLST_ERR_CUDA, "batch graph capture failed: %s",
                cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  b->graph = g;
  CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
  for (int k = 0; k < 4; k++) {
    b->key[k] = in[k];
    b->key[4 + k] = out[k];
  }
  b->key_mode = mode;
  return GLST_OK;
}

extern "C" {

glst_status glst_batch_create(glst_batch **out, uint32_t nsys, const uint32_t *natom, const double *tol,
                              const double *box, const double *rcut, glst_ct ct, uint32_t nstreams) {
  if (!out || (nsys && (!natom || !tol || !box || !rcut)))
    return fail(GLST_ERR_INVALID_ARG, "null argument");
  if (ct != GLST_CT_DOUBLE && ct != GLST_CT_FLOAT) return fail(GLST_ERR_INVALID_ARG, "bad calculation type");
  *out = nullptr;
  auto b = std::make_unique<glst_batch>();
  CUDA_TRY(cudaGetDevice(&b->device));
  std::vector<double> cost(nsys);
  uint64_t acc = 0;
  for (uint32_t i = 0; i < nsys; i++) {
    auto h = std::make_unique<glst_handle>();
    const double bx[3] = {box[3 * i], box[3 * i + 1], box[3 * i + 2]};
    glst_status s = setup(h.get(), natom[i], tol[i], bx, rcut[i], ct == GLST_CT_FLOAT);
    if (s != GLST_OK) {
      release(h.get());
      batch_release(b.get());
      return s;
    }
    b->off.push_back(acc);
    acc += natom[i];
    // cost model: far-field pairs plus near-field pairs (~ N * 27 * N/C)
    const double N = natom[i], C = h->plan.ncell;
    cost[i] = N * (double)h->K + N * 27.0 * N / C * 4.0 + 2e5;
    b->sys.push_back(h.release());
  }
  b->off.push_back(acc);
  const uint32_t ns = std::max<uint32_t>(1, std::min<uint32_t>(nstreams ? nstreams : 16, std::max<uint32_t>(1, nsys)));
  for (uint32_t j = 0; j < ns; j++) {
    cudaStream_t st;
    cudaEvent_t ev;
    CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    b->branch.push_back(st);
    b->branch_done.push_back(ev);
  }
  // Systems large enough to fill the GPU alone run one after another on
  // branch 0 (running two at once only splits the SMs between them); the
  // rest go largest first onto the least loaded of the other branches, where
  // they fill the SMs the large ones leave idle.
  b->order.resize(nsys);
  for (uint32_t i = 0; i < nsys; i++) b->order[i] = i;
  std::stable_sort(b->order.begin(), b->order.end(), [&](uint32_t a, uint32_t c) { return cost[a] > cost[c]; });
  std::vector<double> load(ns, 0.0);
  b->branch_of.assign(nsys, 0);
  for (uint32_t i : b->order) {
    uint32_t j = 0;
    if (ns > 1 && natom[i] < kBatchLargeAtoms)
      j = 1 + (uint32_t)(std::min_element(load.begin() + 1, load.end()) - (load.begin() + 1));
    b->branch_of[i] = j;
    load[j] += cost[i];
  }
  CUDA_TRY(cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking));
  CUDA_TRY(cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming));
  CUDA_TRY(cudaMalloc(&b->energies, sizeof(double) * std::max<uint32_t>(1, nsys)));
  CUDA_TRY(cudaMemset(b->energies, 0, sizeof(double) * std::max<uint32_t>(1, nsys)));
  {
    const glst_status ws = worklist_build(b.get(), cost);
    if (ws != GLST_OK) {
      batch_release(b.get());
      return ws;
    }
  }
  *out = b.release();
  return GLST_OK;
}

glst_status glst_batch_destroy(glst_batch *b) {
  if (!b) return GLST_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(b->device);
  cudaDeviceSynchronize();
  batch_release(b);
  delete b;
  if (prev >= 0) cudaSetDevice(prev);
  return GLST_OK;
}

glst_status glst_batch_compute(glst_batch *b, const double *rx, const double *ry, const double *rz,
                               const double *qc, double *fx, double *fy, double *fz, double *en, int plain,
                               void *stream) {
  if (!b) return fail(GLST_ERR_INVALID_ARG, "null batch");
  if (b->off.back() && (!rx || !ry || !rz || !qc)) return fail(GLST_ERR_INVALID_ARG, "null input pointer");
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != b->device) cudaSetDevice(b->device);
  struct Restore {
    int d;
    ~Restore() {
      if (d >= 0) cudaSetDevice(d);
    }
  } restore{prev != b->device ? prev : -1};
  const double *in[4] = {rx, ry, rz, qc};
  double *out[4] = {fx, fy, fz, en};
  cudaStream_t st = S_(stream);
  if (plain == 1) {
    for (uint32_t i = 0; i < b->sys.size(); i++) GLST_TRY(batch_one(b, i, in, out, st));
    return GLST_OK;
  }
  if (plain != 0 && plain != 2) return fail(GLST_ERR_INVALID_ARG, "mode must be 0, 1 or 2");
  bool same = b->exec != nullptr && b->key_mode == plain;
  for (int k = 0; k < 4 && same; k++) same = b->key[k] == in[k] && b->key[4 + k] == out[k];
  if (!same) GLST_TRY(batch_capture(b, in, out, plain));
  CUDA_TRY(cudaEventRecord(b->ev_in, st));
  CUDA_TRY(cudaStreamWaitEvent(b->own, b->ev_in, 0));
  CUDA_TRY(cudaGraphLaunch(b->exec, b->own));
  CUDA_TRY(cudaEventRecord(b->ev_out, b->own));
  CUDA_TRY(cudaStreamWaitEvent(st, b->ev_out, 0));
  return GLST_OK;
}

glst_status glst_batch_energies(glst_batch *b, double *e, void *stream) {
  if (!b || !e) return fail(GLST_ERR_INVALID_ARG, "null argument");
  if (b->sys.empty()) return GLST_OK;
  CUDA_TRY(cudaMemcpyAsync(e, b->energies, b->sys.size() * sizeof(double), cudaMemcpyDeviceToHost, S_(stream)));
  CUDA_TRY(cudaStreamSynchronize(S_(stream)));
  return GLST_OK;
}

glst_status glst_batch_system(glst_batch *b, uint32_t i, glst_handle **h) {
  if (!b || !h || i >= b->sys.size()) return fail(GLST_ERR_INVALID_ARG, "bad batch index");
  *h = b->sys[i];
  return GLST_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- request server
//
// Continuous batching of independent energy+force requests.  Threads:
//   worker  -- completes finished requests, admits queued ones (reserving
//              device memory against the budget, evicting idle resident
//              systems least recently used first), launches ready requests
//              on free stream slots;
//   builders (kSrvBuilders) -- create the handles (planning + allocation) of admitted
//              requests that need a new system, off the launch path, so the
//              GPU keeps working while new systems are set up.
// A request's life: queued -> building (new system) -> ready -> running -> done.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace {

using SrvClock = std::chrono::steady_clock;

struct SrvSystem {
  uint64_t key = 0;
  glst_handle *h = nullptr;
  uint64_t bytes = 0;
  bool busy = false;
  uint64_t last_use = 0;
  uint32_t natom = 0;
  double tol = 0, box[3] = {0, 0, 0}, rcut = 0;
};

enum class SrvState { Queued, Building, Ready, Running, Done };

struct SrvRequest {
  uint64_t ticket = 0, key = 0;
  uint32_t natom = 0;
  double tol = 0, box[3] = {0, 0, 0}, rcut = 0;
  std::vector<double> in, out;
  double energy = 0.0;
  SrvClock::time_point t_submit, t_done;
  SrvState state = SrvState::Queued;
  glst_status status = GLST_OK;
  std::string err;
  SrvSystem *sys = nullptr;
  uint64_t reserved = 0;  // bytes reserved while its system is being built
};

struct SrvSlot {
  cudaStream_t st = nullptr;
  double *pin = nullptr;  // 4N inputs, then 4N outputs + energy
  size_t cap = 0;         // atoms the pinned buffer holds
  SrvRequest *req = nullptr;
  std::atomic<bool> gpu_done{false};  // set by the stream callback
  SrvClock::time_point t_gpu_done;     // written before gpu_done
  struct glst_server *owner = nullptr;
};

// Device bytes a handle for `p` will hold (an upper bound of setup's sizes).
uint64_t estimate_bytes(const Plan &p, int nsm) {
  const uint64_t N = p.natom, C = p.ncell, K = p.has_far ? p.K() : 0;
  uint64_t b = N * (4 * 4 + 16 + 32 + 32 * (uint64_t)sr_rows_for(C, nsm) + 8 * 8 + 32) + C * 8 + 4096;
  if (K) {
    const uint64_t slots = (uint64_t)nsm * 16;
    const uint64_t kpad = (K + dev::kNodeBlock - 1) / dev::kNodeBlock * dev::kNodeBlock;
    const uint64_t nst = std::max<uint64_t>(1, (C * kpad * 16 + stage_budget() - 1) / stage_budget());
    // the largest stage: ~K / stages, plus up to one structure-factor unit of
    // directions (stages end on unit boundaries)
    uint32_t max_nr = 1;
    for (const auto &g : p.groups) max_nr = std::max(max_nr, g.n_radial);
    const uint64_t stage_k =
        nst == 1 ? kpad : std::min<uint64_t>(kpad, (K + nst - 1) / nst + (uint64_t)dev::kSfThreads * max_nr);
    // gather chunks of a stage (partial rows): enough to fill the GPU, at
    // most kMaxChunkNodes nodes each, one more per group boundary
    const uint64_t chunks = std::max<uint64_t>((8 * slots + C - 1) / C, stage_k / kMaxChunkNodes + 1) +
                            p.groups.size() + 1;
    const uint64_t stage_kpad = (stage_k + dev::kNodeBlock - 1) / dev::kNodeBlock * dev::kNodeBlock;
    b += K * (32 + 4 + 16 + 4) + C * stage_kpad * (8 + 8) + chunks * N * 32;
    // global-memory shell-sum tables (grids whose per-node table exceeds the
    // shared memory of a CTA): 64 MB or one block, and the twiddles
    if ((C + 9 + p.n[0] + p.n[1] + p.n[2]) * 16 > (200ull << 10))
      b += std::max<uint64_t>(64ull << 20, C * dev::kNodeBlock * 16) + stage_kpad * (p.n[0] + p.n[1] + p.n[2]) * 16;
  }
  return b + 64 * 16 * 64;  // per-buffer allocation granularity
}

}  // namespace

struct glst_server {
  int device = 0, nsm = 148;
  uint64_t budget = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_build;
  std::deque<SrvRequest *> queue;      // queued, building and ready requests, arrival order
  std::deque<SrvRequest *> to_build;   // requests whose system the builder creates
  std::unordered_map<uint64_t, SrvRequest *> reqs;
  std::unordered_map<uint64_t, SrvSystem *> resident;  // named systems
  std::unordered_map<uint64_t, bool> building_key;      // keys with a system under construction
  std::deque<SrvSlot> slots;  // stable addresses (stream callbacks point into it)
  std::vector<double *> old_pinned;    // outgrown staging, freed at destroy
  std::thread worker;
  std::vector<std::thread> builders;  // kSrvBuilders, so small builds need not wait behind large ones
  bool stop = false;          // worker: finish what is queued, then exit
  bool stop_builder = false;  // builder: exit (set after the worker has finished)
  uint64_t next_ticket = 1, clock = 0;
  uint64_t reserved = 0;               // bytes promised to systems being built
  std::deque<SrvSystem *> to_free;     // dropped systems, freed by a builder thread
  uint64_t freeing = 0;                // their bytes, until freed
  uint32_t large_in_flight = 0;        // running requests of >= kSrvSmallAtoms atoms
  glst_server_stats stats{};
};

// Take a system out of service (lock held).  Its device memory is freed by
// a builder thread, outside the lock: cudaFree waits for the whole device,
// which in the worker would stall every launch behind it.  Until then its
// bytes count against the budget as `freeing`.
static void srv_drop_system(glst_server *s, SrvSystem *sys) {
  if (sys->key) s->resident.erase(sys->key);
  s->stats.resident_bytes -= sys->bytes;
  s->stats.resident_systems--;
  s->freeing += sys->bytes;
  s->to_free.push_back(sys);
  s->cv_build.notify_one();
}

static void srv_free_now(SrvSystem *sys) {
  release(sys->h, /*device_idle=*/true);  // its last request has completed
  delete sys->h;
  delete sys;
}

static void srv_finish(glst_server *s, SrvRequest *r, glst_status st, const char *err) {
  r->status = st;
  if (err) r->err = err;
  r->t_done = SrvClock::now();
  r->state = SrvState::Done;
  s->stats.completed++;
  s->cv_done.notify_all();
}

// Evict idle named systems, least recently used first, until `need` fits.
static bool srv_make_room(glst_server *s, uint64_t need) {
  while (s->stats.resident_bytes + s->reserved + s->freeing + need > s->budget) {
    SrvSystem *victim = nullptr;
    for (auto &kv : s->resident)
      if (!kv.second->busy && (!victim || kv.second->last_use < victim->last_use)) victim = kv.second;
    if (!victim) return false;  // running requests (or pending frees) will make room
    srv_drop_system(s, victim);
    s->stats.evictions++;
  }
  return true;
}

// Admission of a queued request (lock held).  Returns true when the request
// moved on (ready, building, or finished with an error).
static bool srv_admit(glst_server *s, SrvRequest *r) {
  if (r->key) {
    if (s->building_key.count(r->key)) return false;  // its system is being built
    auto it = s->resident.find(r->key);
    if (it != s->resident.end()) {
      SrvSystem *c = it->second;
      if (c->busy) return false;  // the previous request of this system still runs
      const bool same = c->natom == r->natom && c->tol == r->tol && c->rcut == r->rcut && c->box[0] == r->box[0] &&
                        c->box[1] == r->box[1] && c->box[2] == r->box[2];
      if (same) {
        c->busy = true;
        c->last_use = ++s->clock;
        r->sys = c;
        r->state = SrvState::Ready;
        return true;
      }
      srv_drop_system(s, c);
    }
  }
  Plan p;
  try {
    auto store = get_store();
    p = glst::make_plan(r->natom, r->tol, r->box, r->rcut, 0, *store);
  } catch (const PlanError &e) {
    srv_finish(s, r, static_cast<glst_status>(e.status), e.msg.c_str());
    return true;
  }
  const uint64_t need = estimate_bytes(p, s->nsm);
  if (need > s->budget) {
    srv_finish(s, r, GLST_ERR_OUT_OF_MEMORY, "request larger than the server's memory budget");
    return true;
  }
  if (!srv_make_room(s, need)) return false;  // running requests will free memory
  s->reserved += need;
  r->reserved = need;
  r->state = SrvState::Building;
  if (r->key) s->building_key[r->key] = true;
  s->to_build.push_back(r);
  s->cv_build.notify_one();
  return true;
}

static constexpr int kSrvBuilders = 2;

// Requests of at least this many atoms fill the GPU by themselves.  (Running
// their far field in 8 node ranges, so that smaller requests could start
// between the ranges' launches, measured no better p50 and a worse p99.)
static constexpr uint32_t kSrvSmallAtoms = 20000;

static void srv_builder(glst_server *s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    s->cv_build.wait(lk, [&] { return s->stop_builder || !s->to_build.empty() || !s->to_free.empty(); });
    if (!s->to_free.empty()) {  // frees first: builds may be waiting for the memory
      SrvSystem *sys = s->to_free.front();
      s->to_free.pop_front();
      const uint64_t b = sys->bytes;
      lk.unlock();
      srv_free_now(sys);
      lk.lock();
      s->freeing -= b;
      s->cv_work.notify_all();
      continue;
    }
    if (s->to_build.empty()) {
      if (s->stop_builder) break;
      continue;
    }
    SrvRequest *r = s->to_build.front();
    s->to_build.pop_front();
    lk.unlock();
    auto h = std::make_unique<glst_handle>();
    const glst_status st = setup(h.get(), r->natom, r->tol, r->box, r->rcut, 0);
    const std::string err = st == GLST_OK ? std::string() : g_last_error;
    if (st != GLST_OK) release(h.get(), /*device_idle=*/true);  // nothing ran on it
    lk.lock();
    s->reserved -= r->reserved;
    r->reserved = 0;
    if (r->key) s->building_key.erase(r->key);
    if (st != GLST_OK) {
      for (auto it = s->queue.begin(); it != s->queue.end(); ++it)
        if (*it == r) {
          s->queue.erase(it);
          break;
        }
      srv_finish(s, r, st, err.c_str());
    } else {
      auto *sys = new SrvSystem();
      sys->key = r->key;
      sys->h = h.release();
      sys->bytes = sys->h->bytes;
      sys->natom = r->natom;
      sys->tol = r->tol;
      sys->rcut = r->rcut;
      for (int a = 0; a < 3; a++) sys->box[a] = r->box[a];
      sys->busy = true;
      sys->last_use = ++s->clock;
      s->stats.resident_bytes += sys->bytes;
      s->stats.peak_resident_bytes = std::max(s->stats.peak_resident_bytes, s->stats.resident_bytes);
      s->stats.resident_systems++;
      s->stats.systems_created++;
      if (r->key) s->resident[r->key] = sys;
      r->sys = sys;
      r->state = SrvState::Ready;
    }
    s->cv_work.notify_all();
  }
}

// Stream callback at the end of a request's work: no CUDA calls here, only
// the completion flag and a wake-up of the worker.
// It must not take the server's lock: the worker holds it across CUDA calls
// that may wait for pending callbacks (cudaFree synchronises the device).
static void CUDART_CB srv_done_cb(void *arg) {
  SrvSlot *sl = static_cast<SrvSlot *>(arg);
  sl->t_gpu_done = SrvClock::now();
  sl->gpu_done.store(true, std::memory_order_release);
  sl->owner->cv_work.notify_all();
}


// Launch a ready request on a free slot (lock held).  All slots have equal
// stream priority: giving small requests priority starved the large ones
// under overload (their thread blocks kept losing the SMs).
static void srv_launch(glst_server *s, SrvRequest *r, SrvSlot &sl) {
  SrvSystem *sys = r->sys;
  const size_t N = r->natom;
  if (sl.cap < N || !sl.pin) {
    // grow geometrically; an outgrown buffer is kept until destroy (freeing
    // pinned memory would synchronise the device mid-stream)
    if (sl.pin) s->old_pinned.push_back(sl.pin);
    sl.pin = nullptr;
    sl.cap = std::max<size_t>({N, 2 * sl.cap, 65536});
    if (cudaHostAlloc(reinterpret_cast<void **>(&sl.pin), (8 * sl.cap + 1) * sizeof(double), 0) != cudaSuccess) {
      cudaGetLastError();
      sl.cap = 0;
      sys->busy = false;
      if (!sys->key) srv_drop_system(s, sys);
      srv_finish(s, r, GLST_ERR_OUT_OF_MEMORY, "pinned staging allocation failed");
      return;
    }
  }
  glst_handle *h = sys->h;
  std::memcpy(sl.pin, r->in.data(), 4 * N * sizeof(double));
  glst_status st = GLST_OK;
  if (N && cudaMemcpyAsync(h->in_host, sl.pin, 4 * N * sizeof(double), cudaMemcpyHostToDevice, sl.st) != cudaSuccess)
    st = fail(GLST_ERR_CUDA, "request input copy failed");
  if (st == GLST_OK)
    st = compute_all(h, h->in_host, h->in_host + N, h->in_host + 2 * N, h->in_host + 3 * N, sl.st);
  double *src[4] = {h->ofx, h->ofy, h->ofz, h->oen};
  for (int k = 0; st == GLST_OK && k < 4; k++)
    if (N && cudaMemcpyAsync(sl.pin + (4 + k) * N, src[k], N * sizeof(double), cudaMemcpyDeviceToHost, sl.st) !=
                 cudaSuccess)
      st = fail(GLST_ERR_CUDA, "request output copy failed");
  if (st == GLST_OK &&
      cudaMemcpyAsync(sl.pin + 8 * N, h->energy, sizeof(double), cudaMemcpyDeviceToHost, sl.st) != cudaSuccess)
    st = fail(GLST_ERR_CUDA, "request energy copy failed");
  sl.gpu_done.store(false, std::memory_order_relaxed);
  sl.owner = s;
  if (st == GLST_OK && cudaLaunchHostFunc(sl.st, srv_done_cb, &sl) != cudaSuccess)
    st = fail(GLST_ERR_CUDA, "completion callback failed");
  if (st != GLST_OK) {
    cudaStreamSynchronize(sl.st);
    sys->busy = false;
    if (!sys->key) srv_drop_system(s, sys);
    srv_finish(s, r, st, g_last_error.c_str());
    return;
  }
  r->state = SrvState::Running;
  sl.req = r;
  s->stats.in_flight++;
}

static void srv_worker(glst_server *s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    bool progress = false;
    // 1. complete requests whose work finished (flag set by the callback)
    for (auto &sl : s->slots) {
      if (!sl.req || !sl.gpu_done.load(std::memory_order_acquire)) continue;
      cudaError_t q = cudaStreamQuery(sl.st);
      if (q == cudaErrorNotReady) q = cudaSuccess;  // only the callback itself is still returning
      SrvRequest *r = sl.req;
      const size_t N = r->natom;
      if (r->natom >= kSrvSmallAtoms) s->large_in_flight--;
      if (q == cudaSuccess) {
        r->out.assign(sl.pin + 4 * N, sl.pin + 8 * N);
        r->energy = sl.pin[8 * N];
      }
      r->sys->busy = false;
      if (!r->sys->key) srv_drop_system(s, r->sys);
      r->sys = nullptr;
      sl.req = nullptr;
      s->stats.in_flight--;
      srv_finish(s, r, q == cudaSuccess ? GLST_OK : GLST_ERR_CUDA,
                 q == cudaSuccess ? nullptr : cudaGetErrorString(q));
      r->t_done = sl.t_gpu_done;  // completion time as the GPU finished it
      sl.gpu_done.store(false, std::memory_order_relaxed);
      progress = true;
    }
    // 2. admit queued requests (they keep their place if they cannot start:
    //    system busy or being built, or memory full), launch ready ones
    for (auto it = s->queue.begin(); it != s->queue.end();) {
      SrvRequest *r = *it;
      if (r->state == SrvState::Queued && srv_admit(s, r)) progress = true;
      if (r->state == SrvState::Done) {
        it = s->queue.erase(it);
        continue;
      }
      // A large request fills the GPU by itself: run one at a time (two
      // would only split the SMs between them); small ones fill the gaps.
      const bool large = r->natom >= kSrvSmallAtoms;
      if (r->state == SrvState::Ready && !(large && s->large_in_flight > 0)) {
        SrvSlot *free_slot = nullptr;
        for (auto &sl : s->slots)
          if (!sl.req) {
            free_slot = &sl;
            break;
          }
        if (free_slot) {
          srv_launch(s, r, *free_slot);
          if (large && r->state == SrvState::Running) s->large_in_flight++;
          it = s->queue.erase(it);
          progress = true;
          continue;
        }
      }
      ++it;
    }
    if (s->stop && s->queue.empty() && s->stats.in_flight == 0) break;
    // Sleep, releasing the lock, until a submit, a finished build or a
    // completion callback notifies -- unless this pass made progress, which
    // may unblock more.  The timeout is only a safety net.
    if (!progress) {
      bool any_done = false;
      for (auto &sl : s->slots) any_done |= (sl.req && sl.gpu_done.load(std::memory_order_acquire));
      // short timeout: a callback's notify can land just before this wait
      if (!any_done) s->cv_work.wait_for(lk, std::chrono::microseconds(s->stats.in_flight ? 100 : 5000));
    }
  }
}

extern "C" {

glst_status glst_server_create(glst_server **out, uint64_t budget_bytes, uint32_t nslots) {
  if (!out || !budget_bytes) return fail(GLST_ERR_INVALID_ARG, "null output or zero budget");
  *out = nullptr;
  auto s = std::make_unique<glst_server>();
  CUDA_TRY(cudaGetDevice(&s->device));
  CUDA_TRY(cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, s->device));
  s->budget = budget_bytes;
  for (uint32_t i = 0; i < std::max<uint32_t>(1, nslots); i++) s->slots.emplace_back();
  for (auto &sl : s->slots) {
    CUDA_TRY(cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking));
    // staging for requests up to 262,144 atoms; larger ones grow it
    sl.cap = 262144;
    CUDA_TRY(cudaHostAlloc(reinterpret_cast<void **>(&sl.pin), (8 * sl.cap + 1) * sizeof(double), 0));
  }
  glst_server *raw = s.release();
  raw->worker = std::thread(srv_worker, raw);
  for (int i = 0; i < kSrvBuilders; i++) raw->builders.emplace_back(srv_builder, raw);
  *out = raw;
  return GLST_OK;
}

glst_status glst_server_destroy(glst_server *s) {
  if (!s) return GLST_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();  // drains the queue (needs the builder)
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop_builder = true;
  }
  s->cv_build.notify_all();
  for (auto &b : s->builders)
    if (b.joinable()) b.join();
  cudaSetDevice(s->device);
  cudaDeviceSynchronize();
  std::vector<SrvSystem *> left(s->to_free.begin(), s->to_free.end());
  for (auto &kv : s->resident) left.push_back(kv.second);
  for (auto *sys : left) srv_free_now(sys);
  for (auto &sl : s->slots) {
    if (sl.pin) cudaFreeHost(sl.pin);
    cudaStreamDestroy(sl.st);
  }
  for (double *p : s->old_pinned) cudaFreeHost(p);
  for (auto &kv : s->reqs) delete kv.second;
  delete s;
  return GLST_OK;
}

glst_status glst_server_submit(glst_server *s, uint64_t key, uint32_t natom, double tol, double bx, double by,
                               double bz, double rcut, const double *rx, const double *ry, const double *rz,
                               const double *qc, uint64_t *ticket) {
  if (!s || !ticket || (natom && (!rx || !ry || !rz || !qc))) return fail(GLST_ERR_INVALID_ARG, "null argument");
  auto r = new SrvRequest();
  r->key = key;
  r->natom = natom;
  r->tol = tol;
  r->box[0] = bx;
  r->box[1] = by;
  r->box[2] = bz;
  r->rcut = rcut;
  r->in.resize(4ull * natom);
  const double *src[4] = {rx, ry, rz, qc};
  for (int k = 0; k < 4; k++)
    if (natom) std::memcpy(r->in.data() + (size_t)k * natom, src[k], natom * sizeof(double));
  r->t_submit = SrvClock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      delete r;
      return fail(GLST_ERR_STATE, "server is stopping");
    }
    r->ticket = s->next_ticket++;
    s->reqs[r->ticket] = r;
    s->queue.push_back(r);
    s->stats.submitted++;
    *ticket = r->ticket;
  }
  s->cv_work.notify_all();
  return GLST_OK;
}

glst_status glst_server_wait(glst_server *s, uint64_t ticket, double *fx, double *fy, double *fz, double *en,
                             double *energy, double *latency_us, double timeout_ms) {
  if (!s) return fail(GLST_ERR_INVALID_ARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return fail(GLST_ERR_INVALID_ARG, "unknown ticket");
  SrvRequest *r = it->second;
  auto ready = [&] { return r->state == SrvState::Done; };
  if (timeout_ms < 0)
    s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready))
    return fail(GLST_ERR_STATE, "request not finished within the timeout");
  s->reqs.erase(it);
  lk.unlock();
  std::unique_ptr<SrvRequest> own(r);
  if (r->status != GLST_OK) return fail(r->status, "%s", r->err.c_str());
  const size_t N = r->natom;
  double *dst[4] = {fx, fy, fz, en};
  for (int k = 0; k < 4; k++)
    if (dst[k] && N) std::memcpy(dst[k], r->out.data() + (size_t)k * N, N * sizeof(double));
  if (energy) *energy = r->energy;
  if (latency_us) *latency_us = std::chrono::duration<double, std::micro>(r->t_done - r->t_submit).count();
  return GLST_OK;
}

glst_status glst_server_get_stats(glst_server *s, glst_server_stats *st) {
  if (!s || !st) return fail(GLST_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *st = s->stats;
  return GLST_OK;
}

}  // extern "C"
