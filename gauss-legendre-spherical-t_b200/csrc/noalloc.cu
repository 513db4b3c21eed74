// Allocation-free near field: glst_near_field_noalloc (see glst_c.h).
//
// Some callers cannot allocate device memory at the moment they need the
// near-field forces: code running while a CUDA stream is being captured into
// a graph (cudaMalloc is not allowed during capture), engines that hand the
// whole device to their own memory pool and forbid allocation inside a time
// step, and plugins loaded into such hosts.  This entry point serves them: its
// working memory is one file-scope __device__ array of fixed size, which
// exists on every GPU that loads this library from module load until process
// exit.  The caller passes inputs and outputs only; nothing here calls
// cudaMalloc, cudaFree or any allocating routine.
//
// The near field computed here is the sum over the own cell and its 26
// neighbours of the reference's cell grid (bare Coulomb, open boundary) --
// exactly what glst_compute returns when the grid has at most two cells along
// some axis, where the reference has no far field (src/glst_force.cu:667-670).
#include <cstdint>
#include <cstdio>
#include <mutex>

#include <cuda_runtime.h>

#include "glst_c.h"

// The engine's kernels, compiled again here with internal linkage (this file
// is a translation unit of its own and must not clash with engine.cu).
namespace {
#include "kernels.cuh"
namespace kdev = glst::dev;  // this file's copy of the kernels
}  // namespace

// engine.cu: sets the text glst_last_error returns (hidden, C++ linkage)
void glst_internal_set_last_error(const char *msg);

namespace {

constexpr uint32_t kMaxAtoms = GLST_NOALLOC_MAX_ATOMS;
constexpr uint32_t kMaxCells = GLST_NOALLOC_MAX_CELLS;

// Byte offsets of the pieces of the scratch array (each 256-byte aligned).
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffCount = 0;
constexpr size_t kOffPoint = kOffCount + align256(4ull * kMaxCells);
constexpr size_t kOffCell = kOffPoint + align256(4ull * kMaxCells);
constexpr size_t kOffSlot = kOffCell + align256(4ull * kMaxAtoms);
constexpr size_t kOffPerm = kOffSlot + align256(4ull * kMaxAtoms);
constexpr size_t kOffSorted = kOffPerm + align256(4ull * kMaxAtoms);
constexpr size_t kOffPk = kOffSorted + align256(4ull * kMaxAtoms);
constexpr size_t kOffPd = kOffPk + align256(16ull * kMaxAtoms);
constexpr size_t kOffSr = kOffPd + align256(32ull * kMaxAtoms);
constexpr size_t kOffCellOut = kOffSr + align256(32ull * kdev::kSrRowsPlanes * kMaxAtoms);
constexpr size_t kOffBlockE = kOffCellOut + align256(4ull * 8ull * kMaxAtoms);
constexpr size_t kScratchBytes =
    kOffBlockE + align256(8ull * ((kMaxAtoms + kdev::kCombineAtoms - 1) / kdev::kCombineAtoms));
static_assert(kScratchBytes == GLST_NOALLOC_SCRATCH_BYTES, "scratch size in glst_c.h is stale");

// The scratch.  In host code `g_scratch` names a host-side stand-in, not
// device memory: only the address returned by cudaGetSymbolAddress (taken
// once per device, with that device current) is passed to kernels.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_scratch_dev[kMaxDevices] = {};

thread_local char g_err[256];  // message of the current call, handed to glst_last_error

glst_status failed(glst_status s) {
  glst_internal_set_last_error(g_err);
  return s;
}

glst_status setup_scratch(int device, unsigned char **out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_dev[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) {
      std::snprintf(g_err, sizeof g_err, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
      return failed(GLST_ERR_CUDA);
    }
    g_scratch_dev[device] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch_dev[device];
  return GLST_OK;
}

}  // namespace

extern "C" glst_status glst_near_field_noalloc(uint32_t natom, const double *d_rx, const double *d_ry,
                                               const double *d_rz, const double *d_qc, double box_x,
                                               double box_y, double box_z, double rcut, glst_ct ct,
                                               double *d_fx, double *d_fy, double *d_fz, double *d_en,
                                               void *stream) {
  g_err[0] = 0;
  if (natom > kMaxAtoms) {
    std::snprintf(g_err, sizeof g_err, "natom %u exceeds the allocation-free limit of %u atoms", natom,
                  kMaxAtoms);
    return failed(GLST_ERR_SIZE);
  }
  if (natom && (!d_rx || !d_ry || !d_rz || !d_qc || !d_fx || !d_fy || !d_fz || !d_en)) {
    std::snprintf(g_err, sizeof g_err, "null input or output pointer");
    return failed(GLST_ERR_INVALID_ARG);
  }
  if (!(rcut > 0.0) || !(box_x > 0.0) || !(box_y > 0.0) || !(box_z > 0.0) ||
      (ct != GLST_CT_DOUBLE && ct != GLST_CT_FLOAT)) {
    std::snprintf(g_err, sizeof g_err, "box and rcut must be > 0 and ct valid");
    return failed(GLST_ERR_INVALID_ARG);
  }
  // Cell grid in CT, as glst_create plans it (src/glst_force.cu:223-241).
  // Each axis' cell count is checked against the limit before it is
  // converted to an integer (a ratio beyond the range of `unsigned`, or not
  // finite, would make the conversion undefined), so the product below
  // cannot wrap either.
  const double box[3] = {box_x, box_y, box_z};
  for (int a = 0; a < 3; a++) {
    const double ratio = ct == GLST_CT_FLOAT ? static_cast<double>(static_cast<float>(box[a]) / static_cast<float>(rcut))
                                             : box[a] / rcut;
    if (!(ratio < static_cast<double>(kMaxCells))) {
      std::snprintf(g_err, sizeof g_err, "box / rcut along axis %d exceeds the allocation-free limit of %u cells",
                    a, kMaxCells);
      return failed(GLST_ERR_SIZE);
    }
  }
  uint32_t n[3];
  double l;
  if (ct == GLST_CT_FLOAT) {
    const float lf = static_cast<float>(rcut);
    for (int a = 0; a < 3; a++) {
      const float L = static_cast<float>(box[a]);
      unsigned c = static_cast<unsigned>(L / lf);
      if (static_cast<float>(c) * lf < L) c++;
      n[a] = c;
    }
    l = static_cast<double>(lf);
  } else {
    for (int a = 0; a < 3; a++) {
      unsigned c = static_cast<unsigned>(box[a] / rcut);
      if (static_cast<double>(c) * rcut < box[a]) c++;
      n[a] = c;
    }
    l = rcut;
  }
  const uint64_t ncell = (uint64_t)n[0] * n[1] * n[2];
  if (ncell == 0 || ncell > kMaxCells) {
    std::snprintf(g_err, sizeof g_err, "cell grid of %llu cells exceeds the allocation-free limit of %u",
                  (unsigned long long)ncell, kMaxCells);
    return failed(GLST_ERR_SIZE);
  }
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess || device < 0 || device >= kMaxDevices) {
    std::snprintf(g_err, sizeof g_err, "no usable current device");
    return failed(GLST_ERR_NO_DEVICE);
  }
  unsigned char *base = nullptr;
  const glst_status s = setup_scratch(device, &base);
  if (s != GLST_OK) return s;

  namespace dev = kdev;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const dev::Grid g{n[0], n[1], n[2], (uint32_t)ncell, l, ct == GLST_CT_FLOAT ? 1 : 0};
  uint32_t *cell_count = reinterpret_cast<uint32_t *>(base + kOffCount);
  uint32_t *cell_point = reinterpret_cast<uint32_t *>(base + kOffPoint);
  uint32_t *atom_cell = reinterpret_cast<uint32_t *>(base + kOffCell);
  uint32_t *atom_slot = reinterpret_cast<uint32_t *>(base + kOffSlot);
  uint32_t *perm = reinterpret_cast<uint32_t *>(base + kOffPerm);
  uint32_t *sorted = reinterpret_cast<uint32_t *>(base + kOffSorted);
  float4 *pk = reinterpret_cast<float4 *>(base + kOffPk);
  double4 *pd = reinterpret_cast<double4 *>(base + kOffPd);
  double4 *sr = reinterpret_cast<double4 *>(base + kOffSr);
  double *cell_out = reinterpret_cast<double *>(base + kOffCellOut);
  double *block_e = reinterpret_cast<double *>(base + kOffBlockE);

  // The array keeps the previous call's contents: the cell counts restart at
  // 0 (everything else is written before it is read).
  if ((e = cudaMemsetAsync(cell_count, 0, 4ull * ncell, st)) != cudaSuccess) {
    std::snprintf(g_err, sizeof g_err, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
    return failed(GLST_ERR_CUDA);
  }
  if (natom) {
    const uint32_t nb = (natom + 255) / 256;
    dev::k_bin<<<nb, 256, 0, st>>>(d_rx, d_ry, d_rz, natom, g, atom_cell, atom_slot, cell_count);
    dev::k_scan<<<1, 1024, 0, st>>>(cell_count, (uint32_t)ncell, cell_point);
    dev::k_scatter<<<nb, 256, 0, st>>>(atom_cell, atom_slot, cell_point, natom, perm);
    dev::k_sort_pack<<<(uint32_t)ncell, 256, dev::kSortCap * sizeof(uint32_t), st>>>(
        perm, cell_count, cell_point, g, atom_cell, natom, d_rx, d_ry, d_rz, d_qc, sorted, pk, pd);
    dev::k_short_range<<<dim3((uint32_t)ncell, dev::kSrRowsPlanes), dev::kSrThreads, 0, st>>>(
        pd, cell_count, cell_point, g, natom, sr, dev::kSrRowsPlanes);
    dev::k_combine<<<(natom + dev::kCombineAtoms - 1) / dev::kCombineAtoms, dev::kCombineThreads, 0, st>>>(
        sr, dev::kSrRowsPlanes, nullptr, 0, sorted, natom, 0, cell_out, cell_out + kMaxAtoms, cell_out + 2ull * kMaxAtoms,
        cell_out + 3ull * kMaxAtoms, d_fx, d_fy, d_fz, d_en, block_e);
    if ((e = cudaGetLastError()) != cudaSuccess) {
      std::snprintf(g_err, sizeof g_err, "kernel launch failed: %s", cudaGetErrorString(e));
      return failed(GLST_ERR_CUDA);
    }
  }
  return GLST_OK;
}
