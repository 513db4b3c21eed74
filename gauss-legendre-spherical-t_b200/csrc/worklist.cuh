// Batched work-list kernels: one persistent launch per phase covers many
// independent systems.  Each system is described by a SysDesc (its grid,
// buffers, node tables and where its inputs and outputs live); each phase has
// a list of work items (system, block indices) -- the same block indices the
// system's own launch would use -- and a grid of resident CTAs that take the
// items in a fixed stride (CTA b: items b, b + gridDim.x, ...).  Every item
// runs exactly the code of the one-system kernels (the *_block functions of
// kernels.cuh) on the same tables, so a system's results are bit for bit the
// ones it gets alone.
#pragma once

#include "kernels.cuh"

namespace glst {
namespace dev {

struct SysDesc {
  Grid g;
  uint32_t natom, combine_blocks, part_rows, use_far, sr_rows;
  SatArgs sat;  // shell-sum arguments (S, node tables, nodes per CTA, row stride, R)
  const double *rx, *ry, *rz, *qc;
  uint32_t *atom_cell, *atom_slot, *perm, *sorted_idx, *cell_count, *cell_point;
  float4 *pk;
  double4 *pd;
  const float4 *dirs;
  const float *kappa;
  const LrChunk *chunks;
  const SfUnit *sf_units;
  float2 *S, *R;
  double4 *part, *sr;
  double *cfx, *cfy, *cfz, *cen, *ofx, *ofy, *ofz, *oen, *block_energy, *energy;
};

struct WorkItem {
  uint32_t sys, a, b, pad;
};

// Cell counts to zero before binning: item a = block of 1024 cells.
__global__ void __launch_bounds__(1024) k_zero_counts_multi(const SysDesc *__restrict__ sys,
                                                            const WorkItem *__restrict__ items, uint32_t n) {
  for (uint32_t it = blockIdx.x; it < n; it += gridDim.x) {
    const WorkItem w = items[it];
    const SysDesc &d = sys[w.sys];
    const uint32_t c = w.a * 1024u + threadIdx.x;
    if (c < d.g.ncell) d.cell_count[c] = 0u;
  }
}

__global__ void __launch_bounds__(256) k_bin_multi(const SysDesc *__restrict__ sys,
                                                   const WorkItem *__restrict__ items, uint32_t n) {
  for (uint32_t it = blockIdx.x; it < n; it += gridDim.x) {
    const WorkItem w = items[it];
    const SysDesc &d = sys[w.sys];
    bin_block(d.rx, d.ry, d.rz, d.natom, d.g, d.atom_cell, d.atom_slot, d.cell_count, w.a);
  }
}

__global__ void __launch_bounds__(1024) k_scan_multi(const SysDesc *__restrict__ sys,
                                                     const WorkItem *__restrict__ items, uint32_t n) {
  for (uint32_t it = blockIdx.x; it < n; it += gridDim.x) {
    const SysDesc &d = sys[items[it].sys];
    scan_body(d.cell_count, d.g.ncell, d.cell_point);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_scatter_multi(const SysDesc *__restrict__ sys,
                                                       const WorkItem *__restrict__ items, uint32_t n) {
  for (uint32_t it = blockIdx.x; it < n; it += gridDim.x) {
    const WorkItem w = items[it];
    const SysDesc &d = sys[w.sys];
    scatter_block(d.atom_cell, d.atom_slot, d.cell_point, d.natom, d.perm, w.a);
  }
}

// item a = cell; kSortCap u32 of dynamic shared memory
__global__ void __launch_bounds__(256) k_sort_pack_multi(const SysDesc *__restrict__ sys,
                                                         const WorkItem *__restrict__ items, uint32_t n) {
  for (uint32_t it = blockIdx.x; it < n; it += gridDim.x) {
    const WorkItem w = items[it];
    const SysDesc &d = sys[w.sys];
    sort_pack_block(d.perm, d.cell_count, d.cell_point, d.g, d.atom_cell, d.natom, d.rx, d.ry, d.rz, d.qc,
                    d.sorted_idx, d.pk, d.pd, w.a);
    __syncthreads();
  }
}

// item (a, b) = (structure-factor unit, cell row).  Seven CTAs per SM (72
// registers): the descriptor's pointers take registers the one-system kernel
// reads from its parameters, and at eight CTAs (64 registers) they spilled.
__global__ void __launch_bounds__(kSfThreads, 7) k_structure_factors_multi(const SysDesc *__restrict__ sys,
                                                                          const WorkItem *__restrict__ items,
                                                                          uint32_t n) {
  for (uint32_t it = blockIdx.x; it < n; it += gridDim.x) {
    const WorkItem w = items[it];
    const SysDesc &d = sys[w.sys];
    sf_block(d.pk, d.cell_count, d.cell_point, d.g, d.sf_units, d.dirs, d.kappa, 0, 0, d.S, d.R, w.a, w.b);
    __syncthreads();
  }
}

// item a = block of nb nodes; dynamic shared memory: the largest system's
// rows, twiddles and coordinate table
__global__ void __launch_bounds__(kSatThreads, 3) k_shell_sums_multi(const SysDesc *__restrict__ sys,
                                                                     const WorkItem *__restrict__ items,
                                                                     uint32_t n) {
  for (uint32_t it = blockIdx.x; it < n; it += gridDim.x) {
    const WorkItem w = items[it];
    const SysDesc &d = sys[w.sys];
    shell_block<3>(d.g, d.sat, w.a);
    __syncthreads();
  }
}

// item (a, b) = (block of kLrThreads atoms, long-range chunk); seven CTAs per
// SM, as the structure factors; the default polynomial share (the work
// list takes only systems with the default launch variants)
__global__ void __launch_bounds__(kLrThreads, 7) k_long_range_multi(const SysDesc *__restrict__ sys,
                                                                    const WorkItem *__restrict__ items,
                                                                    uint32_t n) {
  for (uint32_t it = blockIdx.x; it < n; it += gridDim.x) {
    const WorkItem w = items[it];
    const SysDesc &d = sys[w.sys];
    lr_block<kLrPolyMasks[0], false>(d.pk, d.cell_point, d.g.ncell, d.chunks, d.dirs, d.kappa, d.R, 0, d.natom, 0,
                              d.part, w.a, w.b);
    __syncthreads();
  }
}

// item (a, b) = (cell, row of neighbour cells)
__global__ void __launch_bounds__(kSrThreads) k_short_range_multi(const SysDesc *__restrict__ sys,
                                                                  const WorkItem *__restrict__ items,
                                                                  uint32_t n) {
  for (uint32_t it = blockIdx.x; it < n; it += gridDim.x) {
    const WorkItem w = items[it];
    const SysDesc &d = sys[w.sys];
    if (d.sr_rows == kSrRowsLines)
      sr_block<true>(d.pd, d.cell_count, d.cell_point, d.g, d.natom, d.sr, d.sr_rows, w.a, w.b);
    else
      sr_block<false>(d.pd, d.cell_count, d.cell_point, d.g, d.natom, d.sr, d.sr_rows, w.a, w.b);
    __syncthreads();
  }
}

// item a = block of kCombineAtoms atoms
__global__ void __launch_bounds__(kCombineThreads) k_combine_multi(const SysDesc *__restrict__ sys,
                                                                   const WorkItem *__restrict__ items,
                                                                   uint32_t n) {
  for (uint32_t it = blockIdx.x; it < n; it += gridDim.x) {
    const WorkItem w = items[it];
    const SysDesc &d = sys[w.sys];
    combine_block(d.sr, d.sr_rows, d.part, d.part_rows, d.sorted_idx, d.natom, d.use_far, d.cfx, d.cfy, d.cfz, d.cen, d.ofx,
                  d.ofy, d.ofz, d.oen, d.block_energy, w.a);
    __syncthreads();
  }
}

// one item per system
__global__ void __launch_bounds__(256) k_energy_multi(const SysDesc *__restrict__ sys,
                                                      const WorkItem *__restrict__ items, uint32_t n) {
  for (uint32_t it = blockIdx.x; it < n; it += gridDim.x) {
    const SysDesc &d = sys[items[it].sys];
    energy_body(d.block_energy, d.combine_blocks, d.energy);
    __syncthreads();
  }
}

}  // namespace dev
}  // namespace glst
