// GLST device kernels for sm_100a (B200).
//
// Data layout in HBM (one system):
//   pk[N]      float4 (dx, dy, dz, q): cell-ordered atoms, position relative
//              to the centre of the atom's cell, computed in FP64 and rounded
//   pd[N]      double4 (x, y, z, q): cell-ordered atoms, FP64 absolute
//   S[C][K]    float2: cell-relative structure factor sum_j q_j e^{-ik.(r_j - c)}
//              of every cell at every node (FP32 per atom tile, FP64 across
//              tiles, stored rounded to FP32)
//   R[C][K]    float2: shell sum times weight times e^{+ik.c} (cell centre c)
//   part[P][N] double4: long-range partial sums, one row per node chunk
//   sr[W][N]   double4: near-field sums, one row per row of neighbour cells
// Cell c = (ix*ny + iy)*nz + iz, as in the reference (src/glst_force.cu:379-382).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace glst {
namespace dev {

constexpr unsigned kSortCap = 8192;   // atoms per cell the shared-memory cell sort holds

struct Grid {
  uint32_t nx, ny, nz, ncell;
  double l;       // cell edge (CT value widened to double)
  int ct_float;   // bin in float arithmetic (glst_force<float>)
};

// Layout of the structure factors S and shell sums R (C cells x K nodes):
// blocks of kNodeBlock consecutive nodes, each block cell-major, so that a
// cell's run of nodes is contiguous within a block (the structure-factor
// stores and the long-range loads) and one node's values over all cells lie
// in one C x kNodeBlock region (the shell-sum loads and stores; a plain
// cell-major layout put them a whole row apart, one page per cell).
// Buffers hold C x ceil(K / kNodeBlock) x kNodeBlock elements.
constexpr uint32_t kNodeBlock = 32;
__host__ __device__ __forceinline__ size_t sr_index(uint32_t c, uint32_t k, uint32_t ncell) {
  return ((size_t)(k / kNodeBlock) * ncell + c) * kNodeBlock + (k % kNodeBlock);
}

// SFU sine and cosine of an FP32 angle in radians (PTX sin/cos.approx,
// flush-to-zero).  Absolute error ~1e-6 for the |x| < ~30 rad used here,
// below the FP32 rounding of the phase itself at that magnitude.
__device__ __forceinline__ void sfu_sincos(float x, float *s, float *c) {
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(*s) : "f"(x));
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(*c) : "f"(x));
}

__device__ __forceinline__ double cell_centre(uint32_t i, double l) {
  return (static_cast<double>(i) + 0.5) * l;
}

// ----------------------------------------------------------------------------
// Cell assignment.  Binning follows calc_cell_atom_count_kernel
// (src/glst_force.cu:356-386): the coordinate (converted to CT) times 1/l in
// CT, truncated toward zero, clamped to [0, n-1].
__device__ __forceinline__ uint32_t bin_axis(double r, const Grid &g, uint32_t n) {
  int c;
  if (g.ct_float) {
    const float inv = __fdiv_rn(1.0f, static_cast<float>(g.l));
    c = static_cast<int>(__fmul_rn(static_cast<float>(r), inv));
  } else {
    const double inv = __ddiv_rn(1.0, g.l);
    c = static_cast<int>(__dmul_rn(r, inv));
  }
  c = (c >= static_cast<int>(n)) ? static_cast<int>(n) - 1 : c;
  c = (c < 0) ? 0 : c;
  return static_cast<uint32_t>(c);
}

// K_bin: cell of every atom and an (unordered) slot inside the cell.
// (Each kernel's body is a device function of its block indices, so that
// the batched work-list kernels can run the same code for many systems.)
__device__ __forceinline__ void bin_block(const double *__restrict__ rx, const double *__restrict__ ry,
                                          const double *__restrict__ rz, uint32_t n, const Grid &g,
                                          uint32_t *__restrict__ atom_cell, uint32_t *__restrict__ atom_slot,
                                          uint32_t *__restrict__ cell_count, uint32_t bx) {
  const uint32_t i = bx * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t cx = bin_axis(rx[i], g, g.nx);
  const uint32_t cy = bin_axis(ry[i], g, g.ny);
  const uint32_t cz = bin_axis(rz[i], g, g.nz);
  const uint32_t cell = (cx * g.ny + cy) * g.nz + cz;
  atom_cell[i] = cell;
  atom_slot[i] = atomicAdd(&cell_count[cell], 1u);
}

__global__ void k_bin(const double *__restrict__ rx, const double *__restrict__ ry,
                      const double *__restrict__ rz, uint32_t n, Grid g,
                      uint32_t *__restrict__ atom_cell, uint32_t *__restrict__ atom_slot,
                      uint32_t *__restrict__ cell_count) {
  bin_block(rx, ry, rz, n, g, atom_cell, atom_slot, cell_count, blockIdx.x);
}

// K_scan: exclusive offsets of the cell counts (one CTA of 1024 threads,
// chunked block scan).
__device__ __forceinline__ void scan_body(const uint32_t *__restrict__ cell_count, uint32_t ncell,
                                          uint32_t *__restrict__ cell_point) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t base = 0; base < ncell; base += blockDim.x) {
    const uint32_t c = base + threadIdx.x;
    const uint32_t v = (c < ncell) ? cell_count[c] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (unsigned)o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      const unsigned nw = blockDim.x >> 5;
      uint32_t s = (lane < nw) ? warp_sums[lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= (unsigned)o) s += y;
      }
      if (lane < nw) warp_sums[lane] = s;
    }
    __syncthreads();
    const uint32_t before = carry + (warp ? warp_sums[warp - 1] : 0u) + (x - v);
    if (c < ncell) cell_point[c] = before;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + v;
    __syncthreads();
  }
}

__global__ void k_scan(const uint32_t *__restrict__ cell_count, uint32_t ncell,
                       uint32_t *__restrict__ cell_point) {
  scan_body(cell_count, ncell, cell_point);
}

__device__ __forceinline__ void scatter_block(const uint32_t *__restrict__ atom_cell,
                                              const uint32_t *__restrict__ atom_slot,
                                              const uint32_t *__restrict__ cell_point, uint32_t n,
                                              uint32_t *__restrict__ perm, uint32_t bx) {
  const uint32_t i = bx * blockDim.x + threadIdx.x;
  if (i >= n) return;
  perm[cell_point[atom_cell[i]] + atom_slot[i]] = i;
}

__global__ void k_scatter(const uint32_t *__restrict__ atom_cell,
                          const uint32_t *__restrict__ atom_slot,
                          const uint32_t *__restrict__ cell_point, uint32_t n,
                          uint32_t *__restrict__ perm) {
  scatter_block(atom_cell, atom_slot, cell_point, n, perm, blockIdx.x);
}

// K_sort_pack: one CTA per cell.  The atomics of k_bin leave the atoms of a
// cell in arbitrary order; sorting each cell's indices ascending reproduces
// the order of a stable sort by cell id (the reference's CUB radix sort,
// src/glst_force.cu:510-517).  Then writes the packets.  Launched with
// blockDim.x a multiple of 32 and kSortCap u32 of dynamic shared memory.
__device__ __forceinline__ void pack_atom(uint32_t slot, uint32_t a, double cx, double cy, double cz,
                                          const double *__restrict__ rx, const double *__restrict__ ry,
                                          const double *__restrict__ rz, const double *__restrict__ qc,
                                          uint32_t *__restrict__ sorted_idx, float4 *__restrict__ pk,
                                          double4 *__restrict__ pd) {
  const double x = rx[a], y = ry[a], z = rz[a], q = qc[a];
  sorted_idx[slot] = a;
  pd[slot] = make_double4(x, y, z, q);
  pk[slot] = make_float4(static_cast<float>(x - cx), static_cast<float>(y - cy), static_cast<float>(z - cz),
                         static_cast<float>(q));
}

__device__ __forceinline__ void sort_pack_block(const uint32_t *__restrict__ perm,
                                                const uint32_t *__restrict__ cell_count,
                                                const uint32_t *__restrict__ cell_point, const Grid &g,
                                                const uint32_t *__restrict__ atom_cell, uint32_t natom,
                                                const double *__restrict__ rx, const double *__restrict__ ry,
                                                const double *__restrict__ rz, const double *__restrict__ qc,
                                                uint32_t *__restrict__ sorted_idx, float4 *__restrict__ pk,
                                                double4 *__restrict__ pd, uint32_t cell) {
  extern __shared__ uint32_t s_idx[];
  const uint32_t cnt = cell_count[cell];
  const uint32_t start = cell_point[cell];
  if (cnt == 0) return;
  const uint32_t ix = cell / (g.ny * g.nz), iy = (cell / g.nz) % g.ny, iz = cell % g.nz;
  const double cx = cell_centre(ix, g.l), cy = cell_centre(iy, g.l), cz = cell_centre(iz, g.l);
  if (cnt > kSortCap) {
    // Too many atoms for the shared-memory sort: an atom's place in the cell
    // is the number of atoms of the cell with a smaller index, found by one
    // pass over every atom's cell in index order (per step: a warp ballot per
    // warp, then the counts of the warps before).  Stable by construction;
    // O(natom) per such cell, which only dense grids have.
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t seen = 0;
    for (uint32_t i0 = 0; i0 < natom; i0 += blockDim.x) {
      const uint32_t i = i0 + threadIdx.x;
      const bool mine = i < natom && atom_cell[i] == cell;
      const uint32_t bal = __ballot_sync(0xffffffffu, mine);
      if (lane == 0) s_idx[warp] = __popc(bal);
      __syncthreads();
      uint32_t before = seen, total = seen;
      for (uint32_t w = 0; w < nw; w++) {
        const uint32_t c = s_idx[w];
        before += (w < warp) ? c : 0u;
        total += c;
      }
      if (mine) sorted_idx[start + before + __popc(bal & ((1u << lane) - 1u))] = i;
      seen = total;
      __syncthreads();
    }
    for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x)
      pack_atom(start + i, sorted_idx[start + i], cx, cy, cz, rx, ry, rz, qc, sorted_idx, pk, pd);
    return;
  }
  uint32_t np2 = 1;
  while (np2 < cnt) np2 <<= 1;
  for (uint32_t i = threadIdx.x; i < np2; i += blockDim.x)
    s_idx[i] = (i < cnt) ? perm[start + i] : 0xffffffffu;
  __syncthreads();
  // bitonic sort, ascending
  for (uint32_t k = 2; k <= np2; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < np2; i += blockDim.x) {
        const uint32_t p = i ^ j;
        if (p > i) {
          const uint32_t a = s_idx[i], b = s_idx[p];
          const bool up = ((i & k) == 0);
          if ((a > b) == up) {
            s_idx[i] = b;
            s_idx[p] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x)
    pack_atom(start + i, s_idx[i], cx, cy, cz, rx, ry, rz, qc, sorted_idx, pk, pd);
}

__global__ void k_sort_pack(const uint32_t *__restrict__ perm,
                            const uint32_t *__restrict__ cell_count,
                            const uint32_t *__restrict__ cell_point, Grid g,
                            const uint32_t *__restrict__ atom_cell, uint32_t natom,
                            const double *__restrict__ rx, const double *__restrict__ ry,
                            const double *__restrict__ rz, const double *__restrict__ qc,
                            uint32_t *__restrict__ sorted_idx, float4 *__restrict__ pk,
                            double4 *__restrict__ pd) {
  sort_pack_block(perm, cell_count, cell_point, g, atom_cell, natom, rx, ry, rz, qc, sorted_idx, pk, pd,
                  blockIdx.x);
}

// ----------------------------------------------------------------------------
// Sine and cosine on the FP32 FMA pipe, for part of the (atom, node) pairs so
// that the FMA pipe carries some of the work the MUFU pipe would otherwise
// serialise.  Method: theta = n pi + r with n = rint(theta / pi) (rounded by
// adding 1.5 * 2^23), r = theta - n pi in two FMA steps (pi = kPiHi + kPiLo,
// kPiHi with 8 significant bits so n * kPiHi is exact), then
//   sin r = r + r^3 P(r^2),  cos r = Q(r^2)   on |r| <= pi/2,
// with P of degree 3 and Q of degree 4, coefficients fitted by this project
// (Lawson-weighted least squares on [0, (pi/2)^2], csrc/fit_sincos.py).
// sin(theta) = (-1)^n sin r, cos(theta) = (-1)^n cos r: the common sign is
// returned folded into a factor (the atom's charge) instead of applied to
// both results.  Max abs error 1.8e-7 for |theta| <= 30.
constexpr float kInvPi = 0.318309886183790672f;
constexpr float kRoundMagic = 12582912.0f;  // 1.5 * 2^23
constexpr float kPiHi = 3.140625f;
constexpr float kPiLo = 9.67653589793e-4f;
constexpr float kSin1 = -0.16666658222675323f, kSin2 = 0.008333051577210426f,
                kSin3 = -0.000198090827325359f, kSin4 = 2.6052375687868334e-06f;
constexpr float kCos0 = 0.9999999403953552f, kCos1 = -0.4999990463256836f, kCos2 = 0.04166358709335327f,
                kCos3 = -0.0013853712007403374f, kCos4 = 2.3154068912845105e-05f;

__device__ __forceinline__ void fma_sincos_signed(float th, float q, float *s, float *c, float *qs) {
  const float t = fmaf(th, kInvPi, kRoundMagic);
  const float n = t - kRoundMagic;
  float r = fmaf(-n, kPiHi, th);
  r = fmaf(-n, kPiLo, r);
  const float r2 = r * r;
  float p = fmaf(kSin4, r2, kSin3);
  p = fmaf(p, r2, kSin2);
  p = fmaf(p, r2, kSin1);
  *s = fmaf(p * r2, r, r);
  float cc = fmaf(kCos4, r2, kCos3);
  cc = fmaf(cc, r2, kCos2);
  cc = fmaf(cc, r2, kCos1);
  *c = fmaf(cc, r2, kCos0);
  *qs = __int_as_float(__float_as_int(q) ^ (__float_as_int(t) << 31));
}

// The same polynomial on two angles at once with the paired FP32
// instructions of sm_100 (FFMA2/FMUL2/FADD2: two IEEE FP32 operations per
// instruction, each lane bit-identical to the scalar form above).
__device__ __forceinline__ float2 bcast(float v) { return make_float2(v, v); }

__device__ __forceinline__ void fma_sincos_signed2(float2 th, float q, float2 *s, float2 *c, float2 *qs) {
  const float2 t = __ffma2_rn(th, bcast(kInvPi), bcast(kRoundMagic));
  const float2 n = __fadd2_rn(t, bcast(-kRoundMagic));
  float2 r = __ffma2_rn(n, bcast(-kPiHi), th);
  r = __ffma2_rn(n, bcast(-kPiLo), r);
  const float2 r2 = __fmul2_rn(r, r);
  float2 p = __ffma2_rn(bcast(kSin4), r2, bcast(kSin3));
  p = __ffma2_rn(p, r2, bcast(kSin2));
  p = __ffma2_rn(p, r2, bcast(kSin1));
  *s = __ffma2_rn(__fmul2_rn(p, r2), r, r);
  float2 cc = __ffma2_rn(bcast(kCos4), r2, bcast(kCos3));
  cc = __ffma2_rn(cc, r2, bcast(kCos2));
  cc = __ffma2_rn(cc, r2, bcast(kCos1));
  *c = __ffma2_rn(cc, r2, bcast(kCos0));
  const int qi = __float_as_int(q);
  *qs = make_float2(__int_as_float(qi ^ (__float_as_int(t.x) << 31)),
                    __int_as_float(qi ^ (__float_as_int(t.y) << 31)));
}

// ----------------------------------------------------------------------------
// Structure factors.  S_c(k) = sum_{j in c} q_j e^{-i k.r_j}
//                            = e^{-i k.c} sum_j q_j e^{-i k.d_j},  d_j = r_j - c.
// Nodes are k = kappa_r s (group -> direction -> radial), so per atom and
// direction u = s.d_j is formed once and each node's phase is one multiply.
// A CTA takes one work unit -- up to 128 / nb directions of one group, nb
// threads per direction, each thread NPT consecutive radial nodes -- and
// kSfCellsPerCta consecutive cells.  Per (atom, node): one multiply, a sine
// and cosine (SFU, or the FMA-pipe polynomial for the last slot pairs), two
// FMAs, in paired FP32 instructions where two slots go together.  FP32 over a
// tile of <= kSfAtomTile atoms (|k.d| <~ 25 rad), then FP64 over the tiles of
// a denser cell.  S is stored cell-relative in FP32; its twiddle e^{-ik.c}
// is applied by the shell-sum kernel as it loads S.
constexpr int kSfThreads = 128;
constexpr int kSfMaxNpt = 12;     // radial nodes per thread, at most
constexpr int kSfCellsPerCta = 2;
constexpr int kSfAtomTile = 128;

struct SfUnit {
  uint32_t node_begin;   // local internal index of (first direction, r = 0)
  uint32_t dir_begin;    // global direction index of the first direction
  uint32_t n_dir;        // directions in the unit (<= kSfThreads / nb)
  uint32_t n_rad;        // radial nodes per direction in this group
  uint32_t nb;           // threads per direction
  uint32_t npt;          // radial nodes per thread (nb * npt >= n_rad)
  uint32_t kappa_begin;  // offset of this group's radial table
  uint32_t pad;
};

// Slot pairs on the FMA pipe.  Per slot a polynomial costs ~21 FP32
// operations and a SFU slot 4 FP32 operations plus 2 MUFU operations, each of
// which occupies the SFU for 8 cycles of a warp.  Measured on water10k
// (npt 11 / 9 / 10 in its three groups): SF 1.47 ms with no pairs, 1.31 ms
// with (npt - 1) / 4 (2/2/2), 1.25 ms with (npt - 3) / 4 (2/1/1), 1.28 ms
// with one pair everywhere, 1.29 ms with (npt - 3) / 3 (2/2/2 + ...).
// Re-measured with S stored cell-relative in FP32 (no FP64 epilogue): 1.10 ms
// with (npt - 3) / 4, 1.16 with (npt - 5) / 4, 1.17 with npt / 4, 1.19 with
// (npt - 1) / 4, 1.30 with (npt + 1) / 4.
__host__ __device__ constexpr int sf_poly_pairs(int npt) { return (npt - 3) / 4; }

// A cell of several tiles adds them in FP64: the running sum is kept between
// tiles as an unevaluated pair of floats, the leading part in S and the
// remainder in lo_buf (the shell sums' output buffer, which is free until
// the structure factors are done); the last tile stores the sum rounded once
// to FP32.  Out of line, so that the registers of this rare path do not
// count against the hot loop's.
__device__ __noinline__ void sf_store_dense(const float2 *s_f, uint32_t nodes, uint32_t cell, uint32_t node0,
                                            uint32_t ncell, bool add, bool last, float2 *__restrict__ S,
                                            float2 *__restrict__ lo_buf) {
  for (uint32_t m = threadIdx.x; m < nodes; m += kSfThreads) {
    const size_t o = sr_index(cell, node0 + m, ncell);
    const float2 f = s_f[m];
    double vx = f.x, vy = f.y;
    if (add) {
      const float2 h = S[o], l = lo_buf[o];
      vx += (double)h.x + (double)l.x;
      vy += (double)h.y + (double)l.y;
    }
    const float hx = static_cast<float>(vx), hy = static_cast<float>(vy);
    S[o] = make_float2(hx, hy);
    if (!last) lo_buf[o] = make_float2(static_cast<float>(vx - hx), static_cast<float>(vy - hy));
  }
}

template <int NPT>
__device__ __forceinline__ void sf_unit(const SfUnit &u, const float4 *__restrict__ pk,
                                        const uint32_t *__restrict__ cell_count,
                                        const uint32_t *__restrict__ cell_point, const Grid &g,
                                        const float4 *__restrict__ dirs, const float *__restrict__ kappa,
                                        uint32_t c0, uint32_t c1, uint32_t node_off, float2 *__restrict__ S,
                                        float2 *__restrict__ lo_buf, float4 *s_at, float2 *s_f) {
  // Slots are handled in pairs (FMUL2/FFMA2); an odd last slot alone.
  constexpr int NP2 = NPT / 2;
  constexpr bool ODD = (NPT & 1) != 0;
  constexpr int POLY2 = sf_poly_pairs(NPT);  // pairs on the FMA pipe (the last ones)
  const uint32_t d = threadIdx.x / u.nb;
  const uint32_t b = threadIdx.x - d * u.nb;
  const bool act = d < u.n_dir;
  const uint32_t r0 = b * NPT;
  float sx = 0.f, sy = 0.f, sz = 0.f;
  if (act) {
    const float4 sd = dirs[u.dir_begin + d];
    sx = sd.x; sy = sd.y; sz = sd.z;
  }
  float kap[NPT];
#pragma unroll
  for (int i = 0; i < NPT; i++) kap[i] = (act && r0 + i < u.n_rad) ? kappa[u.kappa_begin + r0 + i] : 0.f;
  float2 kap2[NP2 > 0 ? NP2 : 1];
#pragma unroll
  for (int k = 0; k < NP2; k++) kap2[k] = make_float2(kap[2 * k], kap[2 * k + 1]);
  const float kap_odd = kap[NPT - 1];
  const uint32_t nodes = u.n_dir * u.n_rad;
  for (uint32_t cell = c0; cell < c1; cell++) {
    const uint32_t cnt = cell_count[cell];
    const uint32_t start = cell_point[cell];
    uint32_t a0 = 0;
    do {
      const uint32_t na = min((uint32_t)kSfAtomTile, cnt - a0);
      __syncthreads();
      // (the atoms read from the staged tile, one broadcast shared load per
      // atom per thread; broadcast global loads instead measured slower,
      // water10k 1.133 against 1.088 ms, bitwise-equal)
      if (threadIdx.x < na) s_at[threadIdx.x] = pk[start + a0 + threadIdx.x];
      __syncthreads();
      // FR = sum q cos, FI = sum q sin (the sign of S's imaginary part is
      // applied when the sums are stored)
      float2 FR[NP2 > 0 ? NP2 : 1], FI[NP2 > 0 ? NP2 : 1];
#pragma unroll
      for (int k = 0; k < NP2; k++) { FR[k] = make_float2(0.f, 0.f); FI[k] = make_float2(0.f, 0.f); }
      float fr_odd = 0.f, fi_odd = 0.f;
#pragma unroll 1
      for (uint32_t j = 0; j < na; j++) {
        const float4 p = s_at[j];
        const float uu = fmaf(sx, p.x, fmaf(sy, p.y, sz * p.z));
        const float2 uu2 = bcast(uu);
        const float2 q2 = bcast(p.w);
#pragma unroll
        for (int k = 0; k < NP2 - POLY2; k++) {
          const float2 th = __fmul2_rn(kap2[k], uu2);
          float sa, ca, sb, cb;
          sfu_sincos(th.x, &sa, &ca);
          sfu_sincos(th.y, &sb, &cb);
          FR[k] = __ffma2_rn(q2, make_float2(ca, cb), FR[k]);
          FI[k] = __ffma2_rn(q2, make_float2(sa, sb), FI[k]);
        }
#pragma unroll
        for (int k = NP2 - POLY2; k < NP2; k++) {
          float2 sn, cs, qs;
          fma_sincos_signed2(__fmul2_rn(kap2[k], uu2), p.w, &sn, &cs, &qs);
          FR[k] = __ffma2_rn(qs, cs, FR[k]);
          FI[k] = __ffma2_rn(qs, sn, FI[k]);
        }
        if (ODD) {
          float sn, cs;
          sfu_sincos(kap_odd * uu, &sn, &cs);
          fr_odd = fmaf(p.w, cs, fr_odd);
          fi_odd = fmaf(p.w, sn, fi_odd);
        }
      }
      // Tile sums to shared memory in the unit's node order, then one thread
      // per node (coalesced) stores them.  S holds the cell-relative sums in
      // FP32 (an FP32 tile sum; FP64 storage held no more information and
      // doubled the bytes written here and read by the shell sums); the
      // shell-sum kernel applies the twiddle e^{-ik.c} in FP64 from its
      // per-axis tables as it loads S.
      if (act) {
#pragma unroll
        for (int k = 0; k < NP2; k++) {
          if (r0 + 2 * k < u.n_rad) s_f[d * u.n_rad + r0 + 2 * k] = make_float2(FR[k].x, -FI[k].x);
          if (r0 + 2 * k + 1 < u.n_rad) s_f[d * u.n_rad + r0 + 2 * k + 1] = make_float2(FR[k].y, -FI[k].y);
        }
        if (ODD && r0 + NPT - 1 < u.n_rad) s_f[d * u.n_rad + r0 + NPT - 1] = make_float2(fr_odd, -fi_odd);
      }
      __syncthreads();
      if (cnt <= kSfAtomTile) {
        for (uint32_t m = threadIdx.x; m < nodes; m += kSfThreads)
          S[sr_index(cell, u.node_begin + m - node_off, g.ncell)] = s_f[m];
      } else {
        sf_store_dense(s_f, nodes, cell, u.node_begin - node_off, g.ncell, a0 > 0, a0 + kSfAtomTile >= cnt, S,
                       lo_buf);
      }
      a0 += kSfAtomTile;
    } while (a0 < cnt);
  }
}

// Units index nodes by the handle's local node; S holds the nodes from
// node_off on (a node range of the handle: the whole of it, or one stage).
// Cells: kSfCellsPerCta per CTA row from cell_base on (grids of more than
// 65,535 rows take several launches).  lo_buf: scratch of S's size.
__device__ __forceinline__ void sf_block(const float4 *__restrict__ pk, const uint32_t *__restrict__ cell_count,
                                         const uint32_t *__restrict__ cell_point, const Grid &g,
                                         const SfUnit *__restrict__ units, const float4 *__restrict__ dirs,
                                         const float *__restrict__ kappa, uint32_t node_off, uint32_t cell_base,
                                         float2 *__restrict__ S, float2 *__restrict__ lo_buf, uint32_t bx,
                                         uint32_t by) {
  __shared__ float4 s_at[kSfAtomTile];
  __shared__ float2 s_f[kSfThreads * kSfMaxNpt];
  const SfUnit u = units[bx];
  const uint32_t c0 = cell_base + by * kSfCellsPerCta;
  const uint32_t c1 = min(g.ncell, c0 + kSfCellsPerCta);
#define GLST_SF_CASE(n) \
  case n: sf_unit<n>(u, pk, cell_count, cell_point, g, dirs, kappa, c0, c1, node_off, S, lo_buf, s_at, s_f); break;
  switch (u.npt) {
    GLST_SF_CASE(1) GLST_SF_CASE(2) GLST_SF_CASE(3) GLST_SF_CASE(4) GLST_SF_CASE(5) GLST_SF_CASE(6)
    GLST_SF_CASE(7) GLST_SF_CASE(8) GLST_SF_CASE(9) GLST_SF_CASE(10) GLST_SF_CASE(11) GLST_SF_CASE(12)
    default: break;
  }
#undef GLST_SF_CASE
}

__global__ void __launch_bounds__(kSfThreads, 8)
k_structure_factors(const float4 *__restrict__ pk, const uint32_t *__restrict__ cell_count,
                    const uint32_t *__restrict__ cell_point, Grid g, const SfUnit *__restrict__ units,
                    const float4 *__restrict__ dirs, const float *__restrict__ kappa, uint32_t node_off,
                    uint32_t cell_base, float2 *__restrict__ S, float2 *__restrict__ lo_buf) {
  sf_block(pk, cell_count, cell_point, g, units, dirs, kappa, node_off, cell_base, S, lo_buf, blockIdx.x,
           blockIdx.y);
}

// ----------------------------------------------------------------------------
// Shell sums (src/glst_force.cu:702-913 restated for shared memory): per
// node, an inclusive 3-D prefix sum of S over the cell grid (z, y, x), then
// R_c = w * [box(c, r_out) - box(c, r_in)], 8 corners per box, clipped to the
// grid.  All FP64.  Output R'_c(k) = R_c(k) e^{+ik.c} as float2, the twiddle
// built from per-axis tables e^{i kx cx} e^{i ky cy} e^{i kz cz}.
// CTA: nb nodes at once (rows of ncell+1 complex doubles in shared memory).
// (A form with a zero plane in front of each axis, so that corner offsets
// need no clipping tests, measured slower on water10k: 0.50 ms loading all
// eight corners of every box, 0.45 ms skipping the zero-plane corners,
// against 0.42 ms here -- the larger rows and their zeroing cost more than
// the index arithmetic saved.  Per-node tables of per-axis corner offsets,
// three shared loads per cell in place of the clipping arithmetic, measured
// slower too: 0.412 against 0.381 ms, a dependent shared load more per cell
// in a latency-bound loop.)
// Launch shapes: 512 threads, 3 CTAs per SM; 256 threads, 4 CTAs per SM
// where four CTAs' tables fit in shared memory (water10k, 8 nodes per CTA:
// 0.382 against 0.416 ms -- fewer threads per node give each thread more
// cells over which to spread its set-up, and four CTAs overlap their
// barrier-separated phases better; 4 nodes per CTA at any shape measured
// 0.55-0.66 ms); one node per CTA, 512 threads, on large grids (22^3 grid:
// 0.393 ms per 1,534 nodes against 0.399 with 1024 and 0.396 with 768
// threads; there the node's S loads and R stores, 8 bytes at a 256-byte
// stride in the node-block layout, take 25 % and 20 % of the time, the
// corners 19 %, the prefix passes 9 %).
constexpr int kSatThreads = 512;
constexpr int kSatThreadsSmall = 256;
constexpr int kSatThreadsOne = 512;  // one node per CTA (large grids)
// S loads in flight per thread: 8 (a 7-cell line in one batch on water10k),
// 4 in the 512-thread several-nodes form, whose register budget is 40 (8
// spilled there)
template <int kMinBlocks>
struct SatLoadBatch {
  static constexpr int value = kMinBlocks == 3 ? 4 : 8;
};

struct SatArgs {
  const float2 *S;               // cell-relative structure factors
  const double4 *node64;        // (kx, ky, kz, w) FP64
  const uint32_t *node_radii;   // r_in | r_out << 16
  uint32_t K;                   // nodes handled by this launch
  uint32_t kbase;               // local index of the launch's first node in S and R
  uint32_t nb;                  // nodes per CTA (a power of two, <= 32)
  uint32_t lg_nb;               // log2(nb)
  uint32_t xyz_table;           // 1: cell coordinates tabulated in shared memory
  uint32_t stride;              // shared row stride (complex), >= ncell, = 1 (mod 8)
  float2 *R;
};

__device__ __forceinline__ double2 sat_at(const double2 *row, uint32_t x, uint32_t y,
                                          uint32_t z, const Grid &g) {
  return row[(x * g.ny + y) * g.nz + z];
}

__device__ __forceinline__ double2 cube_sum(const double2 *row, uint32_t x, uint32_t y,
                                            uint32_t z, uint32_t r, const Grid &g) {
  const uint32_t x0 = (x < r) ? 0 : x - r, y0 = (y < r) ? 0 : y - r, z0 = (z < r) ? 0 : z - r;
  const uint32_t x1 = min(x + r, g.nx - 1), y1 = min(y + r, g.ny - 1), z1 = min(z + r, g.nz - 1);
  const bool xb = x0 == 0, yb = y0 == 0, zb = z0 == 0;
  const uint32_t xm = xb ? 0 : x0 - 1, ym = yb ? 0 : y0 - 1, zm = zb ? 0 : z0 - 1;
  double2 s = sat_at(row, x1, y1, z1, g);
  double2 t;
  if (!xb) { t = sat_at(row, xm, y1, z1, g); s.x -= t.x; s.y -= t.y; }
  if (!yb) { t = sat_at(row, x1, ym, z1, g); s.x -= t.x; s.y -= t.y; }
  if (!zb) { t = sat_at(row, x1, y1, zm, g); s.x -= t.x; s.y -= t.y; }
  if (!xb && !yb) { t = sat_at(row, xm, ym, z1, g); s.x += t.x; s.y += t.y; }
  if (!xb && !zb) { t = sat_at(row, xm, y1, zm, g); s.x += t.x; s.y += t.y; }
  if (!yb && !zb) { t = sat_at(row, x1, ym, zm, g); s.x += t.x; s.y += t.y; }
  if (!xb && !yb && !zb) { t = sat_at(row, xm, ym, zm, g); s.x -= t.x; s.y -= t.y; }
  return s;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Dynamic shared memory: nb rows of `stride` complex (the SAT), the twiddle
// tables nb x (nx + ny + nz) complex, then, in the several-nodes form
// (kMinBlocks > 1, small grids) when it fits, the cell coordinates (ncell x
// u32, x | y << 10 | z << 20).  nb is a power of two <= 32: lane l of a warp works
// on node l % nb of the CTA and on the (l / nb)-th of the 32 / nb cells or
// lines the warp takes per step, so the per-node values (radii, weight,
// twiddle rows) stay in registers and the S loads and R stores of a warp are
// runs of consecutive nodes.
template <int kMinBlocks>
__device__ __forceinline__ void shell_block(const Grid &g, const SatArgs &a, uint32_t bx) {
  extern __shared__ double2 s_sat[];
  const uint32_t nb = a.nb, lg = a.lg_nb;
  const uint32_t k0 = bx * nb;
  const uint32_t C = g.ncell;
  const uint32_t naxis = g.nx + g.ny + g.nz;
  double2 *s_tw = s_sat + (size_t)nb * a.stride;
  uint32_t *s_xyz = reinterpret_cast<uint32_t *>(s_tw + (size_t)nb * naxis);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t j = lane & (nb - 1u);
  const uint32_t per_warp = 32u >> lg;
  const uint32_t first = warp * per_warp + (lane >> lg);
  const uint32_t step = (blockDim.x >> 5) * per_warp;
  const uint32_t k = k0 + j;         // node within the launch (node tables)
  const uint32_t ks = a.kbase + k;   // node within S and R
  const bool jv = k < a.K;
  // The S loads run as a flat sequence of batches (line l, z from z0) of
  // kLoadBatch cells each; the first is issued before the twiddle tables,
  // whose node loads and FP64 sincos it overlaps (water10k shell sums 0.441
  // vs 0.450 ms; one batch in flight ahead of the one summed, 0.462 ms at a
  // batch of 2 and spilling at 4).
  constexpr int kLoadBatch = SatLoadBatch<kMinBlocks>::value;
  const uint32_t nlines = g.nx * g.ny;
  const double2 zero = make_double2(0.0, 0.0);
  auto fetch = [&](float2 *dst, uint32_t line, uint32_t zb) {
#pragma unroll
    for (int u = 0; u < kLoadBatch; u++)
      dst[u] = (jv && line < nlines && zb + u < g.nz) ? __ldg(a.S + sr_index(line * g.nz + zb + u, ks, C))
                                                      : make_float2(0.f, 0.f);
  };
  float2 v[kLoadBatch];
  uint32_t l = first, z0 = 0;
  fetch(v, l, z0);
  // twiddle tables: e^{i k_a (i + 1/2) l} per node and axis
  for (uint32_t t = threadIdx.x; t < nb * naxis; t += blockDim.x) {
    const uint32_t jj = t / naxis, r = t - jj * naxis;
    const double4 nk = (k0 + jj < a.K) ? a.node64[k0 + jj] : make_double4(0.0, 0.0, 0.0, 0.0);
    double kc;
    if (r < g.nx) kc = nk.x * cell_centre(r, g.l);
    else if (r < g.nx + g.ny) kc = nk.y * cell_centre(r - g.nx, g.l);
    else kc = nk.z * cell_centre(r - g.nx - g.ny, g.l);
    double sn, cs;
    sincos(kc, &sn, &cs);
    s_tw[t] = make_double2(cs, sn);
  }
  auto coords = [&](uint32_t c) {
    const uint32_t x = c / (g.ny * g.nz), rem = c - x * (g.ny * g.nz);
    const uint32_t y = rem / g.nz, z = rem - y * g.nz;
    return x | (y << 10) | (z << 20);
  };
  if (kMinBlocks > 1 && a.xyz_table)
    for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) s_xyz[c] = coords(c);
  double2 *row = s_sat + (size_t)j * a.stride;
  const double2 *twx = s_tw + (size_t)j * naxis, *twy = twx + g.nx, *twz = twy + g.ny;
  __syncthreads();  // twiddle tables
  // S[c][k0 + j] -> row j: the cell-relative structure factors times
  // e^{-ik.c} (the per-axis tables), summed along z on the way in (the z
  // prefix pass without its own shared-memory round trip)
  {
    double2 acc = zero, txy = zero;
    while (l < nlines) {
      uint32_t ln = l, zn = z0 + kLoadBatch;
      if (zn >= g.nz) { ln = l + step; zn = 0; }
      if (z0 == 0) {
        const uint32_t lx = l / g.ny;
        txy = cmul(twx[lx], twy[l - lx * g.ny]);  // e^{+i(kx cx + ky cy)}
        acc = zero;
      }
      const uint32_t base = l * g.nz;
#pragma unroll
      for (int u = 0; u < kLoadBatch; u++) {
        if (z0 + u < g.nz) {
          const double2 t = cmul(txy, twz[z0 + u]);  // e^{+ik.c}
          const double vx = v[u].x, vy = v[u].y;
          acc.x += vx * t.x + vy * t.y;  // v * conj(t)
          acc.y += vy * t.x - vx * t.y;
          row[base + z0 + u] = acc;
        }
      }
      fetch(v, ln, zn);
      l = ln;
      z0 = zn;
    }
  }
  __syncthreads();
  // prefix along y (lines x, z)
  for (uint32_t l = first; l < g.nx * g.nz; l += step) {
    const uint32_t x = l / g.nz, z = l - x * g.nz;
    double2 *p = row + x * g.ny * g.nz + z;
    double2 acc = make_double2(0.0, 0.0);
    for (uint32_t y = 0; y < g.ny; y++) { acc.x += p[y * g.nz].x; acc.y += p[y * g.nz].y; p[y * g.nz] = acc; }
  }
  __syncthreads();
  // prefix along x (lines y, z)
  {
    const uint32_t sx = g.ny * g.nz;
    for (uint32_t l = first; l < sx; l += step) {
      double2 *p = row + l;
      double2 acc = make_double2(0.0, 0.0);
      for (uint32_t x = 0; x < g.nx; x++) { acc.x += p[x * sx].x; acc.y += p[x * sx].y; p[x * sx] = acc; }
    }
  }
  __syncthreads();
  if (!jv) return;
  // shell sums, weight and twiddle
  const uint32_t radii = a.node_radii[k];
  const uint32_t r_out = radii >> 16, r_in = radii & 0xffffu;
  const double w = a.node64[k].w;
  // The thread's cells c = first + i * step.  Small grids (several nodes per
  // CTA) look their coordinates up in the CTA's table.  Large grids (one node
  // per CTA) step them with carries: there the table cost every CTA two
  // divisions per cell of the grid (water333k shell sums 34.8 ms with it,
  // 27.9 ms stepping); on small grids stepping measured slower (water10k
  // 0.43 against 0.42 ms).
  if constexpr (kMinBlocks > 1) {
    for (uint32_t c = first; c < C; c += step) {
      const uint32_t xyz = a.xyz_table ? s_xyz[c] : coords(c);
      const uint32_t x = xyz & 1023u, y = (xyz >> 10) & 1023u, z = xyz >> 20;
      const double2 o = cube_sum(row, x, y, z, r_out, g);
      const double2 i = cube_sum(row, x, y, z, r_in, g);
      const double2 sh = make_double2((o.x - i.x) * w, (o.y - i.y) * w);
      const double2 r = cmul(cmul(sh, twx[x]), cmul(twy[y], twz[z]));
      a.R[sr_index(c, ks, C)] = make_float2(static_cast<float>(r.x), static_cast<float>(r.y));
    }
  } else {
    const uint32_t syz = g.ny * g.nz;
    const uint32_t sx = step / syz, sy = (step - sx * syz) / g.nz, sz = step - sx * syz - sy * g.nz;
    uint32_t x = first / syz, y = (first - x * syz) / g.nz, z = first - x * syz - y * g.nz;
    for (uint32_t c = first; c < C; c += step) {
      const double2 o = cube_sum(row, x, y, z, r_out, g);
      const double2 i = cube_sum(row, x, y, z, r_in, g);
      const double2 sh = make_double2((o.x - i.x) * w, (o.y - i.y) * w);
      const double2 r = cmul(cmul(sh, twx[x]), cmul(twy[y], twz[z]));
      a.R[sr_index(c, ks, C)] = make_float2(static_cast<float>(r.x), static_cast<float>(r.y));
      z += sz;  // sz < nz and sy < ny: one carry at most per axis
      if (z >= g.nz) { z -= g.nz; y++; }
      y += sy;
      if (y >= g.ny) { y -= g.ny; x++; }
      x += sx;
    }
  }
}

template <int kThreads, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
k_shell_sums(Grid g, SatArgs a) {
  shell_block<kMinBlocks>(g, a, blockIdx.x);
}

// ----------------------------------------------------------------------------
// Shell sums for grids whose per-node prefix table does not fit in shared
// memory (the same arithmetic as k_shell_sums, src/glst_force.cu:702-913):
// the FP64 summed-area tables of a batch of node blocks live in global memory
// (laid out like S: per block of kNodeBlock nodes, cell-major, node fastest,
// so every warp access is a contiguous run of 32 nodes), built by three
// line passes (z with the twiddle e^{-ik.c} applied on load, then y, then x)
// and read by a fourth pass that forms the 16-corner shell differences.  The
// per-axis twiddles of the stage's nodes are tabulated once per stage.
struct GsatArgs {
  const float2 *S;              // stage-local structure factors
  const double4 *node64;        // node table of the stage (kx, ky, kz, w)
  const uint32_t *node_radii;   // r_in | r_out << 16, same indexing
  const double2 *tw;            // twiddles e^{+i k_a c_a}: tw[a * K + k], a = 0 .. nx + ny + nz - 1
  double2 *T;                   // tables of the batch: nblk x C x kNodeBlock
  float2 *R;                    // stage-local shell sums
  uint32_t K;                   // nodes of the stage
  uint32_t blk0;                // first node block of the batch (stage-local)
  uint32_t nblk;                // node blocks in the batch
};

// Twiddle table: tw[a * K + k] = e^{+i k_axis (i + 1/2) l} for the a-th of
// the nx + ny + nz per-axis cell indices (node fastest, so the warps of the
// passes, 32 consecutive nodes each, read contiguous runs).
__global__ void k_gsat_twiddles(Grid g, const double4 *__restrict__ node64, uint32_t K,
                                double2 *__restrict__ tw) {
  const uint32_t naxis = g.nx + g.ny + g.nz;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)K * naxis) return;
  const uint32_t r = (uint32_t)(t / K), k = (uint32_t)(t - (size_t)r * K);
  const double4 nk = node64[k];
  double kc;
  if (r < g.nx) kc = nk.x * cell_centre(r, g.l);
  else if (r < g.nx + g.ny) kc = nk.y * cell_centre(r - g.nx, g.l);
  else kc = nk.z * cell_centre(r - g.nx - g.ny, g.l);
  double sn, cs;
  sincos(kc, &sn, &cs);
  tw[t] = make_double2(cs, sn);
}

__device__ __forceinline__ size_t gsat_at(uint32_t bb, uint32_t c, uint32_t j, uint32_t C) {
  return ((size_t)bb * C + c) * kNodeBlock + j;
}

// Pass 1: thread = (line (x, y), block, node j); S x e^{-ik.c}, prefix along z.
__global__ void k_gsat_z(Grid g, GsatArgs a) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t j = (uint32_t)(t % kNodeBlock);
  const size_t lb = t / kNodeBlock;
  const uint32_t bb = (uint32_t)(lb % a.nblk);
  const size_t line = lb / a.nblk;
  if (line >= (size_t)g.nx * g.ny) return;
  const uint32_t blk = a.blk0 + bb;
  const uint32_t k = blk * kNodeBlock + j;  // stage-local node
  const uint32_t C = g.ncell;
  const uint32_t x = (uint32_t)(line / g.ny), y = (uint32_t)(line - (size_t)x * g.ny);
  const uint32_t c0 = (uint32_t)line * g.nz;
  double2 *T = a.T;
  if (k >= a.K) {
    for (uint32_t z = 0; z < g.nz; z++) T[gsat_at(bb, c0 + z, j, C)] = make_double2(0.0, 0.0);
    return;
  }
  const size_t K = a.K;
  const double2 *tk = a.tw + k;  // entry of axis index i: tk[i * K]
  const double2 txy = cmul(tk[(size_t)x * K], tk[(size_t)(g.nx + y) * K]);
  const double2 *twz = tk + (size_t)(g.nx + g.ny) * K;
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll 4
  for (uint32_t z = 0; z < g.nz; z++) {
    const float2 v = a.S[sr_index(c0 + z, k, C)];
    const double2 tt = cmul(txy, twz[(size_t)z * K]);
    const double vx = v.x, vy = v.y;
    acc.x += vx * tt.x + vy * tt.y;  // v * conj(tt)
    acc.y += vy * tt.x - vx * tt.y;
    T[gsat_at(bb, c0 + z, j, C)] = acc;
  }
}

// Passes 2 and 3: prefix along y (axis 1) or x (axis 0), in place.
__global__ void k_gsat_prefix(Grid g, GsatArgs a, int axis) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t j = (uint32_t)(t % kNodeBlock);
  const size_t lb = t / kNodeBlock;
  const uint32_t bb = (uint32_t)(lb % a.nblk);
  const size_t line = lb / a.nblk;
  const uint32_t C = g.ncell;
  uint32_t n, c0, stride;
  if (axis == 1) {  // lines (x, z)
    if (line >= (size_t)g.nx * g.nz) return;
    const uint32_t x = (uint32_t)(line / g.nz), z = (uint32_t)(line - (size_t)x * g.nz);
    n = g.ny; c0 = x * g.ny * g.nz + z; stride = g.nz;
  } else {  // lines (y, z)
    if (line >= (size_t)g.ny * g.nz) return;
    n = g.nx; c0 = (uint32_t)line; stride = g.ny * g.nz;
  }
  double2 *T = a.T;
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll 4
  for (uint32_t i = 0; i < n; i++) {
    double2 *p = T + gsat_at(bb, c0 + i * stride, j, C);
    const double2 v = *p;
    acc.x += v.x;
    acc.y += v.y;
    *p = acc;
  }
}

__device__ __forceinline__ double2 gcube_sum(const double2 *T, uint32_t bb, uint32_t j, uint32_t x, uint32_t y,
                                             uint32_t z, uint32_t r, const Grid &g) {
  const uint32_t C = g.ncell;
  const uint32_t x0 = (x < r) ? 0 : x - r, y0 = (y < r) ? 0 : y - r, z0 = (z < r) ? 0 : z - r;
  const uint32_t x1 = min(x + r, g.nx - 1), y1 = min(y + r, g.ny - 1), z1 = min(z + r, g.nz - 1);
  const bool xb = x0 == 0, yb = y0 == 0, zb = z0 == 0;
  const uint32_t xm = xb ? 0 : x0 - 1, ym = yb ? 0 : y0 - 1, zm = zb ? 0 : z0 - 1;
  auto at = [&](uint32_t a, uint32_t b, uint32_t c) { return T[gsat_at(bb, (a * g.ny + b) * g.nz + c, j, C)]; };
  double2 s = at(x1, y1, z1);
  double2 t;
  if (!xb) { t = at(xm, y1, z1); s.x -= t.x; s.y -= t.y; }
  if (!yb) { t = at(x1, ym, z1); s.x -= t.x; s.y -= t.y; }
  if (!zb) { t = at(x1, y1, zm); s.x -= t.x; s.y -= t.y; }
  if (!xb && !yb) { t = at(xm, ym, z1); s.x += t.x; s.y += t.y; }
  if (!xb && !zb) { t = at(xm, y1, zm); s.x += t.x; s.y += t.y; }
  if (!yb && !zb) { t = at(x1, ym, zm); s.x += t.x; s.y += t.y; }
  if (!xb && !yb && !zb) { t = at(xm, ym, zm); s.x -= t.x; s.y -= t.y; }
  return s;
}

// Pass 4: thread = (cell, block, node j): shell difference x w x e^{+ik.c}.
__global__ void k_gsat_shell(Grid g, GsatArgs a) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t j = (uint32_t)(t % kNodeBlock);
  const size_t cb = t / kNodeBlock;
  const uint32_t bb = (uint32_t)(cb % a.nblk);
  const size_t c = cb / a.nblk;
  if (c >= g.ncell) return;
  const uint32_t k = (a.blk0 + bb) * kNodeBlock + j;
  if (k >= a.K) return;
  const uint32_t syz = g.ny * g.nz;
  const uint32_t x = (uint32_t)(c / syz), rem = (uint32_t)(c - (size_t)x * syz);
  const uint32_t y = rem / g.nz, z = rem - y * g.nz;
  const uint32_t radii = a.node_radii[k];
  const uint32_t r_out = radii >> 16, r_in = radii & 0xffffu;
  const double w = a.node64[k].w;
  const double2 o = gcube_sum(a.T, bb, j, x, y, z, r_out, g);
  const double2 i = gcube_sum(a.T, bb, j, x, y, z, r_in, g);
  const double2 sh = make_double2((o.x - i.x) * w, (o.y - i.y) * w);
  const size_t K = a.K;
  const double2 *tk = a.tw + k;
  const double2 r = cmul(cmul(sh, tk[(size_t)x * K]), cmul(tk[(size_t)(g.nx + y) * K], tk[(size_t)(g.nx + g.ny + z) * K]));
  a.R[sr_index((uint32_t)c, k, g.ncell)] = make_float2(static_cast<float>(r.x), static_cast<float>(r.y));
}

// ----------------------------------------------------------------------------
// Long-range gather (src/glst_force.cu:983-1135 restated):
//   en_i = q_i Re sum_k e^{ik.d_i} R'_c(k),   f_i = q_i sum_k Im(...) k
// Nodes are held in the order group -> direction -> radial, k = kappa_r s_j,
// so per atom and direction u = s_j . d_i is formed once and each node costs
// one multiply, one SFU sin/cos pair and four FMAs:
//   e += c R'x - s R'y,   g += kappa_r (c R'y + s R'x),   f += g s_j.
// FP32 inside a tile, FP64 across tiles.
constexpr int kLrThreads = 128;

struct LrChunk {
  uint32_t node_begin;   // internal index of (first direction, r = 0)
  uint32_t dir_begin;    // global direction index of the first direction
  uint32_t n_dir;        // directions in the chunk
  uint32_t n_rad;        // radial nodes per direction in this group
  uint32_t kappa_begin;  // offset of this group's radial table
  uint32_t pad[3];
};

// A CTA takes 128 consecutive cell-ordered atoms whatever their cells (so
// every warp is full -- one CTA per cell left ~10-15 % of the lanes of last
// warps idle, measured 2.06 vs 1.63 ms on water10k), and stages the R' tiles
// of the up to kLrfCells cells those atoms belong to; lanes read their own
// cell's tile.  Atoms of sparser ranges (more cells) are handled in several
// passes over windows of kLrfCells cells.
//
// Radial nodes go in pairs (r, r+1) -- a direction with an odd count gets a
// zero node -- stored as float4 (R'x_r, R'x_r+1, R'y_r, R'y_r+1) so that the
// paired FP32 instructions (FMUL2/FFMA2) do two nodes at once:
//   EA += c R'x,  EB += s R'y,  G += kappa (c R'y + s R'x),   e = EA - EB.
// One pair in kLrPolyStride takes its sine and cosine from the FMA-pipe
// polynomial, interleaved with the SFU pairs of its group (the FMA pipe
// already carries ~7 FP32 operations per node, so only a small share pays):
// water10k 1.57 ms with none, 1.51 ms with 1 in 7, 1.53 with 1 in 5, 1.66
// with 1 in 3; a separate polynomial loop after the SFU loop (20-40 %)
// measured 1.63-1.87 ms.  The radial scales load as float4 quads (two
// pairs), so groups are even: 14 pairs with 2 on the polynomial, 1.462 ms
// against 1.482 ms with one scale load per pair (groups of 6 / 8 / 12 / 16
// pairs with 1 / 1 / 2 / 2 on the polynomial: 1.503 / 1.483 / 1.476 / 1.498).
// The cell slots of a tile are kLrfSlotPad float4 apart beyond the tile so
// that the up to four addresses a warp reads fall in different shared-memory
// banks (32.9 M bank conflicts per launch without the pad, 0.25 M with).
// Two adjacent atoms per thread (256 atoms per CTA, one R' load serving both
// when they share a cell: 0.75 shared loads per (atom, node pair) instead of
// 1.5) gave bitwise-equal results but ran 14 % slower (water10k 1.67 vs
// 1.465 ms; 96 registers, 5 CTAs per SM): the MUFU latency the 32 resident
// warps hide outweighs the MIO-queue relief.  Staging the tiles with
// asynchronous copies (cp.async, no prefetch registers: 64 registers without
// spills) was bitwise-equal and slower too: 1.570 ms at 8 CTAs per SM, 1.584
// at 9, 1.599 at 10 -- the copies add to the MIO queue, and more resident
// warps do not help a gather bound by that queue.  Reading each lane's R'
// pair straight from global memory (two L1-cached loads per node pair, no
// staging, barriers or window passes) was bitwise-equal and far slower:
// 2.75 against 1.44 ms.
constexpr int kLrfCells = 4;           // cells staged per pass
constexpr int kLrfTilePairs = 128;     // node pairs per cell tile
constexpr int kLrfTileNodes = 2 * kLrfTilePairs;
constexpr int kLrfSlotPad = 2;
constexpr int kLrfSlot = kLrfTilePairs + kLrfSlotPad;
constexpr int kLrfPerThread = (kLrfCells * kLrfTilePairs) / kLrThreads;
constexpr int kLrGroup = 14;      // node pairs per group (even: radial scales load as quads)
static_assert(kLrGroup % 2 == 0, "groups are whole radial-scale quads");
// Which pairs of a group take the FMA-pipe polynomial: bit q of the mask.
// The variants are compiled in and chosen per plan by the autotuner
// (glst_autotune); variant 0, three pairs in fourteen at 1, 5, 10, is the
// default.  With the radial scales in the parameter space (a lighter MIO
// queue) three pairs beat two: water10k 1.397 ms at {1, 5, 10}, 1.406 at
// {0, 5, 10}, against 1.436 at {6, 13} (the earlier default); {2, 7, 12}
// 1.407, {4, 9, 13} 1.410, {0, 4, 9} 1.409, {1, 6, 11} 1.419, {0, 7} 1.420,
// four pairs {2, 6, 10, 13} 1.429, {0, 4, 8, 12} 1.428.
constexpr uint32_t kLrPolyMasks[4] = {(1u << 1) | (1u << 5) | (1u << 10), 0u, (1u << 6) | (1u << 13),
                                      (1u << 1) | (1u << 5) | (1u << 9) | (1u << 13)};
constexpr int kLrVariants = 4;

__device__ __forceinline__ uint32_t cell_of_atom(const uint32_t *__restrict__ cell_point, uint32_t ncell,
                                                 uint32_t p) {
  // last cell whose first atom is <= p (cells may be empty: the last such)
  uint32_t lo = 0, hi = ncell - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (cell_point[mid] <= p) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// The radial scales of every group as quads (kappa_4t .. kappa_4t+3 of a
// group, 0 beyond its last), passed in the gather's parameter space; a
// chunk's quads start at quad_begin.
constexpr int kLrKappaQuads = 128;
struct LrKappaQuads {
  float4 q[kLrKappaQuads];
};

template <uint32_t kPolyMask, bool kParamKappa>
__device__ __forceinline__ void lr_block(const float4 *__restrict__ pk, const uint32_t *__restrict__ cell_point,
                                         uint32_t ncell, const LrChunk *__restrict__ chunks,
                                         const float4 *__restrict__ dirs, const float *__restrict__ kappa,
                                         const float2 *__restrict__ R, uint32_t node_off, uint32_t natom,
                                         int accumulate, double4 *__restrict__ part, uint32_t bx, uint32_t by,
                                         const LrKappaQuads *kpq = nullptr) {
  __shared__ float4 s_n[2][kLrfCells * kLrfSlot];
  __shared__ float4 s_kappa4[kParamKappa ? 1 : kLrfTilePairs / 2];
  __shared__ uint32_t s_cells[kLrThreads];  // each thread's cell, then the distinct cells in order
  __shared__ uint32_t s_heads[kLrThreads / 32];
  const uint32_t a0 = bx * kLrThreads;
  const uint32_t p = a0 + threadIdx.x;
  const bool active = p < natom;
  const LrChunk ch = chunks[by];
  const uint32_t nr = ch.n_rad;
  const uint32_t npr = (nr + 1) >> 1;                                   // pairs per direction
  const uint32_t dirs_per_tile = max(1u, (uint32_t)kLrfTilePairs / npr);  // npr <= kLrfTilePairs (host check)
  const uint32_t ntiles = (ch.n_dir + dirs_per_tile - 1) / dirs_per_tile;
  // radial scales of pairs (2t, 2t+1): kappa_{4t .. 4t+3}, 0 beyond the last
  if constexpr (!kParamKappa) {
    for (uint32_t t = threadIdx.x; 2 * t < npr; t += kLrThreads) {
      float kq[4];
#pragma unroll
      for (int i = 0; i < 4; i++) kq[i] = 4 * t + i < nr ? kappa[ch.kappa_begin + 4 * t + i] : 0.f;
      s_kappa4[t] = make_float4(kq[0], kq[1], kq[2], kq[3]);
    }
  }
  const float4 *kq4 = kParamKappa ? kpq->q + ch.pad[0] : s_kappa4;
  // The distinct cells of the CTA's atoms, in order, and each atom's rank
  // among them: windows of kLrfCells occupied cells.  (Windows of
  // consecutive cell indices made blocks that span empty and sparse cells --
  // the reference's grid of rcut-edged cells leaves the outer layer nearly
  // empty when the box is a little over a multiple of rcut -- take up to six
  // passes over every node tile with most warps idle: 13,500 atoms on 6^3
  // cells, 14 of them empty, 0.834 ms against 0.853 ms for 18,000 atoms.)
  const uint32_t my_cell = active ? cell_of_atom(cell_point, ncell, p) : 0xffffffffu;
  const float4 pa = active ? pk[p] : make_float4(0.f, 0.f, 0.f, 0.f);
  s_cells[threadIdx.x] = my_cell;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const bool head = active && (threadIdx.x == 0 || s_cells[threadIdx.x - 1] != my_cell);
  const uint32_t hmask = __ballot_sync(0xffffffffu, head);
  if (lane == 0) s_heads[warp] = __popc(hmask);
  __syncthreads();  // every thread has read its predecessor's cell
  uint32_t before = 0, ncells = 0;
#pragma unroll
  for (int w = 0; w < kLrThreads / 32; w++) {
    const uint32_t h = s_heads[w];
    before += (w < (int)warp) ? h : 0u;
    ncells += h;
  }
  // rank = heads at or before this thread, less one (active threads only)
  const uint32_t rank = before + __popc(hmask & (0xffffffffu >> (31u - lane))) - 1u;
  if (head) s_cells[rank] = my_cell;
  __syncthreads();
  double ex = 0.0, ey = 0.0, ez = 0.0, ee = 0.0;
  for (uint32_t w0 = 0; w0 < ncells; w0 += kLrfCells) {
    const uint32_t nc = min((uint32_t)kLrfCells, ncells - w0);
    const bool mine = active && rank >= w0 && rank < w0 + nc;
    const uint32_t slot = mine ? rank - w0 : 0;
    const bool warp_live = __any_sync(0xffffffffu, mine);
    float4 pre[kLrfPerThread];
    // prefetch one tile of every cell of this window into registers
    auto prefetch = [&](uint32_t d0) {
      const uint32_t nd = min(dirs_per_tile, ch.n_dir - d0);
#pragma unroll
      for (int k = 0; k < kLrfPerThread; k++) {
        const uint32_t t = threadIdx.x + k * kLrThreads;
        const uint32_t c = t / kLrfTilePairs, i = t % kLrfTilePairs;
        const uint32_t dd = i / npr, r = 2 * (i - dd * npr);
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c < nc && dd < nd) {
          const uint32_t node = ch.node_begin + (d0 + dd) * nr + r - node_off;
          const uint32_t cell = s_cells[w0 + c];
          const float2 x0 = R[sr_index(cell, node, ncell)];
          const float2 x1 = (r + 1 < nr) ? R[sr_index(cell, node + 1, ncell)] : make_float2(0.f, 0.f);
          v = make_float4(x0.x, x1.x, x0.y, x1.y);
        }
        pre[k] = v;
      }
    };
    __syncthreads();  // previous window done with s_n
    prefetch(0);
    for (uint32_t tile = 0; tile < ntiles; tile++) {
      const uint32_t d0 = tile * dirs_per_tile;
      const uint32_t nd = min(dirs_per_tile, ch.n_dir - d0);
      float4 *buf = s_n[tile & 1];
#pragma unroll
      for (int k = 0; k < kLrfPerThread; k++) {
        const uint32_t t = threadIdx.x + k * kLrThreads;
        buf[(t / kLrfTilePairs) * kLrfSlot + t % kLrfTilePairs] = pre[k];
      }
      __syncthreads();
      if (tile + 1 < ntiles) prefetch(d0 + dirs_per_tile);
      if (warp_live) {
        float tx = 0.f, ty = 0.f, tz = 0.f, te = 0.f;
        const float4 *cb = buf + slot * kLrfSlot;
        for (uint32_t d = 0; d < nd; d++) {
          const float4 sj = dirs[ch.dir_begin + d0 + d];
          const float u = fmaf(sj.x, pa.x, fmaf(sj.y, pa.y, sj.z * pa.z));
          const float2 u2 = bcast(u);
          float2 EA = make_float2(0.f, 0.f), EB = make_float2(0.f, 0.f), G = make_float2(0.f, 0.f);
          const float4 *nn = cb + d * npr;
          // Groups of kLrGroup pairs: pair q with bit q of kPolyMask takes
          // its sine and cosine from the FMA-pipe polynomial, interleaved
          // with the SFU pairs of its group; the remaining pairs use the SFU.  The radial scales of two pairs come
          // in one 16-byte load (the R' pair and the scales were two shared
          // loads per node pair in the MIO queue beside four MUFU operations).
          auto sfu_pair = [&](const float4 &v, float2 kp) {
            const float2 th = __fmul2_rn(kp, u2);
            float s0, c0, s1, c1;
            sfu_sincos(th.x, &s0, &c0);
            sfu_sincos(th.y, &s1, &c1);
            const float2 C = make_float2(c0, c1), Sn = make_float2(s0, s1);
            const float2 RX = make_float2(v.x, v.y), RY = make_float2(v.z, v.w);
            EA = __ffma2_rn(C, RX, EA);
            EB = __ffma2_rn(Sn, RY, EB);
            G = __ffma2_rn(kp, __ffma2_rn(C, RY, __fmul2_rn(Sn, RX)), G);
          };
          uint32_t k = 0;  // even throughout
          for (; k + kLrGroup <= npr; k += kLrGroup) {
            float4 kq;
#pragma unroll
            for (int q = 0; q < kLrGroup; q++) {
              if ((q & 1) == 0) kq = kq4[(k + q) >> 1];
              const float2 kp = (q & 1) ? make_float2(kq.z, kq.w) : make_float2(kq.x, kq.y);
              const float4 v = nn[k + q];
              if ((kPolyMask >> q) & 1u) {
                const float2 th = __fmul2_rn(kp, u2);
                float2 C, Sn, sg;
                fma_sincos_signed2(th, 1.0f, &Sn, &C, &sg);  // sg = (+-1, +-1)
                const float2 RX = __fmul2_rn(make_float2(v.x, v.y), sg);
                const float2 RY = __fmul2_rn(make_float2(v.z, v.w), sg);
                EA = __ffma2_rn(C, RX, EA);
                EB = __ffma2_rn(Sn, RY, EB);
                G = __ffma2_rn(kp, __ffma2_rn(C, RY, __fmul2_rn(Sn, RX)), G);
              } else {
                sfu_pair(v, kp);
              }
            }
          }
          // The last, partial group of a direction stays on the SFU: its
          // polynomial pairs, either guarded in a second unrolled copy of the
          // group (water10k 1.491 ms) or one pair per step with a uniform
          // test of the mask (1.511 ms), were slower than none (1.397 ms) --
          // only interleaved with the SFU pairs of a full group does the
          // polynomial's dependent chain hide.
          for (; k + 2 <= npr; k += 2) {
            const float4 kq = kq4[k >> 1];
            sfu_pair(nn[k], make_float2(kq.x, kq.y));
            sfu_pair(nn[k + 1], make_float2(kq.z, kq.w));
          }
          if (k < npr) {
            const float4 kq = kq4[k >> 1];
            sfu_pair(nn[k], make_float2(kq.x, kq.y));
          }
          const float e = (EA.x + EA.y) - (EB.x + EB.y), gsum = G.x + G.y;
          te += e;
          tx = fmaf(gsum, sj.x, tx);
          ty = fmaf(gsum, sj.y, ty);
          tz = fmaf(gsum, sj.z, tz);
        }
        if (mine) {
          ee += te;
          ex += tx;
          ey += ty;
          ez += tz;
        }
      }
      __syncthreads();
    }
  }
  if (active) {
    const double q = static_cast<double>(pa.w);
    double4 *dst = part + (size_t)by * natom + p;
    double4 v = make_double4(q * ex, q * ey, q * ez, q * ee);
    if (accumulate) {  // a later node stage adds into the same rows
      const double4 o = *dst;
      v = make_double4(o.x + v.x, o.y + v.y, o.z + v.z, o.w + v.w);
    }
    *dst = v;
  }
}

template <int kVariant>
__global__ void __launch_bounds__(kLrThreads, 8)
k_long_range_flat(const float4 *__restrict__ pk, const uint32_t *__restrict__ cell_point, uint32_t ncell,
                  const LrChunk *__restrict__ chunks, const float4 *__restrict__ dirs,
                  const float *__restrict__ kappa, const float2 *__restrict__ R, uint32_t node_off,
                  uint32_t natom, int accumulate, double4 *__restrict__ part,
                  const __grid_constant__ LrKappaQuads kpq) {
  lr_block<kLrPolyMasks[kVariant], true>(pk, cell_point, ncell, chunks, dirs, kappa, R, node_off, natom,
                                         accumulate, part, blockIdx.x, blockIdx.y, &kpq);
}

// ----------------------------------------------------------------------------
// Near field (src/glst_force.cu:1170-1544 restated): bare q_i q_j / r over
// the own cell (self skipped) and the up to 26 neighbour cells inside the
// grid (open boundary).  FP64 throughout.  CTA = (cell, row of neighbour
// cells, below); thread = atom; each row writes its own partial row of
// per-atom sums, summed by k_combine in a fixed order.  Smaller CTAs (64 or 96 threads, which
// fit in the registers the shell-sum blocks leave free) measured slower on
// water10k: 3.132 / 3.136 ms per solve against 3.122 ms.
constexpr int kSrThreads = 128;
// One CTA per (cell, row of neighbour cells) writes one row of per-atom
// partial sums: 3 rows (the x planes, 9 cells each) or 9 rows (x, y lines,
// 3 cells each).  Rows are numbered in x-major order of the 27 neighbours;
// the row holding the cell itself starts with it.  Nine rows shorten each
// thread's serial run of pairs threefold and triple the CTAs, for grids too
// small to fill the GPU with three (3,000 atoms on 4^3 cells: 0.076 ->
// 0.033 ms; 9,000 atoms on 5^3: 0.162 -> 0.092 ms; 18,000 on 6^3: 0.244 ->
// 0.117 ms); water10k's 7^3 grid already has 1,029 CTAs, and there nine
// rows measured 0.2 % slower per solve beside the far field.
// In the nine-row form each thread also runs two chains of accumulators
// (pairs j and j+1) instead of one, so the FP64 pipe has more independent
// work (3,000 atoms: near field 0.033 -> 0.025 ms, solve 0.141 -> 0.133 ms;
// 9,000 atoms: solve 0.239 -> 0.223 ms).  The three-row form keeps one
// chain: on water10k two chains made the near field 18 % faster alone but
// the solve 0.2 % slower beside the far field.
constexpr int kSrRowsPlanes = 3;
constexpr int kSrRowsLines = 9;
constexpr int kSrRowsMax = kSrRowsLines;

template <bool kTwoChains>
__device__ __forceinline__ void sr_block(const double4 *__restrict__ pd, const uint32_t *__restrict__ cell_count,
                                         const uint32_t *__restrict__ cell_point, const Grid &g, uint32_t natom,
                                         double4 *__restrict__ sr, uint32_t rows, uint32_t cell, uint32_t by) {
  __shared__ double4 s_at[kSrThreads];
  const int n = 27 / static_cast<int>(rows);  // neighbour cells per row
  const int t0 = static_cast<int>(by) * n;    // x-major index of the row's first neighbour
  const int dx = t0 / 9 - 1;                  // constant along a row
  const bool own_row = static_cast<int>(by) == 13 / n;
  const uint32_t cnt = cell_count[cell];
  const uint32_t start = cell_point[cell];
  const int ix = cell / (g.ny * g.nz), iy = (cell / g.nz) % g.ny, iz = cell % g.nz;
  const int jx = ix + dx;
  const bool plane_in = jx >= 0 && jx < (int)g.nx;
  for (uint32_t a0 = 0; a0 < cnt; a0 += kSrThreads) {
    const uint32_t ai = a0 + threadIdx.x;
    const bool active = ai < cnt;
    const double4 me = active ? pd[start + ai] : make_double4(0., 0., 0., 0.);
    double fx = 0.0, fy = 0.0, fz = 0.0, en = 0.0;
    // (own cell first in its row, as the reference's intra kernel)
    for (int nbi = 0; nbi < n && plane_in; nbi++) {
      const int t = t0 + (own_row ? (nbi + n / 2) % n : nbi);
      const int dyc = (t / 3) % 3 - 1, dzc = t % 3 - 1;
      const int jy = iy + dyc, jz = iz + dzc;
      if (jy < 0 || jz < 0 || jy >= (int)g.ny || jz >= (int)g.nz) continue;
      const bool own = dx == 0 && dyc == 0 && dzc == 0;
      const uint32_t nb = (jx * g.ny + jy) * g.nz + jz;
      const uint32_t bcnt = cell_count[nb];
      const uint32_t bstart = cell_point[nb];
      for (uint32_t b0 = 0; b0 < bcnt; b0 += kSrThreads) {
        const uint32_t nbt = min((uint32_t)kSrThreads, bcnt - b0);
        __syncthreads();
        if (threadIdx.x < nbt) s_at[threadIdx.x] = pd[bstart + b0 + threadIdx.x];
        __syncthreads();
        if (!active) continue;
        auto pair = [&](uint32_t j, double &ax, double &ay, double &az, double &an) {
          if (own && b0 + j == ai) return;  // self
          const double4 o4 = s_at[j];
          const double dx = me.x - o4.x, dy = me.y - o4.y, dz = me.z - o4.z;
          const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
          const double ir = rsqrt(r2);
          const double e = me.w * o4.w * ir;
          const double fs = e * ir * ir;
          ax = fma(fs, dx, ax);
          ay = fma(fs, dy, ay);
          az = fma(fs, dz, az);
          an += e;
        };
        if constexpr (kTwoChains) {
          // branch-free pairs (the self pair selected to zero), so the two
          // chains' instructions interleave
          double gx = 0.0, gy = 0.0, gz = 0.0, gn = 0.0;
          uint32_t j = 0;
          for (; j + 1 < nbt; j += 2) {
            const double4 o4 = s_at[j], p4 = s_at[j + 1];
            const bool sa = own && b0 + j == ai, sb = own && b0 + j + 1 == ai;
            const double dx = me.x - o4.x, dy = me.y - o4.y, dz = me.z - o4.z;
            const double hx = me.x - p4.x, hy = me.y - p4.y, hz = me.z - p4.z;
            const double r2 = sa ? 1.0 : fma(dx, dx, fma(dy, dy, dz * dz));
            const double s2 = sb ? 1.0 : fma(hx, hx, fma(hy, hy, hz * hz));
            const double ir = rsqrt(r2), is = rsqrt(s2);
            const double e = sa ? 0.0 : me.w * o4.w * ir;
            const double h = sb ? 0.0 : me.w * p4.w * is;
            const double fs = e * ir * ir, hs = h * is * is;
            fx = fma(fs, dx, fx);
            gx = fma(hs, hx, gx);
            fy = fma(fs, dy, fy);
            gy = fma(hs, hy, gy);
            fz = fma(fs, dz, fz);
            gz = fma(hs, hz, gz);
            en += e;
            gn += h;
          }
          if (j < nbt) pair(j, fx, fy, fz, en);
          fx += gx;
          fy += gy;
          fz += gz;
          en += gn;
        } else {
          for (uint32_t j = 0; j < nbt; j++) pair(j, fx, fy, fz, en);
        }
      }
    }
    if (active) sr[(size_t)by * natom + start + ai] = make_double4(fx, fy, fz, en);
  }
}

__global__ void __launch_bounds__(kSrThreads)
k_short_range(const double4 *__restrict__ pd, const uint32_t *__restrict__ cell_count,
              const uint32_t *__restrict__ cell_point, Grid g, uint32_t natom,
              double4 *__restrict__ sr, uint32_t rows) {
  if (rows == kSrRowsLines)
    sr_block<true>(pd, cell_count, cell_point, g, natom, sr, rows, blockIdx.x, blockIdx.y);
  else
    sr_block<false>(pd, cell_count, cell_point, g, natom, sr, rows, blockIdx.x, blockIdx.y);
}

// ----------------------------------------------------------------------------
// Combine: near field + long-range partials (fixed order), write the
// cell-ordered outputs and scatter to input order; per-CTA energy sums.
// A CTA takes kCombineAtoms consecutive atoms; its warps split the partial
// rows (warp w sums rows w, w + 8, ... for the warp's 32 atoms, each load a
// coalesced 1 KB run), then warp 0 adds the eight row sums and the near-field
// planes in a fixed order.  (One thread per atom summing every row left small
// systems, with hundreds of rows and a few CTAs, latency-bound.)
constexpr int kCombineThreads = 256;
constexpr int kCombineAtoms = 32;
constexpr int kCombineWarps = kCombineThreads / 32;

__device__ __forceinline__ void combine_block(const double4 *__restrict__ sr, uint32_t sr_rows,
                                              const double4 *__restrict__ part,
                                              uint32_t nsplit, const uint32_t *__restrict__ sorted_idx,
                                              uint32_t natom, int use_far, double *__restrict__ cfx,
                                              double *__restrict__ cfy, double *__restrict__ cfz,
                                              double *__restrict__ cen, double *__restrict__ ofx,
                                              double *__restrict__ ofy, double *__restrict__ ofz,
                                              double *__restrict__ oen, double *__restrict__ block_energy,
                                              uint32_t bx) {
  __shared__ double4 s_rows[kCombineWarps][kCombineAtoms];
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint32_t p = bx * kCombineAtoms + lane;
  const bool live = p < natom;
  double4 acc = make_double4(0., 0., 0., 0.);
  if (live && use_far) {
    for (uint32_t s = w; s < nsplit; s += kCombineWarps) {
      const double4 v = part[(size_t)s * natom + p];
      acc.x += v.x; acc.y += v.y; acc.z += v.z; acc.w += v.w;
    }
  }
  s_rows[w][lane] = acc;
  __syncthreads();
  if (w != 0) return;
  double e = 0.0;
  if (live) {
    double4 t = s_rows[0][lane];
#pragma unroll
    for (int k = 1; k < kCombineWarps; k++) {
      const double4 v = s_rows[k][lane];
      t.x += v.x; t.y += v.y; t.z += v.z; t.w += v.w;
    }
    for (uint32_t pl = 0; pl < sr_rows; pl++) {
      const double4 v = sr[(size_t)pl * natom + p];
      t.x += v.x; t.y += v.y; t.z += v.z; t.w += v.w;
    }
    cfx[p] = t.x; cfy[p] = t.y; cfz[p] = t.z; cen[p] = t.w;
    const uint32_t i = sorted_idx[p];
    if (i < natom) { ofx[i] = t.x; ofy[i] = t.y; ofz[i] = t.z; oen[i] = t.w; }
    e = t.w;
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
  if (lane == 0) block_energy[bx] = e;
}

__global__ void __launch_bounds__(kCombineThreads)
k_combine(const double4 *__restrict__ sr, uint32_t sr_rows, const double4 *__restrict__ part, uint32_t nsplit,
          const uint32_t *__restrict__ sorted_idx, uint32_t natom, int use_far,
          double *__restrict__ cfx, double *__restrict__ cfy, double *__restrict__ cfz,
          double *__restrict__ cen, double *__restrict__ ofx, double *__restrict__ ofy,
          double *__restrict__ ofz, double *__restrict__ oen, double *__restrict__ block_energy) {
  combine_block(sr, sr_rows, part, nsplit, sorted_idx, natom, use_far, cfx, cfy, cfz, cen, ofx, ofy, ofz, oen,
                block_energy, blockIdx.x);
}

// ----------------------------------------------------------------------------
// Sum of the per-atom outputs of the node-range shards of one system (the
// reference's reduce to GPU 0, src/glst_force.cu:1584-1602 with
// src/device_comm.cu:176-201 ncclReduce): dst[i] = src[0][i] + src[1][i] +
// ..., shards in order, for the four input-order and the four cell-order
// arrays.  The sources may live on other GPUs (read over NVLink through peer
// access).  Per-CTA energy sums as k_combine writes them.
constexpr int kMaxShards = 16;
struct ShardSet {
  const double *src[kMaxShards][8];  // per shard: ofx, ofy, ofz, oen, cfx, cfy, cfz, cen
  double *dst[8];
  uint32_t n;
};

__global__ void __launch_bounds__(kCombineThreads)
k_reduce_shards(ShardSet ss, uint32_t natom, double *__restrict__ block_energy) {
  __shared__ double s_red[kCombineThreads / 32];
  const uint32_t i = blockIdx.x * kCombineThreads + threadIdx.x;
  double e = 0.0;
  if (i < natom) {
#pragma unroll
    for (int a = 0; a < 8; a++) {
      double t = 0.0;
      for (uint32_t s = 0; s < ss.n; s++) t += ss.src[s][a][i];
      ss.dst[a][i] = t;
      if (a == 3) e = t;
    }
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kCombineThreads / 32; w++) t += s_red[w];
    block_energy[blockIdx.x] = t;
  }
}

// Total energy 0.5 * sum of the per-CTA sums, fixed order (one CTA).
__device__ __forceinline__ void energy_body(const double *__restrict__ block_energy, uint32_t nblocks,
                                            double *__restrict__ total) {
  __shared__ double s_red[32];
  double e = 0.0;
  for (uint32_t b = threadIdx.x; b < nblocks; b += blockDim.x) e += block_energy[b];
  for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (unsigned w = 0; w < (blockDim.x >> 5); w++) t += s_red[w];
    *total = 0.5 * t;
  }
}

__global__ void k_energy_total(const double *__restrict__ block_energy, uint32_t nblocks,
                               double *__restrict__ total) {
  energy_body(block_energy, nblocks, total);
}

// ----------------------------------------------------------------------------
// Direct all-pairs Coulomb, FP64, open boundary (the reference's physics
// check, utils/coulomb.cu:14-82): thread per atom, the other atoms streamed
// through shared memory.
constexpr int kDirectThreads = 128;

__global__ void __launch_bounds__(kDirectThreads)
k_direct_coulomb(const double *__restrict__ rx, const double *__restrict__ ry, const double *__restrict__ rz,
                 const double *__restrict__ qc, uint32_t n, double *__restrict__ fx, double *__restrict__ fy,
                 double *__restrict__ fz, double *__restrict__ en) {
  __shared__ double4 s_at[kDirectThreads];
  const uint32_t i = blockIdx.x * kDirectThreads + threadIdx.x;
  const bool active = i < n;
  const double xi = active ? rx[i] : 0.0, yi = active ? ry[i] : 0.0, zi = active ? rz[i] : 0.0;
  const double qi = active ? qc[i] : 0.0;
  double f0 = 0.0, f1 = 0.0, f2 = 0.0, e0 = 0.0;
  for (uint32_t j0 = 0; j0 < n; j0 += kDirectThreads) {
    const uint32_t nj = min((uint32_t)kDirectThreads, n - j0);
    __syncthreads();
    if (threadIdx.x < nj) {
      const uint32_t j = j0 + threadIdx.x;
      s_at[threadIdx.x] = make_double4(rx[j], ry[j], rz[j], qc[j]);
    }
    __syncthreads();
    if (!active) continue;
    for (uint32_t k = 0; k < nj; k++) {
      if (j0 + k == i) continue;
      const double4 o = s_at[k];
      const double dx = xi - o.x, dy = yi - o.y, dz = zi - o.z;
      const double ir = rsqrt(fma(dx, dx, fma(dy, dy, dz * dz)));
      const double e = qi * o.w * ir;
      const double fs = e * ir * ir;
      f0 = fma(fs, dx, f0);
      f1 = fma(fs, dy, f1);
      f2 = fma(fs, dz, f2);
      e0 += e;
    }
  }
  if (active) {
    fx[i] = f0;
    fy[i] = f1;
    fz[i] = f2;
    en[i] = e0;
  }
}

// ----------------------------------------------------------------------------
// Pipe-peak probes (roofline denominators).  Eight independent chains per
// thread keep the pipe busy; the results are stored so nothing is removed.
__global__ void k_probe_sfu(float *out, int iters) {
  float a[8];
#pragma unroll
  for (int u = 0; u < 8; u++) a[u] = 0.001f * (threadIdx.x + u);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
      float s, c;
      sfu_sincos(a[u], &s, &c);
      a[u] = s + c;  // 2 MUFU + 1 FADD
    }
  }
  float t = 0.f;
#pragma unroll
  for (int u = 0; u < 8; u++) t += a[u];
  out[blockIdx.x * blockDim.x + threadIdx.x] = t;
}

__global__ void k_probe_fma(float *out, int iters) {
  float a[8];
#pragma unroll
  for (int u = 0; u < 8; u++) a[u] = 0.001f * (threadIdx.x + u);
  const float m = 0.999f, b = 0.0001f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 8; u++) a[u] = fmaf(a[u], m, b);
  }
  float t = 0.f;
#pragma unroll
  for (int u = 0; u < 8; u++) t += a[u];
  out[blockIdx.x * blockDim.x + threadIdx.x] = t;
}

}  // namespace dev
}  // namespace glst
