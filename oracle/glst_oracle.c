/*
 * ORACLE (test infrastructure only) -- FP64 CPU restatement of the GLST sum.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg (and its
 * --impl reference arm) load this library, as the checker / CPU baseline.  The
 * product never links it.
 *
 * It follows the reference's double-precision path step by step, in the same
 * summation order, on the host with OpenMP:
 *   assignment  src/glst_force.cu:356-386 (binning + clamp), :388-400 (offsets),
 *               :510-530 (stable radix sort by cell id => input order in a cell)
 *   SF          src/glst_force.cu:601-664  S_c(k) = sum_j q_j e^{-i k.r_j}
 *   prefix sums src/glst_force.cu:702-772  inclusive z, then y, then x
 *   shell sums  src/glst_force.cu:774-913  cube(r_out) - cube(r_in), 8-corner boxes
 *   LR gather   src/glst_force.cu:1060-1135
 *   SR          src/glst_force.cu:1248-1324 (own cell) and :1436-1544 (26 nbrs)
 *   direct sum  utils/coulomb.cu:14-82 (all pairs, open boundary)
 * Outputs are returned in input order (what get_ef gives, src/glst_force.cu:142-176).
 * oracle_far_arrays returns the two far-field phases' arrays themselves (the
 * reference's sf_re_/sf_im_ and rmt_sum_re_/rmt_sum_im_), for per-phase checks.
 */
#define _GNU_SOURCE /* sincos */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  uint32_t nx, ny, nz;
  double cell_dim;     /* CT-rounded cell edge, as double */
  int ct_float;        /* 1: bin in float like glst_force<float> */
  uint32_t K;          /* number of cubature nodes passed */
  const double *kx, *ky, *kz, *w;
  const uint32_t *group;
  uint32_t ngroup;
  const uint32_t *r_in, *r_out;
  int has_far;
} oracle_plan;

static uint32_t bin_axis(double r, double l, uint32_t n, int ct_float) {
  int c;
  if (ct_float) {
    float rf = (float)r;
    float inv = 1.0f / (float)l;
    c = (int)(rf * inv);
  } else {
    double inv = 1.0 / l;
    c = (int)(r * inv);
  }
  if (c >= (int)n) c = (int)n - 1;
  if (c < 0) c = 0;
  return (uint32_t)c;
}

/* Cell id per atom, counts, exclusive offsets and the stable cell order. */
int oracle_assign(uint32_t natom, const double *rx, const double *ry,
                  const double *rz, const oracle_plan *p, uint32_t *atom_cell,
                  uint32_t *cell_count, uint32_t *cell_point,
                  uint32_t *sorted_idx) {
  uint32_t ncell = p->nx * p->ny * p->nz;
  memset(cell_count, 0, sizeof(uint32_t) * ncell);
  for (uint32_t i = 0; i < natom; i++) {
    uint32_t cx = bin_axis(rx[i], p->cell_dim, p->nx, p->ct_float);
    uint32_t cy = bin_axis(ry[i], p->cell_dim, p->ny, p->ct_float);
    uint32_t cz = bin_axis(rz[i], p->cell_dim, p->nz, p->ct_float);
    uint32_t cell = (cx * p->ny + cy) * p->nz + cz;
    atom_cell[i] = cell;
    cell_count[cell]++;
  }
  uint32_t acc = 0;
  for (uint32_t c = 0; c < ncell; c++) {
    cell_point[c] = acc;
    acc += cell_count[c];
  }
  uint32_t *fill = (uint32_t *)calloc(ncell, sizeof(uint32_t));
  if (!fill) return -1;
  for (uint32_t i = 0; i < natom; i++) {
    uint32_t c = atom_cell[i];
    sorted_idx[cell_point[c] + fill[c]++] = i;
  }
  free(fill);
  return 0;
}

static void box_sum(double *re, double *im, const double *Pre, const double *Pim,
                    uint32_t x0, uint32_t y0, uint32_t z0, uint32_t x1,
                    uint32_t y1, uint32_t z1, uint32_t ny, uint32_t nz,
                    size_t k, size_t K) {
  int xb = (x0 == 0), yb = (y0 == 0), zb = (z0 == 0);
  uint32_t xm = xb ? 0 : x0 - 1, ym = yb ? 0 : y0 - 1, zm = zb ? 0 : z0 - 1;
#define AT(a, b, c) (((size_t)((a) * ny + (b)) * nz + (c)) * K + k)
  double g0r = Pre[AT(x1, y1, z1)], g0i = Pim[AT(x1, y1, z1)];
  double g1r = xb ? 0.0 : Pre[AT(xm, y1, z1)], g1i = xb ? 0.0 : Pim[AT(xm, y1, z1)];
  double g2r = yb ? 0.0 : Pre[AT(x1, ym, z1)], g2i = yb ? 0.0 : Pim[AT(x1, ym, z1)];
  double g3r = zb ? 0.0 : Pre[AT(x1, y1, zm)], g3i = zb ? 0.0 : Pim[AT(x1, y1, zm)];
  double g4r = (xb || yb) ? 0.0 : Pre[AT(xm, ym, z1)], g4i = (xb || yb) ? 0.0 : Pim[AT(xm, ym, z1)];
  double g5r = (xb || zb) ? 0.0 : Pre[AT(xm, y1, zm)], g5i = (xb || zb) ? 0.0 : Pim[AT(xm, y1, zm)];
  double g6r = (yb || zb) ? 0.0 : Pre[AT(x1, ym, zm)], g6i = (yb || zb) ? 0.0 : Pim[AT(x1, ym, zm)];
  double g7r = (xb || yb || zb) ? 0.0 : Pre[AT(xm, ym, zm)];
  double g7i = (xb || yb || zb) ? 0.0 : Pim[AT(xm, ym, zm)];
#undef AT
  *re = g0r - g1r - g2r - g3r + g4r + g5r + g6r - g7r;
  *im = g0i - g1i - g2i - g3i + g4i + g5i + g6i - g7i;
}

static void cube_sum(double *re, double *im, const double *Pre, const double *Pim,
                     uint32_t x, uint32_t y, uint32_t z, uint32_t r,
                     uint32_t nx, uint32_t ny, uint32_t nz, size_t k, size_t K) {
  uint32_t x0 = x < r ? 0 : x - r, y0 = y < r ? 0 : y - r, z0 = z < r ? 0 : z - r;
  uint32_t x1 = x + r, y1 = y + r, z1 = z + r;
  if (x1 >= nx) x1 = nx - 1;
  if (y1 >= ny) y1 = ny - 1;
  if (z1 >= nz) z1 = nz - 1;
  box_sum(re, im, Pre, Pim, x0, y0, z0, x1, y1, z1, ny, nz, k, K);
}

/* Structure factors (src/glst_force.cu:601-664) of cell-ordered atoms X over
 * nodes [k0, k0 + K) into S[c * K + kk], then -- if R is non-NULL -- the
 * inclusive prefix sums z, y, x (:702-772) in place and the shell sums times
 * weight (:774-913) into R.  S_copy (may be NULL) receives S before the
 * prefix sums. */
static void far_arrays(const double *X, const uint32_t *cnt, const uint32_t *pnt, const oracle_plan *p,
                       uint32_t k0, size_t K, double *Sre, double *Sim, double *Rre, double *Rim,
                       double *S_copy_re, double *S_copy_im) {
  const uint32_t nx = p->nx, ny = p->ny, nz = p->nz;
  const uint32_t ncell = nx * ny * nz;
  /* structure factors */
#pragma omp parallel for schedule(dynamic, 1)
  for (uint32_t c = 0; c < ncell; c++) {
    for (size_t kk = 0; kk < K; kk++) {
      const double kx = p->kx[k0 + kk], ky = p->ky[k0 + kk], kz = p->kz[k0 + kk];
      double sr = 0.0, si = 0.0;
      for (uint32_t a = pnt[c]; a < pnt[c] + cnt[c]; a++) {
        double th = kx * X[4 * a] + ky * X[4 * a + 1] + kz * X[4 * a + 2];
        double sn, cs;
        sincos(th, &sn, &cs);
        sr += X[4 * a + 3] * cs;
        si -= X[4 * a + 3] * sn;
      }
      Sre[(size_t)c * K + kk] = sr;
      Sim[(size_t)c * K + kk] = si;
    }
  }
  if (S_copy_re) memcpy(S_copy_re, Sre, sizeof(double) * ncell * K);
  if (S_copy_im) memcpy(S_copy_im, Sim, sizeof(double) * ncell * K);
  if (!Rre || !Rim) return;
  /* inclusive prefix sums: z, then y, then x */
#pragma omp parallel for schedule(static)
  for (size_t kk = 0; kk < K; kk++) {
    for (uint32_t x = 0; x < nx; x++)
      for (uint32_t y = 0; y < ny; y++) {
        double ar = 0.0, ai = 0.0;
        for (uint32_t z = 0; z < nz; z++) {
          size_t o = ((size_t)(x * ny + y) * nz + z) * K + kk;
          ar += Sre[o]; ai += Sim[o]; Sre[o] = ar; Sim[o] = ai;
        }
      }
    for (uint32_t x = 0; x < nx; x++)
      for (uint32_t z = 0; z < nz; z++) {
        double ar = 0.0, ai = 0.0;
        for (uint32_t y = 0; y < ny; y++) {
          size_t o = ((size_t)(x * ny + y) * nz + z) * K + kk;
          ar += Sre[o]; ai += Sim[o]; Sre[o] = ar; Sim[o] = ai;
        }
      }
    for (uint32_t y = 0; y < ny; y++)
      for (uint32_t z = 0; z < nz; z++) {
        double ar = 0.0, ai = 0.0;
        for (uint32_t x = 0; x < nx; x++) {
          size_t o = ((size_t)(x * ny + y) * nz + z) * K + kk;
          ar += Sre[o]; ai += Sim[o]; Sre[o] = ar; Sim[o] = ai;
        }
      }
  }
  /* shell sums times weight */
#pragma omp parallel for schedule(static)
  for (uint32_t c = 0; c < ncell; c++) {
    uint32_t x = c / (ny * nz), y = (c / nz) % ny, z = c % nz;
    for (size_t kk = 0; kk < K; kk++) {
      uint32_t g = p->group[k0 + kk];
      double orr, oi, ir, ii;
      cube_sum(&orr, &oi, Sre, Sim, x, y, z, p->r_out[g], nx, ny, nz, kk, K);
      cube_sum(&ir, &ii, Sre, Sim, x, y, z, p->r_in[g], nx, ny, nz, kk, K);
      Rre[(size_t)c * K + kk] = (orr - ir) * p->w[k0 + kk];
      Rim[(size_t)c * K + kk] = (oi - ii) * p->w[k0 + kk];
    }
  }
}

/* Cell assignment plus the cell-ordered packet array X (x, y, z, q). */
static int assign_pack(uint32_t natom, const double *rx, const double *ry, const double *rz, const double *qc,
                       const oracle_plan *p, uint32_t *atom_cell, uint32_t *cnt, uint32_t *pnt, uint32_t *sidx,
                       double *X) {
  if (oracle_assign(natom, rx, ry, rz, p, atom_cell, cnt, pnt, sidx) != 0) return -1;
  for (uint32_t a = 0; a < natom; a++) {
    uint32_t i = sidx[a];
    X[4 * a + 0] = rx[i];
    X[4 * a + 1] = ry[i];
    X[4 * a + 2] = rz[i];
    X[4 * a + 3] = qc[i];
  }
  return 0;
}

/* The reference's per-phase far-field arrays for all nodes: sf (after
 * calc_sf) and rmt_sum (after sum_rmt_sf), [ncell][K] each, row = cell. */
int oracle_far_arrays(uint32_t natom, const double *rx, const double *ry, const double *rz, const double *qc,
                      const oracle_plan *p, double *sf_re, double *sf_im, double *rmt_re, double *rmt_im) {
  const uint32_t ncell = p->nx * p->ny * p->nz;
  const size_t K = p->K;
  uint32_t *atom_cell = malloc(sizeof(uint32_t) * (natom ? natom : 1));
  uint32_t *cnt = malloc(sizeof(uint32_t) * ncell);
  uint32_t *pnt = malloc(sizeof(uint32_t) * ncell);
  uint32_t *sidx = malloc(sizeof(uint32_t) * (natom ? natom : 1));
  double *X = malloc(sizeof(double) * (natom ? natom : 1) * 4);
  double *Sre = malloc(sizeof(double) * ncell * (K ? K : 1));
  double *Sim = malloc(sizeof(double) * ncell * (K ? K : 1));
  int rc = -1;
  if (atom_cell && cnt && pnt && sidx && X && Sre && Sim &&
      assign_pack(natom, rx, ry, rz, qc, p, atom_cell, cnt, pnt, sidx, X) == 0) {
    far_arrays(X, cnt, pnt, p, 0, K, Sre, Sim, rmt_re, rmt_im, sf_re, sf_im);
    rc = 0;
  }
  free(atom_cell); free(cnt); free(pnt); free(sidx); free(X); free(Sre); free(Sim);
  return rc;
}

/* Far field (SF -> prefix sums -> shell sums -> LR) over nodes [k0, k1), plus
 * (if do_sr) the near field.  Accumulates into cell-ordered outputs, like the
 * reference's += into fx_/fy_/fz_/en_; returned in input order. */
int oracle_glst(uint32_t natom, const double *rx, const double *ry,
                const double *rz, const double *qc, const oracle_plan *p,
                uint32_t k0, uint32_t k1, int do_far, int do_sr, double *fx,
                double *fy, double *fz, double *en) {
  const uint32_t nx = p->nx, ny = p->ny, nz = p->nz;
  const uint32_t ncell = nx * ny * nz;
  uint32_t *atom_cell = malloc(sizeof(uint32_t) * (natom ? natom : 1));
  uint32_t *cnt = malloc(sizeof(uint32_t) * ncell);
  uint32_t *pnt = malloc(sizeof(uint32_t) * ncell);
  uint32_t *sidx = malloc(sizeof(uint32_t) * (natom ? natom : 1));
  double *X = malloc(sizeof(double) * (natom ? natom : 1) * 4);
  double *F = calloc((size_t)(natom ? natom : 1) * 4, sizeof(double));
  if (!atom_cell || !cnt || !pnt || !sidx || !X || !F) return -1;
  assign_pack(natom, rx, ry, rz, qc, p, atom_cell, cnt, pnt, sidx, X);
  if (k1 > p->K) k1 = p->K;
  if (k0 > k1) k0 = k1;
  const size_t K = (size_t)(k1 - k0);
  if (do_far && p->has_far && K > 0) {
    double *Sre = malloc(sizeof(double) * ncell * K);
    double *Sim = malloc(sizeof(double) * ncell * K);
    double *Rre = malloc(sizeof(double) * ncell * K);
    double *Rim = malloc(sizeof(double) * ncell * K);
    if (!Sre || !Sim || !Rre || !Rim) return -1;
    far_arrays(X, cnt, pnt, p, k0, K, Sre, Sim, Rre, Rim, NULL, NULL);
    /* long-range gather */
#pragma omp parallel for schedule(dynamic, 16)
    for (uint32_t a = 0; a < natom; a++) {
      uint32_t c = atom_cell[sidx[a]];
      double xa = X[4 * a], ya = X[4 * a + 1], za = X[4 * a + 2], qa = X[4 * a + 3];
      double f0 = 0.0, f1 = 0.0, f2 = 0.0, e0 = 0.0;
      for (size_t kk = 0; kk < K; kk++) {
        const double kx = p->kx[k0 + kk], ky = p->ky[k0 + kk], kz = p->kz[k0 + kk];
        double th = kx * xa + ky * ya + kz * za;
        double re, im;
        sincos(th, &im, &re);
        double rr = Rre[(size_t)c * K + kk], ri = Rim[(size_t)c * K + kk];
        double dre = qa * (re * rr - im * ri);
        double dim = qa * (re * ri + im * rr);
        f0 += dim * kx; f1 += dim * ky; f2 += dim * kz; e0 += dre;
      }
      F[4 * a + 0] += f0; F[4 * a + 1] += f1; F[4 * a + 2] += f2; F[4 * a + 3] += e0;
    }
    free(Sre); free(Sim); free(Rre); free(Rim);
  }
  if (do_sr) {
#pragma omp parallel for schedule(dynamic, 16)
    for (uint32_t a = 0; a < natom; a++) {
      uint32_t cell = atom_cell[sidx[a]];
      uint32_t xc = cell / (ny * nz), yc = (cell / nz) % ny, zc = cell % nz;
      double xi = X[4 * a], yi = X[4 * a + 1], zi = X[4 * a + 2], qi = X[4 * a + 3];
      double f0 = 0.0, f1 = 0.0, f2 = 0.0, e0 = 0.0;
      /* own cell first (intra kernel), then the 26 neighbours (inter kernel) */
      for (uint32_t b = pnt[cell]; b < pnt[cell] + cnt[cell]; b++) {
        if (b == a) continue;
        double qij = qi * X[4 * b + 3];
        double dx = xi - X[4 * b], dy = yi - X[4 * b + 1], dz = zi - X[4 * b + 2];
        double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2), ir = 1.0 / r;
        double dudr = qij / r2;
        f0 += dudr * (dx * ir); f1 += dudr * (dy * ir); f2 += dudr * (dz * ir);
        e0 += qij * ir;
      }
      double g0 = 0.0, g1 = 0.0, g2 = 0.0, ge = 0.0;
      for (int da = -1; da <= 1; da++) {
        if ((xc == 0 && da == -1) || (xc == nx - 1 && da == 1)) continue;
        for (int db = -1; db <= 1; db++) {
          if ((yc == 0 && db == -1) || (yc == ny - 1 && db == 1)) continue;
          for (int dc = -1; dc <= 1; dc++) {
            if ((zc == 0 && dc == -1) || (zc == nz - 1 && dc == 1)) continue;
            if (da == 0 && db == 0 && dc == 0) continue;
            uint32_t nb = (((uint32_t)((int)xc + da)) * ny + (uint32_t)((int)yc + db)) * nz + (uint32_t)((int)zc + dc);
            for (uint32_t b = pnt[nb]; b < pnt[nb] + cnt[nb]; b++) {
              double qij = qi * X[4 * b + 3];
              double dx = xi - X[4 * b], dy = yi - X[4 * b + 1], dz = zi - X[4 * b + 2];
              double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2), ir = 1.0 / r;
              double dudr = qij / r2;
              g0 += dudr * (dx * ir); g1 += dudr * (dy * ir); g2 += dudr * (dz * ir);
              ge += qij * ir;
            }
          }
        }
      }
      /* intra and inter are separate += into the outputs in the reference */
      F[4 * a + 0] = (F[4 * a + 0] + f0) + g0;
      F[4 * a + 1] = (F[4 * a + 1] + f1) + g1;
      F[4 * a + 2] = (F[4 * a + 2] + f2) + g2;
      F[4 * a + 3] = (F[4 * a + 3] + e0) + ge;
    }
  }
  for (uint32_t a = 0; a < natom; a++) {
    uint32_t i = sidx[a];
    fx[i] = F[4 * a]; fy[i] = F[4 * a + 1]; fz[i] = F[4 * a + 2]; en[i] = F[4 * a + 3];
  }
  free(atom_cell); free(cnt); free(pnt); free(sidx); free(X); free(F);
  return 0;
}

/* FP64 direct all-pairs Coulomb, open boundary (utils/coulomb.cu:14-82). */
void oracle_coulomb(uint32_t natom, const double *rx, const double *ry,
                    const double *rz, const double *qc, double *fx, double *fy,
                    double *fz, double *en) {
#pragma omp parallel for schedule(dynamic, 16)
  for (uint32_t i = 0; i < natom; i++) {
    double f0 = 0.0, f1 = 0.0, f2 = 0.0, e0 = 0.0;
    for (uint32_t j = 0; j < natom; j++) {
      if (j == i) continue;
      double qij = qc[i] * qc[j];
      double dx = rx[i] - rx[j], dy = ry[i] - ry[j], dz = rz[i] - rz[j];
      double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2), ir = 1.0 / r;
      double dudr = qij / r2;
      f0 += dudr * (dx * ir); f1 += dudr * (dy * ir); f2 += dudr * (dz * ir);
      e0 += qij * ir;
    }
    fx[i] = f0; fy[i] = f1; fz[i] = f2; en[i] = e0;
  }
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
