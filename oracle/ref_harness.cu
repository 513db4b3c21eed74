// ORACLE (test infrastructure only): a driver for the UNMODIFIED reference
// library, compiled from the reference's own sources by oracle/Makefile into
// oracle/_ref/.  It runs glst_force<CT> through its public API the way the
// reference driver does (test/full_example.cu:121-236): construct from
// (natom, tol, box, rcut), call calc_ener_force repeatedly with the outputs
// zeroed in between, then get_ef.  It also copies out the cell assignment
// (sorted_idx_, cell_atom_count_, cell_atom_point_) so the assignment can be
// checked bit for bit.  Those members are private in the reference header, so
// this file alone widens access before including it.
//
// The reference reads spherical t-designs from "SS31-Mar-2016/" in the current
// directory (src/cubature.cu:490); the caller runs this binary from a
// directory where that folder holds the project-generated designs.
//
// usage: glst_ref_harness <in.bin> <out.bin> <float|double> <iterations>
//        glst_ref_harness --batch <list.bin> <out.bin> <float|double> <iterations>
//                         [<forces.bin> <every>]
//   in.bin : u32 natom, f64 tol, f64 box[3], f64 rcut, f64 x[N], y[N], z[N], q[N]
//   out.bin: u32 natom, u32 K, u32 nx, ny, nz, u32 iterations,
//            f64 ms_mean[8] (assign, sf, sum, lr, sr, comm, total, events_total),
//            f64 fx[N], fy[N], fz[N], en[N] (input order),
//            u32 sorted_idx[N], u32 cell_count[C], u32 cell_point[C]
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#define private public
#include "glst_force.hcu"
#undef private

template <typename CT>
static int run(const char *out_path, unsigned natom, double tol,
               const double box[3], double rcut, const std::vector<double> &x,
               const std::vector<double> &y, const std::vector<double> &z,
               const std::vector<double> &q, int iters) {
  cuda_container<double> rx(x), ry(y), rz(z), qc(q);
  rx.transfer_to_device();
  ry.transfer_to_device();
  rz.transfer_to_device();
  qc.transfer_to_device();
  glst_force<CT> glst(natom, tol, box[0], box[1], box[2], rcut);
  std::vector<double> acc(8, 0.0);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto now = [] { return std::chrono::high_resolution_clock::now(); };
  auto ms = [](auto a, auto b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
  };
  for (int it = -1; it < iters; it++) {  // it = -1 is an untimed warm-up
    glst.fx()[0].set(0.0);
    glst.fy()[0].set(0.0);
    glst.fz()[0].set(0.0);
    glst.en()[0].set(0.0);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, 0);
    auto t0 = now();
    glst.assign_atoms(rx.d_array().data(), ry.d_array().data(),
                      rz.d_array().data(), qc.d_array().data());
    cudaDeviceSynchronize();
    auto t1 = now();
    glst.calc_sf();
    cudaDeviceSynchronize();
    auto t2 = now();
    glst.sum_rmt_sf();
    cudaDeviceSynchronize();
    auto t3 = now();
    glst.calc_lr_ef();
    cudaDeviceSynchronize();
    auto t4 = now();
    glst.calc_sr_ef();
    cudaDeviceSynchronize();
    auto t5 = now();
    glst.comm_ef();
    cudaDeviceSynchronize();
    auto t6 = now();
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float evms = 0.f;
    cudaEventElapsedTime(&evms, e0, e1);
    if (it >= 0) {
      acc[0] += ms(t0, t1); acc[1] += ms(t1, t2); acc[2] += ms(t2, t3);
      acc[3] += ms(t3, t4); acc[4] += ms(t4, t5); acc[5] += ms(t5, t6);
      acc[6] += ms(t0, t6); acc[7] += evms;
    }
  }
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err));
    return 3;
  }
  for (double &a : acc) a /= (iters > 0 ? iters : 1);
  cuda_container<double> fx, fy, fz, en;
  glst.get_ef(fx, fy, fz, en);
  glst.sorted_idx_[0].transfer_to_host();
  glst.cell_atom_count_[0].transfer_to_host();
  glst.cell_atom_point_[0].transfer_to_host();
  FILE *f = std::fopen(out_path, "wb");
  if (!f) return 2;
  unsigned hdr[6] = {natom, glst.cubature_->tot_num_nodes(), glst.ncell_x_,
                     glst.ncell_y_, glst.ncell_z_, (unsigned)iters};
  std::fwrite(hdr, sizeof(unsigned), 6, f);
  std::fwrite(acc.data(), sizeof(double), 8, f);
  std::fwrite(fx.h_array().data(), sizeof(double), natom, f);
  std::fwrite(fy.h_array().data(), sizeof(double), natom, f);
  std::fwrite(fz.h_array().data(), sizeof(double), natom, f);
  std::fwrite(en.h_array().data(), sizeof(double), natom, f);
  std::fwrite(glst.sorted_idx_[0].h_array().data(), sizeof(unsigned), natom, f);
  std::fwrite(glst.cell_atom_count_[0].h_array().data(), sizeof(unsigned),
              glst.ncell_, f);
  std::fwrite(glst.cell_atom_point_[0].h_array().data(), sizeof(unsigned),
              glst.ncell_, f);
  std::fclose(f);
  return 0;
}

// Batch mode: the reference's plain path on many independent systems, one
// after another (construct, one warm-up solve, `iters` timed solves, get_ef,
// destroy).  Only calc_ener_force is timed, the same host-clock-plus-sync
// method as above.
//   list.bin: u32 nsys, then per system the in.bin record above
//   out.bin : u32 nsys, then per system u32 natom, u32 K, f64 ms_host,
//             f64 ms_events, f64 energy (0.5 * sum en)
//   forces.bin (optional, with every > 0): for systems s with s % every == 0,
//             u32 s, u32 natom, f64 fx[N], fy[N], fz[N], en[N] (input order)
template <typename CT>
static int run_batch(FILE *in, FILE *out, unsigned nsys, int iters, FILE *forces, unsigned every) {
  std::fwrite(&nsys, sizeof(unsigned), 1, out);
  for (unsigned s = 0; s < nsys; s++) {
    unsigned natom = 0;
    double tol = 0, box[3] = {0, 0, 0}, rcut = 0;
    if (std::fread(&natom, sizeof(unsigned), 1, in) != 1) return 2;
    if (std::fread(&tol, sizeof(double), 1, in) != 1) return 2;
    if (std::fread(box, sizeof(double), 3, in) != 3) return 2;
    if (std::fread(&rcut, sizeof(double), 1, in) != 1) return 2;
    std::vector<double> x(natom), y(natom), z(natom), q(natom);
    for (auto *v : {&x, &y, &z, &q})
      if (std::fread(v->data(), sizeof(double), natom, in) != natom) return 2;
    double ms_host = 0, ms_ev = 0, energy = 0;
    unsigned K = 0;
    {
      cuda_container<double> rx(x), ry(y), rz(z), qc(q);
      rx.transfer_to_device();
      ry.transfer_to_device();
      rz.transfer_to_device();
      qc.transfer_to_device();
      glst_force<CT> glst(natom, tol, box[0], box[1], box[2], rcut);
      K = glst.cubature_ ? glst.cubature_->tot_num_nodes() : 0u;
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      for (int it = -1; it < iters; it++) {
        glst.fx()[0].set(0.0);
        glst.fy()[0].set(0.0);
        glst.fz()[0].set(0.0);
        glst.en()[0].set(0.0);
        cudaDeviceSynchronize();
        cudaEventRecord(e0, 0);
        auto t0 = std::chrono::high_resolution_clock::now();
        glst.calc_ener_force(rx.d_array().data(), ry.d_array().data(),
                             rz.d_array().data(), qc.d_array().data());
        cudaDeviceSynchronize();
        auto t1 = std::chrono::high_resolution_clock::now();
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float evms = 0.f;
        cudaEventElapsedTime(&evms, e0, e1);
        if (it >= 0) {
          ms_host += std::chrono::duration<double, std::milli>(t1 - t0).count();
          ms_ev += evms;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      cuda_container<double> fx, fy, fz, en;
      glst.get_ef(fx, fy, fz, en);
      for (unsigned i = 0; i < natom; i++) energy += en.h_array()[i];
      energy *= 0.5;
      if (forces && every && s % every == 0) {
        std::fwrite(&s, sizeof(unsigned), 1, forces);
        std::fwrite(&natom, sizeof(unsigned), 1, forces);
        for (auto *c : {&fx, &fy, &fz, &en}) std::fwrite(c->h_array().data(), sizeof(double), natom, forces);
      }
    }
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
      std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err));
      return 3;
    }
    const double div = iters > 0 ? iters : 1;
    ms_host /= div;
    ms_ev /= div;
    std::fwrite(&natom, sizeof(unsigned), 1, out);
    std::fwrite(&K, sizeof(unsigned), 1, out);
    std::fwrite(&ms_host, sizeof(double), 1, out);
    std::fwrite(&ms_ev, sizeof(double), 1, out);
    std::fwrite(&energy, sizeof(double), 1, out);
  }
  return 0;
}

int main(int argc, char **argv) {
  // --batch list.bin out.bin float|double iterations [forces.bin every]
  if ((argc == 6 || argc == 8) && std::string(argv[1]) == "--batch") {
    FILE *in = std::fopen(argv[2], "rb");
    if (!in) return 2;
    FILE *out = std::fopen(argv[3], "wb");
    if (!out) return 2;
    FILE *forces = nullptr;
    unsigned every = 0;
    if (argc == 8) {
      forces = std::fopen(argv[6], "wb");
      if (!forces) return 2;
      every = (unsigned)std::atoi(argv[7]);
    }
    unsigned nsys = 0;
    if (std::fread(&nsys, sizeof(unsigned), 1, in) != 1) return 2;
    int rc = 0;
    try {
      rc = std::string(argv[4]) == "float"
               ? run_batch<float>(in, out, nsys, std::atoi(argv[5]), forces, every)
               : run_batch<double>(in, out, nsys, std::atoi(argv[5]), forces, every);
    } catch (const std::exception &e) {
      std::fprintf(stderr, "reference threw: %s\n", e.what());
      rc = 4;
    }
    std::fclose(in);
    std::fclose(out);
    if (forces) std::fclose(forces);
    return rc;
  }
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s in.bin out.bin float|double iterations\n",
                 argv[0]);
    return 1;
  }
  FILE *f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  unsigned natom = 0;
  double tol = 0, box[3] = {0, 0, 0}, rcut = 0;
  if (std::fread(&natom, sizeof(unsigned), 1, f) != 1) return 2;
  if (std::fread(&tol, sizeof(double), 1, f) != 1) return 2;
  if (std::fread(box, sizeof(double), 3, f) != 3) return 2;
  if (std::fread(&rcut, sizeof(double), 1, f) != 1) return 2;
  std::vector<double> x(natom), y(natom), z(natom), q(natom);
  for (auto *v : {&x, &y, &z, &q})
    if (std::fread(v->data(), sizeof(double), natom, f) != natom) return 2;
  std::fclose(f);
  const int iters = std::atoi(argv[4]);
  try {
    if (std::string(argv[3]) == "float")
      return run<float>(argv[2], natom, tol, box, rcut, x, y, z, q, iters);
    return run<double>(argv[2], natom, tol, box, rcut, x, y, z, q, iters);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "reference threw: %s\n", e.what());
    return 4;
  }
}
