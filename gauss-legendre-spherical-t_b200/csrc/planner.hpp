// Host-side planning for one GLST system: cell grid, alpha groups and the
// cubature node set.  All FP64, as the reference's host code; see planner.cpp
// for the reference file:line each step follows.
#pragma once

#include <cstdint>
#include <map>
#include <mutex>
#include <memory>
#include <string>
#include <vector>

namespace glst {

struct PlanError {
  int status;  // glst_status
  std::string msg;
};

// Antipodal spherical t-designs keyed by degree; only the free half (m unit
// vectors) is kept, the full design being {p} U {-p}.
class TDesignStore {
 public:
  // `path`: a binary store (magic GLSTTD01) or a directory in the
  // reference's layout (files ssTTT.NNNNN).
  static std::shared_ptr<TDesignStore> open(const std::string &path);
  // Returns nullptr when the degree is not available.
  const std::vector<double> *get(unsigned t);  // 3*m doubles, xyz interleaved
  const std::string &path() const { return path_; }

 private:
  std::string path_;
  bool is_dir_ = false;
  std::map<unsigned, std::string> files_;  // degree -> file (dir layout)
  std::map<unsigned, unsigned> file_m_;    // degree -> N/2 (dir layout)
  std::map<unsigned, std::vector<double>> cache_;  // node-based: pointers stay valid
  std::mutex mu_;  // get() fills cache_ lazily (directory layout) from any thread
};

struct GroupPlan {
  unsigned width = 0;
  double rmax = 0, alpha = 0, zcut = 0;
  unsigned r_in = 0, r_out = 0;
  unsigned gl_degree = 0, t_degree = 0;
  unsigned n_radial = 0, n_dir = 0;
  std::vector<double> kappa;  // radial scales 2 alpha zcut x_i (n_radial)
  std::vector<double> dirs;   // unit directions s_j, xyz interleaved (3 n_dir)
};

struct Plan {
  uint32_t natom = 0;
  double tol = 0;
  double box[3] = {0, 0, 0};
  int ct_float = 0;
  uint32_t n[3] = {0, 0, 0};
  uint32_t ncell = 0;
  double cell_dim = 0;  // CT value widened to double
  bool has_far = false;
  std::vector<GroupPlan> groups;
  // Node set in the reference's order, FP64 (pre-CT-rounding).
  std::vector<double> kx, ky, kz, w;
  std::vector<uint32_t> group;
  uint32_t K() const { return static_cast<uint32_t>(kx.size()); }
};

// Throws PlanError.
Plan make_plan(uint32_t natom, double tol, const double box[3], double rcut,
               int ct_float, TDesignStore &store);
double rcut_from_ncell(const double box[3], const uint32_t ncell[3]);

// Exposed for tests of the numerics set-up.
double erfc_inverse(double y, double tol);
std::vector<double> gauss_legendre_roots(unsigned n);

}  // namespace glst
