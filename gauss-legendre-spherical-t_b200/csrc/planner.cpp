// Host planning for GLST (FP64).  Each function names the reference step it
// must agree with: the node set has to be identical to the reference's for
// the same tol/box/cutoff and the same t-design files, so the order of the
// arithmetic below follows the reference's where it affects rounding.
#include "planner.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <dirent.h>
#include <fstream>
#include <limits>
#include <mutex>
#include <sys/stat.h>
#include <tuple>

#include "glst_c.h"

namespace glst {

static const double kEps = std::numeric_limits<double>::epsilon();
static const double kPi = 3.14159265358979323846;

// ------------------------------------------------------------ t-design store
std::shared_ptr<TDesignStore> TDesignStore::open(const std::string &path) {
  auto s = std::make_shared<TDesignStore>();
  s->path_ = path;
  struct stat st;
  if (stat(path.c_str(), &st) != 0)
    throw PlanError{GLST_ERR_TDESIGN, "t-design path not found: " + path};
  if (S_ISDIR(st.st_mode)) {
    // Reference layout: ".../<anything>TTT.NNNNN" (src/cubature.cu:442-459).
    s->is_dir_ = true;
    DIR *d = opendir(path.c_str());
    if (!d) throw PlanError{GLST_ERR_TDESIGN, "cannot list " + path};
    while (dirent *e = readdir(d)) {
      std::string name = e->d_name;
      if (name == "." || name == "..") continue;
      std::string full = path + (path.back() == '/' ? "" : "/") + name;
      if (full.size() < 9 || full[full.size() - 6] != '.') continue;
      char *end = nullptr;
      std::string ts = full.substr(full.size() - 9, 3);
      std::string ns = full.substr(full.size() - 5, 5);
      unsigned long t = std::strtoul(ts.c_str(), &end, 10);
      if (*end) continue;
      unsigned long nn = std::strtoul(ns.c_str(), &end, 10);
      if (*end) continue;
      if (!s->files_.count((unsigned)t)) {
        s->files_[(unsigned)t] = full;
        s->file_m_[(unsigned)t] = (unsigned)(nn / 2);
      }
    }
    closedir(d);
    return s;
  }
  std::ifstream f(path, std::ios::binary);
  std::vector<char> buf((std::istreambuf_iterator<char>(f)),
                        std::istreambuf_iterator<char>());
  if (buf.size() < 12 || std::memcmp(buf.data(), "GLSTTD01", 8) != 0)
    throw PlanError{GLST_ERR_TDESIGN, "not a t-design store: " + path};
  uint32_t count;
  std::memcpy(&count, buf.data() + 8, 4);
  size_t off = 12;
  for (uint32_t i = 0; i < count; i++) {
    if (off + 20 > buf.size())
      throw PlanError{GLST_ERR_TDESIGN, "truncated t-design store: " + path};
    uint32_t t, m;
    std::memcpy(&t, buf.data() + off, 4);
    std::memcpy(&m, buf.data() + off + 4, 4);
    off += 20;
    if (off + 24ull * m > buf.size())
      throw PlanError{GLST_ERR_TDESIGN, "truncated t-design store: " + path};
    std::vector<double> v(3ull * m);
    std::memcpy(v.data(), buf.data() + off, 24ull * m);
    off += 24ull * m;
    s->cache_[t] = std::move(v);
  }
  return s;
}

const std::vector<double> *TDesignStore::get(unsigned t) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = cache_.find(t);
  if (it != cache_.end()) return &it->second;
  if (!is_dir_) return nullptr;
  auto f = files_.find(t);
  if (f == files_.end()) return nullptr;
  // Only the first N/2 lines: one point of each antipodal pair
  // (src/cubature.cu:423-439, :452); three 25-character columns per line.
  const unsigned m = file_m_[t];
  std::ifstream in(f->second);
  if (!in) return nullptr;
  std::vector<double> v(3ull * m);
  std::string line;
  for (unsigned i = 0; i < m; i++) {
    if (!std::getline(in, line) || line.size() < 75) return nullptr;
    v[3ull * i + 0] = std::stod(line.substr(0, 25));
    v[3ull * i + 1] = std::stod(line.substr(25, 25));
    v[3ull * i + 2] = std::stod(line.substr(50, 25));
  }
  return &(cache_[t] = std::move(v));
}

// ------------------------------------------------------------ erfc inverse
// Newton on 1 - erf(x) - y from x = 0 (src/glst_force.cu:1616-1640).
double erfc_inverse(double y, double tol) {
  const double two_over_sqrtpi = 2.0 / std::sqrt(kPi);
  double x = 0.0;
  double err = std::numeric_limits<double>::max();
  for (unsigned long long it = 0; it < 100000000ull; it++) {
    err = 1.0 - std::erf(x) - y;
    if (std::abs(err) < tol) break;
    const double slope = -std::exp(-x * x) * two_over_sqrtpi;
    x -= err / slope;
  }
  if (!(std::abs(err) < tol))
    throw PlanError{GLST_ERR_NO_CONVERGENCE, "inverse of erfc not found"};
  return x;
}

// ------------------------------------------------------------ Legendre
static void legendre(double &p, double &dp, double x, unsigned n) {
  // Three-term recurrence for P_n and P_n' (src/cubature.cu:161-193).
  if (n == 0) { p = 1.0; dp = 0.0; return; }
  if (n == 1) { p = x; dp = 1.0; return; }
  double pm = 1.0, pc = x, pn = 0.0, dc = 1.0, dn = 0.0;
  for (unsigned i = 1; i < n; i++) {
    const double a1 = static_cast<double>(i) + 1.0;
    const double a2 = 2.0 * static_cast<double>(i) + 1.0;
    pn = (a2 * x * pc - static_cast<double>(i) * pm) / a1;
    dn = a1 * pc + x * dc;
    pm = pc;
    pc = pn;
    dc = dn;
  }
  p = pn;
  dp = dn;
}

static double polish_root(double x, unsigned n) {
  // At most 10 Newton steps; stop when the step or its change is below eps
  // (src/cubature.cu:216-238).
  double p = 1.0, dp = 0.0, step = 0.0, prev = -1.0;
  for (int i = 0; i < 10; i++) {
    legendre(p, dp, x, n);
    prev = step;
    step = p / dp;
    if (std::isnan(step)) step = 0.0;
    x -= step;
    if (std::abs(step) < kEps) break;
    if (std::abs(step - prev) < kEps) break;
  }
  return x;
}

// Walk x forward by dx until P' changes sign (an extremum was passed).
static void walk_past_extremum(double &x, double dx, unsigned n) {
  double p0, d0, p1, d1;
  for (int i = 0; i < 10; i++) {
    legendre(p0, d0, x, n);
    x += dx;
    legendre(p1, d1, x, n);
    if (d0 * d1 < 0.0) return;
  }
}

// Walk x forward by dx until |P| stops decreasing; leave x at the smaller one.
static void walk_to_minimum(double &x, double dx, unsigned n) {
  double p0, d0, p1, d1;
  for (int i = 0; i < 10; i++) {
    legendre(p0, d0, x, n);
    x += dx;
    legendre(p1, d1, x, n);
    if (std::abs(p0) < std::abs(p1)) {
      x -= dx;
      return;
    }
  }
}

// Non-negative roots of P_n in increasing order (src/cubature.cu:240-351).
std::vector<double> gauss_legendre_roots(unsigned n) {
  std::vector<double> roots;
  if (n == 0) throw PlanError{GLST_ERR_INVALID_ARG, "no roots for n == 0"};
  if (n == 1) return {0.0};
  if (n == 2) return {1.0 / std::sqrt(3.0)};
  const unsigned m = (n % 2 == 0) ? n / 2 : (n + 1) / 2;
  double dx = 0.1 / static_cast<double>(m + 1);
  double x = dx;
  if (n % 2 == 1) {
    roots.push_back(0.0);
    walk_past_extremum(x, dx, n);
  }
  walk_to_minimum(x, dx, n);
  double r0 = polish_root(x, n);
  roots.push_back(r0);
  unsigned found = (n % 2 == 0) ? 1 : 2;
  x = r0;
  dx = (n % 2 == 0) ? 0.2 * r0 : 0.1 * r0;
  while (found < m) {
    walk_past_extremum(x, dx, n);
    walk_to_minimum(x, dx, n);
    const double r1 = polish_root(x, n);
    roots.push_back(r1);
    x = r1;
    dx = 0.1 * (r1 - r0);
    r0 = r1;
    found++;
  }
  return roots;
}

static std::vector<double> gauss_legendre_weights(const std::vector<double> &xs,
                                                  unsigned n) {
  // w = 2 / ((1 - x^2) P_n'(x)^2) (src/cubature.cu:195-214).
  std::vector<double> w;
  for (double x : xs) {
    double p, dp;
    legendre(p, dp, x, n);
    w.push_back(2.0 / ((1.0 - x * x) * dp * dp));
  }
  return w;
}

// Smallest even GL degree whose radial rule reproduces (pi/2) erf(alpha d)
// within (pi/2) d tol (src/cubature.cu:353-402).
static unsigned select_gl(std::vector<double> &xs, std::vector<double> &ws,
                          double tol, double dist, double alpha, double zcut) {
  const double target = 0.5 * kPi * std::erf(alpha * dist);
  const double bound = 0.5 * kPi * dist * tol;
  for (unsigned deg = 2; deg <= 324; deg += 2) {
    std::vector<double> x = gauss_legendre_roots(deg);
    std::vector<double> w = gauss_legendre_weights(x, deg);
    const unsigned i0 = (deg % 2 == 0) ? 0 : 1;
    double s = (deg % 2 == 0) ? 0.0 : alpha * dist * zcut * w[0];
    for (size_t i = i0; i < x.size(); i++) {
      const double v = std::exp(-zcut * zcut * x[i] * x[i]) *
                       std::sin(2.0 * alpha * dist * zcut * x[i]) / x[i];
      s += w[i] * v;
    }
    if (std::abs(s - target) < bound) {
      xs = x;
      ws = w;
      return deg;
    }
  }
  throw PlanError{GLST_ERR_NO_CONVERGENCE,
                  "suitable Gauss-Legendre quadrature could not be found"};
}

// t-design degree: walk degrees t = 2n+1 upward from n0 = |xs|/2 until the
// cubature reproduces erf(alpha d)/d within tol for r along x, then y, then z
// (src/cubature.cu:461-523).  Returns the last design read.
static unsigned select_tdesign(const std::vector<double> *&design,
                               TDesignStore &store, unsigned gl_deg,
                               const std::vector<double> &xs,
                               const std::vector<double> &ws, double tol,
                               double dist, double alpha, double zcut) {
  const double zc2 = zcut * zcut;
  const double target = std::erf(alpha * dist) / dist;
  unsigned n0 = static_cast<unsigned>(xs.size()) / 2;
  int nmin = -1;
  double dmin = std::numeric_limits<double>::max();
  const unsigned i0 = (gl_deg % 2 == 0) ? 0 : 1;
  unsigned t_last = 0;
  design = nullptr;
  for (int axis = 0; axis < 3; axis++) {
    for (unsigned n = n0; n < 162; n++) {
      const unsigned t = 2 * n + 1;
      const std::vector<double> *sm = store.get(t);
      if (!sm) {
        char b[160];
        std::snprintf(b, sizeof b,
                      "spherical t-design of degree %u not found in %s", t,
                      store.path().c_str());
        throw PlanError{GLST_ERR_TDESIGN, b};
      }
      design = sm;
      t_last = t;
      const size_t m = sm->size() / 3;
      double s = 0.0;
      for (size_t i = i0; i < xs.size(); i++) {
        const double coef = 2.0 * alpha * zcut * dist * xs[i];
        double v = 0.0;
        for (size_t k = 0; k < m; k++) v += std::cos(coef * (*sm)[3 * k + axis]);
        const double x2 = xs[i] * xs[i];
        s += ws[i] * std::exp(-zc2 * x2) * v;
      }
      s *= (4.0 * alpha * zcut / (kPi * static_cast<double>(m)));
      if (gl_deg % 2 == 1) s += 2.0 * alpha * zcut * ws[0] / kPi;
      const double err = std::abs(s - target);
      if (err < dmin) {
        dmin = err;
        nmin = static_cast<int>(n);
      }
      if (err < tol) {
        n0 = n;
        nmin = -2;
        break;
      }
    }
  }
  if (nmin > 0)
    throw PlanError{GLST_ERR_NO_CONVERGENCE,
                    "suitable t-design could not be found"};
  return t_last;
}

// The rules of a group depend only on (tol, rmax, alpha, zcut) and the store:
// cells of the same edge give the same first groups on every grid, so the
// (costly) selection is kept per parameter set.  Same arithmetic either way.
struct RuleKey {
  double tol, dist, alpha, zcut;
  const TDesignStore *store;
  bool operator<(const RuleKey &o) const {
    return std::tie(tol, dist, alpha, zcut, store) < std::tie(o.tol, o.dist, o.alpha, o.zcut, o.store);
  }
};
struct Rules {
  unsigned gl_degree = 0, t_degree = 0;
  std::vector<double> xs, ws;
  const std::vector<double> *design = nullptr;
};
static std::mutex g_rule_mu;
static std::map<RuleKey, Rules> g_rule_cache;

static void select_rules(GroupPlan &g, std::vector<double> &xs, std::vector<double> &ws,
                         const std::vector<double> *&design, TDesignStore &store, double tol) {
  const RuleKey key{tol, g.rmax, g.alpha, g.zcut, &store};
  {
    std::lock_guard<std::mutex> lk(g_rule_mu);
    auto it = g_rule_cache.find(key);
    if (it != g_rule_cache.end()) {
      g.gl_degree = it->second.gl_degree;
      g.t_degree = it->second.t_degree;
      xs = it->second.xs;
      ws = it->second.ws;
      design = it->second.design;
      return;
    }
  }
  g.gl_degree = select_gl(xs, ws, tol, g.rmax, g.alpha, g.zcut);
  g.t_degree = select_tdesign(design, store, g.gl_degree, xs, ws, tol, g.rmax, g.alpha, g.zcut);
  std::lock_guard<std::mutex> lk(g_rule_mu);
  if (g_rule_cache.size() > 1024) g_rule_cache.clear();
  g_rule_cache[key] = Rules{g.gl_degree, g.t_degree, xs, ws, design};
}

struct PlanKey {
  double tol;
  int ct_float;
  uint32_t n[3];
  double cell_dim;
  const TDesignStore *store;
  bool operator<(const PlanKey &o) const {
    return std::tie(tol, ct_float, n[0], n[1], n[2], cell_dim, store) <
           std::tie(o.tol, o.ct_float, o.n[0], o.n[1], o.n[2], o.cell_dim, o.store);
  }
};
static std::mutex g_plan_mu;
static std::map<PlanKey, Plan> g_plan_cache;

double rcut_from_ncell(const double box[3], const uint32_t ncell[3]) {
  // rcut = min(L/n) (src/glst_force.cu:80-95).
  const double rx = box[0] / static_cast<double>(ncell[0]);
  const double ry = box[1] / static_cast<double>(ncell[1]);
  const double rz = box[2] / static_cast<double>(ncell[2]);
  double r = rx;
  r = (ry < r) ? ry : r;
  r = (rz < r) ? rz : r;
  return r;
}

Plan make_plan(uint32_t natom, double tol, const double box[3], double rcut,
               int ct_float, TDesignStore &store) {
  if (!(tol > 0.0) || !(rcut > 0.0) || !(box[0] > 0.0) || !(box[1] > 0.0) ||
      !(box[2] > 0.0))
    throw PlanError{GLST_ERR_INVALID_ARG, "tol, rcut and box must be > 0"};
  Plan p;
  p.natom = natom;
  p.tol = tol;
  p.ct_float = ct_float;
  for (int a = 0; a < 3; a++) p.box[a] = box[a];

  // Cell grid in CT (src/glst_force.cu:223-241).
  if (ct_float) {
    const float l = static_cast<float>(rcut);
    for (int a = 0; a < 3; a++) {
      const float L = static_cast<float>(box[a]);
      unsigned n = static_cast<unsigned>(L / l);
      if (static_cast<float>(n) * l < L) n++;
      p.n[a] = n;
    }
    p.cell_dim = static_cast<double>(l);
  } else {
    const double l = rcut;
    for (int a = 0; a < 3; a++) {
      unsigned n = static_cast<unsigned>(box[a] / l);
      if (static_cast<double>(n) * l < box[a]) n++;
      p.n[a] = n;
    }
    p.cell_dim = l;
  }
  const uint64_t nc = (uint64_t)p.n[0] * p.n[1] * p.n[2];
  if (nc == 0 || nc > 0xFFFFFFFFull)
    throw PlanError{GLST_ERR_SIZE, "cell grid too large"};
  p.ncell = static_cast<uint32_t>(nc);
  p.has_far = p.n[0] > 2 && p.n[1] > 2 && p.n[2] > 2;

  // The groups and the cubature depend only on (tol, CT, grid, cell edge,
  // t-design source), not on natom or the exact box: reuse earlier plans.
  PlanKey key{tol, ct_float, {p.n[0], p.n[1], p.n[2]}, p.cell_dim, &store};
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = g_plan_cache.find(key);
    if (it != g_plan_cache.end()) {
      const Plan &c = it->second;
      p.groups = c.groups;
      p.kx = c.kx;
      p.ky = c.ky;
      p.kz = c.kz;
      p.w = c.w;
      p.group = c.group;
      return p;
    }
  }

  // Alpha groups (src/glst_force.cu:1643-1724).  Cells are cubes, so the
  // reference's lmin and lmax are both the cell edge.
  {
    int width = 1, tot = 0;
    int remain = static_cast<int>(std::max(p.n[0], std::max(p.n[1], p.n[2]))) - 2;
    const double lmin = p.cell_dim, lmax = p.cell_dim;
    while (remain >= 0) {
      GroupPlan g;
      g.width = static_cast<unsigned>(width);
      const double rmin0 = lmin * static_cast<double>(tot + 1);
      g.rmax = std::sqrt(3.0) * (rmin0 + lmax * static_cast<double>(width + 1));
      g.alpha = erfc_inverse(tol * rmin0, kEps) / rmin0;
      g.zcut = erfc_inverse(0.5 * std::sqrt(kPi) / g.alpha * tol, kEps);
      p.groups.push_back(g);
      remain -= width;
      tot += width;
      if (remain < 1) break;
      const int w1 = 2 * width, w2 = 6 * width;
      if (remain <= w1)
        width = remain;
      else if (w1 < remain && remain < w2)
        width = remain / 2;
      else
        width = w1;
    }
    for (size_t gi = 0; gi < p.groups.size(); gi++) {
      p.groups[gi].r_in = (gi == 0) ? 1u : p.groups[gi - 1].r_out;
      p.groups[gi].r_out = p.groups[gi].r_in + p.groups[gi].width;
    }
  }

  // Cubature per group (src/cubature.cu:100-159): GL radial rule, then the
  // t-design, then nodes k = 2 alpha zcut x_i s_j and equal weights.
  for (size_t gi = 0; gi < p.groups.size(); gi++) {
    GroupPlan &g = p.groups[gi];
    std::vector<double> xs, ws;
    const std::vector<double> *sm = nullptr;
    select_rules(g, xs, ws, sm, store, tol);
    const size_t m = sm->size() / 3;
    g.n_radial = static_cast<unsigned>(xs.size());
    g.n_dir = static_cast<unsigned>(m);
    g.dirs = *sm;
    for (size_t i = 0; i < xs.size(); i++) g.kappa.push_back(2.0 * g.alpha * g.zcut * xs[i]);
    const double zc2 = g.zcut * g.zcut;
    for (size_t i = 0; i < xs.size(); i++) {
      for (size_t j = 0; j < m; j++) {
        p.kx.push_back(2.0 * g.alpha * g.zcut * xs[i] * (*sm)[3 * j + 0]);
        p.ky.push_back(2.0 * g.alpha * g.zcut * xs[i] * (*sm)[3 * j + 1]);
        p.kz.push_back(2.0 * g.alpha * g.zcut * xs[i] * (*sm)[3 * j + 2]);
        p.w.push_back(4.0 * g.alpha * g.zcut * ws[i] *
                      std::exp(-zc2 * xs[i] * xs[i]) /
                      (kPi * static_cast<double>(m)));
        p.group.push_back(static_cast<uint32_t>(gi));
      }
    }
  }
  if (p.kx.size() > 0xFFFFFFFFull)
    throw PlanError{GLST_ERR_SIZE, "too many cubature nodes"};
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    if (g_plan_cache.size() > 256) g_plan_cache.clear();
    g_plan_cache.emplace(key, p);
  }
  return p;
}

}  // namespace glst
