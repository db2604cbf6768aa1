// lp_oracle.cpp - FP64 CPU oracle of the litter-physics MLS-MPM research step.
//
// TEST INFRASTRUCTURE ONLY (checker and CPU baseline, never the product path).
//
// This file restates, in C++, the reference's Rust algorithm step by step so that the
// CUDA product can be checked against it on identical seeded inputs.  Floating-point
// expressions keep the reference's evaluation order (nalgebra evaluates small
// matrix/vector products as left-to-right sums of products, without fused multiply-add;
// this file is compiled with -ffp-contract=off for the same reason), so that FP64
// results can be pinned against the reference's own published values.  Each function
// cites the reference file:line it follows (paths inside nredd/litter-physics).
//
// Parallel loops (OpenMP) are exactly the ones the reference runs with rayon
// (grid update, grid-to-particle, pellet coupling); each writes per-element results that
// are committed serially in index order, so the output does not depend on thread count.
//
// Labelled extensions (defaults reproduce the reference exactly):
//   - Tait EOS exponent for the liquid (gamma == 1 keeps K (1/J - 1) bit for bit);
//   - per-face wall friction / sticky faces (face_mode_enabled == 0 keeps one mu);
//   - per-particle yield stress drawn after placement (yield_random == 0: material value);
//   - configurable HB return tolerance (0 -> 1e-12).

#include "lp_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------- small linear algebra
struct V3 {
  double v[3];
  double& operator[](int i) { return v[i]; }
  double operator[](int i) const { return v[i]; }
};
struct M3 {
  double a[3][3];  // row-major a[row][col]
};

inline V3 v3(double x, double y, double z) { return V3{{x, y, z}}; }
inline V3 zero3() { return v3(0, 0, 0); }
inline V3 add(const V3& a, const V3& b) { return v3(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
inline V3 sub(const V3& a, const V3& b) { return v3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
inline V3 mul(const V3& a, double s) { return v3(a[0] * s, a[1] * s, a[2] * s); }
inline V3 divs(const V3& a, double s) { return v3(a[0] / s, a[1] / s, a[2] / s); }
inline V3 neg(const V3& a) { return v3(-a[0], -a[1], -a[2]); }
// nalgebra 3-vector dot: (a0 b0 + a1 b1) + a2 b2
inline double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double norm2(const V3& a) { return dot(a, a); }
inline double norm(const V3& a) { return std::sqrt(norm2(a)); }
inline V3 cross(const V3& a, const V3& b) {
  return v3(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
inline bool finite3(const V3& a) { return std::isfinite(a[0]) && std::isfinite(a[1]) && std::isfinite(a[2]); }

inline M3 mzero() {
  M3 m;
  std::memset(&m, 0, sizeof(m));
  return m;
}
inline M3 mident() {
  M3 m = mzero();
  m.a[0][0] = m.a[1][1] = m.a[2][2] = 1.0;
  return m;
}
inline M3 mdiag(const V3& d) {
  M3 m = mzero();
  for (int i = 0; i < 3; ++i) m.a[i][i] = d[i];
  return m;
}
inline M3 madd(const M3& x, const M3& y) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.a[i][j] = x.a[i][j] + y.a[i][j];
  return r;
}
inline M3 msub(const M3& x, const M3& y) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.a[i][j] = x.a[i][j] - y.a[i][j];
  return r;
}
inline M3 mscale(const M3& x, double s) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.a[i][j] = x.a[i][j] * s;
  return r;
}
inline M3 mT(const M3& x) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.a[i][j] = x.a[j][i];
  return r;
}
// c_ij = (x_i0 y_0j + x_i1 y_1j) + x_i2 y_2j
inline M3 mmul(const M3& x, const M3& y) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.a[i][j] = x.a[i][0] * y.a[0][j] + x.a[i][1] * y.a[1][j] + x.a[i][2] * y.a[2][j];
  return r;
}
inline V3 mvec(const M3& x, const V3& v) {
  return v3(x.a[0][0] * v[0] + x.a[0][1] * v[1] + x.a[0][2] * v[2],
            x.a[1][0] * v[0] + x.a[1][1] * v[1] + x.a[1][2] * v[2],
            x.a[2][0] * v[0] + x.a[2][1] * v[1] + x.a[2][2] * v[2]);
}
// nalgebra Matrix3::determinant
inline double mdet(const M3& m) {
  const double m11 = m.a[0][0], m12 = m.a[0][1], m13 = m.a[0][2];
  const double m21 = m.a[1][0], m22 = m.a[1][1], m23 = m.a[1][2];
  const double m31 = m.a[2][0], m32 = m.a[2][1], m33 = m.a[2][2];
  const double minor_m12_m23 = m22 * m33 - m32 * m23;
  const double minor_m11_m23 = m21 * m33 - m31 * m23;
  const double minor_m11_m22 = m21 * m32 - m31 * m22;
  return m11 * minor_m12_m23 - m12 * minor_m11_m23 + m13 * minor_m11_m22;
}
// nalgebra Frobenius norm_squared: column-major sequential sum
inline double mnorm2(const M3& m) {
  double r = 0.0;
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) r += m.a[i][j] * m.a[i][j];
  return r;
}
inline bool mfinite(const M3& m) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      if (!std::isfinite(m.a[i][j])) return false;
  return true;
}
inline double rust_signum(double x) {
  if (std::isnan(x)) return x;
  return std::signbit(x) ? -1.0 : 1.0;
}
inline double midpoint(double a, double b) { return (a + b) / 2.0; }

// ---------------------------------------------------------------- rng.rs:35-47
struct SplitMix64 {
  uint64_t state;
  uint64_t next_u64() {
    state += 0x9E3779B97F4A7C15ull;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double next_unit() { return (double)(next_u64() >> 11) * (1.0 / (double)(1ull << 53)); }
};

// ---------------------------------------------------------------- grid.rs
struct Layout {
  double spacing;
  int64_t cells[3];
  int64_t nodes[3];
  int64_t node_count() const { return nodes[0] * nodes[1] * nodes[2]; }
  V3 extents() const {
    return v3((double)cells[0] * spacing, (double)cells[1] * spacing, (double)cells[2] * spacing);
  }
  int64_t index(int64_t i, int64_t j, int64_t k) const { return (i * nodes[1] + j) * nodes[2] + k; }
  V3 node_position(int64_t i, int64_t j, int64_t k) const {
    return v3(((double)i - 1.0) * spacing, ((double)j - 1.0) * spacing, ((double)k - 1.0) * spacing);
  }
  void coords(int64_t index, int64_t& i, int64_t& j, int64_t& k) const {
    k = index % nodes[2];
    int64_t rest = index / nodes[2];
    j = rest % nodes[1];
    i = rest / nodes[1];
  }
  // grid.rs:203-211; returns 0 when free, +1 low face, -1 high face
  double wall_side(int axis, int64_t coord) const {
    if (coord <= 1) return 1.0;
    if (coord > cells[axis]) return -1.0;
    return 0.0;
  }
};

// grid.rs:105-154
bool make_layout(const double domain[3], double spacing, uint64_t max_nodes, Layout& out, std::string& err) {
  if (!(std::isfinite(spacing) && spacing > 0.0)) {
    err = "`grid_spacing_m` must be positive and finite";
    return false;
  }
  for (int axis = 0; axis < 3; ++axis) {
    double extent = domain[axis];
    if (!(std::isfinite(extent) && extent > 0.0)) {
      err = "`domain_m` must be positive and finite";
      return false;
    }
    double ratio = extent / spacing;
    double rounded = std::round(ratio);
    uint64_t capn = max_nodes >= 3 ? max_nodes - 3 : 0;
    double cap = capn > 0xFFFFFFFFull ? (double)0xFFFFFFFFull : (double)capn;
    if (!std::isfinite(ratio) || rounded > cap) {
      err = "grid axis exceeds the node allocation cap";
      return false;
    }
    if (std::fabs(ratio - rounded) > 1e-6 * std::max(rounded, 1.0)) {
      err = "`domain_m` is not an integer multiple of `grid_spacing_m`";
      return false;
    }
    if (rounded < 2.0) {
      err = "`domain_m` must span at least two cells";
      return false;
    }
    out.cells[axis] = (int64_t)rounded;
  }
  for (int a = 0; a < 3; ++a) out.nodes[a] = out.cells[a] + 3;
  out.spacing = spacing;
  double total = (double)out.nodes[0] * (double)out.nodes[1] * (double)out.nodes[2];
  if (total > (double)max_nodes) {
    err = "grid would allocate too many nodes, exceeding the cap";
    return false;
  }
  return true;
}

struct Stencil {
  int64_t base[3];
  double w[3][3];
  double off[3][3];  // off[axis][o] = x_node - x_particle along axis
  double weight(int a, int b, int c) const { return w[0][a] * w[1][b] * w[2][c]; }
  V3 distance(int a, int b, int c) const { return v3(off[0][a], off[1][b], off[2][c]); }
};

// grid.rs:151-182
bool stencil_of(const Layout& L, const V3& x, Stencil& s) {
  for (int axis = 0; axis < 3; ++axis) {
    double scaled = x[axis] / L.spacing;
    double base_f = std::floor(scaled - 0.5);
    double padded = base_f + 1.0;
    if (std::isnan(padded) || padded < 0.0 || padded + 2.0 >= (double)L.nodes[axis]) return false;
    double fx = scaled - base_f;
    double a0 = 1.5 - fx, a1 = fx - 1.0, a2 = fx - 0.5;
    s.w[axis][0] = 0.5 * (a0 * a0);
    s.w[axis][1] = 0.75 - (a1 * a1);
    s.w[axis][2] = 0.5 * (a2 * a2);
    s.base[axis] = (int64_t)padded;
    for (int o = 0; o < 3; ++o) s.off[axis][o] = (fx - (double)o) * -L.spacing;
  }
  return true;
}

struct Grid {
  Layout layout;
  std::vector<double> mass;
  std::vector<V3> momentum;
  std::vector<V3> traction;       // total inward reaction per axis (grid.rs:291)
  std::vector<V3> traction_low;   // extension: per-side split (face mode only)
  std::vector<V3> traction_high;
  std::vector<int64_t> active;
  void init(const Layout& L) {
    layout = L;
    int64_t n = L.node_count();
    mass.assign(n, 0.0);
    momentum.assign(n, zero3());
    traction.assign(n, zero3());
    traction_low.assign(n, zero3());
    traction_high.assign(n, zero3());
    active.clear();
  }
  // grid.rs:243-250
  void clear() {
    for (int64_t i : active) {
      mass[i] = 0.0;
      momentum[i] = zero3();
      traction[i] = zero3();
      traction_low[i] = zero3();
      traction_high[i] = zero3();
    }
    active.clear();
  }
  // grid.rs:254-263
  void deposit(int64_t index, double m, const V3& p) {
    if (m == 0.0) return;
    if (mass[index] == 0.0) active.push_back(index);
    mass[index] += m;
    momentum[index] = add(momentum[index], p);
  }
  // grid.rs:279-295
  bool deposit_reaction(int64_t index, int axis, double inward, double inward_impulse, double& jump) {
    double m = mass[index];
    if (m <= 0.0) return false;
    double impulse = inward_impulse * inward;
    jump = impulse * (momentum[index][axis] / m + impulse / (2.0 * m));
    momentum[index][axis] += impulse;
    traction[index][axis] += inward_impulse;
    if (inward > 0) traction_low[index][axis] += inward_impulse;
    else traction_high[index][axis] += inward_impulse;
    return true;
  }
};

// ---------------------------------------------------------------- constitutive.rs
struct Material {
  int kind;
  double density, mu, lambda, bulk, yield, consistency, n, gamma;
};

Material mat_from(const lp_material& m) {
  return Material{m.kind, m.density, m.shear_modulus, m.lame_lambda, m.bulk_modulus, m.yield_stress,
                  m.consistency, m.flow_index, m.tait_gamma == 0.0 ? 1.0 : m.tait_gamma};
}
lp_material mat_to(const Material& m) {
  lp_material r;
  std::memset(&r, 0, sizeof(r));
  r.kind = m.kind;
  r.density = m.density;
  r.shear_modulus = m.mu;
  r.lame_lambda = m.lambda;
  r.bulk_modulus = m.bulk;
  r.yield_stress = m.yield;
  r.consistency = m.consistency;
  r.flow_index = m.n;
  r.tait_gamma = m.gamma;
  return r;
}
// constitutive.rs:146-167
Material paste(double density, double e, double nu, double ys, double k, double n) {
  double mu = e / (2.0 * (1.0 + nu));
  double lambda = e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  return Material{LP_PASTE, density, mu, lambda, lambda + 2.0 * mu / 3.0, ys, k, n, 1.0};
}
// constitutive.rs:180-197
Material paste_shear(double density, double e, double nu, double tys, double ks, double n) {
  double root3 = std::sqrt(3.0);
  return paste(density, e, nu, root3 * tys, std::pow(3.0, midpoint(1.0, n)) * ks, n);
}
// constitutive.rs:211-223
Material liquid(double density, double e, double nu, double visc) {
  double bulk = e / (3.0 * (1.0 - 2.0 * nu));
  return Material{LP_LIQUID, density, 0.0, 0.0, bulk, 0.0, visc, 1.0, 1.0};
}
// constitutive.rs:227-243
double wave_speed(const Material& m) {
  double modulus = m.kind == LP_PASTE ? m.lambda + 2.0 * m.mu : m.bulk;
  return std::sqrt(modulus / m.density);
}
double diffusivity(const Material& m) { return m.kind == LP_PASTE ? 0.0 : m.consistency / m.density; }

enum ConstErr { CE_OK = 0, CE_INVERTED, CE_EIGEN, CE_STRETCH, CE_NOT_CONVERGED, CE_NONFINITE };
const char* const_err_name(int e) {
  switch (e) {
    case CE_INVERTED: return "trial deformation gradient inverted";
    case CE_EIGEN: return "eigen-decomposition of trial Cauchy-Green tensor did not converge";
    case CE_STRETCH: return "degenerate elastic stretch";
    case CE_NOT_CONVERGED: return "Herschel-Bulkley return did not converge";
    case CE_NONFINITE: return "non-finite constitutive quantity";
  }
  return "ok";
}

struct ReturnSolution {
  double sigma, dep;
  int iterations;
};

// constitutive.rs:280-362 (tolerance configurable; reference value 1e-12)
int hb_return(double trial, double ys, double k, double n, double mu, double dt, double tol_rel,
              ReturnSolution& out) {
  double inputs[6] = {trial, ys, k, n, mu, dt};
  for (double v : inputs)
    if (!std::isfinite(v)) return CE_NONFINITE;
  double viscous_scale = 3.0 * mu * dt;
  if (trial <= ys) {
    out = {trial, 0.0, 0};
    return CE_OK;
  }
  if (k <= 0.0) {
    out = {ys, (trial - ys) / (3.0 * mu), 0};
    return CE_OK;
  }
  double exponent = 1.0 / n;
  auto residual = [&](double sigma) {
    double over = std::fmax((sigma - ys) / k, 0.0);
    return sigma - trial + viscous_scale * std::pow(over, exponent);
  };
  double lower = ys, upper = trial;
  double sigma = midpoint(lower, upper);
  double tolerance = tol_rel * std::fmax(trial, 1.0);
  double last = residual(sigma);
  for (int iteration = 1; iteration <= 200; ++iteration) {
    if (std::fabs(last) <= tolerance || (upper - lower) <= tolerance) {
      out = {sigma, (trial - sigma) / (3.0 * mu), iteration};
      return CE_OK;
    }
    if (last > 0.0) upper = sigma;
    else lower = sigma;
    double over = std::fmax((sigma - ys) / k, 0.0);
    double derivative = over > 0.0 ? 1.0 + viscous_scale * exponent * std::pow(over, exponent - 1.0) / k
                                   : std::numeric_limits<double>::infinity();
    double newton = sigma - last / derivative;
    sigma = (std::isfinite(newton) && newton > lower && newton < upper) ? newton : midpoint(lower, upper);
    last = residual(sigma);
    if (!std::isfinite(last)) return CE_NONFINITE;
  }
  return CE_NOT_CONVERGED;
}

// constitutive.rs:373-425
bool symmetric_eigen3(const M3& m, V3& values, M3& vectors) {
  if (!mfinite(m)) return false;
  // `0.5 * (m + m^T)`: scalar times the elementwise sum
  M3 d;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) d.a[i][j] = 0.5 * (m.a[i][j] + m.a[j][i]);
  M3 v = mident();
  double scale = std::fmax(mnorm2(d), std::numeric_limits<double>::min());
  const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = d.a[0][1] * d.a[0][1] + d.a[0][2] * d.a[0][2] + d.a[1][2] * d.a[1][2];
    if (off <= 1e-30 * scale) {
      values = v3(d.a[0][0], d.a[1][1], d.a[2][2]);
      vectors = v;
      return true;
    }
    for (auto& pq : pairs) {
      int p = pq[0], q = pq[1];
      double apq = d.a[p][q];
      if (apq == 0.0) continue;
      double theta = (d.a[q][q] - d.a[p][p]) / (2.0 * apq);
      double tangent = rust_signum(theta) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
      double cosine = 1.0 / std::sqrt(tangent * tangent + 1.0);
      double sine = tangent * cosine;
      for (int k = 0; k < 3; ++k) {
        double akp = d.a[k][p], akq = d.a[k][q];
        d.a[k][p] = cosine * akp - sine * akq;
        d.a[k][q] = sine * akp + cosine * akq;
      }
      for (int k = 0; k < 3; ++k) {
        double apk = d.a[p][k], aqk = d.a[q][k];
        d.a[p][k] = cosine * apk - sine * aqk;
        d.a[q][k] = sine * apk + cosine * aqk;
      }
      for (int k = 0; k < 3; ++k) {
        double vkp = v.a[k][p], vkq = v.a[k][q];
        v.a[k][p] = cosine * vkp - sine * vkq;
        v.a[k][q] = sine * vkp + cosine * vkq;
      }
    }
  }
  return false;
}

struct PasteUpdate {
  M3 deformation, kirchhoff;
  double dep, dissipation_density, equivalent;
  int iterations;
};

// constitutive.rs:456-531
int update_paste(const M3& trial, const Material& mat, double ys, double dt, double tol, PasteUpdate& out) {
  double det = mdet(trial);
  if (!std::isfinite(det)) return CE_NONFINITE;
  if (det <= 0.0) return CE_INVERTED;
  M3 b = mmul(trial, mT(trial));
  V3 eig;
  M3 u;
  if (!symmetric_eigen3(b, eig, u)) return CE_EIGEN;
  V3 stretches, hencky;
  for (int axis = 0; axis < 3; ++axis) {
    double s = std::sqrt(std::fmax(eig[axis], 0.0));
    if (!std::isfinite(s) || s < 1e-6) return CE_STRETCH;
    stretches[axis] = s;
    hencky[axis] = std::log(s);
  }
  double volumetric = hencky[0] + hencky[1] + hencky[2];
  double mean = volumetric / 3.0;
  V3 dev = v3(hencky[0] - mean, hencky[1] - mean, hencky[2] - mean);
  double mu = mat.mu;
  double dnorm = norm(dev);
  double trial_eq = std::sqrt(1.5) * 2.0 * mu * dnorm;
  double scale = 1.0, dep = 0.0, eq = trial_eq;
  int iterations = 0;
  if (trial_eq > ys && dnorm > 0.0) {
    ReturnSolution sol;
    int e = hb_return(trial_eq, ys, mat.consistency, mat.n, mu, dt, tol, sol);
    if (e != CE_OK) return e;
    scale = sol.sigma / trial_eq;
    dep = sol.dep;
    eq = sol.sigma;
    iterations = sol.iterations;
  }
  V3 dev_new = mul(dev, scale);
  V3 h_new = v3(dev_new[0] + mean, dev_new[1] + mean, dev_new[2] + mean);
  V3 ratio = v3(std::exp(h_new[0]) / stretches[0], std::exp(h_new[1]) / stretches[1],
                std::exp(h_new[2]) / stretches[2]);
  out.deformation = mmul(mmul(mmul(u, mdiag(ratio)), mT(u)), trial);
  double lv = mat.lambda * volumetric;
  V3 principal = v3(h_new[0] * (2.0 * mu) + lv, h_new[1] * (2.0 * mu) + lv, h_new[2] * (2.0 * mu) + lv);
  out.kirchhoff = mmul(mmul(u, mdiag(principal)), mT(u));
  if (!mfinite(out.kirchhoff)) return CE_NONFINITE;
  out.dep = dep;
  out.dissipation_density = eq * dep;
  out.equivalent = eq;
  out.iterations = iterations;
  return CE_OK;
}

struct LiquidUpdate {
  double j;
  M3 kirchhoff;
  double pressure;
};

// liquid pressure: constitutive.rs:593-595; Tait extension for gamma != 1
inline double liquid_pressure(const Material& m, double j) {
  if (m.gamma == 1.0) return m.bulk * (1.0 / j - 1.0);
  return m.bulk / m.gamma * (std::pow(j, -m.gamma) - 1.0);
}

// constitutive.rs:557-589
int update_liquid(double j, const M3& grad, const Material& m, double dt, LiquidUpdate& out) {
  double trace = grad.a[0][0] + grad.a[1][1] + grad.a[2][2];
  double nj = j * (1.0 + dt * trace);
  if (!std::isfinite(nj)) return CE_NONFINITE;
  if (nj <= 1e-6) return CE_INVERTED;
  double pressure = liquid_pressure(m, nj);
  M3 rate;
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) rate.a[i][k] = 0.5 * (grad.a[i][k] + grad.a[k][i]);
  double rtrace = rate.a[0][0] + rate.a[1][1] + rate.a[2][2];
  M3 dev = msub(rate, mscale(mident(), rtrace / 3.0));
  out.kirchhoff = madd(mscale(mident(), -pressure * nj), mscale(dev, 2.0 * m.consistency * nj));
  if (!mfinite(out.kirchhoff)) return CE_NONFINITE;
  out.j = nj;
  out.pressure = pressure;
  return CE_OK;
}

// ---------------------------------------------------------------- particles.rs
struct Particles {
  std::vector<uint32_t> id;
  std::vector<V3> x, v;
  std::vector<M3> C, F;
  std::vector<double> J;
  std::vector<M3> tau;
  std::vector<double> ep, m, V0, ys;  // ys: extension (per-particle yield)
  size_t size() const { return id.size(); }
  void push(const V3& pos, const V3& vel, double mass, double vol0, double yield) {
    id.push_back((uint32_t)id.size());
    x.push_back(pos);
    v.push_back(vel);
    C.push_back(mzero());
    F.push_back(mident());
    J.push_back(1.0);
    tau.push_back(mzero());
    ep.push_back(0.0);
    m.push_back(mass);
    V0.push_back(vol0);
    ys.push_back(yield);
  }
  double total_mass() const {
    double s = 0.0;
    for (double mm : m) s += mm;
    return s;
  }
  V3 linear_momentum() const {
    V3 acc = zero3();
    for (size_t i = 0; i < size(); ++i) acc = add(acc, mul(v[i], m[i]));
    return acc;
  }
  double kinetic_energy() const {
    double s = 0.0;
    for (size_t i = 0; i < size(); ++i) s += 0.5 * m[i] * norm2(v[i]);
    return s;
  }
  template <class T>
  static void apply(std::vector<T>& vals, const std::vector<size_t>& order) {
    std::vector<T> r;
    r.reserve(order.size());
    for (size_t i : order) r.push_back(vals[i]);
    vals.swap(r);
  }
  void permute(const std::vector<size_t>& order) {
    apply(id, order);
    apply(x, order);
    apply(v, order);
    apply(C, order);
    apply(F, order);
    apply(J, order);
    apply(tau, order);
    apply(ep, order);
    apply(m, order);
    apply(V0, order);
    apply(ys, order);
  }
  double remove_sorted(const std::vector<size_t>& idx) {
    if (idx.empty()) return 0.0;
    double removed = 0.0;
    for (size_t i : idx) removed += m[i];
    std::vector<size_t> keep;
    size_t k = 0;
    for (size_t i = 0; i < size(); ++i) {
      if (k < idx.size() && idx[k] == i) {
        ++k;
        continue;
      }
      keep.push_back(i);
    }
    permute(keep);
    return removed;
  }
};

// ---------------------------------------------------------------- rigid.rs
struct Quat {  // (i, j, k, w) like nalgebra coords
  double i, j, k, w;
};
inline Quat qmul(const Quat& a, const Quat& b) {
  return Quat{a.w * b.i + a.i * b.w + a.j * b.k - a.k * b.j, a.w * b.j - a.i * b.k + a.j * b.w + a.k * b.i,
              a.w * b.k + a.i * b.j - a.j * b.i + a.k * b.w, a.w * b.w - a.i * b.i - a.j * b.j - a.k * b.k};
}
// nalgebra UnitQuaternion * Vector3
inline V3 qrot(const Quat& q, const V3& r) {
  V3 qv = v3(q.i, q.j, q.k);
  V3 t = mul(cross(qv, r), 2.0);
  V3 c = cross(qv, t);
  return add(add(mul(t, q.w), c), r);
}
inline M3 qmatrix(const Quat& q) {
  double i = q.i, j = q.j, k = q.k, w = q.w;
  double ww = w * w, ii = i * i, jj = j * j, kk = k * k;
  double ij = i * j * 2.0, wk = w * k * 2.0, wj = w * j * 2.0, ik = i * k * 2.0, jk = j * k * 2.0, wi = w * i * 2.0;
  M3 m;
  m.a[0][0] = ww + ii - jj - kk;
  m.a[0][1] = ij - wk;
  m.a[0][2] = wj + ik;
  m.a[1][0] = wk + ij;
  m.a[1][1] = ww - ii + jj - kk;
  m.a[1][2] = jk - wi;
  m.a[2][0] = ik - wj;
  m.a[2][1] = wi + jk;
  m.a[2][2] = ww - ii - jj + kk;
  return m;
}
// nalgebra UnitQuaternion::from_scaled_axis via the quaternion exponential
inline Quat q_from_scaled_axis(const V3& axisangle) {
  V3 h = divs(axisangle, 2.0);
  double nn = norm2(h);
  double eps = std::numeric_limits<double>::epsilon();
  if (nn <= eps * eps) return Quat{0, 0, 0, 1};
  double w_exp = std::exp(0.0);
  double n = std::sqrt(nn);
  V3 nv = mul(h, w_exp * std::sin(n) / n);
  return Quat{nv[0], nv[1], nv[2], w_exp * std::cos(n)};
}

struct Contact {
  double k, e, mu;
  // rigid.rs:81-91
  double damping(double mass) const {
    double zeta;
    if (e <= 0.0) zeta = 1.0;
    else if (e >= 1.0) zeta = 0.0;
    else {
      double lg = std::log(e);
      zeta = -lg / std::sqrt(kPi * kPi + lg * lg);
    }
    return 2.0 * zeta * std::sqrt(k * mass);
  }
  double stable_dt(double mass) const { return 0.2 * std::sqrt(mass / k); }
};

struct WallContact {
  V3 impulse;
  double work;
  int contacts;
};

struct Pellet {
  double radius, length, mass;
  V3 inertia;
  V3 position;
  Quat q;
  V3 velocity;
  V3 L;
  std::vector<double> offsets;

  M3 rot() const { return qmatrix(q); }
  // rigid.rs:193-198
  V3 angular_velocity() const {
    M3 r = rot();
    V3 bm = mvec(mT(r), L);
    V3 bo = v3(bm[0] / inertia[0], bm[1] / inertia[1], bm[2] / inertia[2]);
    return mvec(r, bo);
  }
  V3 axis() const { return qrot(q, v3(1, 0, 0)); }
  std::vector<V3> centers() const {
    V3 ax = axis();
    std::vector<V3> c;
    for (double o : offsets) c.push_back(add(position, mul(ax, o)));
    return c;
  }
  // rigid.rs:212-230
  double signed_distance(const V3& p, V3& normal) const {
    V3 ax = axis();
    double best = std::numeric_limits<double>::infinity();
    V3 bn = v3(0, 0, 1);
    for (double o : offsets) {
      V3 c = add(position, mul(ax, o));
      V3 d = sub(p, c);
      double dist = norm(d);
      double phi = dist - radius;
      if (phi < best) {
        bn = dist > 1e-12 ? divs(d, dist) : v3(0, 0, 1);
        best = phi;
      }
    }
    normal = bn;
    return best;
  }
  V3 point_velocity(const V3& p) const { return add(velocity, cross(angular_velocity(), sub(p, position))); }
  void bounding_box(V3& lo, V3& hi) const {
    V3 ax = axis();
    double hs = 0.0;
    for (double o : offsets) hs = std::fmax(hs, std::fabs(o));
    V3 reach = add(mul(v3(std::fabs(ax[0]), std::fabs(ax[1]), std::fabs(ax[2])), hs), v3(radius, radius, radius));
    lo = sub(position, reach);
    hi = add(position, reach);
  }
  void apply_impulse(const V3& imp, const V3& ang) {
    velocity = add(velocity, divs(imp, mass));
    L = add(L, ang);
  }
  double kinetic_energy() const {
    V3 om = angular_velocity();
    return 0.5 * mass * norm2(velocity) + 0.5 * dot(om, L);
  }
  bool finite() const {
    return finite3(position) && finite3(velocity) && finite3(L) && std::isfinite(q.i) && std::isfinite(q.j) &&
           std::isfinite(q.k) && std::isfinite(q.w);
  }
  // rigid.rs:279-334; ef / et: pellet-bed sphere-contact force and torque (extension)
  WallContact integrate(double dt, const V3& g, const V3& ext, const Contact& c, const V3* ef = nullptr,
                        const V3* et = nullptr) {
    double damping = c.damping(mass);
    V3 force = zero3(), torque = zero3();
    WallContact led{zero3(), 0.0, 0};
    V3 omega = angular_velocity();
    for (const V3& center : centers()) {
      for (int axis = 0; axis < 3; ++axis) {
        const double faces[2][2] = {{0.0, 1.0}, {ext[axis], -1.0}};
        for (auto& f : faces) {
          double gap = (center[axis] - f[0]) * f[1];
          double pen = radius - gap;
          if (pen <= 0.0) continue;
          V3 normal = zero3();
          normal[axis] = f[1];
          V3 cp = sub(center, mul(normal, radius));
          V3 lever = sub(cp, position);
          V3 pv = add(velocity, cross(omega, lever));
          double ns = dot(pv, normal);
          double nf = std::fmax(c.k * pen - damping * ns, 0.0);
          V3 tang = sub(pv, mul(normal, ns));
          double ts = norm(tang);
          V3 ff = zero3();
          if (ts > 1e-12) {
            double limit = std::fmin(c.mu * nf, mass * ts / dt);
            ff = mul(divs(neg(tang), ts), limit);
          }
          V3 total = add(mul(normal, nf), ff);
          force = add(force, total);
          torque = add(torque, cross(lever, total));
          led.work += dot(total, pv) * dt;
          led.contacts += 1;
        }
      }
    }
    V3 impulse = mul(force, dt);
    led.impulse = impulse;
    V3 applied = ef ? mul(add(force, *ef), dt) : impulse;
    velocity = add(velocity, add(mul(g, dt), divs(applied, mass)));
    L = add(L, mul(et ? add(torque, *et) : torque, dt));
    position = add(position, mul(velocity, dt));
    V3 on = angular_velocity();
    Quat inc = q_from_scaled_axis(mul(on, dt));
    q = qmul(inc, q);
    return led;
  }
};

// rigid.rs:115-182
bool make_pellet(double r, double len, double rho, const V3& pos, Pellet& p, std::string& err) {
  if (!(std::isfinite(r) && r > 0.0)) {
    err = "pellet radius must be positive";
    return false;
  }
  if (!(std::isfinite(len) && len >= 2.0 * r)) {
    err = "pellet length must be at least twice the radius";
    return false;
  }
  if (!(std::isfinite(rho) && rho > 0.0)) {
    err = "pellet density must be positive";
    return false;
  }
  p.radius = r;
  p.length = len;
  p.mass = rho * kPi * r * r * len;
  p.inertia = v3(0.5 * p.mass * r * r, p.mass * (3.0 * r * r + len * len) / 12.0,
                 p.mass * (3.0 * r * r + len * len) / 12.0);
  p.position = pos;
  p.q = Quat{0, 0, 0, 1};
  p.velocity = zero3();
  p.L = zero3();
  double hs = 0.5 * len - r;
  size_t count;
  if (hs <= 0.0) count = 1;
  else {
    double ratio = std::ceil(2.0 * hs / r);
    if (!std::isfinite(ratio) || ratio > 4095.0) {
      err = "pellet proxy exceeds the sphere allocation cap";
      return false;
    }
    count = (size_t)ratio + 1;
  }
  if (count > 64) {
    err = "pellet proxy exceeds 64 spheres";
    return false;
  }
  p.offsets.clear();
  for (size_t i = 0; i < count; ++i)
    p.offsets.push_back(count == 1 ? 0.0 : -hs + 2.0 * hs * (double)i / (double)(count - 1));
  return true;
}

struct Coupling {
  V3 impulse, angular;
  double grid_energy;
  size_t constrained;
};

// ---------------------------------------------------------------- solver.rs
struct Ledger {
  double initial_mass = 0, outflow_mass = 0;
  V3 initial_momentum = zero3();
  double initial_mech = 0;
  V3 gravity_impulse = zero3(), wall_impulse = zero3(), pellet_wall_impulse = zero3(), coupling_impulse = zero3(),
     coupling_angular = zero3();
  double proj = 0, fric = 0, trac = 0, pellet_work = 0, cgrid = 0, cpellet = 0, plastic = 0;
  V3 outflow_momentum = zero3();
  // solver.rs:164-172
  double ledgered() const { return proj - fric + trac + pellet_work + cgrid + cpellet - plastic; }
};

struct Config {
  V3 gravity;
  double friction, cfl, max_dt, min_dt;
  Contact contact;
  bool face_mode;
  bool sticky[6];
  double face_mu[6];
  double tol;
};

struct ParticleTrial {
  V3 x, v;
  M3 C, F;
  double J;
  M3 tau;
  double dep, diss, disp;
  int iterations;
  bool yielded;
};
struct NodeTrial {
  V3 velocity, wall_impulse;
  double proj, fric;
};

enum StepFail { SF_OK = 0, SF_CONST, SF_GRID, SF_DISP, SF_PELLET, SF_TRACTION };

// audit.rs:72-90: kinetic snapshots of one trial
struct AuditStages {
  double transport = 0, stress = 0, traction = 0, gravity = 0, walls = 0, coupling = 0, pellet_after = 0,
         plastic = 0;
};

// pellet bed (extension): tangential spring of one sphere pair
struct HmEntry {
  int other, a, b;
  V3 xi;
};
constexpr int HM_SLOTS = 24, BED_CAND = 64;

struct Simulation {
  Material mat;
  Particles P;
  Grid grid;
  bool has_pellet = false;
  Pellet pellet;
  // pellet bed (extension)
  std::vector<Pellet> bed;
  std::vector<std::vector<HmEntry>> hist;
  double hm_estar = 0, hm_gstar = 0, hm_mu = 0, hm_beta = 0, bed_rb = 0;
  // linear contact law of the household DEM (dem.rs:95-127): stiffness, damping ratio, rolling
  int bed_law = 0;
  double dem_kn = 0, dem_zeta = 0, dem_mur = 0;
  double bed_contact_work = 0.0;
  int bed_contacts = 0;
  uint64_t bed_overflow = 0;
  Config cfg;
  Ledger ledger;
  double time = 0.0;
  uint64_t step_count = 0, limited_steps = 0, rejected_steps = 0;
  double dt_scale = 1.0, min_dt_used = std::numeric_limits<double>::infinity(), max_dt_used = 0.0;
  uint64_t newton_iterations = 0, yielded = 0;
  std::string last_failure;
  AuditStages* audit = nullptr;  // set while an audit trial records its stages

  // audit.rs:360-378 grid_kinetic: active nodes, momentum (or velocity after the walls) plus kick
  double grid_kinetic(bool velocities, const V3& kick) const {
    double e = 0.0;
    for (int64_t i : grid.active) {
      const double m = grid.mass[i];
      if (!(m > 0.0)) continue;
      V3 v = velocities ? grid.momentum[i] : divs(grid.momentum[i], m);
      e += 0.5 * m * norm2(add(v, kick));
    }
    return e;
  }
  // audit.rs:381-398: independent APIC-only deposition on a shadow grid
  double transport_energy() const {
    Grid shadow;
    shadow.init(grid.layout);
    const Layout& L = grid.layout;
    for (size_t p = 0; p < P.size(); ++p) {
      Stencil s;
      if (!stencil_of(L, P.x[p], s)) return std::numeric_limits<double>::quiet_NaN();
      const double mass = P.m[p];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          for (int c = 0; c < 3; ++c) {
            const double w = s.weight(a, b, c);
            V3 vel = add(P.v[p], mvec(P.C[p], s.distance(a, b, c)));
            int64_t index = L.index(s.base[0] + a, s.base[1] + b, s.base[2] + c);
            shadow.deposit(index, w * mass, mul(vel, w * mass));
          }
    }
    double e = 0.0;
    for (int64_t i : shadow.active) {
      const double m = shadow.mass[i];
      if (!(m > 0.0)) continue;
      e += 0.5 * m * norm2(divs(shadow.momentum[i], m));
    }
    return e;
  }
  // audit.rs:38-53 EnergyState::measure: translation, affine norm, elastic, potential, pellet
  void energy_state(double out[5]) const {
    const double h = grid.layout.spacing;
    double aff = 0.0;
    for (size_t p = 0; p < P.size(); ++p) {
      double n2 = 0.0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) n2 += P.C[p].a[i][j] * P.C[p].a[i][j];
      aff += P.m[p] * n2;
    }
    out[0] = P.kinetic_energy();
    out[1] = h * h / 8.0 * aff;
    out[2] = elastic_energy();
    out[3] = potential_energy();
    double pk = has_pellet ? pellet.kinetic_energy() : 0.0;
    for (const Pellet& b : bed) pk += b.kinetic_energy();
    out[4] = pk;
  }

  double ys_of(size_t p) const { return P.ys[p]; }

  double face_mu(int axis, double sign) const {
    int f = 2 * axis + (sign > 0 ? 0 : 1);
    return cfg.face_mu[f];
  }
  bool face_sticky(int axis, double sign) const {
    int f = 2 * axis + (sign > 0 ? 0 : 1);
    return cfg.face_mode && cfg.sticky[f];
  }

  V3 total_momentum() const {
    V3 m = P.linear_momentum();
    if (has_pellet) m = add(m, mul(pellet.velocity, pellet.mass));
    for (const Pellet& b : bed) m = add(m, mul(b.velocity, b.mass));
    return m;
  }
  // solver.rs:1013-1020
  V3 momentum_residual() const {
    return sub(sub(add(sub(sub(total_momentum(), ledger.initial_momentum), ledger.gravity_impulse),
                       ledger.outflow_momentum),
                   ledger.wall_impulse),
               ledger.pellet_wall_impulse);
  }
  double mass_residual() const { return P.total_mass() + ledger.outflow_mass - ledger.initial_mass; }
  double potential_energy() const {
    const V3& g = cfg.gravity;
    double e = 0.0;
    for (size_t p = 0; p < P.size(); ++p) e += -P.m[p] * dot(g, P.x[p]);
    if (has_pellet) e -= pellet.mass * dot(g, pellet.position);
    for (const Pellet& b : bed) e -= b.mass * dot(g, b.position);
    return e;
  }
  double elastic_energy() const {
    double s = 0.0;
    for (size_t p = 0; p < P.size(); ++p) {
      double v0 = P.V0[p], term;
      if (mat.kind == LP_PASTE) {
        const M3& f = P.F[p];
        M3 b = mmul(f, mT(f));
        V3 ev;
        M3 u;
        if (!symmetric_eigen3(b, ev, u)) term = std::numeric_limits<double>::quiet_NaN();
        else {
          V3 h = v3(0.5 * std::log(std::fmax(ev[0], 1e-300)), 0.5 * std::log(std::fmax(ev[1], 1e-300)),
                    0.5 * std::log(std::fmax(ev[2], 1e-300)));
          double trace = h[0] + h[1] + h[2];
          term = v0 * (mat.mu * norm2(h) + 0.5 * mat.lambda * trace * trace);
        }
      } else {
        double j = P.J[p];
        term = v0 * mat.bulk * (j - 1.0 - std::log(j));
      }
      s += term;
    }
    return s;
  }
  double kinetic_energy() const {
    double k = P.kinetic_energy() + (has_pellet ? pellet.kinetic_energy() : 0.0);
    for (const Pellet& b : bed) k += b.kinetic_energy();
    return k;
  }
  double mechanical_energy() const { return kinetic_energy() + potential_energy() + elastic_energy(); }
  double energy_residual() const {
    return mechanical_energy() - ledger.initial_mech - (ledger.ledgered() + bed_contact_work);
  }

  // solver.rs:477-498
  double stability_limit() const {
    double dx = grid.layout.spacing;
    double max_speed = 0.0;
    for (auto& v : P.v) max_speed = std::fmax(max_speed, norm(v));
    double wave = wave_speed(mat);
    double limit = cfg.cfl * dx / (wave + max_speed);
    double d = diffusivity(mat);
    if (d > 0.0) limit = std::fmin(limit, 0.25 * dx * dx / d);
    if (has_pellet) {
      limit = std::fmin(limit, cfg.contact.stable_dt(pellet.mass));
      double ps = norm(pellet.velocity);
      if (ps > 0.0) limit = std::fmin(limit, cfg.cfl * dx / ps);
    }
    // pellet bed: per pellet as above, plus 0.2 sqrt(m*/k_c) for the Hertz stiffness at an
    // overlap of 5 % of the radius, k_c = 2 E* sqrt(R* 0.05 r)
    for (const Pellet& b : bed) {
      limit = std::fmin(limit, cfg.contact.stable_dt(b.mass));
      double ps = norm(b.velocity);
      if (ps > 0.0) limit = std::fmin(limit, cfg.cfl * dx / ps);
      if (bed_law == LP_BED_LINEAR) {
        // World::stable_dt (dem.rs:509-520)
        limit = std::fmin(limit, 0.1 * std::sqrt(b.mass / dem_kn));
      } else {
        double kc = 2.0 * hm_estar * std::sqrt(0.5 * b.radius * 0.05 * b.radius);
        limit = std::fmin(limit, 0.2 * std::sqrt(0.5 * b.mass / kc));
      }
    }
    return limit;
  }

  // solver.rs:501-517
  void sort_particles() {
    const Layout& L = grid.layout;
    std::vector<size_t> order(P.size());
    std::vector<uint64_t> key(P.size());
    for (size_t i = 0; i < P.size(); ++i) {
      order[i] = i;
      uint64_t cell = 0;
      for (int axis = 0; axis < 3; ++axis) {
        double scaled = std::fmax(std::floor(P.x[i][axis] / L.spacing), 0.0);
        uint64_t coord = std::isnan(scaled) ? 0 : (scaled >= 1.8e19 ? UINT64_MAX : (uint64_t)scaled);
        coord = std::min<uint64_t>(coord, (uint64_t)L.cells[axis]);
        cell = cell * (uint64_t)(L.cells[axis] + 1) + coord;
      }
      key[i] = cell;
    }
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
      if (key[a] != key[b]) return key[a] < key[b];
      return P.id[a] < P.id[b];
    });
    P.permute(order);
  }

  // solver.rs:520-532
  void sweep_outflow() {
    std::vector<size_t> escaped;
    Stencil s;
    for (size_t i = 0; i < P.size(); ++i)
      if (!stencil_of(grid.layout, P.x[i], s)) escaped.push_back(i);
    if (escaped.empty()) return;
    for (size_t i : escaped) ledger.outflow_momentum = add(ledger.outflow_momentum, mul(P.v[i], P.m[i]));
    ledger.outflow_mass += P.remove_sorted(escaped);
  }

  // solver.rs:632-661
  void deposit_particles(double dt) {
    grid.clear();
    const Layout& L = grid.layout;
    double dx2_inv = 4.0 / (L.spacing * L.spacing);
    for (size_t p = 0; p < P.size(); ++p) {
      Stencil s;
      if (!stencil_of(L, P.x[p], s)) continue;
      double mass = P.m[p];
      V3 vel = P.v[p];
      M3 am = msub(mscale(P.C[p], mass), mscale(P.tau[p], dt * dx2_inv * P.V0[p]));
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          for (int c = 0; c < 3; ++c) {
            double w = s.weight(a, b, c);
            V3 d = s.distance(a, b, c);
            int64_t index = L.index(s.base[0] + a, s.base[1] + b, s.base[2] + c);
            V3 mom = mul(add(mul(vel, mass), mvec(am, d)), w);
            grid.deposit(index, w * mass, mom);
          }
    }
  }

  // solver.rs:725-819
  void wall_traction(double dt, V3& impulse, double& energy) {
    const Layout& L = grid.layout;
    V3 ext = L.extents();
    double half = 0.5 * L.spacing;
    double force_scale = -dt * 4.0 / (L.spacing * L.spacing);
    const V3& g = cfg.gravity;
    impulse = zero3();
    energy = 0.0;
    for (size_t p = 0; p < P.size(); ++p) {
      V3 pos = P.x[p];
      double mass = P.m[p], vol0 = P.V0[p];
      for (int axis = 0; axis < 3; ++axis) {
        double face;
        if (pos[axis] < half) face = 0.0;
        else if (pos[axis] > ext[axis] - half) face = ext[axis];
        else continue;
        V3 image = pos;
        image[axis] = 2.0 * face - pos[axis];
        Stencil s;
        if (!stencil_of(L, image, s)) continue;
        int64_t plane;
        double inward;
        if (face == 0.0) {
          plane = 1;
          inward = 1.0;
        } else {
          plane = L.cells[axis] + 1;
          inward = -1.0;
        }
        double ns = P.tau[p].a[axis][axis] * vol0 - mass * g[axis] * (image[axis] - pos[axis]);
        if (ns >= 0.0) continue;
        double wm = mass * g[axis] * dt;
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 3; ++c) {
              int64_t co[3] = {s.base[0] + a, s.base[1] + b, s.base[2] + c};
              if (L.wall_side(axis, co[axis]) != 0.0) continue;
              double w = s.weight(a, b, c);
              if (w == 0.0) continue;
              int64_t pc[3] = {co[0], co[1], co[2]};
              pc[axis] = plane;
              int64_t pi = L.index(pc[0], pc[1], pc[2]);
              double pm = grid.mass[pi];
              if (pm <= 0.0) continue;
              double trial = grid.momentum[pi][axis] / pm + g[axis] * dt;
              if (trial * inward >= 0.0) continue;
              double dist = s.distance(a, b, c)[axis];
              double reaction = (ns * dist * force_scale + wm) * w * inward;
              if (reaction <= 0.0) continue;
              int64_t idx = L.index(co[0], co[1], co[2]);
              double jump;
              if (grid.deposit_reaction(idx, axis, inward, reaction, jump)) {
                impulse[axis] += reaction * inward;
                energy += jump;
              }
            }
      }
    }
  }

  static V3 reduce_tangential(const V3& t, double reduction) {
    if (reduction == 0.0) return t;
    double speed = norm(t);
    if (speed <= reduction) return zero3();
    return mul(t, (speed - reduction) / speed);
  }

  // solver.rs:822-892 for one node
  bool update_node(int64_t index, double dt, NodeTrial& out) const {
    const Layout& L = grid.layout;
    double mass = grid.mass[index];
    if (mass <= 0.0) {
      out = NodeTrial{zero3(), zero3(), 0.0, 0.0};
      return true;
    }
    const V3& g = cfg.gravity;
    V3 vel = v3(grid.momentum[index][0] / mass + g[0] * dt, grid.momentum[index][1] / mass + g[1] * dt,
                grid.momentum[index][2] / mass + g[2] * dt);
    if (!finite3(vel)) return false;
    V3 before = vel;
    double proj = 0.0, fric = 0.0;
    int64_t co[3];
    L.coords(index, co[0], co[1], co[2]);
    for (int axis = 0; axis < 3; ++axis) {
      double sign = L.wall_side(axis, co[axis]);
      if (sign == 0.0) continue;
      double nsp = vel[axis] * sign;
      if (nsp >= 0.0) continue;
      proj -= 0.5 * mass * nsp * nsp;
      vel[axis] = 0.0;
      V3 tang = vel;
      if (face_sticky(axis, sign)) vel = zero3();
      else vel = reduce_tangential(tang, (cfg.face_mode ? face_mu(axis, sign) : cfg.friction) * (-nsp));
      fric += 0.5 * mass * (norm2(tang) - norm2(vel));
    }
    for (int axis = 0; axis < 3; ++axis) {
      double reaction = grid.traction[index][axis];
      if (reaction <= 0.0) continue;
      double normal = vel[axis];
      V3 tang = vel;
      tang[axis] = 0.0;
      V3 reduced;
      if (!cfg.face_mode) reduced = reduce_tangential(tang, cfg.friction * reaction / mass);
      else {
        double rl = grid.traction_low[index][axis], rh = grid.traction_high[index][axis];
        bool stick = (rl > 0.0 && cfg.sticky[2 * axis]) || (rh > 0.0 && cfg.sticky[2 * axis + 1]);
        if (stick) reduced = zero3();
        else reduced = reduce_tangential(tang, (cfg.face_mu[2 * axis] * rl + cfg.face_mu[2 * axis + 1] * rh) / mass);
      }
      fric += 0.5 * mass * (norm2(tang) - norm2(reduced));
      vel = reduced;
      vel[axis] = normal;
    }
    out.velocity = vel;
    out.wall_impulse = mul(sub(vel, before), mass);
    out.proj = proj;
    out.fric = fric;
    return true;
  }

  // Pellet bed coupling: couple_grid (rigid.rs:385-438) over all pellets, each node constrained
  // by the pellet of smallest signed distance (ties: lower index); per-pellet sums in node order.
  std::vector<Coupling> couple_bed(const std::vector<Pellet>& pels, double friction) {
    const Layout& L = grid.layout;
    const size_t na = grid.active.size();
    const size_t np = pels.size();
    std::vector<V3> lo(np), hi(np);
    for (size_t q = 0; q < np; ++q) pels[q].bounding_box(lo[q], hi[q]);
    struct Upd {
      int owner;
      V3 nv, dp, lever;
      double energy;
    };
    std::vector<Upd> upd(na);
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < (int64_t)na; ++s) {
      int64_t index = grid.active[s];
      Upd u;
      u.owner = -1;
      double mass = grid.mass[index];
      if (mass > 0.0) {
        int64_t i, j, k;
        L.coords(index, i, j, k);
        V3 node = L.node_position(i, j, k);
        int best_q = -1;
        double best = 0.0;
        V3 best_n = zero3();
        for (size_t q = 0; q < np; ++q) {
          bool outside = false;
          for (int a = 0; a < 3; ++a)
            if (node[a] < lo[q][a] || node[a] > hi[q][a]) outside = true;
          if (outside) continue;
          V3 n;
          double phi = pels[q].signed_distance(node, n);
          if (phi > 0.0) continue;
          if (best_q < 0 || phi < best) {
            best_q = (int)q;
            best = phi;
            best_n = n;
          }
        }
        if (best_q >= 0) {
          const Pellet& pel = pels[best_q];
          V3 vel = grid.momentum[index];
          V3 bv = pel.point_velocity(node);
          V3 rel = sub(vel, bv);
          double nsp = dot(rel, best_n);
          if (nsp < 0.0) {
            V3 tang = sub(rel, mul(best_n, nsp));
            double ts = norm(tang);
            double fr = friction * (-nsp);
            V3 tn = (ts <= fr || ts < 1e-14) ? zero3() : mul(tang, (ts - fr) / ts);
            V3 nv = add(bv, tn);
            V3 dp = mul(sub(nv, vel), mass);
            double energy = 0.5 * mass * (norm2(nv) - norm2(vel));
            u = Upd{best_q, nv, dp, sub(node, pel.position), energy};
          }
        }
      }
      upd[s] = u;
    }
    std::vector<Coupling> r(np, Coupling{zero3(), zero3(), 0.0, 0});
    for (size_t s = 0; s < na; ++s) {
      if (upd[s].owner < 0) continue;
      grid.momentum[grid.active[s]] = upd[s].nv;
      Coupling& c = r[upd[s].owner];
      c.impulse = sub(c.impulse, upd[s].dp);
      c.angular = sub(c.angular, cross(upd[s].lever, upd[s].dp));
      c.grid_energy += upd[s].energy;
      c.constrained += 1;
    }
    return r;
  }

  // Hertz-Mindlin sphere contact on pellet p from the start-of-step states of all pellets:
  // force and torque on p and its new tangential-spring list.  Returns false when more than
  // BED_CAND pellets lie within two bounding radii.
  bool bed_contact(size_t p, double dt, V3& F, V3& T, int& contacts, int& overflow,
                   std::vector<HmEntry>& next) const {
    const Pellet& P = bed[p];
    F = zero3();
    T = zero3();
    contacts = 0;
    overflow = 0;
    next.clear();
    const V3 axp = P.axis(), omp = P.angular_velocity();
    const double rs = 0.5 * P.radius, k56 = 1.8257418583505538;
    int cand = 0;
    for (size_t q = 0; q < bed.size(); ++q) {
      if (q == p) continue;
      const Pellet& Q = bed[q];
      V3 dq = sub(Q.position, P.position);
      if (norm2(dq) > 4.0 * bed_rb * bed_rb) continue;
      if (++cand > BED_CAND) return false;
      const V3 axq = Q.axis(), omq = Q.angular_velocity();
      const double mstar = P.mass * Q.mass / (P.mass + Q.mass);
      for (size_t a = 0; a < P.offsets.size(); ++a) {
        V3 ca = add(P.position, mul(axp, P.offsets[a]));
        for (size_t b = 0; b < Q.offsets.size(); ++b) {
          V3 cb = add(Q.position, mul(axq, Q.offsets[b]));
          V3 d = sub(cb, ca);
          double dist = norm(d);
          double delta = (P.radius + Q.radius) - dist;
          if (!(delta > 0.0) || !(dist > 1e-12)) continue;
          V3 nn = divs(d, dist);
          V3 cp = mul(add(ca, cb), 0.5);
          V3 lp = sub(cp, P.position), lq = sub(cp, Q.position);
          V3 vp = add(P.velocity, cross(omp, lp));
          V3 vrel = sub(add(Q.velocity, cross(omq, lq)), vp);
          double vn = dot(vrel, nn);
          V3 vt = sub(vrel, mul(nn, vn));
          V3 xi = zero3();
          for (const HmEntry& h : hist[p])
            if (h.other == (int)q && h.a == (int)a && h.b == (int)b) {
              xi = h.xi;
              break;
            }
          double xn = dot(xi, nn);
          V3 ft, roll = zero3();
          double fn;
          if (bed_law == LP_BED_LINEAR) {
            // World::contact_force (dem.rs:789-834) with P as the first body: the reference's
            // normal points at P (-nn) and its relative velocity is v_P - v_Q (-vrel), so its
            // tangential velocity is -vt while v_n keeps its sign
            const double cn = 2.0 * dem_zeta * std::sqrt(dem_kn * mstar);
            const double kt = (2.0 / 7.0) * dem_kn, ct = std::sqrt(2.0 / 7.0) * cn;
            fn = std::fmax(dem_kn * delta - cn * vn, 0.0);
            for (int k = 0; k < 3; ++k) {
              xi[k] = (xi[k] - xn * nn[k]) - vt[k] * dt;
              ft[k] = -(xi[k] * kt) + vt[k] * ct;
            }
            double ftn = norm(ft), lim = hm_mu * fn;
            if (ftn > lim) {
              double sc = ftn > std::numeric_limits<double>::epsilon() ? lim / ftn : 0.0;
              for (int k = 0; k < 3; ++k) {
                ft[k] *= sc;
                xi[k] = -ft[k] / kt;
              }
            }
            V3 wr = sub(omp, omq);
            double wn = norm(wr);
            if (wn > std::numeric_limits<double>::epsilon()) roll = mul(divs(wr, -wn), dem_mur * rs * fn);
          } else {
            double sq = std::sqrt(rs * delta);
            double sn = 2.0 * hm_estar * sq, stf = 8.0 * hm_gstar * sq;
            double gn = -k56 * hm_beta * std::sqrt(sn * mstar), gt = -k56 * hm_beta * std::sqrt(stf * mstar);
            fn = std::fmax((4.0 / 3.0) * hm_estar * std::sqrt(rs) * (delta * std::sqrt(delta)) - gn * vn, 0.0);
            for (int k = 0; k < 3; ++k) {
              xi[k] = (xi[k] - xn * nn[k]) + vt[k] * dt;
              ft[k] = stf * xi[k] + gt * vt[k];
            }
            double ftn = norm(ft), lim = hm_mu * fn;
            if (ftn > lim) {
              double sc = lim / ftn;
              for (int k = 0; k < 3; ++k) {
                ft[k] *= sc;
                xi[k] = (ft[k] - gt * vt[k]) / stf;
              }
            }
          }
          V3 f = sub(ft, mul(nn, fn));
          F = add(F, f);
          T = add(add(T, cross(lp, f)), roll);
          ++contacts;
          if ((int)next.size() < HM_SLOTS) next.push_back(HmEntry{(int)q, (int)a, (int)b, xi});
          else ++overflow;
        }
      }
    }
    return true;
  }

  // rigid.rs:385-438
  Coupling couple_grid(const Pellet& pel, double friction) {
    V3 lo, hi;
    pel.bounding_box(lo, hi);
    const Layout& L = grid.layout;
    const size_t na = grid.active.size();
    struct Upd {
      bool some;
      V3 nv, dp, lever;
      double energy;
    };
    std::vector<Upd> upd(na);
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < (int64_t)na; ++s) {
      int64_t index = grid.active[s];
      Upd u;
      u.some = false;
      double mass = grid.mass[index];
      if (mass > 0.0) {
        int64_t i, j, k;
        L.coords(index, i, j, k);
        V3 node = L.node_position(i, j, k);
        bool outside = false;
        for (int a = 0; a < 3; ++a)
          if (node[a] < lo[a] || node[a] > hi[a]) outside = true;
        if (!outside) {
          V3 normal;
          double phi = pel.signed_distance(node, normal);
          if (phi <= 0.0) {
            V3 vel = grid.momentum[index];
            V3 bv = pel.point_velocity(node);
            V3 rel = sub(vel, bv);
            double nsp = dot(rel, normal);
            if (nsp < 0.0) {
              V3 tang = sub(rel, mul(normal, nsp));
              double ts = norm(tang);
              double fr = friction * (-nsp);
              V3 tn = (ts <= fr || ts < 1e-14) ? zero3() : mul(tang, (ts - fr) / ts);
              V3 nv = add(bv, tn);
              V3 dp = mul(sub(nv, vel), mass);
              double energy = 0.5 * mass * (norm2(nv) - norm2(vel));
              u = Upd{true, nv, dp, sub(node, pel.position), energy};
            }
          }
        }
      }
      upd[s] = u;
    }
    Coupling r{zero3(), zero3(), 0.0, 0};
    for (size_t s = 0; s < na; ++s) {
      if (!upd[s].some) continue;
      grid.momentum[grid.active[s]] = upd[s].nv;
      r.impulse = sub(r.impulse, upd[s].dp);
      r.angular = sub(r.angular, cross(upd[s].lever, upd[s].dp));
      r.grid_energy += upd[s].energy;
      r.constrained += 1;
    }
    return r;
  }

  // solver.rs:895-977 for one particle
  int g2p_particle(size_t p, double dt, ParticleTrial& t) const {
    const Layout& L = grid.layout;
    double dx2_inv = 4.0 / (L.spacing * L.spacing);
    Stencil s;
    V3 pos = P.x[p];
    t.iterations = 0;
    t.yielded = false;
    if (!stencil_of(L, pos, s)) {
      t = ParticleTrial{pos, P.v[p], P.C[p], P.F[p], P.J[p], P.tau[p], 0.0, 0.0, 0.0, 0, false};
      return CE_OK;
    }
    V3 vel = zero3();
    M3 aff = mzero();
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        for (int c = 0; c < 3; ++c) {
          double w = s.weight(a, b, c);
          V3 d = s.distance(a, b, c);
          int64_t index = L.index(s.base[0] + a, s.base[1] + b, s.base[2] + c);
          V3 nv = mul(grid.momentum[index], w);
          vel = add(vel, nv);
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) aff.a[i][j] += nv[i] * d[j];
        }
    aff = mscale(aff, dx2_inv);
    t.x = add(pos, mul(vel, dt));
    t.disp = norm(vel) * dt / L.spacing;
    t.v = vel;
    t.C = aff;
    if (mat.kind == LP_PASTE) {
      M3 trial = mmul(madd(mident(), mscale(aff, dt)), P.F[p]);
      PasteUpdate u;
      int e = update_paste(trial, mat, ys_of(p), dt, cfg.tol, u);
      if (e != CE_OK) return e;
      t.F = u.deformation;
      t.J = 1.0;
      t.tau = u.kirchhoff;
      t.dep = u.dep;
      t.diss = u.dissipation_density * P.V0[p];
      t.iterations = u.iterations;
      t.yielded = u.dep > 0.0 || u.iterations > 0;
    } else {
      LiquidUpdate u;
      int e = update_liquid(P.J[p], aff, mat, dt, u);
      if (e != CE_OK) return e;
      t.F = mident();
      t.J = u.j;
      t.tau = u.kirchhoff;
      t.dep = 0.0;
      t.diss = 0.0;
    }
    return CE_OK;
  }

  // solver.rs:540-611 (without the audit hooks)
  int try_step(double dt) {
    sweep_outflow();
    deposit_particles(dt);
    if (audit) audit->stress = grid_kinetic(false, zero3());
    V3 timp;
    double tenergy;
    wall_traction(dt, timp, tenergy);
    if (audit) {
      audit->traction = grid_kinetic(false, zero3());
      audit->gravity = grid_kinetic(false, mul(cfg.gravity, dt));
    }
    if (!std::isfinite(tenergy) || !std::isfinite(ledger.trac + tenergy)) {
      last_failure = "wall traction kinetic-energy jump became non-finite";
      return SF_TRACTION;
    }
    const size_t na = grid.active.size();
    std::vector<NodeTrial> nt(na);
    std::vector<char> okv(na, 1);
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < (int64_t)na; ++s) okv[s] = update_node(grid.active[s], dt, nt[s]) ? 1 : 0;
    for (size_t s = 0; s < na; ++s)
      if (!okv[s]) {
        last_failure = "non-finite grid velocity";
        return SF_GRID;
      }
    V3 wimp = timp;
    double wproj = 0.0, wfric = 0.0, wtrac = tenergy;
    for (size_t s = 0; s < na; ++s) {
      grid.momentum[grid.active[s]] = nt[s].velocity;
      wimp = add(wimp, nt[s].wall_impulse);
      wproj += nt[s].proj;
      wfric += nt[s].fric;
    }
    if (audit) audit->walls = grid_kinetic(true, zero3());
    Pellet ptrial = pellet;
    Coupling coup{zero3(), zero3(), 0.0, 0};
    double pellet_energy = 0.0;
    WallContact pwall{zero3(), 0.0, 0};
    if (has_pellet) {
      coup = couple_grid(ptrial, cfg.friction);
      double kb = ptrial.kinetic_energy();
      ptrial.apply_impulse(coup.impulse, coup.angular);
      pellet_energy = ptrial.kinetic_energy() - kb;
      if (audit) audit->pellet_after = ptrial.kinetic_energy();
      V3 ext = grid.layout.extents();
      pwall = ptrial.integrate(dt, cfg.gravity, ext, cfg.contact);
      if (!ptrial.finite() || !std::isfinite(pellet_energy)) {
        last_failure = "pellet state became non-finite";
        return SF_PELLET;
      }
    }
    // pellet bed (extension): coupling, sphere contacts from the start-of-step states, rigid step
    std::vector<Pellet> btrial = bed;
    std::vector<std::vector<HmEntry>> htrial(bed.size());
    std::vector<Coupling> bcoup;
    std::vector<double> bpe(bed.size(), 0.0), bwork(bed.size(), 0.0);
    std::vector<WallContact> bwall(bed.size(), WallContact{zero3(), 0.0, 0});
    int bcontacts = 0;
    uint64_t boverflow = 0;
    if (!bed.empty()) {
      bcoup = couple_bed(bed, cfg.friction);
      V3 ext = grid.layout.extents();
      for (size_t p = 0; p < bed.size(); ++p) {
        V3 F, T;
        int nc, ov;
        if (!bed_contact(p, dt, F, T, nc, ov, htrial[p])) {
          last_failure = "pellet state became non-finite";
          return SF_PELLET;
        }
        bcontacts += nc;
        boverflow += (uint64_t)ov;
        Pellet& b = btrial[p];
        double kb = b.kinetic_energy();
        b.apply_impulse(bcoup[p].impulse, bcoup[p].angular);
        bpe[p] = b.kinetic_energy() - kb;
        if (audit) audit->pellet_after += b.kinetic_energy();
        bwall[p] = b.integrate(dt, cfg.gravity, ext, cfg.contact, &F, &T);
        // contact work at the step's mean linear and angular velocity
        const V3 om0 = bed[p].angular_velocity(), om1 = b.angular_velocity();
        double W = 0.0;
        for (int k = 0; k < 3; ++k)
          W += (F[k] * (0.5 * (bed[p].velocity[k] + b.velocity[k])) + T[k] * (0.5 * (om0[k] + om1[k]))) * dt;
        bwork[p] = W;
        if (!b.finite() || !std::isfinite(bpe[p]) || !std::isfinite(W)) {
          last_failure = "pellet state became non-finite";
          return SF_PELLET;
        }
      }
    }
    if (audit) audit->coupling = grid_kinetic(true, zero3());
    const size_t np = P.size();
    std::vector<ParticleTrial> tr(np);
    std::vector<int> err(np, CE_OK);
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < (int64_t)np; ++p) err[p] = g2p_particle((size_t)p, dt, tr[p]);
    for (size_t p = 0; p < np; ++p)
      if (err[p] != CE_OK) {
        last_failure = std::string("constitutive update failed: ") + const_err_name(err[p]);
        return SF_CONST;
      }
    if (audit) {
      double d = 0.0;
      for (size_t p = 0; p < np; ++p) d += tr[p].diss;
      audit->plastic = d;
    }
    double max_cells = 0.0;
    for (size_t p = 0; p < np; ++p) max_cells = std::fmax(max_cells, tr[p].disp);
    if (max_cells > 1.0) {
      char buf[128];
      std::snprintf(buf, sizeof(buf), "particle moved '%g' cells in one step", max_cells);
      last_failure = buf;
      return SF_DISP;
    }
    // commit (solver.rs:980-998)
    double dissipation = 0.0;
    uint64_t iters = 0, yielded_now = 0;
    for (size_t p = 0; p < np; ++p) {
      P.x[p] = tr[p].x;
      P.v[p] = tr[p].v;
      P.C[p] = tr[p].C;
      P.F[p] = tr[p].F;
      P.J[p] = tr[p].J;
      P.tau[p] = tr[p].tau;
      P.ep[p] += tr[p].dep;
      dissipation += tr[p].diss;
      iters += (uint64_t)tr[p].iterations;
      yielded_now += tr[p].iterations > 0 ? 1 : 0;
    }
    newton_iterations += iters;
    yielded = yielded_now;
    ledger.plastic += dissipation;
    ledger.wall_impulse = add(ledger.wall_impulse, wimp);
    ledger.proj += wproj;
    ledger.fric += wfric;
    ledger.trac += wtrac;
    ledger.gravity_impulse = add(ledger.gravity_impulse, mul(cfg.gravity, P.total_mass() * dt));
    if (has_pellet) {
      ledger.gravity_impulse = add(ledger.gravity_impulse, mul(cfg.gravity, ptrial.mass * dt));
      ledger.pellet_wall_impulse = add(ledger.pellet_wall_impulse, pwall.impulse);
      ledger.pellet_work += pwall.work;
      ledger.coupling_impulse = add(ledger.coupling_impulse, coup.impulse);
      ledger.coupling_angular = add(ledger.coupling_angular, coup.angular);
      ledger.cgrid += coup.grid_energy;
      ledger.cpellet += pellet_energy;
      pellet = ptrial;
    }
    if (!bed.empty()) {
      double bm = 0.0;
      for (size_t p = 0; p < bed.size(); ++p) {
        bm += btrial[p].mass;
        ledger.pellet_wall_impulse = add(ledger.pellet_wall_impulse, bwall[p].impulse);
        ledger.pellet_work += bwall[p].work;
        ledger.coupling_impulse = add(ledger.coupling_impulse, bcoup[p].impulse);
        ledger.coupling_angular = add(ledger.coupling_angular, bcoup[p].angular);
        ledger.cgrid += bcoup[p].grid_energy;
        ledger.cpellet += bpe[p];
        bed_contact_work += bwork[p];
      }
      ledger.gravity_impulse = add(ledger.gravity_impulse, mul(cfg.gravity, bm * dt));
      bed_contacts = bcontacts;
      bed_overflow += boverflow;
      bed = btrial;
      hist = htrial;
    }
    return SF_OK;
  }

  // solver.rs:413-472; max_accepted > 0 acts as the caller's budget
  int advance(double target, int64_t max_accepted, bool& reached, std::string& err) {
    reached = false;
    if (!std::isfinite(target) || target < time) {
      err = "invalid solver state: invalid target time";
      return LP_INVALID;
    }
    int64_t accepted = 0;
    while (time < target) {
      if (max_accepted > 0 && accepted >= max_accepted) return LP_BUDGET;
      double remaining = target - time;
      double limit = stability_limit();
      double scaled = dt_scale * limit;
      bool limited = scaled < cfg.max_dt;
      double dt = std::fmin(std::fmin(scaled, cfg.max_dt), remaining);
      if (remaining - dt < 1e-12 * std::fmax(target, 1.0)) dt = remaining;
      if (!std::isfinite(dt) || dt <= 0.0 || (dt < cfg.min_dt && remaining > cfg.min_dt)) {
        err = "solver aborted: stability limit is nonfinite, nonpositive or below minimum";
        return LP_MIN_STEP;
      }
      int f = try_step(dt);
      if (f == SF_OK) {
        time += dt;
        step_count += 1;
        limited_steps += limited ? 1 : 0;
        min_dt_used = std::fmin(min_dt_used, dt);
        max_dt_used = std::fmax(max_dt_used, dt);
        dt_scale = std::fmin(dt_scale * 1.25, 1.0);
        ++accepted;
        if (step_count % 32 == 0) sort_particles();
      } else {
        rejected_steps += 1;
        dt_scale *= 0.5;
        if (dt_scale * limit < cfg.min_dt) {
          err = "solver aborted: step below minimum; last failure: " + last_failure;
          return LP_MIN_STEP;
        }
      }
    }
    time = target;
    reached = true;
    return LP_OK;
  }
};

// ---------------------------------------------------------------- fixtures.rs
struct Fixture {
  lp_fixture_spec spec;
  Material mat;
};

int64_t axis_count(double size, double spacing) {
  double sub = spacing / 2.0;
  return (int64_t)std::fmax(std::round(size / sub), 1.0);
}

// fixtures.rs:152-229
bool validate_spec(const lp_fixture_spec& s, std::string& err) {
  for (int a = 0; a < 3; ++a) {
    if (s.initial_size[a] > s.domain[a] + 1e-12) {
      err = "`initial_size_m` exceeds `domain_m`";
      return false;
    }
    if (s.initial_size[a] < s.grid_spacing) {
      err = "`initial_size_m` must span at least one cell";
      return false;
    }
  }
  double count = 1;
  for (int a = 0; a < 3; ++a) count *= (double)axis_count(s.initial_size[a], s.grid_spacing);
  if (count > (double)s.max_particles) {
    err = "fixture would allocate too many particles, exceeding the cap";
    return false;
  }
  switch (s.fixture) {
    case LP_HYDROSTATIC:
      for (int a = 0; a < 2; ++a)
        if (std::fabs(s.initial_size[a] - s.domain[a]) > 1e-9) {
          err = "`hydrostatic` requires `initial_size_m` to equal `domain_m` so the column spans the domain";
          return false;
        }
      if (norm(v3(s.initial_velocity[0], s.initial_velocity[1], s.initial_velocity[2])) > 0.0) {
        err = "`hydrostatic` requires zero `initial_velocity_m_s`";
        return false;
      }
      if (s.initial_size[2] >= s.domain[2]) {
        err = "`hydrostatic` requires free space above the column";
        return false;
      }
      break;
    case LP_COUPLED_PATCH: {
      if (!s.has_pellet) {
        err = "`coupled_patch` requires exactly one box supplying pellet geometry";
        return false;
      }
      if (s.material.kind != LP_PASTE) {
        err = "`coupled_patch` is implemented for `paste` only";
        return false;
      }
      if (s.pellet_radius < 1.5 * s.grid_spacing) {
        err = "`pellet_radius_m` is under-resolved";
        return false;
      }
      double top = s.initial_size[2] + 2.0 * s.grid_spacing + 2.0 * s.pellet_radius;
      if (top > s.domain[2] || s.pellet_length > s.domain[0] || 2.0 * s.pellet_radius > s.domain[1]) {
        err = "`coupled_patch` pellet does not fit above the block inside `domain_m`";
        return false;
      }
      break;
    }
    default:
      if (s.has_pellet && !(s.fixture == LP_SLUMP && s.bed_count >= 2)) {
        err = "fixture does not accept boxes; only `coupled_patch` uses pellet geometry";
        return false;
      }
  }
  if (s.bed_count >= 2) {
    if (s.fixture != LP_SLUMP || !s.has_pellet || s.bed_count > 4096) {
      err = "a pellet bed needs the slump fixture, a pellet geometry and at most 4096 pellets";
      return false;
    }
    if (s.bed_law == LP_BED_LINEAR) {
      if (!(std::isfinite(s.dem_stiffness) && s.dem_stiffness > 0.0) ||
          !(std::isfinite(s.dem_rolling) && s.dem_rolling >= 0.0) || !(s.hm_friction >= 0.0) ||
          !std::isfinite(s.hm_restitution)) {
        err = "invalid linear contact parameters (stiffness > 0, rolling friction >= 0, friction >= 0, finite restitution)";
        return false;
      }
    } else if (s.bed_law != LP_BED_HERTZ_MINDLIN) {
      err = "unknown pellet-bed contact law";
      return false;
    } else if (!(s.hm_young > 0.0) || !(s.hm_poisson >= 0.0 && s.hm_poisson < 0.5) || !(s.hm_friction >= 0.0) ||
               !(s.hm_restitution > 0.0 && s.hm_restitution <= 1.0)) {
      err = "invalid Hertz-Mindlin parameters (young > 0, 0 <= poisson < 0.5, friction >= 0, 0 < restitution <= 1)";
      return false;
    }
  }
  return true;
}

// Damping parameter of the Hertz-Mindlin normal force, calibrated so that a head-on impact
// rebounds with restitution e: in scaled units the overlap obeys
// x'' = -max(x^1.5 + c x^0.25 x', 0), c = -sqrt(5) beta, x(0) = 0, x'(0) = 1, independent of
// speed, masses and moduli; e = -x' at separation (RK4, step 2e-4), bisection on beta.
// ContactParams::damping_ratio (dem.rs:112-120)
static double dem_damping_ratio(double e) {
  e = std::fmin(std::fmax(e, 0.0), 1.0);
  if (e <= std::numeric_limits<double>::epsilon()) return 1.0;
  const double l = std::log(e);
  return std::fmin(-l / std::sqrt(M_PI * M_PI + l * l), 1.0);
}

static double hm_restitution_of(double beta) {
  const double c = -std::sqrt(5.0) * beta, h = 2e-4;
  auto acc = [c](double x, double v) {
    if (x <= 0.0) return 0.0;
    const double f = std::pow(x, 1.5) + c * std::pow(x, 0.25) * v;
    return f > 0.0 ? -f : 0.0;
  };
  double x = 0.0, v = 1.0;
  for (int n = 1; n <= 1000000; ++n) {
    const double k1x = v, k1v = acc(x, v);
    const double k2x = v + 0.5 * h * k1v, k2v = acc(x + 0.5 * h * k1x, v + 0.5 * h * k1v);
    const double k3x = v + 0.5 * h * k2v, k3v = acc(x + 0.5 * h * k2x, v + 0.5 * h * k2v);
    const double k4x = v + h * k3v, k4v = acc(x + h * k3x, v + h * k3v);
    x += h / 6.0 * (k1x + 2.0 * k2x + 2.0 * k3x + k4x);
    v += h / 6.0 * (k1v + 2.0 * k2v + 2.0 * k3v + k4v);
    if (x <= 0.0) break;
  }
  return -v;
}
static double hm_beta_for(double e) {
  if (e >= 1.0) return 0.0;
  double lo = -20.0, hi = 0.0;
  for (int it = 0; it < 60; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (hm_restitution_of(mid) < e) lo = mid;
    else hi = mid;
  }
  return 0.5 * (lo + hi);
}

// Pellet bed placement (extension): per pellet, centre (x y z uniforms in [bed_lo, bed_hi]) then
// orientation (Shoemake: three uniforms) from one SplitMix64 stream seeded with bed_seed,
// redrawn until every sphere is a radius inside the walls and 2.02 radii from placed spheres.
bool make_bed(const lp_fixture_spec& s, const V3& extent, std::vector<Pellet>& bed, std::string& err) {
  SplitMix64 rng{s.bed_seed};
  Pellet proto;
  if (!make_pellet(s.pellet_radius, s.pellet_length, s.pellet_density, zero3(), proto, err)) return false;
  const double r = proto.radius;
  std::vector<V3> centres;
  bed.clear();
  for (int p = 0; p < s.bed_count; ++p) {
    bool placed = false;
    for (int attempt = 0; attempt < 10000 && !placed; ++attempt) {
      Pellet P = proto;
      for (int a = 0; a < 3; ++a) P.position[a] = s.bed_lo[a] + (s.bed_hi[a] - s.bed_lo[a]) * rng.next_unit();
      double u1 = rng.next_unit(), u2 = rng.next_unit(), u3 = rng.next_unit();
      double s1 = std::sqrt(1.0 - u1), s2 = std::sqrt(u1), t1 = 2.0 * kPi * u2, t2 = 2.0 * kPi * u3;
      P.q = Quat{s1 * std::sin(t1), s1 * std::cos(t1), s2 * std::sin(t2), s2 * std::cos(t2)};
      M3 R = qmatrix(P.q);
      std::vector<V3> mine;
      bool ok = true;
      for (size_t k = 0; k < P.offsets.size() && ok; ++k) {
        V3 c;
        for (int a = 0; a < 3; ++a) {
          c[a] = P.position[a] + R.a[a][0] * P.offsets[k];
          if (c[a] < r || c[a] > extent[a] - r) ok = false;
        }
        for (const V3& o : centres) {
          double dx = c[0] - o[0], dy = c[1] - o[1], dz = c[2] - o[2];
          if (dx * dx + dy * dy + dz * dz < (2.02 * r) * (2.02 * r)) ok = false;
        }
        mine.push_back(c);
      }
      if (!ok) continue;
      centres.insert(centres.end(), mine.begin(), mine.end());
      bed.push_back(P);
      placed = true;
    }
    if (!placed) {
      err = "pellet bed: pellet " + std::to_string(p) + " does not fit in the region without overlap after 10000 draws";
      return false;
    }
  }
  return true;
}

// fixtures.rs:238-349
bool build(const lp_fixture_spec& s, Simulation& sim, std::string& err) {
  if (!validate_spec(s, err)) return false;
  Layout L;
  if (!make_layout(s.domain, s.grid_spacing, s.max_nodes, L, err)) return false;
  Material mat = mat_from(s.material);
  SplitMix64 rng{s.seed};
  int64_t counts[3];
  for (int a = 0; a < 3; ++a) counts[a] = axis_count(s.initial_size[a], s.grid_spacing);
  double sub = s.grid_spacing / 2.0;
  V3 origin = zero3();
  if (s.fixture == LP_SLUMP || s.fixture == LP_COUPLED_PATCH)
    origin = v3(0.5 * (s.domain[0] - s.initial_size[0]), 0.5 * (s.domain[1] - s.initial_size[1]), 0.0);
  double jitter = s.fixture == LP_HYDROSTATIC ? 0.0 : 0.1 * sub;
  double height = s.initial_size[2];
  double gnorm = norm(v3(s.gravity[0], s.gravity[1], s.gravity[2]));
  V3 v0 = v3(s.initial_velocity[0], s.initial_velocity[1], s.initial_velocity[2]);
  Particles& P = sim.P;
  for (int64_t i = 0; i < counts[0]; ++i)
    for (int64_t j = 0; j < counts[1]; ++j)
      for (int64_t k = 0; k < counts[2]; ++k) {
        V3 pos = add(origin, v3(((double)i + 0.5) * sub, ((double)j + 0.5) * sub, ((double)k + 0.5) * sub));
        if (jitter > 0.0)
          for (int a = 0; a < 3; ++a) pos[a] += (rng.next_unit() - 0.5) * 2.0 * jitter;
        double cur = sub * sub * sub;
        double J = 1.0;
        M3 F = mident(), tau = mzero();
        if (s.fixture == LP_HYDROSTATIC) {
          double depth = height - pos[2];
          if (mat.kind == LP_LIQUID) {
            J = std::exp(-mat.density * gnorm * depth / mat.bulk);
            double pr = liquid_pressure(mat, J);
            tau = mscale(mident(), -pr * J);
          } else {
            double modulus = mat.lambda + 2.0 * mat.mu;
            double strain = -mat.density * gnorm * depth / modulus;
            double stretch = std::exp(strain);
            F = mdiag(v3(1.0, 1.0, stretch));
            tau = mdiag(v3(mat.lambda * strain, mat.lambda * strain, modulus * strain));
            J = stretch;
          }
        }
        double vol0 = cur / J;
        P.push(pos, v0, mat.density * vol0, vol0, mat.yield);
        size_t idx = P.size() - 1;
        P.J[idx] = J;
        P.F[idx] = F;
        P.tau[idx] = tau;
      }
  // extension: per-particle yield stress, drawn after placement in particle order
  if (s.yield_random) {
    for (size_t p = 0; p < P.size(); ++p) P.ys[p] = s.yield_min + (s.yield_max - s.yield_min) * rng.next_unit();
  }
  sim.mat = mat;
  sim.grid.init(L);
  sim.has_pellet = false;
  sim.bed.clear();
  sim.hist.clear();
  if (s.bed_count >= 2) {
    if (!make_bed(s, L.extents(), sim.bed, err)) return false;
    sim.hist.assign(sim.bed.size(), std::vector<HmEntry>());
    sim.hm_mu = s.hm_friction;
    sim.bed_law = s.bed_law;
    if (s.bed_law == LP_BED_LINEAR) {
      sim.dem_kn = s.dem_stiffness;
      sim.dem_zeta = dem_damping_ratio(s.hm_restitution);
      sim.dem_mur = s.dem_rolling;
    } else {
      const double nu = s.hm_poisson, E = s.hm_young, G = E / (2.0 * (1.0 + nu));
      sim.hm_estar = E / (2.0 * (1.0 - nu * nu));
      sim.hm_gstar = G / (2.0 * (2.0 - nu));
      sim.hm_beta = hm_beta_for(s.hm_restitution);
    }
    double hs = 0.0;
    for (double o : sim.bed[0].offsets) hs = std::fmax(hs, std::fabs(o));
    sim.bed_rb = hs + sim.bed[0].radius;
  }
  if (s.fixture == LP_COUPLED_PATCH && s.has_pellet) {
    V3 center = v3(0.5 * s.domain[0], 0.5 * s.domain[1], s.initial_size[2] + 2.0 * s.grid_spacing + s.pellet_radius);
    if (!make_pellet(s.pellet_radius, s.pellet_length, s.pellet_density, center, sim.pellet, err)) return false;
    sim.has_pellet = true;
  }
  Config& c = sim.cfg;
  c.gravity = v3(s.gravity[0], s.gravity[1], s.gravity[2]);
  c.friction = s.wall_friction;
  c.cfl = s.cfl;
  c.max_dt = s.max_dt;
  c.min_dt = s.min_dt;
  c.contact = Contact{s.contact_stiffness, s.contact_restitution, s.contact_friction};
  c.face_mode = s.face_mode_enabled != 0;
  for (int f = 0; f < 6; ++f) {
    c.sticky[f] = s.face_sticky[f] != 0;
    c.face_mu[f] = c.face_mode ? s.face_friction[f] : s.wall_friction;
  }
  c.tol = s.newton_tolerance > 0.0 ? s.newton_tolerance : 1e-12;
  // Simulation::new (solver.rs:357-394)
  V3 mom = P.linear_momentum();
  if (sim.has_pellet) mom = add(mom, mul(sim.pellet.velocity, sim.pellet.mass));
  for (const Pellet& b : sim.bed) mom = add(mom, mul(b.velocity, b.mass));
  sim.ledger = Ledger();
  sim.ledger.initial_mass = P.total_mass();
  sim.ledger.initial_momentum = mom;
  sim.ledger.initial_mech = sim.mechanical_energy();
  return true;
}

// audit.rs:214-243 EnergyTerms::measure
void audit_terms(lp_energy_audit& a) {
  const double* b = a.before;
  const double* f = a.after;
  const double* s = a.stages;
  const double p2g = b[0] + b[1] - s[0];
  const double g2p = s[5] - f[0] - f[1];
  const double stress = s[1] - s[0] + f[2] - b[2] + s[7];
  const double gravity = s[3] - s[2] + f[3] - b[3];
  const double integrator = f[4] - s[6];
  const double traction = s[2] - s[1];
  const double walls = s[4] - s[3];
  const double coupling = s[5] - s[4] + s[6] - b[4];
  const double change = (f[0] + f[1] + f[2] + f[3] + f[4]) - (b[0] + b[1] + b[2] + b[3] + b[4]);
  const double sum = -p2g - g2p + stress - s[7] + gravity + integrator + traction + walls + coupling;
  const double nan = std::numeric_limits<double>::quiet_NaN();
  const double t[12] = {p2g,      g2p,       stress, a.coupled ? nan : gravity, a.coupled ? gravity : nan,
                        integrator, traction, walls,  coupling, change, sum, change - sum};
  for (int k = 0; k < 12; ++k) a.terms[k] = t[k];
}

// audit.rs:284-353 Simulation::audit_step on a copy of the simulation
bool audit_step(const Simulation& sim, double dt, lp_energy_audit& out, std::string& err) {
  std::memset(&out, 0, sizeof(out));
  const Config& c = sim.cfg;
  const double stability = sim.stability_limit();
  if (!finite3(c.gravity) || !std::isfinite(c.cfl) || c.cfl <= 0.0 || !std::isfinite(c.friction) || c.friction < 0.0 ||
      !std::isfinite(c.min_dt) || c.min_dt <= 0.0 || !std::isfinite(c.max_dt) || c.max_dt < c.min_dt ||
      !std::isfinite(stability) || stability <= 0.0) {
    err = "invalid solver state: invalid audit step configuration or stability limit";
    return false;
  }
  const double limit = std::fmin(sim.dt_scale * stability, c.max_dt);
  if (!std::isfinite(dt) || dt <= 0.0 || dt < c.min_dt || !std::isfinite(limit) || dt > limit) {
    char buf[200];
    std::snprintf(buf, sizeof(buf), "invalid solver state: audit `dt`='%.17g' outside finite accepted range ending at '%.17g'",
                  dt, limit);
    err = buf;
    return false;
  }
  out.time = sim.time;
  out.dt = dt;
  out.coupled = (sim.has_pellet || !sim.bed.empty()) ? 1 : 0;
  sim.energy_state(out.before);
  for (double v : out.before)
    if (!std::isfinite(v)) {
      err = "invalid solver state: nonfinite initial audit energy";
      return false;
    }
  AuditStages st;
  st.transport = sim.transport_energy();
  Simulation trial = sim;
  trial.audit = &st;
  const int f = trial.try_step(dt);
  trial.audit = nullptr;
  if (f != SF_OK) {
    err = "invalid solver state: audit trial rejected: " + trial.last_failure;
    return false;
  }
  trial.energy_state(out.after);
  const double stg[8] = {st.transport, st.stress, st.traction, st.gravity, st.walls, st.coupling, st.pellet_after,
                         st.plastic};
  for (int k = 0; k < 8; ++k) out.stages[k] = stg[k];
  const Ledger& l0 = sim.ledger;
  const Ledger& l1 = trial.ledger;
  const double inc[7] = {l1.plastic - l0.plastic, l1.fric - l0.fric, l1.proj - l0.proj, l1.trac - l0.trac,
                         l1.cgrid - l0.cgrid, l1.cpellet - l0.cpellet, l1.pellet_work - l0.pellet_work};
  for (int k = 0; k < 7; ++k) out.increments[k] = inc[k];
  audit_terms(out);
  bool finite = true;
  for (double v : out.after) finite = finite && std::isfinite(v);
  for (double v : out.stages) finite = finite && std::isfinite(v);
  for (double v : out.increments) finite = finite && std::isfinite(v);
  for (int k = 0; k < 12; ++k)
    if (!((k == 3 && out.coupled) || (k == 4 && !out.coupled))) finite = finite && std::isfinite(out.terms[k]);
  if (!finite) {
    err = "invalid solver state: audit energy became nonfinite";
    return false;
  }
  return true;
}

// fixtures.rs:354-364
double hydrostatic_reference(const Simulation& sim, double depth) {
  double g = norm(sim.cfg.gravity);
  const Material& m = sim.mat;
  if (m.kind == LP_LIQUID) return m.bulk * (std::exp(m.density * g * depth / m.bulk) - 1.0);
  return m.density * g * depth;
}

// fixtures.rs:369-606
std::map<std::string, double> observables(const Fixture& fx, const Simulation& sim) {
  std::map<std::string, double> out;
  const lp_fixture_spec& s = fx.spec;
  const Particles& P = sim.P;
  double sub = s.grid_spacing / 2.0;
  out["mass_residual_kg"] = sim.mass_residual();
  out["momentum_residual_kg_m_s"] = norm(sim.momentum_residual());
  out["kinetic_energy_j"] = sim.kinetic_energy();
  out["potential_energy_j"] = sim.potential_energy();
  out["elastic_energy_j"] = sim.elastic_energy();
  out["mechanical_energy_j"] = sim.mechanical_energy();
  out["plastic_dissipation_j"] = sim.ledger.plastic;
  out["wall_normal_projection_energy_j"] = sim.ledger.proj;
  out["wall_friction_dissipation_j"] = sim.ledger.fric;
  out["wall_normal_traction_energy_j"] = sim.ledger.trac;
  out["energy_residual_j"] = sim.energy_residual();
  out["outflow_kg"] = sim.ledger.outflow_mass;
  out["particle_count"] = (double)P.size();
  out["step_count"] = (double)sim.step_count;
  out["limited_steps"] = (double)sim.limited_steps;
  out["rejected_steps"] = (double)sim.rejected_steps;
  out["min_dt_s"] = std::isfinite(sim.min_dt_used) ? sim.min_dt_used : 0.0;
  out["max_dt_s"] = sim.max_dt_used;
  double max_speed = 0.0, max_plastic = 0.0;
  size_t yielded = 0;
  for (size_t p = 0; p < P.size(); ++p) {
    max_speed = std::fmax(max_speed, norm(P.v[p]));
    max_plastic = std::fmax(max_plastic, P.ep[p]);
    if (P.ep[p] > 0.0) ++yielded;
  }
  out["max_speed_m_s"] = max_speed;
  out["max_plastic_strain"] = max_plastic;
  out["yielded_fraction"] = P.size() == 0 ? 0.0 : (double)yielded / (double)P.size();
  double inf = std::numeric_limits<double>::infinity();
  double min_x = inf, max_x = -inf, min_y = inf, max_y = -inf, max_z = -inf;
  for (size_t p = 0; p < P.size(); ++p) {
    min_x = std::fmin(min_x, P.x[p][0]);
    max_x = std::fmax(max_x, P.x[p][0]);
    min_y = std::fmin(min_y, P.x[p][1]);
    max_y = std::fmax(max_y, P.x[p][1]);
    max_z = std::fmax(max_z, P.x[p][2]);
  }
  double height = P.size() == 0 ? 0.0 : max_z + 0.5 * sub;
  out["height_m"] = height;
  out["spread_x_m"] = P.size() == 0 ? 0.0 : max_x - min_x + sub;
  out["spread_y_m"] = P.size() == 0 ? 0.0 : max_y - min_y + sub;
  double g = norm(sim.cfg.gravity);
  if (s.fixture == LP_SLUMP) {
    double h0 = s.initial_size[2];
    out["slump_m"] = h0 - height;
    double shear_yield = sim.mat.yield / std::sqrt(3.0);
    double tp = shear_yield / (sim.mat.density * g * h0);
    out["dimensionless_yield_stress"] = tp;
    double pashias;
    if (tp >= 0.5) pashias = 0.0;
    else if (tp <= 0.0) pashias = h0;
    else pashias = h0 * (1.0 - 2.0 * tp * (1.0 - std::log(2.0 * tp)));
    out["pashias_slump_m"] = pashias;
  } else if (s.fixture == LP_HYDROSTATIC) {
    double h0 = s.initial_size[2];
    double scale = sim.mat.density * g * h0;
    double sum_sq = 0.0, max_err = 0.0;
    for (size_t p = 0; p < P.size(); ++p) {
      double depth = std::fmax(h0 - P.x[p][2], 0.0);
      double reference = hydrostatic_reference(sim, depth);
      double measured = sim.mat.kind == LP_LIQUID ? liquid_pressure(sim.mat, P.J[p]) : -P.tau[p].a[2][2];
      double e = (measured - reference) / scale;
      sum_sq += e * e;
      max_err = std::fmax(max_err, std::fabs(e));
    }
    out["hydrostatic_rms_relative_error"] = P.size() == 0 ? 0.0 : std::sqrt(sum_sq / (double)P.size());
    out["hydrostatic_max_relative_error"] = max_err;
    out["reference_bottom_stress_pa"] = hydrostatic_reference(sim, h0);
    out["wave_speed_m_s"] = wave_speed(sim.mat);
  } else if (s.fixture == LP_DAM_BREAK) {
    out["front_x_m"] = P.size() == 0 ? 0.0 : max_x + 0.5 * sub;
    double ritter = s.initial_size[0] + 2.0 * std::sqrt(g * s.initial_size[2]) * sim.time;
    out["ritter_front_bound_m"] = std::fmin(ritter, s.domain[0]);
    double column = 0.0;
    for (size_t p = 0; p < P.size(); ++p)
      if (P.x[p][0] < s.grid_spacing) column = std::fmax(column, P.x[p][2] + 0.5 * sub);
    out["column_height_m"] = column;
  } else if (s.fixture == LP_COUPLED_PATCH && sim.has_pellet) {
    const Pellet& pl = sim.pellet;
    out["pellet_x_m"] = pl.position[0];
    out["pellet_y_m"] = pl.position[1];
    out["pellet_z_m"] = pl.position[2];
    out["pellet_speed_m_s"] = norm(pl.velocity);
    out["pellet_angular_speed_rad_s"] = norm(pl.angular_velocity());
    out["pellet_kinetic_energy_j"] = pl.kinetic_energy();
    out["pellet_penetration_m"] = std::fmax(s.initial_size[2] + pl.radius - pl.position[2], 0.0);
    V3 ax = pl.axis();
    out["pellet_axis_tilt_rad"] = std::asin(std::fmin(std::fabs(ax[2]), 1.0));
    const Ledger& l = sim.ledger;
    out["coupling_impulse_x_kg_m_s"] = l.coupling_impulse[0];
    out["coupling_impulse_y_kg_m_s"] = l.coupling_impulse[1];
    out["coupling_impulse_z_kg_m_s"] = l.coupling_impulse[2];
    out["coupling_angular_impulse_x_kg_m2_s"] = l.coupling_angular[0];
    out["coupling_angular_impulse_y_kg_m2_s"] = l.coupling_angular[1];
    out["coupling_angular_impulse_z_kg_m2_s"] = l.coupling_angular[2];
    out["pellet_wall_impulse_z_kg_m_s"] = l.pellet_wall_impulse[2];
    out["pellet_wall_work_j"] = l.pellet_work;
    out["coupling_grid_energy_j"] = l.cgrid;
    out["coupling_pellet_energy_j"] = l.cpellet;
  }
  if (!sim.bed.empty()) {
    double zs = 0.0, zmin = 1e300, vmax = 0.0, ke = 0.0;
    for (const Pellet& b : sim.bed) {
      zs += b.position[2];
      zmin = std::fmin(zmin, b.position[2]);
      vmax = std::fmax(vmax, norm(b.velocity));
      ke += b.kinetic_energy();
    }
    const Ledger& l = sim.ledger;
    out["pellet_count"] = (double)sim.bed.size();
    out["pellet_mean_z_m"] = zs / (double)sim.bed.size();
    out["pellet_min_z_m"] = zmin;
    out["pellet_max_speed_m_s"] = vmax;
    out["pellet_kinetic_energy_j"] = ke;
    out["pellet_contact_work_j"] = sim.bed_contact_work;
    out["pellet_contacts"] = (double)sim.bed_contacts;
    out["pellet_history_overflow"] = (double)sim.bed_overflow;
    out["pellet_wall_work_j"] = l.pellet_work;
    out["coupling_grid_energy_j"] = l.cgrid;
    out["coupling_pellet_energy_j"] = l.cpellet;
    out["coupling_impulse_z_kg_m_s"] = l.coupling_impulse[2];
  }
  return out;
}

void m3_out(const M3& m, double* dst) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) dst[3 * i + j] = m.a[i][j];
}
M3 m3_in(const double* src) {
  M3 m;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) m.a[i][j] = src[3 * i + j];
  return m;
}
void set_err(char* err, int32_t len, const std::string& msg) {
  if (err && len > 0) {
    std::snprintf(err, (size_t)len, "%s", msg.c_str());
  }
}

}  // namespace

struct ora_sim {
  Fixture fx;
  Simulation sim;
};

extern "C" {

int32_t ora_sim_create(const lp_fixture_spec* spec, ora_sim** out, char* err, int32_t errlen) {
  *out = nullptr;
  ora_sim* s = new ora_sim();
  s->fx.spec = *spec;
  std::string e;
  if (!build(*spec, s->sim, e)) {
    set_err(err, errlen, e);
    delete s;
    return LP_INVALID;
  }
  s->fx.mat = s->sim.mat;
  *out = s;
  return LP_OK;
}

void ora_sim_destroy(ora_sim* s) { delete s; }

int32_t ora_sim_advance(ora_sim* s, double target, int64_t max_accepted, int32_t* reached, char* err,
                        int32_t errlen) {
  bool r = false;
  std::string e;
  int st = s->sim.advance(target, max_accepted, r, e);
  if (reached) *reached = r ? 1 : 0;
  if (st != LP_OK) set_err(err, errlen, e);
  return st;
}

int32_t ora_sim_try_step(ora_sim* s, double dt, int32_t* accepted, char* reason, int32_t len) {
  int f = s->sim.try_step(dt);
  *accepted = f == SF_OK ? 1 : 0;
  if (f != SF_OK) set_err(reason, len, s->sim.last_failure);
  return LP_OK;
}

double ora_sim_stability_limit(ora_sim* s) { return s->sim.stability_limit(); }

int32_t ora_sim_audit_step(ora_sim* s, double dt, lp_energy_audit* out, char* err, int32_t errlen) {
  std::string e;
  if (!audit_step(s->sim, dt, *out, e)) {
    set_err(err, errlen, e);
    return LP_INVALID;
  }
  return LP_OK;
}

void ora_sim_counters(ora_sim* s, lp_counters* out) {
  const Simulation& m = s->sim;
  out->time = m.time;
  out->step_count = m.step_count;
  out->limited_steps = m.limited_steps;
  out->rejected_steps = m.rejected_steps;
  out->dt_scale = m.dt_scale;
  out->min_dt_used = m.min_dt_used;
  out->max_dt_used = m.max_dt_used;
  out->particle_count = m.P.size();
  out->newton_iterations = m.newton_iterations;
  out->yielded_particles = m.yielded;
}

int32_t ora_sim_set_counters(ora_sim* s, const lp_counters* in) {
  Simulation& m = s->sim;
  if (!(in->dt_scale > 0.0 && in->dt_scale <= 1.0) || !std::isfinite(in->time) || in->time < 0.0) return LP_INVALID;
  m.time = in->time;
  m.step_count = in->step_count;
  m.limited_steps = in->limited_steps;
  m.rejected_steps = in->rejected_steps;
  m.dt_scale = in->dt_scale;
  m.min_dt_used = in->min_dt_used;
  m.max_dt_used = in->max_dt_used;
  return LP_OK;
}

static void v3_out(const V3& v, double* d) {
  d[0] = v[0];
  d[1] = v[1];
  d[2] = v[2];
}
static V3 v3_in(const double* d) { return v3(d[0], d[1], d[2]); }

void ora_sim_ledger(ora_sim* s, lp_ledger* o) {
  const Ledger& l = s->sim.ledger;
  o->initial_mass = l.initial_mass;
  o->outflow_mass = l.outflow_mass;
  v3_out(l.initial_momentum, o->initial_momentum);
  o->initial_mechanical_energy = l.initial_mech;
  v3_out(l.gravity_impulse, o->gravity_impulse);
  v3_out(l.wall_impulse, o->wall_impulse);
  v3_out(l.pellet_wall_impulse, o->pellet_wall_impulse);
  v3_out(l.coupling_impulse, o->coupling_impulse);
  v3_out(l.coupling_angular, o->coupling_angular_impulse);
  o->wall_normal_projection_energy = l.proj;
  o->wall_friction_dissipation = l.fric;
  o->wall_normal_traction_energy = l.trac;
  o->pellet_wall_work = l.pellet_work;
  o->coupling_grid_energy = l.cgrid;
  o->coupling_pellet_energy = l.cpellet;
  o->plastic_dissipation = l.plastic;
  v3_out(l.outflow_momentum, o->outflow_momentum);
}

void ora_sim_set_ledger(ora_sim* s, const lp_ledger* o) {
  Ledger& l = s->sim.ledger;
  l.initial_mass = o->initial_mass;
  l.outflow_mass = o->outflow_mass;
  l.initial_momentum = v3_in(o->initial_momentum);
  l.initial_mech = o->initial_mechanical_energy;
  l.gravity_impulse = v3_in(o->gravity_impulse);
  l.wall_impulse = v3_in(o->wall_impulse);
  l.pellet_wall_impulse = v3_in(o->pellet_wall_impulse);
  l.coupling_impulse = v3_in(o->coupling_impulse);
  l.coupling_angular = v3_in(o->coupling_angular_impulse);
  l.proj = o->wall_normal_projection_energy;
  l.fric = o->wall_friction_dissipation;
  l.trac = o->wall_normal_traction_energy;
  l.pellet_work = o->pellet_wall_work;
  l.cgrid = o->coupling_grid_energy;
  l.cpellet = o->coupling_pellet_energy;
  l.plastic = o->plastic_dissipation;
  l.outflow_momentum = v3_in(o->outflow_momentum);
}

uint64_t ora_sim_particle_count(ora_sim* s) { return s->sim.P.size(); }

void ora_sim_export_particles(ora_sim* s, lp_particles* o) {
  const Particles& P = s->sim.P;
  size_t n = std::min<size_t>(P.size(), (size_t)o->count);
  for (size_t p = 0; p < n; ++p) {
    if (o->id) o->id[p] = P.id[p];
    if (o->position) v3_out(P.x[p], o->position + 3 * p);
    if (o->velocity) v3_out(P.v[p], o->velocity + 3 * p);
    if (o->affine) m3_out(P.C[p], o->affine + 9 * p);
    if (o->deformation) m3_out(P.F[p], o->deformation + 9 * p);
    if (o->volume_ratio) o->volume_ratio[p] = P.J[p];
    if (o->kirchhoff) m3_out(P.tau[p], o->kirchhoff + 9 * p);
    if (o->plastic_strain) o->plastic_strain[p] = P.ep[p];
    if (o->mass) o->mass[p] = P.m[p];
    if (o->volume0) o->volume0[p] = P.V0[p];
    if (o->yield_stress) o->yield_stress[p] = P.ys[p];
  }
  o->count = n;
}

int32_t ora_sim_import_particles(ora_sim* s, const lp_particles* in) {
  Particles P;
  for (size_t p = 0; p < in->count; ++p) {
    P.id.push_back(in->id[p]);
    P.x.push_back(v3_in(in->position + 3 * p));
    P.v.push_back(v3_in(in->velocity + 3 * p));
    P.C.push_back(m3_in(in->affine + 9 * p));
    P.F.push_back(m3_in(in->deformation + 9 * p));
    P.J.push_back(in->volume_ratio[p]);
    P.tau.push_back(m3_in(in->kirchhoff + 9 * p));
    P.ep.push_back(in->plastic_strain[p]);
    P.m.push_back(in->mass[p]);
    P.V0.push_back(in->volume0[p]);
    P.ys.push_back(in->yield_stress ? in->yield_stress[p] : s->sim.mat.yield);
  }
  s->sim.P = P;
  return LP_OK;
}

int32_t ora_sim_get_pellet(ora_sim* s, lp_pellet* o) {
  if (!s->sim.has_pellet) return 0;
  const Pellet& p = s->sim.pellet;
  std::memset(o, 0, sizeof(*o));
  o->radius = p.radius;
  o->length = p.length;
  o->mass = p.mass;
  v3_out(p.inertia, o->inertia_body);
  v3_out(p.position, o->position);
  o->orientation[0] = p.q.i;
  o->orientation[1] = p.q.j;
  o->orientation[2] = p.q.k;
  o->orientation[3] = p.q.w;
  v3_out(p.velocity, o->velocity);
  v3_out(p.L, o->angular_momentum);
  o->sphere_count = (int32_t)p.offsets.size();
  for (size_t i = 0; i < p.offsets.size(); ++i) o->sphere_offsets[i] = p.offsets[i];
  return 1;
}

void ora_sim_set_pellet(ora_sim* s, const lp_pellet* o) {
  Pellet& p = s->sim.pellet;
  p.radius = o->radius;
  p.length = o->length;
  p.mass = o->mass;
  p.inertia = v3_in(o->inertia_body);
  p.position = v3_in(o->position);
  p.q = Quat{o->orientation[0], o->orientation[1], o->orientation[2], o->orientation[3]};
  p.velocity = v3_in(o->velocity);
  p.L = v3_in(o->angular_momentum);
  p.offsets.assign(o->sphere_offsets, o->sphere_offsets + o->sphere_count);
  s->sim.has_pellet = true;
}

int32_t ora_sim_get_pellets(ora_sim* s, lp_pellet* out, int32_t cap) {
  const std::vector<Pellet>& B = s->sim.bed;
  for (int32_t i = 0; i < std::min<int32_t>(cap, (int32_t)B.size()); ++i) {
    const Pellet& p = B[i];
    lp_pellet* o = out + i;
    std::memset(o, 0, sizeof(*o));
    o->radius = p.radius;
    o->length = p.length;
    o->mass = p.mass;
    v3_out(p.inertia, o->inertia_body);
    v3_out(p.position, o->position);
    o->orientation[0] = p.q.i;
    o->orientation[1] = p.q.j;
    o->orientation[2] = p.q.k;
    o->orientation[3] = p.q.w;
    v3_out(p.velocity, o->velocity);
    v3_out(p.L, o->angular_momentum);
    o->sphere_count = (int32_t)p.offsets.size();
    for (size_t k = 0; k < p.offsets.size(); ++k) o->sphere_offsets[k] = p.offsets[k];
  }
  return (int32_t)B.size();
}

int32_t ora_sim_set_pellets(ora_sim* s, const lp_pellet* in, int32_t count) {
  std::vector<Pellet>& B = s->sim.bed;
  if (count != (int32_t)B.size()) return LP_INVALID;
  for (int32_t i = 0; i < count; ++i) {
    B[i].position = v3_in(in[i].position);
    B[i].velocity = v3_in(in[i].velocity);
    B[i].L = v3_in(in[i].angular_momentum);
    B[i].q = Quat{in[i].orientation[0], in[i].orientation[1], in[i].orientation[2], in[i].orientation[3]};
  }
  s->sim.hist.assign(B.size(), std::vector<HmEntry>());
  return LP_OK;
}

int32_t ora_sim_observables(ora_sim* s, char* names, double* values, int32_t capacity) {
  auto obs = observables(s->fx, s->sim);
  int32_t n = 0;
  for (auto& kv : obs) {
    if (n >= capacity) break;
    std::snprintf(names + 64 * n, 64, "%s", kv.first.c_str());
    values[n] = kv.second;
    ++n;
  }
  return n;
}

void ora_sim_energies(ora_sim* s, double out[9]) {
  const Simulation& m = s->sim;
  out[0] = m.kinetic_energy();
  out[1] = m.potential_energy();
  out[2] = m.elastic_energy();
  out[3] = m.mechanical_energy();
  out[4] = m.mass_residual();
  V3 r = m.momentum_residual();
  out[5] = r[0];
  out[6] = r[1];
  out[7] = r[2];
  out[8] = m.energy_residual();
}

void ora_set_threads(int32_t threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
}

// deposit_particles (solver.rs:632-661) then wall_traction_to_grid (solver.rs:725-819) on a copy:
// node mass, node momentum without the wall reactions, and the signed reaction impulse each node
// received (Grid::deposit_reaction, grid.rs:279-295: impulse = inward_impulse * inward, so the
// reference's post-traction momentum is momentum + reaction).
int64_t ora_sim_probe_grid(ora_sim* s, double dt, double* mass, double* momentum, double* reaction) {
  Simulation copy = s->sim;
  copy.sweep_outflow();
  copy.deposit_particles(dt);
  const int64_t n = copy.grid.layout.node_count();
  if (momentum)
    for (int64_t i = 0; i < n; ++i) v3_out(copy.grid.momentum[i], momentum + 3 * i);
  V3 imp;
  double e;
  copy.wall_traction(dt, imp, e);
  if (mass)
    for (int64_t i = 0; i < n; ++i) mass[i] = copy.grid.mass[i];
  if (reaction)
    for (int64_t i = 0; i < n; ++i)
      v3_out(sub(copy.grid.traction_low[i], copy.grid.traction_high[i]), reaction + 3 * i);
  return (int64_t)copy.grid.active.size();
}

int64_t ora_sim_probe_p2g(ora_sim* s, double dt, double* mass, double* momentum, double* traction_energy,
                          double traction_impulse[3]) {
  Simulation copy = s->sim;
  copy.sweep_outflow();
  copy.deposit_particles(dt);
  V3 imp;
  double e;
  copy.wall_traction(dt, imp, e);
  int64_t n = copy.grid.layout.node_count();
  if (mass)
    for (int64_t i = 0; i < n; ++i) mass[i] = copy.grid.mass[i];
  if (momentum)
    for (int64_t i = 0; i < n; ++i) v3_out(copy.grid.momentum[i], momentum + 3 * i);
  if (traction_energy) *traction_energy = e;
  if (traction_impulse) v3_out(imp, traction_impulse);
  return (int64_t)copy.grid.active.size();
}

int32_t ora_hb_return(double trial, double yield, double consistency, double flow_index, double mu, double dt,
                      double tol_rel, double out[3]) {
  ReturnSolution r{0, 0, 0};
  int e = hb_return(trial, yield, consistency, flow_index, mu, dt, tol_rel > 0 ? tol_rel : 1e-12, r);
  out[0] = r.sigma;
  out[1] = r.dep;
  out[2] = r.iterations;
  return e;
}

int32_t ora_update_paste(const double f_trial[9], const lp_material* m, double yield_override, double dt,
                         double tol_rel, double f_new[9], double tau[9], double out[3]) {
  Material mat = mat_from(*m);
  PasteUpdate u;
  double ys = yield_override >= 0.0 ? yield_override : mat.yield;
  int e = update_paste(m3_in(f_trial), mat, ys, dt, tol_rel > 0 ? tol_rel : 1e-12, u);
  if (e != CE_OK) return e;
  m3_out(u.deformation, f_new);
  m3_out(u.kirchhoff, tau);
  out[0] = u.dep;
  out[1] = u.dissipation_density;
  out[2] = u.equivalent;
  return CE_OK;
}

int32_t ora_update_liquid(double volume_ratio, const double grad[9], const lp_material* m, double dt, double* j_new,
                          double tau[9], double* pressure) {
  LiquidUpdate u;
  int e = update_liquid(volume_ratio, m3_in(grad), mat_from(*m), dt, u);
  if (e != CE_OK) return e;
  *j_new = u.j;
  m3_out(u.kirchhoff, tau);
  *pressure = u.pressure;
  return CE_OK;
}

int32_t ora_eigen3(const double m[9], double values[3], double vectors[9]) {
  V3 ev;
  M3 u;
  if (!symmetric_eigen3(m3_in(m), ev, u)) return 1;
  v3_out(ev, values);
  m3_out(u, vectors);
  return 0;
}

int32_t ora_stencil(double spacing, const int32_t nodes[3], const double x[3], int32_t base[3], double weights[9],
                    double offsets[9]) {
  Layout L;
  L.spacing = spacing;
  for (int a = 0; a < 3; ++a) {
    L.nodes[a] = nodes[a];
    L.cells[a] = nodes[a] - 3;
  }
  Stencil s;
  if (!stencil_of(L, v3_in(x), s)) return 1;
  for (int a = 0; a < 3; ++a) {
    base[a] = (int32_t)s.base[a];
    for (int o = 0; o < 3; ++o) {
      weights[3 * a + o] = s.w[a][o];
      offsets[3 * a + o] = s.off[a][o];
    }
  }
  return 0;
}

double ora_splitmix_next_unit(uint64_t* state) {
  SplitMix64 r{*state};
  double u = r.next_unit();
  *state = r.state;
  return u;
}
uint64_t ora_splitmix_next_u64(uint64_t* state) {
  SplitMix64 r{*state};
  uint64_t u = r.next_u64();
  *state = r.state;
  return u;
}

lp_material ora_material_paste(double density, double e, double nu, double ys, double k, double n) {
  return mat_to(paste(density, e, nu, ys, k, n));
}
lp_material ora_material_paste_shear(double density, double e, double nu, double tys, double ks, double n) {
  return mat_to(paste_shear(density, e, nu, tys, ks, n));
}
lp_material ora_material_liquid(double density, double e, double nu, double visc) {
  return mat_to(liquid(density, e, nu, visc));
}

int32_t ora_grid_update_node(const lp_fixture_spec* spec, const int32_t coords[3], double mass,
                             const double momentum[3], const double traction[3], double dt, double out[8]) {
  ora_sim* s = nullptr;
  char err[256];
  lp_fixture_spec sp = *spec;
  Simulation sim;
  Layout L;
  std::string e;
  if (!make_layout(sp.domain, sp.grid_spacing, sp.max_nodes, L, e)) return 1;
  (void)s;
  (void)err;
  sim.grid.init(L);
  sim.cfg.gravity = v3(sp.gravity[0], sp.gravity[1], sp.gravity[2]);
  sim.cfg.friction = sp.wall_friction;
  sim.cfg.face_mode = sp.face_mode_enabled != 0;
  for (int f = 0; f < 6; ++f) {
    sim.cfg.sticky[f] = sp.face_sticky[f] != 0;
    sim.cfg.face_mu[f] = sim.cfg.face_mode ? sp.face_friction[f] : sp.wall_friction;
  }
  int64_t idx = L.index(coords[0], coords[1], coords[2]);
  sim.grid.mass[idx] = mass;
  sim.grid.momentum[idx] = v3_in(momentum);
  sim.grid.traction[idx] = v3_in(traction);
  sim.grid.traction_low[idx] = v3_in(traction);
  NodeTrial t;
  if (!sim.update_node(idx, dt, t)) return 2;
  v3_out(t.velocity, out);
  v3_out(t.wall_impulse, out + 3);
  out[6] = t.proj;
  out[7] = t.fric;
  return 0;
}

}  // extern "C"
