// lp_host.cu - host runtime and C ABI (include/lp_mpm.h) of the B200 MLS-MPM substep.
//
// The runtime owns every device buffer of an "ensemble" (one simulation, or a batch of
// independent simulations sharing one launch sequence), builds fixtures (setup only, host FP64
// restatement of fixtures.rs:272-349 so that GPU and reference start from identical seeded
// inputs), drives advance_while's loop in chunks of device-controlled attempts (optionally
// replayed from a CUDA graph), and converts state to and from the reference's FP64 particle
// layout at the boundary.  It never computes a substep on the host: without a CUDA device every
// entry point that needs one fails with LP_DEVICE.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lp_mpm.h"
#include "lp_kernels.h"

using lp::Control;
using lp::InstDesc;

namespace {

thread_local std::string g_err;

lp_status set_error(lp_status s, const std::string& msg) {
  g_err = msg;
  return s;
}

#define CUDA_CK(expr)                                                                                   \
  do {                                                                                                  \
    cudaError_t _e = (expr);                                                                            \
    if (_e != cudaSuccess) return set_error(LP_DEVICE, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------- SplitMix64 (rng.rs:35-47)
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

// ---------------------------------------------------------------- host fixture
struct HostParticles {
  std::vector<double> x, v, H, tau;  // 3, 3, 9 (F - I), 9 per particle
  std::vector<double> jm1, m, V0, ys;
  std::vector<uint32_t> id;
  size_t size() const { return id.size(); }
};

struct HostInstance {
  lp_fixture_spec spec;
  int64_t cells[3], nodes[3];
  HostParticles P;
  bool has_pellet = false;
  lp::PelletState pellet;
  std::vector<lp::PelletState> bed;  // pellet bed (extension)
};

int64_t axis_count(double size, double spacing) {
  double sub = spacing / 2.0;
  return (int64_t)std::fmax(std::round(size / sub), 1.0);
}

// grid.rs:105-154
lp_status make_layout(const lp_fixture_spec& s, HostInstance& h) {
  if (!(std::isfinite(s.grid_spacing) && s.grid_spacing > 0.0))
    return set_error(LP_INVALID, "`grid_spacing_m` must be positive and finite");
  double total = 1.0;
  for (int a = 0; a < 3; ++a) {
    double extent = s.domain[a];
    if (!(std::isfinite(extent) && extent > 0.0)) return set_error(LP_INVALID, "`domain_m` must be positive and finite");
    double ratio = extent / s.grid_spacing, rounded = std::round(ratio);
    if (!std::isfinite(ratio) || rounded > 4294967295.0)
      return set_error(LP_INVALID, "grid axis exceeds the node allocation cap");
    if (std::fabs(ratio - rounded) > 1e-6 * std::fmax(rounded, 1.0))
      return set_error(LP_INVALID, "`domain_m` is not an integer multiple of `grid_spacing_m`");
    if (rounded < 2.0) return set_error(LP_INVALID, "`domain_m` must span at least two cells");
    h.cells[a] = (int64_t)rounded;
    h.nodes[a] = h.cells[a] + 3;
    total *= (double)h.nodes[a];
  }
  if (total > (double)s.max_nodes) return set_error(LP_INVALID, "grid would allocate too many nodes, exceeding the cap");
  return LP_OK;
}

// fixtures.rs:152-229
lp_status validate_spec(const lp_fixture_spec& s) {
  for (int a = 0; a < 3; ++a) {
    if (s.initial_size[a] > s.domain[a] + 1e-12) return set_error(LP_INVALID, "`initial_size_m` exceeds `domain_m`");
    if (s.initial_size[a] < s.grid_spacing) return set_error(LP_INVALID, "`initial_size_m` must span at least one cell");
  }
  double count = 1.0;
  for (int a = 0; a < 3; ++a) count *= (double)axis_count(s.initial_size[a], s.grid_spacing);
  if (count > (double)s.max_particles)
    return set_error(LP_INVALID, "fixture would allocate too many particles, exceeding the cap");
  if (count > 2147483647.0) return set_error(LP_INVALID, "particle count exceeds the 32-bit slot range");
  const double m = s.material.kind;
  if (m != LP_PASTE && m != LP_LIQUID) return set_error(LP_INVALID, "unknown material kind");
  switch (s.fixture) {
    case LP_HYDROSTATIC: {
      for (int a = 0; a < 2; ++a)
        if (std::fabs(s.initial_size[a] - s.domain[a]) > 1e-9)
          return set_error(LP_INVALID,
                           "`hydrostatic` requires `initial_size_m` to equal `domain_m` so the column spans the domain");
      double v2 = 0;
      for (int a = 0; a < 3; ++a) v2 += s.initial_velocity[a] * s.initial_velocity[a];
      if (v2 > 0.0) return set_error(LP_INVALID, "`hydrostatic` requires zero `initial_velocity_m_s`");
      if (s.initial_size[2] >= s.domain[2]) return set_error(LP_INVALID, "`hydrostatic` requires free space above the column");
      if (s.material.kind == LP_LIQUID && s.material.tait_gamma != 0.0 && s.material.tait_gamma != 1.0)
        return set_error(LP_UNSUPPORTED, "`hydrostatic` prestress is defined for the linear EOS only");
      break;
    }
    case LP_COUPLED_PATCH: {
      if (!s.has_pellet) return set_error(LP_INVALID, "`coupled_patch` requires exactly one box supplying pellet geometry");
      if (s.material.kind != LP_PASTE) return set_error(LP_INVALID, "`coupled_patch` is implemented for `paste` only");
      if (s.pellet_radius < 1.5 * s.grid_spacing) return set_error(LP_INVALID, "`pellet_radius_m` is under-resolved");
      double top = s.initial_size[2] + 2.0 * s.grid_spacing + 2.0 * s.pellet_radius;
      if (top > s.domain[2] || s.pellet_length > s.domain[0] || 2.0 * s.pellet_radius > s.domain[1])
        return set_error(LP_INVALID, "`coupled_patch` pellet does not fit above the block inside `domain_m`");
      break;
    }
    case LP_SLUMP:
    case LP_DAM_BREAK:
      if (s.has_pellet && !(s.fixture == LP_SLUMP && s.bed_count >= 2))
        return set_error(LP_INVALID, "fixture does not accept boxes; only `coupled_patch` uses pellet geometry");
      break;
    default:
      return set_error(LP_INVALID, "unknown fixture");
  }
  if (s.bed_count >= 2) {
    if (s.fixture != LP_SLUMP || !s.has_pellet)
      return set_error(LP_UNSUPPORTED, "a pellet bed needs the slump fixture and a pellet geometry");
    if (s.bed_count > lp::BED_MAX) return set_error(LP_INVALID, "pellet bed exceeds 4096 pellets per simulation");
    for (int a = 0; a < 3; ++a)
      if (!(std::isfinite(s.bed_lo[a]) && std::isfinite(s.bed_hi[a]) && s.bed_lo[a] <= s.bed_hi[a] &&
            s.bed_lo[a] >= 0.0 && s.bed_hi[a] <= s.domain[a]))
        return set_error(LP_INVALID, "pellet bed region must lie inside `domain_m`");
    if (s.bed_law == LP_BED_LINEAR) {
      if (!(std::isfinite(s.dem_stiffness) && s.dem_stiffness > 0.0) ||
          !(std::isfinite(s.dem_rolling) && s.dem_rolling >= 0.0) ||
          !(std::isfinite(s.hm_friction) && s.hm_friction >= 0.0) || !std::isfinite(s.hm_restitution))
        return set_error(LP_INVALID, "invalid linear contact parameters (stiffness > 0, rolling friction >= 0, "
                                     "friction >= 0, finite restitution)");
    } else if (s.bed_law != LP_BED_HERTZ_MINDLIN) {
      return set_error(LP_INVALID, "unknown pellet-bed contact law");
    } else if (!(std::isfinite(s.hm_young) && s.hm_young > 0.0) || !(s.hm_poisson >= 0.0 && s.hm_poisson < 0.5) ||
               !(std::isfinite(s.hm_friction) && s.hm_friction >= 0.0) ||
               !(s.hm_restitution > 0.0 && s.hm_restitution <= 1.0)) {
      return set_error(LP_INVALID, "invalid Hertz-Mindlin parameters (young > 0, 0 <= poisson < 0.5, "
                                   "friction >= 0, 0 < restitution <= 1)");
    }
  }
  return LP_OK;
}

// Damping of the Hertz-Mindlin normal force, F = (4/3) E* sqrt(R*) d^1.5 - gamma v_n with
// gamma = -2 sqrt(5/6) beta sqrt(2 E* sqrt(R* d) m*), calibrated so that a head-on impact
// rebounds with the requested restitution e.  In scaled units the overlap obeys
// x'' = -max(x^1.5 + c x^0.25 x', 0), c = -sqrt(5) beta, x(0) = 0, x'(0) = 1, whatever the
// impact speed, masses and moduli (the damping scales with the contact stiffness), and
// e = -x' when the spheres separate.  The closed form beta = ln e / sqrt(ln^2 e + pi^2) of the
// linear spring-dashpot would give e = 0.40 for a requested 0.3 under Hertz contact.
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
  double lo = -20.0, hi = 0.0;  // restitution rises from lo to hi
  for (int it = 0; it < 60; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (hm_restitution_of(mid) < e) lo = mid;
    else hi = mid;
  }
  return 0.5 * (lo + hi);
}

lp_status make_pellet(double r, double len, double rho, const double pos[3], lp::PelletState& p);
void q_matrix(const double* q, double R[3][3]);

// Pellet bed placement (extension).  Pellet p draws its centre (three uniforms, x y z) and then
// its orientation (three uniforms, Shoemake's uniform random rotation: q = (sqrt(1-u1) sin 2pi u2,
// sqrt(1-u1) cos 2pi u2, sqrt(u1) sin 2pi u3, sqrt(u1) cos 2pi u3) as (i, j, k, w)) from one
// SplitMix64 stream seeded with bed_seed, and redraws until every sphere lies at least one
// radius inside the walls and at least 2.02 radii from every sphere of the pellets placed so far.
lp_status make_bed(const lp_fixture_spec& s, const double extent[3], std::vector<lp::PelletState>& bed) {
  SplitMix64 rng{s.bed_seed};
  bed.clear();
  const double zero[3] = {0.0, 0.0, 0.0};
  lp::PelletState proto;
  lp_status st = make_pellet(s.pellet_radius, s.pellet_length, s.pellet_density, zero, proto);
  if (st != LP_OK) return st;
  const double r = proto.radius;
  std::vector<double> centres;  // 3 per placed sphere
  for (int p = 0; p < s.bed_count; ++p) {
    bool placed = false;
    for (int attempt = 0; attempt < 10000 && !placed; ++attempt) {
      lp::PelletState P = proto;
      for (int a = 0; a < 3; ++a) P.pos[a] = s.bed_lo[a] + (s.bed_hi[a] - s.bed_lo[a]) * rng.next_unit();
      const double u1 = rng.next_unit(), u2 = rng.next_unit(), u3 = rng.next_unit();
      const double s1 = std::sqrt(1.0 - u1), s2 = std::sqrt(u1), t1 = 2.0 * kPi * u2, t2 = 2.0 * kPi * u3;
      P.q[0] = s1 * std::sin(t1);
      P.q[1] = s1 * std::cos(t1);
      P.q[2] = s2 * std::sin(t2);
      P.q[3] = s2 * std::cos(t2);
      double R[3][3];
      q_matrix(P.q, R);
      std::vector<double> mine;
      bool ok = true;
      for (int k = 0; k < P.nsph && ok; ++k) {
        double c[3];
        for (int a = 0; a < 3; ++a) {
          c[a] = P.pos[a] + R[a][0] * P.off[k];
          if (c[a] < r || c[a] > extent[a] - r) ok = false;
        }
        for (size_t o = 0; o < centres.size() && ok; o += 3) {
          const double dx = c[0] - centres[o], dy = c[1] - centres[o + 1], dz = c[2] - centres[o + 2];
          if (dx * dx + dy * dy + dz * dz < (2.02 * r) * (2.02 * r)) ok = false;
        }
        mine.insert(mine.end(), c, c + 3);
      }
      if (!ok) continue;
      centres.insert(centres.end(), mine.begin(), mine.end());
      bed.push_back(P);
      placed = true;
    }
    if (!placed)
      return set_error(LP_INVALID, "pellet bed: pellet " + std::to_string(p) +
                                       " does not fit in the region without overlap after 10000 draws");
  }
  return LP_OK;
}

// rigid.rs:115-182
lp_status make_pellet(double r, double len, double rho, const double pos[3], lp::PelletState& p) {
  if (!(std::isfinite(r) && r > 0.0)) return set_error(LP_INVALID, "pellet radius must be positive");
  if (!(std::isfinite(len) && len >= 2.0 * r)) return set_error(LP_INVALID, "pellet length must be at least twice the radius");
  if (!(std::isfinite(rho) && rho > 0.0)) return set_error(LP_INVALID, "pellet density must be positive");
  std::memset(&p, 0, sizeof(p));
  p.radius = r;
  p.length = len;
  p.mass = rho * kPi * r * r * len;
  p.inertia[0] = 0.5 * p.mass * r * r;
  p.inertia[1] = p.mass * (3.0 * r * r + len * len) / 12.0;
  p.inertia[2] = p.inertia[1];
  for (int a = 0; a < 3; ++a) p.pos[a] = pos[a];
  p.q[3] = 1.0;
  double hs = 0.5 * len - r;
  int count = 1;
  if (hs > 0.0) {
    double ratio = std::ceil(2.0 * hs / r);
    if (!std::isfinite(ratio) || ratio > 63.0) return set_error(LP_INVALID, "pellet proxy exceeds the sphere cap");
    count = (int)ratio + 1;
  }
  p.nsph = count;
  for (int i = 0; i < count; ++i) p.off[i] = count == 1 ? 0.0 : -hs + 2.0 * hs * (double)i / (double)(count - 1);
  return LP_OK;
}

// fixtures.rs:238-349 (placement with SplitMix64 jitter, hydrostatic prestress)
lp_status build_instance(const lp_fixture_spec& s, HostInstance& h) {
  lp_status st = validate_spec(s);
  if (st != LP_OK) return st;
  st = make_layout(s, h);
  if (st != LP_OK) return st;
  h.spec = s;
  const lp_material& M = s.material;
  SplitMix64 rng{s.seed};
  int64_t counts[3];
  for (int a = 0; a < 3; ++a) counts[a] = axis_count(s.initial_size[a], s.grid_spacing);
  const double sub = s.grid_spacing / 2.0;
  double origin[3] = {0, 0, 0};
  if (s.fixture == LP_SLUMP || s.fixture == LP_COUPLED_PATCH) {
    origin[0] = 0.5 * (s.domain[0] - s.initial_size[0]);
    origin[1] = 0.5 * (s.domain[1] - s.initial_size[1]);
  }
  const double jitter = s.fixture == LP_HYDROSTATIC ? 0.0 : 0.1 * sub;
  const double height = s.initial_size[2];
  const double gnorm = std::sqrt(s.gravity[0] * s.gravity[0] + s.gravity[1] * s.gravity[1] + s.gravity[2] * s.gravity[2]);
  const size_t n = (size_t)(counts[0] * counts[1] * counts[2]);
  HostParticles& P = h.P;
  P.x.resize(3 * n);
  P.v.resize(3 * n);
  P.H.assign(9 * n, 0.0);
  P.tau.assign(9 * n, 0.0);
  P.jm1.assign(n, 0.0);
  P.m.resize(n);
  P.V0.resize(n);
  P.ys.assign(n, M.yield_stress);
  P.id.resize(n);
  size_t idx = 0;
  for (int64_t i = 0; i < counts[0]; ++i)
    for (int64_t j = 0; j < counts[1]; ++j)
      for (int64_t k = 0; k < counts[2]; ++k) {
        double pos[3] = {origin[0] + ((double)i + 0.5) * sub, origin[1] + ((double)j + 0.5) * sub,
                         origin[2] + ((double)k + 0.5) * sub};
        if (jitter > 0.0)
          for (int a = 0; a < 3; ++a) pos[a] += (rng.next_unit() - 0.5) * 2.0 * jitter;
        const double cur = sub * sub * sub;
        double J = 1.0;
        if (s.fixture == LP_HYDROSTATIC) {
          const double depth = height - pos[2];
          if (M.kind == LP_LIQUID) {
            const double arg = -M.density * gnorm * depth / M.bulk_modulus;
            J = std::exp(arg);
            P.jm1[idx] = std::expm1(arg);
            const double pr = M.bulk_modulus * (1.0 / J - 1.0);
            for (int a = 0; a < 3; ++a) P.tau[9 * idx + 4 * a] = -pr * J;
          } else {
            const double modulus = M.lame_lambda + 2.0 * M.shear_modulus;
            const double strain = -M.density * gnorm * depth / modulus;
            J = std::exp(strain);
            P.H[9 * idx + 8] = std::expm1(strain);
            P.tau[9 * idx + 0] = M.lame_lambda * strain;
            P.tau[9 * idx + 4] = M.lame_lambda * strain;
            P.tau[9 * idx + 8] = modulus * strain;
          }
        }
        const double vol0 = cur / J;
        for (int a = 0; a < 3; ++a) {
          P.x[3 * idx + a] = pos[a];
          P.v[3 * idx + a] = s.initial_velocity[a];
        }
        P.m[idx] = M.density * vol0;
        P.V0[idx] = vol0;
        P.id[idx] = (uint32_t)idx;
        ++idx;
      }
  if (s.yield_random)
    for (size_t p = 0; p < n; ++p) P.ys[p] = s.yield_min + (s.yield_max - s.yield_min) * rng.next_unit();
  h.has_pellet = false;
  h.bed.clear();
  if (s.bed_count >= 2) {
    const double extent[3] = {(double)h.cells[0] * s.grid_spacing, (double)h.cells[1] * s.grid_spacing,
                              (double)h.cells[2] * s.grid_spacing};
    st = make_bed(s, extent, h.bed);
    if (st != LP_OK) return st;
  }
  if (s.fixture == LP_COUPLED_PATCH && s.has_pellet) {
    const double center[3] = {0.5 * s.domain[0], 0.5 * s.domain[1],
                              s.initial_size[2] + 2.0 * s.grid_spacing + s.pellet_radius};
    st = make_pellet(s.pellet_radius, s.pellet_length, s.pellet_density, center, h.pellet);
    if (st != LP_OK) return st;
    h.has_pellet = true;
  }
  return LP_OK;
}

int64_t round_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

// ---------------------------------------------------------------- ensemble
struct Ensemble {
  int n = 0;
  std::vector<lp_fixture_spec> specs;
  std::vector<InstDesc> desc;
  std::vector<int> has_pellet;
  lp::DeviceArrays A;
  std::vector<void*> allocs;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  // graph of `graph_steps` attempts
  int graph_steps = 0;
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraph_t graph = nullptr;
  cudaStream_t graph_stream = nullptr;
  int graph_kernels = 0;
  std::vector<Control> ctrl_h;
  double* d_diag = nullptr;
  double* d_audit = nullptr;  // energy-audit partials, 6 per grid-update CTA
  // staging of host-layout particle chunks for import / export (38 doubles + 1 id per particle),
  // two slots so that the host copies of one chunk overlap the transfer and conversion of the
  // other; stage_ev[s] marks the end of the device work that last used slot s
  double* d_stage = nullptr;
  double* h_stage = nullptr;  // pinned host twin of d_stage
  int64_t stage_particles = 0;  // particles per slot
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  unsigned long long* d_bad = nullptr;
  float* d_mlp = nullptr;
  lp::MlpPacked* d_mlp_pk = nullptr;
  int warm = 0;

  ~Ensemble() { release(); }
  void release() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
    for (void* p : allocs) cudaFree(p);
    allocs.clear();
    if (h_stage) cudaFreeHost(h_stage);
    h_stage = nullptr;
    for (cudaEvent_t& ev : stage_ev) {
      if (ev) cudaEventDestroy(ev);
      ev = nullptr;
    }
    if (own_stream) cudaStreamDestroy(own_stream);
    own_stream = nullptr;
  }
  template <class T>
  lp_status alloc(T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return set_error(LP_DEVICE, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(q);
    *p = (T*)q;
    e = cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(T), stream);
    if (e != cudaSuccess) return set_error(LP_DEVICE, std::string("cudaMemset: ") + cudaGetErrorString(e));
    return LP_OK;
  }
  void invalidate_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
  }
};

lp_status pull_ctrl(Ensemble& E) {
  E.ctrl_h.resize(E.n);
  CUDA_CK(cudaMemcpyAsync(E.ctrl_h.data(), E.A.ctrl, sizeof(Control) * E.n, cudaMemcpyDeviceToHost, E.stream));
  CUDA_CK(cudaStreamSynchronize(E.stream));
  return LP_OK;
}
lp_status push_ctrl(Ensemble& E) {
  CUDA_CK(cudaMemcpyAsync(E.A.ctrl, E.ctrl_h.data(), sizeof(Control) * E.n, cudaMemcpyHostToDevice, E.stream));
  CUDA_CK(cudaStreamSynchronize(E.stream));
  return LP_OK;
}

// refresh bbound / max speed / total mass of the committed state
lp_status refresh_stats(Ensemble& E) {
  lp::launch_state_stats(E.A, E.stream);
  CUDA_CK(cudaGetLastError());
  std::vector<lp::ParticlePartial> part(E.A.n_pcta);
  CUDA_CK(cudaMemcpyAsync(part.data(), E.A.ppart, sizeof(lp::ParticlePartial) * E.A.n_pcta, cudaMemcpyDeviceToHost,
                          E.stream));
  lp_status st = pull_ctrl(E);
  if (st != LP_OK) return st;
  for (int i = 0; i < E.n; ++i) {
    const InstDesc& D = E.desc[i];
    double bb = 0.0, mass = 0.0;
    float ms = 0.0f;
    for (int64_t c = 0; c < D.pcta_cnt; ++c) {
      const lp::ParticlePartial& P = part[D.pcta_off + c];
      bb += P.bbound;
      mass += P.mass;
      ms = std::max(ms, P.max_speed);
    }
    E.ctrl_h[i].bbound = bb;
    E.ctrl_h[i].max_speed = ms;
    E.ctrl_h[i].total_mass = mass;
  }
  return push_ctrl(E);
}

struct Diag {
  double ke, pe, ee, mass, mom[3], max_speed, max_ep, yielded, min_x, max_x, min_y, max_y, max_z, hsq, hmax, column,
      cnorm;
};

lp_status diagnostics(Ensemble& E, std::vector<Diag>& out) {
  if (!E.d_diag) {
    lp_status st = E.alloc(&E.d_diag, (size_t)E.A.n_pcta * lp::DIAG_N);
    if (st != LP_OK) return st;
  }
  // hydrostatic / dam-break flags are per ensemble: batch members share fixture kind
  const lp_fixture_spec& s0 = E.specs[0];
  lp::launch_diagnostics(E.A, s0.fixture == LP_HYDROSTATIC, s0.initial_size[2], s0.fixture == LP_DAM_BREAK, E.d_diag,
                         E.stream);
  CUDA_CK(cudaGetLastError());
  std::vector<double> raw((size_t)E.A.n_pcta * lp::DIAG_N);
  CUDA_CK(cudaMemcpyAsync(raw.data(), E.d_diag, sizeof(double) * raw.size(), cudaMemcpyDeviceToHost, E.stream));
  CUDA_CK(cudaStreamSynchronize(E.stream));
  out.assign(E.n, Diag{});
  for (int i = 0; i < E.n; ++i) {
    const InstDesc& D = E.desc[i];
    Diag d{};
    d.min_x = d.min_y = 1e300;
    d.max_x = d.max_y = d.max_z = -1e300;
    d.column = -1e300;
    for (int64_t c = 0; c < D.pcta_cnt; ++c) {
      const double* v = &raw[(size_t)(D.pcta_off + c) * lp::DIAG_N];
      d.ke += v[0];
      d.pe += v[1];
      d.ee += v[2];
      d.mass += v[3];
      d.mom[0] += v[4];
      d.mom[1] += v[5];
      d.mom[2] += v[6];
      d.max_speed = std::max(d.max_speed, v[7]);
      d.max_ep = std::max(d.max_ep, v[8]);
      d.min_x = std::min(d.min_x, v[9]);
      d.max_x = std::max(d.max_x, v[10]);
      d.min_y = std::min(d.min_y, v[11]);
      d.max_y = std::max(d.max_y, v[12]);
      d.max_z = std::max(d.max_z, v[13]);
      d.yielded += v[14];
      d.hsq += v[15];
      d.hmax = std::max(d.hmax, v[16]);
      d.column = std::max(d.column, v[17]);
      d.cnorm += v[18];
    }
    out[i] = d;
  }
  return LP_OK;
}

// pellet kinetic energy (rigid.rs:256-261) and helpers on the host FP64 copy
void q_matrix(const double* q, double R[3][3]) {
  const double i = q[0], j = q[1], k = q[2], w = q[3];
  const double ww = w * w, ii = i * i, jj = j * j, kk = k * k;
  const double ij = i * j * 2.0, wk = w * k * 2.0, wj = w * j * 2.0, ik = i * k * 2.0, jk = j * k * 2.0, wi = w * i * 2.0;
  R[0][0] = ww + ii - jj - kk;
  R[0][1] = ij - wk;
  R[0][2] = wj + ik;
  R[1][0] = wk + ij;
  R[1][1] = ww - ii + jj - kk;
  R[1][2] = jk - wi;
  R[2][0] = ik - wj;
  R[2][1] = wi + jk;
  R[2][2] = ww - ii - jj + kk;
}
void pellet_omega_h(const lp::PelletState& P, double om[3]) {
  double R[3][3];
  q_matrix(P.q, R);
  double bm[3], bo[3];
  for (int a = 0; a < 3; ++a) bm[a] = R[0][a] * P.L[0] + R[1][a] * P.L[1] + R[2][a] * P.L[2];
  for (int a = 0; a < 3; ++a) bo[a] = bm[a] / P.inertia[a];
  for (int a = 0; a < 3; ++a) om[a] = R[a][0] * bo[0] + R[a][1] * bo[1] + R[a][2] * bo[2];
}
double pellet_ke_h(const lp::PelletState& P) {
  double om[3];
  pellet_omega_h(P, om);
  return 0.5 * P.mass * (P.vel[0] * P.vel[0] + P.vel[1] * P.vel[1] + P.vel[2] * P.vel[2]) +
         0.5 * (om[0] * P.L[0] + om[1] * P.L[1] + om[2] * P.L[2]);
}

struct Energies {
  double ke, pe, ee, mech, mass_res, mom_res[3], e_res;
};

// committed pellet-bed states of instance i (host copy)
std::vector<lp::PelletState> bed_pull(const Ensemble& E, int i) {
  const InstDesc& D = E.desc[i];
  std::vector<lp::PelletState> out((size_t)std::max(D.bed_np, 0));
  if (D.bed_np < 2) return out;
  const int par = E.ctrl_h[i].bed_parity;
  cudaStreamSynchronize(E.stream);
  cudaMemcpy(out.data(), E.A.bed.state[par] + D.bed_off, sizeof(lp::PelletState) * out.size(),
             cudaMemcpyDeviceToHost);
  return out;
}

Energies energies_of(const Ensemble& E, int i, const Diag& d) {
  const Control& c = E.ctrl_h[i];
  const InstDesc& D = E.desc[i];
  Energies r{};
  r.ke = d.ke;
  r.pe = d.pe;
  r.ee = d.ee;
  double mom[3] = {d.mom[0], d.mom[1], d.mom[2]};
  if (D.has_pellet) {
    r.ke += pellet_ke_h(c.pellet);
    r.pe -= c.pellet.mass * (D.gravity[0] * c.pellet.pos[0] + D.gravity[1] * c.pellet.pos[1] + D.gravity[2] * c.pellet.pos[2]);
    for (int a = 0; a < 3; ++a) mom[a] += c.pellet.vel[a] * c.pellet.mass;
  }
  if (D.bed_np >= 2)
    for (const lp::PelletState& P : bed_pull(E, i)) {
      r.ke += pellet_ke_h(P);
      r.pe -= P.mass * (D.gravity[0] * P.pos[0] + D.gravity[1] * P.pos[1] + D.gravity[2] * P.pos[2]);
      for (int a = 0; a < 3; ++a) mom[a] += P.vel[a] * P.mass;
    }
  r.mech = r.ke + r.pe + r.ee;
  const lp::LedgerD& L = c.ledger;
  r.mass_res = d.mass + L.outflow_mass - L.initial_mass;
  for (int a = 0; a < 3; ++a)
    r.mom_res[a] = mom[a] - L.initial_momentum[a] - L.gravity_impulse[a] + L.outflow_momentum[a] - L.wall_impulse[a] -
                   L.pellet_wall_impulse[a];
  // the pellet bed's sphere-contact work (dissipation plus energy stored in the contacts) is
  // ledgered beside the reference channels
  const double ledgered =
      L.proj - L.fric + L.trac + L.pellet_work + L.cgrid + L.cpellet - L.plastic + c.bed_contact_work;
  r.e_res = r.mech - L.initial_mech - ledgered;
  return r;
}

lp_status ensemble_create(const lp_fixture_spec* specs, int count, Ensemble& E) {
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
    return set_error(LP_DEVICE, "no CUDA device: the MLS-MPM substep runs on the GPU only");
  if (count <= 0) return set_error(LP_INVALID, "ensemble needs at least one instance");
  std::vector<HostInstance> H(count);
  for (int i = 0; i < count; ++i) {
    lp_status st = build_instance(specs[i], H[i]);
    if (st != LP_OK) return count > 1 ? set_error(st, "instance " + std::to_string(i) + ": " + g_err) : st;
    if (specs[i].fixture != specs[0].fixture)
      return set_error(LP_UNSUPPORTED, "batched instances must share one fixture kind");
  }
  E.n = count;
  E.specs.assign(specs, specs + count);
  lp::configure_kernels();
  CUDA_CK(cudaStreamCreateWithFlags(&E.own_stream, cudaStreamNonBlocking));
  E.stream = E.own_stream;
  // geometry and offsets
  E.desc.resize(count);
  int64_t node_off = 0, tile_off = 0, key_off = 0, blk_off = 0, gcta_off = 0, slot_off = 0;
  std::vector<int> tile_inst, gcta_inst, pcta_inst, chunk_inst;
  std::vector<lp::SegDesc> segs;
  int any_pellet = 0, any_bed = 0;
  int64_t bed_off = 0;
  std::vector<int> bed_inst;
  for (int i = 0; i < count; ++i) {
    const lp_fixture_spec& s = specs[i];
    HostInstance& h = H[i];
    InstDesc D;
    std::memset(&D, 0, sizeof(D));
    D.dx = s.grid_spacing;
    D.inv_dx = 1.0 / s.grid_spacing;
    {
      const float f = (float)s.grid_spacing;
      int e = 0;
      D.pow2_inv_dx = (std::isfinite(f) && f > 0.f && std::frexp(f, &e) == 0.5f) ? 1.0f / f : 0.0f;
    }
    for (int a = 0; a < 3; ++a) {
      D.cells[a] = (int)h.cells[a];
      D.nodes[a] = (int)h.nodes[a];
      D.bins[a] = D.cells[a] + 1;
      D.extent[a] = (double)h.cells[a] * s.grid_spacing;
    }
    D.tiles[0] = (D.bins[0] + lp::TX - 1) / lp::TX;
    D.tiles[1] = (D.bins[1] + lp::TY - 1) / lp::TY;
    D.tiles[2] = (D.bins[2] + lp::TZ - 1) / lp::TZ;
    for (int a = 0; a < 3; ++a) D.nblk[a] = (D.nodes[a] + lp::NB - 1) / lp::NB;
    D.kind = s.material.kind;
    D.per_particle_yield = s.yield_random ? 1 : 0;
    D.face_mode = s.face_mode_enabled ? 1 : 0;
    D.has_pellet = h.has_pellet ? 1 : 0;
    any_pellet |= D.has_pellet;
    D.bed_np = (int)h.bed.size();
    D.bed_off = bed_off;
    if (D.bed_np >= 2) {
      any_bed = 1;
      const lp::PelletState& P0 = h.bed[0];
      double hs = 0.0;
      for (int k = 0; k < P0.nsph; ++k) hs = std::fmax(hs, std::fabs(P0.off[k]));
      D.bed_rb = hs + P0.radius;
      D.bed_h = 2.0 * D.bed_rb;
      for (int a = 0; a < 3; ++a)
        D.bed_nc[a] = std::max(1, (int)std::ceil((double)h.cells[a] * s.grid_spacing / D.bed_h));
      D.hm_mu = s.hm_friction;
      D.bed_law = s.bed_law;
      if (s.bed_law == LP_BED_LINEAR) {
        D.dem_kn = s.dem_stiffness;
        D.dem_zeta = lp::dem_damping_ratio(s.hm_restitution);
        D.dem_mur = s.dem_rolling;
      } else {
        const double nu = s.hm_poisson, E = s.hm_young, G = E / (2.0 * (1.0 + nu));
        D.hm_estar = E / (2.0 * (1.0 - nu * nu));
        D.hm_gstar = G / (2.0 * (2.0 - nu));
        D.hm_beta = hm_beta_for(s.hm_restitution);
      }
      for (int p = 0; p < D.bed_np; ++p) bed_inst.push_back(i);
      bed_off += D.bed_np;
    }
    const int64_t ntiles = (int64_t)D.tiles[0] * D.tiles[1] * D.tiles[2];
    const int64_t nnodes = (int64_t)D.nodes[0] * D.nodes[1] * D.nodes[2];
    const int64_t nblk = (int64_t)D.nblk[0] * D.nblk[1] * D.nblk[2];
    D.node_off = node_off;
    D.tile_off = tile_off;
    D.key_off = key_off;
    D.nkeys = round_up(ntiles * lp::TB + 1, lp::KEY_CHUNK);
    D.blk_off = blk_off;
    D.gcta_off = gcta_off;
    D.gcta_cnt = (nblk + lp::GU_BLOCKS_PER_CTA * lp::GU_PASSES - 1) / (lp::GU_BLOCKS_PER_CTA * lp::GU_PASSES);
    D.slot_off = slot_off;
    D.slot_cap = round_up(std::max<int64_t>((int64_t)h.P.size(), 1), lp::SLOT_ALIGN);
    D.pcta_off = slot_off / lp::G2P_THREADS;
    D.pcta_cnt = D.slot_cap / lp::G2P_THREADS;
    const lp_material& M = s.material;
    D.density = M.density;
    D.mu = M.shear_modulus;
    D.lambda = M.lame_lambda;
    D.bulk = M.bulk_modulus;
    D.yield = M.yield_stress;
    D.consistency = M.consistency;
    D.flow_index = M.flow_index;
    D.tait_gamma = M.tait_gamma == 0.0 ? 1.0 : M.tait_gamma;
    for (int a = 0; a < 3; ++a) D.gravity[a] = s.gravity[a];
    D.friction = s.wall_friction;
    for (int f = 0; f < 6; ++f) {
      D.face_mu[f] = s.face_mode_enabled ? s.face_friction[f] : s.wall_friction;
      D.face_sticky[f] = s.face_mode_enabled ? s.face_sticky[f] : 0;
    }
    D.cfl = s.cfl;
    D.max_dt = s.max_dt;
    D.min_dt = s.min_dt;
    D.tol = s.newton_tolerance > 0.0 ? s.newton_tolerance : 1e-12;
    D.contact_k = s.contact_stiffness;
    D.contact_e = s.contact_restitution;
    D.contact_mu = s.contact_friction;
    double mass = 0.0;
    for (size_t p = 0; p < h.P.size(); ++p) mass += (double)(float)h.P.m[p];
    D.s_mass = std::ldexp(1.0, (int)std::floor(std::log2(4.611686018427388e18 / std::max(mass, 1e-300))));
    D.seg_off = (int64_t)segs.size();
    D.seg_cnt_g = (D.gcta_cnt + lp::SEG_SPAN - 1) / lp::SEG_SPAN;
    for (int64_t b = 0; b < D.gcta_cnt; b += lp::SEG_SPAN)
      segs.push_back(lp::SegDesc{D.gcta_off + b, D.gcta_off + std::min<int64_t>(b + lp::SEG_SPAN, D.gcta_cnt), i, 0});
    for (int64_t b = 0; b < ntiles; b += lp::SEG_SPAN)
      segs.push_back(lp::SegDesc{D.tile_off + b, D.tile_off + std::min<int64_t>(b + lp::SEG_SPAN, ntiles), i, 1});
    D.seg_cnt = (int64_t)segs.size() - D.seg_off;
    E.desc[i] = D;
    for (int64_t t = 0; t < ntiles; ++t) tile_inst.push_back(i);
    for (int64_t t = 0; t < D.gcta_cnt; ++t) gcta_inst.push_back(i);
    for (int64_t t = 0; t < D.pcta_cnt; ++t) pcta_inst.push_back(i);
    for (int64_t t = 0; t < D.nkeys / lp::KEY_CHUNK; ++t) chunk_inst.push_back(i);
    node_off += nnodes;
    tile_off += ntiles;
    key_off += D.nkeys;
    blk_off += nblk;
    gcta_off += D.gcta_cnt;
    slot_off += D.slot_cap;
    E.has_pellet.push_back(D.has_pellet);
  }
  if (slot_off > 0xFFFFFFFFll || key_off > 0xFFFFFFFFll) return set_error(LP_INVALID, "ensemble exceeds 32-bit slot/key range");
  lp::DeviceArrays& A = E.A;
  A.n_inst = count;
  A.any_pellet = any_pellet;
  A.any_bed = any_bed;
  A.kinds = 0;
  for (int i = 0; i < count; ++i) A.kinds |= E.desc[i].kind == 0 ? 1 : 2;
  A.n_bed = bed_off;
  A.cap = slot_off;
  A.n_pcta = (int64_t)pcta_inst.size();
  A.n_tiles = (int64_t)tile_inst.size();
  A.n_gcta = (int64_t)gcta_inst.size();
  A.n_chunks = (int64_t)chunk_inst.size();
  A.node_total = node_off;
  A.n_blk = blk_off;
  lp_status st;
#define ALLOC(ptr, n)                 \
  st = E.alloc(&(ptr), (size_t)(n)); \
  if (st != LP_OK) return st;
  ALLOC(A.desc, count);
  ALLOC(A.ctrl, count);
  ALLOC(A.pcta_inst, A.n_pcta);
  ALLOC(A.tile_inst, A.n_tiles);
  ALLOC(A.gcta_inst, A.n_gcta);
  ALLOC(A.chunk_inst, A.n_chunks);
  ALLOC(A.st[0], (size_t)lp::NCOMP * A.cap);
  ALLOC(A.st[1], (size_t)lp::NCOMP * A.cap);
  ALLOC(A.id[0], A.cap);
  ALLOC(A.id[1], A.cap);
  ALLOC(A.keys, A.cap);
  ALLOC(A.count, key_off);
  ALLOC(A.start, key_off);
  ALLOC(A.chunk_sum, A.n_chunks);
  ALLOC(A.chunk_base, A.n_chunks);
  ALLOC(A.perm, A.cap);
  ALLOC(A.nw_list, A.cap);
  ALLOC(A.nw_count, 6);
  A.tile_count = A.nw_count + 1;
  ALLOC(A.tile_rec, A.n_tiles);
  ALLOC(A.defer_rec, A.n_tiles);
  ALLOC(A.acc, 4 * A.node_total);
  ALLOC(A.trac, 6 * A.node_total);
  ALLOC(A.blk_epoch, A.n_blk);
  ALLOC(A.vel, A.node_total);
  ALLOC(A.gpart, A.n_gcta);
  ALLOC(A.ppart, A.n_pcta);
  ALLOC(A.tpart, A.n_tiles);
  A.n_seg = (int64_t)segs.size();
  ALLOC(A.segs, A.n_seg);
  ALLOC(A.seg, A.n_seg);
  for (int b = 0; b < 2; ++b) {
    ALLOC(A.bed.state[b], A.n_bed);
    ALLOC(A.bed.hist[b], A.n_bed * lp::HM_SLOTS);
    ALLOC(A.bed.hist_n[b], A.n_bed);
  }
  ALLOC(A.bed_step, A.n_bed);
  ALLOC(A.bed_key, A.n_bed);
  ALLOC(A.bed_idx, A.n_bed);
  ALLOC(A.bed_inst, A.n_bed);
#undef ALLOC
  if (any_bed) {
    std::vector<lp::PelletState> all;
    for (int i = 0; i < count; ++i) all.insert(all.end(), H[i].bed.begin(), H[i].bed.end());
    CUDA_CK(cudaMemcpyAsync(A.bed.state[0], all.data(), sizeof(lp::PelletState) * all.size(), cudaMemcpyHostToDevice,
                            E.stream));
    CUDA_CK(cudaMemcpyAsync(A.bed_inst, bed_inst.data(), sizeof(int) * bed_inst.size(), cudaMemcpyHostToDevice,
                            E.stream));
    CUDA_CK(cudaStreamSynchronize(E.stream));
  }
  CUDA_CK(cudaMemcpyAsync(A.segs, segs.data(), sizeof(lp::SegDesc) * segs.size(), cudaMemcpyHostToDevice, E.stream));
  CUDA_CK(cudaMemcpyAsync(A.desc, E.desc.data(), sizeof(InstDesc) * count, cudaMemcpyHostToDevice, E.stream));
  CUDA_CK(cudaMemcpyAsync(A.pcta_inst, pcta_inst.data(), sizeof(int) * pcta_inst.size(), cudaMemcpyHostToDevice, E.stream));
  CUDA_CK(cudaMemcpyAsync(A.tile_inst, tile_inst.data(), sizeof(int) * tile_inst.size(), cudaMemcpyHostToDevice, E.stream));
  CUDA_CK(cudaMemcpyAsync(A.gcta_inst, gcta_inst.data(), sizeof(int) * gcta_inst.size(), cudaMemcpyHostToDevice, E.stream));
  CUDA_CK(cudaMemcpyAsync(A.chunk_inst, chunk_inst.data(), sizeof(int) * chunk_inst.size(), cudaMemcpyHostToDevice,
                          E.stream));
  // particle state (FP32, component-major), ids
  {
    std::vector<float> st32((size_t)lp::NCOMP * A.cap, 0.0f);
    std::vector<uint32_t> ids(A.cap, 0u);
    for (int i = 0; i < count; ++i) {
      const HostParticles& P = H[i].P;
      const int64_t off = E.desc[i].slot_off;
      for (size_t p = 0; p < P.size(); ++p) {
        const int64_t s = off + (int64_t)p;
        auto put = [&](int c, double v) { st32[(size_t)c * A.cap + s] = (float)v; };
        for (int a = 0; a < 3; ++a) {
          put(lp::C_X + a, P.x[3 * p + a]);
          put(lp::C_V + a, P.v[3 * p + a]);
        }
        for (int a = 0; a < 9; ++a) put(lp::C_H + a, P.H[9 * p + a]);
        const double* T = &P.tau[9 * p];
        put(lp::C_TAU + 0, T[0]);
        put(lp::C_TAU + 1, T[4]);
        put(lp::C_TAU + 2, T[8]);
        put(lp::C_TAU + 3, T[1]);
        put(lp::C_TAU + 4, T[2]);
        put(lp::C_TAU + 5, T[5]);
        put(lp::C_M, P.m[p]);
        put(lp::C_V0, P.V0[p]);
        put(lp::C_YS, P.ys[p]);
        put(lp::C_JM1, P.jm1[p]);
        ids[s] = P.id[p];
      }
    }
    CUDA_CK(cudaMemcpyAsync(A.st[0], st32.data(), sizeof(float) * st32.size(), cudaMemcpyHostToDevice, E.stream));
    CUDA_CK(cudaMemcpyAsync(A.id[0], ids.data(), sizeof(uint32_t) * ids.size(), cudaMemcpyHostToDevice, E.stream));
    CUDA_CK(cudaStreamSynchronize(E.stream));
  }
  // control blocks
  E.ctrl_h.assign(count, Control{});
  for (int i = 0; i < count; ++i) {
    Control& c = E.ctrl_h[i];
    std::memset(&c, 0, sizeof(c));
    c.dt_scale = 1.0;
    c.min_dt_used = std::numeric_limits<double>::infinity();
    c.count = (int64_t)H[i].P.size();
    c.status = lp::S_RUNNING;
    if (H[i].has_pellet) c.pellet = H[i].pellet;
    if (E.desc[i].bed_np >= 2) c.bed_limit = lp::bed_limit(E.desc[i], H[i].bed.data());
  }
  lp_status s2 = push_ctrl(E);
  if (s2 != LP_OK) return s2;
  s2 = refresh_stats(E);
  if (s2 != LP_OK) return s2;
  // initial ledger (Simulation::new, solver.rs:357-394)
  std::vector<Diag> d;
  s2 = diagnostics(E, d);
  if (s2 != LP_OK) return s2;
  for (int i = 0; i < count; ++i) {
    Control& c = E.ctrl_h[i];
    Energies en = energies_of(E, i, d[i]);
    c.ledger.initial_mass = d[i].mass;
    for (int a = 0; a < 3; ++a)
      c.ledger.initial_momentum[a] = d[i].mom[a] + (E.desc[i].has_pellet ? c.pellet.vel[a] * c.pellet.mass : 0.0);
    for (const lp::PelletState& P : H[i].bed)
      for (int a = 0; a < 3; ++a) c.ledger.initial_momentum[a] += P.vel[a] * P.mass;
    c.ledger.initial_mech = en.mech;
  }
  return push_ctrl(E);
}

// Capture and instantiate the graph of G attempts when the launch shape asks for one and none is
// built; launches nothing.  The kernel launches counted while capturing are taken back, so that
// each replay counts its own.
lp_status ensure_graph(Ensemble& E) {
  const int G = E.graph_steps;
  if (G <= 1 || E.graph_exec) return LP_OK;
  const uint64_t before = lp::kernel_launch_count();
  cudaStream_t cs = E.stream;
  CUDA_CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int kernels = 0;
  for (int s = 0; s < G; ++s) kernels += lp::launch_attempt(E.A, cs);
  cudaGraph_t g = nullptr;
  CUDA_CK(cudaStreamEndCapture(cs, &g));
  E.graph = g;
  CUDA_CK(cudaGraphInstantiate(&E.graph_exec, g, 0));
  E.graph_kernels = kernels;
  lp::add_kernel_launches(before - lp::kernel_launch_count());  // unsigned wrap: subtracts the capture's count
  return LP_OK;
}

// Queue `steps` attempts: with a graph length G > 1, floor(steps / G) replays of a CUDA graph of G
// attempts (captured on first use unless ensure_graph built it earlier) and the remainder as plain
// launches.
lp_status run_attempts(Ensemble& E, int steps) {
  if (steps <= 0) return LP_OK;
  const int G = E.graph_steps;
  if (G > 1 && steps >= G) {
    const lp_status st = ensure_graph(E);
    if (st != LP_OK) return st;
    for (; steps >= G; steps -= G) {
      CUDA_CK(cudaGraphLaunch(E.graph_exec, E.stream));
      lp::add_kernel_launches((uint64_t)E.graph_kernels);
    }
  }
  for (int s = 0; s < steps; ++s) lp::launch_attempt(E.A, E.stream);
  CUDA_CK(cudaGetLastError());
  return LP_OK;
}

// ---------------------------------------------------------------- launch shapes and autotuner
lp_status set_targets(Ensemble& E, double target, bool forced_reset);

static lp_status set_launch_shape(Ensemble& E, const lp_launch_shape* in) {
  if (!in) return set_error(LP_INVALID, "null launch shape");
  if (in->g2p_variant < 0 || in->g2p_variant >= lp::G2P_VARIANTS || in->p2g_variant < 0 || in->p2g_variant >= lp::P2G_VARIANTS || in->dynamic_tiles < 0 ||
      in->dynamic_tiles > 1 || in->g2p_per_sm < 0 || in->p2g_per_sm < 0 || in->graph_attempts < 0)
    return set_error(LP_INVALID, "launch shape fields out of range");
  E.invalidate_graph();
  E.A.shape.g2p_variant = in->g2p_variant;
  E.A.shape.g2p_per_sm = in->g2p_per_sm;
  E.A.shape.p2g_variant = in->p2g_variant;
  E.A.shape.p2g_per_sm = in->p2g_per_sm;
  E.A.shape.dynamic = in->dynamic_tiles;
  E.graph_steps = in->graph_attempts > 1 ? in->graph_attempts : 0;
  return LP_OK;
}
static lp_status get_launch_shape(Ensemble& E, lp_launch_shape* out) {
  if (!out) return set_error(LP_INVALID, "null launch shape");
  int lim[lp::LAUNCH_LIMITS];
  lp::launch_shape_limits(lim);
  const lp::LaunchShape& L = E.A.shape;
  out->g2p_variant = L.g2p_variant;
  out->p2g_variant = L.p2g_variant;
  out->dynamic_tiles = L.dynamic;
  // the CTAs per SM the launches use: the request, at most the resident limit
  const int g2p_lim = lim[lp::LIM_G2P + L.g2p_variant], p2g_lim = lim[lp::LIM_P2G + L.p2g_variant];
  out->g2p_per_sm = (L.g2p_per_sm > 0 && L.g2p_per_sm < g2p_lim) ? L.g2p_per_sm : g2p_lim;
  out->p2g_per_sm = (L.p2g_per_sm > 0 && L.p2g_per_sm < p2g_lim) ? L.p2g_per_sm : p2g_lim;
  out->graph_attempts = E.graph_steps > 1 ? E.graph_steps : 1;
  return LP_OK;
}
static std::string shape_text(const lp_launch_shape& s) {
  char b[192];
  static const char* const g2p_names[4] = {"256", "128", "128_regs_for_5", "128_regs_for_6"};
  const int gv = s.g2p_variant >= 0 && s.g2p_variant < 4 ? s.g2p_variant : 0;
  std::snprintf(b, sizeof(b),
                "g2p_threads=%s g2p_per_sm=%d p2g_chunk=%d%s p2g_per_sm=%d dynamic_tiles=%d graph_attempts=%d",
                g2p_names[gv], s.g2p_per_sm, (s.p2g_variant == 1 || s.p2g_variant == 2) ? 512 : 1024,
                s.p2g_variant == 2 ? "_staged" : "",
                s.p2g_per_sm, s.dynamic_tiles, s.graph_attempts);
  return b;
}

// Coordinate search over the launch shape on the live ensemble: one knob at a time (tile
// scheduling, G2P block shape and CTAs per SM, P2G chunk and CTAs per SM, attempts per graph
// replay), each candidate timed over trial_steps attempts with CUDA events after two untimed
// ones, keeping the fastest value before moving to the next knob.  The attempts are real steps,
// and the work per attempt changes as the trajectory moves on (a collapsing column yields more
// from step to step), so every candidate starts from the same state: the ensemble's device
// state (both particle buffers and ids, the control blocks, the pellet-bed buffers) is copied
// aside once and put back before each candidate and at the end.  Every candidate then runs the
// same attempts, and since the tile kernels' results do not depend on the launch shape, only the
// speed differs; tuning leaves the simulation where it found it.  A candidate replaces the
// incumbent only when it is faster by more than the timing noise (TUNE_MARGIN).
static lp_status autotune(Ensemble& E, int32_t trial_steps, char* report, size_t report_len) {
  constexpr float TUNE_MARGIN = 0.005f;
  if (trial_steps < 1) return set_error(LP_INVALID, "trial_steps must be at least 1");
  lp_status st = pull_ctrl(E);
  if (st != LP_OK) return st;
  const std::vector<Control> ctrl_before = E.ctrl_h;  // the caller's targets, put back at the end
  if (E.ctrl_h.empty() || !std::isinf(E.ctrl_h[0].target)) {
    st = set_targets(E, std::numeric_limits<double>::infinity(), true);
    if (st != LP_OK) return st;
  }
  // the device state every candidate starts from; the control blocks are kept on the host and
  // put back with the attempt epoch left advanced, so that node blocks marked by a tuning attempt
  // never look active to a later one
  st = pull_ctrl(E);
  if (st != LP_OK) return st;
  const std::vector<Control> ctrl_start = E.ctrl_h;
  lp::DeviceArrays& A = E.A;
  std::vector<std::pair<void*, size_t>> live = {
      {A.st[0], sizeof(float) * (size_t)lp::NCOMP * A.cap}, {A.st[1], sizeof(float) * (size_t)lp::NCOMP * A.cap},
      {A.id[0], sizeof(uint32_t) * (size_t)A.cap},           {A.id[1], sizeof(uint32_t) * (size_t)A.cap}};
  if (A.any_bed)
    for (int b = 0; b < 2; ++b) {
      live.push_back({A.bed.state[b], sizeof(lp::PelletState) * (size_t)A.n_bed});
      live.push_back({A.bed.hist[b], sizeof(lp::HmContact) * (size_t)A.n_bed * lp::HM_SLOTS});
      live.push_back({A.bed.hist_n[b], sizeof(int) * (size_t)A.n_bed});
    }
  size_t total = 0;
  for (auto& l : live) total += (l.second + 255) & ~(size_t)255;
  char* saved = nullptr;
  if (cudaMalloc(&saved, total) != cudaSuccess) {
    cudaGetLastError();
    return set_error(LP_DEVICE, "autotune needs device memory for a copy of the ensemble's state");
  }
  auto copy_state = [&](bool restore) -> lp_status {
    size_t off = 0;
    for (auto& l : live) {
      void* dst = restore ? l.first : (void*)(saved + off);
      const void* src = restore ? (const void*)(saved + off) : l.first;
      CUDA_CK(cudaMemcpyAsync(dst, src, l.second, cudaMemcpyDeviceToDevice, E.stream));
      off += (l.second + 255) & ~(size_t)255;
    }
    if (!restore) return LP_OK;
    lp_status r = pull_ctrl(E);
    if (r != LP_OK) return r;
    for (int i = 0; i < E.n; ++i) {
      const int epoch = E.ctrl_h[i].epoch;
      E.ctrl_h[i] = ctrl_start[i];
      E.ctrl_h[i].epoch = epoch;
    }
    return push_ctrl(E);
  };
  int lim[lp::LAUNCH_LIMITS];
  lp::launch_shape_limits(lim);
  lp_launch_shape best;
  st = get_launch_shape(E, &best);
  best.g2p_per_sm = best.p2g_per_sm = 0;  // 0: as many as fit
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (st == LP_OK && cudaEventCreate(&e0) != cudaSuccess) st = set_error(LP_DEVICE, "cudaEventCreate failed");
  if (st == LP_OK && cudaEventCreate(&e1) != cudaSuccess) st = set_error(LP_DEVICE, "cudaEventCreate failed");
  if (st == LP_OK) st = copy_state(false);
  std::string rep;
  auto measure = [&](const lp_launch_shape& s, float* ms_per_attempt) -> lp_status {
    lp_status r = copy_state(true);
    if (r != LP_OK) return r;
    r = set_launch_shape(E, &s);
    if (r != LP_OK) return r;
    const int per = std::max(1, s.graph_attempts);
    const int reps = std::max(1, trial_steps / per);
    r = run_attempts(E, per);  // untimed (captures the graph)
    if (r != LP_OK) return r;
    r = run_attempts(E, per);
    if (r != LP_OK) return r;
    CUDA_CK(cudaEventRecord(e0, E.stream));
    for (int k = 0; k < reps; ++k) {
      r = run_attempts(E, per);
      if (r != LP_OK) return r;
    }
    CUDA_CK(cudaEventRecord(e1, E.stream));
    CUDA_CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CUDA_CK(cudaEventElapsedTime(&ms, e0, e1));
    *ms_per_attempt = ms / (float)(reps * per);
    return LP_OK;
  };
  float best_ms = 0.f;
  if (st == LP_OK) st = measure(best, &best_ms);
  if (st == LP_OK) rep += shape_text(best) + " ms_per_attempt=" + std::to_string(best_ms) + "\n";
  // one knob at a time; each candidate list holds complete field values for that knob
  struct Knob {
    std::vector<std::array<int, 2>> values;  // (small / dynamic / graph, per-SM) pairs
    int which;                               // 0 dynamic, 1 G2P, 2 P2G, 3 graph
  };
  std::vector<Knob> knobs = {
      {{{0, 0}, {1, 0}}, 0},
      {{{0, 0}, {0, 1}, {1, 0}, {1, std::max(1, lim[lp::LIM_G2P + 1] - 1)}, {2, 0}, {3, 0}}, 1},
      {{{0, 0}, {0, 1}, {1, 0}, {2, 0}}, 2},
      {{{1, 0}, {4, 0}, {16, 0}}, 3},
  };
  for (const Knob& kb : knobs) {
    if (st != LP_OK) break;
    for (const auto& v : kb.values) {
      lp_launch_shape c = best;
      if (kb.which == 0) c.dynamic_tiles = v[0];
      else if (kb.which == 1) c.g2p_variant = v[0], c.g2p_per_sm = v[1];
      else if (kb.which == 2) c.p2g_variant = v[0], c.p2g_per_sm = v[1];
      else c.graph_attempts = v[0];
      if (std::memcmp(&c, &best, sizeof(c)) == 0) continue;  // measured already
      float ms = 0.f;
      st = measure(c, &ms);
      if (st != LP_OK) break;
      rep += shape_text(c) + " ms_per_attempt=" + std::to_string(ms) + " incumbent=" + std::to_string(best_ms) + "\n";
      if (ms < (1.0f - TUNE_MARGIN) * best_ms) {
        best = c;
        best_ms = ms;
      }
    }
  }
  // back to the state and targets tuning found
  if (saved) {
    const lp_status r = copy_state(true);
    if (st == LP_OK) st = r;
    cudaStreamSynchronize(E.stream);
    cudaFree(saved);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st != LP_OK) return st;
  st = pull_ctrl(E);
  if (st != LP_OK) return st;
  for (int i = 0; i < E.n; ++i) {
    E.ctrl_h[i].target = ctrl_before[i].target;
    E.ctrl_h[i].status = ctrl_before[i].status;
    E.ctrl_h[i].forced_dt = ctrl_before[i].forced_dt;
  }
  st = push_ctrl(E);
  if (st != LP_OK) return st;
  st = set_launch_shape(E, &best);
  if (st != LP_OK) return st;
  rep += "chosen: " + shape_text(best) + " ms_per_attempt=" + std::to_string(best_ms) + "\n";
  if (report && report_len) std::snprintf(report, report_len, "%s", rep.c_str());
  return LP_OK;
}

lp_status set_targets(Ensemble& E, double target, bool forced_reset) {
  lp_status st = pull_ctrl(E);
  if (st != LP_OK) return st;
  for (int i = 0; i < E.n; ++i) {
    Control& c = E.ctrl_h[i];
    if (forced_reset) c.forced_dt = 0.0;
    if (c.status == lp::S_REACHED || c.status == lp::S_RUNNING) {
      c.target = target;
      c.status = (c.time < target) ? lp::S_RUNNING : lp::S_REACHED;
    }
  }
  return push_ctrl(E);
}

lp_status ensemble_advance(Ensemble& E, double target, lp_keep_going_fn keep, void* ctx, int32_t* reached) {
  if (reached) *reached = 0;
  if (!std::isfinite(target)) return set_error(LP_INVALID, "invalid solver state: invalid target time");
  lp_status st = pull_ctrl(E);
  if (st != LP_OK) return st;
  for (int i = 0; i < E.n; ++i)
    if (target < E.ctrl_h[i].time) return set_error(LP_INVALID, "invalid solver state: invalid target time");
  st = set_targets(E, target, true);
  if (st != LP_OK) return st;
  const int chunk = E.graph_steps > 0 ? E.graph_steps : 16;
  while (true) {
    bool running = false;
    for (int i = 0; i < E.n; ++i) running |= E.ctrl_h[i].status == lp::S_RUNNING;
    if (!running) break;
    if (keep && !keep(ctx)) return set_error(LP_BUDGET, "budget stop at a resumable step boundary");
    st = run_attempts(E, chunk);
    if (st != LP_OK) return st;
    st = pull_ctrl(E);
    if (st != LP_OK) return st;
  }
  bool all = true;
  for (int i = 0; i < E.n; ++i) {
    const Control& c = E.ctrl_h[i];
    if (c.status == lp::S_MIN_STEP) {
      char buf[256];
      std::snprintf(buf, sizeof(buf),
                    "solver aborted at t='%.17g' s: step '%.17g' s below minimum after '%llu' rejections; last failure code %d",
                    c.time, c.dt, (unsigned long long)c.rejected_steps, c.last_fail);
      return set_error(LP_MIN_STEP, (E.n > 1 ? "instance " + std::to_string(i) + ": " : std::string()) + buf);
    }
    if (c.status == lp::S_ERROR)
      return set_error(LP_INVALID, "closed fixture leaked particles beyond the padded grid (outflow)");
    all &= c.status == lp::S_REACHED;
  }
  if (reached) *reached = all ? 1 : 0;
  return LP_OK;
}

const char* fail_text(int f) {
  switch (f) {
    case lp::F_CONST_INVERTED: return "constitutive update failed: trial deformation gradient inverted";
    case lp::F_CONST_EIGEN: return "constitutive update failed: eigen-decomposition did not converge";
    case lp::F_CONST_STRETCH: return "constitutive update failed: degenerate elastic stretch";
    case lp::F_CONST_NOT_CONVERGED: return "constitutive update failed: Herschel-Bulkley return did not converge";
    case lp::F_CONST_NONFINITE: return "constitutive update failed: non-finite constitutive quantity";
    case lp::F_GRID_NONFINITE: return "non-finite grid velocity";
    case lp::F_DISPLACEMENT: return "particle moved more than one cell in one step";
    case lp::F_PELLET_NONFINITE: return "pellet state became non-finite";
    case lp::F_TRACTION_NONFINITE: return "wall traction kinetic-energy jump became non-finite";
    case lp::F_OUTFLOW: return "particle left the padded grid";
  }
  return "ok";
}

// ---------------------------------------------------------------- export / import
// Particles per staging slot of import and export: 2^20 x 308 B = 323 MB of device memory and
// as much pinned host memory, twice (two slots).
static const int64_t STAGE_CHUNK = (int64_t)1 << 20;

// Two staging slots of up to STAGE_CHUNK particles on the device, their pinned host twins and
// the slot events (allocated once, grown when a larger set arrives).
static lp_status stage_alloc(Ensemble& E, int64_t count) {
  const int64_t want = std::min<int64_t>(std::max<int64_t>(count, 1), STAGE_CHUNK);
  if (E.stage_particles < want) {
    cudaStreamSynchronize(E.stream);
    if (E.d_stage) {
      cudaFree(E.d_stage);
      E.allocs.erase(std::remove(E.allocs.begin(), E.allocs.end(), (void*)E.d_stage), E.allocs.end());
      E.d_stage = nullptr;
    }
    if (E.h_stage) cudaFreeHost(E.h_stage);
    E.h_stage = nullptr;
    E.stage_particles = 0;
    lp_status st = E.alloc(&E.d_stage, (size_t)want * 39 * 2);
    if (st != LP_OK) return st;
    if (cudaHostAlloc((void**)&E.h_stage, sizeof(double) * 39 * 2 * (size_t)want, cudaHostAllocDefault) !=
        cudaSuccess) {
      E.h_stage = nullptr;
      return set_error(LP_DEVICE, "cudaHostAlloc of the particle staging buffer failed");
    }
    E.stage_particles = want;
  }
  for (cudaEvent_t& ev : E.stage_ev)
    if (!ev) CUDA_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  if (!E.d_bad) {
    lp_status st = E.alloc(&E.d_bad, 1);
    if (st != LP_OK) return st;
  }
  return LP_OK;
}

// The host-layout arrays of staging slot `slot` (0 or 1), carved out of the device buffer.
static void stage_slot(Ensemble& E, int slot, lp::HostParticleChunk& h) {
  const int64_t c = E.stage_particles;
  double* b = E.d_stage + (size_t)slot * 39 * (size_t)c;
  h.position = b;
  h.velocity = b + 3 * c;
  h.affine = b + 6 * c;
  h.deformation = b + 15 * c;
  h.kirchhoff = b + 24 * c;
  h.volume_ratio = b + 33 * c;
  h.plastic_strain = b + 34 * c;
  h.mass = b + 35 * c;
  h.volume0 = b + 36 * c;
  h.yield_stress = b + 37 * c;
  h.id = reinterpret_cast<uint32_t*>(b + 38 * c);
}

// memcpy of the listed (destination, source, bytes) spans over up to 16 host threads
struct CopySpan {
  void* dst;
  const void* src;
  size_t bytes;
};
static void parallel_copy(const std::vector<CopySpan>& spans) {
  size_t total = 0;
  for (const CopySpan& c : spans) total += c.bytes;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned nt = (unsigned)std::min<size_t>(std::min(16u, hw), std::max<size_t>(1, total >> 23));
  auto run = [&](unsigned k) {
    // thread k copies bytes [k total / nt, (k + 1) total / nt) of the concatenated spans
    const size_t lo = total * k / nt, hi = total * (k + 1) / nt;
    size_t base = 0;
    for (const CopySpan& c : spans) {
      const size_t a = std::max(lo, base), b = std::min(hi, base + c.bytes);
      if (a < b) std::memcpy((char*)c.dst + (a - base), (const char*)c.src + (a - base), b - a);
      base += c.bytes;
    }
  };
  if (nt == 1) {
    run(0);
    return;
  }
  std::vector<std::thread> pool;
  for (unsigned k = 1; k < nt; ++k) pool.emplace_back(run, k);
  run(0);
  for (std::thread& t : pool) t.join();
}

// the host twin of a device staging pointer
static inline void* host_twin(const Ensemble& E, const void* dev) {
  return (char*)E.h_stage + ((const char*)dev - (const char*)E.d_stage);
}

// A caller's host span is page-locked (cudaHostAlloc'd or cudaHostRegister'ed, for example with
// lp_host_pin) from its first to its last byte: then import and export move it by DMA directly,
// without the staging copy by host threads.  A wrong answer would cost speed only: a copy from
// pageable memory is still correct.
static bool page_locked(const void* p, size_t bytes) {
  if (!p || bytes == 0) return true;
  for (const char* q : {(const char*)p, (const char*)p + bytes - 1}) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (a.type != cudaMemoryTypeHost) return false;
  }
  return true;
}
static bool particles_page_locked(const lp_particles* p, int64_t n) {
  const size_t d1 = sizeof(double) * (size_t)n;
  return page_locked(p->id, sizeof(uint32_t) * (size_t)n) && page_locked(p->position, 3 * d1) &&
         page_locked(p->velocity, 3 * d1) && page_locked(p->affine, 9 * d1) && page_locked(p->deformation, 9 * d1) &&
         page_locked(p->kirchhoff, 9 * d1) && page_locked(p->volume_ratio, d1) && page_locked(p->plastic_strain, d1) &&
         page_locked(p->mass, d1) && page_locked(p->volume0, d1) && page_locked(p->yield_stress, d1);
}

// Export instance i's committed particles into the caller's FP64 arrays (null fields are
// skipped).  Chunk k is converted on the device into staging slot k % 2 and copied to its pinned
// twin (one copy per requested field); while those run, host threads copy chunk k - 1 from the
// other slot's pinned twin into the caller's arrays.
lp_status export_particles(Ensemble& E, int i, lp_particles* out) {
  lp_status st = pull_ctrl(E);
  if (st != LP_OK) return st;
  const Control& c = E.ctrl_h[i];
  const InstDesc& D = E.desc[i];
  const int64_t n = c.count;
  if ((int64_t)out->count < n) return set_error(LP_INVALID, "particle buffer too small");
  st = stage_alloc(E, n);
  if (st != LP_OK) return st;
  // page-locked caller arrays: each chunk is converted into its staging slot and copied by DMA
  // straight into them, all in stream order (a slot is rewritten only after its copies ran)
  const bool direct = particles_page_locked(out, n);
  std::vector<CopySpan> pending[2];  // host copies waiting for slot s's device-to-host copies
  int64_t k = 0;
  for (int64_t first = 0; first < n; first += E.stage_particles, ++k) {
    const int slot = (int)(k & 1);
    const int64_t m = std::min(E.stage_particles, n - first);
    lp::HostParticleChunk h;
    stage_slot(E, slot, h);
    lp::launch_export(h, m, first, E.A.st[c.parity], E.A.id[c.parity], E.A.cap, D.slot_off, D.kind == 0,
                      D.per_particle_yield, D.yield, E.stream);
    CUDA_CK(cudaGetLastError());
    // device staging -> pinned twin (one copy per requested field); the host copy to the caller
    // arrays runs after the slot's event, one chunk later
    std::vector<CopySpan>& spans = pending[slot];
    spans.clear();
    auto back = [&](void* dst, const void* src, size_t bytes) -> lp_status {
      if (!dst) return LP_OK;
      if (direct) {
        CUDA_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, E.stream));
        return LP_OK;
      }
      void* pinned = host_twin(E, src);
      CUDA_CK(cudaMemcpyAsync(pinned, src, bytes, cudaMemcpyDeviceToHost, E.stream));
      spans.push_back({dst, pinned, bytes});
      return LP_OK;
    };
    const size_t d1 = sizeof(double) * (size_t)m;
    if (back(out->id ? out->id + first : nullptr, h.id, sizeof(uint32_t) * (size_t)m) != LP_OK ||
        back(out->position ? out->position + 3 * first : nullptr, h.position, 3 * d1) != LP_OK ||
        back(out->velocity ? out->velocity + 3 * first : nullptr, h.velocity, 3 * d1) != LP_OK ||
        back(out->affine ? out->affine + 9 * first : nullptr, h.affine, 9 * d1) != LP_OK ||
        back(out->deformation ? out->deformation + 9 * first : nullptr, h.deformation, 9 * d1) != LP_OK ||
        back(out->kirchhoff ? out->kirchhoff + 9 * first : nullptr, h.kirchhoff, 9 * d1) != LP_OK ||
        back(out->volume_ratio ? out->volume_ratio + first : nullptr, h.volume_ratio, d1) != LP_OK ||
        back(out->plastic_strain ? out->plastic_strain + first : nullptr, h.plastic_strain, d1) != LP_OK ||
        back(out->mass ? out->mass + first : nullptr, h.mass, d1) != LP_OK ||
        back(out->volume0 ? out->volume0 + first : nullptr, h.volume0, d1) != LP_OK ||
        back(out->yield_stress ? out->yield_stress + first : nullptr, h.yield_stress, d1) != LP_OK)
      return LP_DEVICE;
    if (direct) continue;
    CUDA_CK(cudaEventRecord(E.stage_ev[slot], E.stream));
    if (k > 0) {  // chunk k - 1: its copies have landed once the other slot's event has
      CUDA_CK(cudaEventSynchronize(E.stage_ev[slot ^ 1]));
      parallel_copy(pending[slot ^ 1]);
    }
  }
  if (direct) {
    CUDA_CK(cudaStreamSynchronize(E.stream));
  } else if (k > 0) {
    const int last = (int)((k - 1) & 1);
    CUDA_CK(cudaEventSynchronize(E.stage_ev[last]));
    parallel_copy(pending[last]);
  }
  out->count = (uint64_t)n;
  return LP_OK;
}

// Import the caller's FP64 arrays as instance i's committed particles.  They are converted on
// the device into the instance's scratch (other-parity) buffers, which become the committed
// ones only when every particle has finite positive mass and volume and finite kinematics, so a
// refused import leaves the simulation as it was.
lp_status import_particles(Ensemble& E, int i, const lp_particles* in) {
  lp_status st = pull_ctrl(E);
  if (st != LP_OK) return st;
  Control& c = E.ctrl_h[i];
  const InstDesc& D = E.desc[i];
  const int64_t n = (int64_t)in->count;
  if (n > D.slot_cap) return set_error(LP_INVALID, "imported particle count exceeds the instance capacity");
  if (n > 0 && (!in->id || !in->position || !in->velocity || !in->affine || !in->deformation || !in->kirchhoff ||
                !in->volume_ratio || !in->plastic_strain || !in->mass || !in->volume0))
    return set_error(LP_INVALID, "imported particles need every array but yield_stress");
  st = stage_alloc(E, n);
  if (st != LP_OK) return st;
  const int par = c.parity ^ 1;
  const unsigned long long none = ~0ull;
  CUDA_CK(cudaMemcpyAsync(E.d_bad, &none, sizeof(none), cudaMemcpyHostToDevice, E.stream));
  // Chunk k goes through staging slot k % 2: host threads fill the slot's pinned twin while the
  // device still copies and converts chunk k - 1 from the other slot; a slot is refilled only
  // after the event of the chunk that last used it.  Page-locked caller arrays go to the slot by
  // DMA directly, in stream order, with no host copy and no wait.
  const bool direct = particles_page_locked(in, n);
  int64_t k = 0;
  for (int64_t first = 0; first < n; first += E.stage_particles, ++k) {
    const int slot = (int)(k & 1);
    const int64_t m = std::min(E.stage_particles, n - first);
    const size_t d1 = sizeof(double) * (size_t)m;
    lp::HostParticleChunk h;
    stage_slot(E, slot, h);
    if (direct) {
      lp::HostParticleChunk hc = h;
      auto up = [&](void* dst, const void* src, size_t bytes) -> lp_status {
        CUDA_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, E.stream));
        return LP_OK;
      };
      if (up(h.id, in->id + first, sizeof(uint32_t) * (size_t)m) != LP_OK ||
          up(h.position, in->position + 3 * first, 3 * d1) != LP_OK ||
          up(h.velocity, in->velocity + 3 * first, 3 * d1) != LP_OK ||
          up(h.affine, in->affine + 9 * first, 9 * d1) != LP_OK ||
          up(h.deformation, in->deformation + 9 * first, 9 * d1) != LP_OK ||
          up(h.kirchhoff, in->kirchhoff + 9 * first, 9 * d1) != LP_OK ||
          up(h.volume_ratio, in->volume_ratio + first, d1) != LP_OK ||
          up(h.plastic_strain, in->plastic_strain + first, d1) != LP_OK ||
          up(h.mass, in->mass + first, d1) != LP_OK || up(h.volume0, in->volume0 + first, d1) != LP_OK)
        return LP_DEVICE;
      if (in->yield_stress) {
        if (up(h.yield_stress, in->yield_stress + first, d1) != LP_OK) return LP_DEVICE;
      } else {
        hc.yield_stress = nullptr;
      }
      lp::launch_import(hc, m, first, E.A.st[par], E.A.id[par], E.A.cap, D.slot_off, D.yield, E.d_bad, E.stream);
      CUDA_CK(cudaGetLastError());
      continue;
    }
    if (k >= 2) CUDA_CK(cudaEventSynchronize(E.stage_ev[slot]));
    // caller arrays -> pinned twin (host threads) -> device staging (one copy per field)
    std::vector<CopySpan> spans = {
        {host_twin(E, h.id), in->id + first, sizeof(uint32_t) * (size_t)m},
        {host_twin(E, h.position), in->position + 3 * first, 3 * d1},
        {host_twin(E, h.velocity), in->velocity + 3 * first, 3 * d1},
        {host_twin(E, h.affine), in->affine + 9 * first, 9 * d1},
        {host_twin(E, h.deformation), in->deformation + 9 * first, 9 * d1},
        {host_twin(E, h.kirchhoff), in->kirchhoff + 9 * first, 9 * d1},
        {host_twin(E, h.volume_ratio), in->volume_ratio + first, d1},
        {host_twin(E, h.plastic_strain), in->plastic_strain + first, d1},
        {host_twin(E, h.mass), in->mass + first, d1},
        {host_twin(E, h.volume0), in->volume0 + first, d1}};
    lp::HostParticleChunk hc = h;
    if (in->yield_stress) spans.push_back({host_twin(E, h.yield_stress), in->yield_stress + first, d1});
    else hc.yield_stress = nullptr;
    parallel_copy(spans);
    for (const CopySpan& c : spans)
      CUDA_CK(cudaMemcpyAsync((char*)E.d_stage + ((const char*)c.dst - (const char*)E.h_stage), c.dst, c.bytes,
                              cudaMemcpyHostToDevice, E.stream));
    lp::launch_import(hc, m, first, E.A.st[par], E.A.id[par], E.A.cap, D.slot_off, D.yield, E.d_bad, E.stream);
    CUDA_CK(cudaGetLastError());
    CUDA_CK(cudaEventRecord(E.stage_ev[slot], E.stream));  // the slot is free again after this
  }
  unsigned long long bad = none;
  CUDA_CK(cudaMemcpyAsync(&bad, E.d_bad, sizeof(bad), cudaMemcpyDeviceToHost, E.stream));
  CUDA_CK(cudaStreamSynchronize(E.stream));
  if (bad != none)
    return set_error(LP_INVALID, "particle id '" + std::to_string(in->id[bad]) + "' has non-finite state");
  c.parity = par;
  c.count = n;
  st = push_ctrl(E);
  if (st != LP_OK) return st;
  return refresh_stats(E);
}

void ledger_out(const lp::LedgerD& L, lp_ledger* o) {
  static_assert(sizeof(lp::LedgerD) == sizeof(lp_ledger), "ledger layouts differ");
  std::memcpy(o, &L, sizeof(L));
}

void counters_out(const Control& c, lp_counters* o) {
  o->time = c.time;
  o->step_count = c.step_count;
  o->limited_steps = c.limited_steps;
  o->rejected_steps = c.rejected_steps;
  o->dt_scale = c.dt_scale;
  o->min_dt_used = c.min_dt_used;
  o->max_dt_used = c.max_dt_used;
  o->particle_count = (uint64_t)c.count;
  o->newton_iterations = c.newton_iterations;
  o->yielded_particles = c.yielded;
}

// fixtures.rs:369-606 assembled from device reductions
lp_status observables(Ensemble& E, int i, std::map<std::string, double>& out) {
  std::vector<Diag> d;
  lp_status st = diagnostics(E, d);
  if (st != LP_OK) return st;
  st = pull_ctrl(E);
  if (st != LP_OK) return st;
  const Control& c = E.ctrl_h[i];
  const InstDesc& D = E.desc[i];
  const lp_fixture_spec& s = E.specs[i];
  const Diag& g = d[i];
  Energies en = energies_of(E, i, g);
  const lp::LedgerD& L = c.ledger;
  const double sub = s.grid_spacing / 2.0;
  const double n = (double)c.count;
  out["mass_residual_kg"] = en.mass_res;
  out["momentum_residual_kg_m_s"] =
      std::sqrt(en.mom_res[0] * en.mom_res[0] + en.mom_res[1] * en.mom_res[1] + en.mom_res[2] * en.mom_res[2]);
  out["kinetic_energy_j"] = en.ke;
  out["potential_energy_j"] = en.pe;
  out["elastic_energy_j"] = en.ee;
  out["mechanical_energy_j"] = en.mech;
  out["plastic_dissipation_j"] = L.plastic;
  out["wall_normal_projection_energy_j"] = L.proj;
  out["wall_friction_dissipation_j"] = L.fric;
  out["wall_normal_traction_energy_j"] = L.trac;
  out["energy_residual_j"] = en.e_res;
  out["outflow_kg"] = L.outflow_mass;
  out["particle_count"] = n;
  out["step_count"] = (double)c.step_count;
  out["limited_steps"] = (double)c.limited_steps;
  out["rejected_steps"] = (double)c.rejected_steps;
  out["min_dt_s"] = std::isfinite(c.min_dt_used) ? c.min_dt_used : 0.0;
  out["max_dt_s"] = c.max_dt_used;
  out["max_speed_m_s"] = g.max_speed;
  out["max_plastic_strain"] = g.max_ep;
  out["yielded_fraction"] = n > 0 ? g.yielded / n : 0.0;
  const double height = n > 0 ? g.max_z + 0.5 * sub : 0.0;
  out["height_m"] = height;
  out["spread_x_m"] = n > 0 ? g.max_x - g.min_x + sub : 0.0;
  out["spread_y_m"] = n > 0 ? g.max_y - g.min_y + sub : 0.0;
  const double gn = std::sqrt(D.gravity[0] * D.gravity[0] + D.gravity[1] * D.gravity[1] + D.gravity[2] * D.gravity[2]);
  if (s.fixture == LP_SLUMP) {
    const double h0 = s.initial_size[2];
    out["slump_m"] = h0 - height;
    const double tp = (D.yield / std::sqrt(3.0)) / (D.density * gn * h0);
    out["dimensionless_yield_stress"] = tp;
    out["pashias_slump_m"] = tp >= 0.5 ? 0.0 : (tp <= 0.0 ? h0 : h0 * (1.0 - 2.0 * tp * (1.0 - std::log(2.0 * tp))));
  } else if (s.fixture == LP_HYDROSTATIC) {
    const double h0 = s.initial_size[2];
    out["hydrostatic_rms_relative_error"] = n > 0 ? std::sqrt(g.hsq / n) : 0.0;
    out["hydrostatic_max_relative_error"] = g.hmax;
    out["reference_bottom_stress_pa"] =
        D.kind == 1 ? D.bulk * (std::exp(D.density * gn * h0 / D.bulk) - 1.0) : D.density * gn * h0;
    out["wave_speed_m_s"] = D.kind == 0 ? std::sqrt((D.lambda + 2.0 * D.mu) / D.density) : std::sqrt(D.bulk / D.density);
  } else if (s.fixture == LP_DAM_BREAK) {
    out["front_x_m"] = n > 0 ? g.max_x + 0.5 * sub : 0.0;
    const double ritter = s.initial_size[0] + 2.0 * std::sqrt(gn * s.initial_size[2]) * c.time;
    out["ritter_front_bound_m"] = std::min(ritter, s.domain[0]);
    out["column_height_m"] = g.column > -1e299 ? g.column + 0.5 * sub : 0.0;
  } else if (s.fixture == LP_COUPLED_PATCH && D.has_pellet) {
    const lp::PelletState& P = c.pellet;
    out["pellet_x_m"] = P.pos[0];
    out["pellet_y_m"] = P.pos[1];
    out["pellet_z_m"] = P.pos[2];
    out["pellet_speed_m_s"] = std::sqrt(P.vel[0] * P.vel[0] + P.vel[1] * P.vel[1] + P.vel[2] * P.vel[2]);
    double om[3];
    pellet_omega_h(P, om);
    out["pellet_angular_speed_rad_s"] = std::sqrt(om[0] * om[0] + om[1] * om[1] + om[2] * om[2]);
    out["pellet_kinetic_energy_j"] = pellet_ke_h(P);
    out["pellet_penetration_m"] = std::max(s.initial_size[2] + P.radius - P.pos[2], 0.0);
    // tilt of the body axis R x_hat out of the horizontal plane
    double R[3][3];
    q_matrix(P.q, R);
    out["pellet_axis_tilt_rad"] = std::asin(std::min(std::fabs(R[2][0]), 1.0));
    out["coupling_impulse_x_kg_m_s"] = L.coupling_impulse[0];
    out["coupling_impulse_y_kg_m_s"] = L.coupling_impulse[1];
    out["coupling_impulse_z_kg_m_s"] = L.coupling_impulse[2];
    out["coupling_angular_impulse_x_kg_m2_s"] = L.coupling_angular[0];
    out["coupling_angular_impulse_y_kg_m2_s"] = L.coupling_angular[1];
    out["coupling_angular_impulse_z_kg_m2_s"] = L.coupling_angular[2];
    out["pellet_wall_impulse_z_kg_m_s"] = L.pellet_wall_impulse[2];
    out["pellet_wall_work_j"] = L.pellet_work;
    out["coupling_grid_energy_j"] = L.cgrid;
    out["coupling_pellet_energy_j"] = L.cpellet;
  }
  if (D.bed_np >= 2) {
    const std::vector<lp::PelletState> B = bed_pull(E, i);
    double zs = 0.0, zmin = 1e300, vmax = 0.0, ke = 0.0;
    for (const lp::PelletState& P : B) {
      zs += P.pos[2];
      zmin = std::min(zmin, P.pos[2]);
      vmax = std::max(vmax, std::sqrt(P.vel[0] * P.vel[0] + P.vel[1] * P.vel[1] + P.vel[2] * P.vel[2]));
      ke += pellet_ke_h(P);
    }
    out["pellet_count"] = (double)B.size();
    out["pellet_mean_z_m"] = zs / (double)B.size();
    out["pellet_min_z_m"] = zmin;
    out["pellet_max_speed_m_s"] = vmax;
    out["pellet_kinetic_energy_j"] = ke;
    out["pellet_contact_work_j"] = c.bed_contact_work;
    out["pellet_contacts"] = (double)c.bed_contacts;
    out["pellet_history_overflow"] = (double)c.bed_overflow;
    out["pellet_wall_work_j"] = L.pellet_work;
    out["coupling_grid_energy_j"] = L.cgrid;
    out["coupling_pellet_energy_j"] = L.cpellet;
    out["coupling_impulse_z_kg_m_s"] = L.coupling_impulse[2];
  }
  return LP_OK;
}

}  // namespace

void lp::set_last_error(const char* msg) { g_err = msg; }

// ================================================================ C ABI
struct lp_sim {
  Ensemble E;
};
struct lp_batch {
  Ensemble E;
};

extern "C" {

int32_t lp_abi_version(void) { return LP_ABI_VERSION; }
const char* lp_last_error(void) { return g_err.c_str(); }
uint64_t lp_kernel_launches(void) { return lp::kernel_launch_count(); }
void lp_abi_struct_sizes(uint64_t out[6]) {
  out[0] = sizeof(lp_material);
  out[1] = sizeof(lp_fixture_spec);
  out[2] = sizeof(lp_ledger);
  out[3] = sizeof(lp_counters);
  out[4] = sizeof(lp_particles);
  out[5] = sizeof(lp_pellet);
}

lp_material lp_material_paste(double density, double e, double nu, double ys, double k, double n) {
  lp_material m;
  std::memset(&m, 0, sizeof(m));
  m.kind = LP_PASTE;
  m.density = density;
  m.shear_modulus = e / (2.0 * (1.0 + nu));
  m.lame_lambda = e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  m.bulk_modulus = m.lame_lambda + 2.0 * m.shear_modulus / 3.0;
  m.yield_stress = ys;
  m.consistency = k;
  m.flow_index = n;
  m.tait_gamma = 1.0;
  return m;
}
lp_material lp_material_paste_from_shear_rheology(double density, double e, double nu, double tys, double ks, double n) {
  return lp_material_paste(density, e, nu, std::sqrt(3.0) * tys, std::pow(3.0, (1.0 + n) / 2.0) * ks, n);
}
lp_material lp_material_liquid(double density, double e, double nu, double viscosity) {
  lp_material m;
  std::memset(&m, 0, sizeof(m));
  m.kind = LP_LIQUID;
  m.density = density;
  m.bulk_modulus = e / (3.0 * (1.0 - 2.0 * nu));
  m.consistency = viscosity;
  m.flow_index = 1.0;
  m.tait_gamma = 1.0;
  return m;
}
double lp_material_wave_speed(const lp_material* m) {
  const double modulus = m->kind == LP_PASTE ? m->lame_lambda + 2.0 * m->shear_modulus : m->bulk_modulus;
  return std::sqrt(modulus / m->density);
}
double lp_material_diffusivity(const lp_material* m) { return m->kind == LP_PASTE ? 0.0 : m->consistency / m->density; }

lp_status lp_sim_create(const lp_fixture_spec* spec, lp_sim** out) {
  if (!spec || !out) return set_error(LP_INVALID, "null argument");
  *out = nullptr;
  lp_sim* s = new lp_sim();
  lp_status st = ensemble_create(spec, 1, s->E);
  if (st != LP_OK) {
    delete s;
    return st;
  }
  *out = s;
  return LP_OK;
}
void lp_sim_destroy(lp_sim* sim) { delete sim; }

lp_status lp_sim_set_stream(lp_sim* sim, void* stream) {
  sim->E.invalidate_graph();
  sim->E.stream = stream ? (cudaStream_t)stream : sim->E.own_stream;
  return LP_OK;
}

lp_status lp_sim_advance(lp_sim* sim, double target, lp_keep_going_fn keep, void* ctx, int32_t* reached) {
  return ensemble_advance(sim->E, target, keep, ctx, reached);
}

lp_status lp_sim_try_step(lp_sim* sim, double dt, int32_t* accepted, char* reason, size_t reason_len) {
  Ensemble& E = sim->E;
  if (!(dt > 0.0) || !std::isfinite(dt)) return set_error(LP_INVALID, "dt must be positive and finite");
  lp_status st = pull_ctrl(E);
  if (st != LP_OK) return st;
  E.ctrl_h[0].forced_dt = dt;
  st = push_ctrl(E);
  if (st != LP_OK) return st;
  lp::launch_attempt(E.A, E.stream);
  CUDA_CK(cudaGetLastError());
  st = pull_ctrl(E);
  if (st != LP_OK) return st;
  Control& c = E.ctrl_h[0];
  const int ok = c.fail == lp::F_OK && c.status != lp::S_ERROR;
  if (accepted) *accepted = ok;
  if (reason && reason_len) std::snprintf(reason, reason_len, "%s", ok ? "" : fail_text(c.fail));
  c.forced_dt = 0.0;
  return push_ctrl(E);
}

lp_status lp_sim_run_substeps(lp_sim* sim, int32_t steps) {
  Ensemble& E = sim->E;
  if (E.ctrl_h.empty() || !std::isinf(E.ctrl_h[0].target)) {
    lp_status st = set_targets(E, std::numeric_limits<double>::infinity(), true);
    if (st != LP_OK) return st;
  }
  return run_attempts(E, steps);
}
lp_status lp_sim_sync(lp_sim* sim) {
  CUDA_CK(cudaStreamSynchronize(sim->E.stream));
  return pull_ctrl(sim->E);
}

lp_status lp_sim_stability_limit(lp_sim* sim, double* out) {
  lp_status st = pull_ctrl(sim->E);
  if (st != LP_OK) return st;
  const Control& c = sim->E.ctrl_h[0];
  const InstDesc& D = sim->E.desc[0];
  const double wave = D.kind == 0 ? std::sqrt((D.lambda + 2.0 * D.mu) / D.density) : std::sqrt(D.bulk / D.density);
  double limit = D.cfl * D.dx / (wave + c.max_speed);
  const double diff = D.kind == 0 ? 0.0 : D.consistency / D.density;
  if (diff > 0.0) limit = std::fmin(limit, 0.25 * D.dx * D.dx / diff);
  if (D.has_pellet) {
    limit = std::fmin(limit, 0.2 * std::sqrt(c.pellet.mass / D.contact_k));
    const double ps = std::sqrt(c.pellet.vel[0] * c.pellet.vel[0] + c.pellet.vel[1] * c.pellet.vel[1] + c.pellet.vel[2] * c.pellet.vel[2]);
    if (ps > 0.0) limit = std::fmin(limit, D.cfl * D.dx / ps);
  }
  if (D.bed_np >= 2) {
    const std::vector<lp::PelletState> B = bed_pull(sim->E, 0);
    limit = std::fmin(limit, lp::bed_limit(D, B.data()));
  }
  *out = limit;
  return LP_OK;
}

lp_status lp_sim_get_ledger(lp_sim* sim, lp_ledger* out) {
  lp_status st = pull_ctrl(sim->E);
  if (st != LP_OK) return st;
  ledger_out(sim->E.ctrl_h[0].ledger, out);
  return LP_OK;
}
lp_status lp_sim_set_ledger(lp_sim* sim, const lp_ledger* in) {
  lp_status st = pull_ctrl(sim->E);
  if (st != LP_OK) return st;
  std::memcpy(&sim->E.ctrl_h[0].ledger, in, sizeof(lp_ledger));
  return push_ctrl(sim->E);
}
lp_status lp_sim_get_counters(lp_sim* sim, lp_counters* out) {
  lp_status st = pull_ctrl(sim->E);
  if (st != LP_OK) return st;
  counters_out(sim->E.ctrl_h[0], out);
  return LP_OK;
}
lp_status lp_sim_set_counters(lp_sim* sim, const lp_counters* in) {
  lp_status st = pull_ctrl(sim->E);
  if (st != LP_OK) return st;
  Control& c = sim->E.ctrl_h[0];
  if (!(in->dt_scale > 0.0 && in->dt_scale <= 1.0) || !std::isfinite(in->time) || in->time < 0.0)
    return set_error(LP_INVALID, "invalid counters");
  c.time = in->time;
  c.step_count = in->step_count;
  c.limited_steps = in->limited_steps;
  c.rejected_steps = in->rejected_steps;
  c.dt_scale = in->dt_scale;
  c.min_dt_used = in->min_dt_used;
  c.max_dt_used = in->max_dt_used;
  c.status = lp::S_RUNNING;
  return push_ctrl(sim->E);
}
lp_status lp_sim_particle_count(lp_sim* sim, uint64_t* out) {
  lp_status st = pull_ctrl(sim->E);
  if (st != LP_OK) return st;
  *out = (uint64_t)sim->E.ctrl_h[0].count;
  return LP_OK;
}
lp_status lp_sim_export_particles(lp_sim* sim, lp_particles* out) { return export_particles(sim->E, 0, out); }
lp_status lp_host_pin(void* ptr, uint64_t bytes) {
  if (!ptr || bytes == 0) return set_error(LP_INVALID, "lp_host_pin needs a non-empty buffer");
  const cudaError_t e = cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(LP_DEVICE, std::string("cudaHostRegister: ") + cudaGetErrorString(e));
  }
  return LP_OK;
}

lp_status lp_host_unpin(void* ptr) {
  if (!ptr) return set_error(LP_INVALID, "lp_host_unpin needs a buffer");
  const cudaError_t e = cudaHostUnregister(ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(LP_DEVICE, std::string("cudaHostUnregister: ") + cudaGetErrorString(e));
  }
  return LP_OK;
}

lp_status lp_sim_import_particles(lp_sim* sim, const lp_particles* in) { return import_particles(sim->E, 0, in); }

static void pellet_out(const lp::PelletState& P, lp_pellet* out) {
  std::memset(out, 0, sizeof(*out));
  out->radius = P.radius;
  out->length = P.length;
  out->mass = P.mass;
  for (int a = 0; a < 3; ++a) {
    out->inertia_body[a] = P.inertia[a];
    out->position[a] = P.pos[a];
    out->velocity[a] = P.vel[a];
    out->angular_momentum[a] = P.L[a];
  }
  for (int a = 0; a < 4; ++a) out->orientation[a] = P.q[a];
  out->sphere_count = P.nsph;
  for (int k = 0; k < P.nsph; ++k) out->sphere_offsets[k] = P.off[k];
}
lp_status lp_sim_get_pellets(lp_sim* sim, lp_pellet* out, int32_t cap, int32_t* count) {
  if (!count) return set_error(LP_INVALID, "null count");
  lp_status st = pull_ctrl(sim->E);
  if (st != LP_OK) return st;
  const std::vector<lp::PelletState> B = bed_pull(sim->E, 0);
  *count = (int32_t)B.size();
  for (int32_t p = 0; p < std::min<int32_t>(cap, (int32_t)B.size()); ++p) pellet_out(B[p], out + p);
  return LP_OK;
}
lp_status lp_sim_set_pellets(lp_sim* sim, const lp_pellet* in, int32_t count) {
  Ensemble& E = sim->E;
  lp_status st = pull_ctrl(E);
  if (st != LP_OK) return st;
  const InstDesc& D = E.desc[0];
  if (D.bed_np < 2 || count != D.bed_np || !in) return set_error(LP_INVALID, "pellet count differs from the bed's");
  std::vector<lp::PelletState> B = bed_pull(E, 0);
  for (int32_t p = 0; p < count; ++p) {
    const lp_pellet& q = in[p];
    if (q.sphere_count != B[p].nsph || q.radius != B[p].radius || q.mass != B[p].mass)
      return set_error(LP_INVALID, "pellet geometry differs from the bed's");
    for (int a = 0; a < 3; ++a) {
      B[p].pos[a] = q.position[a];
      B[p].vel[a] = q.velocity[a];
      B[p].L[a] = q.angular_momentum[a];
    }
    for (int a = 0; a < 4; ++a) B[p].q[a] = q.orientation[a];
  }
  E.invalidate_graph();
  const int par = E.ctrl_h[0].bed_parity;
  CUDA_CK(cudaMemcpy(E.A.bed.state[par] + D.bed_off, B.data(), sizeof(lp::PelletState) * B.size(),
                     cudaMemcpyHostToDevice));
  CUDA_CK(cudaMemset(E.A.bed.hist_n[par] + D.bed_off, 0, sizeof(int) * B.size()));
  E.ctrl_h[0].bed_limit = lp::bed_limit(D, B.data());
  return push_ctrl(E);
}
static lp_status get_pellet(Ensemble& E, int i, lp_pellet* out, int32_t* has) {
  lp_status st = pull_ctrl(E);
  if (st != LP_OK) return st;
  *has = E.desc[i].has_pellet;
  if (!*has) return LP_OK;
  const lp::PelletState& P = E.ctrl_h[i].pellet;
  std::memset(out, 0, sizeof(*out));
  out->radius = P.radius;
  out->length = P.length;
  out->mass = P.mass;
  for (int a = 0; a < 3; ++a) {
    out->inertia_body[a] = P.inertia[a];
    out->position[a] = P.pos[a];
    out->velocity[a] = P.vel[a];
    out->angular_momentum[a] = P.L[a];
  }
  for (int a = 0; a < 4; ++a) out->orientation[a] = P.q[a];
  out->sphere_count = P.nsph;
  for (int k = 0; k < P.nsph; ++k) out->sphere_offsets[k] = P.off[k];
  return LP_OK;
}
lp_status lp_sim_get_pellet(lp_sim* sim, lp_pellet* out, int32_t* has) { return get_pellet(sim->E, 0, out, has); }
lp_status lp_sim_set_pellet(lp_sim* sim, const lp_pellet* in) {
  lp_status st = pull_ctrl(sim->E);
  if (st != LP_OK) return st;
  if (!sim->E.desc[0].has_pellet) return set_error(LP_INVALID, "simulation has no pellet");
  if (in->sphere_count < 1 || in->sphere_count > 64) return set_error(LP_INVALID, "invalid pellet sphere count");
  lp::PelletState& P = sim->E.ctrl_h[0].pellet;
  P.radius = in->radius;
  P.length = in->length;
  P.mass = in->mass;
  for (int a = 0; a < 3; ++a) {
    P.inertia[a] = in->inertia_body[a];
    P.pos[a] = in->position[a];
    P.vel[a] = in->velocity[a];
    P.L[a] = in->angular_momentum[a];
  }
  for (int a = 0; a < 4; ++a) P.q[a] = in->orientation[a];
  P.nsph = in->sphere_count;
  for (int k = 0; k < P.nsph; ++k) P.off[k] = in->sphere_offsets[k];
  return push_ctrl(sim->E);
}

lp_status lp_sim_observables(lp_sim* sim, char* names, double* values, int32_t capacity, int32_t* count) {
  std::map<std::string, double> obs;
  lp_status st = observables(sim->E, 0, obs);
  if (st != LP_OK) return st;
  int32_t n = 0;
  for (auto& kv : obs) {
    if (n >= capacity) break;
    std::snprintf(names + 64 * n, 64, "%s", kv.first.c_str());
    values[n] = kv.second;
    ++n;
  }
  *count = n;
  return LP_OK;
}

lp_status lp_sim_energies(lp_sim* sim, double out[9]) {
  std::vector<Diag> d;
  lp_status st = diagnostics(sim->E, d);
  if (st != LP_OK) return st;
  st = pull_ctrl(sim->E);
  if (st != LP_OK) return st;
  Energies en = energies_of(sim->E, 0, d[0]);
  out[0] = en.ke;
  out[1] = en.pe;
  out[2] = en.ee;
  out[3] = en.mech;
  out[4] = en.mass_res;
  out[5] = en.mom_res[0];
  out[6] = en.mom_res[1];
  out[7] = en.mom_res[2];
  out[8] = en.e_res;
  return LP_OK;
}

// ---------------------------------------------------------------- energy audit (audit.rs)
// EnergyState::measure (audit.rs:38-53) of the committed state of instance 0: translation,
// APIC affine norm h^2/8 sum m |C|^2, elastic, potential (material and pellets), pellet kinetic.
static lp_status audit_state(Ensemble& E, double out[5]) {
  std::vector<Diag> d;
  lp_status st = diagnostics(E, d);
  if (st != LP_OK) return st;
  st = pull_ctrl(E);
  if (st != LP_OK) return st;
  const Energies en = energies_of(E, 0, d[0]);
  const InstDesc& D = E.desc[0];
  double pellet = 0.0;
  if (D.has_pellet) pellet += pellet_ke_h(E.ctrl_h[0].pellet);
  if (D.bed_np >= 2)
    for (const lp::PelletState& P : bed_pull(E, 0)) pellet += pellet_ke_h(P);
  out[0] = d[0].ke;
  out[1] = D.dx * D.dx / 8.0 * d[0].cnorm;
  out[2] = d[0].ee;
  out[3] = en.pe;
  out[4] = pellet;
  return LP_OK;
}

// EnergyTerms::measure (audit.rs:214-243)
static void audit_terms(lp_energy_audit& a) {
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
  const double t[12] = {p2g,        g2p,      stress, a.coupled ? nan : gravity, a.coupled ? gravity : nan,
                        integrator, traction, walls,  coupling,                  change, sum, change - sum};
  for (int k = 0; k < 12; ++k) a.terms[k] = t[k];
}

// Simulation::audit_step (audit.rs:284-353): one trial step of exactly dt with its stage energies;
// the committed state (particles, pellets, ledger, counters) is left as it was.
lp_status lp_sim_audit_step(lp_sim* sim, double dt, lp_energy_audit* out) {
  if (!sim || !out) return set_error(LP_INVALID, "null argument");
  Ensemble& E = sim->E;
  std::memset(out, 0, sizeof(*out));
  double stability = 0.0;
  lp_status st = lp_sim_stability_limit(sim, &stability);
  if (st != LP_OK) return st;
  const Control saved = E.ctrl_h[0];
  const InstDesc& D = E.desc[0];
  const lp_fixture_spec& S = E.specs[0];
  if (!(std::isfinite(S.gravity[0]) && std::isfinite(S.gravity[1]) && std::isfinite(S.gravity[2])) ||
      !std::isfinite(S.cfl) || S.cfl <= 0.0 || !std::isfinite(S.wall_friction) || S.wall_friction < 0.0 ||
      !std::isfinite(S.min_dt) || S.min_dt <= 0.0 || !std::isfinite(S.max_dt) || S.max_dt < S.min_dt ||
      !std::isfinite(stability) || stability <= 0.0)
    return set_error(LP_INVALID, "invalid solver state: invalid audit step configuration or stability limit");
  const double limit = std::fmin(saved.dt_scale * stability, D.max_dt);
  if (!std::isfinite(dt) || dt <= 0.0 || dt < D.min_dt || !std::isfinite(limit) || dt > limit) {
    char buf[200];
    std::snprintf(buf, sizeof(buf),
                  "invalid solver state: audit `dt`='%.17g' outside finite accepted range ending at '%.17g'", dt, limit);
    return set_error(LP_INVALID, buf);
  }
  if (saved.status != lp::S_RUNNING && saved.status != lp::S_REACHED)
    return set_error(LP_INVALID, "invalid solver state: the simulation has stopped");
  out->time = saved.time;
  out->dt = dt;
  out->coupled = (D.has_pellet || D.bed_np >= 2) ? 1 : 0;
  st = audit_state(E, out->before);
  if (st != LP_OK) return st;
  for (double v : out->before)
    if (!std::isfinite(v)) return set_error(LP_INVALID, "invalid solver state: nonfinite initial audit energy");
  if (!E.d_audit) {
    st = E.alloc(&E.d_audit, (size_t)6 * E.A.n_gcta);
    if (st != LP_OK) return st;
  }
  CUDA_CK(cudaMemsetAsync(E.d_audit, 0, sizeof(double) * 6 * E.A.n_gcta, E.stream));
  E.ctrl_h[0].forced_dt = dt;
  st = push_ctrl(E);
  if (st != LP_OK) return st;
  lp::launch_audit(E.A, E.d_audit, E.stream);
  CUDA_CK(cudaGetLastError());
  std::vector<double> raw((size_t)6 * E.A.n_gcta);
  CUDA_CK(cudaMemcpyAsync(raw.data(), E.d_audit, sizeof(double) * raw.size(), cudaMemcpyDeviceToHost, E.stream));
  std::vector<lp::BedStep> bstep((size_t)std::max(D.bed_np, 0));
  if (D.bed_np >= 2)
    CUDA_CK(cudaMemcpyAsync(bstep.data(), E.A.bed_step + D.bed_off, sizeof(lp::BedStep) * bstep.size(),
                            cudaMemcpyDeviceToHost, E.stream));
  st = pull_ctrl(E);
  if (st != LP_OK) return st;
  const Control trial = E.ctrl_h[0];
  // put the committed state back; the trial wrote only the other particle and bed buffers.
  // The attempt epoch stays advanced so that node blocks marked by the trial never look active.
  auto restore = [&]() {
    Control r = saved;
    r.epoch = trial.epoch;
    r.forced_dt = 0.0;
    E.ctrl_h[0] = r;
    return push_ctrl(E);
  };
  if (trial.fail != lp::F_OK || trial.status == lp::S_ERROR) {
    const int f = trial.fail != lp::F_OK ? trial.fail : lp::F_OUTFLOW;
    st = restore();
    if (st != LP_OK) return st;
    return set_error(LP_INVALID, std::string("invalid solver state: audit trial rejected: ") + fail_text(f));
  }
  st = audit_state(E, out->after);
  if (st != LP_OK) {
    restore();
    return st;
  }
  const int64_t g0 = D.gcta_off, g1 = D.gcta_off + D.gcta_cnt, ng = E.A.n_gcta;
  double stage[5] = {0, 0, 0, 0, 0}, transport = 0.0;
  for (int64_t c = g0; c < g1; ++c) {
    for (int k = 0; k < 4; ++k) stage[k] += raw[(size_t)(4 * c + k)];
    stage[4] += raw[(size_t)(4 * ng + c)];
    transport += raw[(size_t)(5 * ng + c)];
  }
  double pellet_after = 0.0;
  if (D.has_pellet) pellet_after += pellet_ke_h(saved.pellet) + trial.c_pellet_energy;
  if (D.bed_np >= 2) {
    E.ctrl_h[0].bed_parity = saved.bed_parity;
    const std::vector<lp::PelletState> B0 = bed_pull(E, 0);
    for (size_t p = 0; p < B0.size(); ++p) pellet_after += pellet_ke_h(B0[p]) + bstep[p].cpellet;
  }
  const double stg[8] = {transport, stage[0], stage[1], stage[2], stage[3], stage[4], pellet_after, trial.step_diss};
  for (int k = 0; k < 8; ++k) out->stages[k] = stg[k];
  const lp::LedgerD& l0 = saved.ledger;
  const lp::LedgerD& l1 = trial.ledger;
  const double inc[7] = {l1.plastic - l0.plastic, l1.fric - l0.fric, l1.proj - l0.proj, l1.trac - l0.trac,
                         l1.cgrid - l0.cgrid, l1.cpellet - l0.cpellet, l1.pellet_work - l0.pellet_work};
  for (int k = 0; k < 7; ++k) out->increments[k] = inc[k];
  audit_terms(*out);
  st = restore();
  if (st != LP_OK) return st;
  bool finite = true;
  for (double v : out->after) finite = finite && std::isfinite(v);
  for (double v : out->stages) finite = finite && std::isfinite(v);
  for (double v : out->increments) finite = finite && std::isfinite(v);
  for (int k = 0; k < 12; ++k)
    if (!((k == 3 && out->coupled) || (k == 4 && !out->coupled))) finite = finite && std::isfinite(out->terms[k]);
  if (!finite) return set_error(LP_INVALID, "invalid solver state: audit energy became nonfinite");
  return LP_OK;
}

static lp_status set_warm(Ensemble& E, const float* w, int32_t nw, int32_t enable) {
  if (enable) {
    if (!w || nw != lp::MLP_NW) return set_error(LP_INVALID, "warm start needs the full MLP weight vector");
    if (!E.d_mlp) {
      lp_status st = E.alloc(&E.d_mlp, lp::MLP_NW);
      if (st != LP_OK) return st;
    }
    if (!E.d_mlp_pk) {
      lp_status st = E.alloc(&E.d_mlp_pk, 1);
      if (st != LP_OK) return st;
    }
    if (!E.A.mlp_tab) {
      lp_status st = E.alloc(&E.A.mlp_tab, (size_t)E.A.n_inst * lp::MLP_TAB_FLOATS);
      if (st != LP_OK) return st;
      st = E.alloc(&E.A.mlp_tab_dt, (size_t)E.A.n_inst);
      if (st != LP_OK) return st;
    }
    CUDA_CK(cudaMemcpyAsync(E.d_mlp, w, sizeof(float) * lp::MLP_NW, cudaMemcpyHostToDevice, E.stream));
    lp::launch_mlp_pack(E.d_mlp, E.d_mlp_pk, E.stream);
    CUDA_CK(cudaGetLastError());
    // new weights: every instance's logit table is rebuilt on its next attempt (NaN never equals dt)
    CUDA_CK(cudaMemsetAsync(E.A.mlp_tab_dt, 0xff, sizeof(double) * (size_t)E.A.n_inst, E.stream));
    E.A.mlp = E.d_mlp_pk;
  }
  E.invalidate_graph();
  lp_status st = pull_ctrl(E);
  if (st != LP_OK) return st;
  for (auto& c : E.ctrl_h) c.warm_start = enable ? 1 : 0;
  E.A.warm = enable ? 1 : 0;
  return push_ctrl(E);
}
lp_status lp_sim_set_warm_start(lp_sim* sim, const float* w, int32_t nw, int32_t enable) {
  return set_warm(sim->E, w, nw, enable);
}
static_assert(LP_MLP_TAB_N == lp::MLP_TAB_N, "table size of the C header");
static lp_status warm_table(Ensemble& E, int32_t inst, float* out, int32_t capacity, double* dt) {
  if (!out || !dt) return set_error(LP_INVALID, "null output");
  if (inst < 0 || inst >= E.A.n_inst) return set_error(LP_INVALID, "instance out of range");
  if (capacity < lp::MLP_TAB_N) return set_error(LP_INVALID, "capacity below LP_MLP_TAB_N");
  *dt = std::numeric_limits<double>::quiet_NaN();
  if (!E.A.mlp_tab) return LP_OK;
  double built = 0.0;
  CUDA_CK(cudaMemcpyAsync(&built, E.A.mlp_tab_dt + inst, sizeof(double), cudaMemcpyDeviceToHost, E.stream));
  CUDA_CK(cudaStreamSynchronize(E.stream));
  if (!(built > 0.0)) return LP_OK;  // never built (0) or stale (NaN)
  CUDA_CK(cudaMemcpyAsync(out, E.A.mlp_tab + (size_t)inst * lp::MLP_TAB_FLOATS, sizeof(float) * lp::MLP_TAB_N,
                          cudaMemcpyDeviceToHost, E.stream));
  CUDA_CK(cudaStreamSynchronize(E.stream));
  *dt = built;
  return LP_OK;
}
lp_status lp_sim_warm_table(lp_sim* sim, float* out, int32_t capacity, double* dt) {
  return warm_table(sim->E, 0, out, capacity, dt);
}
lp_status lp_sim_grid_totals(lp_sim* sim, double dt, double out[8]) {
  Ensemble& E = sim->E;
  if (!(dt > 0.0)) return set_error(LP_INVALID, "dt must be positive");
  lp_status st = pull_ctrl(E);
  if (st != LP_OK) return st;
  E.ctrl_h[0].forced_dt = dt;
  st = push_ctrl(E);
  if (st != LP_OK) return st;
  long long* d = nullptr;
  CUDA_CK(cudaMalloc(&d, 4 * sizeof(long long)));
  CUDA_CK(cudaMemsetAsync(d, 0, 4 * sizeof(long long), E.stream));
  lp::launch_grid_totals(E.A, d, E.stream);
  CUDA_CK(cudaGetLastError());
  long long h[4];
  CUDA_CK(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, E.stream));
  CUDA_CK(cudaMemsetAsync(E.A.acc, 0, sizeof(long long) * 4 * E.A.node_total, E.stream));
  CUDA_CK(cudaMemsetAsync(E.A.trac, 0, sizeof(long long) * 6 * E.A.node_total, E.stream));
  CUDA_CK(cudaStreamSynchronize(E.stream));
  cudaFree(d);
  st = pull_ctrl(E);
  if (st != LP_OK) return st;
  const Control& c = E.ctrl_h[0];
  out[0] = (double)h[0] / E.desc[0].s_mass;
  for (int a = 0; a < 3; ++a) out[1 + a] = (double)h[1 + a] / c.s_mom;
  std::vector<Diag> dg;
  st = diagnostics(E, dg);
  if (st != LP_OK) return st;
  out[4] = dg[0].mass;
  for (int a = 0; a < 3; ++a) out[5 + a] = dg[0].mom[a];
  E.ctrl_h[0].forced_dt = 0.0;
  return push_ctrl(E);
}

// Mean per-kernel duration of `steps` attempts of the whole ensemble, CUDA events between the
// kernels on the ensemble's stream.
static lp_status ensemble_kernel_times(Ensemble& E, int32_t steps, double* ms, char* names, int32_t capacity,
                                       int32_t* count) {
  if (E.ctrl_h.empty() || !std::isinf(E.ctrl_h[0].target)) {
    lp_status st = set_targets(E, std::numeric_limits<double>::infinity(), true);
    if (st != LP_OK) return st;
  }
  cudaEvent_t ev[24];
  for (int k = 0; k < 24; ++k) CUDA_CK(cudaEventCreate(&ev[k]));
  std::vector<double> acc(24, 0.0);
  int nk = 0;
  for (int s = 0; s < steps; ++s) {
    nk = lp::launch_attempt(E.A, E.stream, ev);
    CUDA_CK(cudaGetLastError());
    CUDA_CK(cudaEventSynchronize(ev[nk]));
    for (int k = 0; k < nk; ++k) {
      float t = 0.f;
      CUDA_CK(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
      acc[k] += t;
    }
  }
  for (int k = 0; k < 24; ++k) cudaEventDestroy(ev[k]);
  const int n = std::min(nk, (int)capacity);
  for (int k = 0; k < n; ++k) {
    ms[k] = acc[k] / std::max(steps, 1);
    std::snprintf(names + 32 * k, 32, "%s", lp::attempt_kernel_name(k, E.A.any_pellet, E.A.any_bed,
                                                                    E.A.mlp && E.A.mlp_tab && E.A.warm));
  }
  *count = n;
  return pull_ctrl(E);
}

lp_status lp_sim_kernel_times(lp_sim* sim, int32_t steps, double* ms, char* names, int32_t capacity,
                              int32_t* count) {
  return ensemble_kernel_times(sim->E, steps, ms, names, capacity, count);
}

lp_status lp_batch_kernel_times(lp_batch* b, int32_t steps, double* ms, char* names, int32_t capacity,
                                int32_t* count) {
  return ensemble_kernel_times(b->E, steps, ms, names, capacity, count);
}

lp_status lp_sim_grid_dump(lp_sim* sim, double dt, double* mass, double* momentum, double* reaction,
                           int64_t node_count) {
  Ensemble& E = sim->E;
  const int64_t nn = (int64_t)E.desc[0].nodes[0] * E.desc[0].nodes[1] * E.desc[0].nodes[2];
  if (node_count != nn) return set_error(LP_INVALID, "node_count does not match the grid");
  lp_status st = pull_ctrl(E);
  if (st != LP_OK) return st;
  E.ctrl_h[0].forced_dt = dt;
  st = push_ctrl(E);
  if (st != LP_OK) return st;
  lp::launch_p2g_traction(E.A, E.stream);
  CUDA_CK(cudaGetLastError());
  std::vector<long long> acc(4 * nn), tr(6 * nn);
  for (int k = 0; k < 4; ++k)
    CUDA_CK(cudaMemcpyAsync(acc.data() + k * nn, E.A.acc + k * E.A.node_total, sizeof(long long) * nn,
                            cudaMemcpyDeviceToHost, E.stream));
  for (int k = 0; k < 6; ++k)
    CUDA_CK(cudaMemcpyAsync(tr.data() + k * nn, E.A.trac + k * E.A.node_total, sizeof(long long) * nn,
                            cudaMemcpyDeviceToHost, E.stream));
  CUDA_CK(cudaMemsetAsync(E.A.acc, 0, sizeof(long long) * 4 * E.A.node_total, E.stream));
  CUDA_CK(cudaMemsetAsync(E.A.trac, 0, sizeof(long long) * 6 * E.A.node_total, E.stream));
  st = pull_ctrl(E);
  if (st != LP_OK) return st;
  const double sm = E.desc[0].s_mass, sp = E.ctrl_h[0].s_mom;
  for (int64_t g = 0; g < nn; ++g) {
    if (mass) mass[g] = (double)acc[g] / sm;
    for (int a = 0; a < 3; ++a) {
      if (momentum) momentum[3 * g + a] = (double)acc[(1 + a) * nn + g] / sp;
      if (reaction) reaction[3 * g + a] = ((double)tr[a * nn + g] - (double)tr[(a + 3) * nn + g]) / sp;
    }
  }
  E.ctrl_h[0].forced_dt = 0.0;
  return push_ctrl(E);
}

lp_status lp_sim_use_graph(lp_sim* sim, int32_t steps) {
  sim->E.invalidate_graph();
  sim->E.graph_steps = steps > 0 ? steps : 0;
  return LP_OK;
}

lp_status lp_sim_prepare(lp_sim* sim) { return ensure_graph(sim->E); }

lp_status lp_sim_enable_newton_log(lp_sim* sim, int64_t capacity) {
  Ensemble& E = sim->E;
  E.invalidate_graph();
  if (capacity <= 0) {
    E.A.log_n = nullptr;
    return LP_OK;
  }
  lp_status st = E.alloc(&E.A.log_x, (size_t)capacity * 6);
  if (st != LP_OK) return st;
  st = E.alloc(&E.A.log_y, (size_t)capacity);
  if (st != LP_OK) return st;
  st = E.alloc(&E.A.log_n, 1);
  if (st != LP_OK) return st;
  E.A.log_cap = capacity;
  return LP_OK;
}
lp_status lp_sim_read_newton_log(lp_sim* sim, float* x, float* y, int64_t capacity, int64_t* count) {
  Ensemble& E = sim->E;
  if (!E.A.log_n) return set_error(LP_INVALID, "newton log not enabled");
  unsigned long long n = 0;
  CUDA_CK(cudaMemcpyAsync(&n, E.A.log_n, sizeof(n), cudaMemcpyDeviceToHost, E.stream));
  CUDA_CK(cudaStreamSynchronize(E.stream));
  int64_t m = std::min<int64_t>((int64_t)n, std::min<int64_t>(capacity, E.A.log_cap));
  if (m > 0) {
    CUDA_CK(cudaMemcpyAsync(x, E.A.log_x, sizeof(float) * 6 * m, cudaMemcpyDeviceToHost, E.stream));
    CUDA_CK(cudaMemcpyAsync(y, E.A.log_y, sizeof(float) * m, cudaMemcpyDeviceToHost, E.stream));
    CUDA_CK(cudaStreamSynchronize(E.stream));
  }
  *count = m;
  return LP_OK;
}

// ---------------- batch
lp_status lp_batch_create(const lp_fixture_spec* specs, int32_t count, lp_batch** out) {
  if (!specs || !out) return set_error(LP_INVALID, "null argument");
  *out = nullptr;
  lp_batch* b = new lp_batch();
  lp_status st = ensemble_create(specs, count, b->E);
  if (st != LP_OK) {
    delete b;
    return st;
  }
  *out = b;
  return LP_OK;
}
void lp_batch_destroy(lp_batch* b) { delete b; }
lp_status lp_batch_set_stream(lp_batch* b, void* stream) {
  b->E.invalidate_graph();
  b->E.stream = stream ? (cudaStream_t)stream : b->E.own_stream;
  return LP_OK;
}
lp_status lp_batch_advance(lp_batch* b, double target, lp_keep_going_fn keep, void* ctx, int32_t* all) {
  return ensemble_advance(b->E, target, keep, ctx, all);
}
lp_status lp_batch_run_substeps(lp_batch* b, int32_t steps) {
  Ensemble& E = b->E;
  if (E.ctrl_h.empty() || !std::isinf(E.ctrl_h[0].target)) {
    lp_status st = set_targets(E, std::numeric_limits<double>::infinity(), true);
    if (st != LP_OK) return st;
  }
  return run_attempts(E, steps);
}
lp_status lp_batch_sync(lp_batch* b) {
  CUDA_CK(cudaStreamSynchronize(b->E.stream));
  return pull_ctrl(b->E);
}
lp_status lp_batch_get_counters(lp_batch* b, int32_t i, lp_counters* out) {
  if (i < 0 || i >= b->E.n) return set_error(LP_INVALID, "instance index out of range");
  lp_status st = pull_ctrl(b->E);
  if (st != LP_OK) return st;
  counters_out(b->E.ctrl_h[i], out);
  return LP_OK;
}
lp_status lp_batch_get_ledger(lp_batch* b, int32_t i, lp_ledger* out) {
  if (i < 0 || i >= b->E.n) return set_error(LP_INVALID, "instance index out of range");
  lp_status st = pull_ctrl(b->E);
  if (st != LP_OK) return st;
  ledger_out(b->E.ctrl_h[i].ledger, out);
  return LP_OK;
}
lp_status lp_batch_export_particles(lp_batch* b, int32_t i, lp_particles* out) {
  if (i < 0 || i >= b->E.n) return set_error(LP_INVALID, "instance index out of range");
  return export_particles(b->E, i, out);
}
lp_status lp_batch_get_pellet(lp_batch* b, int32_t i, lp_pellet* out, int32_t* has) {
  if (i < 0 || i >= b->E.n) return set_error(LP_INVALID, "instance index out of range");
  return get_pellet(b->E, i, out, has);
}
lp_status lp_batch_observables(lp_batch* b, int32_t i, char* names, double* values, int32_t capacity, int32_t* count) {
  if (i < 0 || i >= b->E.n) return set_error(LP_INVALID, "instance index out of range");
  std::map<std::string, double> obs;
  lp_status st = observables(b->E, i, obs);
  if (st != LP_OK) return st;
  int32_t n = 0;
  for (auto& kv : obs) {
    if (n >= capacity) break;
    std::snprintf(names + 64 * n, 64, "%s", kv.first.c_str());
    values[n] = kv.second;
    ++n;
  }
  *count = n;
  return LP_OK;
}
lp_status lp_batch_energies(lp_batch* b, int32_t i, double out[9]) {
  if (i < 0 || i >= b->E.n) return set_error(LP_INVALID, "instance index out of range");
  std::vector<Diag> d;
  lp_status st = diagnostics(b->E, d);
  if (st != LP_OK) return st;
  st = pull_ctrl(b->E);
  if (st != LP_OK) return st;
  const Energies en = energies_of(b->E, i, d[i]);
  const double v[9] = {en.ke, en.pe, en.ee, en.mech, en.mass_res, en.mom_res[0], en.mom_res[1], en.mom_res[2],
                       en.e_res};
  for (int k = 0; k < 9; ++k) out[k] = v[k];
  return LP_OK;
}
lp_status lp_batch_instance_state(lp_batch* b, int32_t i, int32_t* state, char* message, size_t message_len) {
  if (i < 0 || i >= b->E.n) return set_error(LP_INVALID, "instance index out of range");
  lp_status st = pull_ctrl(b->E);
  if (st != LP_OK) return st;
  const Control& c = b->E.ctrl_h[i];
  char buf[256] = "";
  switch (c.status) {
    case lp::S_RUNNING: *state = 0; break;
    case lp::S_REACHED: *state = 1; break;
    case lp::S_MIN_STEP:
      *state = 2;
      std::snprintf(buf, sizeof(buf),
                    "solver aborted at t='%.17g' s: step '%.17g' s below minimum after '%llu' rejections; last failure code %d",
                    c.time, c.dt, (unsigned long long)c.rejected_steps, c.last_fail);
      break;
    default:
      *state = 3;
      std::snprintf(buf, sizeof(buf), "closed fixture leaked particles beyond the padded grid (outflow)");
      break;
  }
  if (message && message_len) std::snprintf(message, message_len, "%s", buf);
  return LP_OK;
}
lp_status lp_batch_total_particles(lp_batch* b, uint64_t* out) {
  lp_status st = pull_ctrl(b->E);
  if (st != LP_OK) return st;
  uint64_t t = 0;
  for (auto& c : b->E.ctrl_h) t += (uint64_t)c.count;
  *out = t;
  return LP_OK;
}
lp_status lp_batch_set_warm_start(lp_batch* b, const float* w, int32_t nw, int32_t enable) {
  return set_warm(b->E, w, nw, enable);
}
lp_status lp_batch_warm_table(lp_batch* b, int32_t instance, float* out, int32_t capacity, double* dt) {
  return warm_table(b->E, instance, out, capacity, dt);
}
lp_status lp_batch_use_graph(lp_batch* b, int32_t steps) {
  b->E.invalidate_graph();
  b->E.graph_steps = steps > 0 ? steps : 0;
  return LP_OK;
}
lp_status lp_batch_prepare(lp_batch* b) { return ensure_graph(b->E); }
lp_status lp_sim_g2p_return_share(lp_sim* sim, int32_t steps, double* share) {
  Ensemble& E = sim->E;
  if (!share || steps < 1) return set_error(LP_INVALID, "need steps >= 1 and an output");
  if (E.ctrl_h.empty() || !std::isinf(E.ctrl_h[0].target)) {
    lp_status st = set_targets(E, std::numeric_limits<double>::infinity(), true);
    if (st != LP_OK) return st;
  }
  unsigned long long* d = nullptr;
  CUDA_CK(cudaMalloc(&d, 2 * sizeof(unsigned long long)));
  CUDA_CK(cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), E.stream));
  E.invalidate_graph();
  E.A.g2p_clk = d;
  lp_status st = LP_OK;
  for (int s = 0; s < steps && st == LP_OK; ++s) {
    lp::launch_attempt(E.A, E.stream);
    if (cudaGetLastError() != cudaSuccess) st = set_error(LP_DEVICE, "launch failed in the return-share measurement");
  }
  E.A.g2p_clk = nullptr;
  unsigned long long h[2] = {0, 0};
  const cudaError_t e1 = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, E.stream);
  const cudaError_t e2 = cudaStreamSynchronize(E.stream);
  cudaFree(d);
  if (st != LP_OK) return st;
  if (e1 != cudaSuccess || e2 != cudaSuccess) return set_error(LP_DEVICE, "return-share measurement failed");
  *share = h[0] > 0 ? (double)h[1] / (double)h[0] : 0.0;
  return pull_ctrl(E);
}

lp_status lp_batch_autotune(lp_batch* b, int32_t trial_steps, char* report, size_t report_len) {
  return autotune(b->E, trial_steps, report, report_len);
}
lp_status lp_sim_autotune(lp_sim* sim, int32_t trial_steps, char* report, size_t report_len) {
  return autotune(sim->E, trial_steps, report, report_len);
}
lp_status lp_batch_set_launch_shape(lp_batch* b, const lp_launch_shape* shape) {
  return set_launch_shape(b->E, shape);
}
lp_status lp_batch_get_launch_shape(lp_batch* b, lp_launch_shape* out) { return get_launch_shape(b->E, out); }
lp_status lp_sim_set_launch_shape(lp_sim* sim, const lp_launch_shape* shape) {
  return set_launch_shape(sim->E, shape);
}
lp_status lp_sim_get_launch_shape(lp_sim* sim, lp_launch_shape* out) { return get_launch_shape(sim->E, out); }

// ---------------- constitutive unit kernels on host arrays
lp_status lp_hb_return_batch(int64_t n, const double* trial, const double* yield, const double* consistency,
                             const double* flow_index, const double* mu, const double* dt, double tol_rel,
                             const float* mlp_weights, int32_t nweights, double* out, int32_t* status) {
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) return set_error(LP_DEVICE, "no CUDA device");
  if (n <= 0) return LP_OK;
  if (mlp_weights && nweights != lp::MLP_NW) return set_error(LP_INVALID, "MLP weight count mismatch");
  double* d = nullptr;
  float* w = nullptr;
  lp::MlpPacked* pk = nullptr;
  int* s = nullptr;
  const size_t nb = sizeof(double) * (size_t)n;
  CUDA_CK(cudaMalloc(&d, nb * 9));
  CUDA_CK(cudaMalloc(&s, sizeof(int) * n));
  if (mlp_weights) {
    CUDA_CK(cudaMalloc(&w, sizeof(float) * lp::MLP_NW));
    CUDA_CK(cudaMalloc(&pk, sizeof(lp::MlpPacked)));
    CUDA_CK(cudaMemcpy(w, mlp_weights, sizeof(float) * lp::MLP_NW, cudaMemcpyHostToDevice));
    lp::launch_mlp_pack(w, pk, 0);
  }
  const double* src[6] = {trial, yield, consistency, flow_index, mu, dt};
  for (int k = 0; k < 6; ++k) CUDA_CK(cudaMemcpy(d + k * n, src[k], nb, cudaMemcpyHostToDevice));
  lp::launch_hb_return_batch(n, d, d + n, d + 2 * n, d + 3 * n, d + 4 * n, d + 5 * n, tol_rel > 0 ? tol_rel : 1e-12, pk,
                             d + 6 * n, s, 0);
  CUDA_CK(cudaGetLastError());
  CUDA_CK(cudaMemcpy(out, d + 6 * n, nb * 3, cudaMemcpyDeviceToHost));
  CUDA_CK(cudaMemcpy(status, s, sizeof(int) * n, cudaMemcpyDeviceToHost));
  cudaFree(d);
  cudaFree(s);
  if (w) cudaFree(w);
  if (pk) cudaFree(pk);
  return LP_OK;
}

lp_status lp_update_paste_batch(int64_t n, const double* f_trial, const lp_material* m, double dt, double* f_new,
                                double* tau, double* dep, double* diss, double* eq, int32_t* status) {
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) return set_error(LP_DEVICE, "no CUDA device");
  if (n <= 0) return LP_OK;
  double *df = nullptr, *dfn = nullptr, *dt9 = nullptr, *ds = nullptr;
  int* st = nullptr;
  CUDA_CK(cudaMalloc(&df, sizeof(double) * 9 * n));
  CUDA_CK(cudaMalloc(&dfn, sizeof(double) * 9 * n));
  CUDA_CK(cudaMalloc(&dt9, sizeof(double) * 9 * n));
  CUDA_CK(cudaMalloc(&ds, sizeof(double) * 3 * n));
  CUDA_CK(cudaMalloc(&st, sizeof(int) * n));
  CUDA_CK(cudaMemcpy(df, f_trial, sizeof(double) * 9 * n, cudaMemcpyHostToDevice));
  lp::launch_update_paste_batch(n, df, m->shear_modulus, m->lame_lambda, m->yield_stress, m->consistency, m->flow_index,
                                dt, 1e-12, dfn, dt9, ds, st, 0);
  CUDA_CK(cudaGetLastError());
  std::vector<double> sc(3 * n);
  CUDA_CK(cudaMemcpy(f_new, dfn, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost));
  CUDA_CK(cudaMemcpy(tau, dt9, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost));
  CUDA_CK(cudaMemcpy(sc.data(), ds, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
  CUDA_CK(cudaMemcpy(status, st, sizeof(int) * n, cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < n; ++i) {
    if (dep) dep[i] = sc[3 * i];
    if (diss) diss[i] = sc[3 * i + 1];
    if (eq) eq[i] = sc[3 * i + 2];
  }
  cudaFree(df);
  cudaFree(dfn);
  cudaFree(dt9);
  cudaFree(ds);
  cudaFree(st);
  return LP_OK;
}

lp_status lp_update_liquid_batch(int64_t n, const double* volume_ratio, const double* grad, const lp_material* m,
                                 double dt, double* j_new, double* tau, double* pressure, int32_t* status) {
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) return set_error(LP_DEVICE, "no CUDA device");
  if (n <= 0) return LP_OK;
  double *dj, *dg, *djn, *dtau, *dp;
  int* st;
  CUDA_CK(cudaMalloc(&dj, sizeof(double) * n));
  CUDA_CK(cudaMalloc(&dg, sizeof(double) * 9 * n));
  CUDA_CK(cudaMalloc(&djn, sizeof(double) * n));
  CUDA_CK(cudaMalloc(&dtau, sizeof(double) * 9 * n));
  CUDA_CK(cudaMalloc(&dp, sizeof(double) * n));
  CUDA_CK(cudaMalloc(&st, sizeof(int) * n));
  CUDA_CK(cudaMemcpy(dj, volume_ratio, sizeof(double) * n, cudaMemcpyHostToDevice));
  CUDA_CK(cudaMemcpy(dg, grad, sizeof(double) * 9 * n, cudaMemcpyHostToDevice));
  lp::launch_update_liquid_batch(n, dj, dg, m->bulk_modulus, m->consistency, m->tait_gamma == 0.0 ? 1.0 : m->tait_gamma,
                                 dt, djn, dtau, dp, st, 0);
  CUDA_CK(cudaGetLastError());
  CUDA_CK(cudaMemcpy(j_new, djn, sizeof(double) * n, cudaMemcpyDeviceToHost));
  CUDA_CK(cudaMemcpy(tau, dtau, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost));
  CUDA_CK(cudaMemcpy(pressure, dp, sizeof(double) * n, cudaMemcpyDeviceToHost));
  CUDA_CK(cudaMemcpy(status, st, sizeof(int) * n, cudaMemcpyDeviceToHost));
  cudaFree(dj);
  cudaFree(dg);
  cudaFree(djn);
  cudaFree(dtau);
  cudaFree(dp);
  cudaFree(st);
  return LP_OK;
}

void lp_hb_features(double trial, double yield, double consistency, double flow_index, double mu, double dt,
                    float out[6]) {
  lp::hb_features(trial, yield, consistency, flow_index, mu, dt, out);
}

}  // extern "C"
