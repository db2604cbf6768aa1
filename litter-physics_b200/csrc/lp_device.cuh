// lp_device.cuh - device data layout and per-particle constitutive math of the B200 MLS-MPM step.
//
// Layout (one "ensemble" = one or more independent simulations, "instances"):
//   * particle state: FP32 structure of arrays, component-major (component c of slot s at
//     state[c * cap + s]); two buffers (current / trial) selected per instance by a parity bit
//     so a rejected trial never touches the committed state (solver.rs:11-14);
//   * grid: dense padded node arrays per instance (grid.rs:71, n+3 nodes per axis):
//     int64 fixed-point mass / momentum accumulators, int64 wall-reaction accumulators split by
//     face side, and a float4 (velocity, mass) array written by the grid update;
//   * bins: particles are counting-sorted every attempt by their stencil base cell
//     (floor(x/dx - 0.5) + 1 per axis), bins grouped in tiles of TX x TY x TZ so that one
//     CTA of the scatter owns one tile and its (TX+2)(TY+2)(TZ+2)-node halo.
//
// Precision: particle and grid arithmetic in FP32.  The deformation gradient is stored as
// H = F - I and the liquid volume ratio as J - 1, so that near-identity strains keep full FP32
// relative precision.  The Herschel-Bulkley scalar return runs in FP64, and so do the ledger
// reductions.  Grid mass/momentum accumulate as exact int64 fixed-point sums (order
// independent, hence deterministic).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lp_mlp.cuh"

namespace lp {

// ---------------------------------------------------------------- tiling constants
constexpr int TX = 4, TY = 4, TZ = 8;            // bins per tile
constexpr int TB = TX * TY * TZ;                 // 128 bins per tile
constexpr int HX = TX + 2, HY = TY + 2, HZ = TZ + 2;
constexpr int HN = HX * HY * HZ;                 // 360 halo nodes per tile
constexpr int P2G_THREADS = 3 * TB;              // 3 slab threads per bin
constexpr int NB = 4;                            // node block edge (grid update / activity)
constexpr int GU_BLOCKS_PER_CTA = 4;             // node blocks per grid-update CTA pass
constexpr int GU_PASSES = 8;                     // passes per grid-update CTA
constexpr int GU_THREADS = NB * NB * NB * GU_BLOCKS_PER_CTA;  // 256
constexpr int G2P_THREADS = 256;
constexpr int SLOT_ALIGN = G2P_THREADS;          // instance slot ranges are aligned to this
constexpr int KEY_CHUNK = 1024;                  // scan chunk; instance key ranges aligned to it

// state components (component-major)
enum Comp : int {
  C_X = 0,    // 3
  C_V = 3,    // 3
  C_C = 6,    // 9 (row-major)
  C_H = 15,   // 9 (F - I, row-major)
  C_TAU = 24, // 6: xx yy zz xy xz yz
  C_EP = 30,
  C_M = 31,
  C_V0 = 32,
  C_YS = 33,
  C_JM1 = 34,
  NCOMP = 35
};

// failure codes (worst wins)
enum Fail : int {
  F_OK = 0,
  F_CONST_INVERTED = 1,
  F_CONST_EIGEN = 2,
  F_CONST_STRETCH = 3,
  F_CONST_NOT_CONVERGED = 4,
  F_CONST_NONFINITE = 5,
  F_GRID_NONFINITE = 6,
  F_DISPLACEMENT = 7,
  F_PELLET_NONFINITE = 8,
  F_TRACTION_NONFINITE = 9,
  F_OUTFLOW = 10
};

enum Status : int { S_RUNNING = 0, S_REACHED = 1, S_MIN_STEP = 2, S_ERROR = 3 };

// per-instance constants (set at creation)
struct InstDesc {
  double dx, inv_dx;
  float pow2_inv_dx;  // 1 / (float)dx when (float)dx is a power of two (then x * it == x / dx), else 0
  int cells[3], nodes[3];
  int bins[3], tiles[3];
  int nblk[3];
  int kind;  // 0 paste, 1 liquid
  int per_particle_yield;
  int face_mode;
  int has_pellet;
  int64_t node_off;   // first node of this instance in the global node arrays
  int64_t tile_off;   // first global tile
  int64_t key_off;    // first global bin key (= tile_off * TB)
  int64_t nkeys;      // keys incl. the trailing outflow key, aligned to KEY_CHUNK
  int64_t blk_off;    // first global node block
  int64_t gcta_off, gcta_cnt;  // grid-update CTAs
  int64_t slot_off, slot_cap;  // particle slots
  int64_t pcta_off, pcta_cnt;  // G2P CTAs
  int64_t seg_off, seg_cnt, seg_cnt_g;  // reduction segments (grid segments first)
  // material (constitutive.rs:111-131), FP64 master copy
  double density, mu, lambda, bulk, yield, consistency, flow_index, tait_gamma;
  // config (solver.rs:48-62)
  double gravity[3];
  double friction;
  double face_mu[6];
  int face_sticky[6];
  double cfl, max_dt, min_dt, tol;
  double contact_k, contact_e, contact_mu;
  double extent[3];
  double s_mass;  // fixed-point scale of node mass
  // pellet bed (extension): bed_np >= 2 pellets of one geometry, Hertz-Mindlin sphere contact
  int bed_np;
  int bed_nc[3];             // coarse cells per axis (cell edge bed_h = two bounding radii)
  int64_t bed_off;           // first pellet of this instance in the global bed arrays
  double bed_h, bed_rb;      // coarse cell edge, pellet bounding radius
  double hm_estar, hm_gstar, hm_mu, hm_beta;  // effective moduli, friction, damping parameter
  // contact law: 0 Hertz-Mindlin, 1 linear spring-dashpot (stiffness, damping ratio, rolling
  // friction; friction is hm_mu)
  int bed_law;
  double dem_kn, dem_zeta, dem_mur;
};

// pellet state (rigid.rs:30-49), FP64
struct PelletState {
  double radius, length, mass;
  double inertia[3];
  double pos[3];
  double q[4];  // i j k w
  double vel[3];
  double L[3];
  int nsph;
  int pad;
  double off[64];
};

// FP64 ledger, same order as lp_ledger
struct LedgerD {
  double initial_mass, outflow_mass, initial_momentum[3], initial_mech, gravity_impulse[3], wall_impulse[3],
      pellet_wall_impulse[3], coupling_impulse[3], coupling_angular[3], proj, fric, trac, pellet_work, cgrid,
      cpellet, plastic, outflow_momentum[3];
};

// Constants of the HB return (hb_return_d) that depend on the material (consistency K, flow
// index n, shear modulus mu) and dt only: hb_const computes them once per instance and attempt
// (k_begin) instead of per particle, with the expressions of the per-particle form, so the
// results are the same.
struct HbConst {
  double k, mu3, viscous_scale, exponent, log_k, c1;  // K, 3 mu, 3 mu dt, 1/n, log K, 3 mu dt / n
  int finite;                                         // K, n, mu and dt are finite
  int pad;
};

// per-instance mutable control block (device resident)
struct Control {
  double time, target;
  double dt, dt_scale, limit;
  double forced_dt;      // > 0: lp_sim_try_step mode (exact dt, no control)
  double max_speed;      // of the committed state
  double bbound;         // momentum bound of the committed state (for the fixed-point scale)
  double s_mom;          // fixed-point scale of node momentum for the current attempt
  double total_mass;     // FP64 sum of particle masses
  double min_dt_used, max_dt_used;
  uint64_t step_count, limited_steps, rejected_steps;
  uint64_t newton_iterations, yielded;
  int active, status, limited, parity;
  int fail, last_fail, epoch, pad;
  int64_t count;         // particle count
  int64_t outflow;       // particles detected outside the padded grid this attempt
  double fail_value;
  LedgerD ledger;
  PelletState pellet, pellet_trial;
  // pellet-step results of the current attempt
  double c_impulse[3], c_angular[3], c_grid_energy, c_pellet_energy, pw_impulse[3], pw_work;
  int pellet_fail, warm_start;
  // pellet bed: committed buffer parity, cumulative sphere-contact work, last accepted step's
  // contact count and history overflows
  int bed_parity, bed_contacts;
  double bed_contact_work;
  uint64_t bed_overflow;
  double bed_limit;  // step limit of the committed pellets (set on commit and by the host)
  double step_diss;  // plastic work of the last attempt, accepted or not (energy audit)
  HbConst hb;        // HB return constants of the current attempt's dt (set by k_begin)
};

// pellet bed: tangential spring of one sphere pair (pellet-local sphere a, other pellet's b)
constexpr int HM_SLOTS = 24;
constexpr int BED_MAX = 4096;  // pellets per instance
struct HmContact {
  int other, a, b, pad;
  double xi[3];
};
// pellet bed: double-buffered device arrays (index = buffer parity), passed to kernels by value
struct BedPtrs {
  PelletState* state[2];  // [pellet]
  HmContact* hist[2];     // [pellet * HM_SLOTS]
  int* hist_n[2];         // [pellet]
};
// pellet bed: per-pellet results of one attempt
struct BedStep {
  double imp[3], ang[3], cgrid, cpellet, wimp[3], wwork, ppwork, limit;
  int contacts, overflow, fail, pad;
};

// partial results of one grid-update CTA
struct GridPartial {
  double wall_impulse[3];
  double proj, fric, trac;
  int fail;
  int pad;
};
// a reduction segment: [begin, end) of grid (kind 0) or particle (kind 1) partials of one instance
struct SegDesc {
  int64_t begin, end;
  int inst, kind;
};
struct SegPartial {
  double v[13];
};
constexpr int SEG_SPAN = 2048;
// partial results of one G2P CTA
struct ParticlePartial {
  double diss, bbound, mass;
  float max_speed, max_disp;
  int fail;
  int iterations;
  int yielded;
  int pad;
  double fail_value;
};

// Pellet-bed step limit: per pellet the reference's wall-contact and pellet-CFL limits
// (solver.rs:477-498), plus for Hertz-Mindlin 0.2 sqrt(m*/k_c) at the stiffness of an overlap
// of 5 % of the sphere radius, k_c = 2 E* sqrt(R* 0.05 r), and for the linear law the household
// DEM's 0.1 sqrt(m/k_n) (World::stable_dt, dem.rs:509-520).
__host__ __device__ inline double pellet_bed_limit(const InstDesc& D, const PelletState& P) {
  double limit = 0.2 * sqrt(P.mass / D.contact_k);
  const double ps = sqrt(P.vel[0] * P.vel[0] + P.vel[1] * P.vel[1] + P.vel[2] * P.vel[2]);
  if (ps > 0.0) limit = fmin(limit, D.cfl * D.dx / ps);
  if (D.bed_law == 1) return fmin(limit, 0.1 * sqrt(P.mass / D.dem_kn));
  const double kc = 2.0 * D.hm_estar * sqrt(0.5 * P.radius * 0.05 * P.radius);
  return fmin(limit, 0.2 * sqrt(0.5 * P.mass / kc));
}

// Damping ratio of a linear dashpot for restitution e (ContactParams::damping_ratio,
// dem.rs:112-120): e clamped to [0, 1], critical damping at e = 0.
__host__ __device__ inline double dem_damping_ratio(double e) {
  e = fmin(fmax(e, 0.0), 1.0);
  if (e <= 2.220446049250313e-16) return 1.0;
  const double l = log(e);
  return fmin(-l / sqrt(3.14159265358979323846 * 3.14159265358979323846 + l * l), 1.0);
}
__host__ __device__ inline double bed_limit(const InstDesc& D, const PelletState* S) {
  double limit = 1e300;
  for (int p = 0; p < D.bed_np; ++p) limit = fmin(limit, pellet_bed_limit(D, S[p]));
  return limit;
}

// ---------------------------------------------------------------- small helpers
__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }

// fixed-point conversion of an FP64 value (round to nearest)
__device__ __forceinline__ long long to_fixed(double v, double scale) { return __double2ll_rn(v * scale); }

__device__ __forceinline__ void atomic_add_ll(long long* p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

// ---------------------------------------------------------------- HB scalar return (FP64)
__device__ inline HbConst hb_const(double k, double n, double mu, double dt) {
  HbConst h;
  h.finite = (isfinite(k) && isfinite(n) && isfinite(mu) && isfinite(dt)) ? 1 : 0;
  h.k = k;
  h.mu3 = 3.0 * mu;
  h.viscous_scale = 3.0 * mu * dt;
  h.exponent = 1.0 / n;
  h.log_k = log(k);
  h.c1 = h.viscous_scale * h.exponent;
  h.pad = 0;
  return h;
}

// (1 - q)^a for |q| <= 2^-7 and |a q| <= 2^-7, as exp(a log1p(-q)) from the Taylor series of
// log1p and exp, each cut after the eighth power: log1p(-q) = -q (1 + q/2 + ... + q^7/8) and
// exp(t) = 1 + t + ... + t^8/8!.  At these arguments the omitted terms are below 1e-19, so the
// result is the FP64 power to rounding.
__device__ __forceinline__ double pow_one_minus_small(double q, double a) {
  double s = 1.0 / 8.0;
  s = fma(s, q, 1.0 / 7.0);
  s = fma(s, q, 1.0 / 6.0);
  s = fma(s, q, 1.0 / 5.0);
  s = fma(s, q, 1.0 / 4.0);
  s = fma(s, q, 1.0 / 3.0);
  s = fma(s, q, 1.0 / 2.0);
  s = fma(s, q, 1.0);
  const double t = -a * q * s;
  double e = 1.0 / 40320.0;
  e = fma(e, t, 1.0 / 5040.0);
  e = fma(e, t, 1.0 / 720.0);
  e = fma(e, t, 1.0 / 120.0);
  e = fma(e, t, 1.0 / 24.0);
  e = fma(e, t, 1.0 / 6.0);
  e = fma(e, t, 1.0 / 2.0);
  e = fma(e, t, 1.0);
  return fma(e, t, 1.0);
}

// Bracketed Newton of constitutive.rs:280-362, with an optional start value sigma0 in
// (yield, trial) (the learned warm start); the plain solver starts at the midpoint.
// Returns failure code; iterations through *iters.
//
// The iteration runs on the excess stress x = sigma - yield over the bracket [0, trial - yield]:
// the residual f = sigma - trial + 3 mu dt (x/K)^(1/n) = x - (trial - yield) + 3 mu dt p with
// p = (x/K)^(1/n), and the Newton step x - f / f', f' = 1 + (3 mu dt / n) p / x, is
// x (1 - q) with q = f / (x + (3 mu dt / n) p): one division per iterate.  The same bracket
// updates, bisection safeguard and stopping rule as the reference's solver.  After a Newton
// step the new power is the old one times (1 - q)^(1/n); once |q| is small (quadratic
// convergence makes it so within a few iterates, and a good warm start from the first) that
// factor comes from two short series instead of a logarithm and an exponential.
__device__ inline int hb_return_d(double trial, double ys, const HbConst& h, double tol_rel, double sigma0,
                                  double* sigma_out, double* dep_out, int* iters) {
  *iters = 0;
  if (!(isfinite(trial) && isfinite(ys) && h.finite)) return F_CONST_NONFINITE;
  const double viscous_scale = h.viscous_scale;
  if (trial <= ys) {
    *sigma_out = trial;
    *dep_out = 0.0;
    return F_OK;
  }
  if (h.k <= 0.0) {
    *sigma_out = ys;
    *dep_out = (trial - ys) / h.mu3;
    return F_OK;
  }
  const double exponent = h.exponent, log_k = h.log_k, c1 = h.c1;
  const double span = trial - ys;  // the bracket [0, span] of the excess stress
  const double small_q = 0.0078125 / fmax(exponent, 1.0);  // |q| and |q / n| at most 2^-7
  double lo = 0.0, hi = span;
  double x = (sigma0 > ys && sigma0 < trial) ? sigma0 - ys : 0.5 * span;
  const double tolerance = tol_rel * fmax(trial, 1.0);
  double pw = 0.0;
  bool full = true;  // the power at x needs the logarithm and the exponential
  // Pass `it` evaluates the residual of the iterate that pass it - 1 chose (pass 1: the start),
  // so the FP64 logarithm and exponential have one call site and the kernels' code stays small.
  for (int it = 1; it <= 201; ++it) {
    if (full) pw = x > 0.0 ? exp(exponent * (log(x) - log_k)) : 0.0;
    const double last = x - span + viscous_scale * pw;
    if (it > 1 && !isfinite(last)) {
      *iters = it - 1;
      return F_CONST_NONFINITE;
    }
    if (it == 201) break;
    if (fabs(last) <= tolerance || (hi - lo) <= tolerance) {
      const double sigma = ys + x;
      *sigma_out = sigma;
      *dep_out = (trial - sigma) / h.mu3;
      *iters = it;
      return F_OK;
    }
    if (last > 0.0) hi = x;
    else lo = x;
    // at x = 0 the derivative is infinite and the reference's Newton step is a no-op: bisect
    const double q = x > 0.0 ? last / (x + c1 * pw) : 0.0;
    const double xn = fma(-q, x, x);
    if (x > 0.0 && isfinite(xn) && xn > lo && xn < hi) {
      full = fabs(q) > small_q;
      if (!full) pw *= pow_one_minus_small(q, exponent);
      x = xn;
    } else {
      x = 0.5 * (lo + hi);
      full = true;
    }
  }
  *iters = 200;
  return F_CONST_NOT_CONVERGED;
}
// the same with the constants computed here (one return problem per material)
__device__ inline int hb_return_d(double trial, double ys, double k, double n, double mu, double dt, double tol_rel,
                                  double sigma0, double* sigma_out, double* dep_out, int* iters) {
  return hb_return_d(trial, ys, hb_const(k, n, mu, dt), tol_rel, sigma0, sigma_out, dep_out, iters);
}

// ---------------------------------------------------------------- symmetric 3x3 eigen (Jacobi)
// Cyclic Jacobi as constitutive.rs:373-425; FP32 version with an FP32-appropriate stopping
// rule, FP64 version with the reference's rule (used when FP32 stalls).
template <typename T>
__device__ inline bool jacobi3(T d[3][3], T v[3][3], int max_sweeps, T tol) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) v[i][j] = (i == j) ? T(1) : T(0);
  T scale = T(0);
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) scale += d[i][j] * d[i][j];
  const int P[3] = {0, 0, 1}, Q[3] = {1, 2, 2};
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    T off = d[0][1] * d[0][1] + d[0][2] * d[0][2] + d[1][2] * d[1][2];
    if (off <= tol * scale) return true;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int p = P[r], q = Q[r];
      T apq = d[p][q];
      if (apq == T(0)) continue;
      T theta = (d[q][q] - d[p][p]) / (T(2) * apq);
      T at = theta < T(0) ? -theta : theta;
      T sgn = signbit(theta) ? T(-1) : T(1);
      T tangent = at > T(1e18) ? sgn / (T(2) * at) : sgn / (at + sqrt(theta * theta + T(1)));
      T c = T(1) / sqrt(tangent * tangent + T(1));
      T s = tangent * c;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        T akp = d[k][p], akq = d[k][q];
        d[k][p] = c * akp - s * akq;
        d[k][q] = s * akp + c * akq;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        T apk = d[p][k], aqk = d[q][k];
        d[p][k] = c * apk - s * aqk;
        d[q][k] = s * apk + c * aqk;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        T vkp = v[k][p], vkq = v[k][q];
        v[k][p] = c * vkp - s * vkq;
        v[k][q] = s * vkp + c * vkq;
      }
    }
  }
  return false;
}

// ---------------------------------------------------------------- paste update (H = F - I)
// update_paste of constitutive.rs:456-531 rewritten on the displacement gradient:
//   H_tr = H + dt C + dt C H            (F_tr = (I + dt C) F)
//   B    = H_tr + H_tr^T + H_tr H_tr^T  (b - I, b = F_tr F_tr^T)
//   eps_i = log1p(beta_i) / 2           (Hencky strain from the eigenvalues beta of B)
//   F_new = U diag(exp(eps_new - eps)) U^T F_tr  ->  H_new = H_tr + U diag(expm1(delta)) U^T (I + H_tr)
// Identical mathematics, FP32 rounding kept relative to the strain rather than to 1.
struct PasteOut {
  float H[9];
  float tau[6];
  double dep, diss_density, eq, trial;
  int iters;
  int fail;
  int yielded;
};

// Eigen-decomposition path (any strain size).  sigma0: Newton start in (yield, trial), or -1 for
// the reference's midpoint start.  trial_only: stop after the trial equivalent stress (o.trial).
static __device__ __noinline__ void paste_update_jacobi(const float Htr[9], float mu, float lambda, double mu_d, double ys,
                                                        const HbConst& h, double tol, double sigma0, bool trial_only,
                                                        PasteOut& o) {
  o.fail = F_OK;
  o.iters = 0;
  o.yielded = 0;
  o.dep = 0.0;
  o.diss_density = 0.0;
  // det(I + H_tr) > 0
  const float f00 = 1.f + Htr[0], f01 = Htr[1], f02 = Htr[2];
  const float f10 = Htr[3], f11 = 1.f + Htr[4], f12 = Htr[5];
  const float f20 = Htr[6], f21 = Htr[7], f22 = 1.f + Htr[8];
  const float det = f00 * (f11 * f22 - f21 * f12) - f01 * (f10 * f22 - f20 * f12) + f02 * (f10 * f21 - f20 * f11);
  if (!isfinite(det)) {
    o.fail = F_CONST_NONFINITE;
    return;
  }
  if (det <= 0.f) {
    o.fail = F_CONST_INVERTED;
    return;
  }
  // B = H + H^T + H H^T
  float B[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      float hh = Htr[3 * i + 0] * Htr[3 * j + 0] + Htr[3 * i + 1] * Htr[3 * j + 1] + Htr[3 * i + 2] * Htr[3 * j + 2];
      B[i][j] = Htr[3 * i + j] + Htr[3 * j + i] + hh;
    }
  float U[3][3];
  float beta[3];
  {
    float d[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) d[i][j] = 0.5f * (B[i][j] + B[j][i]);
    bool ok = jacobi3<float>(d, U, 12, 1e-13f);
    if (ok) {
      beta[0] = d[0][0];
      beta[1] = d[1][1];
      beta[2] = d[2][2];
    } else {
      double dd[3][3], uu[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) dd[i][j] = 0.5 * ((double)B[i][j] + (double)B[j][i]);
      if (!jacobi3<double>(dd, uu, 64, 1e-30)) {
        o.fail = F_CONST_EIGEN;
        return;
      }
      for (int i = 0; i < 3; ++i) {
        beta[i] = (float)dd[i][i];
        for (int j = 0; j < 3; ++j) U[i][j] = (float)uu[i][j];
      }
    }
  }
  float eps[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float lam = 1.f + beta[a];  // squared stretch
    if (!isfinite(beta[a]) || !(lam >= 1e-12f)) {
      o.fail = F_CONST_STRETCH;
      return;
    }
    eps[a] = 0.5f * log1pf(beta[a]);
  }
  const float vol = eps[0] + eps[1] + eps[2];
  const float mean = vol / 3.f;
  float dev[3] = {eps[0] - mean, eps[1] - mean, eps[2] - mean};
  const float dnorm = sqrtf(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
  const double trial_eq = 1.2247448713915890 * 2.0 * mu_d * (double)dnorm;  // sqrt(3/2) 2 mu |dev|
  double scale = 1.0;
  o.eq = trial_eq;
  o.trial = trial_eq;
  if (trial_only) return;
  if (trial_eq > ys && dnorm > 0.f) {
    double sigma, dep;
    int iters;
    int e = hb_return_d(trial_eq, ys, h, tol, sigma0, &sigma, &dep, &iters);
    o.iters = iters;
    if (e != F_OK) {
      o.fail = e;
      return;
    }
    scale = sigma / trial_eq;
    o.dep = dep;
    o.eq = sigma;
    o.yielded = 1;
  }
  const float sc = (float)scale;
  float eps_new[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) eps_new[a] = dev[a] * sc + mean;
  // Kirchhoff stress tau = U diag(2 mu eps_new + lambda vol) U^T
  float ps[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) ps[a] = eps_new[a] * (2.f * mu) + lambda * vol;
  float T[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) T[i][j] = U[i][0] * ps[0] * U[j][0] + U[i][1] * ps[1] * U[j][1] + U[i][2] * ps[2] * U[j][2];
  o.tau[0] = T[0][0];
  o.tau[1] = T[1][1];
  o.tau[2] = T[2][2];
  o.tau[3] = 0.5f * (T[0][1] + T[1][0]);
  o.tau[4] = 0.5f * (T[0][2] + T[2][0]);
  o.tau[5] = 0.5f * (T[1][2] + T[2][1]);
  for (int i = 0; i < 6; ++i)
    if (!isfinite(o.tau[i])) {
      o.fail = F_CONST_NONFINITE;
      return;
    }
  if (o.yielded) {
    // H_new = H_tr + U diag(expm1(delta)) U^T (I + H_tr), delta = dev (scale - 1)
    float r[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) r[a] = expm1f(dev[a] * (sc - 1.f));
    float M[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) M[i][j] = U[i][0] * r[0] * U[j][0] + U[i][1] * r[1] * U[j][1] + U[i][2] * r[2] * U[j][2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        float s = M[i][j] + (M[i][0] * Htr[0 * 3 + j] + M[i][1] * Htr[1 * 3 + j] + M[i][2] * Htr[2 * 3 + j]);
        o.H[3 * i + j] = Htr[3 * i + j] + s;
      }
  } else {
#pragma unroll
    for (int i = 0; i < 9; ++i) o.H[i] = Htr[i];
  }
  o.diss_density = o.eq * o.dep;
}

// ---------------------------------------------------------------- paste update, series path
// For ||B||_F <= 0.25 the isotropic tensor functions of update_paste need no eigenvectors:
//   E = log(I + B) / 2                    (Hencky strain tensor, Horner series in B)
//   tau = 2 mu (mean I + s dev E) + lambda tr(E) I,  s = sigma / sigma_tr
//   F_new = exp((s - 1) dev E) F_tr  ->  H_new = H_tr + G (I + H_tr),  G = exp((s-1) dev E) - I
// These are the same functions of the same matrix as U diag(.) U^T in constitutive.rs:456-531;
// all the polynomials in B commute, so their products stay symmetric (6 stored entries).
struct Sym {
  float xx, yy, zz, xy, xz, yz;
};
// product of two commuting symmetric matrices
__device__ __forceinline__ Sym sym_mul(const Sym& p, const Sym& q) {
  Sym r;
  r.xx = p.xx * q.xx + p.xy * q.xy + p.xz * q.xz;
  r.yy = p.xy * q.xy + p.yy * q.yy + p.yz * q.yz;
  r.zz = p.xz * q.xz + p.yz * q.yz + p.zz * q.zz;
  r.xy = p.xx * q.xy + p.xy * q.yy + p.xz * q.yz;
  r.xz = p.xx * q.xz + p.xy * q.yz + p.xz * q.zz;
  r.yz = p.xy * q.xz + p.yy * q.yz + p.yz * q.zz;
  return r;
}
__device__ __forceinline__ float sym_norm(const Sym& a) {
  return sqrtf(a.xx * a.xx + a.yy * a.yy + a.zz * a.zz + 2.f * (a.xy * a.xy + a.xz * a.xz + a.yz * a.yz));
}

// Series coefficients, correctly rounded like the FP32 divisions they replace:
// kLogSeries[j] = (-1)^(j+1) / j (log(I + B)), kInverse[j] = 1 / j (exp(M) by Horner).
__constant__ const float kLogSeries[13] = {0.0f,         1.0f,         -1.0f / 2.0f,  1.0f / 3.0f,  -1.0f / 4.0f,
                                           1.0f / 5.0f,  -1.0f / 6.0f, 1.0f / 7.0f,   -1.0f / 8.0f, 1.0f / 9.0f,
                                           -1.0f / 10.0f, 1.0f / 11.0f, -1.0f / 12.0f};
__constant__ const float kInverse[10] = {0.0f,        1.0f,        1.0f / 2.0f, 1.0f / 3.0f, 1.0f / 4.0f,
                                         1.0f / 5.0f, 1.0f / 6.0f, 1.0f / 7.0f, 1.0f / 8.0f, 1.0f / 9.0f};

// Trial part of the paste update: the Hencky strain of H_tr and its equivalent stress.  The
// Newton start (the learned warm start) is chosen from t.trial_eq between paste_trial and
// paste_finish, which lets a warp evaluate the network for all its lanes at one call site.
// PT_DEFER (DEFER instantiations only): the strain is outside the series path and the caller
// leaves the particle to a separate eigen-decomposition pass, so that its own code carries no
// call of paste_update_jacobi.
enum { PT_SERIES = 0, PT_JACOBI = 1, PT_DONE = 2, PT_DEFER = 3 };
struct PasteTrial {
  Sym dev;
  float mean, vol, dnorm;
  double trial_eq;
  int path;
};

template <bool DEFER = false>
__device__ inline void paste_trial(const float Htr[9], double mu_d, PasteTrial& t, PasteOut& o) {
  o.fail = F_OK;
  o.iters = 0;
  o.yielded = 0;
  o.dep = 0.0;
  o.diss_density = 0.0;
  Sym B;
  B.xx = 2.f * Htr[0] + (Htr[0] * Htr[0] + Htr[1] * Htr[1] + Htr[2] * Htr[2]);
  B.yy = 2.f * Htr[4] + (Htr[3] * Htr[3] + Htr[4] * Htr[4] + Htr[5] * Htr[5]);
  B.zz = 2.f * Htr[8] + (Htr[6] * Htr[6] + Htr[7] * Htr[7] + Htr[8] * Htr[8]);
  B.xy = Htr[1] + Htr[3] + (Htr[0] * Htr[3] + Htr[1] * Htr[4] + Htr[2] * Htr[5]);
  B.xz = Htr[2] + Htr[6] + (Htr[0] * Htr[6] + Htr[1] * Htr[7] + Htr[2] * Htr[8]);
  B.yz = Htr[5] + Htr[7] + (Htr[3] * Htr[6] + Htr[4] * Htr[7] + Htr[5] * Htr[8]);
  const float r = sym_norm(B);
  if (!(r <= 0.25f)) {  // large or non-finite strain: eigen-decomposition path
    if constexpr (DEFER) {
      t.path = PT_DEFER;
      t.trial_eq = 0.0;
    } else {
      // the out-of-line call works on copies, so that the caller's arrays need no stack home
      float Hj[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) Hj[i] = Htr[i];
      PasteOut oj = o;
      const HbConst none = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0, 0};  // the trial stops before the return
      paste_update_jacobi(Hj, 0.f, 0.f, mu_d, 0.0, none, 0.0, -1.0, true, oj);
      o = oj;
      t.path = o.fail == F_OK ? PT_JACOBI : PT_DONE;
      t.trial_eq = o.trial;
    }
    return;
  }
  const float f00 = 1.f + Htr[0], f01 = Htr[1], f02 = Htr[2];
  const float f10 = Htr[3], f11 = 1.f + Htr[4], f12 = Htr[5];
  const float f20 = Htr[6], f21 = Htr[7], f22 = 1.f + Htr[8];
  const float det = f00 * (f11 * f22 - f21 * f12) - f01 * (f10 * f22 - f20 * f12) + f02 * (f10 * f21 - f20 * f11);
  if (!(det > 0.f)) {
    o.fail = isfinite(det) ? F_CONST_INVERTED : F_CONST_NONFINITE;
    t.path = PT_DONE;
    t.trial_eq = 0.0;
    return;
  }
  // log(I + B) = B (c1 I + B (c2 I + ... + B cK)), c_j = (-1)^(j+1) / j; K from the truncation
  // bound r^(K+1) / ((K+1)(1-r)) <= 2e-8 r
  const int K = r <= 0.01f ? 4 : (r <= 0.05f ? 6 : (r <= 0.1f ? 7 : (r <= 0.18f ? 10 : 12)));
  Sym P;
  {
    const float cK = kLogSeries[K];
    P.xx = P.yy = P.zz = cK;
    P.xy = P.xz = P.yz = 0.f;
    for (int j = K - 1; j >= 1; --j) {
      Sym q = sym_mul(B, P);
      const float cj = kLogSeries[j];
      q.xx += cj;
      q.yy += cj;
      q.zz += cj;
      P = q;
    }
  }
  Sym E = sym_mul(B, P);
  E.xx *= 0.5f;
  E.yy *= 0.5f;
  E.zz *= 0.5f;
  E.xy *= 0.5f;
  E.xz *= 0.5f;
  E.yz *= 0.5f;
  const float vol = E.xx + E.yy + E.zz;
  const float mean = vol / 3.f;
  t.vol = vol;
  t.mean = mean;
  Sym& dev = t.dev;
  dev = E;
  dev.xx -= mean;
  dev.yy -= mean;
  dev.zz -= mean;
  t.dnorm = sym_norm(dev);
  t.trial_eq = 1.2247448713915890 * 2.0 * mu_d * (double)t.dnorm;  // sqrt(3/2) 2 mu |dev|
  t.path = PT_SERIES;
}

// The Herschel-Bulkley return of the series path after paste_trial, started at sigma0 (in
// (yield, trial), or -1 for the midpoint): sets o.eq, o.trial, and for a yielding particle
// o.dep, o.iters, o.yielded (or o.fail), and returns the deviatoric scale sigma / sigma_tr.
// newton_cycles (measurement builds only, else null): clock64 cycles spent in the return are
// added to it.
__device__ __forceinline__ double paste_return(double trial_eq, float dnorm, double ys, const HbConst& h, double tol,
                                               double sigma0, PasteOut& o, long long* newton_cycles = nullptr) {
  o.eq = trial_eq;
  o.trial = trial_eq;
  double scale = 1.0;
  if (trial_eq > ys && dnorm > 0.f) {
    double sigma, dep;
    int iters;
    const long long c0 = newton_cycles ? clock64() : 0;
    const int e = hb_return_d(trial_eq, ys, h, tol, sigma0, &sigma, &dep, &iters);
    if (newton_cycles) *newton_cycles += clock64() - c0;
    o.iters = iters;
    if (e != F_OK) {
      o.fail = e;
      return 1.0;
    }
    scale = sigma / trial_eq;
    o.dep = dep;
    o.eq = sigma;
    o.yielded = 1;
  }
  return scale;
}

// The stress and the plastic correction of H after paste_return (series path): tau from the
// scaled deviatoric Hencky strain, and for a yielding particle H_new = H_tr + G (I + H_tr) with
// G = exp((scale - 1) dev E) - I.
__device__ __forceinline__ void paste_stress(const float Htr[9], const Sym& dev, float mean, float vol, float mu,
                                             float lambda, double scale, PasteOut& o) {
  const float sc = (float)scale;
  const float lv = lambda * vol;
  o.tau[0] = 2.f * mu * (dev.xx * sc + mean) + lv;
  o.tau[1] = 2.f * mu * (dev.yy * sc + mean) + lv;
  o.tau[2] = 2.f * mu * (dev.zz * sc + mean) + lv;
  o.tau[3] = 2.f * mu * dev.xy * sc;
  o.tau[4] = 2.f * mu * dev.xz * sc;
  o.tau[5] = 2.f * mu * dev.yz * sc;
  for (int i = 0; i < 6; ++i)
    if (!isfinite(o.tau[i])) {
      o.fail = F_CONST_NONFINITE;
      return;
    }
  if (o.yielded) {
    // G = exp(M) - I, M = (s - 1) dev E, Horner: M (I + M/2 (I + M/3 (I + ...)))
    Sym M = dev;
    const float a = sc - 1.f;
    M.xx *= a;
    M.yy *= a;
    M.zz *= a;
    M.xy *= a;
    M.xz *= a;
    M.yz *= a;
    const float mn = sym_norm(M);
    const int T = mn <= 0.02f ? 4 : (mn <= 0.1f ? 6 : 9);
    Sym Q;
    Q.xx = Q.yy = Q.zz = 1.f;
    Q.xy = Q.xz = Q.yz = 0.f;
    for (int j = T; j >= 2; --j) {
      Sym q = sym_mul(M, Q);
      const float inv = kInverse[j];
      Q.xx = 1.f + q.xx * inv;
      Q.yy = 1.f + q.yy * inv;
      Q.zz = 1.f + q.zz * inv;
      Q.xy = q.xy * inv;
      Q.xz = q.xz * inv;
      Q.yz = q.yz * inv;
    }
    const Sym G = sym_mul(M, Q);
    const float Gm[9] = {G.xx, G.xy, G.xz, G.xy, G.yy, G.yz, G.xz, G.yz, G.zz};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const float s2 = Gm[3 * i + j] + (Gm[3 * i + 0] * Htr[0 * 3 + j] + Gm[3 * i + 1] * Htr[1 * 3 + j] +
                                          Gm[3 * i + 2] * Htr[2 * 3 + j]);
        o.H[3 * i + j] = Htr[3 * i + j] + s2;
      }
  } else {
#pragma unroll
    for (int i = 0; i < 9; ++i) o.H[i] = Htr[i];
  }
  o.diss_density = o.eq * o.dep;
}

// Rest of the paste update after paste_trial: the return (paste_return) and the stress and
// plastic correction (paste_stress), or the eigen-decomposition path for PT_JACOBI.
template <bool DEFER = false>
__device__ inline void paste_finish(const float Htr[9], float mu, float lambda, double mu_d, double ys, const HbConst& h,
                                    double tol, double sigma0, const PasteTrial& t, PasteOut& o,
                                    long long* newton_cycles = nullptr) {
  if (t.path == PT_DONE || t.path == PT_DEFER) return;
  if constexpr (!DEFER) {
    if (t.path == PT_JACOBI) {
      float Hj[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) Hj[i] = Htr[i];
      PasteOut oj = o;
      paste_update_jacobi(Hj, mu, lambda, mu_d, ys, h, tol, sigma0, false, oj);
      o = oj;
      return;
    }
  }
  const double scale = paste_return(t.trial_eq, t.dnorm, ys, h, tol, sigma0, o, newton_cycles);
  if (o.fail != F_OK) return;
  paste_stress(Htr, t.dev, t.mean, t.vol, mu, lambda, scale, o);
}

// whole paste update (constitutive.rs:456-531) with the reference's midpoint Newton start
__device__ inline void paste_update(const float Htr[9], float mu, float lambda, double mu_d, double ys, double k,
                                    double n, double dt, double tol, PasteOut& o) {
  PasteTrial t;
  paste_trial(Htr, mu_d, t, o);
  paste_finish(Htr, mu, lambda, mu_d, ys, hb_const(k, n, mu_d, dt), tol, -1.0, t, o);
}

// ---------------------------------------------------------------- liquid update (J - 1)
// update_liquid of constitutive.rs:557-589 on jm1 = J - 1, plus the Tait EOS extension
// p = (K/gamma) (J^-gamma - 1) (gamma == 1 is the reference's K (1/J - 1)).
struct LiquidOut {
  float jm1;
  float tau[6];
  float pressure;
  int fail;
};
__device__ inline void liquid_update(float jm1, const float C[9], float bulk, float visc, float gamma, float dt,
                                     LiquidOut& o) {
  o.fail = F_OK;
  const float tr = C[0] + C[4] + C[8];
  const float g = dt * tr;
  const float nj = jm1 + g + jm1 * g;  // (1 + jm1)(1 + g) - 1
  const float J = 1.f + nj;
  if (!isfinite(nj)) {
    o.fail = F_CONST_NONFINITE;
    return;
  }
  if (J <= 1e-6f) {
    o.fail = F_CONST_INVERTED;
    return;
  }
  float p;
  if (gamma == 1.f) p = -bulk * nj / J;
  else p = bulk / gamma * expm1f(-gamma * log1pf(nj));
  const float third = (C[0] + C[4] + C[8]) / 3.f;
  const float s = 2.f * visc * J;
  o.tau[0] = -p * J + s * (C[0] - third);
  o.tau[1] = -p * J + s * (C[4] - third);
  o.tau[2] = -p * J + s * (C[8] - third);
  o.tau[3] = s * 0.5f * (C[1] + C[3]);
  o.tau[4] = s * 0.5f * (C[2] + C[6]);
  o.tau[5] = s * 0.5f * (C[5] + C[7]);
  for (int i = 0; i < 6; ++i)
    if (!isfinite(o.tau[i])) {
      o.fail = F_CONST_NONFINITE;
      return;
    }
  o.jm1 = nj;
  o.pressure = p;
}

}  // namespace lp
