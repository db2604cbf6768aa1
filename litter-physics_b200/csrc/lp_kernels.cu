// lp_kernels.cu - CUDA kernels of one MLS-MPM substep attempt (sm_100a).
//
// Attempt = begin -> bin (count, scan, scatter, slot sort) -> P2G -> wall traction -> grid update
//           -> pellet coupling -> (warm-start table) -> G2P + constitutive -> end (reduce,
//           accept / reject, commit).
// Every kernel reads dt, the fixed-point scales and the buffer parity of its instance from the
// device control block, so one attempt is a fixed launch sequence that a CUDA graph can replay.
//
// Reference mapping (nredd/litter-physics):
//   k_begin        solver.rs:418-441 (dt selection of advance_while), 477-498 (stability_limit)
//   k_bin_*        replaces sort_particles (solver.rs:501-517): a counting sort by stencil cell
//                  every attempt; ties ordered by slot in the committed state, so the order is
//                  deterministic
//   k_p2g          deposit_particles (solver.rs:632-661), Grid::deposit (grid.rs:254-263)
//   k_traction     wall_traction_to_grid (solver.rs:725-819), Grid::deposit_reaction (grid.rs:279-295)
//   k_grid_update  grid_update (solver.rs:822-892), reduce_tangential_velocity (solver.rs:1145-1155)
//   k_couple       couple_grid (rigid.rs:385-438), apply_impulse / integrate (rigid.rs:251-334)
//   k_mlp_table    learned warm start of the HB return: the network tabulated per instance and dt
//                  (no reference counterpart)
//   k_g2p          grid_to_particle (solver.rs:895-977) + update_paste / update_liquid
//   k_end          try_step_captured's accept/reject and commit (solver.rs:540-611, 980-998),
//                  advance_while's bookkeeping (solver.rs:442-468)
#include "lp_device.cuh"
#include "lp_kernels.h"

#include <cstdio>

namespace lp {

// ============================================================== helpers
__device__ __forceinline__ float* comp(float* base, int64_t cap, int c) { return base + (int64_t)c * cap; }
__device__ __forceinline__ const float* comp(const float* base, int64_t cap, int c) {
  return base + (int64_t)c * cap;
}

__device__ __forceinline__ int64_t node_index(const InstDesc& D, int i, int j, int k) {
  return D.node_off + ((int64_t)i * D.nodes[1] + j) * D.nodes[2] + k;
}

// Stencil base (padded) of a coordinate: floor(x/dx - 0.5) + 1 (grid.rs:151-182).
// x / dx in grid units.  For a power-of-two dx (pow2_inv_dx != 0) the product with its exact
// reciprocal is the same correctly rounded quotient, without the division.
__device__ __forceinline__ float scaled_of(float x, float dx, float pow2_inv_dx) {
  return pow2_inv_dx != 0.0f ? x * pow2_inv_dx : x / dx;
}

__device__ __forceinline__ void weights_of(float fx, float dx, float w[3], float d[3]) {
  const float a0 = 1.5f - fx, a1 = fx - 1.0f, a2 = fx - 0.5f;
  w[0] = 0.5f * (a0 * a0);
  w[1] = 0.75f - (a1 * a1);
  w[2] = 0.5f * (a2 * a2);
  d[0] = fx * -dx;
  d[1] = (fx - 1.0f) * -dx;
  d[2] = (fx - 2.0f) * -dx;
}

// block-wide deterministic reductions (fixed tree); NT need not be a power of two: the
// entries above the largest power of two are folded in first.
template <int NT>
struct Pow2Floor {
  static constexpr int value = (NT & (NT - 1)) == 0 ? NT : Pow2Floor<NT & (NT - 1)>::value;
};
template <>
struct Pow2Floor<0> {
  static constexpr int value = 0;
};

template <int NT, typename T, typename Op>
__device__ T block_reduce(T v, T* sh, Op op) {
  constexpr int P = Pow2Floor<NT>::value;
  const int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
  if (P < NT) {
    if (t < NT - P) sh[t] = op(sh[t], sh[t + P]);
    __syncthreads();
  }
  for (int s = P / 2; s > 0; s >>= 1) {
    if (t < s) sh[t] = op(sh[t], sh[t + s]);
    __syncthreads();
  }
  T r = sh[0];
  __syncthreads();
  return r;
}
struct AddOp {
  template <typename T>
  __device__ T operator()(T a, T b) const { return a + b; }
};
struct MaxFOp {
  __device__ float operator()(float a, float b) const { return fmaxf(a, b); }
};
struct MaxIOp {
  __device__ int operator()(int a, int b) const { return max(a, b); }
};
template <int NT>
__device__ double block_sum_d(double v, double* sh) { return block_reduce<NT>(v, sh, AddOp()); }
template <int NT>
__device__ long long block_sum_ll(long long v, long long* sh) { return block_reduce<NT>(v, sh, AddOp()); }
template <int NT>
__device__ float block_max_f(float v, float* sh) { return block_reduce<NT>(v, sh, MaxFOp()); }
template <int NT>
__device__ int block_max_i(int v, int* sh) { return block_reduce<NT>(v, sh, MaxIOp()); }

// Multi-value block reductions with a fixed warp butterfly (__shfl_xor_sync) followed by one
// shared-memory pass in warp 0: deterministic, two barriers.  Bit k of max_mask selects max
// instead of sum for value k.  The results are returned to every thread.
template <int K>
__device__ __forceinline__ void warp_reduce_multi(double (&v)[K], unsigned max_mask) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double other = __shfl_xor_sync(0xffffffffu, v[k], o);
      v[k] = ((max_mask >> k) & 1u) ? fmax(v[k], other) : v[k] + other;
    }
  }
}
template <int NT, int K>
__device__ void block_reduce_multi(double (&v)[K], unsigned max_mask, double* sh /* NT/32*K + K */) {
  constexpr int NW = NT / 32;
  static_assert(NT % 32 == 0 && NW <= 32, "block size");
  warp_reduce_multi<K>(v, max_mask);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sh[w * K + k] = v[k];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = lane < NW ? sh[lane * K + k] : (((max_mask >> k) & 1u) ? -1e300 : 0.0);
    warp_reduce_multi<K>(v, max_mask);
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < K; ++k) sh[NW * K + k] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = sh[NW * K + k];
  __syncthreads();
}
// block_reduce_multi for a caller that reads the result in thread 0 only: one barrier, the
// totals end in warp 0, and sh must not be rewritten before the caller's next barrier
template <int NT, int K>
__device__ void block_reduce_multi_to0(double (&v)[K], unsigned max_mask, double* sh /* NT/32*K */) {
  constexpr int NW = NT / 32;
  static_assert(NT % 32 == 0 && NW <= 32, "block size");
  warp_reduce_multi<K>(v, max_mask);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sh[w * K + k] = v[k];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = lane < NW ? sh[lane * K + k] : (((max_mask >> k) & 1u) ? -1e300 : 0.0);
    warp_reduce_multi<K>(v, max_mask);
  }
}
template <int K>
__device__ __forceinline__ void warp_sum_ll_multi(long long (&v)[K]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
}
// Exact int64 sum over a full warp by the integer reduction unit (redux.sync): the value is split
// into 22-, 22- and 20-bit (signed) limbs, whose 32-lane sums fit 32 bits; the recombination
// is exact modulo 2^64, hence exact whenever the total fits int64.
__device__ __forceinline__ long long warp_sum_ll_redux(long long v) {
  const unsigned long long u = (unsigned long long)v;
  const unsigned s0 = __reduce_add_sync(0xffffffffu, (unsigned)(u & 0x3fffffull));
  const unsigned s1 = __reduce_add_sync(0xffffffffu, (unsigned)((u >> 22) & 0x3fffffull));
  const int s2 = __reduce_add_sync(0xffffffffu, (int)(v >> 44));
  return (long long)((unsigned long long)s0 + ((unsigned long long)s1 << 22) +
                     ((unsigned long long)(long long)s2 << 44));
}
// TRAIL = false leaves out the closing barrier: the caller must not rewrite sh[NW K .. NW K + K)
// before another barrier (the partial sums below it may be rewritten at once)
template <int NT, int K, bool TRAIL = true>
__device__ void block_sum_ll_multi(long long (&v)[K], long long* sh /* NT/32*K + K */) {
  constexpr int NW = NT / 32;
  warp_sum_ll_multi<K>(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sh[w * K + k] = v[k];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = lane < NW ? sh[lane * K + k] : 0;
    warp_sum_ll_multi<K>(v);
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < K; ++k) sh[NW * K + k] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = sh[NW * K + k];
  if (TRAIL) __syncthreads();
}
// Sums of K int64 values over the block and, in the same pass, the argmax of (value, index):
// largest value, lowest index on ties.  sh holds NW K + NW + K values and shi NW + 1 ints (NW
// warps).  Two barriers; the caller must not rewrite sh or shi before another barrier.
template <int NT, int K>
__device__ int block_sum_argmax_ll(long long (&v)[K], long long value, int index, long long* sh, int* shi) {
  constexpr int NW = NT / 32;
  warp_sum_ll_multi<K>(v);
  auto better = [](long long ov, int oi, long long bv, int bi) { return ov > bv || (ov == bv && oi < bi); };
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const long long ov = __shfl_xor_sync(0xffffffffu, value, o);
    const int oi = __shfl_xor_sync(0xffffffffu, index, o);
    if (better(ov, oi, value, index)) {
      value = ov;
      index = oi;
    }
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) sh[w * K + k] = v[k];
    sh[NW * K + w] = value;
    shi[w] = index;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = lane < NW ? sh[lane * K + k] : 0;
    warp_sum_ll_multi<K>(v);
    long long bv = lane < NW ? sh[NW * K + lane] : LLONG_MIN;
    int bi = lane < NW ? shi[lane] : INT_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const long long ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (better(ov, oi, bv, bi)) {
        bv = ov;
        bi = oi;
      }
    }
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < K; ++k) sh[NW * K + NW + k] = v[k];
      shi[NW] = bi;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = sh[NW * K + NW + k];
  return shi[NW];
}

// Per-particle bound of the node momentum one particle can deposit (mass times speed, affine and
// stress terms over the stencil, one gravity kick).  The norms are taken in FP32 and, where a
// square overflows FP32, again in FP64, so that no magnitude a finite FP32 state holds overflows
// the bound; the sum is FP64.  k_g2p and k_state_stats evaluate these same expressions, so an
// imported state gets the bound of the run that wrote it.
__device__ __forceinline__ float affine_norm(const float Cm[9]) {
  float c2 = 0.f;
#pragma unroll
  for (int a = 0; a < 9; ++a) c2 = fmaf(Cm[a], Cm[a], c2);
  if (isfinite(c2)) return sqrtf(c2);
  double d2 = 0.0;
#pragma unroll
  for (int a = 0; a < 9; ++a) d2 += (double)Cm[a] * Cm[a];
  return (float)sqrt(d2);
}
// |v| with explicit roundings, so that k_g2p and k_g2p_defer get the same value from the same v
__device__ __forceinline__ float particle_speed(const float v[3]) {
  return sqrtf(__fmaf_rn(v[2], v[2], __fmaf_rn(v[1], v[1], __fmul_rn(v[0], v[0]))));
}
__device__ __forceinline__ double momentum_bound(float m, float speed, float cn, const float tau[6], float v0,
                                                 float c_tau, float c_dx, float c_g) {
  const float f2 = tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2] +
                   2.f * (tau[3] * tau[3] + tau[4] * tau[4] + tau[5] * tau[5]);
  double tn;
  if (isfinite(f2)) {
    tn = (double)sqrtf(f2);
  } else {
    const double t2 = (double)tau[0] * tau[0] + (double)tau[1] * tau[1] + (double)tau[2] * tau[2] +
                      2.0 * ((double)tau[3] * tau[3] + (double)tau[4] * tau[4] + (double)tau[5] * tau[5]);
    tn = sqrt(t2);
  }
  return (double)m * speed + ((double)m * cn + tn * c_tau * v0) * c_dx + (double)m * c_g;
}

// Tile loop of a persistent CTA over the entries of the attempt's occupied-tile list:
//   for (uint32_t i = tile_first(cursor, &slot); i < n; i = tile_next(cursor, i, &slot)) {
//     ...one tile...; __syncthreads();
//   }
// With a cursor the CTAs take entries from it one at a time (atomicAdd; k_begin resets it), so a
// CTA that drew light tiles takes more of them; without one they take every gridDim.x-th entry.
// Results are per tile, so the order and the CTA that processes a tile change nothing.  The
// barrier that ends each tile also orders every thread's read of *slot before thread 0 writes it
// again.
__device__ __forceinline__ uint32_t tile_take(uint32_t* cursor, uint32_t* slot) {
  if (threadIdx.x == 0) *slot = atomicAdd(cursor, 1u);
  __syncthreads();
  return *slot;
}
__device__ __forceinline__ uint32_t tile_first(uint32_t* cursor, uint32_t* slot) {
  return cursor ? tile_take(cursor, slot) : blockIdx.x;
}
__device__ __forceinline__ uint32_t tile_next(uint32_t* cursor, uint32_t i, uint32_t* slot) {
  return cursor ? tile_take(cursor, slot) : i + gridDim.x;
}

// ============================================================== begin
// One thread per instance: decides whether the instance attempts a step and with which dt.
__global__ void k_begin(const InstDesc* __restrict__ desc, Control* __restrict__ ctrl, int n_inst,
                        uint32_t* __restrict__ nw_count, BedPtrs bed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    nw_count[0] = 0u;  // near-wall particle list of this attempt
    nw_count[1] = 0u;  // occupied-tile list of this attempt
    nw_count[2] = 0u;  // tile cursors of the bin sort, P2G and G2P
    nw_count[3] = 0u;
    nw_count[4] = 0u;
    nw_count[5] = 0u;  // tiles left to k_g2p_defer
  }
  if (i >= n_inst) return;
  const InstDesc& D = desc[i];
  Control& c = ctrl[i];
  c.fail = F_OK;
  c.outflow = 0;
  c.pellet_fail = 0;
  c.epoch += 1;
  // fixed-point momentum scale from the committed state's momentum bound
  {
    // a non-finite bound (non-finite state) fails the attempt in k_end; any scale does meanwhile
    double b = c.bbound > 0.0 ? fmin(c.bbound, 1e300) : 1e-300;
    int e = (int)floor(log2(2.305843009213694e18 / b));  // 2^61 / b
    e = e > 200 ? 200 : (e < -200 ? -200 : e);
    c.s_mom = ldexp(1.0, e);
  }
  if (c.forced_dt > 0.0) {
    c.active = (c.status == S_RUNNING || c.status == S_REACHED) ? 1 : 0;
    c.dt = c.forced_dt;
    c.hb = hb_const(D.consistency, D.flow_index, D.mu, c.dt);
    c.limited = 0;
    return;
  }
  if (c.status != S_RUNNING || !(c.time < c.target)) {
    c.active = 0;
    return;
  }
  // stability_limit (solver.rs:477-498)
  const double dx = D.dx;
  const double wave = D.kind == 0 ? sqrt((D.lambda + 2.0 * D.mu) / D.density) : sqrt(D.bulk / D.density);
  double limit = D.cfl * dx / (wave + c.max_speed);
  const double diff = D.kind == 0 ? 0.0 : D.consistency / D.density;
  if (diff > 0.0) limit = fmin(limit, 0.25 * dx * dx / diff);
  if (D.has_pellet) {
    limit = fmin(limit, 0.2 * sqrt(c.pellet.mass / D.contact_k));
    const double ps = sqrt(c.pellet.vel[0] * c.pellet.vel[0] + c.pellet.vel[1] * c.pellet.vel[1] +
                           c.pellet.vel[2] * c.pellet.vel[2]);
    if (ps > 0.0) limit = fmin(limit, D.cfl * dx / ps);
  }
  if (D.bed_np >= 2) limit = fmin(limit, c.bed_limit);
  // advance_while dt choice (solver.rs:424-441)
  const double remaining = c.target - c.time;
  const double scaled = c.dt_scale * limit;
  const int limited = scaled < D.max_dt ? 1 : 0;
  double dt = fmin(fmin(scaled, D.max_dt), remaining);
  if (remaining - dt < 1e-12 * fmax(c.target, 1.0)) dt = remaining;
  if (!isfinite(dt) || dt <= 0.0 || (dt < D.min_dt && remaining > D.min_dt)) {
    c.status = S_MIN_STEP;
    c.active = 0;
    c.last_fail = -1;
    c.fail_value = dt;
    return;
  }
  c.limit = limit;
  c.dt = dt;
  c.hb = hb_const(D.consistency, D.flow_index, D.mu, dt);
  c.limited = limited;
  c.active = 1;
}

// ============================================================== binning
// Runs of equal values among the active lanes (a prefix of the warp): the first lane of each run
// gets the run's length, the others 0.
__device__ __forceinline__ uint32_t run_length(unsigned am, unsigned lane, uint32_t v) {
  const uint32_t prev = __shfl_up_sync(am, v, 1);
  const unsigned heads = __ballot_sync(am, lane == 0 || prev != v) | ~am;
  if (!((heads >> lane) & 1u) || !((am >> lane) & 1u)) return 0u;
  const unsigned later = heads & ~((2u << lane) - 1u);  // heads after this lane (lane 31: none)
  const unsigned next = later ? (unsigned)(__ffs(later) - 1) : 32u;
  return next - lane;
}

// The binning passes run 2 warps per block of G2P_THREADS slots; each warp takes 4 rounds of 32
// consecutive slots and issues the loads (and, in the scatter, the atomics) of all its rounds
// before using them, so that each warp keeps several memory requests in flight.
constexpr int BIN_THREADS = 64, BIN_ROUNDS = 4;
static_assert(BIN_THREADS * BIN_ROUNDS == G2P_THREADS, "a binning CTA covers one slot block");

// stencil-cell key of a particle at x (the instance's outflow key when the stencil leaves the
// grid) and whether it lies within dx/2 of a wall
__device__ __forceinline__ uint32_t bin_key(const InstDesc& D, const float (&x)[3], float dx, bool& ok, bool& near) {
  int b[3];
  ok = true;
  near = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float s = scaled_of(x[a], dx, D.pow2_inv_dx);
    const float bf = floorf(s - 0.5f);
    const float padded = bf + 1.0f;
    if (!(padded >= 0.0f) || padded + 2.0f >= (float)D.nodes[a]) ok = false;
    b[a] = ok ? (int)padded : 0;
    const float half = 0.5f * dx;
    if (x[a] < half || x[a] > (float)D.extent[a] - half) near = true;
  }
  if (!ok) return (uint32_t)(D.key_off + D.nkeys - 1);
  const int tx = b[0] / TX, ty = b[1] / TY, tz = b[2] / TZ;
  const int lx = b[0] % TX, ly = b[1] % TY, lz = b[2] % TZ;
  const int64_t tile = ((int64_t)tx * D.tiles[1] + ty) * D.tiles[2] + tz;
  return (uint32_t)(D.key_off + tile * TB + (lx * TY + ly) * TZ + lz);
}

// 32 registers: 32 CTAs (the full 64 warps) per SM to cover the position loads
__global__ void __launch_bounds__(BIN_THREADS, 32)
    k_bin_count(const InstDesc* __restrict__ desc, Control* __restrict__ ctrl, const int* __restrict__ pcta_inst,
                const float* __restrict__ st0, const float* __restrict__ st1, int64_t cap,
                uint32_t* __restrict__ keys, uint32_t* __restrict__ count, uint32_t* __restrict__ chunk_sum,
                uint32_t* __restrict__ nw_list, uint32_t* __restrict__ nw_count) {
  const int inst = pcta_inst[blockIdx.x];
  const Control& c = ctrl[inst];
  if (!c.active) return;
  const InstDesc& D = desc[inst];
  const unsigned lane = threadIdx.x & 31;
  const int64_t base = (int64_t)blockIdx.x * G2P_THREADS + (threadIdx.x >> 5) * (32 * BIN_ROUNDS) + lane;
  const int64_t lim = D.slot_off + c.count;  // slots below lim hold particles
  const float* cur = c.parity ? st1 : st0;
  float xs[BIN_ROUNDS][3];
#pragma unroll
  for (int q = 0; q < BIN_ROUNDS; ++q)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int64_t slot = base + 32 * q;
      xs[q][a] = slot < lim ? cur[(int64_t)(C_X + a) * cap + slot] : 0.f;
    }
  // lanes holding a particle in each round (a prefix of the warp), taken while the warp is converged
  unsigned amq[BIN_ROUNDS];
#pragma unroll
  for (int q = 0; q < BIN_ROUNDS; ++q) amq[q] = __ballot_sync(0xffffffffu, base + 32 * q < lim);
  const float dx = (float)D.dx;
#pragma unroll
  for (int q = 0; q < BIN_ROUNDS; ++q) {
    const unsigned am = amq[q];
    if (!am) break;  // warp-uniform
    const int64_t slot = base + 32 * q;
    if (slot < lim) {
      bool ok, near;
      const uint32_t key = bin_key(D, xs[q], dx, ok, near);
      if (!ok) atomicAdd((unsigned long long*)&ctrl[inst].outflow, 1ull);
      keys[slot] = key;
      // near-wall particles go to the traction list: one atomic per warp on the shared counter
      const unsigned nb = __ballot_sync(am, ok && near);
      if (nb) {
        const unsigned first = (unsigned)(__ffs(nb) - 1);
        uint32_t w = 0u;
        if (lane == first) w = atomicAdd(nw_count, (uint32_t)__popc(nb));
        w = __shfl_sync(am, w, first);
        if (ok && near) nw_list[w + __popc(nb & ((1u << lane) - 1u))] = (uint32_t)slot;
      }
      // particles arrive in binned order, so a warp's keys come in runs: one atomic per run of
      // equal keys, and one per run of equal key chunks
      uint32_t len = run_length(am, lane, key);
      if (len) atomicAdd(&count[key], len);
      const uint32_t ch = key / KEY_CHUNK;
      len = run_length(am, lane, ch);
      if (len) atomicAdd(&chunk_sum[ch], len);
    }
    __syncwarp();  // the warp reconverges before the next round's masked collectives
  }
}

// per instance: exclusive scan of its key-chunk sums (accumulated by k_bin_count), offset by the
// instance's first slot.  1024 threads take 4 consecutive chunks each per pass: warp shuffles scan
// the thread sums, one warp scans the 32 warp totals.
__global__ void __launch_bounds__(1024) k_scan_instances(const InstDesc* __restrict__ desc,
                                                         const Control* __restrict__ ctrl,
                                                         uint32_t* __restrict__ chunk_sum,
                                                         uint32_t* __restrict__ chunk_base) {
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t pass_total;
  const int inst = blockIdx.x;
  if (!ctrl[inst].active) return;
  const InstDesc& D = desc[inst];
  const int64_t c0 = D.key_off / KEY_CHUNK, nc = D.nkeys / KEY_CHUNK;
  const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t carry = (uint32_t)D.slot_off;
  for (int64_t base = 0; base < nc; base += 4 * 1024) {
    const int64_t j0 = base + 4 * (int64_t)threadIdx.x;
    uint32_t v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      v[q] = 0u;
      if (j0 + q < nc) {
        v[q] = chunk_sum[c0 + j0 + q];
        chunk_sum[c0 + j0 + q] = 0u;  // k_bin_count of the next attempt accumulates from zero
      }
    }
    const uint32_t tsum = v[0] + v[1] + v[2] + v[3];
    uint32_t x = tsum;  // inclusive scan of the thread sums within the warp
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
      if (lane >= (unsigned)off) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
      const uint32_t w = wsum[lane];
      uint32_t t = w;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, t, off);
        if (lane >= (unsigned)off) t += y;
      }
      wsum[lane] = t - w;  // exclusive prefix of the warp totals
      if (lane == 31) pass_total = t;
    }
    __syncthreads();
    uint32_t e = carry + wsum[wid] + x - tsum;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (j0 + q < nc) chunk_base[c0 + j0 + q] = e;
      e += v[q];
    }
    carry += pass_total;
    __syncthreads();  // wsum and pass_total are rewritten by the next pass
  }
}

// per chunk: exclusive scan of counts -> bin start slots; 256 threads, four keys each
__global__ void __launch_bounds__(256) k_scan_apply(const uint32_t* __restrict__ count,
                                                   const uint32_t* __restrict__ chunk_base,
                                                   uint32_t* __restrict__ start, const int* __restrict__ chunk_inst,
                                                   const Control* __restrict__ ctrl) {
  __shared__ uint32_t sh[16];
  const int64_t chunk = blockIdx.x;
  if (!ctrl[chunk_inst[chunk]].active) return;
  const int64_t base = chunk * KEY_CHUNK;
  const uint4 c4 = reinterpret_cast<const uint4*>(count + base)[threadIdx.x];
  const uint32_t tsum = c4.x + c4.y + c4.z + c4.w;
  const uint32_t cb = chunk_base[chunk];
  if (!__syncthreads_or(tsum != 0u)) {  // no particle in this chunk (CTA-uniform)
    reinterpret_cast<uint4*>(start + base)[threadIdx.x] = make_uint4(cb, cb, cb, cb);
    return;
  }
  const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = tsum;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= (unsigned)off) x += y;
  }
  if (lane == 31) sh[wid] = x;
  __syncthreads();
  if (wid == 0) {
    const uint32_t w = lane < 8 ? sh[lane] : 0u;
    uint32_t t = w;
#pragma unroll
    for (int off = 1; off < 8; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, t, off);
      if (lane >= (unsigned)off) t += y;
    }
    if (lane < 8) sh[8 + lane] = t - w;  // exclusive prefix of the warp totals
  }
  __syncthreads();
  const uint32_t e0 = cb + sh[8 + wid] + x - tsum;
  reinterpret_cast<uint4*>(start + base)[threadIdx.x] =
      make_uint4(e0, e0 + c4.x, e0 + c4.x + c4.y, e0 + c4.x + c4.y + c4.z);
}

// Each particle takes a place in its bin: one atomicSub per run of equal keys in a round, which
// also leaves count at zero for the next attempt.  The order inside a bin follows the atomics and
// is made deterministic by k_bin_sort.
__global__ void __launch_bounds__(BIN_THREADS)
    k_bin_scatter(const InstDesc* __restrict__ desc, const Control* __restrict__ ctrl,
                  const int* __restrict__ pcta_inst, const uint32_t* __restrict__ keys, uint32_t* __restrict__ count,
                  const uint32_t* __restrict__ start, uint32_t* __restrict__ perm) {
  const int inst = pcta_inst[blockIdx.x];
  const Control& c = ctrl[inst];
  if (!c.active) return;
  const InstDesc& D = desc[inst];
  const unsigned lane = threadIdx.x & 31;
  const int64_t base = (int64_t)blockIdx.x * G2P_THREADS + (threadIdx.x >> 5) * (32 * BIN_ROUNDS) + lane;
  const int64_t lim = D.slot_off + c.count;
  uint32_t key[BIN_ROUNDS], top[BIN_ROUNDS], lead[BIN_ROUNDS], st[BIN_ROUNDS];
  unsigned am[BIN_ROUNDS];
#pragma unroll
  for (int q = 0; q < BIN_ROUNDS; ++q) key[q] = base + 32 * q < lim ? keys[base + 32 * q] : 0u;
#pragma unroll
  for (int q = 0; q < BIN_ROUNDS; ++q) {
    am[q] = __ballot_sync(0xffffffffu, base + 32 * q < lim);
    top[q] = lead[q] = st[q] = 0u;
  }
#pragma unroll
  for (int q = 0; q < BIN_ROUNDS; ++q) {
    if (base + 32 * q < lim) {
      const uint32_t len = run_length(am[q], lane, key[q]);
      const unsigned prev = __shfl_up_sync(am[q], key[q], 1);
      const unsigned heads = __ballot_sync(am[q], lane == 0 || prev != key[q]);
      lead[q] = 31u - __clz(heads & ((2u << lane) - 1u));  // first lane of this lane's run
      if (len) top[q] = atomicSub(&count[key[q]], len);
    }
    __syncwarp();
  }
#pragma unroll
  for (int q = 0; q < BIN_ROUNDS; ++q) {
    if (base + 32 * q < lim) {
      top[q] = __shfl_sync(am[q], top[q], lead[q]);
      st[q] = start[key[q]];
    }
    __syncwarp();
  }
#pragma unroll
  for (int q = 0; q < BIN_ROUNDS; ++q)
    if (base + 32 * q < lim) perm[st[q] + top[q] - 1u - (lane - lead[q])] = (uint32_t)(base + 32 * q);
}

// sort n <= R slot indices in registers (unrolled insertion network; unused entries sort last)
template <int R>
__device__ __forceinline__ void bin_sort_small(uint32_t* __restrict__ p, int n) {
  uint32_t v[R];
#pragma unroll
  for (int i = 0; i < R; ++i) v[i] = i < n ? p[i] : 0xffffffffu;
#pragma unroll
  for (int i = 1; i < R; ++i)
#pragma unroll
    for (int j = i; j > 0; --j) {
      const uint32_t a = v[j - 1], b = v[j];
      v[j - 1] = min(a, b);
      v[j] = max(a, b);
    }
#pragma unroll
  for (int i = 0; i < R; ++i)
    if (i < n) p[i] = v[i];
}

// Order each bin by slot, that is by the particles' order in the committed state, which makes the
// binned order deterministic after the atomic scatter.  The committed state is itself in binned
// order, so a particle keeps its place relative to the others of its bin from step to step.
// Persistent CTAs of TB threads walk the occupied-tile list, one thread per bin.
__global__ void __launch_bounds__(TB) k_bin_sort(const InstDesc* __restrict__ desc, const uint32_t* __restrict__ start,
                                                 uint32_t* __restrict__ perm, const uint4* __restrict__ tile_rec,
                                                 const uint32_t* __restrict__ tile_count, uint32_t* cursor) {
  __shared__ uint32_t slot;
  const uint32_t n = *tile_count;
  for (uint32_t i = tile_first(cursor, &slot); i < n; i = tile_next(cursor, i, &slot)) {
    const uint4 rec = tile_rec[i];
    const int tile = (int)rec.x;
    const InstDesc& D = desc[rec.y];
    // a tile's keys are followed by at least the instance's outflow key, so key + 1 is valid
    const int64_t key = D.key_off + (int64_t)(tile - D.tile_off) * TB + threadIdx.x;
    const uint32_t s = start[key], e = start[key + 1];
    if (e - s > 1u) {
      if (e - s <= 8u) {  // the common case at 8 particles per cell
        bin_sort_small<8>(perm + s, (int)(e - s));
      } else if (e - s <= 16u) {
        bin_sort_small<16>(perm + s, (int)(e - s));
      } else {
        for (uint32_t j = s + 1; j < e; ++j) {
          const uint32_t pj = perm[j];
          uint32_t k = j;
          while (k > s && perm[k - 1] > pj) {
            perm[k] = perm[k - 1];
            --k;
          }
          perm[k] = pj;
        }
      }
    }
    if (cursor) __syncthreads();  // only the cursor's slot needs the barrier
  }
}

// The attempt's occupied tiles of the active instances, for the persistent bin-sort, P2G and G2P
// CTAs (the list order does not matter: their results are per tile).  Each entry is the record
// (tile, instance, first sorted slot, end slot), so that a CTA learns what it needs of a tile from
// one load.  Empty tiles get zero G2P partials.
__global__ void k_tiles(const InstDesc* __restrict__ desc, const Control* __restrict__ ctrl,
                        const int* __restrict__ tile_inst, int64_t n_tiles, const uint32_t* __restrict__ start,
                        uint4* __restrict__ tile_rec, uint32_t* __restrict__ tile_count,
                        ParticlePartial* __restrict__ tpart) {
  const int64_t tile = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool busy = false;
  int inst = 0;
  uint32_t ts = 0, te = 0;
  if (tile < n_tiles) {
    inst = tile_inst[tile];
    const Control& c = ctrl[inst];
    if (c.active) {
      const InstDesc& D = desc[inst];
      const int64_t key0 = D.key_off + (tile - D.tile_off) * TB;
      ts = start[key0];
      te = start[key0 + TB];
      busy = te > ts;
      if (!busy) {
        ParticlePartial& P = tpart[tile];
        P.diss = P.bbound = P.mass = 0.0;
        P.max_speed = P.max_disp = 0.f;
        P.fail = F_OK;
        P.iterations = P.yielded = 0;
        P.fail_value = 0.0;
      }
    }
  }
  const unsigned lane = threadIdx.x & 31;
  const unsigned bal = __ballot_sync(0xffffffffu, busy);
  uint32_t base = 0u;
  if (lane == 0 && bal) base = atomicAdd(tile_count, (uint32_t)__popc(bal));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (busy) tile_rec[base + __popc(bal & ((1u << lane) - 1u))] = make_uint4((uint32_t)tile, (uint32_t)inst, ts, te);
}

// ============================================================== P2G
// Persistent CTAs take the occupied tiles of TX x TY x TZ bins from the attempt's tile list.  A
// tile's particles (contiguous in sorted slot order) are taken in chunks of P2G_CHUNK:
//   phase 1: the CTA loads each particle once (coalesced in slot order) and writes a 16-float
//            record to shared memory: mass, momentum m v, the affine matrix
//            A = C m - tau (dt 4/dx^2 V0), and the position relative to its stencil base;
//   phase 2: three threads per bin, one per slab a of the 3x3x3 stencil, accumulate their 9
//            nodes x (mass, momentum) in registers over the bin's records in sorted order.
// All particles of a bin share the same 27 target nodes.  The partial sums then go to shared
// memory (aliasing the records); one thread per halo node adds its 27 contributors in a fixed
// order (deterministic, no atomics), converts to int64 fixed point, the tile's exact particle
// totals are restored by a proportional correction, and each node component is flushed with
// one global atomic.
// Chunk sizes (particles per chunk) of the two P2G instantiations the launch shape chooses from.
constexpr int P2G_CHUNK = 1024, P2G_CHUNK_SMALL = 512;
constexpr int P2G_REC = 16;  // m, q[3], A[9], f[3]
constexpr size_t P2G_PART_BYTES = sizeof(float4) * TB * 27;
// dynamic shared memory of a chunk size: the records, which the partial node sums alias later
__host__ __device__ constexpr size_t p2g_smem(int chunk) {
  return P2G_PART_BYTES > sizeof(float) * P2G_REC * chunk ? P2G_PART_BYTES : sizeof(float) * P2G_REC * chunk;
}
// Slot of chunk particle i in each record row: within each 32-word segment the slots rotate by
// the segment number, so bins whose particles start 32 apart (8 per bin in a lattice fill) read
// different shared-memory banks in the per-bin pass; consecutive i still fill a segment.
__device__ __forceinline__ uint32_t rec_slot(uint32_t i) { return (i & ~31u) | ((i + (i >> 5)) & 31u); }

// Asynchronous 4-byte global -> shared copies (cp.async) of this GPU's own memory, used by the
// staged P2G and by G2P to prefetch particle inputs while the CTA computes.
__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// State components P2G reads, in the order of the staged (prefetched) copies: x3 v3 C9 tau6 m V0.
constexpr int P2G_RAW = 23;
__device__ __forceinline__ int p2g_raw_comp(int r) {
  return r < 15 ? C_X + r : (r < 21 ? C_TAU + (r - 15) : (r == 21 ? C_M : C_V0));
}
__host__ __device__ constexpr size_t p2g_raw_bytes(int chunk) { return sizeof(float) * P2G_RAW * chunk; }

// APIC record of one particle, the quantities the per-bin pass scatters: momentum q = m v, the
// affine matrix A = C m - tau sv (sv = dt 4/dx^2 V0) and the position f relative to the stencil
// base (floor(x/dx - 0.5)).  Every rounding is explicit, so the variants that build the record in
// different places scatter bit-identical values.
__device__ __forceinline__ void p2g_record(const float v[3], const float Cm[9], const float tau[6], float m, float sv,
                                           float q[3], float A[9]) {
  const float T[9] = {tau[0], tau[3], tau[4], tau[3], tau[1], tau[5], tau[4], tau[5], tau[2]};
#pragma unroll
  for (int a = 0; a < 3; ++a) q[a] = __fmul_rn(v[a], m);
#pragma unroll
  for (int a = 0; a < 9; ++a) A[a] = __fmaf_rn(Cm[a], m, -__fmul_rn(T[a], sv));
}
__device__ __forceinline__ float p2g_frac(float x, float dx, float pow2_inv_dx) {
  const float sc = scaled_of(x, dx, pow2_inv_dx);
  return __fsub_rn(sc, floorf(__fsub_rn(sc, 0.5f)));
}
// Scatter of one record by the thread of slab `slab` (x offset) of its bin: the 9 nodes
// (slab, b, c) x (mass, momentum), accumulated in acc[b][c] as the pairs (p_x, p_y), (p_z, m).
// The sums run on Blackwell's paired FP32 units (fma.rn.f32x2): each lane of a pair is the
// single-precision FMA of the scalar form, p_r += w_ab w_c (q_r + A_r0 d_a + A_r1 d_b + A_r2 d_c)
// and m_node += w_ab w_c m, and the mass rides in the second lane of the z pair as m + 0 d.
__device__ __forceinline__ void p2g_scatter(float m, const float q[3], const float A[9], float fx, float fy, float fz,
                                            int slab, float dx, float2 (&acc)[3][3][2]) {
  float w[3][3], d[3][3];
  weights_of(fy, dx, w[1], d[1]);
  weights_of(fz, dx, w[2], d[2]);
  // x weight of this thread's slab only (the expressions of weights_of for offset `slab`)
  const float ao = slab == 0 ? 1.5f - fx : (slab == 1 ? fx - 1.0f : fx - 0.5f);
  const float wa = slab == 1 ? 0.75f - ao * ao : 0.5f * (ao * ao);
  const float da = (fx - (float)slab) * -dx;
  float u[3];
#pragma unroll
  for (int rr = 0; rr < 3; ++rr) u[rr] = __fmaf_rn(A[3 * rr + 0], da, q[rr]);
  const float2 a14 = make_float2(A[1], A[4]), a70 = make_float2(A[7], 0.0f);
  const float2 a25 = make_float2(A[2], A[5]), a80 = make_float2(A[8], 0.0f);
  const float2 u01 = make_float2(u[0], u[1]), u2m = make_float2(u[2], m);
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    const float wab = __fmul_rn(wa, w[1][b]);
    const float2 db = make_float2(d[1][b], d[1][b]);
    const float2 ub01 = __ffma2_rn(a14, db, u01);  // (q_x + .. + A_01 d_b, q_y + .. + A_11 d_b)
    const float2 ub2m = __ffma2_rn(a70, db, u2m);  // (q_z + .. + A_21 d_b, m)
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
      const float2 dc = make_float2(d[2][cc], d[2][cc]);
      const float2 ww = __fmul2_rn(make_float2(wab, wab), make_float2(w[2][cc], w[2][cc]));
      acc[b][cc][0] = __ffma2_rn(ww, __ffma2_rn(a25, dc, ub01), acc[b][cc][0]);
      acc[b][cc][1] = __ffma2_rn(ww, __ffma2_rn(a80, dc, ub2m), acc[b][cc][1]);
    }
  }
}

// Staged P2G: asynchronous copies (cp.async, 4 bytes each) of the state components of chunk
// [c0, c0 + cn) of a tile into raw[P2G_RAW][CHUNK], particle i of the chunk copied by thread
// i % P2G_THREADS, which is the thread that reads it back in phase 1.  The caller commits.
template <int CHUNK>
__device__ __forceinline__ void p2g_stage(float* __restrict__ raw, const float* __restrict__ cur,
                                          const uint32_t* __restrict__ perm, int64_t cap, uint32_t c0, uint32_t cn) {
  constexpr int PER = (CHUNK + P2G_THREADS - 1) / P2G_THREADS;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const uint32_t i = threadIdx.x + q * P2G_THREADS;
    if (i < cn) {
      const int64_t src = perm[c0 + i];
#pragma unroll
      for (int r = 0; r < P2G_RAW; ++r) cp_async4(raw + r * CHUNK + i, cur + (int64_t)p2g_raw_comp(r) * cap + src);
    }
  }
}
// the first chunk of the occupied tile of tile-list record `rec`
template <int CHUNK>
__device__ __forceinline__ void p2g_stage_tile(float* __restrict__ raw, const uint4 rec,
                                               const Control* __restrict__ ctrl, const float* __restrict__ st0,
                                               const float* __restrict__ st1, int64_t cap,
                                               const uint32_t* __restrict__ perm) {
  p2g_stage<CHUNK>(raw, ctrl[rec.y].parity ? st1 : st0, perm, cap, rec.z, min((uint32_t)CHUNK, rec.w - rec.z));
}

// one tile of k_p2g, chunks of CHUNK particles.  STAGED: the particle state of each chunk
// arrives by the asynchronous copies of p2g_stage, issued one chunk ahead: the tile's first
// chunk by the caller (or the previous tile), each later chunk, and after the last one the
// first chunk of the next tile (next: its tile-list record, or null), right after the thread has
// read its copies of the current chunk, so that the copies fly while the CTA scatters.
template <int CHUNK, bool STAGED>
__device__ __forceinline__ void p2g_tile(const uint4 trec, const InstDesc* __restrict__ desc,
                                         const Control* __restrict__ ctrl, const float* __restrict__ st0,
                                         const float* __restrict__ st1, int64_t cap,
                                         const uint32_t* __restrict__ start, const uint32_t* __restrict__ perm,
                                         long long* __restrict__ acc, int64_t node_total,
                                         uint32_t* __restrict__ blk_epoch, int transport_only,
                                         const uint4* __restrict__ next) {
  constexpr int P2G_PER_THREAD = (CHUNK + P2G_THREADS - 1) / P2G_THREADS;  // phase-1 particles per thread
  static_assert(CHUNK % 32 == 0, "record rows rotate within 32-word segments");
  extern __shared__ float4 part[];  // particle records during the chunks, then TB * 27 partial node sums
  float* rec = reinterpret_cast<float*>(part);  // [P2G_REC][CHUNK]
  // STAGED: the raw copies sit after the records / partials region
  float* raw = reinterpret_cast<float*>(reinterpret_cast<char*>(part) + p2g_smem(CHUNK));
  __shared__ long long red[(P2G_THREADS / 32) * 8 + 8];

  const int tile = (int)trec.x, inst = (int)trec.y;
  const Control& c = ctrl[inst];
  const InstDesc& D = desc[inst];
  const int64_t ltile = tile - D.tile_off;
  const int64_t key0 = D.key_off + ltile * TB;
  const uint32_t ts = trec.z, te = trec.w;
  if (!c.active || ts == te) {  // inactive instance or empty tile (uniform across the CTA)
    if constexpr (STAGED) {      // the tile list holds neither, but keep the staging chain whole
      cp_async_wait<0>();        // this tile's copies land before the next tile's reuse the buffer
      if (next) p2g_stage_tile<CHUNK>(raw, *next, ctrl, st0, st1, cap, perm);
      cp_async_commit();
    }
    return;
  }

  const int tz = (int)(ltile % D.tiles[2]);
  const int ty = (int)((ltile / D.tiles[2]) % D.tiles[1]);
  const int tx = (int)(ltile / ((int64_t)D.tiles[2] * D.tiles[1]));
  const int t = threadIdx.x;
  const int bin = t / 3, slab = t % 3;

  const float* cur = c.parity ? st1 : st0;
  const float dx = (float)D.dx;
  // the energy audit's transport pass deposits APIC momentum only (audit.rs:381-398)
  const float stress_scale = transport_only ? 0.0f : (float)(c.dt * 4.0 / (D.dx * D.dx));
  const double s_m = D.s_mass, s_p = c.s_mom;

  float2 acc9[3][3][2];  // per node (b, c) of the slab: (p_x, p_y), (p_z, m)
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
      for (int k = 0; k < 2; ++k) acc9[b][q][k] = make_float2(0.0f, 0.0f);
  // this thread's particle totals (mass, momentum, fixed point), kept in shared memory between the
  // chunks' load phases so that they hold no registers during the scatter
  __shared__ long long tot_s[4 * P2G_THREADS];
  volatile long long* tot = tot_s + threadIdx.x;
#pragma unroll
  for (int k = 0; k < 4; ++k) tot[k * P2G_THREADS] = 0;

  const uint32_t s = start[key0 + bin], e = start[key0 + bin + 1];  // this bin's sorted range
  for (uint32_t c0 = ts; c0 < te; c0 += CHUNK) {
    const uint32_t cn = min((uint32_t)CHUNK, te - c0);
    if (c0 != ts) __syncthreads();  // the previous chunk's records are consumed
    // phase 1: one thread per particle.  The thread's permutation entries of the chunk are loaded
    // first, so that each particle's state loads issue without waiting for its entry.
    uint32_t srcs[P2G_PER_THREAD];
    if constexpr (STAGED) {
      cp_async_wait<0>();  // this thread's copies of the chunk have landed
    } else {
#pragma unroll
      for (int q = 0; q < P2G_PER_THREAD; ++q)
        srcs[q] = t + q * P2G_THREADS < cn ? perm[c0 + t + q * P2G_THREADS] : 0u;
    }
#pragma unroll
    for (int q = 0; q < P2G_PER_THREAD; ++q) {
      const uint32_t i = t + q * P2G_THREADS;
      if (i >= cn) break;
      float x[3], v[3], Cm[9], tau[6], m, v0;
      if constexpr (STAGED) {
        const float* in = raw + i;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          x[a] = in[a * CHUNK];
          v[a] = in[(3 + a) * CHUNK];
        }
#pragma unroll
        for (int a = 0; a < 9; ++a) Cm[a] = in[(6 + a) * CHUNK];
#pragma unroll
        for (int a = 0; a < 6; ++a) tau[a] = in[(15 + a) * CHUNK];
        m = in[21 * CHUNK];
        v0 = in[22 * CHUNK];
      } else {
        const int64_t src = srcs[q];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          x[a] = cur[(C_X + a) * cap + src];
          v[a] = cur[(C_V + a) * cap + src];
        }
#pragma unroll
        for (int a = 0; a < 9; ++a) Cm[a] = cur[(C_C + a) * cap + src];
#pragma unroll
        for (int a = 0; a < 6; ++a) tau[a] = cur[(C_TAU + a) * cap + src];
        m = cur[C_M * cap + src];
        v0 = cur[C_V0 * cap + src];
      }
      float qv[3], A[9];
      p2g_record(v, Cm, tau, m, stress_scale * v0, qv, A);
      float* r = rec + rec_slot(i);
      r[0] = m;
#pragma unroll
      for (int a = 0; a < 3; ++a) r[(1 + a) * CHUNK] = qv[a];
#pragma unroll
      for (int a = 0; a < 9; ++a) r[(4 + a) * CHUNK] = A[a];
#pragma unroll
      for (int a = 0; a < 3; ++a) r[(13 + a) * CHUNK] = p2g_frac(x[a], dx, D.pow2_inv_dx);
      // exact per-particle totals: FP64 products of the stored FP32 mass and velocity
      tot[0] = tot[0] + to_fixed((double)m, s_m);
      tot[P2G_THREADS] = tot[P2G_THREADS] + to_fixed((double)m * (double)v[0], s_p);
      tot[2 * P2G_THREADS] = tot[2 * P2G_THREADS] + to_fixed((double)m * (double)v[1], s_p);
      tot[3 * P2G_THREADS] = tot[3 * P2G_THREADS] + to_fixed((double)m * (double)v[2], s_p);
    }
    if constexpr (STAGED) {
      // this thread has read its copies: the next chunk (of this tile or of the next) may land
      if (c0 + CHUNK < te) p2g_stage<CHUNK>(raw, cur, perm, cap, c0 + CHUNK, min((uint32_t)CHUNK, te - c0 - CHUNK));
      else if (next)
        p2g_stage_tile<CHUNK>(raw, *next, ctrl, st0, st1, cap, perm);
      cp_async_commit();
    }
    __syncthreads();
    // phase 2: this bin's particles inside the chunk, in sorted order
    const uint32_t j0 = max(s, c0), j1 = min(e, c0 + cn);
    for (uint32_t j = j0; j < j1; ++j) {
      const float* r = rec + rec_slot(j - c0);
      const float q[3] = {r[CHUNK], r[2 * CHUNK], r[3 * CHUNK]};
      float A[9];
#pragma unroll
      for (int a = 0; a < 9; ++a) A[a] = r[(4 + a) * CHUNK];
      p2g_scatter(r[0], q, A, r[13 * CHUNK], r[14 * CHUNK], r[15 * CHUNK], slab, dx, acc9);
    }
  }
  __syncthreads();  // the last chunk's records (aliasing part[]) are consumed
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
      part[bin * 27 + slab * 9 + b * 3 + cc] =
          make_float4(acc9[b][cc][1].y, acc9[b][cc][0].x, acc9[b][cc][0].y, acc9[b][cc][1].x);
  __syncthreads();
  // one thread per halo node: sum the 27 contributing (bin, slab) partials in a fixed order
  long long nv[4] = {0, 0, 0, 0};
  int hx = 0, hy = 0, hz = 0;
  const bool has_node = t < HN;
  if (has_node) {
    hz = t % HZ;
    hy = (t / HZ) % HY;
    hx = t / (HZ * HY);
    float2 s01 = make_float2(0.f, 0.f), s23 = make_float2(0.f, 0.f);  // (mass, p_x), (p_y, p_z)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int lbx = hx - a;
      if (lbx < 0 || lbx >= TX) continue;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const int lby = hy - b;
        if (lby < 0 || lby >= TY) continue;
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const int lbz = hz - cc;
          if (lbz < 0 || lbz >= TZ) continue;
          const float4 q = part[((lbx * TY + lby) * TZ + lbz) * 27 + a * 9 + b * 3 + cc];
          s01 = __fadd2_rn(s01, make_float2(q.x, q.y));
          s23 = __fadd2_rn(s23, make_float2(q.z, q.w));
        }
      }
    }
    nv[0] = to_fixed((double)s01.x, s_m);
    nv[1] = to_fixed((double)s01.y, s_p);
    nv[2] = to_fixed((double)s23.x, s_p);
    nv[3] = to_fixed((double)s23.y, s_p);
  }
  // Exact conservation per tile.  The tile's particle totals (tot, exact int64) minus its halo's
  // node sums (nv) is the FP32 rounding discrepancy D of each component.  It is spread over the
  // halo nodes in proportion to node mass by a telescoping rule: with P the inclusive prefix sum
  // of the node masses in thread order and M their total, the node of thread i receives
  // f(P_i) - f(P_i - m_i), f(P) = floor(D (P / M)) in FP64.  The shares sum to f(M) - f(0) = D
  // exactly and each has the sign of D.  Integer sums do not depend on their order, so the warp
  // sums may take any route; the prefix is taken in thread order.  Two barriers.
  constexpr int NW = P2G_THREADS / 32;
  const int lane = t & 31, w = t >> 5;
  long long dif[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) dif[k] = warp_sum_ll_redux(tot[k * P2G_THREADS] - nv[k]);
  long long pin = nv[0];  // inclusive warp prefix of node masses
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, pin, o);
    if (lane >= o) pin += y;
  }
  if (lane == 31) red[w] = pin;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) red[NW + 4 * w + k] = dif[k];
  __syncthreads();
  if (w == 0) {
    const long long wm = lane < NW ? red[lane] : 0;
    long long incl = wm;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    long long dd[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) dd[k] = warp_sum_ll_redux(lane < NW ? red[NW + 4 * lane + k] : 0);
    const long long mtot = __shfl_sync(0xffffffffu, incl, NW - 1);
    if (lane < NW) red[5 * NW + lane] = incl - wm;  // node mass before warp `lane`
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < 4; ++k) red[6 * NW + k] = dd[k];
      red[6 * NW + 4] = mtot;
    }
  }
  __syncthreads();
  static_assert(6 * NW + 5 <= NW * 8 + 8, "the conservation scratch fits red");
  const long long Dk[4] = {red[6 * NW + 0], red[6 * NW + 1], red[6 * NW + 2], red[6 * NW + 3]};
  if (has_node && (Dk[0] | Dk[1] | Dk[2] | Dk[3]) != 0) {
    const long long mtot = red[6 * NW + 4];
    if (mtot > 0) {
      const long long p1 = red[5 * NW + w] + pin, p0 = p1 - nv[0];
      // f(P) = floor(D r(P)) with r(P) = P / M as a product with 1 / M, exactly 1 at P = M: r stays
      // monotone with r(0) = 0 and r(M) = 1, so the shares still telescope to D
      const double inv = 1.0 / (double)mtot;
      const double r1 = p1 >= mtot ? 1.0 : (double)p1 * inv, r0 = p0 >= mtot ? 1.0 : (double)p0 * inv;
#pragma unroll
      for (int k = 0; k < 4; ++k) nv[k] += __double2ll_rd((double)Dk[k] * r1) - __double2ll_rd((double)Dk[k] * r0);
    } else if (t == 0) {  // no node mass to weigh by: the tile's first halo node takes it all
#pragma unroll
      for (int k = 0; k < 4; ++k) nv[k] += Dk[k];
    }
  }
  // flush to the global grid
  if (has_node && (nv[0] | nv[1] | nv[2] | nv[3]) != 0) {
    const int nx = tx * TX + hx, ny = ty * TY + hy, nz = tz * TZ + hz;
    if (nx < D.nodes[0] && ny < D.nodes[1] && nz < D.nodes[2]) {
      const int64_t g = node_index(D, nx, ny, nz);
      // the node's block takes part in this attempt's grid update
      blk_epoch[D.blk_off + ((int64_t)(nx / NB) * D.nblk[1] + ny / NB) * D.nblk[2] + nz / NB] = (uint32_t)c.epoch;
      atomic_add_ll(acc + g, nv[0]);
      atomic_add_ll(acc + node_total + g, nv[1]);
      atomic_add_ll(acc + 2 * node_total + g, nv[2]);
      atomic_add_ll(acc + 3 * node_total + g, nv[3]);
    }
  }
}

// Persistent CTAs (as many as the launch shape asks, at most as many as fit the GPU at once)
// walk the attempt's list of occupied tiles.
// STAGED: each tile's next tile is known before the tile starts (two cursor slots, used
// alternately, so that the slot a CTA reads is not rewritten before every thread has read it),
// and the first chunk of the next tile is copied while the current tile scatters.
template <int CHUNK, bool STAGED>
__global__ void __launch_bounds__(P2G_THREADS, 2)
    k_p2g(const InstDesc* __restrict__ desc, const Control* __restrict__ ctrl, const float* __restrict__ st0, const float* __restrict__ st1, int64_t cap,
          const uint32_t* __restrict__ start, const uint32_t* __restrict__ perm, long long* __restrict__ acc,
          int64_t node_total, uint32_t* __restrict__ blk_epoch, int transport_only,
          const uint4* __restrict__ tile_rec, const uint32_t* __restrict__ tile_count, uint32_t* cursor) {
  const uint32_t n = *tile_count;
  if constexpr (!STAGED) {
    __shared__ uint32_t slot;
    for (uint32_t i = tile_first(cursor, &slot); i < n; i = tile_next(cursor, i, &slot)) {
      p2g_tile<CHUNK, false>(tile_rec[i], desc, ctrl, st0, st1, cap, start, perm, acc, node_total, blk_epoch,
                             transport_only, nullptr);
      __syncthreads();  // the next tile reuses the shared memory
    }
  } else {
    __shared__ uint32_t slots[2];
    extern __shared__ float4 part[];
    float* raw = reinterpret_cast<float*>(reinterpret_cast<char*>(part) + p2g_smem(CHUNK));
    int which = 0;
    uint32_t i = tile_first(cursor, &slots[0]);
    if (i < n) p2g_stage_tile<CHUNK>(raw, tile_rec[i], ctrl, st0, st1, cap, perm);
    cp_async_commit();
    while (i < n) {
      which ^= 1;
      const uint32_t nx = tile_next(cursor, i, &slots[which]);
      p2g_tile<CHUNK, true>(tile_rec[i], desc, ctrl, st0, st1, cap, start, perm, acc, node_total, blk_epoch,
                            transport_only, nx < n ? tile_rec + nx : nullptr);
      __syncthreads();  // the next tile reuses the shared memory
      i = nx;
    }
    cp_async_wait<0>();  // no copy may land after the CTA's shared memory is released
  }
}

// ============================================================== wall traction
__device__ __forceinline__ void traction_particle(const InstDesc* __restrict__ desc,
                                                  const Control* __restrict__ ctrl,
                                                  const int* __restrict__ pcta_inst, const float* __restrict__ st0,
                                                  const float* __restrict__ st1, int64_t cap, int64_t slot, int row,
                                                  const long long* __restrict__ acc, long long* __restrict__ trac,
                                                  int64_t node_total);
// Nine threads per particle within half a cell of a face (listed while binning): thread `row`
// of a particle takes the stencil row (a, b) = (row / 3, row % 3) of each face image, three
// nodes, and issues the node loads of all three before it tests any of them.  A particle's 27
// node reads thus overlap instead of running as one thread's chain of dependent loads.  The
// reactions are int64 sums, so the split changes no result.
constexpr int TRACTION_ROWS = 9, TRACTION_THREADS = 128, TRACTION_CTAS_PER_SM = 6;  // one wave at 78 registers
__global__ void __launch_bounds__(TRACTION_THREADS)
    k_traction(const InstDesc* __restrict__ desc, const Control* __restrict__ ctrl,
               const int* __restrict__ pcta_inst, const float* __restrict__ st0,
               const float* __restrict__ st1, int64_t cap, const uint32_t* __restrict__ nw_list,
               const uint32_t* __restrict__ nw_count, const long long* __restrict__ acc,
               long long* __restrict__ trac, int64_t node_total) {
  const uint64_t work = (uint64_t)*nw_count * TRACTION_ROWS;
  for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < work; g += (uint64_t)gridDim.x * blockDim.x)
    traction_particle(desc, ctrl, pcta_inst, st0, st1, cap, nw_list[g / TRACTION_ROWS], (int)(g % TRACTION_ROWS), acc,
                      trac, node_total);
}

__device__ __forceinline__ void traction_particle(const InstDesc* __restrict__ desc,
                                                  const Control* __restrict__ ctrl,
                                                  const int* __restrict__ pcta_inst, const float* __restrict__ st0,
                                                  const float* __restrict__ st1, int64_t cap, int64_t slot, int row,
                                                  const long long* __restrict__ acc, long long* __restrict__ trac,
                                                  int64_t node_total) {
  const int inst = pcta_inst[slot / G2P_THREADS];
  const Control& c = ctrl[inst];
  if (!c.active) return;
  const InstDesc& D = desc[inst];
  const float* cur = c.parity ? st1 : st0;
  const float dx = (float)D.dx;
  const float dt = (float)c.dt;
  const float half = 0.5f * dx;
  const float force_scale = (float)(-c.dt * 4.0 / (D.dx * D.dx));
  const float m = cur[C_M * cap + slot], v0 = cur[C_V0 * cap + slot];
  float x[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) x[a] = cur[(C_X + a) * cap + slot];
  const double s_m = D.s_mass, s_p = c.s_mom;
  // unrolled axis and node loops: the stencil arrays stay in registers (no stack frame)
#pragma unroll
  for (int axis = 0; axis < 3; ++axis) {
    const float ext = (float)D.extent[axis];
    float face;
    if (x[axis] < half) face = 0.0f;
    else if (x[axis] > ext - half) face = ext;
    else continue;
    float img[3] = {x[0], x[1], x[2]};
    img[axis] = 2.0f * face - x[axis];
    int base[3];
    float w[3][3], d[3][3];
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float sc = scaled_of(img[a], dx, D.pow2_inv_dx);
      const float bf = floorf(sc - 0.5f);
      const float padded = bf + 1.0f;
      if (!(padded >= 0.0f) || padded + 2.0f >= (float)D.nodes[a]) ok = false;
      base[a] = (int)padded;
      weights_of(sc - bf, dx, w[a], d[a]);
    }
    if (!ok) continue;
    const int plane = face == 0.0f ? 1 : D.cells[axis] + 1;
    const float inward = face == 0.0f ? 1.0f : -1.0f;
    const float gax = (float)D.gravity[axis];
    const float tau_aa = cur[(C_TAU + axis) * cap + slot];
    const float ns = tau_aa * v0 - m * gax * (img[axis] - x[axis]);
    if (ns >= 0.0f) continue;
    const float wm = m * gax * dt;
    long long* dst = trac + (int64_t)(axis + (inward > 0.f ? 0 : 3)) * node_total;
    // this thread's row (a, b): the three nodes' loads first, then their tests
    const int a = row / 3, b = row % 3;
    const int c0 = base[0] + a, c1 = base[1] + b;
    const float wab = (a == 0 ? w[0][0] : (a == 1 ? w[0][1] : w[0][2])) * (b == 0 ? w[1][0] : (b == 1 ? w[1][1] : w[1][2]));
    long long pmf[3], pmo[3], tmf[3];
    int64_t tix[3];
    bool use[3];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
      const int c2 = base[2] + cc;
      const int ca = axis == 0 ? c0 : (axis == 1 ? c1 : c2);
      use[cc] = !(ca <= 1 || ca > D.cells[axis]) && wab * w[2][cc] != 0.0f;
      const int64_t pi = node_index(D, axis == 0 ? plane : c0, axis == 1 ? plane : c1, axis == 2 ? plane : c2);
      tix[cc] = node_index(D, c0, c1, c2);
      pmf[cc] = use[cc] ? acc[pi] : 0;
      pmo[cc] = use[cc] ? acc[(1 + axis) * node_total + pi] : 0;
      tmf[cc] = use[cc] ? acc[tix[cc]] : 0;
    }
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
      if (!use[cc] || pmf[cc] <= 0) continue;
      const float wt = wab * w[2][cc];
      const float pm = (float)((double)pmf[cc] / s_m);
      const float pp = (float)((double)pmo[cc] / s_p);
      const float trial = pp / pm + gax * dt;
      if (trial * inward >= 0.0f) continue;
      const int o = axis == 0 ? a : (axis == 1 ? b : cc);
      const float dist = axis == 0 ? (o == 0 ? d[0][0] : (o == 1 ? d[0][1] : d[0][2]))
                                   : (axis == 1 ? (o == 0 ? d[1][0] : (o == 1 ? d[1][1] : d[1][2])) : d[2][cc]);
      const float reaction = (ns * dist * force_scale + wm) * wt * inward;
      if (!(reaction > 0.0f)) continue;
      if (tmf[cc] <= 0) continue;
      atomic_add_ll(dst + tix[cc], to_fixed((double)reaction, s_p));
    }
  }
}

// ============================================================== grid update
__device__ __forceinline__ void reduce_tangential(float t[3], float reduction) {
  if (reduction == 0.0f) return;
  const float speed = sqrtf(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  if (speed <= reduction) {
    t[0] = t[1] = t[2] = 0.0f;
  } else {
    const float f = (speed - reduction) / speed;
    t[0] *= f;
    t[1] *= f;
    t[2] *= f;
  }
}

// AUDIT (energy audit, audit.rs:72-90): each CTA also sums the grid kinetic energy after the
// stress deposit, after wall traction, with the gravity kick, and after the wall projection and
// friction, into audit[4 * CTA + 0..3].
// Registers for 4 CTAs per SM (64): the update waits on its node loads, so resident warps count
// more than registers; the FP64 tallies live in shared memory and the next live pass's sums are
// loaded while the current pass works (0.168 -> 0.112 ms on the 16.8M-particle slump against
// 2 CTAs per SM at 84 registers, one pass in flight).
template <bool AUDIT>
__global__ void __launch_bounds__(GU_THREADS, 4)
    k_grid_update(const InstDesc* __restrict__ desc, const Control* __restrict__ ctrl,
                  const int* __restrict__ gcta_inst, long long* __restrict__ acc, long long* __restrict__ trac,
                  int64_t node_total, const uint32_t* __restrict__ blk_epoch, float4* __restrict__ vel,
                  GridPartial* __restrict__ part, double* __restrict__ audit) {
  constexpr int RK = AUDIT ? 11 : 7;
  __shared__ double shd[(GU_THREADS / 32) * RK + RK];
  const int inst = gcta_inst[blockIdx.x];
  const Control& c = ctrl[inst];
  if (!c.active) return;
  const InstDesc& D = desc[inst];
  const int t = threadIdx.x;
  const int64_t nblk = (int64_t)D.nblk[0] * D.nblk[1] * D.nblk[2];
  // this thread's FP64 tallies, kept in shared memory (volatile accesses) so that they hold no
  // registers while the node loads are in flight
  constexpr int NTAL = AUDIT ? 10 : 6;
  __shared__ double tally[10 * GU_THREADS];  // the audit tallies have their own rows in both forms
  volatile double& wi0 = tally[0 * GU_THREADS + t];
  volatile double& wi1 = tally[1 * GU_THREADS + t];
  volatile double& wi2 = tally[2 * GU_THREADS + t];
  volatile double& proj = tally[3 * GU_THREADS + t];
  volatile double& fric = tally[4 * GU_THREADS + t];
  volatile double& tren = tally[5 * GU_THREADS + t];
  volatile double& e_stress = tally[6 * GU_THREADS + t];
  volatile double& e_trac = tally[7 * GU_THREADS + t];
  volatile double& e_grav = tally[8 * GU_THREADS + t];
  volatile double& e_walls = tally[9 * GU_THREADS + t];
#pragma unroll
  for (int k = 0; k < NTAL; ++k) tally[k * GU_THREADS + t] = 0.0;
  int fail = F_OK;
  // GU_PASSES passes of GU_BLOCKS_PER_CTA node blocks each.  The activity marks of all the
  // passes are read up front (independent loads, one latency), and a pass whose block holds no
  // mass in this attempt is skipped by its two warps alone: most CTAs of a sparse grid find no
  // live block and leave after one round trip instead of one per pass.
  const int64_t lblk0 = ((int64_t)(blockIdx.x - D.gcta_off) * GU_PASSES) * GU_BLOCKS_PER_CTA + t / 64;
  uint32_t live_mask = 0;
#pragma unroll
  for (int pass = 0; pass < GU_PASSES; ++pass) {
    const int64_t lblk = lblk0 + (int64_t)pass * GU_BLOCKS_PER_CTA;
    if (lblk < nblk && blk_epoch[D.blk_off + lblk] == (uint32_t)c.epoch) live_mask |= 1u << pass;
  }
  const bool any_live = __syncthreads_or(live_mask != 0u) != 0;  // CTA-uniform
  // The live passes run in order; each prefetches the next live pass's four sums while it works.
  // Every node belongs to one thread and one pass, so the prefetch never reads a node that this
  // kernel has already written.
  const int l64 = t % 64;
  auto node_of = [&](int pass, int& ni, int& nj, int& nk, int64_t& g) -> bool {
    const int64_t lblk = lblk0 + (int64_t)pass * GU_BLOCKS_PER_CTA;
    const int bk = (int)(lblk % D.nblk[2]), bj = (int)((lblk / D.nblk[2]) % D.nblk[1]),
              bi = (int)(lblk / ((int64_t)D.nblk[2] * D.nblk[1]));
    ni = bi * NB + l64 / 16;
    nj = bj * NB + (l64 / 4) % 4;
    nk = bk * NB + l64 % 4;
    const bool in = ni < D.nodes[0] && nj < D.nodes[1] && nk < D.nodes[2];
    g = in ? node_index(D, ni, nj, nk) : 0;
    return in;
  };
  int pass = live_mask ? __ffs(live_mask) - 1 : GU_PASSES;
  long long q0 = 0, q1 = 0, q2 = 0, q3 = 0;
  int64_t qg = 0;
  bool ql = false;
  if (pass < GU_PASSES) {
    int qi, qj, qk;
    ql = node_of(pass, qi, qj, qk, qg);
    if (ql) {
      q0 = acc[qg];
      q1 = acc[node_total + qg];
      q2 = acc[2 * node_total + qg];
      q3 = acc[3 * node_total + qg];
    }
  }
  while (pass < GU_PASSES) {
    const bool live = ql;
    const int this_pass = pass;
    const int64_t g = qg;
    const long long mf = q0, pf0 = q1, pf1 = q2, pf2 = q3;
    const uint32_t rest = live_mask & ~((2u << pass) - 1u);
    pass = rest ? __ffs(rest) - 1 : GU_PASSES;
    if (pass < GU_PASSES) {
      int qi, qj, qk;
      ql = node_of(pass, qi, qj, qk, qg);
      if (ql) {
        q0 = acc[qg];
        q1 = acc[node_total + qg];
        q2 = acc[2 * node_total + qg];
        q3 = acc[3 * node_total + qg];
      }
    }
    if (live) {
      int ni, nj, nk;
      int64_t g_unused;
      node_of(this_pass, ni, nj, nk, g_unused);
      if (mf <= 0) {
        vel[g] = make_float4(0.f, 0.f, 0.f, 0.f);
        acc[g] = 0;
        acc[node_total + g] = 0;
        acc[2 * node_total + g] = 0;
        acc[3 * node_total + g] = 0;
      } else {
        const double s_m = D.s_mass, s_p = c.s_mom;
        const double md = (double)mf / s_m;
        double p[3] = {(double)pf0 / s_p, (double)pf1 / s_p, (double)pf2 / s_p};
        acc[g] = 0;
        acc[node_total + g] = 0;
        acc[2 * node_total + g] = 0;
        acc[3 * node_total + g] = 0;
        if (AUDIT) e_stress += 0.5 * (p[0] * p[0] + p[1] * p[1] + p[2] * p[2]) / md;
        const int co[3] = {ni, nj, nk};
        float Tl[3] = {0.f, 0.f, 0.f}, Th[3] = {0.f, 0.f, 0.f};
        bool shell = false;
  #pragma unroll
        for (int a = 0; a < 3; ++a)
          if (co[a] == 2 || co[a] == 3 || co[a] == D.cells[a] - 1 || co[a] == D.cells[a]) shell = true;
        if (shell) {
  #pragma unroll
          for (int a = 0; a < 3; ++a) {
            const long long l = trac[(int64_t)a * node_total + g], h = trac[(int64_t)(a + 3) * node_total + g];
            if (l | h) {
              trac[(int64_t)a * node_total + g] = 0;
              trac[(int64_t)(a + 3) * node_total + g] = 0;
              const double dl = (double)l / s_p, dh = (double)h / s_p;
              const double S = dl - dh;
              // telescoped kinetic-energy jump of the reaction deposits (grid.rs:279-295)
              tren += S * (p[a] / md + S / (2.0 * md));
              if (a == 0) wi0 += S;
              if (a == 1) wi1 += S;
              if (a == 2) wi2 += S;
              p[a] += S;
              Tl[a] = (float)dl;
              Th[a] = (float)dh;
            }
          }
        }
        if (AUDIT) {
          e_trac += 0.5 * (p[0] * p[0] + p[1] * p[1] + p[2] * p[2]) / md;
          double k2 = 0.0;
          for (int a = 0; a < 3; ++a) {
            const double u = p[a] / md + D.gravity[a] * c.dt;
            k2 += u * u;
          }
          e_grav += 0.5 * md * k2;
        }
        const float m = (float)md;
        const float dt = (float)c.dt;
        float v[3];
  #pragma unroll
        for (int a = 0; a < 3; ++a) v[a] = (float)p[a] / m + (float)D.gravity[a] * dt;
        if (!(isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]))) {
          fail = F_GRID_NONFINITE;
          vel[g] = make_float4(0.f, 0.f, 0.f, m);
        } else {
          const float before[3] = {v[0], v[1], v[2]};
  #pragma unroll
          for (int a = 0; a < 3; ++a) {
            float sign = 0.0f;
            if (co[a] <= 1) sign = 1.0f;
            else if (co[a] > D.cells[a]) sign = -1.0f;
            if (sign == 0.0f) continue;
            const float nsp = v[a] * sign;
            if (nsp >= 0.0f) continue;
            proj -= 0.5 * (double)m * (double)nsp * (double)nsp;
            v[a] = 0.0f;
            const float t0 = v[0], t1 = v[1], t2 = v[2];
            const int face = 2 * a + (sign > 0.f ? 0 : 1);
            if (D.face_mode && D.face_sticky[face]) {
              v[0] = v[1] = v[2] = 0.0f;
            } else {
              const float mu = D.face_mode ? (float)D.face_mu[face] : (float)D.friction;
              reduce_tangential(v, mu * (-nsp));
            }
            fric += 0.5 * (double)m *
                    ((double)(t0 * t0 + t1 * t1 + t2 * t2) - (double)(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
          }
  #pragma unroll
          for (int a = 0; a < 3; ++a) {
            const float R = Tl[a] + Th[a];
            if (!(R > 0.0f)) continue;
            const float normal = v[a];
            float tg[3] = {v[0], v[1], v[2]};
            tg[a] = 0.0f;
            const double t2b = (double)(tg[0] * tg[0] + tg[1] * tg[1] + tg[2] * tg[2]);
            if (D.face_mode) {
              const bool stick = (Tl[a] > 0.f && D.face_sticky[2 * a]) || (Th[a] > 0.f && D.face_sticky[2 * a + 1]);
              if (stick) tg[0] = tg[1] = tg[2] = 0.0f;
              else reduce_tangential(tg, ((float)D.face_mu[2 * a] * Tl[a] + (float)D.face_mu[2 * a + 1] * Th[a]) / m);
            } else {
              reduce_tangential(tg, (float)D.friction * R / m);
            }
            fric += 0.5 * (double)m * (t2b - (double)(tg[0] * tg[0] + tg[1] * tg[1] + tg[2] * tg[2]));
            v[0] = tg[0];
            v[1] = tg[1];
            v[2] = tg[2];
            v[a] = normal;
          }
          wi0 += (double)(v[0] - before[0]) * (double)m;
          wi1 += (double)(v[1] - before[1]) * (double)m;
          wi2 += (double)(v[2] - before[2]) * (double)m;
          vel[g] = make_float4(v[0], v[1], v[2], m);
          if (AUDIT)
            e_walls += 0.5 * (double)m * ((double)v[0] * v[0] + (double)v[1] * v[1] + (double)v[2] * v[2]);
        }
      }
    }
  }
  if (!any_live) {  // CTA-uniform
    if (t == 0) {
      GridPartial& P = part[blockIdx.x];
      P.wall_impulse[0] = P.wall_impulse[1] = P.wall_impulse[2] = 0.0;
      P.proj = P.fric = P.trac = 0.0;
      P.fail = F_OK;
      if (AUDIT)
        for (int k = 0; k < 4; ++k) audit[4 * (int64_t)blockIdx.x + k] = 0.0;
    }
    return;
  }
  double rv[RK];
  rv[0] = wi0;
  rv[1] = wi1;
  rv[2] = wi2;
  rv[3] = proj;
  rv[4] = fric;
  rv[5] = tren;
  rv[6] = (double)fail;
  if (AUDIT) {
    rv[RK - 4] = e_stress;
    rv[RK - 3] = e_trac;
    rv[RK - 2] = e_grav;
    rv[RK - 1] = e_walls;
  }
  block_reduce_multi_to0<GU_THREADS, RK>(rv, 1u << 6, shd);  // kernel end: thread 0 writes
  if (t == 0) {
    GridPartial& P = part[blockIdx.x];
    P.wall_impulse[0] = rv[0];
    P.wall_impulse[1] = rv[1];
    P.wall_impulse[2] = rv[2];
    P.proj = rv[3];
    P.fric = rv[4];
    P.trac = rv[5];
    P.fail = (int)rv[6];
    if (AUDIT)
      for (int k = 0; k < 4; ++k) audit[4 * (int64_t)blockIdx.x + k] = rv[RK - 4 + k];
  }
}

// Energy audit: grid kinetic energy of the nodes that hold mass in this attempt, one partial per
// grid-update CTA (audit.rs:360-378 grid_kinetic).  from_acc: from the deposited momentum of the
// transport pass, clearing the accumulators as the grid update does; otherwise from the node
// velocities and masses of vel[].
__global__ void __launch_bounds__(GU_THREADS)
    k_audit_kinetic(const InstDesc* __restrict__ desc, const Control* __restrict__ ctrl,
                    const int* __restrict__ gcta_inst, long long* __restrict__ acc, const float4* __restrict__ vel,
                    int64_t node_total, const uint32_t* __restrict__ blk_epoch, int from_acc,
                    double* __restrict__ out) {
  __shared__ double shd[(GU_THREADS / 32) + 1];
  const int inst = gcta_inst[blockIdx.x];
  const Control& c = ctrl[inst];
  const InstDesc& D = desc[inst];
  const int t = threadIdx.x;
  double e = 0.0;
  const int64_t nblk = (int64_t)D.nblk[0] * D.nblk[1] * D.nblk[2];
  for (int pass = 0; pass < GU_PASSES; ++pass) {
    const int64_t lblk = ((blockIdx.x - D.gcta_off) * GU_PASSES + pass) * GU_BLOCKS_PER_CTA + t / 64;
    if (c.active && lblk < nblk && blk_epoch[D.blk_off + lblk] == (uint32_t)c.epoch) {
      const int bk = (int)(lblk % D.nblk[2]), bj = (int)((lblk / D.nblk[2]) % D.nblk[1]),
                bi = (int)(lblk / ((int64_t)D.nblk[2] * D.nblk[1]));
      const int l = t % 64;
      const int ni = bi * NB + l / 16, nj = bj * NB + (l / 4) % 4, nk = bk * NB + l % 4;
      if (ni < D.nodes[0] && nj < D.nodes[1] && nk < D.nodes[2]) {
        const int64_t g = node_index(D, ni, nj, nk);
        if (from_acc) {
          const long long mf = acc[g];
          if (mf > 0) {
            const double md = (double)mf / D.s_mass;
            double p2 = 0.0;
            for (int a = 1; a <= 3; ++a) {
              const double pa = (double)acc[a * node_total + g] / c.s_mom;
              p2 += pa * pa;
            }
            e += 0.5 * p2 / md;
          }
          for (int a = 0; a < 4; ++a) acc[a * node_total + g] = 0;
        } else {
          const float4 v = vel[g];
          if (v.w > 0.0f) e += 0.5 * (double)v.w * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
        }
      }
    }
  }
  double r[1] = {e};
  block_reduce_multi_to0<GU_THREADS, 1>(r, 0u, shd);
  if (t == 0) out[blockIdx.x] = r[0];
}

// ============================================================== pellet (FP64 rigid body)
struct Q4 {
  double i, j, k, w;
};
__device__ inline void qmat(const double* q, double R[3][3]) {
  const double i = q[0], j = q[1], k = q[2], w = q[3];
  const double ww = w * w, ii = i * i, jj = j * j, kk = k * k;
  const double ij = i * j * 2.0, wk = w * k * 2.0, wj = w * j * 2.0, ik = i * k * 2.0, jk = j * k * 2.0,
               wi = w * i * 2.0;
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
__device__ inline void cross3(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ inline void qrotv(const double* q, const double* r, double* o) {
  double qv[3] = {q[0], q[1], q[2]}, t[3], cc[3];
  cross3(qv, r, t);
  t[0] *= 2.0;
  t[1] *= 2.0;
  t[2] *= 2.0;
  cross3(qv, t, cc);
  for (int a = 0; a < 3; ++a) o[a] = t[a] * q[3] + cc[a] + r[a];
}
__device__ inline void pellet_omega(const PelletState& P, double* om) {
  double R[3][3];
  qmat(P.q, R);
  double bm[3], bo[3];
  for (int a = 0; a < 3; ++a) bm[a] = R[0][a] * P.L[0] + R[1][a] * P.L[1] + R[2][a] * P.L[2];
  for (int a = 0; a < 3; ++a) bo[a] = bm[a] / P.inertia[a];
  for (int a = 0; a < 3; ++a) om[a] = R[a][0] * bo[0] + R[a][1] * bo[1] + R[a][2] * bo[2];
}
__device__ inline double pellet_ke(const PelletState& P) {
  double om[3];
  pellet_omega(P, om);
  return 0.5 * P.mass * (P.vel[0] * P.vel[0] + P.vel[1] * P.vel[1] + P.vel[2] * P.vel[2]) +
         0.5 * (om[0] * P.L[0] + om[1] * P.L[1] + om[2] * P.L[2]);
}
// rigid.rs:279-334
// ef / et: extra force and torque (pellet-bed sphere contacts) or null (the reference's single
// pellet); impulse_out and work_out book the wall contacts only.
__device__ inline void pellet_integrate(PelletState& P, double dt, const double* g, const double* ext, double k,
                                        double e, double mu, double* impulse_out, double* work_out,
                                        const double* ef = nullptr, const double* et = nullptr) {
  double zeta;
  if (e <= 0.0) zeta = 1.0;
  else if (e >= 1.0) zeta = 0.0;
  else {
    const double lg = log(e);
    zeta = -lg / sqrt(3.14159265358979323846 * 3.14159265358979323846 + lg * lg);
  }
  const double damping = 2.0 * zeta * sqrt(k * P.mass);
  double force[3] = {0, 0, 0}, torque[3] = {0, 0, 0}, work = 0.0;
  double om[3];
  pellet_omega(P, om);
  double ax[3];
  const double ex[3] = {1.0, 0.0, 0.0};
  qrotv(P.q, ex, ax);
  for (int s = 0; s < P.nsph; ++s) {
    double cen[3];
    for (int a = 0; a < 3; ++a) cen[a] = P.pos[a] + ax[a] * P.off[s];
    for (int axis = 0; axis < 3; ++axis) {
      for (int f = 0; f < 2; ++f) {
        const double fp = f == 0 ? 0.0 : ext[axis], sign = f == 0 ? 1.0 : -1.0;
        const double gap = (cen[axis] - fp) * sign;
        const double pen = P.radius - gap;
        if (pen <= 0.0) continue;
        double normal[3] = {0, 0, 0};
        normal[axis] = sign;
        double cp[3], lever[3], tmp[3], pv[3];
        for (int a = 0; a < 3; ++a) cp[a] = cen[a] - normal[a] * P.radius;
        for (int a = 0; a < 3; ++a) lever[a] = cp[a] - P.pos[a];
        cross3(om, lever, tmp);
        for (int a = 0; a < 3; ++a) pv[a] = P.vel[a] + tmp[a];
        const double ns = pv[0] * normal[0] + pv[1] * normal[1] + pv[2] * normal[2];
        const double nf = fmax(k * pen - damping * ns, 0.0);
        double tg[3];
        for (int a = 0; a < 3; ++a) tg[a] = pv[a] - normal[a] * ns;
        const double ts = sqrt(tg[0] * tg[0] + tg[1] * tg[1] + tg[2] * tg[2]);
        double ff[3] = {0, 0, 0};
        if (ts > 1e-12) {
          const double limit = fmin(mu * nf, P.mass * ts / dt);
          for (int a = 0; a < 3; ++a) ff[a] = -tg[a] / ts * limit;
        }
        double total[3];
        for (int a = 0; a < 3; ++a) total[a] = normal[a] * nf + ff[a];
        for (int a = 0; a < 3; ++a) force[a] += total[a];
        cross3(lever, total, tmp);
        for (int a = 0; a < 3; ++a) torque[a] += tmp[a];
        work += (total[0] * pv[0] + total[1] * pv[1] + total[2] * pv[2]) * dt;
      }
    }
  }
  for (int a = 0; a < 3; ++a) {
    impulse_out[a] = force[a] * dt;
    const double applied = ef ? (force[a] + ef[a]) * dt : impulse_out[a];
    P.vel[a] = P.vel[a] + (g[a] * dt + applied / P.mass);
  }
  for (int a = 0; a < 3; ++a) P.L[a] += (et ? torque[a] + et[a] : torque[a]) * dt;
  for (int a = 0; a < 3; ++a) P.pos[a] += P.vel[a] * dt;
  double on[3];
  pellet_omega(P, on);
  double h[3] = {on[0] * dt / 2.0, on[1] * dt / 2.0, on[2] * dt / 2.0};
  const double nn = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
  const double eps = 2.220446049250313e-16;
  double inc[4] = {0, 0, 0, 1};
  if (!(nn <= eps * eps)) {
    const double n = sqrt(nn);
    const double f = 1.0 * sin(n) / n;
    inc[0] = h[0] * f;
    inc[1] = h[1] * f;
    inc[2] = h[2] * f;
    inc[3] = cos(n);
  }
  const double* b = P.q;
  double r[4];
  r[0] = inc[3] * b[0] + inc[0] * b[3] + inc[1] * b[2] - inc[2] * b[1];
  r[1] = inc[3] * b[1] - inc[0] * b[2] + inc[1] * b[3] + inc[2] * b[0];
  r[2] = inc[3] * b[2] + inc[0] * b[1] - inc[1] * b[0] + inc[2] * b[3];
  r[3] = inc[3] * b[3] - inc[0] * b[0] - inc[1] * b[1] - inc[2] * b[2];
  for (int a = 0; a < 4; ++a) P.q[a] = r[a];
  *work_out = work;
}

// One CTA per instance that has a pellet: constrain grid nodes inside the pellet against its
// (start-of-step) surface velocity, reduce the equal and opposite impulses in FP64, then apply
// them and integrate the pellet (the trial state is committed by k_end on acceptance).
__global__ void k_couple(const InstDesc* __restrict__ desc, Control* __restrict__ ctrl,
                         const uint32_t* __restrict__ blk_epoch, float4* __restrict__ vel) {
  __shared__ double shd[256];
  const int inst = blockIdx.x;
  Control& c = ctrl[inst];
  const InstDesc& D = desc[inst];
  if (!c.active || !D.has_pellet) return;
  const PelletState& P = c.pellet;
  double ax[3];
  const double ex[3] = {1.0, 0.0, 0.0};
  qrotv(P.q, ex, ax);
  double hs = 0.0;
  for (int s = 0; s < P.nsph; ++s) hs = fmax(hs, fabs(P.off[s]));
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    const double reach = fabs(ax[a]) * hs + P.radius;
    lo[a] = P.pos[a] - reach;
    hi[a] = P.pos[a] + reach;
  }
  int i0[3], n[3];
  for (int a = 0; a < 3; ++a) {
    int a0 = (int)floor(lo[a] / D.dx + 1.0) - 1, a1 = (int)ceil(hi[a] / D.dx + 1.0) + 1;
    a0 = a0 < 0 ? 0 : a0;
    a1 = a1 > D.nodes[a] - 1 ? D.nodes[a] - 1 : a1;
    i0[a] = a0;
    n[a] = a1 >= a0 ? a1 - a0 + 1 : 0;
  }
  double om[3];
  pellet_omega(P, om);
  double imp[3] = {0, 0, 0}, ang[3] = {0, 0, 0}, energy = 0.0;
  const int64_t total = (int64_t)n[0] * n[1] * n[2];
  for (int64_t l = threadIdx.x; l < total; l += blockDim.x) {
    const int k = i0[2] + (int)(l % n[2]);
    const int j = i0[1] + (int)((l / n[2]) % n[1]);
    const int i = i0[0] + (int)(l / ((int64_t)n[2] * n[1]));
    const int64_t blk = D.blk_off + ((int64_t)(i / NB) * D.nblk[1] + j / NB) * D.nblk[2] + k / NB;
    if (blk_epoch[blk] != (uint32_t)c.epoch) continue;
    const int64_t g = node_index(D, i, j, k);
    const float4 nv = vel[g];
    const double mass = nv.w;
    if (!(mass > 0.0)) continue;
    const double node[3] = {((double)i - 1.0) * D.dx, ((double)j - 1.0) * D.dx, ((double)k - 1.0) * D.dx};
    bool outside = false;
    for (int a = 0; a < 3; ++a)
      if (node[a] < lo[a] || node[a] > hi[a]) outside = true;
    if (outside) continue;
    double best = 1e300, normal[3] = {0, 0, 1};
    for (int s = 0; s < P.nsph; ++s) {
      double d[3];
      for (int a = 0; a < 3; ++a) d[a] = node[a] - (P.pos[a] + ax[a] * P.off[s]);
      const double dist = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      const double phi = dist - P.radius;
      if (phi < best) {
        best = phi;
        if (dist > 1e-12) {
          normal[0] = d[0] / dist;
          normal[1] = d[1] / dist;
          normal[2] = d[2] / dist;
        } else {
          normal[0] = 0;
          normal[1] = 0;
          normal[2] = 1;
        }
      }
    }
    if (best > 0.0) continue;
    double lever[3], tmp[3], bv[3];
    for (int a = 0; a < 3; ++a) lever[a] = node[a] - P.pos[a];
    cross3(om, lever, tmp);
    for (int a = 0; a < 3; ++a) bv[a] = P.vel[a] + tmp[a];
    const double v[3] = {nv.x, nv.y, nv.z};
    double rel[3];
    for (int a = 0; a < 3; ++a) rel[a] = v[a] - bv[a];
    const double nsp = rel[0] * normal[0] + rel[1] * normal[1] + rel[2] * normal[2];
    if (nsp >= 0.0) continue;
    double tg[3];
    for (int a = 0; a < 3; ++a) tg[a] = rel[a] - normal[a] * nsp;
    const double ts = sqrt(tg[0] * tg[0] + tg[1] * tg[1] + tg[2] * tg[2]);
    const double fr = D.friction * (-nsp);
    double tn[3] = {0, 0, 0};
    if (!(ts <= fr || ts < 1e-14))
      for (int a = 0; a < 3; ++a) tn[a] = tg[a] * ((ts - fr) / ts);
    double nvv[3], dp[3];
    for (int a = 0; a < 3; ++a) {
      nvv[a] = bv[a] + tn[a];
      dp[a] = (nvv[a] - v[a]) * mass;
    }
    energy += 0.5 * mass * ((nvv[0] * nvv[0] + nvv[1] * nvv[1] + nvv[2] * nvv[2]) - (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    double lx[3];
    cross3(lever, dp, lx);
    for (int a = 0; a < 3; ++a) {
      imp[a] -= dp[a];
      ang[a] -= lx[a];
    }
    vel[g] = make_float4((float)nvv[0], (float)nvv[1], (float)nvv[2], nv.w);
  }
  for (int a = 0; a < 3; ++a) imp[a] = block_sum_d<256>(imp[a], shd);
  for (int a = 0; a < 3; ++a) ang[a] = block_sum_d<256>(ang[a], shd);
  energy = block_sum_d<256>(energy, shd);
  if (threadIdx.x == 0) {
    PelletState T = P;
    const double kb = pellet_ke(T);
    for (int a = 0; a < 3; ++a) {
      T.vel[a] += imp[a] / T.mass;
      T.L[a] += ang[a];
    }
    const double pe = pellet_ke(T) - kb;
    double wimp[3], work;
    pellet_integrate(T, c.dt, D.gravity, D.extent, D.contact_k, D.contact_e, D.contact_mu, wimp, &work);
    bool finite = isfinite(pe);
    for (int a = 0; a < 3; ++a)
      finite = finite && isfinite(T.pos[a]) && isfinite(T.vel[a]) && isfinite(T.L[a]);
    for (int a = 0; a < 4; ++a) finite = finite && isfinite(T.q[a]);
    c.pellet_trial = T;
    for (int a = 0; a < 3; ++a) {
      c.c_impulse[a] = imp[a];
      c.c_angular[a] = ang[a];
      c.pw_impulse[a] = wimp[a];
    }
    c.c_grid_energy = energy;
    c.c_pellet_energy = pe;
    c.pw_work = work;
    c.pellet_fail = finite ? 0 : 1;
  }
}

// ============================================================== pellet bed (extension)
// Many pellets of one multisphere geometry (rigid.rs:115-182 per pellet).  Per attempt:
//   k_bed_bin    : pellets sorted by coarse cell (edge = two bounding radii), ties by index;
//   k_bed_couple : one CTA per pellet applies couple_grid (rigid.rs:385-438) to the grid nodes it
//                  owns: a node inside several proxies belongs to the pellet of smallest signed
//                  distance (ties: lower index), so every node is constrained at most once;
//   k_bed_step   : one thread per pellet: sphere contact (Hertz-Mindlin or the linear law) with the other pellets
//                  (start-of-step states, tangential spring history per sphere pair), then
//                  apply_impulse and integrate (rigid.rs:251-334) with the contact force added.
// The two sides of a contact evaluate mirrored expressions (d -> -d, v_rel -> -v_rel, the
// contact point is the sphere midpoint), so their forces are exact negatives.
__device__ inline double pellet_phi(const PelletState& P, const double ax[3], const double y[3], double nrm[3]) {
  double best = 1e300;
  nrm[0] = 0.0;
  nrm[1] = 0.0;
  nrm[2] = 1.0;
  for (int s = 0; s < P.nsph; ++s) {
    double d[3];
    for (int a = 0; a < 3; ++a) d[a] = y[a] - (P.pos[a] + ax[a] * P.off[s]);
    const double dist = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    const double phi = dist - P.radius;
    if (phi < best) {
      best = phi;
      if (dist > 1e-12) {
        nrm[0] = d[0] / dist;
        nrm[1] = d[1] / dist;
        nrm[2] = d[2] / dist;
      } else {
        nrm[0] = 0;
        nrm[1] = 0;
        nrm[2] = 1;
      }
    }
  }
  return best;
}
__device__ inline void bed_cell(const InstDesc& D, const double x[3], int cc[3]) {
  for (int a = 0; a < 3; ++a) {
    const double f = floor(x[a] / D.bed_h);
    cc[a] = f < 0.0 ? 0 : (f > (double)(D.bed_nc[a] - 1) ? D.bed_nc[a] - 1 : (int)f);
  }
}
__device__ inline long long bed_key_of(const InstDesc& D, const int cc[3]) {
  return ((long long)cc[0] * D.bed_nc[1] + cc[1]) * D.bed_nc[2] + cc[2];
}
// [lo, hi) of sorted entries with this key
__device__ inline void bed_range(const long long* __restrict__ keys, int np, long long key, int& lo, int& hi) {
  int a = 0, b = np;
  while (a < b) {
    const int m = (a + b) >> 1;
    if (keys[m] < key) a = m + 1;
    else b = m;
  }
  lo = a;
  b = np;
  while (a < b) {
    const int m = (a + b) >> 1;
    if (keys[m] <= key) a = m + 1;
    else b = m;
  }
  hi = a;
}

__global__ void __launch_bounds__(1024) k_bed_bin(const InstDesc* __restrict__ desc, const Control* __restrict__ ctrl,
                                                  BedPtrs bed, long long* __restrict__ key, int* __restrict__ idx) {
  __shared__ long long sk[BED_MAX];
  const int inst = blockIdx.x;
  const InstDesc& D = desc[inst];
  const Control& c = ctrl[inst];
  if (D.bed_np < 2 || !c.active) return;
  const PelletState* S = bed.state[c.bed_parity] + D.bed_off;
  const int np = D.bed_np;
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    int cc[3];
    bed_cell(D, S[p].pos, cc);
    sk[p] = bed_key_of(D, cc);
  }
  __syncthreads();
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    const long long kp = sk[p];
    int rank = 0;
    for (int q = 0; q < np; ++q) {
      const long long kq = sk[q];
      rank += (kq < kp) || (kq == kp && q < p);
    }
    key[D.bed_off + rank] = kp;
    idx[D.bed_off + rank] = p;
  }
}

__global__ void __launch_bounds__(128) k_bed_couple(const InstDesc* __restrict__ desc, Control* __restrict__ ctrl,
                                                    const int* __restrict__ bed_inst, BedPtrs bed,
                                                    const long long* __restrict__ key, const int* __restrict__ idx,
                                                    BedStep* __restrict__ step, const uint32_t* __restrict__ blk_epoch,
                                                    float4* __restrict__ vel) {
  __shared__ double shd[128];
  const int64_t gp = blockIdx.x;
  const int inst = bed_inst[gp];
  const Control& c = ctrl[inst];
  const InstDesc& D = desc[inst];
  if (!c.active) return;
  const int p = (int)(gp - D.bed_off);
  const PelletState* S = bed.state[c.bed_parity] + D.bed_off;
  const long long* K = key + D.bed_off;
  const int* I = idx + D.bed_off;
  const PelletState& P = S[p];
  double ax[3];
  const double ex[3] = {1.0, 0.0, 0.0};
  qrotv(P.q, ex, ax);
  double hs = 0.0;
  for (int s = 0; s < P.nsph; ++s) hs = fmax(hs, fabs(P.off[s]));
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    const double reach = fabs(ax[a]) * hs + P.radius;
    lo[a] = P.pos[a] - reach;
    hi[a] = P.pos[a] + reach;
  }
  int i0[3], n[3];
  for (int a = 0; a < 3; ++a) {
    int a0 = (int)floor(lo[a] / D.dx + 1.0) - 1, a1 = (int)ceil(hi[a] / D.dx + 1.0) + 1;
    a0 = a0 < 0 ? 0 : a0;
    a1 = a1 > D.nodes[a] - 1 ? D.nodes[a] - 1 : a1;
    i0[a] = a0;
    n[a] = a1 >= a0 ? a1 - a0 + 1 : 0;
  }
  double om[3];
  pellet_omega(P, om);
  double imp[3] = {0, 0, 0}, ang[3] = {0, 0, 0}, energy = 0.0;
  const int64_t total = (int64_t)n[0] * n[1] * n[2];
  for (int64_t l = threadIdx.x; l < total; l += blockDim.x) {
    const int k = i0[2] + (int)(l % n[2]);
    const int j = i0[1] + (int)((l / n[2]) % n[1]);
    const int i = i0[0] + (int)(l / ((int64_t)n[2] * n[1]));
    const int64_t blk = D.blk_off + ((int64_t)(i / NB) * D.nblk[1] + j / NB) * D.nblk[2] + k / NB;
    if (blk_epoch[blk] != (uint32_t)c.epoch) continue;
    const int64_t g = node_index(D, i, j, k);
    const float4 nv = vel[g];
    const double mass = nv.w;
    if (!(mass > 0.0)) continue;
    const double node[3] = {((double)i - 1.0) * D.dx, ((double)j - 1.0) * D.dx, ((double)k - 1.0) * D.dx};
    bool outside = false;
    for (int a = 0; a < 3; ++a)
      if (node[a] < lo[a] || node[a] > hi[a]) outside = true;
    if (outside) continue;
    double normal[3];
    const double best = pellet_phi(P, ax, node, normal);
    if (best > 0.0) continue;
    // ownership: the pellet of smallest signed distance, ties to the lower index
    bool own = true;
    int cc[3];
    bed_cell(D, node, cc);
    for (int di = -1; di <= 1 && own; ++di)
      for (int dj = -1; dj <= 1 && own; ++dj)
        for (int dk = -1; dk <= 1 && own; ++dk) {
          const int c3[3] = {cc[0] + di, cc[1] + dj, cc[2] + dk};
          if (c3[0] < 0 || c3[1] < 0 || c3[2] < 0 || c3[0] >= D.bed_nc[0] || c3[1] >= D.bed_nc[1] ||
              c3[2] >= D.bed_nc[2])
            continue;
          int r0, r1;
          bed_range(K, D.bed_np, bed_key_of(D, c3), r0, r1);
          for (int r = r0; r < r1 && own; ++r) {
            const int q = I[r];
            if (q == p) continue;
            const PelletState& Q = S[q];
            const double dq[3] = {node[0] - Q.pos[0], node[1] - Q.pos[1], node[2] - Q.pos[2]};
            if (dq[0] * dq[0] + dq[1] * dq[1] + dq[2] * dq[2] > D.bed_rb * D.bed_rb) continue;
            double axq[3], nq[3];
            qrotv(Q.q, ex, axq);
            const double phq = pellet_phi(Q, axq, node, nq);
            if (phq < best || (phq == best && q < p)) own = false;
          }
        }
    if (!own) continue;
    double lever[3], tmp[3], bv[3];
    for (int a = 0; a < 3; ++a) lever[a] = node[a] - P.pos[a];
    cross3(om, lever, tmp);
    for (int a = 0; a < 3; ++a) bv[a] = P.vel[a] + tmp[a];
    const double v[3] = {nv.x, nv.y, nv.z};
    double rel[3];
    for (int a = 0; a < 3; ++a) rel[a] = v[a] - bv[a];
    const double nsp = rel[0] * normal[0] + rel[1] * normal[1] + rel[2] * normal[2];
    if (nsp >= 0.0) continue;
    double tg[3];
    for (int a = 0; a < 3; ++a) tg[a] = rel[a] - normal[a] * nsp;
    const double ts = sqrt(tg[0] * tg[0] + tg[1] * tg[1] + tg[2] * tg[2]);
    const double fr = D.friction * (-nsp);
    double tn[3] = {0, 0, 0};
    if (!(ts <= fr || ts < 1e-14))
      for (int a = 0; a < 3; ++a) tn[a] = tg[a] * ((ts - fr) / ts);
    double nvv[3], dp[3];
    for (int a = 0; a < 3; ++a) {
      nvv[a] = bv[a] + tn[a];
      dp[a] = (nvv[a] - v[a]) * mass;
    }
    energy += 0.5 * mass * ((nvv[0] * nvv[0] + nvv[1] * nvv[1] + nvv[2] * nvv[2]) - (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    double lx[3];
    cross3(lever, dp, lx);
    for (int a = 0; a < 3; ++a) {
      imp[a] -= dp[a];
      ang[a] -= lx[a];
    }
    vel[g] = make_float4((float)nvv[0], (float)nvv[1], (float)nvv[2], nv.w);
  }
  for (int a = 0; a < 3; ++a) imp[a] = block_sum_d<128>(imp[a], shd);
  for (int a = 0; a < 3; ++a) ang[a] = block_sum_d<128>(ang[a], shd);
  energy = block_sum_d<128>(energy, shd);
  if (threadIdx.x == 0) {
    BedStep& st = step[gp];
    for (int a = 0; a < 3; ++a) {
      st.imp[a] = imp[a];
      st.ang[a] = ang[a];
    }
    st.cgrid = energy;
  }
}

constexpr int BED_CAND = 64;  // neighbour pellets examined per pellet

__global__ void __launch_bounds__(64) k_bed_step(const InstDesc* __restrict__ desc, Control* __restrict__ ctrl,
                                                 const int* __restrict__ bed_inst, int64_t n_bed, BedPtrs bed,
                                                 const long long* __restrict__ key, const int* __restrict__ idx,
                                                 BedStep* __restrict__ step) {
  const int64_t gp = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gp >= n_bed) return;
  const int inst = bed_inst[gp];
  const Control& c = ctrl[inst];
  const InstDesc& D = desc[inst];
  if (!c.active) return;
  const int par = c.bed_parity;
  const int p = (int)(gp - D.bed_off);
  const PelletState* S = bed.state[par] + D.bed_off;
  PelletState* T = bed.state[par ^ 1] + D.bed_off;
  const HmContact* hold = bed.hist[par] + gp * HM_SLOTS;
  const int nold = bed.hist_n[par][gp];
  HmContact* hnew = bed.hist[par ^ 1] + gp * HM_SLOTS;
  const long long* K = key + D.bed_off;
  const int* I = idx + D.bed_off;
  const PelletState& P = S[p];
  const double dt = c.dt;
  const double ex[3] = {1.0, 0.0, 0.0};
  double axp[3], omp[3];
  qrotv(P.q, ex, axp);
  pellet_omega(P, omp);
  BedStep& st = step[gp];
  int fail = 0, overflow = 0, contacts = 0, nnew = 0;
  // neighbours within two bounding radii, in increasing index
  int cand[BED_CAND];
  int nc = 0;
  int cc[3];
  bed_cell(D, P.pos, cc);
  for (int di = -1; di <= 1; ++di)
    for (int dj = -1; dj <= 1; ++dj)
      for (int dk = -1; dk <= 1; ++dk) {
        const int c3[3] = {cc[0] + di, cc[1] + dj, cc[2] + dk};
        if (c3[0] < 0 || c3[1] < 0 || c3[2] < 0 || c3[0] >= D.bed_nc[0] || c3[1] >= D.bed_nc[1] ||
            c3[2] >= D.bed_nc[2])
          continue;
        int r0, r1;
        bed_range(K, D.bed_np, bed_key_of(D, c3), r0, r1);
        for (int r = r0; r < r1; ++r) {
          const int q = I[r];
          if (q == p) continue;
          const double dq[3] = {S[q].pos[0] - P.pos[0], S[q].pos[1] - P.pos[1], S[q].pos[2] - P.pos[2]};
          if (dq[0] * dq[0] + dq[1] * dq[1] + dq[2] * dq[2] > 4.0 * D.bed_rb * D.bed_rb) continue;
          if (nc == BED_CAND) {
            fail = 1;
            continue;
          }
          int w = nc++;
          while (w > 0 && cand[w - 1] > q) {
            cand[w] = cand[w - 1];
            --w;
          }
          cand[w] = q;
        }
      }
  const double rs = 0.5 * P.radius;       // effective radius of two equal spheres
  const double k56 = 1.8257418583505538;  // 2 sqrt(5/6)
  double F[3] = {0, 0, 0}, Tq[3] = {0, 0, 0}, W = 0.0;
  for (int ci = 0; ci < nc; ++ci) {
    const int q = cand[ci];
    const PelletState& Q = S[q];
    double axq[3], omq[3];
    qrotv(Q.q, ex, axq);
    pellet_omega(Q, omq);
    const double mstar = P.mass * Q.mass / (P.mass + Q.mass);
    for (int a = 0; a < P.nsph; ++a) {
      double ca[3];
      for (int k = 0; k < 3; ++k) ca[k] = P.pos[k] + axp[k] * P.off[a];
      for (int b = 0; b < Q.nsph; ++b) {
        double cb[3], d[3];
        for (int k = 0; k < 3; ++k) {
          cb[k] = Q.pos[k] + axq[k] * Q.off[b];
          d[k] = cb[k] - ca[k];
        }
        const double dist = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        const double delta = (P.radius + Q.radius) - dist;
        if (!(delta > 0.0) || !(dist > 1e-12)) continue;
        double nn[3], cp[3], lp[3], lq[3], t1[3], t2[3], vp[3], vrel[3];
        for (int k = 0; k < 3; ++k) {
          nn[k] = d[k] / dist;
          cp[k] = 0.5 * (ca[k] + cb[k]);
          lp[k] = cp[k] - P.pos[k];
          lq[k] = cp[k] - Q.pos[k];
        }
        cross3(omp, lp, t1);
        cross3(omq, lq, t2);
        for (int k = 0; k < 3; ++k) {
          vp[k] = P.vel[k] + t1[k];
          vrel[k] = (Q.vel[k] + t2[k]) - vp[k];
        }
        const double vn = vrel[0] * nn[0] + vrel[1] * nn[1] + vrel[2] * nn[2];
        double vt[3];
        for (int k = 0; k < 3; ++k) vt[k] = vrel[k] - vn * nn[k];
        double xi[3] = {0.0, 0.0, 0.0};
        for (int h = 0; h < nold; ++h)
          if (hold[h].other == q && hold[h].a == a && hold[h].b == b) {
            xi[0] = hold[h].xi[0];
            xi[1] = hold[h].xi[1];
            xi[2] = hold[h].xi[2];
            break;
          }
        const double xn = xi[0] * nn[0] + xi[1] * nn[1] + xi[2] * nn[2];
        double fn, ft[3], roll[3] = {0.0, 0.0, 0.0};
        if (D.bed_law == 1) {
          // linear spring-dashpot, tangential spring with Coulomb sliding and constant rolling
          // resistance (dem.rs:789-834).  xi follows the reference's first-body convention (this
          // pellet first, contact normal pointing at it), in which the tangential velocity is -vt.
          const double cn = 2.0 * D.dem_zeta * sqrt(D.dem_kn * mstar);
          const double kt = (2.0 / 7.0) * D.dem_kn, ct = 0.5345224838248488 * cn;  // sqrt(2/7) cn
          fn = fmax(D.dem_kn * delta - cn * vn, 0.0);
          for (int k = 0; k < 3; ++k) {
            xi[k] = (xi[k] - xn * nn[k]) - vt[k] * dt;
            ft[k] = -(xi[k] * kt) + vt[k] * ct;
          }
          const double ftn = sqrt(ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2]);
          const double lim = D.hm_mu * fn;
          if (ftn > lim) {
            const double sc = ftn > 2.220446049250313e-16 ? lim / ftn : 0.0;
            for (int k = 0; k < 3; ++k) {
              ft[k] *= sc;
              xi[k] = -ft[k] / kt;
            }
          }
          double wr[3];
          for (int k = 0; k < 3; ++k) wr[k] = omp[k] - omq[k];
          const double wn = sqrt(wr[0] * wr[0] + wr[1] * wr[1] + wr[2] * wr[2]);
          if (wn > 2.220446049250313e-16)
            for (int k = 0; k < 3; ++k) roll[k] = -wr[k] / wn * (D.dem_mur * rs * fn);
        } else {
          const double sq = sqrt(rs * delta);
          const double sn = 2.0 * D.hm_estar * sq, stf = 8.0 * D.hm_gstar * sq;
          const double gn = -k56 * D.hm_beta * sqrt(sn * mstar), gt = -k56 * D.hm_beta * sqrt(stf * mstar);
          fn = fmax((4.0 / 3.0) * D.hm_estar * sqrt(rs) * (delta * sqrt(delta)) - gn * vn, 0.0);
          for (int k = 0; k < 3; ++k) {
            xi[k] = (xi[k] - xn * nn[k]) + vt[k] * dt;
            ft[k] = stf * xi[k] + gt * vt[k];
          }
          const double ftn = sqrt(ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2]);
          const double lim = D.hm_mu * fn;
          if (ftn > lim) {
            const double sc = lim / ftn;
            for (int k = 0; k < 3; ++k) {
              ft[k] *= sc;
              xi[k] = (ft[k] - gt * vt[k]) / stf;
            }
          }
        }
        double f[3], tq[3];
        for (int k = 0; k < 3; ++k) f[k] = ft[k] - fn * nn[k];
        cross3(lp, f, tq);
        for (int k = 0; k < 3; ++k) {
          F[k] += f[k];
          Tq[k] += tq[k] + roll[k];
        }
        ++contacts;
        if (nnew < HM_SLOTS) {
          HmContact& hc = hnew[nnew++];
          hc.other = q;
          hc.a = a;
          hc.b = b;
          hc.pad = 0;
          for (int k = 0; k < 3; ++k) hc.xi[k] = xi[k];
        } else {
          ++overflow;
        }
      }
    }
  }
  bed.hist_n[par ^ 1][gp] = nnew;
  // coupling impulse, then the rigid step with the contact force (rigid.rs:251-334)
  PelletState Tp = P;
  const double kb = pellet_ke(Tp);
  for (int a = 0; a < 3; ++a) {
    Tp.vel[a] += st.imp[a] / Tp.mass;
    Tp.L[a] += st.ang[a];
  }
  const double pe = pellet_ke(Tp) - kb;
  double wimp[3], work;
  pellet_integrate(Tp, dt, D.gravity, D.extent, D.contact_k, D.contact_e, D.contact_mu, wimp, &work, F, Tq);
  // contact work over the step at the step's mean linear and angular velocity: for the
  // explicit update this is the kinetic-energy change the contact force causes
  double ome[3];
  pellet_omega(Tp, ome);
  for (int k = 0; k < 3; ++k) W += (F[k] * (0.5 * (P.vel[k] + Tp.vel[k])) + Tq[k] * (0.5 * (omp[k] + ome[k]))) * dt;
  bool finite = isfinite(pe) && isfinite(W);
  for (int a = 0; a < 3; ++a) finite = finite && isfinite(Tp.pos[a]) && isfinite(Tp.vel[a]) && isfinite(Tp.L[a]);
  for (int a = 0; a < 4; ++a) finite = finite && isfinite(Tp.q[a]);
  T[p] = Tp;
  st.cpellet = pe;
  for (int a = 0; a < 3; ++a) st.wimp[a] = wimp[a];
  st.wwork = work;
  st.ppwork = W;
  st.contacts = contacts;
  st.overflow = overflow;
  st.limit = pellet_bed_limit(D, Tp);
  st.fail = (fail || !finite) ? 1 : 0;
}

// ============================================================== G2P + constitutive
// Persistent CTAs take the occupied P2G tiles from the attempt's tile list.  Per tile, the
// (TX+2)(TY+2)(TZ+2) node velocities are staged in shared memory once, then the CTA walks the
// tile's particles (contiguous in sorted slot order),
// gathers from shared memory, advects, runs the constitutive update and writes the trial state
// in sorted slot order.  The next round's particle inputs are prefetched by cp.async while the
// current round computes.

// G2P input slots per particle, [slot][thread] in shared memory, two rounds in flight
enum {
  PF_X = 0,    // 3: position
  PF_H = 3,    // 9: F - I (paste)
  PF_JM1 = 3,  // 1: J - 1 (liquid)
  PF_EP = 12,
  PF_M = 13,
  PF_V0 = 14,
  PF_YS = 15,  // per-particle yield stress
  PF_ID = 16,
  PF_SLOTS = 17
};
// dynamic shared memory of a G2P CTA of nt threads
constexpr size_t g2p_smem(int nt) { return sizeof(float) * 2 * PF_SLOTS * nt; }
// threads per CTA of the two G2P instantiations the launch shape chooses from
constexpr int G2P_THREADS_SMALL = 128;
// threads per CTA of G2P variant v: 0 256 threads (2 CTAs per SM), 1-3 128 threads with registers
// sized for 4, 5 or 6 CTAs per SM (more resident warps, some registers spilled)
constexpr int g2p_threads(int v) { return v == 0 ? G2P_THREADS : G2P_THREADS_SMALL; }

template <int NT>
__device__ __forceinline__ void g2p_prefetch(float* __restrict__ buf, const float* __restrict__ cur,
                                             const uint32_t* __restrict__ idc, int64_t cap, int64_t src, bool paste,
                                             bool pyield) {
  float* b = buf + threadIdx.x;
#pragma unroll
  for (int a = 0; a < 3; ++a) cp_async4(b + (PF_X + a) * NT, cur + (C_X + a) * cap + src);
  if (paste) {
#pragma unroll
    for (int a = 0; a < 9; ++a) cp_async4(b + (PF_H + a) * NT, cur + (C_H + a) * cap + src);
    if (pyield) cp_async4(b + PF_YS * NT, cur + C_YS * cap + src);
  } else {
    cp_async4(b + PF_JM1 * NT, cur + C_JM1 * cap + src);
  }
  cp_async4(b + PF_EP * NT, cur + C_EP * cap + src);
  cp_async4(b + PF_M * NT, cur + C_M * cap + src);
  cp_async4(b + PF_V0 * NT, cur + C_V0 * cap + src);
  cp_async4(b + PF_ID * NT, idc + src);
}

// Paste particles whose trial strain is outside the series path of paste_trial (||B||_F > 0.25:
// large elastic strain, or a non-finite state) take the eigen-decomposition path.  k_g2p leaves
// them to k_g2p_defer: it stores H_tr in the trial state's H, the unchanged plastic strain, and
// DEFER_MARK in tau_xx, and lists the tile.  So the hot kernel carries no call of
// paste_update_jacobi (no call frame, no copies on the stack), and a strain that needs the
// eigenvectors costs one more pass over the tiles that hold one.
constexpr uint32_t DEFER_MARK = 0x7fc0defeu;  // a quiet NaN payload that no arithmetic produces

// Warm start (WARM instantiation): each yielding lane reads the network's logit at its la8 from
// its instance's table (k_mlp_table), interpolated between the two neighbouring nodes.
// one tile of k_g2p, CTAs of NT threads.  CLOCKS (a measurement instantiation, not used by the
// solver): every warp adds its clock64 cycles in the tile to clk[0] and, per round, the longest
// lane time in the Herschel-Bulkley return to clk[1], so clk[1] / clk[0] is the share of warp
// time the return takes.
// Material kinds a G2P instantiation handles: paste only, liquid only, or both (an ensemble whose
// instances mix them).  The single-kind instantiations carry no code of the other kind's update,
// which keeps the kernel small (its instruction fetch, not its arithmetic, limits it).
enum G2pKind : int { G2P_PASTE = 0, G2P_LIQUID = 1, G2P_MIXED = 2 };

template <bool WARM, int NT, bool CLOCKS, int KIND>
__device__ __forceinline__ void g2p_tile(const uint4 rec, const InstDesc* __restrict__ desc,
                                         const Control* __restrict__ ctrl, float* __restrict__ st0, float* __restrict__ st1,
                                         uint32_t* __restrict__ id0, uint32_t* __restrict__ id1, int64_t cap,
                                         const uint32_t* __restrict__ perm, const float4* __restrict__ vel,
                                         ParticlePartial* __restrict__ part, const float* __restrict__ mlp_tab,
                                         float* __restrict__ log_x,
                                         float* __restrict__ log_y, unsigned long long* __restrict__ log_n,
                                         long long log_cap, unsigned long long* __restrict__ clk,
                                         uint4* __restrict__ defer_rec, uint32_t* __restrict__ defer_count) {
  __shared__ float4 hv[HN];
  __shared__ int defer_flag;  // some particle of the tile is left to k_g2p_defer
  // per thread, the deviatoric Hencky strain (6), its mean and the volumetric strain, parked
  // during the Herschel-Bulkley return (with H_tr, parked over the dead H of the prefetch slot)
  __shared__ float park[8 * NT];
  extern __shared__ float4 g2p_dyn[];  // prefetched inputs of two rounds
  float* pf = reinterpret_cast<float*>(g2p_dyn);
  const int tile = (int)rec.x, inst = (int)rec.y;
  const Control& c = ctrl[inst];
  if (!c.active) return;
  const long long clk_begin = CLOCKS ? clock64() : 0;
  unsigned long long clk_newton = 0;  // CLOCKS: this warp's return cycles in the tile
  const InstDesc& D = desc[inst];
  const int64_t ltile = tile - D.tile_off;
  const uint32_t s0 = rec.z, e0 = rec.w;
  if (s0 == e0) {
    if (threadIdx.x == 0) {
      ParticlePartial& P = part[tile];
      P.diss = P.bbound = P.mass = 0.0;
      P.max_speed = P.max_disp = 0.f;
      P.fail = F_OK;
      P.iterations = P.yielded = 0;
      P.fail_value = 0.0;
    }
    return;
  }
  const float* cur = c.parity ? st1 : st0;
  float* nxt = c.parity ? st0 : st1;
  const uint32_t* idc = c.parity ? id1 : id0;
  uint32_t* idn = c.parity ? id0 : id1;
  const bool paste = KIND == G2P_PASTE || (KIND == G2P_MIXED && D.kind == 0);
  const bool pyield = paste && D.per_particle_yield;
  const int nround = (int)((e0 - s0 + NT - 1) / NT);
  // slot of this thread in round r (clamped to the tile's last particle) and warp liveness
  auto slot_of = [&](int r) -> int64_t {
    const int64_t kk = (int64_t)s0 + (int64_t)r * NT + threadIdx.x;
    return kk < (int64_t)e0 ? kk : (int64_t)e0 - 1;
  };
  auto live_of = [&](int r) -> bool {
    return (int64_t)s0 + (int64_t)r * NT + (threadIdx.x & ~31u) < (int64_t)e0;
  };
  // pipeline: copies of round r+1 are in flight while round r computes; perm of round r+2 is
  // loaded a round ahead of its copies.  The first round's copies are issued before the halo is
  // staged, so that the two overlap.
  int64_t src_next = 0;
  if (live_of(0)) g2p_prefetch<NT>(pf, cur, idc, cap, perm[slot_of(0)], paste, pyield);
  cp_async_commit();
  if (nround > 1 && live_of(1)) src_next = perm[slot_of(1)];
  const int tz = (int)(ltile % D.tiles[2]);
  const int ty = (int)((ltile / D.tiles[2]) % D.tiles[1]);
  const int tx = (int)(ltile / ((int64_t)D.tiles[2] * D.tiles[1]));
  const int ox = tx * TX, oy = ty * TY, oz = tz * TZ;
  if (threadIdx.x == 0) defer_flag = 0;
  for (int n = threadIdx.x; n < HN; n += NT) {
    const int hz = n % HZ, hy = (n / HZ) % HY, hx = n / (HZ * HY);
    const int gi = ox + hx, gj = oy + hy, gk = oz + hz;
    hv[n] = (gi < D.nodes[0] && gj < D.nodes[1] && gk < D.nodes[2]) ? __ldg(&vel[node_index(D, gi, gj, gk)])
                                                                    : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  const bool use_mlp = WARM && D.kind == 0 && c.warm_start && mlp_tab != nullptr;  // CTA-uniform
  const float2* tab =
      use_mlp ? reinterpret_cast<const float2*>(mlp_tab + (int64_t)inst * MLP_TAB_FLOATS + MLP_TAB_STRIDE) : nullptr;
  const float inv_k = (float)(1.0 / D.consistency);
  const float dx = (float)D.dx;
  const float dt = (float)c.dt;
  // this thread's sums over its particles of the tile, kept in shared memory (through volatile
  // accesses) instead of registers: each is touched once per round, and the registers are worth
  // more to the FP64 return
  __shared__ double acc_d[4 * NT];  // plastic work, momentum bound, mass, failure value
  __shared__ float acc_f[2 * NT];   // largest speed, largest displacement
  __shared__ int acc_i[3 * NT];     // failure code, Newton iterations, yielded particles
  volatile double& diss = acc_d[threadIdx.x];
  volatile double& bb = acc_d[NT + threadIdx.x];
  volatile double& mass_sum = acc_d[2 * NT + threadIdx.x];
  volatile double& fail_value = acc_d[3 * NT + threadIdx.x];
  volatile float& max_speed = acc_f[threadIdx.x];
  volatile float& max_disp = acc_f[NT + threadIdx.x];
  volatile int& fail = acc_i[threadIdx.x];
  volatile int& iters = acc_i[NT + threadIdx.x];
  volatile int& yielded = acc_i[2 * NT + threadIdx.x];
  diss = 0.0;
  bb = 0.0;
  mass_sum = 0.0;
  fail_value = 0.0;
  max_speed = 0.0f;
  max_disp = 0.0f;
  fail = F_OK;
  iters = 0;
  yielded = 0;
  const float c_tau = (float)(D.max_dt * 4.0 / (D.dx * D.dx));
  const float c_dx = (float)(2.6 * D.dx);
  const float c_g =
      (float)(6.0 * sqrt(D.gravity[0] * D.gravity[0] + D.gravity[1] * D.gravity[1] + D.gravity[2] * D.gravity[2]) *
              D.max_dt);
  for (int r = 0; r < nround; ++r) {
    // a warp leaves once its slots are past the tile; lanes past the end of a live warp redo the
    // tile's last particle and store nothing
    const bool warp_live = live_of(r);
    if (!warp_live) break;
    if (r + 1 < nround && live_of(r + 1))
      g2p_prefetch<NT>(pf + ((r + 1) & 1) * PF_SLOTS * NT, cur, idc, cap, src_next, paste, pyield);
    cp_async_commit();
    if (r + 2 < nround && live_of(r + 2)) src_next = perm[slot_of(r + 2)];
    cp_async_wait<1>();  // this thread's copies of round r have landed
    const float* in = pf + (r & 1) * PF_SLOTS * NT + threadIdx.x;
    const bool valid = (int64_t)s0 + (int64_t)r * NT + threadIdx.x < (int64_t)e0;
    const int64_t k = slot_of(r);
    float Htr[9];
    float tau[6];
    float ep = 0.f, speed = 0.f, disp = 0.f, m = 0.f, v0 = 0.f, cn = 0.f;
    double ys = 0.0;
    PasteTrial pt;
    PasteOut o;
    pt.path = PT_DONE;
    pt.trial_eq = 0.0;
    if (warp_live) {
      float x[3];
      int base[3];
      float w[3][3], d[3][3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        x[a] = in[(PF_X + a) * NT];
        const float sc = scaled_of(x[a], dx, D.pow2_inv_dx);
        const float bf = floorf(sc - 0.5f);
        base[a] = (int)(bf + 1.0f);
        weights_of(sc - bf, dx, w[a], d[a]);
      }
      float v[3], Cm[9];
      const int lbx = base[0] - ox, lby = base[1] - oy, lbz = base[2] - oz;
      // separable gather: per (a, b) row, z sums S0 = sum_c w_c v and S1 = sum_c w_c d_c v, then
      // v += w_ab S0, C[:,0] += w_ab d_a S0, C[:,1] += w_ab d_b S0, C[:,2] += w_ab S1.  The x and y
      // components run as pairs on the paired FP32 units (fma.rn.f32x2, each lane the scalar FMA);
      // C is held as the pairs (C_00, C_10), (C_01, C_11), (C_02, C_12) and the z row alone.
      const float wdz[3] = {w[2][0] * d[2][0], w[2][1] * d[2][1], w[2][2] * d[2][2]};
      float2 vxy = make_float2(0.f, 0.f), c0 = vxy, c1 = vxy, c2 = vxy;
      float vz = 0.f, cz0 = 0.f, cz1 = 0.f, cz2 = 0.f;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          const int row = ((lbx + a) * HY + (lby + b)) * HZ + lbz;
          float2 s0 = make_float2(0.f, 0.f), s1 = s0;
          float s0z = 0.f, s1z = 0.f;
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) {
            const float4 nv = hv[row + cc];
            const float2 nxy = make_float2(nv.x, nv.y);
            s0 = __ffma2_rn(make_float2(w[2][cc], w[2][cc]), nxy, s0);
            s1 = __ffma2_rn(make_float2(wdz[cc], wdz[cc]), nxy, s1);
            s0z = __fmaf_rn(w[2][cc], nv.z, s0z);
            s1z = __fmaf_rn(wdz[cc], nv.z, s1z);
          }
          const float wab = w[0][a] * w[1][b];
          const float wa0 = wab * d[0][a], wa1 = wab * d[1][b];
          const float2 wab2 = make_float2(wab, wab);
          vxy = __ffma2_rn(wab2, s0, vxy);
          c0 = __ffma2_rn(make_float2(wa0, wa0), s0, c0);
          c1 = __ffma2_rn(make_float2(wa1, wa1), s0, c1);
          c2 = __ffma2_rn(wab2, s1, c2);
          vz = __fmaf_rn(wab, s0z, vz);
          cz0 = __fmaf_rn(wa0, s0z, cz0);
          cz1 = __fmaf_rn(wa1, s0z, cz1);
          cz2 = __fmaf_rn(wab, s1z, cz2);
        }
      v[0] = vxy.x;
      v[1] = vxy.y;
      v[2] = vz;
      Cm[0] = c0.x;
      Cm[1] = c1.x;
      Cm[2] = c2.x;
      Cm[3] = c0.y;
      Cm[4] = c1.y;
      Cm[5] = c2.y;
      Cm[6] = cz0;
      Cm[7] = cz1;
      Cm[8] = cz2;
      const float dx2_inv = 4.0f / (dx * dx);
#pragma unroll
      for (int a = 0; a < 9; ++a) Cm[a] *= dx2_inv;
      speed = particle_speed(v);
      disp = scaled_of(speed * dt, dx, D.pow2_inv_dx);
      m = in[PF_M * NT];
      v0 = in[PF_V0 * NT];
      ep = in[PF_EP * NT];
      // kinematic part of the trial state, stored before the constitutive update (sorted slot order)
      if (valid) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          nxt[(C_X + a) * cap + k] = x[a] + v[a] * dt;
          nxt[(C_V + a) * cap + k] = v[a];
        }
#pragma unroll
        for (int a = 0; a < 9; ++a) nxt[(C_C + a) * cap + k] = Cm[a];
        nxt[C_M * cap + k] = m;
        nxt[C_V0 * cap + k] = v0;
        if (pyield) nxt[C_YS * cap + k] = in[PF_YS * NT];
        idn[k] = __float_as_uint(in[PF_ID * NT]);
      }
      cn = affine_norm(Cm);
      if (paste) {
        float H[9];
#pragma unroll
        for (int a = 0; a < 9; ++a) H[a] = in[(PF_H + a) * NT];
        // H_tr = H + dt C + dt C H
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const float ch =
                Cm[3 * i + 0] * H[0 * 3 + j] + Cm[3 * i + 1] * H[1 * 3 + j] + Cm[3 * i + 2] * H[2 * 3 + j];
            Htr[3 * i + j] = H[3 * i + j] + dt * (Cm[3 * i + j] + ch);
          }
        ys = pyield ? (double)in[PF_YS * NT] : D.yield;
        paste_trial<true>(Htr, D.mu, pt, o);
        // park what the stress update needs after the return in shared memory, written and read
        // back through volatile accesses so that it holds no registers during the FP64 Newton
        volatile float* pk = pf + (r & 1) * PF_SLOTS * NT + threadIdx.x;  // this thread's prefetch slot
#pragma unroll
        for (int a = 0; a < 9; ++a) pk[(PF_H + a) * NT] = Htr[a];
        volatile float* pd = park + threadIdx.x;
        pd[0 * NT] = pt.dev.xx;
        pd[1 * NT] = pt.dev.yy;
        pd[2 * NT] = pt.dev.zz;
        pd[3 * NT] = pt.dev.xy;
        pd[4 * NT] = pt.dev.xz;
        pd[5 * NT] = pt.dev.yz;
        pd[6 * NT] = pt.mean;
        pd[7 * NT] = pt.vol;
      } else {
        const float jm1 = in[PF_JM1 * NT];
        LiquidOut lo;
        liquid_update(jm1, Cm, (float)D.bulk, (float)D.consistency, (float)D.tait_gamma, dt, lo);
#pragma unroll
        for (int a = 0; a < 6; ++a) tau[a] = lo.tau[a];
        if (valid) {
          if (lo.fail != F_OK) fail = max((int)fail, lo.fail);
          nxt[C_JM1 * cap + k] = lo.jm1;
        }
      }
    }
    double sigma0 = -1.0;
    if constexpr (WARM) {
      // learned warm start of the yielding lanes (the network's root fraction from the table)
      if (use_mlp && valid && pt.path != PT_DONE && pt.trial_eq > ys && pt.trial_eq > 0.0) {
        const float t = mlp_table_fraction(tab, hb_la8(inv_k, pt.trial_eq, ys));
        if (t > 0.0f && t < 1.0f) sigma0 = ys + (double)t * (pt.trial_eq - ys);
      }
    }
    if (paste) {
      long long nc = 0;
      // paste_finish of the series path, split around the parked values
      double scale = 1.0;
      if (pt.path == PT_SERIES) scale = paste_return(pt.trial_eq, pt.dnorm, ys, c.hb, D.tol, sigma0, o,
                                                     CLOCKS ? &nc : nullptr);
      if constexpr (CLOCKS) clk_newton += __reduce_max_sync(0xffffffffu, (unsigned)nc);  // the warp is converged
      const volatile float* pk = pf + (r & 1) * PF_SLOTS * NT + threadIdx.x;
      const volatile float* pd = park + threadIdx.x;
      float Hr[9];
#pragma unroll
      for (int a = 0; a < 9; ++a) Hr[a] = pk[(PF_H + a) * NT];
      if (pt.path == PT_SERIES && o.fail == F_OK) {
        const Sym dev = {pd[0 * NT], pd[1 * NT], pd[2 * NT], pd[3 * NT], pd[4 * NT], pd[5 * NT]};
        paste_stress(Hr, dev, pd[6 * NT], pd[7 * NT], (float)D.mu, (float)D.lambda, scale, o);
      }
      if (pt.path == PT_DEFER) {  // k_g2p_defer finishes it (paste_trial zeroed o's scalars)
#pragma unroll
        for (int a = 0; a < 9; ++a) o.H[a] = Hr[a];
        o.tau[0] = __uint_as_float(DEFER_MARK);
#pragma unroll
        for (int a = 1; a < 6; ++a) o.tau[a] = 0.0f;
        if (valid) defer_flag = 1;
      }
#pragma unroll
      for (int a = 0; a < 6; ++a) tau[a] = o.tau[a];
      if (valid) {
        if (o.fail != F_OK) {
          fail = max((int)fail, o.fail);
          fail_value = o.eq;
        }
#pragma unroll
        for (int a = 0; a < 9; ++a) nxt[(C_H + a) * cap + k] = o.H[a];
        ep += (float)o.dep;
        diss = diss + o.diss_density * (double)v0;
        iters = iters + o.iters;
        yielded = yielded + o.yielded;
        if (log_n != nullptr && o.yielded && o.fail == F_OK) {
          const unsigned long long slot = atomicAdd(log_n, 1ull);
          if ((long long)slot < log_cap) {
            // (trial stress, yield, consistency, flow index, mu, dt) -> returned stress
            log_x[6 * slot + 0] = (float)o.trial;
            log_x[6 * slot + 1] = (float)ys;
            log_x[6 * slot + 2] = (float)D.consistency;
            log_x[6 * slot + 3] = (float)D.flow_index;
            log_x[6 * slot + 4] = (float)D.mu;
            log_x[6 * slot + 5] = (float)c.dt;
            log_y[slot] = (float)o.eq;
          }
        }
      }
    }
    if (!valid) continue;
#pragma unroll
    for (int a = 0; a < 6; ++a) nxt[(C_TAU + a) * cap + k] = tau[a];
    nxt[C_EP * cap + k] = ep;
    // momentum bound of the new state for the next attempt's fixed-point scale (its factors of
    // 2.6 and 6 leave ample room for rounding); k_g2p_defer adds the deferred particles'
    if (pt.path != PT_DEFER) bb = bb + momentum_bound(m, speed, cn, tau, v0, c_tau, c_dx, c_g);
    mass_sum = mass_sum + (double)m;
    max_speed = fmaxf(max_speed, speed);
    max_disp = fmaxf(max_disp, disp);
  }
  cp_async_wait<0>();  // no copy may land after the CTA's shared memory is released
  // the tile's sums: a warp butterfly (one short loop over the five offsets), then thread 0 adds
  // the warps' results in warp order (a fixed order: deterministic, one barrier)
  {
    double d0 = diss, d1 = bb, d2 = mass_sum, d3 = fail_value;
    float f0 = max_speed, f1 = max_disp;
    int i0 = fail, i1 = iters, i2 = yielded;
#pragma unroll 1
    for (int o = 16; o > 0; o >>= 1) {
      d0 += __shfl_xor_sync(0xffffffffu, d0, o);
      d1 += __shfl_xor_sync(0xffffffffu, d1, o);
      d2 += __shfl_xor_sync(0xffffffffu, d2, o);
      d3 = fmax(d3, __shfl_xor_sync(0xffffffffu, d3, o));
      f0 = fmaxf(f0, __shfl_xor_sync(0xffffffffu, f0, o));
      f1 = fmaxf(f1, __shfl_xor_sync(0xffffffffu, f1, o));
      i0 = max(i0, __shfl_xor_sync(0xffffffffu, i0, o));
      i1 += __shfl_xor_sync(0xffffffffu, i1, o);
      i2 += __shfl_xor_sync(0xffffffffu, i2, o);
    }
    if ((threadIdx.x & 31) == 0) {  // the warp's sums, in lane 0's own slots (thread 32 w)
      const int t = threadIdx.x;
      acc_d[t] = d0;
      acc_d[NT + t] = d1;
      acc_d[2 * NT + t] = d2;
      acc_d[3 * NT + t] = d3;
      acc_f[t] = f0;
      acc_f[NT + t] = f1;
      acc_i[t] = i0;
      acc_i[NT + t] = i1;
      acc_i[2 * NT + t] = i2;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll 1
    for (int w = 32; w < NT; w += 32) {
      acc_d[0] += acc_d[w];
      acc_d[NT] += acc_d[NT + w];
      acc_d[2 * NT] += acc_d[2 * NT + w];
      acc_d[3 * NT] = fmax(acc_d[3 * NT], acc_d[3 * NT + w]);
      acc_f[0] = fmaxf(acc_f[0], acc_f[w]);
      acc_f[NT] = fmaxf(acc_f[NT], acc_f[NT + w]);
      acc_i[0] = max(acc_i[0], acc_i[w]);
      acc_i[NT] += acc_i[NT + w];
      acc_i[2 * NT] += acc_i[2 * NT + w];
    }
  }
  if (threadIdx.x == 0) {
    ParticlePartial& P = part[tile];
    P.diss = acc_d[0];
    P.bbound = acc_d[NT];
    P.mass = acc_d[2 * NT];
    P.max_speed = acc_f[0];
    P.max_disp = acc_f[NT];
    P.fail = acc_i[0];
    P.iterations = acc_i[NT];
    P.yielded = acc_i[2 * NT];
    P.fail_value = acc_d[3 * NT];
    // the barrier above ordered every lane's write of defer_flag before this read
    if (defer_flag) defer_rec[atomicAdd(defer_count, 1u)] = rec;
  }
  if constexpr (CLOCKS) {
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(clk, (unsigned long long)(clock64() - clk_begin));
      atomicAdd(clk + 1, clk_newton);
    }
  }
}

// Persistent CTAs (as many as the launch shape asks, at most as many as fit the GPU at once)
// walk the attempt's list of occupied tiles; the partial results are per tile, so they do not
// depend on which CTA took which tile.  Both block shapes hold 16 warps per SM at the 128
// registers a thread needs.
template <bool WARM, int NT, int MINB = 512 / NT, bool CLOCKS = false, int KIND = G2P_MIXED>
__global__ void __launch_bounds__(NT, MINB)
    k_g2p(const InstDesc* __restrict__ desc, const Control* __restrict__ ctrl, float* __restrict__ st0,
          float* __restrict__ st1, uint32_t* __restrict__ id0, uint32_t* __restrict__ id1, int64_t cap,
          const uint32_t* __restrict__ perm, const float4* __restrict__ vel, ParticlePartial* __restrict__ part, const float* __restrict__ mlp_tab,
          float* __restrict__ log_x, float* __restrict__ log_y, unsigned long long* __restrict__ log_n,
          long long log_cap, const uint4* __restrict__ tile_rec, const uint32_t* __restrict__ tile_count,
          uint32_t* cursor, unsigned long long* __restrict__ clk, uint4* __restrict__ defer_rec,
          uint32_t* __restrict__ defer_count) {
  __shared__ uint32_t slot;
  const uint32_t n = *tile_count;
  for (uint32_t i = tile_first(cursor, &slot); i < n; i = tile_next(cursor, i, &slot)) {
    g2p_tile<WARM, NT, CLOCKS, KIND>(tile_rec[i], desc, ctrl, st0, st1, id0, id1, cap, perm, vel, part, mlp_tab, log_x,
                                     log_y, log_n, log_cap, clk, defer_rec, defer_count);
    __syncthreads();  // the next tile reuses the shared memory
  }
}

// The eigen-decomposition path of the paste update for the particles k_g2p left (DEFER_MARK in
// the trial state's tau_xx): one CTA per listed tile, over the tile's slots in order.  It
// finishes each such particle as k_g2p would have (the same paste_trial / warm start /
// paste_finish on the stored H_tr, with the call of paste_update_jacobi) and adds their plastic
// work, momentum bound, failure, Newton iterations and yield count to the tile's partial with a
// fixed-order block reduction, so the result does not depend on which CTA took the tile.
constexpr int G2P_DEFER_THREADS = 128;
template <bool WARM>
__global__ void __launch_bounds__(G2P_DEFER_THREADS)
    k_g2p_defer(const InstDesc* __restrict__ desc, const Control* __restrict__ ctrl, float* __restrict__ st0,
                float* __restrict__ st1, int64_t cap, ParticlePartial* __restrict__ part,
                const float* __restrict__ mlp_tab, float* __restrict__ log_x, float* __restrict__ log_y,
                unsigned long long* __restrict__ log_n, long long log_cap, const uint4* __restrict__ defer_rec,
                const uint32_t* __restrict__ defer_count) {
  constexpr int NT = G2P_DEFER_THREADS;
  __shared__ double shd[(NT / 32) * 6 + 6];
  const uint32_t n = *defer_count;
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const uint4 rec = defer_rec[i];
    const int tile = (int)rec.x, inst = (int)rec.y;
    const Control& c = ctrl[inst];
    const InstDesc& D = desc[inst];
    float* nxt = c.parity ? st0 : st1;  // the trial state k_g2p wrote
    const bool use_mlp = WARM && c.warm_start && mlp_tab != nullptr;
    const float2* tab =
        use_mlp ? reinterpret_cast<const float2*>(mlp_tab + (int64_t)inst * MLP_TAB_FLOATS + MLP_TAB_STRIDE) : nullptr;
    const float inv_k = (float)(1.0 / D.consistency);
    const float c_tau = (float)(D.max_dt * 4.0 / (D.dx * D.dx));
    const float c_dx = (float)(2.6 * D.dx);
    const float c_g =
        (float)(6.0 * sqrt(D.gravity[0] * D.gravity[0] + D.gravity[1] * D.gravity[1] + D.gravity[2] * D.gravity[2]) *
                D.max_dt);
    double diss = 0.0, bb = 0.0, fail_value = 0.0;
    int fail = F_OK, iters = 0, yielded = 0;
    for (int64_t k = (int64_t)rec.z + threadIdx.x; k < (int64_t)rec.w; k += NT) {
      if (__float_as_uint(nxt[C_TAU * cap + k]) != DEFER_MARK) continue;
      float Htr[9];
#pragma unroll
      for (int a = 0; a < 9; ++a) Htr[a] = nxt[(C_H + a) * cap + k];
      const double ys = D.per_particle_yield ? (double)nxt[C_YS * cap + k] : D.yield;
      PasteTrial pt;
      PasteOut o;
      paste_trial<false>(Htr, D.mu, pt, o);
      double sigma0 = -1.0;
      if (use_mlp && pt.path != PT_DONE && pt.trial_eq > ys && pt.trial_eq > 0.0) {
        const float t = mlp_table_fraction(tab, hb_la8(inv_k, pt.trial_eq, ys));
        if (t > 0.0f && t < 1.0f) sigma0 = ys + (double)t * (pt.trial_eq - ys);
      }
      paste_finish<false>(Htr, (float)D.mu, (float)D.lambda, D.mu, ys, c.hb, D.tol, sigma0, pt, o);
      if (o.fail != F_OK) {
        fail = max(fail, o.fail);
        fail_value = o.eq;
      }
#pragma unroll
      for (int a = 0; a < 9; ++a) nxt[(C_H + a) * cap + k] = o.H[a];
#pragma unroll
      for (int a = 0; a < 6; ++a) nxt[(C_TAU + a) * cap + k] = o.tau[a];
      nxt[C_EP * cap + k] += (float)o.dep;
      const float v0 = nxt[C_V0 * cap + k], m = nxt[C_M * cap + k];
      diss += o.diss_density * (double)v0;
      iters += o.iters;
      yielded += o.yielded;
      if (log_n != nullptr && o.yielded && o.fail == F_OK) {
        const unsigned long long slot = atomicAdd(log_n, 1ull);
        if ((long long)slot < log_cap) {
          log_x[6 * slot + 0] = (float)o.trial;
          log_x[6 * slot + 1] = (float)ys;
          log_x[6 * slot + 2] = (float)D.consistency;
          log_x[6 * slot + 3] = (float)D.flow_index;
          log_x[6 * slot + 4] = (float)D.mu;
          log_x[6 * slot + 5] = (float)c.dt;
          log_y[slot] = (float)o.eq;
        }
      }
      // the momentum bound k_g2p left out, from the stored velocity and affine field
      float v[3], Cm[9];
#pragma unroll
      for (int a = 0; a < 3; ++a) v[a] = nxt[(C_V + a) * cap + k];
#pragma unroll
      for (int a = 0; a < 9; ++a) Cm[a] = nxt[(C_C + a) * cap + k];
      bb += momentum_bound(m, particle_speed(v), affine_norm(Cm), o.tau, v0, c_tau, c_dx, c_g);
    }
    double rv[6] = {diss, bb, (double)fail, (double)iters, (double)yielded, fail_value};
    block_reduce_multi_to0<NT, 6>(rv, (1u << 2) | (1u << 5), shd);
    if (threadIdx.x == 0) {
      ParticlePartial& P = part[tile];
      P.diss += rv[0];
      P.bbound += rv[1];
      P.fail = max(P.fail, (int)rv[2]);
      P.iterations += (int)rv[3];
      P.yielded += (int)rv[4];
      P.fail_value = fmax(P.fail_value, rv[5]);
    }
    __syncthreads();  // shd is reused by the next tile
  }
}

// Warm-start table, one CTA per instance: the tensor-core network pass at the MLP_TAB_N nodes
// of la8 with the instance's material constants and this attempt's dt, then the root fractions.  A
// table built for the same dt is kept (tab_dt holds the dt of each built table; the host sets it
// to NaN when the weights change).
constexpr int MLP_TAB_THREADS = 256;
__global__ void __launch_bounds__(MLP_TAB_THREADS) k_mlp_table(const InstDesc* __restrict__ desc,
                                                               const Control* __restrict__ ctrl,
                                                               const MlpPacked* __restrict__ mlp,
                                                               float* __restrict__ tab, double* __restrict__ tab_dt) {
  __shared__ MlpPacked w;
  __shared__ uint32_t xs[(MLP_TAB_THREADS / 32) * MLP_XS_WORDS];
  const int inst = blockIdx.x;
  const Control& c = ctrl[inst];
  const InstDesc& D = desc[inst];
  if (!c.active || !c.warm_start || D.kind != 0 || tab_dt[inst] == c.dt) return;  // CTA-uniform
  mlp_stage(mlp, w);
  const HbFeatureConst h = hb_feature_const(D.consistency, D.flow_index, D.mu, c.dt);
  __syncthreads();
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* out = tab + (int64_t)inst * MLP_TAB_FLOATS;
  for (int r0 = wid * 32; r0 < MLP_TAB_N; r0 += MLP_TAB_THREADS) {  // warp-uniform
    const int r = r0 + lane;
    float f[6];
    hb_features_la8(h, mlp_table_node(min(r, MLP_TAB_N - 1)), f);
    const float y = warp_mlp_logit(w, xs + wid * MLP_XS_WORDS, f);
    if (r < MLP_TAB_N) out[r] = y;
  }
  __syncthreads();
  // root fractions and their node differences (the sigmoid of warm_fraction_of)
  float2* pairs = reinterpret_cast<float2*>(out + MLP_TAB_STRIDE);
  for (int r = threadIdx.x; r < MLP_TAB_N; r += MLP_TAB_THREADS) {
    const float t0 = 1.0f / (1.0f + __expf(-out[r]));
    const float t1 = r + 1 < MLP_TAB_N ? 1.0f / (1.0f + __expf(-out[r + 1])) : t0;
    pairs[r] = make_float2(t0, t1 - t0);
  }
  __syncthreads();
  if (threadIdx.x == 0) tab_dt[inst] = c.dt;
}

// ============================================================== end of attempt
// Level 1: one CTA per segment of at most SEG_SPAN grid or particle partials of one instance,
// reduced in a fixed order.  Level 2 (k_end): the instance's segments in order.
__global__ void k_segments(const Control* __restrict__ ctrl, const SegDesc* __restrict__ segs,
                           const GridPartial* __restrict__ gpart, const ParticlePartial* __restrict__ ppart,
                           SegPartial* __restrict__ out) {
  __shared__ double shd[(256 / 32) * 13 + 13];
  const SegDesc sd = segs[blockIdx.x];
  if (!ctrl[sd.inst].active) return;
  const int t = threadIdx.x;
  // sums: wi0 wi1 wi2 proj fric trac diss bb its yl; max: ms md fail
  double v[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (sd.kind == 0) {
    for (int64_t j = sd.begin + t; j < sd.end; j += 256) {
      const GridPartial& P = gpart[j];
      v[0] += P.wall_impulse[0];
      v[1] += P.wall_impulse[1];
      v[2] += P.wall_impulse[2];
      v[3] += P.proj;
      v[4] += P.fric;
      v[5] += P.trac;
      v[12] = fmax(v[12], (double)P.fail);
    }
  } else {
    for (int64_t j = sd.begin + t; j < sd.end; j += 256) {
      const ParticlePartial& P = ppart[j];
      v[6] += P.diss;
      v[7] += P.bbound;
      v[8] += (double)P.iterations;
      v[9] += (double)P.yielded;
      v[10] = fmax(v[10], (double)P.max_speed);
      v[11] = fmax(v[11], (double)P.max_disp);
      v[12] = fmax(v[12], (double)P.fail);
    }
  }
  block_reduce_multi_to0<256, 13>(v, (1u << 10) | (1u << 11) | (1u << 12), shd);
  if (t == 0) {
    SegPartial& o = out[blockIdx.x];
    for (int k = 0; k < 13; ++k) o.v[k] = v[k];
  }
}

__global__ void k_end(const InstDesc* __restrict__ desc, Control* __restrict__ ctrl,
                      const SegPartial* __restrict__ seg, const BedStep* __restrict__ bed_step, BedPtrs bed) {
  __shared__ double shd[(256 / 32) * 18 + 18];
  const int inst = blockIdx.x;
  Control& c = ctrl[inst];
  if (!c.active) return;
  const InstDesc& D = desc[inst];
  const int t = threadIdx.x;
  // v: wi0 wi1 wi2 proj fric trac diss bb its yl | ms md | grid fail, particle fail (max)
  double v[14] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t j = t; j < D.seg_cnt; j += 256) {
    const SegPartial& P = seg[D.seg_off + j];
    const bool grid = j < D.seg_cnt_g;
    for (int k = 0; k < 10; ++k) v[k] += P.v[k];
    v[10] = fmax(v[10], P.v[10]);
    v[11] = fmax(v[11], P.v[11]);
    if (grid) v[12] = fmax(v[12], P.v[12]);
    else v[13] = fmax(v[13], P.v[12]);
  }
  block_reduce_multi<256, 14>(v, (1u << 10) | (1u << 11) | (1u << 12) | (1u << 13), shd);
  // pellet bed: imp3 ang3 cgrid cpellet wimp3 wwork ppwork contacts overflow mass | fail (max)
  double bv[18] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1e300};
  if (D.bed_np >= 2) {
    const PelletState* S = bed.state[c.bed_parity] + D.bed_off;
    for (int p = t; p < D.bed_np; p += 256) {
      const BedStep& B = bed_step[D.bed_off + p];
      for (int a = 0; a < 3; ++a) {
        bv[a] += B.imp[a];
        bv[3 + a] += B.ang[a];
        bv[8 + a] += B.wimp[a];
      }
      bv[6] += B.cgrid;
      bv[7] += B.cpellet;
      bv[11] += B.wwork;
      bv[12] += B.ppwork;
      bv[13] += (double)B.contacts;
      bv[14] += (double)B.overflow;
      bv[15] += S[p].mass;
      bv[16] = fmax(bv[16], (double)B.fail);
      bv[17] = fmax(bv[17], -B.limit);  // smallest step limit of the trial pellets
    }
    block_reduce_multi<256, 18>(bv, (1u << 16) | (1u << 17), shd);
  }
  if (t != 0) return;
  const double wi[3] = {v[0], v[1], v[2]};
  const double proj = v[3], fric = v[4], trac = v[5], diss = v[6], bb = v[7];
  const long long its = (long long)v[8], yl = (long long)v[9];
  const float ms = (float)v[10], md = (float)v[11];
  const int fail = (int)v[12], pfail = (int)v[13];
  c.step_diss = diss;
  int f = F_OK;
  if (!isfinite(trac) || !isfinite(c.ledger.trac + trac)) f = F_TRACTION_NONFINITE;
  else if (!isfinite(c.bbound)) f = F_GRID_NONFINITE;  // the deposit could not be represented
  else if (fail != F_OK) f = fail;
  else if (D.has_pellet && c.pellet_fail) f = F_PELLET_NONFINITE;
  else if (D.bed_np >= 2 && bv[16] > 0.0) f = F_PELLET_NONFINITE;
  else if (pfail != F_OK) f = pfail;
  else if (md > 1.0f) f = F_DISPLACEMENT;
  else if (c.outflow > 0) f = F_OUTFLOW;
  const bool forced = c.forced_dt > 0.0;
  if (f != F_OK) {
    c.fail = f;
    c.last_fail = f;
    c.fail_value = f == F_DISPLACEMENT ? (double)md : 0.0;
    if (f == F_OUTFLOW) {
      c.status = S_ERROR;
      return;
    }
    if (!forced) {
      c.rejected_steps += 1;
      c.dt_scale *= 0.5;
      if (c.dt_scale * c.limit < D.min_dt) c.status = S_MIN_STEP;
    }
    return;
  }
  // commit (solver.rs:980-998 + pellet ledger of try_step_captured)
  const double dt = c.dt;
  c.parity ^= 1;
  LedgerD& L = c.ledger;
  L.plastic += diss;
  for (int a = 0; a < 3; ++a) L.wall_impulse[a] += wi[a];
  L.proj += proj;
  L.fric += fric;
  L.trac += trac;
  for (int a = 0; a < 3; ++a) L.gravity_impulse[a] += D.gravity[a] * (c.total_mass * dt);
  if (D.has_pellet) {
    for (int a = 0; a < 3; ++a) {
      L.gravity_impulse[a] += D.gravity[a] * (c.pellet_trial.mass * dt);
      L.pellet_wall_impulse[a] += c.pw_impulse[a];
      L.coupling_impulse[a] += c.c_impulse[a];
      L.coupling_angular[a] += c.c_angular[a];
    }
    L.pellet_work += c.pw_work;
    L.cgrid += c.c_grid_energy;
    L.cpellet += c.c_pellet_energy;
    c.pellet = c.pellet_trial;
  }
  if (D.bed_np >= 2) {
    for (int a = 0; a < 3; ++a) {
      L.gravity_impulse[a] += D.gravity[a] * (bv[15] * dt);
      L.pellet_wall_impulse[a] += bv[8 + a];
      L.coupling_impulse[a] += bv[a];
      L.coupling_angular[a] += bv[3 + a];
    }
    L.pellet_work += bv[11];
    L.cgrid += bv[6];
    L.cpellet += bv[7];
    c.bed_contact_work += bv[12];
    c.bed_contacts = (int)bv[13];
    c.bed_overflow += (uint64_t)bv[14];
    c.bed_limit = -bv[17];
    c.bed_parity ^= 1;
  }
  c.max_speed = ms;
  c.bbound = bb;
  c.newton_iterations += (uint64_t)its;
  c.yielded = (uint64_t)yl;
  if (!forced) {
    c.time += dt;
    c.step_count += 1;
    c.limited_steps += (uint64_t)c.limited;
    c.min_dt_used = fmin(c.min_dt_used, dt);
    c.max_dt_used = fmax(c.max_dt_used, dt);
    c.dt_scale = fmin(c.dt_scale * 1.25, 1.0);
    if (!(c.time < c.target)) {
      c.time = c.target;
      c.status = S_REACHED;
    }
  }
}

// ============================================================== setup / diagnostics
// Committed-state reductions: max speed and the momentum bound (used by k_begin), FP64.
__global__ void k_state_stats(const InstDesc* __restrict__ desc, const Control* __restrict__ ctrl,
                              const int* __restrict__ pcta_inst, const float* __restrict__ st0,
                              const float* __restrict__ st1, int64_t cap, ParticlePartial* __restrict__ part) {
  __shared__ double shd[G2P_THREADS];
  __shared__ float shf[G2P_THREADS];
  const int inst = pcta_inst[blockIdx.x];
  const Control& c = ctrl[inst];
  const InstDesc& D = desc[inst];
  const int64_t k = (int64_t)blockIdx.x * G2P_THREADS + threadIdx.x;
  double bb = 0.0, ms = 0.0;
  float sp = 0.0f;
  if (k - D.slot_off < c.count) {
    const float* cur = c.parity ? st1 : st0;
    float v[3], Cm[9], tau[6];
    for (int a = 0; a < 3; ++a) v[a] = cur[(C_V + a) * cap + k];
    for (int a = 0; a < 9; ++a) Cm[a] = cur[(C_C + a) * cap + k];
    for (int a = 0; a < 6; ++a) tau[a] = cur[(C_TAU + a) * cap + k];
    const float m = cur[C_M * cap + k], v0 = cur[C_V0 * cap + k];
    // the same FP32 expressions as the end of k_g2p, so that a state imported from a
    // checkpoint gets the same speed and per-particle bound as the run that wrote it
    const float speed = particle_speed(v);
    const float c_tau = (float)(D.max_dt * 4.0 / (D.dx * D.dx));
    const float c_dx = (float)(2.6 * D.dx);
    const float c_g =
        (float)(6.0 * sqrt(D.gravity[0] * D.gravity[0] + D.gravity[1] * D.gravity[1] + D.gravity[2] * D.gravity[2]) *
                D.max_dt);
    bb = momentum_bound(m, speed, affine_norm(Cm), tau, v0, c_tau, c_dx, c_g);
    sp = speed;
    ms = (double)m;
  }
  bb = block_sum_d<G2P_THREADS>(bb, shd);
  ms = block_sum_d<G2P_THREADS>(ms, shd);
  sp = block_max_f<G2P_THREADS>(sp, shf);
  if (threadIdx.x == 0) {
    ParticlePartial& P = part[blockIdx.x];
    P.bbound = bb;
    P.mass = ms;
    P.max_speed = sp;
    P.diss = 0.0;
    P.max_disp = 0.f;
    P.fail = 0;
    P.iterations = 0;
    P.yielded = 0;
  }
}

// Energies and observables of the committed state (FP64 partials per CTA).
// out per CTA (DIAG_N doubles): ke, pe, ee, mass, mom xyz, max speed, max ep, yielded count,
// min x, max x, min y, max y, max z, hydro sum sq, hydro max, column height (dam break),
// sum of m |C|^2 (the APIC affine norm before its h^2/8 factor)
__global__ void k_diagnostics(const InstDesc* __restrict__ desc, const Control* __restrict__ ctrl,
                              const int* __restrict__ pcta_inst, const float* __restrict__ st0,
                              const float* __restrict__ st1, int64_t cap, int fixture_hydro, double h0,
                              int fixture_dam, double* __restrict__ out) {
  __shared__ double shd[G2P_THREADS];
  const int inst = pcta_inst[blockIdx.x];
  const Control& c = ctrl[inst];
  const InstDesc& D = desc[inst];
  const int64_t k = (int64_t)blockIdx.x * G2P_THREADS + threadIdx.x;
  double vals[DIAG_N];
  for (int j = 0; j < DIAG_N; ++j) vals[j] = 0.0;
  vals[9] = 1e300;
  vals[10] = -1e300;
  vals[11] = 1e300;
  vals[12] = -1e300;
  vals[13] = -1e300;
  if (k - D.slot_off < c.count) {
    const float* cur = c.parity ? st1 : st0;
    double x[3], v[3];
    for (int a = 0; a < 3; ++a) {
      x[a] = cur[(C_X + a) * cap + k];
      v[a] = cur[(C_V + a) * cap + k];
    }
    const double m = cur[C_M * cap + k], v0 = cur[C_V0 * cap + k];
    const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    vals[0] = 0.5 * m * v2;
    vals[1] = -m * (D.gravity[0] * x[0] + D.gravity[1] * x[1] + D.gravity[2] * x[2]);
    if (D.kind == 0) {
      float Hh[9];
      for (int a = 0; a < 9; ++a) Hh[a] = cur[(C_H + a) * cap + k];
      double B[3][3], U[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double hh = (double)Hh[3 * i] * Hh[3 * j] + (double)Hh[3 * i + 1] * Hh[3 * j + 1] +
                      (double)Hh[3 * i + 2] * Hh[3 * j + 2];
          B[i][j] = (double)Hh[3 * i + j] + (double)Hh[3 * j + i] + hh;
        }
      double e = 0.0;
      if (jacobi3<double>(B, U, 64, 1e-30)) {
        double h[3], tr = 0.0, n2 = 0.0;
        for (int a = 0; a < 3; ++a) {
          h[a] = 0.5 * log1p(fmax(B[a][a], -1.0 + 1e-300));
          tr += h[a];
          n2 += h[a] * h[a];
        }
        e = v0 * (D.mu * n2 + 0.5 * D.lambda * tr * tr);
      } else {
        e = nan("");
      }
      vals[2] = e;
    } else {
      const double jm1 = cur[C_JM1 * cap + k];
      const double j = 1.0 + jm1;
      vals[2] = v0 * D.bulk * (jm1 - log1p(jm1));
      (void)j;
    }
    vals[3] = m;
    vals[4] = m * v[0];
    vals[5] = m * v[1];
    vals[6] = m * v[2];
    vals[7] = sqrt(v2);
    const double ep = cur[C_EP * cap + k];
    vals[8] = ep;
    vals[14] = ep > 0.0 ? 1.0 : 0.0;
    vals[9] = x[0];
    vals[10] = x[0];
    vals[11] = x[1];
    vals[12] = x[1];
    vals[13] = x[2];
    if (fixture_hydro) {
      const double g = sqrt(D.gravity[0] * D.gravity[0] + D.gravity[1] * D.gravity[1] + D.gravity[2] * D.gravity[2]);
      const double depth = fmax(h0 - x[2], 0.0);
      double ref, meas;
      if (D.kind == 1) {
        ref = D.bulk * expm1(D.density * g * depth / D.bulk);
        const double jm1 = cur[C_JM1 * cap + k];
        meas = D.tait_gamma == 1.0 ? -D.bulk * jm1 / (1.0 + jm1) : D.bulk / D.tait_gamma * expm1(-D.tait_gamma * log1p(jm1));
      } else {
        ref = D.density * g * depth;
        meas = -(double)cur[(C_TAU + 2) * cap + k];
      }
      const double scale = D.density * g * h0;
      const double er = (meas - ref) / scale;
      vals[15] = er * er;
      vals[16] = fabs(er);
    }
    if (fixture_dam && x[0] < D.dx) vals[17] = x[2];
    else vals[17] = -1e300;
    double c2 = 0.0;
    for (int a = 0; a < 9; ++a) {
      const double ca = cur[(C_C + a) * cap + k];
      c2 += ca * ca;
    }
    vals[18] = m * c2;
  } else {
    vals[17] = -1e300;
  }
  // reduce: sums 0-6, 14, 15, 18; max 7, 8, 10, 12, 13, 16, 17; min 9, 11
  for (int j = 0; j < DIAG_N; ++j) {
    const int t = threadIdx.x;
    shd[t] = vals[j];
    __syncthreads();
    for (int s = G2P_THREADS / 2; s > 0; s >>= 1) {
      if (t < s) {
        const double a = shd[t], b = shd[t + s];
        double r;
        if (j <= 6 || j == 14 || j == 15 || j == 18) r = a + b;
        else if (j == 9 || j == 11) r = fmin(a, b);
        else r = fmax(a, b);
        shd[t] = r;
      }
      __syncthreads();
    }
    if (t == 0) out[(int64_t)blockIdx.x * DIAG_N + j] = shd[0];
    __syncthreads();
  }
}


// ============================================================== host-layout import / export
// Conversion between the reference's FP64 particle arrays (ParticleSet layout, matrices
// row-major) staged in device memory and the FP32 component-major state, one thread per
// particle of a chunk.  The FP64 -> FP32 roundings are those of a host-side cast.
__global__ void k_import(HostParticleChunk h, int64_t n, int64_t first, float* __restrict__ dst,
                         uint32_t* __restrict__ ids, int64_t cap, int64_t slot_off, double yield_default,
                         unsigned long long* __restrict__ bad) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int64_t k = slot_off + first + p;
  bool ok = isfinite(h.mass[p]) && h.mass[p] > 0.0 && isfinite(h.volume0[p]) && h.volume0[p] > 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double x = h.position[3 * p + a], v = h.velocity[3 * p + a];
    ok = ok && isfinite(x) && isfinite(v);
    dst[(C_X + a) * cap + k] = (float)x;
    dst[(C_V + a) * cap + k] = (float)v;
  }
  if (!ok) atomicMin(bad, (unsigned long long)(first + p));
#pragma unroll
  for (int a = 0; a < 9; ++a) {
    dst[(C_C + a) * cap + k] = (float)h.affine[9 * p + a];
    dst[(C_H + a) * cap + k] = (float)(h.deformation[9 * p + a] - ((a % 4) == 0 ? 1.0 : 0.0));
  }
  const double* T = h.kirchhoff + 9 * p;
  dst[(C_TAU + 0) * cap + k] = (float)T[0];
  dst[(C_TAU + 1) * cap + k] = (float)T[4];
  dst[(C_TAU + 2) * cap + k] = (float)T[8];
  dst[(C_TAU + 3) * cap + k] = (float)(0.5 * (T[1] + T[3]));
  dst[(C_TAU + 4) * cap + k] = (float)(0.5 * (T[2] + T[6]));
  dst[(C_TAU + 5) * cap + k] = (float)(0.5 * (T[5] + T[7]));
  dst[C_EP * cap + k] = (float)h.plastic_strain[p];
  dst[C_M * cap + k] = (float)h.mass[p];
  dst[C_V0 * cap + k] = (float)h.volume0[p];
  dst[C_YS * cap + k] = (float)(h.yield_stress ? h.yield_stress[p] : yield_default);
  dst[C_JM1 * cap + k] = (float)(h.volume_ratio[p] - 1.0);
  ids[k] = h.id[p];
}

__global__ void k_export(HostParticleChunk h, int64_t n, int64_t first, const float* __restrict__ src,
                         const uint32_t* __restrict__ ids, int64_t cap, int64_t slot_off, int paste,
                         int per_particle_yield, double yield_default) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int64_t k = slot_off + first + p;
  auto g = [&](int comp) { return (double)src[comp * cap + k]; };
  h.id[p] = ids[k];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    h.position[3 * p + a] = g(C_X + a);
    h.velocity[3 * p + a] = g(C_V + a);
  }
#pragma unroll
  for (int a = 0; a < 9; ++a) {
    const double eye = (a % 4) == 0 ? 1.0 : 0.0;
    h.affine[9 * p + a] = g(C_C + a);
    h.deformation[9 * p + a] = paste ? g(C_H + a) + eye : eye;
  }
  const int map[9] = {0, 3, 4, 3, 1, 5, 4, 5, 2};
#pragma unroll
  for (int a = 0; a < 9; ++a) h.kirchhoff[9 * p + a] = g(C_TAU + map[a]);
  h.volume_ratio[p] = paste ? 1.0 : 1.0 + g(C_JM1);
  h.plastic_strain[p] = g(C_EP);
  h.mass[p] = g(C_M);
  h.volume0[p] = g(C_V0);
  h.yield_stress[p] = per_particle_yield ? g(C_YS) : yield_default;
}

// ============================================================== unit kernels (host arrays API)
// One return problem per lane; with weights, each warp starts its lanes' Newton solves from one
// tensor-core network pass (the same call as in k_g2p).
__global__ void __launch_bounds__(128) k_hb_batch(int64_t n, const double* trial, const double* ys, const double* k,
                                                  const double* nn, const double* mu, const double* dt, double tol,
                                                  const MlpPacked* mlp, double* out, int* status) {
  __shared__ MlpPacked mlp_s;
  __shared__ uint32_t mlp_xs[4 * MLP_XS_WORDS];
  if (mlp != nullptr) mlp_stage(mlp, mlp_s);
  __syncthreads();
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u) >= n) return;  // warp-uniform
  const bool valid = i0 < n;
  const int64_t i = valid ? i0 : n - 1;
  double sigma0 = -1.0;
  if (mlp != nullptr) {
    const bool need = valid && trial[i] > ys[i] && k[i] > 0.0;
    if (__any_sync(0xffffffffu, need)) {
      float f[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (need) hb_features(trial[i], ys[i], k[i], nn[i], mu[i], dt[i], f);
      const float y = warp_mlp_logit(mlp_s, mlp_xs + (threadIdx.x >> 5) * MLP_XS_WORDS, f);
      const double frac = warm_fraction_of(y);
      if (need && frac > 0.0) sigma0 = ys[i] + frac * (trial[i] - ys[i]);
    }
  }
  if (!valid) return;
  double sigma = 0.0, dep = 0.0;
  int it = 0;
  status[i] = hb_return_d(trial[i], ys[i], k[i], nn[i], mu[i], dt[i], tol, sigma0, &sigma, &dep, &it);
  out[3 * i + 0] = sigma;
  out[3 * i + 1] = dep;
  out[3 * i + 2] = (double)it;
}
__global__ void k_paste_batch(int64_t n, const double* f, double mu, double lambda, double ys, double k, double nn,
                              double dt, double tol, double* fnew, double* tau, double* scal, int* status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float Htr[9];
  for (int a = 0; a < 9; ++a) Htr[a] = (float)(f[9 * i + a] - ((a % 4) == 0 ? 1.0 : 0.0));
  PasteOut o;
  paste_update(Htr, (float)mu, (float)lambda, mu, ys, k, nn, dt, tol, o);
  status[i] = o.fail;
  if (o.fail != F_OK) return;
  for (int a = 0; a < 9; ++a) fnew[9 * i + a] = (double)o.H[a] + ((a % 4) == 0 ? 1.0 : 0.0);
  const int map[9] = {0, 3, 4, 3, 1, 5, 4, 5, 2};
  for (int a = 0; a < 9; ++a) tau[9 * i + a] = o.tau[map[a]];
  scal[3 * i + 0] = o.dep;
  scal[3 * i + 1] = o.diss_density;
  scal[3 * i + 2] = o.eq;
}
__global__ void k_liquid_batch(int64_t n, const double* j, const double* grad, double bulk, double visc,
                               double gamma, double dt, double* jnew, double* tau, double* p, int* status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float C[9];
  for (int a = 0; a < 9; ++a) C[a] = (float)grad[9 * i + a];
  LiquidOut o;
  liquid_update((float)(j[i] - 1.0), C, (float)bulk, (float)visc, (float)gamma, (float)dt, o);
  status[i] = o.fail;
  if (o.fail != F_OK) return;
  jnew[i] = 1.0 + (double)o.jm1;
  const int map[9] = {0, 3, 4, 3, 1, 5, 4, 5, 2};
  for (int a = 0; a < 9; ++a) tau[9 * i + a] = o.tau[map[a]];
  p[i] = o.pressure;
}

// ============================================================== launchers
static uint64_t g_launches = 0;

static inline unsigned grid_of(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// Resident CTAs per SM of the persistent kernels' instantiations (from the occupancy calculator;
// the defaults are the B200 figures) and the SM count.
static int g_sms = 148, g_sort_per_sm = 16;
static int g_p2g_per_sm[P2G_VARIANTS] = {2, 2, 2};  // [p2g_variant]
// [kind][g2p_variant][warm] (mixed-kind ensembles run the 256-thread instantiation, variant 0)
static int g_g2p_per_sm[3][G2P_VARIANTS][2] = {{{2, 2}, {4, 4}, {5, 5}, {6, 6}},
                                               {{2, 2}, {4, 4}, {5, 5}, {6, 6}},
                                               {{2, 2}, {2, 2}, {2, 2}, {2, 2}}};

// The G2P instantiation of a kind, launch-shape variant and warm start (liquid: no warm start;
// mixed kinds: the 256-thread block shape whatever the variant), as a function pointer.
template <int KIND>
static const void* g2p_fn(int v, bool warm) {
  if constexpr (KIND == G2P_MIXED) {
    return warm ? (const void*)k_g2p<true, G2P_THREADS, 2, false, KIND> : (const void*)k_g2p<false, G2P_THREADS, 2, false, KIND>;
  } else {
    constexpr bool W = KIND == G2P_PASTE;  // the warm instantiations exist for paste only
    if (v == 3) return (warm && W) ? (const void*)k_g2p<W, G2P_THREADS_SMALL, 6, false, KIND> : (const void*)k_g2p<false, G2P_THREADS_SMALL, 6, false, KIND>;
    if (v == 2) return (warm && W) ? (const void*)k_g2p<W, G2P_THREADS_SMALL, 5, false, KIND> : (const void*)k_g2p<false, G2P_THREADS_SMALL, 5, false, KIND>;
    if (v == 1) return (warm && W) ? (const void*)k_g2p<W, G2P_THREADS_SMALL, 4, false, KIND> : (const void*)k_g2p<false, G2P_THREADS_SMALL, 4, false, KIND>;
    return (warm && W) ? (const void*)k_g2p<W, G2P_THREADS, 2, false, KIND> : (const void*)k_g2p<false, G2P_THREADS, 2, false, KIND>;
  }
}
static const void* g2p_fn(int kind, int v, bool warm) {
  return kind == G2P_PASTE ? g2p_fn<G2P_PASTE>(v, warm) : (kind == G2P_LIQUID ? g2p_fn<G2P_LIQUID>(v, false) : g2p_fn<G2P_MIXED>(v, warm));
}
static int g2p_fn_threads(int kind, int v) { return kind == G2P_MIXED ? G2P_THREADS : g2p_threads(v); }

// dynamic shared memory of each P2G variant: records / partials, plus the staged copies
static size_t p2g_variant_smem(int v) {
  return v == 0 ? p2g_smem(P2G_CHUNK) : p2g_smem(P2G_CHUNK_SMALL) + (v == 2 ? p2g_raw_bytes(P2G_CHUNK_SMALL) : 0);
}

static void occupancy(int* out, const void* fn, int threads, size_t smem) {
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem) == cudaSuccess && per > 0) *out = per;
}

void configure_kernels() {
  const void* p2g[P2G_VARIANTS] = {(const void*)k_p2g<P2G_CHUNK, false>, (const void*)k_p2g<P2G_CHUNK_SMALL, false>,
                                   (const void*)k_p2g<P2G_CHUNK_SMALL, true>};
  for (int v = 0; v < P2G_VARIANTS; ++v)
    cudaFuncSetAttribute(p2g[v], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p2g_variant_smem(v));
  for (int k = 0; k < 3; ++k)
    for (int v = 0; v < G2P_VARIANTS; ++v)
      for (int w = 0; w < 2; ++w)
        cudaFuncSetAttribute(g2p_fn(k, v, w), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)g2p_smem(g2p_fn_threads(k, v)));
  // the clock-instrumented instantiations of the return-share measurement (any kind)
  const void* g2p_clk[2] = {(const void*)k_g2p<false, G2P_THREADS, 2, true>,
                            (const void*)k_g2p<true, G2P_THREADS, 2, true>};
  for (const void* f : g2p_clk)
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g2p_smem(G2P_THREADS));
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return;
  g_sms = sms;
  occupancy(&g_sort_per_sm, (const void*)k_bin_sort, TB, 0);
  for (int v = 0; v < P2G_VARIANTS; ++v) occupancy(&g_p2g_per_sm[v], p2g[v], P2G_THREADS, p2g_variant_smem(v));
  for (int k = 0; k < 3; ++k)
    for (int v = 0; v < G2P_VARIANTS; ++v)
      for (int w = 0; w < 2; ++w)
        occupancy(&g_g2p_per_sm[k][v][w], g2p_fn(k, v, w), g2p_fn_threads(k, v), g2p_smem(g2p_fn_threads(k, v)));
}

// persistent grid size: the requested CTAs per SM, at most the resident limit, times the SMs
static unsigned persistent_ctas(int requested, int limit) {
  const int per = (requested > 0 && requested < limit) ? requested : limit;
  return (unsigned)(per * g_sms);
}

int launch_shape_limits(int out[LAUNCH_LIMITS]) {
  out[0] = g_sms;
  out[1] = g_sort_per_sm;
  for (int v = 0; v < P2G_VARIANTS; ++v) out[LIM_P2G + v] = g_p2g_per_sm[v];
  for (int v = 0; v < G2P_VARIANTS; ++v) out[LIM_G2P + v] = g_g2p_per_sm[G2P_PASTE][v][1];
  return LAUNCH_LIMITS;
}

// the occupied-tile list, then P2G over it
static int launch_tiles_p2g(const DeviceArrays& A, cudaStream_t s, int transport_only, cudaEvent_t* ev, int& n) {
  const LaunchShape& L = A.shape;
  uint32_t* cur = L.dynamic ? A.nw_count + 2 : nullptr;  // cursors: [0] bin sort, [1] P2G, [2] G2P
  k_tiles<<<grid_of(A.n_tiles, 256), 256, 0, s>>>(A.desc, A.ctrl, A.tile_inst, A.n_tiles, A.start, A.tile_rec,
                                                   A.tile_count, A.tpart);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  k_bin_sort<<<(unsigned)(g_sort_per_sm * g_sms), TB, 0, s>>>(A.desc, A.start, A.perm, A.tile_rec, A.tile_count,
                                                               cur);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  const int v = (L.p2g_variant >= 0 && L.p2g_variant < P2G_VARIANTS) ? L.p2g_variant : 0;
  const unsigned ctas = persistent_ctas(L.p2g_per_sm, g_p2g_per_sm[v]);
  uint32_t* pc = cur ? cur + 1 : nullptr;
#define LP_P2G_ARGS                                                                                          \
  A.desc, A.ctrl, A.st[0], A.st[1], A.cap, A.start, A.perm, A.acc, A.node_total, A.blk_epoch, transport_only, \
      A.tile_rec, A.tile_count, pc
  if (v == 2) k_p2g<P2G_CHUNK_SMALL, true><<<ctas, P2G_THREADS, p2g_variant_smem(2), s>>>(LP_P2G_ARGS);
  else if (v == 1) k_p2g<P2G_CHUNK_SMALL, false><<<ctas, P2G_THREADS, p2g_variant_smem(1), s>>>(LP_P2G_ARGS);
  else k_p2g<P2G_CHUNK, false><<<ctas, P2G_THREADS, p2g_variant_smem(0), s>>>(LP_P2G_ARGS);
#undef LP_P2G_ARGS
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  return 3;
}

// G2P in the launch shape's instantiation for the ensemble's material kinds
template <int KIND>
static void launch_g2p_kind(const DeviceArrays& A, bool warm, cudaStream_t s) {
  const LaunchShape& L = A.shape;
  uint32_t* cur = L.dynamic ? A.nw_count + 4 : nullptr;
  const float* tab = warm ? A.mlp_tab : nullptr;
  const int v = (L.g2p_variant >= 0 && L.g2p_variant < G2P_VARIANTS) ? L.g2p_variant : 0;
  const unsigned ctas = persistent_ctas(L.g2p_per_sm, g_g2p_per_sm[KIND][v][warm ? 1 : 0]);
#define LP_G2P_ARGS                                                                                               \
  A.desc, A.ctrl, A.st[0], A.st[1], A.id[0], A.id[1], A.cap, A.perm, A.vel, A.tpart, tab, A.log_x, A.log_y, \
      A.log_n, A.log_cap, A.tile_rec, A.tile_count, cur, A.g2p_clk, A.defer_rec, A.nw_count + 5
#define LP_G2P_LAUNCH(T, MB)                                                                                 \
  (warm ? k_g2p<KIND == G2P_LIQUID ? false : true, T, MB, false, KIND> : k_g2p<false, T, MB, false, KIND>) \
      <<<ctas, T, g2p_smem(T), s>>>(LP_G2P_ARGS)
  if constexpr (KIND == G2P_MIXED) {
    LP_G2P_LAUNCH(G2P_THREADS, 2);
  } else {
    if (v == 3) LP_G2P_LAUNCH(G2P_THREADS_SMALL, 6);
    else if (v == 2) LP_G2P_LAUNCH(G2P_THREADS_SMALL, 5);
    else if (v == 1) LP_G2P_LAUNCH(G2P_THREADS_SMALL, 4);
    else LP_G2P_LAUNCH(G2P_THREADS, 2);
  }
#undef LP_G2P_LAUNCH
#undef LP_G2P_ARGS
}
static void launch_g2p(const DeviceArrays& A, bool warm, cudaStream_t s) {
  if (A.g2p_clk) {  // measurement of the return's share of G2P warp time (256-thread CTAs, any kind)
    const LaunchShape& L = A.shape;
    uint32_t* cur = L.dynamic ? A.nw_count + 4 : nullptr;
    const float* tab = warm ? A.mlp_tab : nullptr;
    const unsigned ctas = persistent_ctas(L.g2p_per_sm, g_g2p_per_sm[G2P_MIXED][0][warm ? 1 : 0]);
    (warm ? k_g2p<true, G2P_THREADS, 2, true> : k_g2p<false, G2P_THREADS, 2, true>)<<<ctas, G2P_THREADS,
                                                                                       g2p_smem(G2P_THREADS), s>>>(
        A.desc, A.ctrl, A.st[0], A.st[1], A.id[0], A.id[1], A.cap, A.perm, A.vel, A.tpart, tab, A.log_x, A.log_y,
        A.log_n, A.log_cap, A.tile_rec, A.tile_count, cur, A.g2p_clk, A.defer_rec, A.nw_count + 5);
    return;
  }
  if (A.kinds == 1) launch_g2p_kind<G2P_PASTE>(A, warm, s);
  else if (A.kinds == 2) launch_g2p_kind<G2P_LIQUID>(A, false, s);
  else launch_g2p_kind<G2P_MIXED>(A, warm, s);
}
// the particles G2P left to the eigen-decomposition pass (normally none: every CTA exits at once)
static void launch_g2p_defer(const DeviceArrays& A, bool warm, cudaStream_t s) {
  (warm ? k_g2p_defer<true> : k_g2p_defer<false>)<<<(unsigned)g_sms, G2P_DEFER_THREADS, 0, s>>>(
      A.desc, A.ctrl, A.st[0], A.st[1], A.cap, A.tpart, warm ? A.mlp_tab : nullptr, A.log_x, A.log_y, A.log_n,
      A.log_cap, A.defer_rec, A.nw_count + 5);
}
uint64_t kernel_launch_count() { return g_launches; }
void add_kernel_launches(uint64_t n) { g_launches += n; }


// audit (energy audit) or null: the grid-update stage energies go to audit[4 * CTA + k] and the
// kinetic energy after the pellet coupling to audit[4 * n_gcta + CTA].
static int attempt_sequence(const DeviceArrays& A, cudaStream_t s, cudaEvent_t* ev, double* audit) {
  int n = 0;
  if (ev) cudaEventRecord(ev[0], s);
  k_begin<<<grid_of(A.n_inst, 64), 64, 0, s>>>(A.desc, A.ctrl, A.n_inst, A.nw_count, A.bed);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  k_bin_count<<<(unsigned)A.n_pcta, BIN_THREADS, 0, s>>>(A.desc, A.ctrl, A.pcta_inst, A.st[0], A.st[1], A.cap,
                                                          A.keys, A.count, A.chunk_sum, A.nw_list, A.nw_count);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  k_scan_instances<<<A.n_inst, 1024, 0, s>>>(A.desc, A.ctrl, A.chunk_sum, A.chunk_base);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  k_scan_apply<<<(unsigned)A.n_chunks, 256, 0, s>>>(A.count, A.chunk_base, A.start, A.chunk_inst, A.ctrl);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  k_bin_scatter<<<(unsigned)A.n_pcta, BIN_THREADS, 0, s>>>(A.desc, A.ctrl, A.pcta_inst, A.keys, A.count, A.start,
                                                            A.perm);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  launch_tiles_p2g(A, s, 0, ev, n);
  k_traction<<<(unsigned)(g_sms * TRACTION_CTAS_PER_SM), TRACTION_THREADS, 0, s>>>(A.desc, A.ctrl, A.pcta_inst, A.st[0], A.st[1], A.cap, A.nw_list, A.nw_count,
                                     A.acc, A.trac, A.node_total);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  if (audit)
    k_grid_update<true><<<(unsigned)A.n_gcta, GU_THREADS, 0, s>>>(A.desc, A.ctrl, A.gcta_inst, A.acc, A.trac,
                                                                 A.node_total, A.blk_epoch, A.vel, A.gpart, audit);
  else
    k_grid_update<false><<<(unsigned)A.n_gcta, GU_THREADS, 0, s>>>(A.desc, A.ctrl, A.gcta_inst, A.acc, A.trac,
                                                                  A.node_total, A.blk_epoch, A.vel, A.gpart, nullptr);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  if (A.any_pellet) {
    k_couple<<<A.n_inst, 256, 0, s>>>(A.desc, A.ctrl, A.blk_epoch, A.vel);
    ++n;
    if (ev) cudaEventRecord(ev[n], s);
  }
  if (A.any_bed) {
    k_bed_bin<<<A.n_inst, 1024, 0, s>>>(A.desc, A.ctrl, A.bed, A.bed_key, A.bed_idx);
    ++n;
    if (ev) cudaEventRecord(ev[n], s);
    k_bed_couple<<<(unsigned)A.n_bed, 128, 0, s>>>(A.desc, A.ctrl, A.bed_inst, A.bed, A.bed_key, A.bed_idx,
                                                   A.bed_step, A.blk_epoch, A.vel);
    ++n;
    if (ev) cudaEventRecord(ev[n], s);
    k_bed_step<<<grid_of(A.n_bed, 64), 64, 0, s>>>(A.desc, A.ctrl, A.bed_inst, A.n_bed, A.bed, A.bed_key,
                                                   A.bed_idx, A.bed_step);
    ++n;
    if (ev) cudaEventRecord(ev[n], s);
  }
  if (audit) {
    k_audit_kinetic<<<(unsigned)A.n_gcta, GU_THREADS, 0, s>>>(A.desc, A.ctrl, A.gcta_inst, A.acc, A.vel, A.node_total,
                                                             A.blk_epoch, 0, audit + 4 * A.n_gcta);
    ++n;
  }
  const bool warm_g2p = A.mlp != nullptr && A.mlp_tab != nullptr && A.warm;
  if (warm_g2p) {
    k_mlp_table<<<A.n_inst, MLP_TAB_THREADS, 0, s>>>(A.desc, A.ctrl, A.mlp, A.mlp_tab, A.mlp_tab_dt);
    ++n;
    if (ev) cudaEventRecord(ev[n], s);
  }
  launch_g2p(A, warm_g2p, s);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  launch_g2p_defer(A, warm_g2p, s);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  k_segments<<<(unsigned)A.n_seg, 256, 0, s>>>(A.ctrl, A.segs, A.gpart, A.tpart, A.seg);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  k_end<<<A.n_inst, 256, 0, s>>>(A.desc, A.ctrl, A.seg, A.bed_step, A.bed);
  ++n;
  if (ev) cudaEventRecord(ev[n], s);
  g_launches += (uint64_t)n;
  return n;
}

int launch_attempt(const DeviceArrays& A, cudaStream_t s, cudaEvent_t* ev) { return attempt_sequence(A, s, ev, nullptr); }

int launch_audit(const DeviceArrays& A, double* buf, cudaStream_t s) {
  // transport pass: binning and an APIC-only deposit, its grid kinetic energy to buf[5 n_gcta + CTA]
  k_begin<<<grid_of(A.n_inst, 64), 64, 0, s>>>(A.desc, A.ctrl, A.n_inst, A.nw_count, A.bed);
  k_bin_count<<<(unsigned)A.n_pcta, BIN_THREADS, 0, s>>>(A.desc, A.ctrl, A.pcta_inst, A.st[0], A.st[1], A.cap,
                                                          A.keys, A.count, A.chunk_sum, A.nw_list, A.nw_count);
  k_scan_instances<<<A.n_inst, 1024, 0, s>>>(A.desc, A.ctrl, A.chunk_sum, A.chunk_base);
  k_scan_apply<<<(unsigned)A.n_chunks, 256, 0, s>>>(A.count, A.chunk_base, A.start, A.chunk_inst, A.ctrl);
  k_bin_scatter<<<(unsigned)A.n_pcta, BIN_THREADS, 0, s>>>(A.desc, A.ctrl, A.pcta_inst, A.keys, A.count, A.start,
                                                            A.perm);
  int nt = 0;
  launch_tiles_p2g(A, s, 1, nullptr, nt);
  k_audit_kinetic<<<(unsigned)A.n_gcta, GU_THREADS, 0, s>>>(A.desc, A.ctrl, A.gcta_inst, A.acc, A.vel, A.node_total,
                                                           A.blk_epoch, 1, buf + 5 * A.n_gcta);
  g_launches += 9;
  // the audited trial step, without the Newton log
  DeviceArrays B = A;
  B.log_cap = 0;
  return 9 + attempt_sequence(B, s, nullptr, buf);
}

__global__ void k_grid_sums(const long long* __restrict__ acc, int64_t node_total, unsigned long long* __restrict__ out) {
  long long v[4] = {0, 0, 0, 0};
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < node_total; g += (int64_t)gridDim.x * blockDim.x)
    for (int k = 0; k < 4; ++k) v[k] += acc[k * node_total + g];
  for (int k = 0; k < 4; ++k) atomicAdd(out + k, (unsigned long long)v[k]);
}

int launch_p2g_traction(const DeviceArrays& A, cudaStream_t s) {
  k_begin<<<grid_of(A.n_inst, 64), 64, 0, s>>>(A.desc, A.ctrl, A.n_inst, A.nw_count, A.bed);
  k_bin_count<<<(unsigned)A.n_pcta, BIN_THREADS, 0, s>>>(A.desc, A.ctrl, A.pcta_inst, A.st[0], A.st[1], A.cap,
                                                          A.keys, A.count, A.chunk_sum, A.nw_list, A.nw_count);
  k_scan_instances<<<A.n_inst, 1024, 0, s>>>(A.desc, A.ctrl, A.chunk_sum, A.chunk_base);
  k_scan_apply<<<(unsigned)A.n_chunks, 256, 0, s>>>(A.count, A.chunk_base, A.start, A.chunk_inst, A.ctrl);
  k_bin_scatter<<<(unsigned)A.n_pcta, BIN_THREADS, 0, s>>>(A.desc, A.ctrl, A.pcta_inst, A.keys, A.count, A.start,
                                                            A.perm);
  {
    int nt = 0;
    launch_tiles_p2g(A, s, 0, nullptr, nt);
  }
  k_traction<<<(unsigned)(g_sms * TRACTION_CTAS_PER_SM), TRACTION_THREADS, 0, s>>>(A.desc, A.ctrl, A.pcta_inst, A.st[0], A.st[1], A.cap, A.nw_list, A.nw_count,
                                     A.acc, A.trac, A.node_total);
  g_launches += 9;
  return 9;
}

int launch_grid_totals(const DeviceArrays& A, long long* out, cudaStream_t s) {
  k_begin<<<grid_of(A.n_inst, 64), 64, 0, s>>>(A.desc, A.ctrl, A.n_inst, A.nw_count, A.bed);
  k_bin_count<<<(unsigned)A.n_pcta, BIN_THREADS, 0, s>>>(A.desc, A.ctrl, A.pcta_inst, A.st[0], A.st[1], A.cap,
                                                          A.keys, A.count, A.chunk_sum, A.nw_list, A.nw_count);
  k_scan_instances<<<A.n_inst, 1024, 0, s>>>(A.desc, A.ctrl, A.chunk_sum, A.chunk_base);
  k_scan_apply<<<(unsigned)A.n_chunks, 256, 0, s>>>(A.count, A.chunk_base, A.start, A.chunk_inst, A.ctrl);
  k_bin_scatter<<<(unsigned)A.n_pcta, BIN_THREADS, 0, s>>>(A.desc, A.ctrl, A.pcta_inst, A.keys, A.count, A.start,
                                                            A.perm);
  {
    int nt = 0;
    launch_tiles_p2g(A, s, 0, nullptr, nt);
  }
  k_grid_sums<<<148 * 4, 256, 0, s>>>(A.acc, A.node_total, (unsigned long long*)out);
  g_launches += 9;
  return 9;
}

int launch_attempt(const DeviceArrays& A, cudaStream_t s) { return attempt_sequence(A, s, nullptr, nullptr); }

const char* attempt_kernel_name(int k, int any_pellet, int any_bed, int warm) {
  static const char* a[] = {"k_begin", "k_bin_count", "k_scan_instances", "k_scan_apply", "k_bin_scatter",
                            "k_tiles", "k_bin_sort", "k_p2g", "k_traction", "k_grid_update", "k_couple",
                            "k_bed_bin", "k_bed_couple", "k_bed_step", "k_mlp_table", "k_g2p", "k_g2p_defer",
                            "k_segments", "k_end"};
  if (!any_pellet && k >= 10) ++k;
  if (!any_bed && k >= 11) k += 3;
  if (!warm && k >= 14) ++k;
  return k < 19 ? a[k] : "?";
}

int launch_state_stats(const DeviceArrays& A, cudaStream_t s) {
  k_state_stats<<<(unsigned)A.n_pcta, G2P_THREADS, 0, s>>>(A.desc, A.ctrl, A.pcta_inst, A.st[0], A.st[1], A.cap,
                                                            A.ppart);
  g_launches += 1;
  return 1;
}

int launch_diagnostics(const DeviceArrays& A, int hydro, double h0, int dam, double* out, cudaStream_t s) {
  k_diagnostics<<<(unsigned)A.n_pcta, G2P_THREADS, 0, s>>>(A.desc, A.ctrl, A.pcta_inst, A.st[0], A.st[1], A.cap,
                                                            hydro, h0, dam, out);
  g_launches += 1;
  return 1;
}

int launch_hb_return_batch(int64_t n, const double* trial, const double* ys, const double* k, const double* nn,
                           const double* mu, const double* dt, double tol, const MlpPacked* mlp, double* out,
                           int* status, cudaStream_t s) {
  k_hb_batch<<<grid_of(n, 128), 128, 0, s>>>(n, trial, ys, k, nn, mu, dt, tol, mlp, out, status);
  g_launches += 1;
  return 1;
}
int launch_update_paste_batch(int64_t n, const double* f, double mu, double lambda, double ys, double k, double nn,
                              double dt, double tol, double* fnew, double* tau, double* scal, int* status,
                              cudaStream_t s) {
  k_paste_batch<<<grid_of(n, 128), 128, 0, s>>>(n, f, mu, lambda, ys, k, nn, dt, tol, fnew, tau, scal, status);
  g_launches += 1;
  return 1;
}
int launch_update_liquid_batch(int64_t n, const double* j, const double* grad, double bulk, double visc, double gamma,
                               double dt, double* jnew, double* tau, double* p, int* status, cudaStream_t s) {
  k_liquid_batch<<<grid_of(n, 128), 128, 0, s>>>(n, j, grad, bulk, visc, gamma, dt, jnew, tau, p, status);
  g_launches += 1;
  return 1;
}

int launch_import(const HostParticleChunk& h, int64_t n, int64_t first, float* dst, uint32_t* ids, int64_t cap,
                  int64_t slot_off, double yield_default, unsigned long long* bad, cudaStream_t s) {
  k_import<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(h, n, first, dst, ids, cap, slot_off, yield_default, bad);
  g_launches += 1;
  return 1;
}
int launch_export(const HostParticleChunk& h, int64_t n, int64_t first, const float* src, const uint32_t* ids,
                  int64_t cap, int64_t slot_off, int paste, int per_particle_yield, double yield_default,
                  cudaStream_t s) {
  k_export<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(h, n, first, src, ids, cap, slot_off, paste, per_particle_yield,
                                           yield_default);
  g_launches += 1;
  return 1;
}

}  // namespace lp
