// lp_kernels.h - launch interface between the host runtime and the substep kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lp_device.cuh"

namespace lp {

constexpr int DIAG_N = 19;

// Launch shape of the persistent tile kernels, chosen per ensemble (by default, or by the
// autotuner on the live batch).  Per-SM counts of 0, or above what fits, mean as many as fit.
struct LaunchShape {
  int g2p_variant = 0;  // G2P CTAs of 0: G2P_THREADS (256) threads, 1-3: G2P_THREADS_SMALL (128)
                        // threads with registers sized for 4, 5 or 6 CTAs per SM
  int g2p_per_sm = 0;  // persistent G2P CTAs per SM
  int p2g_variant = 0;  // P2G chunks of 0: P2G_CHUNK (1024) particles, 1: P2G_CHUNK_SMALL (512),
                        // 2: P2G_CHUNK_SMALL with each chunk's particle state copied one chunk ahead
  int p2g_per_sm = 0;  // persistent P2G CTAs per SM
  int dynamic = 1;     // 1: CTAs take tiles from the attempt's cursors, 0: round robin
};

// All device buffers of one ensemble (owned by the host runtime).
struct DeviceArrays {
  InstDesc* desc = nullptr;
  Control* ctrl = nullptr;
  int n_inst = 0;
  int any_pellet = 0;
  int kinds = 3;  // material kinds of the instances: bit 0 paste, bit 1 liquid
  int* pcta_inst = nullptr;  // G2P / per-slot CTA -> instance
  int64_t n_pcta = 0;
  int* tile_inst = nullptr;  // P2G tile -> instance
  int64_t n_tiles = 0;
  int* gcta_inst = nullptr;  // grid-update CTA -> instance
  int64_t n_gcta = 0;
  int* chunk_inst = nullptr;  // scan chunk -> instance
  int64_t n_chunks = 0;
  float* st[2] = {nullptr, nullptr};
  uint32_t* id[2] = {nullptr, nullptr};
  int64_t cap = 0;  // slots (multiple of SLOT_ALIGN)
  uint32_t* keys = nullptr;
  uint32_t* count = nullptr;
  uint32_t* start = nullptr;
  uint32_t* chunk_sum = nullptr;
  uint32_t* chunk_base = nullptr;
  uint32_t* perm = nullptr;
  uint32_t* nw_list = nullptr;
  uint32_t* nw_count = nullptr;    // [0] near-wall particles, [1] occupied tiles of the attempt,
                                   // [2..4] tile cursors of the bin sort, P2G and G2P,
                                   // [5] tiles listed in defer_rec
  uint32_t* tile_count = nullptr;  // = nw_count + 1
  uint4* tile_rec = nullptr;       // occupied tiles of the attempt: (tile, instance, first slot, end slot)
  uint4* defer_rec = nullptr;      // tiles whose particles k_g2p left to the eigen-decomposition pass
  long long* acc = nullptr;   // 4 x node_total: mass, momentum xyz (int64 fixed point)
  long long* trac = nullptr;  // 6 x node_total: reactions per axis, low faces then high faces
  int64_t node_total = 0;
  uint32_t* blk_epoch = nullptr;
  int64_t n_blk = 0;
  float4* vel = nullptr;
  GridPartial* gpart = nullptr;
  ParticlePartial* ppart = nullptr;  // per slot-CTA (state statistics)
  ParticlePartial* tpart = nullptr;  // per tile (G2P)
  SegDesc* segs = nullptr;  // reduction segments
  SegPartial* seg = nullptr;
  int64_t n_seg = 0;
  const MlpPacked* mlp = nullptr;  // packed warm-start weights (device) or null
  float* mlp_tab = nullptr;         // [n_inst][MLP_TAB_FLOATS] warm-start tables (logits, fractions)
  double* mlp_tab_dt = nullptr;     // [n_inst] dt each table was built for (NaN: stale)
  int warm = 0;                     // some instance has the warm start on: launch the WARM G2P
  float* log_x = nullptr;
  float* log_y = nullptr;
  unsigned long long* log_n = nullptr;
  long long log_cap = 0;
  LaunchShape shape;
  unsigned long long* g2p_clk = nullptr;  // non-null: G2P runs its clock-measurement instantiation
  // pellet bed (instances with InstDesc::bed_np >= 2)
  int any_bed = 0;
  int64_t n_bed = 0;                                 // pellets of all instances
  int* bed_inst = nullptr;                           // pellet -> instance
  BedPtrs bed = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
  BedStep* bed_step = nullptr;                       // [pellet]
  long long* bed_key = nullptr;                      // coarse-cell keys sorted per instance
  int* bed_idx = nullptr;                            // instance-local pellet index per sorted key
};

// One substep attempt for every active instance; returns the number of kernels launched.
int launch_attempt(const DeviceArrays& A, cudaStream_t s);
// same, recording ev[0] before the first kernel and ev[k] after kernel k (at most 20 events)
int launch_attempt(const DeviceArrays& A, cudaStream_t s, cudaEvent_t* ev);
const char* attempt_kernel_name(int k, int any_pellet, int any_bed, int warm);
// Energy audit of one forced-dt trial: a transport pass (binning + APIC-only deposit) and the
// attempt with stage energies.  buf holds 6 * n_gcta doubles: [0, 4 n_gcta) the grid-update
// stages per CTA (stress, traction, gravity kick, walls), [4 n_gcta, 5 n_gcta) the kinetic energy
// after the pellet coupling, [5 n_gcta, 6 n_gcta) the transport pass.
int launch_audit(const DeviceArrays& A, double* buf, cudaStream_t s);
int launch_state_stats(const DeviceArrays& A, cudaStream_t s);
// begin + binning + P2G only (conservation probe), then exact node sums into out[4] (int64)
int launch_grid_totals(const DeviceArrays& A, long long* out, cudaStream_t s);
int launch_p2g_traction(const DeviceArrays& A, cudaStream_t s);
int launch_diagnostics(const DeviceArrays& A, int hydro, double h0, int dam, double* out, cudaStream_t s);
// FP64 particle arrays of one chunk in the reference's host layout (device pointers)
struct HostParticleChunk {
  uint32_t* id;
  double *position, *velocity, *affine, *deformation, *volume_ratio, *kirchhoff, *plastic_strain, *mass, *volume0,
      *yield_stress;  // yield_stress may be null on import (instance default)
};
// FP64 host-layout chunk [first, first + n) of an instance <-> its FP32 component-major state.
// Import writes dst/ids and records the smallest index whose mass, volume or kinematics are not
// finite and positive in *bad.
int launch_import(const HostParticleChunk& h, int64_t n, int64_t first, float* dst, uint32_t* ids, int64_t cap,
                  int64_t slot_off, double yield_default, unsigned long long* bad, cudaStream_t s);
int launch_export(const HostParticleChunk& h, int64_t n, int64_t first, const float* src, const uint32_t* ids,
                  int64_t cap, int64_t slot_off, int paste, int per_particle_yield, double yield_default,
                  cudaStream_t s);
uint64_t kernel_launch_count();
void configure_kernels();              // one-time function attributes (dynamic shared memory)
// launch-shape variants of the persistent P2G and G2P kernels
constexpr int P2G_VARIANTS = 3, G2P_VARIANTS = 4;
// out = SMs, resident CTAs per SM of the bin sort, of the P2G variants (from out[LIM_P2G]) and of
// the warm G2P variants (from out[LIM_G2P]); returns LAUNCH_LIMITS
constexpr int LIM_P2G = 2, LIM_G2P = LIM_P2G + P2G_VARIANTS, LAUNCH_LIMITS = LIM_G2P + G2P_VARIANTS;
int launch_shape_limits(int out[LAUNCH_LIMITS]);
void set_last_error(const char* msg);  // message returned by lp_last_error()
void add_kernel_launches(uint64_t n);

// FP32 warm-start weights -> packed BF16 layout of the tensor-core inference
void launch_mlp_pack(const float* W, MlpPacked* P, cudaStream_t s);

// constitutive unit kernels on device arrays
int launch_hb_return_batch(int64_t n, const double* trial, const double* ys, const double* k, const double* nn,
                           const double* mu, const double* dt, double tol, const MlpPacked* mlp, double* out, int* status,
                           cudaStream_t s);
int launch_update_paste_batch(int64_t n, const double* f, double mu, double lambda, double ys, double k, double nn,
                              double dt, double tol, double* fnew, double* tau, double* scal, int* status,
                              cudaStream_t s);
int launch_update_liquid_batch(int64_t n, const double* j, const double* grad, double bulk, double visc, double gamma,
                               double dt, double* jnew, double* tau, double* p, int* status, cudaStream_t s);

}  // namespace lp
