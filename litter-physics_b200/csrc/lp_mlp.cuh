// lp_mlp.cuh - learned warm start of the Herschel-Bulkley return (no reference counterpart).
//
// The scalar return of constitutive.rs:280-362 solves
//     f(sigma) = sigma - sigma_tr + 3 mu dt ((sigma - sigma_y) / K)^(1/n) = 0  on [sigma_y, sigma_tr].
// With s = (sigma - sigma_y)/K, a = (sigma_tr - sigma_y)/K and b = 3 mu dt / K it becomes
// s + b s^(1/n) = a, so the root fraction t = s / a in (0, 1) depends on (a, b, n) only.  The
// network maps six dimensionless features of the six return inputs (trial stress, yield stress,
// consistency, flow index, shear modulus, dt) to logit(t); the Newton solve then starts at
// sigma_y + t (sigma_tr - sigma_y) instead of the bracket midpoint, keeping the same bracket,
// safeguard and stopping rule, so every particle converges to the same tolerance.  The mean
// pressure does not enter the J2 return and is therefore not an input.
//
// Network: 6 -> 64 -> 64 -> 1, SiLU, FP32 weights, flat layout below.
#pragma once

#include <cuda_runtime.h>

namespace lp {

constexpr int MLP_IN = 6, MLP_H = 64;
constexpr int MLP_W1 = 0;                       // [64][6]
constexpr int MLP_B1 = MLP_W1 + MLP_H * MLP_IN;  // [64]
constexpr int MLP_W2 = MLP_B1 + MLP_H;           // [64][64]
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;   // [64]
constexpr int MLP_W3 = MLP_B2 + MLP_H;           // [64]
constexpr int MLP_B3 = MLP_W3 + MLP_H;           // [1]
constexpr int MLP_NW = MLP_B3 + 1;               // 4673

__host__ __device__ inline void hb_features(double trial, double ys, double k, double n, double mu, double dt,
                                            float f[6]) {
  const double a = fmax((trial - ys) / k, 1e-300);
  const double b = fmax(3.0 * mu * dt / k, 1e-300);
  const double la = log(a), lb = log(b);
  f[0] = (float)(la / 8.0);
  f[1] = (float)(lb / 8.0);
  f[2] = (float)n;
  f[3] = (float)((lb + (1.0 / n - 1.0) * la) / 8.0);
  f[4] = (float)(1.0 / (3.0 * n));
  f[5] = (float)log(n);
}

__device__ __forceinline__ float silu(float x) { return x / (1.0f + __expf(-x)); }

// Scalar FP32 forward pass; returns logit(t).
__device__ inline float mlp_forward(const float* __restrict__ W, const float f[6]) {
  float h1[MLP_H];
#pragma unroll 4
  for (int j = 0; j < MLP_H; ++j) {
    float s = W[MLP_B1 + j];
#pragma unroll
    for (int i = 0; i < MLP_IN; ++i) s += W[MLP_W1 + j * MLP_IN + i] * f[i];
    h1[j] = silu(s);
  }
  float out = W[MLP_B3];
#pragma unroll 2
  for (int j = 0; j < MLP_H; ++j) {
    float s = W[MLP_B2 + j];
#pragma unroll 8
    for (int i = 0; i < MLP_H; ++i) s += W[MLP_W2 + j * MLP_H + i] * h1[i];
    out += W[MLP_W3 + j] * silu(s);
  }
  return out;
}

// Warm-start fraction in (0, 1) for the Newton start, from the network output.
static __device__ __noinline__ double warm_fraction(const float* __restrict__ W, double trial, double ys, double k,
                                                double n, double mu, double dt) {
  if (W == nullptr || !(trial > ys) || !(k > 0.0)) return -1.0;
  float f[6];
  hb_features(trial, ys, k, n, mu, dt, f);
  const float y = mlp_forward(W, f);
  const double t = 1.0 / (1.0 + exp(-(double)y));
  return (t > 0.0 && t < 1.0) ? t : -1.0;
}

}  // namespace lp
