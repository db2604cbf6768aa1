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

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

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

// ---------------------------------------------------------------- warp-cooperative inference
// One warp evaluates the network for its 32 lanes at once on the tensor cores with
// mma.sync.m16n8k16 (BF16 operands, FP32 accumulation); rows are lanes:
//   layer 1: [32 x 16] x [16 x 64].  Each FP32 feature enters as a BF16 pair hi + lo (columns
//            k and k + 6, both multiplying the same W1 column), so the inputs keep ~16 bits;
//   layer 2: [32 x 64] x [64 x 64], A fragments are the layer-1 accumulators after bias + SiLU,
//            re-packed to BF16 in registers (the C layout of one n-tile pair is the A layout of
//            one k-step);
//   layer 3: 64-wide FP32 dot product, reduced across each lane quad.
// SiLU uses the hardware tanh: silu(z) = z/2 (1 + tanh(z/2)).
// Packed weights (MlpPacked, built once per weight upload by k_mlp_pack) are BF16 pairs with
// padded row strides of 12 and 36 words, so that fragment loads are free of bank conflicts.
constexpr int MLP_S1 = 12, MLP_S2 = 36;
struct __align__(16) MlpPacked {
  uint32_t w1[MLP_H * MLP_S1];  // [n][k/2]: words 0-2 W1[n][0..5], 3-5 the same again, rest 0
  uint32_t w2[MLP_H * MLP_S2];  // [n][k/2], k < 64
  float b1[MLP_H], b2[MLP_H], w3[MLP_H], b3[4];
};
static_assert(sizeof(MlpPacked) % 16 == 0, "MlpPacked is staged with 16-byte copies");
constexpr int MLP_XS_WORDS = 32 * MLP_S1;  // per-warp feature rows (BF16 pairs, 12-word stride)

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float silu_hw(float z) {
  const float h = 0.5f * z;
  return fmaf(h, tanh_hw(h), h);
}

// FP32 weights -> packed BF16 layout (any grid; grid-stride over the words)
__device__ inline void mlp_pack_words(const float* __restrict__ W, MlpPacked& P, int tid, int stride) {
  for (int i = tid; i < MLP_H * MLP_S1; i += stride) {
    const int n = i / MLP_S1, w = i % MLP_S1, k = 2 * (w < 3 ? w : w - 3);
    P.w1[i] = w < 6 ? pack_bf16(W[MLP_W1 + n * MLP_IN + k], W[MLP_W1 + n * MLP_IN + k + 1]) : 0u;
  }
  for (int i = tid; i < MLP_H * MLP_S2; i += stride) {
    const int n = i / MLP_S2, w = i % MLP_S2;
    P.w2[i] = w < 32 ? pack_bf16(W[MLP_W2 + n * MLP_H + 2 * w], W[MLP_W2 + n * MLP_H + 2 * w + 1]) : 0u;
  }
  for (int i = tid; i < MLP_H; i += stride) {
    P.b1[i] = W[MLP_B1 + i];
    P.b2[i] = W[MLP_B2 + i];
    P.w3[i] = W[MLP_W3 + i];
  }
  if (tid < 4) P.b3[tid] = tid == 0 ? W[MLP_B3] : 0.f;
}

// copy of the packed weights into shared memory by all threads of the CTA (caller syncs)
__device__ inline void mlp_stage(const MlpPacked* __restrict__ g, MlpPacked& s) {
  const uint4* src = reinterpret_cast<const uint4*>(g);
  uint4* dst = reinterpret_cast<uint4*>(&s);
  for (int i = threadIdx.x; i < (int)(sizeof(MlpPacked) / 16); i += blockDim.x) dst[i] = __ldg(src + i);
}

// One feature row in the BF16 hi + lo layout of the first layer's A operand.
__device__ __forceinline__ void mlp_write_row(uint32_t* row, const float (&f)[6]) {
  float hi[6], lo[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    hi[i] = __bfloat162float(__float2bfloat16_rn(f[i]));
    lo[i] = f[i] - hi[i];
  }
  row[0] = pack_bf16(hi[0], hi[1]);
  row[1] = pack_bf16(hi[2], hi[3]);
  row[2] = pack_bf16(hi[4], hi[5]);
  row[3] = pack_bf16(lo[0], lo[1]);
  row[4] = pack_bf16(lo[2], lo[3]);
  row[5] = pack_bf16(lo[4], lo[5]);
  row[6] = 0u;
  row[7] = 0u;
}

// Network output (logit of the root fraction) of the 32 feature rows at xs (row stride MLP_S1
// words) for the lane's own row.  Every lane of the warp calls it, converged, after the rows
// are visible to the warp.
__device__ __forceinline__ float warp_mlp_rows(const MlpPacked& S, const uint32_t* xs) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float part[2][2];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    const int r0 = mt * 16 + g, r1 = r0 + 8;
    const uint32_t a[4] = {xs[r0 * MLP_S1 + t], xs[r1 * MLP_S1 + t], xs[r0 * MLP_S1 + t + 4],
                           xs[r1 * MLP_S1 + t + 4]};
    uint32_t a2[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const int nn = 2 * kk + half;
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        mma_bf16_16816(c, a, S.w1[(nn * 8 + g) * MLP_S1 + t], S.w1[(nn * 8 + g) * MLP_S1 + t + 4]);
        const int col = nn * 8 + 2 * t;
        const float bb0 = S.b1[col], bb1 = S.b1[col + 1];
        a2[kk][2 * half + 0] = pack_bf16(silu_hw(c[0] + bb0), silu_hw(c[1] + bb1));
        a2[kk][2 * half + 1] = pack_bf16(silu_hw(c[2] + bb0), silu_hw(c[3] + bb1));
      }
    float p0 = 0.f, p1 = 0.f;
#pragma unroll
    for (int nn = 0; nn < 8; ++nn) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        mma_bf16_16816(c, a2[kk], S.w2[(nn * 8 + g) * MLP_S2 + kk * 8 + t],
                       S.w2[(nn * 8 + g) * MLP_S2 + kk * 8 + t + 4]);
      const int col = nn * 8 + 2 * t;
      const float bb0 = S.b2[col], bb1 = S.b2[col + 1], u0 = S.w3[col], u1 = S.w3[col + 1];
      p0 = fmaf(silu_hw(c[0] + bb0), u0, fmaf(silu_hw(c[1] + bb1), u1, p0));
      p1 = fmaf(silu_hw(c[2] + bb0), u0, fmaf(silu_hw(c[3] + bb1), u1, p1));
    }
    p0 += __shfl_xor_sync(0xffffffffu, p0, 1);
    p0 += __shfl_xor_sync(0xffffffffu, p0, 2);
    p1 += __shfl_xor_sync(0xffffffffu, p1, 1);
    p1 += __shfl_xor_sync(0xffffffffu, p1, 2);
    part[mt][0] = p0;
    part[mt][1] = p1;
  }
  // row r of m-tile mt sits in lane quad (r % 8) as p0 (r < 8) or p1
  const int src = (lane & 7) * 4;
  const float v00 = __shfl_sync(0xffffffffu, part[0][0], src), v01 = __shfl_sync(0xffffffffu, part[0][1], src);
  const float v10 = __shfl_sync(0xffffffffu, part[1][0], src), v11 = __shfl_sync(0xffffffffu, part[1][1], src);
  const float out = lane < 16 ? ((lane & 8) ? v01 : v00) : ((lane & 8) ? v11 : v10);
  return out + S.b3[0];
}

// Network output for this lane's features, rows staged in this warp's scratch xs
// (MLP_XS_WORDS words); every lane of the warp calls it, converged.
__device__ __forceinline__ float warp_mlp_logit(const MlpPacked& S, uint32_t* xs, const float (&f)[6]) {
  const int lane = threadIdx.x & 31;
  mlp_write_row(xs + lane * MLP_S1, f);
  __syncwarp();
  const float y = warp_mlp_rows(S, xs);
  __syncwarp();  // xs may be rewritten by the next call
  return y;
}

// Features of many return problems that share consistency, flow index, mu and dt (one
// material, one attempt): the per-problem part is log a only.  FP32 restatement of hb_features.
struct HbFeatureConst {
  float lb8, n, inv_n_m1, f4, f5;
};
__device__ inline HbFeatureConst hb_feature_const(double k, double n, double mu, double dt) {
  HbFeatureConst h;
  const double b = fmax(3.0 * mu * dt / k, 1e-300);
  h.lb8 = (float)(log(b) / 8.0);
  h.n = (float)n;
  h.inv_n_m1 = (float)(1.0 / n - 1.0);
  h.f4 = (float)(1.0 / (3.0 * n));
  h.f5 = (float)log(n);
  return h;
}
// log(a) / 8 of one return problem, a = (trial - yield) / K floored at 1e-37; the hardware
// logarithm suffices, since la8 only places the problem between table nodes 0.011 apart
__device__ __forceinline__ float hb_la8(float inv_k, double trial, double ys) {
  const float a = fmaxf((float)(trial - ys) * inv_k, 1e-37f);
  return __logf(a) * 0.125f;
}
__device__ __forceinline__ void hb_features_la8(const HbFeatureConst& h, float la8, float (&f)[6]) {
  f[0] = la8;
  f[1] = h.lb8;
  f[2] = h.n;
  f[3] = h.lb8 + h.inv_n_m1 * la8;
  f[4] = h.f4;
  f[5] = h.f5;
}

// Warm-start table of one instance.  For one material and one dt, four of the six features are
// constants, the first is la8 = log(a)/8 and the fourth is affine in it, so the network is a
// smooth function of la8 alone.  It is evaluated (the same tensor-core pass) at MLP_TAB_N nodes
// la8_j = MLP_TAB_LO + j MLP_TAB_H, which cover every finite FP32 a >= 1e-37
// (la8 in [-10.66, 11.10]); the node spacing is exact in FP32.  Per instance the table holds the
// logits (MLP_TAB_STRIDE floats), then one float2 per node: the root fraction
// t_j = 1 / (1 + exp(-logit_j)) and t_(j+1) - t_j, which the solver interpolates linearly.
constexpr int MLP_TAB_N = 2049, MLP_TAB_STRIDE = 2056;
constexpr int MLP_TAB_FLOATS = 3 * MLP_TAB_STRIDE;  // per instance: logits, then (t, dt) pairs
constexpr float MLP_TAB_LO = -10.75f, MLP_TAB_H = 11.0f / 1024.0f, MLP_TAB_INV_H = 1024.0f / 11.0f;
__device__ __forceinline__ float mlp_table_node(int j) { return MLP_TAB_LO + (float)j * MLP_TAB_H; }
// interpolated root fraction at la8 of the instance's (t, dt) pairs; NaN outside the table (a
// non-finite la8 included)
__device__ __forceinline__ float mlp_table_fraction(const float2* __restrict__ pairs, float la8) {
  const float u = (la8 - MLP_TAB_LO) * MLP_TAB_INV_H;
  if (!(u >= 0.0f && u <= (float)(MLP_TAB_N - 1))) return __int_as_float(0x7fc00000);
  const int i = min((int)u, MLP_TAB_N - 2);
  const float2 p = __ldg(pairs + i);
  return fmaf(u - (float)i, p.y, p.x);
}

// warm-start fraction in (0, 1) from the network output, or -1 (midpoint start)
__device__ __forceinline__ double warm_fraction_of(float logit) {
  const float t = 1.0f / (1.0f + __expf(-logit));
  return (t > 0.f && t < 1.f) ? (double)t : -1.0;
}

}  // namespace lp
