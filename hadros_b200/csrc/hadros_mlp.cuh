// hadros_mlp.cuh — the surrogate network's fixed shape, parameter layouts and
// the device helpers its training kernels (tcgen05, hadros_mlp.cu) and its
// fused inference kernel (tcgen05, hadros_mlp_umma.cu) share.
//
// The surrogate has no counterpart in the reference: it predicts
// ln tau_E and ln I_E of one (pixel, bin) sample from 16 raw features
//   0 alpha, 1 beta (screen coordinates u*r_obs, v*r_obs, in M; the camera of
//     src/kerr_camera.cpp:110-116), 2 a, 3 cos(theta_obs), 4 log10 rho0,
//   5..12 one-hot torus profile kind, 13 r0 (M), 14 H/R, 15 log10 E_mid (GeV).
// Each normalized feature x enters as two BF16 columns, hi = bf16(x) and
// lo = bf16(x - hi), with tied first-layer weights, so the network sees x to
// ~16 bits (a pixel of a 4096-wide image) although its operands are BF16.
// The normalized screen coordinates also enter as Fourier features
// sin(pi 2^(k-1) x), cos(pi 2^(k-1) x), k = 0..7, so the first layer can
// resolve image structure down to ~1/100 of the field of view.
// Network: 64 -> 256 -> 256 -> 256 -> 256 (SiLU) -> 2, BF16 weights and
// activations, FP32 accumulation, FP32 biases, plus an FP32 linear skip from
// the 16 normalized features (x = hi + lo) to the 2 outputs.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#include <cuda_bf16.h>
#endif

namespace hadros {
namespace mlp {

constexpr int kF = 16;      // raw features
constexpr int kFreq = 8;    // Fourier frequencies per screen coordinate
constexpr int kFour = 4 * kFreq;   // sin and cos of alpha and beta
constexpr int kW1In = kF + kFour;  // master first-layer inputs (hi/lo tied)
constexpr int kIn = 2 * kF + kFour;   // BF16 input columns: hi, lo, Fourier
constexpr int kW = 256;     // hidden width
constexpr int kDepth = 4;   // hidden layers
constexpr int kOut = 2;     // ln tau_E, ln I_E (standardized)
constexpr int kOutPad = 16; // rows of the packed last-layer matrix

// FP32 master parameters (what Adam updates), one network:
//   W1 [256][48] (16 tied hi/lo columns, 32 Fourier columns), b1 [256],
//   W_l [256][256], b_l [256] for l = 2..4,
//   W5 [2][256], b5 [2], Ws [2][16] (linear skip).
constexpr long kOffW1 = 0;
constexpr long kOffB1 = kOffW1 + long(kW) * kW1In;
constexpr long kOffW2 = kOffB1 + kW;
constexpr long kHidStride = long(kW) * kW + kW;   // W_l then b_l
constexpr long kOffW5 = kOffW2 + 3 * kHidStride;
constexpr long kOffB5 = kOffW5 + long(kOut) * kW;
constexpr long kOffWs = kOffB5 + kOut;
constexpr long kParamsUsed = kOffWs + long(kOut) * kF;
constexpr long kParams = (kParamsUsed + 7) / 8 * 8;   // padded for vector access

__host__ __device__ constexpr long off_w(int layer)   // layer 1..4 weights
{
    return layer == 1 ? kOffW1 : kOffW2 + (layer - 2) * kHidStride;
}
__host__ __device__ constexpr long off_b(int layer)   // layer 1..4 bias
{
    return layer == 1 ? kOffB1 : off_w(layer) + long(kW) * kW;
}

// Row-major BF16 working copy (training kernels and tests):
//   W1 [256][64] (the 16 feature columns twice, then the 32 Fourier
//   columns), W2..W4 [256][256],
//   W5 [16][256] (rows 0..1 from the master, rows 2..15 zero).
constexpr long kPW1 = 0;
constexpr long kPW2 = kPW1 + long(kW) * kIn;
constexpr long kPW5 = kPW2 + 3L * kW * kW;
constexpr long kPacked = kPW5 + long(kOutPad) * kW;   // elements

__host__ __device__ constexpr long pw(int layer)       // layer 1..5
{
    return layer == 1 ? kPW1 : (layer == 5 ? kPW5 : kPW2 + (layer - 2) * long(kW) * kW);
}

// Training workspace (bytes) for a batch of n samples: Z1..Z4, H1..H4,
// two dZ buffers (BF16 [n][256] each) and the [256][kIn] FP32 layer-1 weight
// gradient before the hi/lo columns are folded.
// The input row X [kIn] = hi[16], lo[16], then for each screen coordinate
// (alpha, beta) sin and cos of its kFreq frequencies.
constexpr long kWsAlign = 256;
__host__ __device__ constexpr long ws_act_bytes(long n) { return n * kW * 2; }
__host__ __device__ constexpr long ws_bytes(long n) { return 10 * ws_act_bytes(n) + long(kW) * kIn * 4 + kWsAlign; }
// Batch buffers of one member in hadros_mlp_train_members: X [n][kIn] BF16,
// targets, weights, outputs and their gradients (FP32), kWsAlign-rounded.
__host__ __device__ constexpr long members_batch_bytes(long n)
{
    return (n * kIn * 2 + n * (3 * kOut + 1) * 4 + 64 + kWsAlign - 1) / kWsAlign * kWsAlign;
}

// Normalization of one model (FP32): features x = (raw - mu) * inv_sd;
// targets t = (y - out_mu) / out_sd with y = ln(value + floor).
struct Norm {
    float feat_mu[kF];
    float feat_inv_sd[kF];
    float out_mu[kOut];
    float out_sd[kOut];
    float out_floor[kOut];
};

#ifdef __CUDACC__

// SiLU(z) = z sigma(z) = h + h tanh(h) with h = z / 2, evaluated on a pair of
// values in packed BF16: h is rounded to BF16, tanh runs on the paired unit
// (tanh.approx.bf16x2) and the result is one fused multiply-add rounded to
// BF16, the activation's storage type.  Takes h (FP32) and returns the packed
// BF16 pair.  The same function in every kernel, so the trained network and
// the inferred one agree; the inference kernel folds the 1/2 into its weights.
__device__ __forceinline__ uint32_t silu_half_bf16x2(float h0, float h1)
{
    uint32_t hb, t, y;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(hb) : "f"(h1), "f"(h0));
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(hb));
    asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(y) : "r"(hb), "r"(t));
    return y;
}
// d SiLU / dz at z (FP32 tanh): (1 + tanh(h) + h (1 - tanh(h)^2)) / 2.
__device__ __forceinline__ float silu_grad_f(float z)
{
    const float h = 0.5f * z;
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(h));
    return 0.5f * (1.0f + t + h * fmaf(-t, t, 1.0f));
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float2 unpack_bf16x2(uint32_t u)
{
    const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(&u);
    return __bfloat1622float2(v);
}

// Fourier features of a normalized screen coordinate x: out[2k] =
// sin(pi t), out[2k+1] = cos(pi t), t = 2^(k-1) x reduced to [-1, 1].
__device__ __forceinline__ void fourier(float x, float* out)
{
#pragma unroll
    for (int k = 0; k < kFreq; ++k) {
        const float t = x * float(1 << k) * 0.5f;
        const float r = t - 2.0f * rintf(0.5f * t);
        float sn, cs;
        __sincosf(3.14159265358979f * r, &sn, &cs);
        out[2 * k] = sn;
        out[2 * k + 1] = cs;
    }
}

// One input row of kIn BF16 values from the 16 normalized features.
__device__ __forceinline__ void input_row(const float* xn, __nv_bfloat16* row)
{
#pragma unroll
    for (int j = 0; j < kF; ++j) {
        const __nv_bfloat16 hi = __float2bfloat16_rn(xn[j]);
        row[j] = hi;
        row[kF + j] = __float2bfloat16_rn(xn[j] - __bfloat162float(hi));
    }
    float f[2 * kFreq];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        fourier(xn[c], f);
#pragma unroll
        for (int q = 0; q < 2 * kFreq; ++q) row[2 * kF + c * 2 * kFreq + q] = __float2bfloat16_rn(f[q]);
    }
}

// Normalized feature x split into (hi, lo) BF16 parts.
__device__ __forceinline__ void split_hi_lo(float x, __nv_bfloat16& hi, __nv_bfloat16& lo)
{
    hi = __float2bfloat16_rn(x);
    lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

#endif  // __CUDACC__

}  // namespace mlp
}  // namespace hadros
