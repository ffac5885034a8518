// hadros_mlp.cu — training kernels of the surrogate network and their C-ABI
// entry points (no counterpart in the reference).
//
// Every product of the 256-wide layers runs on the tensor cores through one
// BF16 GEMM kernel (mma.sync m16n8k16, FP32 accumulation, cp.async double
// buffering, ldmatrix with or without transposition for the three operand
// layouts of a forward and backward pass) whose epilogue is fused with the
// surrounding elementwise work:
//   forward      Z_l = H_{l-1} W_l^T + b_l,  H_l = SiLU(Z_l)     (both BF16;
//                SiLU in packed BF16 from h = Z_l / 2, hadros_mlp.cuh)
//   data grad    dZ_{l-1} = (dZ_l W_l) * SiLU'(Z_{l-1})          (BF16)
//   weight grad  G_Wl += dZ_l^T H_{l-1}   (split over the batch, FP32 atomics)
// The 2-output last layer, the loss, bias gradients and Adam are small
// CUDA-core kernels.  The FP32 master parameters live in one flat array
// (layout in hadros_mlp.cuh) so Adam is one elementwise pass.
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "hadros_b200.h"
#include "hadros_internal.h"
#include "hadros_mlp.cuh"

namespace hadros {
namespace mlp {
namespace {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16-byte global->shared copy; zero-fills when !valid (src-size 0).
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void ldsm_x4(uint32_t r[4], const void* p)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t r[4], const void* p)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ---- GEMM: C[m][n] = sum_k A(m,k) B(k,n), then epi(m, n, c[n], c[n+1]) ------
//   A_K: A(m,k) = A[m*lda + k]  (else A[k*lda + m])
//   B_K: B(k,n) = B[n*ldb + k]  (else B[k*ldb + n])
// M, N, K and the split length are multiples of 8 (16-byte chunks); rows and
// columns past M, N, K are zero-filled on load and skipped on store.
constexpr int BM = 128, BN = 128, BK = 32, kGemmThreads = 256;
constexpr int LDK = BK + 8;    // K-contiguous smem rows (80 B: conflict-free ldmatrix)
constexpr int LDMN = BM + 8;   // MN-contiguous smem rows (272 B)
constexpr int kTile = (BM * LDK > BK * LDMN) ? BM * LDK : BK * LDMN;

template <bool A_K, bool B_K, class Epi>
__global__ void __launch_bounds__(kGemmThreads)
    gemm_kernel(const bf16* __restrict__ A, long lda, const bf16* __restrict__ B, long ldb, int M,
                int N, int K, int k_split, Epi epi)
{
    __shared__ __align__(16) bf16 sA[2][kTile];
    __shared__ __align__(16) bf16 sB[2][kTile];
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kb = blockIdx.z * k_split;
    const int ke = min(K, kb + k_split);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = warp >> 2, wn = warp & 3;   // 2 x 4 warps, 64 x 32 each

    auto load = [&](int st, int k0) {
        for (int c = tid; c < 512; c += kGemmThreads) {
            if (A_K) {
                const int row = c >> 2, kc = (c & 3) * 8, gm = m0 + row, gk = k0 + kc;
                const bool v = gm < M && gk < ke;
                cp_async16(&sA[st][row * LDK + kc], v ? A + long(gm) * lda + gk : A, v);
            } else {
                const int row = c >> 4, mc = (c & 15) * 8, gk = k0 + row, gm = m0 + mc;
                const bool v = gk < ke && gm < M;
                cp_async16(&sA[st][row * LDMN + mc], v ? A + long(gk) * lda + gm : A, v);
            }
            if (B_K) {
                const int row = c >> 2, kc = (c & 3) * 8, gn = n0 + row, gk = k0 + kc;
                const bool v = gn < N && gk < ke;
                cp_async16(&sB[st][row * LDK + kc], v ? B + long(gn) * ldb + gk : B, v);
            } else {
                const int row = c >> 4, nc = (c & 15) * 8, gk = k0 + row, gn = n0 + nc;
                const bool v = gk < ke && gn < N;
                cp_async16(&sB[st][row * LDMN + nc], v ? B + long(gk) * ldb + gn : B, v);
            }
        }
    };

    float acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0f;

    const int nk = ke > kb ? (ke - kb + BK - 1) / BK : 0;
    if (nk > 0) load(0, kb);
    cp_async_commit();
    for (int t = 0; t < nk; ++t) {
        if (t + 1 < nk) load((t + 1) & 1, kb + (t + 1) * BK);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const int s = t & 1;
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
            uint32_t af[4][4], bfr[4][2];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt) {
                if (A_K) {
                    const int row = wm * 64 + mt * 16 + (lane & 15), col = ks * 16 + (lane >> 4) * 8;
                    ldsm_x4(af[mt], &sA[s][row * LDK + col]);
                } else {
                    const int krow = ks * 16 + (lane & 7) + (lane >> 4) * 8;
                    const int m = wm * 64 + mt * 16 + ((lane >> 3) & 1) * 8;
                    ldsm_x4_t(af[mt], &sA[s][krow * LDMN + m]);
                }
            }
#pragma unroll
            for (int np = 0; np < 2; ++np) {
                uint32_t r[4];
                if (B_K) {
                    const int n = wn * 32 + np * 16 + (lane & 7) + (lane >> 4) * 8;
                    const int k = ks * 16 + ((lane >> 3) & 1) * 8;
                    ldsm_x4(r, &sB[s][n * LDK + k]);
                } else {
                    const int krow = ks * 16 + (lane & 7) + ((lane >> 3) & 1) * 8;
                    const int n = wn * 32 + np * 16 + (lane >> 4) * 8;
                    ldsm_x4_t(r, &sB[s][krow * LDMN + n]);
                }
                bfr[np * 2][0] = r[0];
                bfr[np * 2][1] = r[1];
                bfr[np * 2 + 1][0] = r[2];
                bfr[np * 2 + 1][1] = r[3];
            }
#pragma unroll
            for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[mt][nt], af[mt], bfr[nt]);
        }
        __syncthreads();
    }
    cp_async_wait<0>();

    const int g = lane >> 2, c2 = (lane & 3) * 2;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int m = m0 + wm * 64 + mt * 16 + g, n = n0 + wn * 32 + nt * 8 + c2;
            if (n < N) {
                if (m < M) epi(m, n, acc[mt][nt][0], acc[mt][nt][1]);
                if (m + 8 < M) epi(m + 8, n, acc[mt][nt][2], acc[mt][nt][3]);
            }
        }
}

struct EpiHidden {   // Z = acc + b (BF16, for the backward pass), H = SiLU(acc + b)
    const float* bias;
    bf16* Z;
    bf16* H;
    __device__ void operator()(int m, int n, float v0, float v1) const
    {
        const float z0 = v0 + bias[n], z1 = v1 + bias[n + 1];
        const long o = long(m) * kW + n;
        if (Z) *reinterpret_cast<uint32_t*>(Z + o) = pack_bf16x2(z0, z1);
        *reinterpret_cast<uint32_t*>(H + o) = silu_half_bf16x2(0.5f * z0, 0.5f * z1);
    }
};

struct EpiBwdData {   // dZ_prev = acc * SiLU'(Z_prev)
    const bf16* Zp;
    bf16* dZp;
    __device__ void operator()(int m, int n, float v0, float v1) const
    {
        const long o = long(m) * kW + n;
        const float2 z = unpack_bf16x2(*reinterpret_cast<const uint32_t*>(Zp + o));
        *reinterpret_cast<uint32_t*>(dZp + o) = pack_bf16x2(v0 * silu_grad_f(z.x), v1 * silu_grad_f(z.y));
    }
};

struct EpiWgrad {   // G[m][n] += acc (partial sums over a slice of the batch)
    float* G;
    int ldg;
    __device__ void operator()(int m, int n, float v0, float v1) const
    {
        atomicAdd(G + long(m) * ldg + n, v0);
        atomicAdd(G + long(m) * ldg + n + 1, v1);
    }
};

template <bool A_K, bool B_K, class Epi>
void gemm(const bf16* A, long lda, const bf16* B, long ldb, int M, int N, int K, int splits, Epi epi,
          cudaStream_t st)
{
    int k_split = (K + splits - 1) / splits;
    k_split = (k_split + BK - 1) / BK * BK;
    splits = (K + k_split - 1) / k_split;
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, std::max(splits, 1));
    gemm_kernel<A_K, B_K, Epi><<<grid, kGemmThreads, 0, st>>>(A, lda, B, ldb, M, N, K, k_split, epi);
}

// ---- small kernels ----------------------------------------------------------

__global__ void k_pack(const float* __restrict__ master, bf16* __restrict__ packed)
{
    const long idx = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= kPacked) return;
    float v;
    if (idx < kPW2) {   // [hi 16 | lo 16 | Fourier 32] <- master [16 | 32]
        const long o = idx / kIn, c = idx % kIn;
        const long j = c < 2 * kF ? c % kF : c - kF;
        v = master[kOffW1 + o * kW1In + j];
    } else if (idx < kPW5) {
        const long r = idx - kPW2;
        const int l = 2 + int(r / (long(kW) * kW));
        v = master[off_w(l) + r % (long(kW) * kW)];
    } else {
        const long r = idx - kPW5, o = r / kW, i = r % kW;
        v = o < kOut ? master[kOffW5 + o * kW + i] : 0.0f;
    }
    packed[idx] = __float2bfloat16_rn(v);
}

__global__ void k_featurize(const float* __restrict__ raw, long n, Norm nm, bf16* __restrict__ X)
{
    const long s = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float xn[kF];
#pragma unroll
    for (int j = 0; j < kF; ++j) xn[j] = (raw[s * kF + j] - nm.feat_mu[j]) * nm.feat_inv_sd[j];
    bf16 row[kIn];
    input_row(xn, row);
#pragma unroll
    for (int q = 0; q < kIn / 8; ++q)
        reinterpret_cast<uint4*>(X + s * kIn)[q] = reinterpret_cast<const uint4*>(row)[q];
}

// out[s][o] = W5[o] . H4[s] + b5[o] + Ws[o] . x[s]   (one warp per sample)
__global__ void k_top_forward(const bf16* __restrict__ H4, const bf16* __restrict__ X,
                              const bf16* __restrict__ W5b, const float* __restrict__ master, long n,
                              float* __restrict__ out)
{
    const long s = (long(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= n) return;
    const uint4 h = *reinterpret_cast<const uint4*>(H4 + s * kW + lane * 8);
    const uint4 w0 = *reinterpret_cast<const uint4*>(W5b + lane * 8);
    const uint4 w1 = *reinterpret_cast<const uint4*>(W5b + kW + lane * 8);
    const uint32_t hv[4] = {h.x, h.y, h.z, h.w}, av[4] = {w0.x, w0.y, w0.z, w0.w},
                   bv[4] = {w1.x, w1.y, w1.z, w1.w};
    float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float2 hh = unpack_bf16x2(hv[q]), ww0 = unpack_bf16x2(av[q]), ww1 = unpack_bf16x2(bv[q]);
        a0 = fmaf(hh.x, ww0.x, fmaf(hh.y, ww0.y, a0));
        a1 = fmaf(hh.x, ww1.x, fmaf(hh.y, ww1.y, a1));
    }
    if (lane < kF) {
        const float x = __bfloat162float(X[s * kIn + lane]) + __bfloat162float(X[s * kIn + kF + lane]);
        a0 = fmaf(master[kOffWs + lane], x, a0);
        a1 = fmaf(master[kOffWs + kF + lane], x, a1);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    }
    if (lane == 0) {
        out[s * kOut] = a0 + master[kOffB5];
        out[s * kOut + 1] = a1 + master[kOffB5 + 1];
    }
}

// Weighted squared error: loss += scale * w * (out - t)^2, dout = 2 scale w (out - t).
__global__ void k_loss(const float* __restrict__ out, const float* __restrict__ t,
                       const float* __restrict__ w, long n, float scale, float* __restrict__ dout,
                       float* __restrict__ loss)
{
    __shared__ float red[32];
    float l = 0.0f;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n * kOut; i += long(gridDim.x) * blockDim.x) {
        const float ws = w ? w[i / kOut] : 1.0f;
        const float d = out[i] - t[i];
        dout[i] = 2.0f * scale * ws * d;
        l += scale * ws * d * d;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x < 32) {
        l = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
        if (threadIdx.x == 0 && loss) atomicAdd(loss, l);
    }
}

// Last layer backward over a chunk of samples; thread i = hidden unit i.
//   dZ4 = (dout . W5[:, i]) * SiLU'(Z4);  G_W5 += dout^T H4;  G_b5 += sum dout;
//   G_Ws += dout^T x.
__global__ void __launch_bounds__(kW) k_top_backward(const float* __restrict__ dout, const bf16* __restrict__ W5b,
                                                      const bf16* __restrict__ Z4, const bf16* __restrict__ H4,
                                                      const bf16* __restrict__ X, long n, int chunk,
                                                      bf16* __restrict__ dZ4, float* __restrict__ G)
{
    const int i = threadIdx.x;
    const long s0 = long(blockIdx.x) * chunk, s1 = min(n, s0 + chunk);
    const float w0 = __bfloat162float(W5b[i]), w1 = __bfloat162float(W5b[kW + i]);
    float gw0 = 0.0f, gw1 = 0.0f, gx = 0.0f;
    for (long s = s0; s < s1; ++s) {
        const float d0 = dout[s * kOut], d1 = dout[s * kOut + 1];
        const float z = __bfloat162float(Z4[s * kW + i]), h = __bfloat162float(H4[s * kW + i]);
        dZ4[s * kW + i] = __float2bfloat16_rn(fmaf(d0, w0, d1 * w1) * silu_grad_f(z));
        gw0 = fmaf(d0, h, gw0);
        gw1 = fmaf(d1, h, gw1);
        if (i < 2 * kF) {
            const int j = i & (kF - 1);
            const float x = __bfloat162float(X[s * kIn + j]) + __bfloat162float(X[s * kIn + kF + j]);
            gx = fmaf(i < kF ? d0 : d1, x, gx);
        } else if (i < 2 * kF + kOut) {
            gx += (i == 2 * kF) ? d0 : d1;
        }
    }
    atomicAdd(G + kOffW5 + i, gw0);
    atomicAdd(G + kOffW5 + kW + i, gw1);
    if (i < 2 * kF) atomicAdd(G + kOffWs + i, gx);
    else if (i < 2 * kF + kOut) atomicAdd(G + kOffB5 + (i - 2 * kF), gx);
}

__global__ void __launch_bounds__(kW) k_bias_grad(const bf16* __restrict__ dZ, long n, int chunk,
                                                   float* __restrict__ Gb)
{
    const int i = threadIdx.x;
    const long s0 = long(blockIdx.x) * chunk, s1 = min(n, s0 + chunk);
    float g = 0.0f;
    for (long s = s0; s < s1; ++s) g += __bfloat162float(dZ[s * kW + i]);
    atomicAdd(Gb + i, g);
}

// Tied hi/lo first-layer weights: G_W1[o][j] += dW[o][j] + dW[o][j+16] for
// the features, G_W1[o][16+q] += dW[o][32+q] for the Fourier columns.
__global__ void k_fold_w1(const float* __restrict__ dW1, float* __restrict__ G)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= kW * kW1In) return;
    const int o = idx / kW1In, j = idx % kW1In;
    G[kOffW1 + idx] += j < kF ? dW1[o * kIn + j] + dW1[o * kIn + kF + j] : dW1[o * kIn + kF + j];
}

__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, long count, float lr, float b1, float b2, float eps,
                       float inv_bc1, float inv_bc2)
{
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i];
    const float mi = fmaf(b1, m[i], (1.0f - b1) * gi);
    const float vi = fmaf(b2, v[i], (1.0f - b2) * gi * gi);
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * inv_bc1) / (sqrtf(vi * inv_bc2) + eps);
}

struct Workspace {
    bf16* Z[kDepth + 1];
    bf16* H[kDepth + 1];
    bf16* dZa;
    bf16* dZb;
    float* dW1;
};

Workspace carve(void* ws, long n)
{
    char* p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(ws) + kWsAlign - 1) / kWsAlign * kWsAlign);
    const long a = ws_act_bytes(n);
    Workspace w{};
    for (int l = 1; l <= kDepth; ++l) {
        w.Z[l] = reinterpret_cast<bf16*>(p + (l - 1) * a);
        w.H[l] = reinterpret_cast<bf16*>(p + (kDepth + l - 1) * a);
    }
    w.dZa = reinterpret_cast<bf16*>(p + 8 * a);
    w.dZb = reinterpret_cast<bf16*>(p + 9 * a);
    w.dW1 = reinterpret_cast<float*>(p + 10 * a);
    return w;
}

int32_t cuda_status(const char* what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(HADROS_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return HADROS_OK;
}

int blocks_for(long count, int threads) { return int((count + threads - 1) / threads); }

void forward_impl(const float* master, const bf16* packed, const bf16* X, long n, const Workspace& w,
                  float* out, cudaStream_t st)
{
    const int M = int(n);
    gemm<true, true>(X, kIn, packed + pw(1), kIn, M, kW, kIn, 1,
                     EpiHidden{master + off_b(1), w.Z[1], w.H[1]}, st);
    for (int l = 2; l <= kDepth; ++l)
        gemm<true, true>(w.H[l - 1], kW, packed + pw(l), kW, M, kW, kW, 1,
                         EpiHidden{master + off_b(l), w.Z[l], w.H[l]}, st);
    k_top_forward<<<blocks_for(n * 32, 256), 256, 0, st>>>(w.H[kDepth], X, packed + pw(5), master, n, out);
}

void backward_impl(const bf16* packed, const bf16* X, long n, const float* dout, const Workspace& w,
                   float* G, cudaStream_t st)
{
    const int M = int(n);
    const int chunk = 64;
    const int wsplits = int(std::min<long>(64, std::max<long>(1, n / 512)));
    bf16* dZ = w.dZa;
    bf16* dZn = w.dZb;
    k_top_backward<<<blocks_for(n, chunk), kW, 0, st>>>(dout, packed + pw(5), w.Z[kDepth], w.H[kDepth], X, n,
                                                        chunk, dZ, G);
    for (int l = kDepth; l >= 2; --l) {
        gemm<false, false>(dZ, kW, w.H[l - 1], kW, kW, kW, M, wsplits, EpiWgrad{G + off_w(l), kW}, st);
        k_bias_grad<<<blocks_for(n, chunk), kW, 0, st>>>(dZ, n, chunk, G + off_b(l));
        gemm<true, false>(dZ, kW, packed + pw(l), kW, M, kW, kW, 1, EpiBwdData{w.Z[l - 1], dZn}, st);
        std::swap(dZ, dZn);
    }
    cudaMemsetAsync(w.dW1, 0, sizeof(float) * kW * kIn, st);
    gemm<false, false>(dZ, kW, X, kIn, kW, kIn, M, wsplits, EpiWgrad{w.dW1, kIn}, st);
    k_bias_grad<<<blocks_for(n, chunk), kW, 0, st>>>(dZ, n, chunk, G + off_b(1));
    k_fold_w1<<<blocks_for(kW * kW1In, 256), 256, 0, st>>>(w.dW1, G);
}

Norm to_norm(const hadros_mlp_norm& a)
{
    Norm nm{};
    for (int j = 0; j < kF; ++j) {
        nm.feat_mu[j] = a.feat_mu[j];
        nm.feat_inv_sd[j] = a.feat_inv_sd[j];
    }
    for (int o = 0; o < kOut; ++o) {
        nm.out_mu[o] = a.out_mu[o];
        nm.out_sd[o] = a.out_sd[o];
        nm.out_floor[o] = a.out_floor[o];
    }
    return nm;
}

}  // namespace
}  // namespace mlp
}  // namespace hadros

using namespace hadros;
using namespace hadros::mlp;

static_assert(sizeof(hadros_mlp_norm) == sizeof(Norm), "hadros_mlp_norm must mirror mlp::Norm");

extern "C" {

int64_t hadros_mlp_param_count(void) { return kParams; }
int64_t hadros_mlp_packed_count(void) { return kPacked; }
int64_t hadros_mlp_workspace_bytes(int64_t batch) { return batch > 0 ? ws_bytes(batch) : 0; }

int32_t hadros_mlp_layout(int64_t* offsets, int32_t n)
{
    const int64_t v[12] = {kOffW1, kOffB1, off_w(2), off_b(2), off_w(3), off_b(3), off_w(4), off_b(4),
                           kOffW5, kOffB5, kOffWs, kParamsUsed};
    if (!offsets || n < 12) return set_error(HADROS_E_ARG, "hadros_mlp_layout needs 12 slots");
    for (int i = 0; i < 12; ++i) offsets[i] = v[i];
    return HADROS_OK;
}

int32_t hadros_mlp_pack(const float* master, void* packed, void* stream)
{
    if (!master || !packed) return set_error(HADROS_E_ARG, "NULL argument");
    auto st = static_cast<cudaStream_t>(stream);
    k_pack<<<blocks_for(kPacked, 256), 256, 0, st>>>(master, static_cast<bf16*>(packed));
    return cuda_status("hadros_mlp_pack");
}

int32_t hadros_mlp_featurize(const float* raw, int64_t n, const hadros_mlp_norm* norm, void* X, void* stream)
{
    if (!raw || !norm || !X || n < 0) return set_error(HADROS_E_ARG, "bad argument");
    if (n == 0) return HADROS_OK;
    auto st = static_cast<cudaStream_t>(stream);
    k_featurize<<<blocks_for(n, 256), 256, 0, st>>>(raw, n, to_norm(*norm), static_cast<bf16*>(X));
    return cuda_status("hadros_mlp_featurize");
}

int32_t hadros_mlp_forward(const float* master, const void* packed, const void* X, int64_t n,
                           void* workspace, float* out, void* stream)
{
    if (!master || !packed || !X || !workspace || !out || n <= 0 || n > (int64_t(1) << 30))
        return set_error(HADROS_E_ARG, "bad argument (n must be in 1..2^30)");
    const Workspace w = carve(workspace, n);
    forward_impl(master, static_cast<const bf16*>(packed), static_cast<const bf16*>(X), n, w, out,
                 static_cast<cudaStream_t>(stream));
    return cuda_status("hadros_mlp_forward");
}

int32_t hadros_mlp_backward(const void* packed, const void* X, int64_t n, const float* dout, void* workspace,
                            float* grad, void* stream)
{
    if (!packed || !X || !dout || !workspace || !grad || n <= 0 || n > (int64_t(1) << 30))
        return set_error(HADROS_E_ARG, "bad argument (n must be in 1..2^30)");
    const Workspace w = carve(workspace, n);
    backward_impl(static_cast<const bf16*>(packed), static_cast<const bf16*>(X), n, dout, w, grad,
                  static_cast<cudaStream_t>(stream));
    return cuda_status("hadros_mlp_backward");
}

int32_t hadros_mlp_loss(const float* out, const float* target, const float* weight, int64_t n, float* dout,
                        float* loss, void* stream)
{
    if (!out || !target || !dout || n <= 0) return set_error(HADROS_E_ARG, "bad argument");
    const int blocks = std::min(blocks_for(n * kOut, 256), 1024);
    k_loss<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(out, target, weight, n,
                                                                   1.0f / float(n * kOut), dout, loss);
    return cuda_status("hadros_mlp_loss");
}

int32_t hadros_mlp_adam(float* master, float* m, float* v, const float* grad, const hadros_adam* opt,
                        int64_t step, void* stream)
{
    if (!master || !m || !v || !grad || !opt || step < 1) return set_error(HADROS_E_ARG, "bad argument");
    const float bc1 = 1.0f - std::pow(opt->beta1, float(step));
    const float bc2 = 1.0f - std::pow(opt->beta2, float(step));
    k_adam<<<blocks_for(kParamsUsed, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        master, m, v, grad, kParamsUsed, opt->lr, opt->beta1, opt->beta2, opt->eps, 1.0f / bc1, 1.0f / bc2);
    return cuda_status("hadros_mlp_adam");
}

int32_t hadros_mlp_train_step(float* master, void* packed, float* m, float* v, const void* X,
                              const float* target, const float* weight, int64_t n, const hadros_adam* opt,
                              int64_t step, void* workspace, float* grad, float* out, float* dout, float* loss,
                              void* stream)
{
    if (!master || !packed || !m || !v || !X || !target || !opt || !workspace || !grad || !out || !dout ||
        n <= 0 || n > (int64_t(1) << 30) || step < 1)
        return set_error(HADROS_E_ARG, "bad argument");
    auto st = static_cast<cudaStream_t>(stream);
    const Workspace w = carve(workspace, n);
    auto* pk = static_cast<bf16*>(packed);
    auto* x = static_cast<const bf16*>(X);
    forward_impl(master, pk, x, n, w, out, st);
    if (int32_t rc = hadros_mlp_loss(out, target, weight, n, dout, loss, stream)) return rc;
    cudaMemsetAsync(grad, 0, sizeof(float) * kParams, st);
    backward_impl(pk, x, n, dout, w, grad, st);
    if (int32_t rc = hadros_mlp_adam(master, m, v, grad, opt, step, stream)) return rc;
    k_pack<<<blocks_for(kPacked, 256), 256, 0, st>>>(master, pk);
    return cuda_status("hadros_mlp_train_step");
}

}  // extern "C"
