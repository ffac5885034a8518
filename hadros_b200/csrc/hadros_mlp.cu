// hadros_mlp.cu — training kernels of the surrogate network and their C-ABI
// entry points (no counterpart in the reference).
//
// Every product of the 256-wide layers runs on the 5th-generation tensor
// cores through one GEMM kernel (tcgen05.mma into tensor memory, BF16
// operands, FP32 accumulation; operands staged by cp.async in the 128-byte
// swizzled K-major or MN-major layouts the three products of a forward and
// backward pass need) whose epilogue is fused with the surrounding
// elementwise work:
//   forward      Z_l = H_{l-1} W_l^T + b_l,  H_l = SiLU(Z_l)     (both BF16;
//                SiLU in packed BF16 from h = Z_l / 2, hadros_mlp.cuh)
//   data grad    dZ_{l-1} = (dZ_l W_l) * SiLU'(Z_{l-1})          (BF16)
//   weight grad  G_Wl += dZ_l^T H_{l-1}   (split over the batch, FP32 vector
//                reductions)
// Several networks (the members of an ensemble) train side by side in the
// same launches (hadros_mlp_train_members).  The 2-output last layer, the
// loss, bias gradients and Adam are small CUDA-core kernels.  The FP32 master
// parameters live in one flat array (layout in hadros_mlp.cuh) so Adam is one
// elementwise pass.
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "hadros_b200.h"
#include "hadros_internal.h"
#include "hadros_mlp.cuh"
#include "hadros_umma.cuh"

namespace hadros {
namespace mlp {
namespace {

using bf16 = __nv_bfloat16;

// 16-byte global->shared copy; zero-fills when !valid (src-size 0).
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ---- GEMM on the 5th-generation tensor cores -----------------------------------
// C[m][n] = sum_k A(m,k) B(k,n) for k in one split [kb, kb + k_split), then
// epi(member, m, n0, 32 FP32 values of columns n0..n0+31).
//   A_MN: A(m,k) = A[k*lda + m] (MN-major), else A[m*lda + k] (K-major)
//   B_MN: B(k,n) = B[k*ldb + n] (MN-major), else B[n*ldb + k] (K-major)
// One CTA computes a 128 x BN tile (BN = 256 or 64) of one member
// (grid.z = member * splits + split).  K runs in chunks of 64 through a
// two-stage shared-memory ring that all eight warps fill with cp.async, each
// 16-byte unit written where the 128-byte swizzle of the UMMA layout puts it:
// K-major tiles are rows of 64 k (128 B) in 8-row groups 1024 B apart;
// MN-major tiles are atoms of 64 m or n (one 128-byte row per k) by 8 k,
// atoms along K 1024 B apart and along MN 8 KB apart.  One thread issues
// tcgen05.mma (M = 128, N = BN, K = 16, BF16 -> FP32) into a TMEM accumulator
// and commits each chunk to that stage's mbarrier, which frees the stage for
// the chunk two ahead.  In the epilogue warp w reads, with tcgen05.ld, the 32
// rows of TMEM lane quarter w % 4 in column half w / 4.  Two stages (98 KB of
// shared memory) let two CTAs share an SM (2 x BN <= 512 TMEM columns), so one
// CTA's epilogue overlaps the other's loads and MMAs: the tiles here have
// only K = 256 (four chunks), and with one CTA per SM the epilogue and the
// load latency left the tensor pipe idle ~90 % of the time.
// Rows and k beyond M, K load as zeros and are not stored.
// Every wait is bounded; a timeout stores NaN in *fail (the step's loss),
// which the host sees.
constexpr int UM = 128, UK = 64, kUStages = 2, kUThreads = 256;
constexpr int kMnLbo = (UK / 8) * 1024;   // MN-major: bytes between 64-wide MN blocks

template <int BN>
struct UTile {
    static constexpr int kA = UM * UK * 2;
    static constexpr int kB = BN * UK * 2;
    static constexpr int kStage = kA + kB;
    static constexpr int kSmem = kUStages * kStage + 1024 + 128;
};

template <bool A_MN, bool B_MN, int BN, class Epi>
__global__ void __launch_bounds__(kUThreads, 2)
    umma_gemm(const bf16* __restrict__ A, long lda, long a_mem, const bf16* __restrict__ B, long ldb, long b_mem,
              int M, int N, int K, int k_split, int splits, Epi epi, float* fail)
{
    using namespace umma;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kUStages * UTile<BN>::kStage);
    uint64_t* mma_done = bars;                    // [kUStages]
    uint64_t* acc_ready = bars + kUStages;
    uint64_t* drain = bars + kUStages + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + kUStages + 2);
    __shared__ int s_abort;
    volatile int* abort_flag = &s_abort;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mem = blockIdx.z / splits, split = blockIdx.z % splits;
    A += mem * a_mem;
    B += mem * b_mem;
    const int m0 = blockIdx.y * UM, n0 = blockIdx.x * BN;
    const int kb = split * k_split;
    const int ke = min(K, kb + k_split);
    const int nk = ke > kb ? (ke - kb + UK - 1) / UK : 0;

    if (tid == 0) {
        s_abort = 0;
        for (int s = 0; s < kUStages; ++s) mbar_init(saddr(&mma_done[s]), 1);
        mbar_init(saddr(acc_ready), 1);
        mbar_init(saddr(drain), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(tmem_slot)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    auto load = [&](int st, int k0) {
        const uint32_t sa = saddr(smem + st * UTile<BN>::kStage);
        const uint32_t sb = sa + UTile<BN>::kA;
        if (!A_MN) {
            for (int c = tid; c < UM * 8; c += kUThreads) {
                const int row = c >> 3, u = c & 7, gm = m0 + row, gk = k0 + u * 8;
                const bool v = gm < M && gk < ke;
                cp_async16(sa + row * 128 + ((u ^ (row & 7)) << 4), v ? A + long(gm) * lda + gk : A, v);
            }
        } else {
            for (int c = tid; c < UK * (UM / 8); c += kUThreads) {
                const int kr = c / (UM / 8), u = c % (UM / 8), gk = k0 + kr, gm = m0 + u * 8;
                const bool v = gk < ke && gm < M;
                cp_async16(sa + (u >> 3) * kMnLbo + (kr >> 3) * 1024 + (kr & 7) * 128 + (((u & 7) ^ (kr & 7)) << 4),
                           v ? A + long(gk) * lda + gm : A, v);
            }
        }
        if (!B_MN) {
            for (int c = tid; c < BN * 8; c += kUThreads) {
                const int row = c >> 3, u = c & 7, gn = n0 + row, gk = k0 + u * 8;
                const bool v = gn < N && gk < ke;
                cp_async16(sb + row * 128 + ((u ^ (row & 7)) << 4), v ? B + long(gn) * ldb + gk : B, v);
            }
        } else {
            for (int c = tid; c < UK * (BN / 8); c += kUThreads) {
                const int kr = c / (BN / 8), u = c % (BN / 8), gk = k0 + kr, gn = n0 + u * 8;
                const bool v = gk < ke && gn < N;
                cp_async16(sb + (u >> 3) * kMnLbo + (kr >> 3) * 1024 + (kr & 7) * 128 + (((u & 7) ^ (kr & 7)) << 4),
                           v ? B + long(gk) * ldb + gn : B, v);
            }
        }
    };

    constexpr uint32_t idesc = idesc_bf16_major(UM, BN, A_MN, B_MN);
    bool mma_issued = false;
    for (int t = 0; t < kUStages - 1; ++t) {
        if (t < nk) load(t, kb + t * UK);
        cp_async_commit();
    }
    for (int t = 0; t < nk; ++t) {
        const int tl = t + kUStages - 1;   // the chunk loaded now, into the stage chunk t-1 used
        if (tl < nk) {
            const int st = tl % kUStages;
            bool ok = true;
            if (tl >= kUStages) ok = mbar_wait(saddr(&mma_done[st]), uint32_t((tl / kUStages - 1) & 1), abort_flag);
            if (ok) load(st, kb + tl * UK);
        }
        cp_async_commit();
        cp_async_wait<kUStages - 1>();    // this thread's copies of chunk t have landed
        fence_async_smem();               // and are visible to the tensor cores
        __syncthreads();
        if (tid == 0 && !*abort_flag) {
            tc_fence_after();
            const uint32_t sa = saddr(smem + (t % kUStages) * UTile<BN>::kStage);
            const uint32_t sb = sa + UTile<BN>::kA;
            for (int kk = 0; kk < UK / 16; ++kk) {
                const uint64_t da = A_MN ? sdesc_mn(sa + kk * 2048, kMnLbo, 1024) : sdesc(sa + kk * 32);
                const uint64_t db = B_MN ? sdesc_mn(sb + kk * 2048, kMnLbo, 1024) : sdesc(sb + kk * 32);
                tc_mma(tmem, da, db, idesc, (t | kk) != 0);
            }
            mma_issued = true;
            tc_commit(saddr(&mma_done[t % kUStages]));
        }
    }
    cp_async_wait<0>();
    if (tid == 0) {
        if (mma_issued) tc_commit(saddr(acc_ready));
        else mbar_arrive(saddr(acc_ready));   // nothing accumulated: the epilogue adds zeros
    }
    const bool ok = warp_wait(saddr(acc_ready), 0, abort_flag);
    tc_fence_after();
    if (ok && !*abort_flag) {
        const int quarter = warp & 3, half = warp >> 2;
        const uint32_t lane_base = tmem + (uint32_t(quarter * 32) << 16);
        const int m = m0 + quarter * 32 + lane;
        uint32_t v[32];
#pragma unroll 1
        for (int cb = half * (BN / 2); cb < (half + 1) * (BN / 2); cb += 32) {
            tc_ld32(lane_base + uint32_t(cb), v);
            tc_wait_ld(v);
            if (nk == 0) {
#pragma unroll
                for (int q = 0; q < 32; ++q) v[q] = 0u;
            }
            if (m < M && n0 + cb < N) epi(mem, m, n0 + cb, reinterpret_cast<const float*>(v));
        }
    }
    if (*abort_flag && tid == 0) {
        *fail = __int_as_float(0x7fc00000);
        if (mma_issued) {   // let the MMAs in flight finish before TMEM is released
            tc_commit(saddr(drain));
            mbar_wait_plain(saddr(drain), 0);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(BN) : "memory");
}

struct EpiHidden {   // Z = acc + b (BF16, for the backward pass), H = SiLU(acc + b)
    const float* bias;
    long bias_mem;    // floats between members' biases
    bf16* Z;
    bf16* H;
    long act_mem;     // elements between members' activations
    __device__ void operator()(int mem, int m, int n, const float* v) const
    {
        const float* b = bias + mem * bias_mem + n;
        const long o = mem * act_mem + long(m) * kW + n;
        uint32_t z[16], h[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const float z0 = v[2 * q] + b[2 * q], z1 = v[2 * q + 1] + b[2 * q + 1];
            z[q] = pack_bf16x2(z0, z1);
            h[q] = silu_half_bf16x2(0.5f * z0, 0.5f * z1);
        }
        if (Z)
#pragma unroll
            for (int u = 0; u < 4; ++u)
                *reinterpret_cast<uint4*>(Z + o + 8 * u) = make_uint4(z[4 * u], z[4 * u + 1], z[4 * u + 2], z[4 * u + 3]);
#pragma unroll
        for (int u = 0; u < 4; ++u)
            *reinterpret_cast<uint4*>(H + o + 8 * u) = make_uint4(h[4 * u], h[4 * u + 1], h[4 * u + 2], h[4 * u + 3]);
    }
};

struct EpiBwdData {   // dZ_prev = acc * SiLU'(Z_prev)
    const bf16* Zp;
    bf16* dZp;
    long act_mem;
    __device__ void operator()(int mem, int m, int n, const float* v) const
    {
        const long o = mem * act_mem + long(m) * kW + n;
        uint32_t d[16];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint4 zz = *reinterpret_cast<const uint4*>(Zp + o + 8 * u);
            const uint32_t zw[4] = {zz.x, zz.y, zz.z, zz.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float2 z = unpack_bf16x2(zw[q]);
                const int c = 8 * u + 2 * q;
                d[4 * u + q] = pack_bf16x2(v[c] * silu_grad_f(z.x), v[c + 1] * silu_grad_f(z.y));
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            *reinterpret_cast<uint4*>(dZp + o + 8 * u) = make_uint4(d[4 * u], d[4 * u + 1], d[4 * u + 2], d[4 * u + 3]);
    }
};

struct EpiWgrad {   // G[m][n] += acc (partial sums over a slice of the batch)
    float* G;
    int ldg;
    long g_mem;       // floats between members' gradients
    __device__ void operator()(int mem, int m, int n, const float* v) const
    {
        float* g = G + mem * g_mem + long(m) * ldg + n;
#pragma unroll
        for (int q = 0; q < 32; q += 4)
            asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"l"(g + q), "f"(v[q]), "f"(v[q + 1]),
                         "f"(v[q + 2]), "f"(v[q + 3])
                         : "memory");
    }
};

template <bool A_MN, bool B_MN, int BN, class Epi>
void gemm(const bf16* A, long lda, long a_mem, const bf16* B, long ldb, long b_mem, int M, int N, int K, int splits,
          int members, Epi epi, float* fail, cudaStream_t st)
{
    int k_split = (K + splits - 1) / splits;
    k_split = (k_split + UK - 1) / UK * UK;
    splits = std::max((K + k_split - 1) / k_split, 1);
    auto kern = umma_gemm<A_MN, B_MN, BN, Epi>;
    // set once per process (and device 0's context first): later launches,
    // such as those captured into a CUDA graph, only enqueue the kernel
    static thread_local int attr_device = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_device != dev) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, UTile<BN>::kSmem);
        attr_device = dev;
    }
    dim3 grid((N + BN - 1) / BN, (M + UM - 1) / UM, members * splits);
    kern<<<grid, kUThreads, UTile<BN>::kSmem, st>>>(A, lda, a_mem, B, ldb, b_mem, M, N, K, k_split, splits, epi,
                                                   fail);
}

// ---- small kernels ----------------------------------------------------------

__global__ void k_pack(const float* __restrict__ master, bf16* __restrict__ packed)
{
    master += long(blockIdx.y) * kParams;
    packed += long(blockIdx.y) * kPacked;
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

// Strides between the arrays of networks trained side by side; the small
// kernels take their member from blockIdx.y.
struct Mem {
    long x;     // input rows X (elements)
    long p;     // packed weights (elements)
    long m;     // master parameters and gradients (floats)
    long act;   // workspace activations (elements)
    long n;     // samples per member
};

// out[s][o] = W5[o] . H4[s] + b5[o] + Ws[o] . x[s]   (one warp per sample)
__global__ void k_top_forward(const bf16* __restrict__ H4, const bf16* __restrict__ X,
                              const bf16* __restrict__ W5b, const float* __restrict__ master, Mem mm,
                              float* __restrict__ out)
{
    const int k = blockIdx.y;
    H4 += k * mm.act;
    X += k * mm.x;
    W5b += k * mm.p;
    master += k * mm.m;
    out += k * mm.n * kOut;
    const long n = mm.n;
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

// Weighted squared error: loss[k] += scale * w * (out - t)^2, dout = 2 scale w (out - t).
__global__ void k_loss(const float* __restrict__ out, const float* __restrict__ t,
                       const float* __restrict__ w, long n, float scale, float* __restrict__ dout,
                       float* __restrict__ loss)
{
    __shared__ float red[32];
    const int k = blockIdx.y;
    out += k * n * kOut;
    t += k * n * kOut;
    dout += k * n * kOut;
    if (w) w += k * n;
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
        if (threadIdx.x == 0 && loss) atomicAdd(loss + k, l);
    }
}

// Last layer backward over a chunk of samples; thread i = hidden unit i.
//   dZ4 = (dout . W5[:, i]) * SiLU'(Z4);  G_W5 += dout^T H4;  G_b5 += sum dout;
//   G_Ws += dout^T x.
__global__ void __launch_bounds__(kW) k_top_backward(const float* __restrict__ dout, const bf16* __restrict__ W5b,
                                                      const bf16* __restrict__ Z4, const bf16* __restrict__ H4,
                                                      const bf16* __restrict__ X, Mem mm, int chunk,
                                                      bf16* __restrict__ dZ4, float* __restrict__ G)
{
    const int k = blockIdx.y;
    const long n = mm.n;
    dout += k * n * kOut;
    W5b += k * mm.p;
    Z4 += k * mm.act;
    H4 += k * mm.act;
    X += k * mm.x;
    dZ4 += k * mm.act;
    G += k * mm.m;
    const int i = threadIdx.x;
    const long s0 = long(blockIdx.x) * chunk, s1 = min(n, s0 + chunk);
    const float w0 = __bfloat162float(W5b[i]), w1 = __bfloat162float(W5b[kW + i]);
    float gw0 = 0.0f, gw1 = 0.0f, gx = 0.0f;
    // unrolled so that several samples' loads are in flight at once (the
    // loop is otherwise bound by one load latency per sample)
#pragma unroll 8
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

__global__ void __launch_bounds__(kW) k_bias_grad(const bf16* __restrict__ dZ, Mem mm, int chunk, long g_off,
                                                   float* __restrict__ G)
{
    const int k = blockIdx.y;
    dZ += k * mm.act;
    float* Gb = G + k * mm.m + g_off;
    const int i = threadIdx.x;
    const long s0 = long(blockIdx.x) * chunk, s1 = min(mm.n, s0 + chunk);
    // four partial sums, so that four samples' loads are in flight at once
    float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f, g3 = 0.0f;
    long s = s0;
    for (; s + 4 <= s1; s += 4) {
        g0 += __bfloat162float(dZ[s * kW + i]);
        g1 += __bfloat162float(dZ[(s + 1) * kW + i]);
        g2 += __bfloat162float(dZ[(s + 2) * kW + i]);
        g3 += __bfloat162float(dZ[(s + 3) * kW + i]);
    }
    for (; s < s1; ++s) g0 += __bfloat162float(dZ[s * kW + i]);
    atomicAdd(Gb + i, (g0 + g1) + (g2 + g3));
}

// Tied hi/lo first-layer weights: G_W1[o][j] += dW[o][j] + dW[o][j+16] for
// the features, G_W1[o][16+q] += dW[o][32+q] for the Fourier columns.
// dW1 of member k at dW1 + k * dw_mem floats.
__global__ void k_fold_w1(const float* __restrict__ dW1, long dw_mem, float* __restrict__ G, long g_mem)
{
    const int k = blockIdx.y;
    dW1 += k * dw_mem;
    G += k * g_mem;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= kW * kW1In) return;
    const int o = idx / kW1In, j = idx % kW1In;
    G[kOffW1 + idx] += j < kF ? dW1[o * kIn + j] + dW1[o * kIn + kF + j] : dW1[o * kIn + kF + j];
}

__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, long count, long stride, float lr, float b1, float b2,
                       float eps, float inv_bc1, float inv_bc2)
{
    const long off = long(blockIdx.y) * stride;
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[off + i];
    const float mi = fmaf(b1, m[off + i], (1.0f - b1) * gi);
    const float vi = fmaf(b2, v[off + i], (1.0f - b2) * gi * gi);
    m[off + i] = mi;
    v[off + i] = vi;
    w[off + i] -= lr * (mi * inv_bc1) / (sqrtf(vi * inv_bc2) + eps);
}

// Per-step values of a graph-replayed training run, written on the device by
// k_step_begin (so a captured step reads the values of the step it runs).
struct StepDev {
    float lr, inv_bc1, inv_bc2;
    int64_t idx_off;   // first row of this step's batch in each member's index list
};

// ++step; the cosine learning rate lr_min + (lr_max - lr_min)(1 + cos(pi t))/2,
// t = (step - 1) / (total - 1); Adam's bias corrections; the batch offset.
__global__ void k_step_begin(int64_t* step, hadros_train_sched sc, long n, StepDev* out)
{
    const int64_t st = ++*step;
    const double t = double(st - 1) / double(sc.total_steps > 1 ? sc.total_steps - 1 : 1);
    out->lr = float(sc.lr_min + 0.5 * (sc.lr_max - sc.lr_min) * (1.0 + cos(3.141592653589793 * (t < 1.0 ? t : 1.0))));
    out->inv_bc1 = 1.0f / (1.0f - powf(sc.beta1, float(st)));
    out->inv_bc2 = 1.0f / (1.0f - powf(sc.beta2, float(st)));
    out->idx_off = ((st - 1) % (sc.steps_per_epoch > 0 ? sc.steps_per_epoch : 1)) * n;
}

// Adam with the step's values from the device.
__global__ void k_adam_dev(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ g, long count, long stride, const StepDev* sd, float b1,
                           float b2, float eps)
{
    const long off = long(blockIdx.y) * stride;
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float lr = sd->lr, inv_bc1 = sd->inv_bc1, inv_bc2 = sd->inv_bc2;
    const float gi = g[off + i];
    const float mi = fmaf(b1, m[off + i], (1.0f - b1) * gi);
    const float vi = fmaf(b2, v[off + i], (1.0f - b2) * gi * gi);
    m[off + i] = mi;
    v[off + i] = vi;
    w[off + i] -= lr * (mi * inv_bc1) / (sqrtf(vi * inv_bc2) + eps);
}

// Rows idx[k][s] of the shared inputs and targets -> member k's batch.
__global__ void k_gather(const bf16* __restrict__ X_all, const float* __restrict__ T_all,
                         const float* __restrict__ W_all, const int64_t* __restrict__ idx, long idx_mem, long n,
                         bf16* __restrict__ X, float* __restrict__ T, float* __restrict__ Wt,
                         const StepDev* sd)
{
    const int k = blockIdx.y;
    const long s = long(blockIdx.x) * (blockDim.x / 8) + threadIdx.x / 8;
    const int u = threadIdx.x & 7;   // 16-byte unit of the 128-byte row
    if (s >= n) return;
    const int64_t r = idx[k * idx_mem + (sd ? sd->idx_off : 0) + s];
    reinterpret_cast<uint4*>(X + (k * n + s) * kIn)[u] = reinterpret_cast<const uint4*>(X_all + r * kIn)[u];
    if (u < kOut) T[(k * n + s) * kOut + u] = T_all[r * kOut + u];
    if (u == kOut && W_all) Wt[k * n + s] = W_all[r];
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

// One training step's buffers of `members` networks trained side by side
// (each member's arrays follow one another at the given strides).
struct Batch {
    int members;
    long n;                 // samples per member
    long x_mem;             // elements between members' input rows X [n][kIn]
    long p_mem;             // elements between members' packed weights
    long m_mem;             // floats between members' master parameters / gradients
    long ws_mem;            // bytes between members' workspaces (a multiple of kWsAlign)
    Mem mem() const { return Mem{x_mem, p_mem, m_mem, ws_mem / 2, n}; }
};

void forward_impl(const float* master, const bf16* packed, const bf16* X, const Batch& bt, void* ws, float* out,
                  float* fail, cudaStream_t st)
{
    const int M = int(bt.n);
    const Workspace w = carve(ws, bt.n);
    const Mem mm = bt.mem();
    gemm<false, false, 256>(X, kIn, bt.x_mem, packed + pw(1), kIn, bt.p_mem, M, kW, kIn, 1, bt.members,
                            EpiHidden{master + off_b(1), bt.m_mem, w.Z[1], w.H[1], mm.act}, fail, st);
    for (int l = 2; l <= kDepth; ++l)
        gemm<false, false, 256>(w.H[l - 1], kW, mm.act, packed + pw(l), kW, bt.p_mem, M, kW, kW, 1, bt.members,
                                EpiHidden{master + off_b(l), bt.m_mem, w.Z[l], w.H[l], mm.act}, fail, st);
    k_top_forward<<<dim3(blocks_for(bt.n * 32, 256), bt.members), 256, 0, st>>>(w.H[kDepth], X, packed + pw(5),
                                                                                master, mm, out);
}

void backward_impl(const bf16* packed, const bf16* X, const Batch& bt, const float* dout, void* ws, float* G,
                   float* fail, cudaStream_t st)
{
    const int M = int(bt.n);
    const long n = bt.n;
    const int chunk = 64;
    const int wsplits = int(std::min<long>(32, std::max<long>(1, n / 256)));
    const Mem mm = bt.mem();
    const dim3 gchunk(blocks_for(n, chunk), bt.members);
    const Workspace w = carve(ws, n);
    bf16* dZ = w.dZa;
    bf16* dZn = w.dZb;
    k_top_backward<<<gchunk, kW, 0, st>>>(dout, packed + pw(5), w.Z[kDepth], w.H[kDepth], X, mm, chunk, dZ, G);
    for (int l = kDepth; l >= 2; --l) {
        // G_l += dZ_l^T H_{l-1}: both operands MN-major (the samples are K)
        gemm<true, true, 256>(dZ, kW, mm.act, w.H[l - 1], kW, mm.act, kW, kW, M, wsplits, bt.members,
                              EpiWgrad{G + off_w(l), kW, bt.m_mem}, fail, st);
        k_bias_grad<<<gchunk, kW, 0, st>>>(dZ, mm, chunk, off_b(l), G);
        // dZ_{l-1} = (dZ_l W_l) * SiLU'(Z_{l-1}): W_l[out][in] is the MN-major B
        gemm<false, true, 256>(dZ, kW, mm.act, packed + pw(l), kW, bt.p_mem, M, kW, kW, 1, bt.members,
                               EpiBwdData{w.Z[l - 1], dZn, mm.act}, fail, st);
        std::swap(dZ, dZn);
    }
    const long dw_mem = bt.ws_mem / 4;   // floats between members' dW1
    for (int k = 0; k < bt.members; ++k) cudaMemsetAsync(w.dW1 + k * dw_mem, 0, sizeof(float) * kW * kIn, st);
    gemm<true, true, 64>(dZ, kW, mm.act, X, kIn, bt.x_mem, kW, kIn, M, wsplits, bt.members,
                         EpiWgrad{w.dW1, kIn, dw_mem}, fail, st);
    k_bias_grad<<<gchunk, kW, 0, st>>>(dZ, mm, chunk, off_b(1), G);
    k_fold_w1<<<dim3(blocks_for(kW * kW1In, 256), bt.members), 256, 0, st>>>(w.dW1, dw_mem, G, bt.m_mem);
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
    const Batch bt{1, n, 0, 0, 0, 0};
    // a timed-out wait in a GEMM stores NaN in out[0]
    forward_impl(master, static_cast<const bf16*>(packed), static_cast<const bf16*>(X), bt, workspace, out, out,
                 static_cast<cudaStream_t>(stream));
    return cuda_status("hadros_mlp_forward");
}

int32_t hadros_mlp_backward(const void* packed, const void* X, int64_t n, const float* dout, void* workspace,
                            float* grad, void* stream)
{
    if (!packed || !X || !dout || !workspace || !grad || n <= 0 || n > (int64_t(1) << 30))
        return set_error(HADROS_E_ARG, "bad argument (n must be in 1..2^30)");
    const Batch bt{1, n, 0, 0, 0, 0};
    // a timed-out wait in a GEMM stores NaN in grad[0]
    backward_impl(static_cast<const bf16*>(packed), static_cast<const bf16*>(X), bt, dout, workspace, grad, grad,
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
        master, m, v, grad, kParamsUsed, kParams, opt->lr, opt->beta1, opt->beta2, opt->eps, 1.0f / bc1,
        1.0f / bc2);
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
    auto* pk = static_cast<bf16*>(packed);
    auto* x = static_cast<const bf16*>(X);
    const Batch bt{1, n, 0, 0, 0, 0};
    forward_impl(master, pk, x, bt, workspace, out, loss ? loss : out, st);
    if (int32_t rc = hadros_mlp_loss(out, target, weight, n, dout, loss, stream)) return rc;
    cudaMemsetAsync(grad, 0, sizeof(float) * kParams, st);
    backward_impl(pk, x, bt, dout, workspace, grad, loss ? loss : grad, st);
    if (int32_t rc = hadros_mlp_adam(master, m, v, grad, opt, step, stream)) return rc;
    k_pack<<<blocks_for(kPacked, 256), 256, 0, st>>>(master, pk);
    return cuda_status("hadros_mlp_train_step");
}

int64_t hadros_mlp_members_workspace_bytes(int32_t members, int64_t batch)
{
    if (members < 1 || batch < 1) return 0;
    return int64_t(members) * (ws_bytes(batch) + members_batch_bytes(batch)) + kWsAlign;
}

int32_t hadros_mlp_train_members(int32_t members, int64_t n, const void* X_all, const float* T_all,
                                 const float* W_all, const int64_t* idx, int64_t idx_stride, float* masters,
                                 void* packed, float* m, float* v, float* grad, const hadros_adam* opt,
                                 int64_t step, void* workspace, float* loss, void* stream)
{
    if (members < 1 || members > 64 || n <= 0 || n > (int64_t(1) << 26) || !X_all || !T_all || !idx ||
        !masters || !packed || !m || !v || !grad || !opt || !workspace || !loss || step < 1 || idx_stride < n)
        return set_error(HADROS_E_ARG, "bad argument");
    auto st = static_cast<cudaStream_t>(stream);
    // workspace: each member's layer workspace, then the members' batch buffers
    char* base =
        reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(workspace) + kWsAlign - 1) / kWsAlign * kWsAlign);
    const long wsb = ws_bytes(n);
    char* bb = base + long(members) * wsb;
    auto* X = reinterpret_cast<bf16*>(bb);
    auto* T = reinterpret_cast<float*>(bb + long(members) * n * kIn * 2);
    auto* Wt = T + long(members) * n * kOut;
    auto* out = Wt + long(members) * n;
    auto* dout = out + long(members) * n * kOut;
    k_gather<<<dim3(blocks_for(n * 8, 256), members), 256, 0, st>>>(
        static_cast<const bf16*>(X_all), T_all, W_all, idx, idx_stride, n, X, T, W_all ? Wt : nullptr, nullptr);
    auto* pk = static_cast<bf16*>(packed);
    const Batch bt{members, n, n * kIn, kPacked, kParams, wsb};
    forward_impl(masters, pk, X, bt, base, out, loss, st);
    k_loss<<<dim3(std::min(blocks_for(n * kOut, 256), 1024), members), 256, 0, st>>>(
        out, T, W_all ? Wt : nullptr, n, 1.0f / float(n * kOut), dout, loss);
    cudaMemsetAsync(grad, 0, sizeof(float) * kParams * members, st);
    backward_impl(pk, X, bt, dout, base, grad, loss, st);
    const float bc1 = 1.0f - std::pow(opt->beta1, float(step));
    const float bc2 = 1.0f - std::pow(opt->beta2, float(step));
    k_adam<<<dim3(blocks_for(kParamsUsed, 256), members), 256, 0, st>>>(
        masters, m, v, grad, kParamsUsed, kParams, opt->lr, opt->beta1, opt->beta2, opt->eps, 1.0f / bc1,
        1.0f / bc2);
    k_pack<<<dim3(blocks_for(kPacked, 256), members), 256, 0, st>>>(masters, pk);
    return cuda_status("hadros_mlp_train_members");
}

int32_t hadros_mlp_train_members_dev(int32_t members, int64_t n, const void* X_all, const float* T_all,
                                     const float* W_all, const int64_t* idx, int64_t idx_stride, float* masters,
                                     void* packed, float* m, float* v, float* grad, const hadros_train_sched* sched,
                                     int64_t* step_dev, void* workspace, float* loss, void* stream)
{
    if (members < 1 || members > 64 || n <= 0 || n > (int64_t(1) << 26) || !X_all || !T_all || !idx ||
        !masters || !packed || !m || !v || !grad || !sched || !step_dev || !workspace || !loss ||
        sched->steps_per_epoch < 1 || sched->total_steps < 1 || idx_stride < n * sched->steps_per_epoch)
        return set_error(HADROS_E_ARG, "bad argument");
    auto st = static_cast<cudaStream_t>(stream);
    char* base =
        reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(workspace) + kWsAlign - 1) / kWsAlign * kWsAlign);
    const long wsb = ws_bytes(n);
    char* bb = base + long(members) * wsb;
    auto* X = reinterpret_cast<bf16*>(bb);
    auto* T = reinterpret_cast<float*>(bb + long(members) * n * kIn * 2);
    auto* Wt = T + long(members) * n * kOut;
    auto* out = Wt + long(members) * n;
    auto* dout = out + long(members) * n * kOut;
    // the step's values sit past the members' batch buffers (members_batch_bytes rounds up)
    auto* sd = reinterpret_cast<StepDev*>(
        (reinterpret_cast<uintptr_t>(dout + long(members) * n * kOut) + 15) / 16 * 16);
    k_step_begin<<<1, 1, 0, st>>>(step_dev, *sched, n, sd);
    k_gather<<<dim3(blocks_for(n * 8, 256), members), 256, 0, st>>>(
        static_cast<const bf16*>(X_all), T_all, W_all, idx, idx_stride, n, X, T, W_all ? Wt : nullptr, sd);
    auto* pk = static_cast<bf16*>(packed);
    const Batch bt{members, n, n * kIn, kPacked, kParams, wsb};
    forward_impl(masters, pk, X, bt, base, out, loss, st);
    k_loss<<<dim3(std::min(blocks_for(n * kOut, 256), 1024), members), 256, 0, st>>>(
        out, T, W_all ? Wt : nullptr, n, 1.0f / float(n * kOut), dout, loss);
    cudaMemsetAsync(grad, 0, sizeof(float) * kParams * members, st);
    backward_impl(pk, X, bt, dout, base, grad, loss, st);
    k_adam_dev<<<dim3(blocks_for(kParamsUsed, 256), members), 256, 0, st>>>(
        masters, m, v, grad, kParamsUsed, kParams, sd, sched->beta1, sched->beta2, sched->eps);
    k_pack<<<dim3(blocks_for(kPacked, 256), members), 256, 0, st>>>(masters, pk);
    return cuda_status("hadros_mlp_train_members_dev");
}

}  // extern "C"
