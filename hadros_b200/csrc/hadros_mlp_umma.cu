// hadros_mlp_umma.cu — surrogate inference on the 5th-generation tensor cores
// (tcgen05), plus the sample features shared with training (no counterpart
// in the reference).
//
// One persistent CTA per SM evaluates every ensemble member on 256 samples
// (pixel, bin) at a time, the whole network chain without leaving the SM:
//   - the epilogue warps build each sample's features in the kernel (the same
//     device function as hadros_mlp_raw_features, which feeds training), and
//     write them, then each layer's SiLU activations, as BF16 into shared
//     memory in the UMMA K-major 128-byte-swizzled layout;
//   - one thread issues tcgen05.mma (M=128, N=256, K=16, BF16 in, FP32 out)
//     for the two 128-row halves into two TMEM accumulators (512 columns);
//   - one thread streams the weights (pre-swizzled "images", 32 KB stages)
//     with cp.async.bulk into a two-slot ring; both halves use each stage;
//   - the epilogue reads TMEM with tcgen05.ld, adds bias, applies SiLU and
//     stores the next layer's operand; after the last layer it de-standardizes
//     ln tau_E and ln I_E, and reduces each pixel's bins (log-sum-exp of
//     ln I_E + ln dE) per member, giving the ensemble spread of ln I_obs.
// Pixels whose spread exceeds the threshold are appended to a fallback list
// for the exact tracer.  Every wait is bounded: on timeout the kernel sets an
// abort flag that the host reports as HADROS_E_TIMEOUT.
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "hadros_b200.h"
#include "hadros_internal.h"
#include "hadros_mlp.cuh"
#include "hadros_umma.cuh"

namespace hadros {
namespace mlp {
namespace {

using bf16 = __nv_bfloat16;
using namespace umma;

constexpr int kMaxBinsS = 128;   // bins of a surrogate camera
constexpr int kTileRows = 128;   // rows of one TMEM accumulator
constexpr int kPair = 2;         // accumulators per CTA pass (256 samples)
constexpr int kStageBytes = 32768;           // [256 rows x 64 K] BF16, 128B-swizzled
constexpr int kStages = 2;                   // weight ring slots
constexpr int kStagesPerMember = 14;         // L1: 1, L2..L4: 4 each, L5: 1
constexpr int kLastStageBytes = 8192;        // L5: 4 chunks of [16 x 64]
constexpr long kImageBytes = long(kStagesPerMember - 1) * kStageBytes + kLastStageBytes;
constexpr int kActBytes = 4 * 16384;         // [128 rows x 256 K] as 4 swizzled chunks
constexpr int kEpiWarps = 16;   // 4 per 32-row TMEM lane quarter: 2 accumulators x 2 column halves
constexpr int kThreads = (kEpiWarps + 2) * 32;   // + MMA warp + producer warp
constexpr int kMaxMembers = 8;

// Camera and bins of one surrogate image (kernel parameter).
struct SurCam {
    int32_t nx, ny, n_bins, profile;
    float inv_nx, inv_ny, c_alpha, c_beta;
    float a, cos_i, log_rho0, r0, h_over_r;
    float log10E[kMaxBinsS];
    float ln_dE[kMaxBinsS];   // -inf for bins outside the aggregates
    float w[kMaxBinsS];       // aggregation weight (0 outside)
    float wsum;               // sum of w
    float ln_sw[kMaxBinsS];   // spread: log-sum-exp over bins of out + ln_sw
    int32_t spread_out;       // 0: ln I_E (ln_sw = ln dE), 1: ln tau_E (ln w / sum w)
};

// The 16 raw features of sample (pixel, bin): the single definition used for
// training rows and inference rows.
__device__ __forceinline__ void raw_features(const SurCam& c, long pixel, int bin, float f[kF])
{
    const int i = int(pixel % c.nx), j = int(pixel / c.nx);
    f[0] = (float(2 * i + 1) * c.inv_nx - 1.0f) * c.c_alpha;
    f[1] = (float(2 * j + 1) * c.inv_ny - 1.0f) * c.c_beta;
    f[2] = c.a;
    f[3] = c.cos_i;
    f[4] = c.log_rho0;
#pragma unroll
    for (int q = 0; q < 8; ++q) f[5 + q] = (q == c.profile) ? 1.0f : 0.0f;
    f[13] = c.r0;
    f[14] = c.h_over_r;
    f[15] = c.log10E[bin];
}

__global__ void k_raw_features(SurCam c, const int32_t* __restrict__ pixel_ids, long n_pixels,
                               float* __restrict__ raw)
{
    const long idx = long(blockIdx.x) * blockDim.x + threadIdx.x;
    const long n = n_pixels * c.n_bins;
    if (idx >= n) return;
    const long p = idx / c.n_bins;
    const int b = int(idx % c.n_bins);
    float f[kF];
    raw_features(c, pixel_ids ? long(pixel_ids[p]) : p, b, f);
#pragma unroll
    for (int q = 0; q < kF; ++q) raw[idx * kF + q] = f[q];
}

// ---- weight images ------------------------------------------------------------
// A K-major 128B-swizzled block has rows of 64 BF16 (128 B); the 16-byte unit
// u of row r is stored at unit u ^ (r % 8).
// One thread per 16-byte unit of the image of one network.
__global__ void k_pack_image(const bf16* __restrict__ packed, uint8_t* __restrict__ image)
{
    const long u = long(blockIdx.x) * blockDim.x + threadIdx.x;   // 16-byte unit
    if (u >= kImageBytes / 16) return;
    const long byte = u * 16;
    const int q = int(byte / kStageBytes);
    const int in = int(byte % kStageBytes);
    uint4 v = make_uint4(0, 0, 0, 0);
    bf16 e[8];
    int row, unit, c, l;
    if (q < kStagesPerMember - 1) {
        row = in / 128;                       // 0..255 = output unit n
        unit = (in % 128) / 16;               // physical unit
        const int kunit = unit ^ (row & 7);   // logical 16-byte unit
        if (q == 0) {                         // W1 [256][64]
            for (int t = 0; t < 8; ++t) e[t] = packed[pw(1) + long(row) * kIn + kunit * 8 + t];
        } else {
            l = 2 + (q - 1) / 4;
            c = (q - 1) % 4;
            for (int t = 0; t < 8; ++t) e[t] = packed[pw(l) + long(row) * kW + c * 64 + kunit * 8 + t];
        }
    } else {                                  // W5 [16][256]: chunk c at c * 2048
        c = in / 2048;
        const int r = in % 2048;
        row = r / 128;
        unit = (r % 128) / 16;
        const int kunit = unit ^ (row & 7);
        for (int t = 0; t < 8; ++t) e[t] = packed[pw(5) + long(row) * kW + c * 64 + kunit * 8 + t];
    }
    if (q < kStagesPerMember - 1)   // hidden layers: weights / 2 (exact), see epi_chunk
        for (int t = 0; t < 8; ++t) e[t] = __float2bfloat16_rn(0.5f * __bfloat162float(e[t]));
    v = *reinterpret_cast<const uint4*>(e);
    *reinterpret_cast<uint4*>(image + byte) = v;
}

// Bias, SiLU and BF16 store of 32 accumulator columns [cb, cb+32) of row r.
// The weights and biases of the hidden layers are pre-scaled by 1/2, so the
// accumulator plus bias is h = z / 2.
__device__ __forceinline__ void epi_chunk(uint32_t (&v)[32], const float* sb, int cb, uint8_t* act, int r)
{
    uint32_t h[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        add_f32x2(v[2 * q], v[2 * q + 1], *reinterpret_cast<const float2*>(sb + cb + 2 * q));
        h[q] = silu_half_bf16x2(__uint_as_float(v[2 * q]), __uint_as_float(v[2 * q + 1]));
    }
    uint8_t* chunk = act + (cb >> 6) * 16384 + r * 128;
    const int u0 = (cb & 63) >> 3;   // logical 16-byte unit of column cb
#pragma unroll
    for (int u = 0; u < 4; ++u)
        *reinterpret_cast<uint4*>(chunk + (((u0 + u) ^ (r & 7)) << 4)) =
            make_uint4(h[4 * u], h[4 * u + 1], h[4 * u + 2], h[4 * u + 3]);
}

struct InferArgs {
    SurCam cam;
    Norm norm;
    const float* masters;     // [members][kParams]
    const uint8_t* images;    // [members][kImageBytes]
    int32_t members;
    int64_t pixel_begin, n_pixels;
    float spread_threshold;
    float* ln_tau_E;          // [n_pixels][B] (may be NULL)
    float* ln_I_E;            // [n_pixels][B] (may be NULL)
    double* tau;
    double* P_surv;
    double* I_obs;
    float* spread;
    int32_t* fallback_ids;
    int32_t* counters;        // [0] fallback count, [1] abort flag
};

constexpr int kBiasFloats = 4 * kW + kOut + kOut * kF + 6;   // + padding to 8 bytes
constexpr int kSmemBytes = kPair * kActBytes + kStages * kStageBytes + 2 * 256 * 4 + 4 * kBiasFloats * 4 + 256 + 1024;

// First stage (in a member's weight image) of layer L and its stage count.
__host__ __device__ constexpr int stage_of(int L) { return L == 1 ? 0 : (L == 5 ? kStagesPerMember - 1 : 1 + (L - 2) * 4); }
__host__ __device__ constexpr int stages_in(int L) { return (L == 1 || L == 5) ? 1 : 4; }
static_assert(kSmemBytes <= 232448, "shared memory above the sm_100 per-block limit");

// PP = false: the two 128-row halves go through each layer together, each
// weight stage feeding both (half the weight traffic, but the tensor cores
// idle during the epilogue).  PP = true ("ping-pong"): the halves take turns,
// so one half's epilogue overlaps the other half's MMAs; every weight stage
// is streamed once per half.
template <bool PP>
__global__ void __launch_bounds__(kThreads, 1) k_infer(const InferArgs A)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* act = smem;                                      // [2][64 KB]
    uint8_t* stage = smem + kPair * kActBytes;                // [2][32 KB]
    float* red_a = reinterpret_cast<float*>(stage + kStages * kStageBytes);   // [256]
    float* red_b = red_a + 256;                                               // [256]
    float* sbias = red_b + 256;        // per epilogue group and member parity: b1..b4 [4][256], b5 [2], Ws [2][16]
    uint64_t* bars = reinterpret_cast<uint64_t*>(sbias + 4 * kBiasFloats);
    uint64_t* full = bars;                 // [kStages]
    uint64_t* empty = bars + kStages;      // [kStages]
    uint64_t* acc_full = bars + 2 * kStages;        // [2] (PP: one per half)
    uint64_t* act_ready = bars + 2 * kStages + 2;   // [2]
    uint64_t* epi_bar = bars + 2 * kStages + 4;     // [2] barrier of an epilogue group
    uint64_t* drain = bars + 2 * kStages + 6;       // abort path: MMAs in flight
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 7);
    constexpr int kGroups = PP ? 2 : 1;             // epilogue groups (and MMA turns per layer)
    constexpr int kGroupWarps = kEpiWarps / kGroups;
    volatile int* abort_flag = A.counters + 1;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int B = A.cam.n_bins;
    const long n_samples = A.n_pixels * B;
    const long n_tiles = (n_samples + kPair * kTileRows - 1) / (kPair * kTileRows);
    const int K = A.members;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(saddr(&full[s]), 1);
            mbar_init(saddr(&empty[s]), 1);
        }
        for (int g = 0; g < 2; ++g) {
            mbar_init(saddr(&acc_full[g]), 1);
            mbar_init(saddr(&act_ready[g]), kGroupWarps);
            mbar_init(saddr(&epi_bar[g]), kGroupWarps * 32);
        }
        mbar_init(saddr(drain), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        fence_async_smem();
    }
    if (warp == 0) {   // 512 TMEM columns: two 128 x 256 FP32 accumulators
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(tmem_slot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    long issued = 0;          // producer: stages issued
    bool mma_issued = false;  // MMA thread: any tcgen05.mma issued
    uint32_t epi_phase = 0;   // epilogue barrier phase
    const int grp = PP ? (warp >> 2) & 1 : 0;
    auto epi_sync = [&]() -> bool {
        mbar_arrive(saddr(&epi_bar[grp]));
        const bool ok = warp_wait(saddr(&epi_bar[grp]), epi_phase, abort_flag);
        epi_phase ^= 1u;
        return ok;
    };

    if (warp == kEpiWarps + 1) {
        // ---- producer: per member, each layer's stages (once per MMA turn) ---
        if (lane == 0) {
            for (long tile = blockIdx.x; tile < n_tiles && !*abort_flag; tile += gridDim.x)
                for (int k = 0; k < K; ++k)
                    for (int L = 1; L <= 5; ++L)
                        for (int tt = 0; tt < kGroups; ++tt)
                            for (int c = 0; c < stages_in(L); ++c, ++issued) {
                        const int q = stage_of(L) + c;
                        const long i = issued;
                        const int slot = int(i % kStages);
                        const uint32_t ph = uint32_t((i / kStages) & 1);
                        if (!mbar_wait(saddr(&empty[slot]), ph ^ 1u, abort_flag)) goto done;
                        const uint32_t bytes = q == kStagesPerMember - 1 ? kLastStageBytes : kStageBytes;
                        mbar_expect_tx(saddr(&full[slot]), bytes);
                        bulk_g2s(saddr(stage + slot * kStageBytes), A.images + k * kImageBytes + long(q) * kStageBytes,
                                 bytes, saddr(&full[slot]));
                    }
        }
    } else if (warp == kEpiWarps) {
        // ---- MMA issuer ---------------------------------------------------------
        if (lane == 0) {
            long i = 0, layer_count = 0;
            const uint32_t id256 = idesc_bf16(128, 256), id16 = idesc_bf16(128, 16);
            for (long tile = blockIdx.x; tile < n_tiles && !*abort_flag; tile += gridDim.x)
                for (int k = 0; k < K; ++k)
                    for (int L = 1; L <= 5; ++L, ++layer_count)
                      for (int tt = 0; tt < kGroups; ++tt) {
                        if (!mbar_wait(saddr(&act_ready[tt]), uint32_t(layer_count & 1), abort_flag)) goto done;
                        tc_fence_after();
                        const int nst = stages_in(L);
                        for (int c = 0; c < nst; ++c, ++i) {
                            const int slot = int(i % kStages);
                            if (!mbar_wait(saddr(&full[slot]), uint32_t((i / kStages) & 1), abort_flag)) goto done;
                            tc_fence_after();
                            const uint32_t sb = saddr(stage + slot * kStageBytes);
                            mma_issued = true;
                            for (int t = PP ? tt : 0; t < (PP ? tt + 1 : kPair); ++t) {
                                const uint32_t ab = saddr(act + t * kActBytes);
                                const uint32_t d = tmem + uint32_t(t * 256);
                                if (L == 1) {          // K = 64 from chunk 0
                                    for (int kk = 0; kk < 4; ++kk)
                                        tc_mma(d, sdesc(ab + kk * 32), sdesc(sb + kk * 32), id256, kk > 0);
                                } else if (L == 5) {   // N = 16, K = 256 over 4 chunks of the stage
                                    for (int cc = 0; cc < 4; ++cc)
                                        for (int kk = 0; kk < 4; ++kk)
                                            tc_mma(d, sdesc(ab + cc * 16384 + kk * 32), sdesc(sb + cc * 2048 + kk * 32),
                                                   id16, (cc | kk) != 0);
                                } else {               // K chunk c of 64
                                    for (int kk = 0; kk < 4; ++kk)
                                        tc_mma(d, sdesc(ab + c * 16384 + kk * 32), sdesc(sb + kk * 32), id256,
                                               (c | kk) != 0);
                                }
                            }
                            tc_commit(saddr(&empty[slot]));   // slot free once these MMAs finish
                        }
                        tc_commit(saddr(&acc_full[tt]));       // layer done (for this turn)
                      }
        }
    } else {
        // ---- epilogue warps ------------------------------------------------------
        // Warp w takes TMEM lane quarter w % 4 (rows qw*32..+31) of accumulator
        // t = (w / 4) % 2 and column half cpart = w / 8 (columns cpart*128..+127):
        // two warps share each row, each evaluating half of its columns, which
        // doubles the warps that hide the TMEM-load and barrier latency of the
        // epilogue.  The column-half-0 ("lead") warp also does the row's last
        // layer, the skip connection and the per-pixel reductions.
        const int qw = warp & 3, t = (warp >> 2) & 1, cpart = warp >> 3;
        const bool lead = cpart == 0;
        const int r = qw * 32 + lane;                 // row in the 128-row half
        const int trow = t * kTileRows + r;           // row in the 256-sample tile
        uint8_t* my_act = act + t * kActBytes;
        long member_count = 0;   // biases are double-buffered by member parity
        // Segmented reduction over the B consecutive rows (threads) of a pixel:
        // on entry m = this row's log-sum-exp term, x1, x2 this row's plain
        // terms; on exit m = the pixel's maximum, se = sum exp(term - m), x1, x2
        // the pixel's sums.  Pixels of <= 32 bins reduce within a warp; larger
        // ones combine their warps through shared memory.
        // Only the lead warps hold the values; the others take part in the
        // group's barriers.
        auto pixel_reduce = [&](float& m, float& se, float& x1, float& x2) -> bool {
            if (lead) {
                const int width = B < 32 ? B : 32;
                const float v = m;
                for (int off = 1; off < width; off <<= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
                se = (m == -INFINITY) ? 0.0f : __expf(v - m);
                for (int off = 1; off < width; off <<= 1) {
                    se += __shfl_xor_sync(0xffffffffu, se, off);
                    x1 += __shfl_xor_sync(0xffffffffu, x1, off);
                    x2 += __shfl_xor_sync(0xffffffffu, x2, off);
                }
            }
            if (B > 32) {
                float* wr = red_a + (t * 4 + qw) * 4;
                if (lead && lane == 0) {
                    wr[0] = m;
                    wr[1] = se;
                    wr[2] = x1;
                    wr[3] = x2;
                }
                if (!epi_sync()) return false;
                if (lead) {
                    const int nw = B / 32, w0 = t * 4 + (qw / nw) * nw;
                    float M = -INFINITY;
                    for (int j = 0; j < nw; ++j) M = fmaxf(M, red_a[(w0 + j) * 4]);
                    float S = 0.0f, X1 = 0.0f, X2 = 0.0f;
                    for (int j = 0; j < nw; ++j) {
                        const float* q = red_a + (w0 + j) * 4;
                        S += (q[0] == -INFINITY) ? 0.0f : q[1] * __expf(q[0] - M);
                        X1 += q[2];
                        X2 += q[3];
                    }
                    m = M;
                    se = S;
                    x1 = X1;
                    x2 = X2;
                }
                if (!epi_sync()) return false;   // slots free for the next reduction
            }
            return true;
        };
        const uint32_t lane_base = tmem + (uint32_t(qw * 32) << 16) + uint32_t(t * 256);
        long layer_count = 0;
        const bool leader_possible = lead && (trow % B) == 0;
        for (long tile = blockIdx.x; tile < n_tiles && __all_sync(0xffffffffu, *abort_flag == 0);
             tile += gridDim.x) {
            const long s = tile * (kPair * kTileRows) + trow;
            const bool valid = s < n_samples;
            const long lp = valid ? s / B : 0;
            const int b = valid ? int(s % B) : 0;
            // this warp's half of the input row: units 0..3 (hi, lo) for column
            // half 0, units 4..7 (Fourier features) for column half 1
            uint32_t feat[kIn / 4];
            {
                float f[kF], xn[kF];
                raw_features(A.cam, A.pixel_begin + lp, b, f);
#pragma unroll
                for (int q = 0; q < kF; ++q) xn[q] = valid ? (f[q] - A.norm.feat_mu[q]) * A.norm.feat_inv_sd[q] : 0.0f;
                __align__(16) bf16 row[kIn];
                input_row(xn, row);
#pragma unroll
                for (int q = 0; q < kIn / 4; ++q)
                    feat[q] = reinterpret_cast<const uint32_t*>(row)[cpart * (kIn / 4) + q];
            }
            float sum_tau = 0.0f, sum_lnI = 0.0f;
            float w_ref = 0.0f, w_s1 = 0.0f, w_s2 = 0.0f;   // pixel leader: shifted sums of ln I_k
            for (int k = 0; k < K; ++k, ++member_count) {
                const float* P = A.masters + long(k) * kParams;
                float* my_bias = sbias + (grp * 2 + int(member_count & 1)) * kBiasFloats;
                // this member's biases and skip weights -> shared memory (this
                // buffer was last read two members ago, before the barrier below
                // of the previous member)
                {
                    const int gt = PP ? cpart * kTileRows + r : cpart * 2 * kTileRows + trow;   // thread in the group
                    for (int e = gt; e < 4 * kW; e += kGroupWarps * 32)   // hidden biases / 2
                        my_bias[e] = 0.5f * P[off_b(1 + e / kW) + e % kW];
                    if (gt < kOut) my_bias[4 * kW + gt] = P[kOffB5 + gt];
                    if (gt < kOut * kF) my_bias[4 * kW + kOut + gt] = P[kOffWs + gt];
                }
                // features -> chunk 0: this warp's four 16-byte units of row r
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int uu = cpart * 4 + u;
                    *reinterpret_cast<uint4*>(my_act + r * 128 + ((uu ^ (r & 7)) << 4)) =
                        make_uint4(feat[4 * u], feat[4 * u + 1], feat[4 * u + 2], feat[4 * u + 3]);
                }
                fence_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(saddr(&act_ready[grp]));
                if (!epi_sync()) goto done;   // biases visible to every epilogue thread
                for (int L = 1; L <= 4; ++L, ++layer_count) {
                    if (!warp_wait(saddr(&acc_full[grp]), uint32_t(layer_count & 1), abort_flag)) goto done;
                    tc_fence_after();
                    const float* sb = my_bias + (L - 1) * kW;
                    // this warp's 128 columns, 32 at a time (the warp that shares
                    // the row hides this warp's TMEM-load latency)
                    const int c0 = cpart * (kW / 2), c1 = c0 + kW / 2;
                    uint32_t v[32];
#pragma unroll 1
                    for (int cb = c0; cb < c1; cb += 32) {
                        tc_ld32(lane_base + uint32_t(cb), v);
                        tc_wait_ld(v);
                        epi_chunk(v, sb, cb, my_act, r);
                    }
                    tc_fence_before();
                    fence_async_smem();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(saddr(&act_ready[grp]));
                }
                // last layer: 2 outputs (+ bias + FP32 skip), de-standardized
                if (!warp_wait(saddr(&acc_full[grp]), uint32_t(layer_count & 1), abort_flag)) goto done;
                ++layer_count;
                tc_fence_after();
                float ltau = 0.0f, lnI = 0.0f;
                if (lead) {   // the lead warp holds the hi and lo units of the skip input
                    uint32_t o0, o1;
                    tc_ld2(lane_base, o0, o1);
                    tc_wait_ld(o0, o1);
                    const float* st = my_bias + 4 * kW;
                    float a0 = __uint_as_float(o0) + st[0], a1 = __uint_as_float(o1) + st[1];
#pragma unroll
                    for (int q = 0; q < kF / 2; ++q) {   // skip input x = hi + lo, from the feature registers
                        const float2 hi = unpack_bf16x2(feat[q]), lo = unpack_bf16x2(feat[kF / 2 + q]);
                        const float x0 = hi.x + lo.x, x1 = hi.y + lo.y;
                        a0 = fmaf(st[kOut + 2 * q], x0, fmaf(st[kOut + 2 * q + 1], x1, a0));
                        a1 = fmaf(st[kOut + kF + 2 * q], x0, fmaf(st[kOut + kF + 2 * q + 1], x1, a1));
                    }
                    ltau = fmaf(a0, A.norm.out_sd[0], A.norm.out_mu[0]);
                    lnI = fmaf(a1, A.norm.out_sd[1], A.norm.out_mu[1]);
                }
                tc_fence_before();
                sum_tau += ltau;
                sum_lnI += lnI;
                // this member's ln I_obs (or ln tau) per pixel: log-sum-exp over the bins
                {
                    float m = valid ? (A.cam.spread_out ? ltau : lnI) + A.cam.ln_sw[b] : -INFINITY;
                    float se, x1 = 0.0f, x2 = 0.0f;
                    if (!pixel_reduce(m, se, x1, x2)) goto done;
                    if (leader_possible && valid) {
                        const float Lk = m + __logf(se);
                        if (k == 0) w_ref = Lk;
                        const float d = Lk - w_ref;
                        w_s1 += d;
                        w_s2 += d * d;
                    }
                }
            }
            // ensemble means -> per-sample outputs and per-pixel aggregates
            const float inv_k = 1.0f / float(K);
            const float ltau = sum_tau * inv_k, lnI = sum_lnI * inv_k;
            if (valid && lead) {
                if (A.ln_tau_E) A.ln_tau_E[s] = ltau;
                if (A.ln_I_E) A.ln_I_E[s] = lnI;
            }
            {
                const float tau_b = valid ? fmaxf(__expf(ltau) - A.norm.out_floor[0], 0.0f) : 0.0f;
                const float wb = valid ? A.cam.w[b] : 0.0f;
                float m = valid ? lnI + A.cam.ln_dE[b] : -INFINITY;
                float se, x1 = wb * tau_b, x2 = wb * __expf(-tau_b);
                if (!pixel_reduce(m, se, x1, x2)) goto done;
                if (leader_possible && valid) {
                    const double wsum = A.cam.wsum;
                    const double I = m > -INFINITY ? exp(double(m)) * double(se) : 0.0;
                    const float mean = w_s1 * inv_k;
                    const float sd = sqrtf(fmaxf(w_s2 * inv_k - mean * mean, 0.0f));
                    A.tau[lp] = wsum > 0.0 ? double(x1) / wsum : 0.0;
                    A.P_surv[lp] = wsum > 0.0 ? double(x2) / wsum : 1.0;
                    A.I_obs[lp] = I;
                    A.spread[lp] = sd;
                    if (sd > A.spread_threshold) {
                        const int slot = atomicAdd(A.counters, 1);
                        A.fallback_ids[slot] = int32_t(A.pixel_begin + lp);
                    }
                }
            }
        }
    }
done:
    if (*abort_flag) {
        // Abort path: let the MMAs and bulk copies this CTA issued finish
        // before its shared memory and TMEM are released.
        if (warp == kEpiWarps && lane == 0 && mma_issued) {
            tc_commit(saddr(drain));
            mbar_wait_plain(saddr(drain), 0);
        }
        if (warp == kEpiWarps + 1 && lane == 0)
            for (long j = issued - 1; j >= 0 && j >= issued - kStages; --j)
                mbar_wait_plain(saddr(&full[j % kStages]), uint32_t((j / kStages) & 1));
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512) : "memory");
}

std::atomic<int32_t> g_schedule{HADROS_SURROGATE_PINGPONG};

int32_t cuda_status(const char* what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(HADROS_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return HADROS_OK;
}

// Camera constants and bins of a surrogate image from the tracer's params.
int32_t make_surcam(const hadros_params* p, const hadros_sigma* s, SurCam* c, int32_t spread_out = 0)
{
    if (int32_t rc = hadros_params_validate(p)) return rc;
    const int B = p->spectral_kind == HADROS_SPECTRAL_MONOCHROMATIC ? 1 : p->n_bins;
    if (B < 1 || B > kMaxBinsS)
        return set_error(HADROS_E_ARG, "the surrogate handles 1.." + std::to_string(kMaxBinsS) + " bins");
    std::vector<double> E(B), dE(B), w(B);
    std::vector<int8_t> valid(B);
    int32_t nb = 0;
    if (int32_t rc = hadros_spectral_bins(p, s, E.data(), dE.data(), w.data(), valid.data(), &nb)) return rc;
    *c = SurCam{};
    c->nx = p->nx;
    c->ny = p->ny;
    c->n_bins = nb;
    c->profile = p->profile_kind;
    c->inv_nx = 1.0f / float(p->nx);
    c->inv_ny = 1.0f / float(p->ny);
    const double th = std::tan(0.5 * p->fov_deg * M_PI / 180.0) * p->r_obs_rg;
    c->c_alpha = float(th);
    c->c_beta = float(th);
    c->a = float(p->a_spin);
    c->cos_i = float(std::cos(p->theta_obs_rad));
    c->log_rho0 = float(std::log10(p->rho0_gcm3));
    c->r0 = float(p->r0_rg);
    c->h_over_r = float(p->H_over_R);
    double wsum = 0.0;
    for (int b = 0; b < nb; ++b) {
        c->log10E[b] = E[b] > 0.0 ? float(std::log10(E[b])) : 0.0f;
        const bool in = valid[b] != 0 && dE[b] > 0.0;
        c->ln_dE[b] = in ? float(std::log(dE[b])) : -INFINITY;
        c->w[b] = in ? float(w[b]) : 0.0f;
        if (in && w[b] > 0.0) wsum += w[b];
    }
    c->spread_out = spread_out;
    c->wsum = float(wsum);
    for (int b = 0; b < nb; ++b) {
        const bool in = valid[b] != 0 && dE[b] > 0.0;
        if (spread_out == 0) c->ln_sw[b] = c->ln_dE[b];
        else c->ln_sw[b] = (in && w[b] > 0.0 && wsum > 0.0) ? float(std::log(w[b] / wsum)) : -INFINITY;
    }
    return HADROS_OK;
}

}  // namespace
}  // namespace mlp
}  // namespace hadros

using namespace hadros;
using namespace hadros::mlp;

extern "C" {

int64_t hadros_mlp_image_bytes(void) { return kImageBytes; }

int32_t hadros_surrogate_schedule(int32_t schedule)
{
    if (schedule == -1) return g_schedule.load();
    if (schedule != HADROS_SURROGATE_LOCKSTEP && schedule != HADROS_SURROGATE_PINGPONG)
        return set_error(HADROS_E_ARG, "unknown surrogate schedule");
    g_schedule.store(schedule);
    return HADROS_OK;
}

int32_t hadros_mlp_pack_image(const void* packed, void* image, void* stream)
{
    if (!packed || !image) return set_error(HADROS_E_ARG, "NULL argument");
    if (reinterpret_cast<uintptr_t>(image) % 16 != 0) return set_error(HADROS_E_ARG, "image must be 16-byte aligned");
    const long units = kImageBytes / 16;
    k_pack_image<<<int((units + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const bf16*>(packed), static_cast<uint8_t*>(image));
    return cuda_status("hadros_mlp_pack_image");
}

int32_t hadros_mlp_raw_features(const hadros_params* p, const hadros_sigma* s, const int32_t* pixel_ids,
                                int64_t n_pixels, float* raw, void* stream)
{
    if (!p || !s || !raw || n_pixels < 0) return set_error(HADROS_E_ARG, "bad argument");
    SurCam c;
    if (int32_t rc = make_surcam(p, s, &c)) return rc;
    const long n = n_pixels * c.n_bins;
    if (n == 0) return HADROS_OK;
    k_raw_features<<<int((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(c, pixel_ids, n_pixels, raw);
    return cuda_status("hadros_mlp_raw_features");
}

int32_t hadros_surrogate_image(const hadros_params* p, const hadros_sigma* s, int32_t n_members,
                               const float* masters, const void* images, const hadros_mlp_norm* norm,
                               int64_t pixel_begin, int64_t pixel_end, float spread_threshold,
                               int32_t spread_of, const hadros_surrogate_out* out, void* stream)
{
    if (!p || !s || !masters || !images || !norm || !out || !out->tau || !out->P_surv || !out->I_obs ||
        !out->spread || !out->fallback_ids || !out->counters)
        return set_error(HADROS_E_ARG, "NULL argument");
    if (n_members < 1 || n_members > kMaxMembers)
        return set_error(HADROS_E_ARG, "n_members must be in 1.." + std::to_string(kMaxMembers));
    if (reinterpret_cast<uintptr_t>(images) % 16 != 0) return set_error(HADROS_E_ARG, "images must be 16-byte aligned");
    if (spread_of != 0 && spread_of != 1) return set_error(HADROS_E_ARG, "spread_of must be 0 (ln I_obs) or 1 (ln tau)");
    InferArgs a{};
    if (int32_t rc = make_surcam(p, s, &a.cam, spread_of)) return rc;
    const long P = long(p->nx) * p->ny;
    if (pixel_begin < 0 || pixel_end > P || pixel_end < pixel_begin)
        return set_error(HADROS_E_ARG, "pixel range outside the image");
    if ((kPair * kTileRows) % a.cam.n_bins != 0)
        return set_error(HADROS_E_ARG, "surrogate inference needs a bin count that divides 256");
    int dev = 0, n_sm = 0, max_smem = 0, major = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) return set_error(HADROS_E_CUDA, "surrogate inference needs an sm_100 GPU");
    if (max_smem < kSmemBytes) return set_error(HADROS_E_CUDA, "not enough shared memory per block");
    auto st = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(out->counters, 0, 2 * sizeof(int32_t), st);
    const long n_px = pixel_end - pixel_begin;
    if (n_px == 0) return cuda_status("hadros_surrogate_image");
    static_assert(sizeof(hadros_mlp_norm) == sizeof(Norm), "hadros_mlp_norm must mirror mlp::Norm");
    std::memcpy(&a.norm, norm, sizeof(Norm));
    a.masters = masters;
    a.images = static_cast<const uint8_t*>(images);
    a.members = n_members;
    a.pixel_begin = pixel_begin;
    a.n_pixels = n_px;
    a.spread_threshold = spread_threshold;
    a.ln_tau_E = out->ln_tau_E;
    a.ln_I_E = out->ln_I_E;
    a.tau = out->tau;
    a.P_surv = out->P_surv;
    a.I_obs = out->I_obs;
    a.spread = out->spread;
    a.fallback_ids = out->fallback_ids;
    a.counters = out->counters;
    const long tiles = (n_px * a.cam.n_bins + kPair * kTileRows - 1) / (kPair * kTileRows);
    const int grid = int(std::min<long>(tiles, n_sm));
    if (g_schedule.load() == HADROS_SURROGATE_PINGPONG) {
        cudaFuncSetAttribute(k_infer<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        k_infer<true><<<grid, kThreads, kSmemBytes, st>>>(a);
    } else {
        cudaFuncSetAttribute(k_infer<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        k_infer<false><<<grid, kThreads, kSmemBytes, st>>>(a);
    }
    return cuda_status("hadros_surrogate_image");
}

}  // extern "C"
