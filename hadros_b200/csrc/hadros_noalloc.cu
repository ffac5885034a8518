// hadros_noalloc.cu — hadros_image_device_noalloc(): the trace kernel for
// callers that cannot allocate GPU memory.
//
// Who needs it: code that links this library into a process whose device
// memory is owned by someone else — a framework with its own caching
// allocator (a cudaMalloc/cudaFree behind its back fragments the pool and can
// synchronize the device), a service that reserves a fixed memory budget per
// tenant and forbids further allocation, or a host thread that must not block
// on the allocator.  Such callers already own their input and output buffers;
// what the ordinary entry points add on top is a context with device scratch
// (the work cursor and counters, the camera and bin tables, the sigma table).
// Here that scratch is one file-scope __device__ array instead.
//
// The array (kNoAllocScratchBytes, about 60 KB) is part of the library image:
// every GPU that loads the library holds it until the process exits.  Limits:
// at most 1024 sigma-table rows and 64 spectral bins per call; larger
// requests are rejected with HADROS_E_ARG before anything runs.  All calls
// share the one array and each leaves its contents behind; the work counters
// are cleared at the start of every call.  Two calls whose work overlaps on
// the GPU (different streams, or different host threads on one device) race
// on the array and corrupt each other's results: serialize them.
//
// Set-up: every call looks up the array's device address in the current
// context with cudaGetSymbolAddress (the array's name in host code is only a
// host-side stand-in, not a device address).  The first call on a device
// loads the library's module there; make that first call outside any stream
// capture.
//
// No cudaMalloc, cudaFree or other allocating routine is called: the plan is
// built in fixed-size local arrays and copied into the array with
// cudaMemcpyAsync; the only heap use is the text of an error message when a
// call fails.  The call waits on the caller's stream before returning, so it
// can report HADROS_E_TIMEOUT.
#include <cstring>
#include <limits>

#include "hadros_trace_kernel.cuh"

namespace hadros {
namespace {

constexpr int kNoAllocMaxSigma = 1024;
constexpr int kNoAllocMaxBins = 64;

constexpr size_t al256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffCounters = 0;
constexpr size_t kOffCam = 256;
constexpr size_t kOffBins = al256(kOffCam + sizeof(DevCam));
constexpr size_t kOffE = al256(kOffBins + sizeof(DevBin) * kNoAllocMaxBins);
constexpr size_t kOffS = al256(kOffE + 8 * kNoAllocMaxSigma);
constexpr size_t kOffLnE = al256(kOffS + 8 * kNoAllocMaxSigma);
constexpr size_t kOffLnS = al256(kOffLnE + 8 * kNoAllocMaxSigma);
constexpr size_t kOffLx = al256(kOffLnS + 8 * kNoAllocMaxSigma);
constexpr size_t kOffSeg = al256(kOffLx + 4 * kNoAllocMaxSigma);
constexpr size_t kNoAllocScratchBytes = al256(kOffSeg + 16 * kNoAllocMaxSigma);

// The scratch of every no-alloc call (see the file comment).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch in the current context, looked up on
// every call: cudaGetSymbolAddress allocates nothing, and a cached address
// would go stale when the caller resets the device or makes another context
// current (the library's module then loads at a different address).
int32_t scratch_address(unsigned char** out)
{
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return set_error(HADROS_E_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                                            cudaGetErrorString(e));
    *out = static_cast<unsigned char*>(p);
    return HADROS_OK;
}

}  // namespace
}  // namespace hadros

using namespace hadros;

extern "C" int32_t hadros_image_device_noalloc(const hadros_params* p, const hadros_sigma* s,
                                               const hadros_image_out* dev_out, void* stream)
{
    if (!p || !s || !dev_out) return set_error(HADROS_E_ARG, "NULL argument");
    int32_t rc = hadros_params_validate(p);
    if (rc) return rc;
    if (p->fast_geodesic)
        return set_error(HADROS_E_ARG, "the no-alloc entry point runs the reference-arithmetic kernel only "
                                       "(fast_geodesic must be 0)");
    const int n_sig = static_cast<int>(s->h.E.size());
    if (n_sig > kNoAllocMaxSigma)
        return set_error(HADROS_E_ARG, "sigma table has more rows than the no-alloc maximum of 1024");
    const int want_bins = p->spectral_kind == HADROS_SPECTRAL_MONOCHROMATIC ? 1 : std::max(p->n_bins, 1);
    if (want_bins > kNoAllocMaxBins)
        return set_error(HADROS_E_ARG, "n_bins exceeds the no-alloc maximum of 64 spectral bins");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(HADROS_E_CUDA, "no usable current CUDA device");
    int n_sm = 0;
    e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return set_error(HADROS_E_CUDA, cudaGetErrorString(e));

    DevCam cam;
    DevBin bins[kNoAllocMaxBins];
    int nb = 0;
    const char* perr = "";
    rc = build_cam_into(*p, s->h, cam, bins, kNoAllocMaxBins, &nb, &perr);
    if (rc) return set_error(rc, perr);
    const int64_t P = static_cast<int64_t>(p->nx) * p->ny;
    cam.item_begin = 0;
    cam.item_end = P;
    cam.out_offset = 0;
    cam.binout_offset = 0;

    unsigned char* base = nullptr;
    if ((rc = scratch_address(&base))) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const SigmaHost& h = s->h;
    struct Up { size_t off; const void* src; size_t n; } ups[] = {
        {kOffCam, &cam, sizeof(DevCam)}, {kOffBins, bins, sizeof(DevBin) * nb},
        {kOffE, h.E.data(), 8u * n_sig}, {kOffS, h.s_cm2.data(), 8u * n_sig},
        {kOffLnE, h.lnE.data(), 8u * n_sig}, {kOffLnS, h.lnS.data(), 8u * n_sig},
        {kOffLx, h.lx.data(), 4u * n_sig}, {kOffSeg, h.seg.data(), 16u * n_sig}};
    for (const Up& u : ups) {
        e = cudaMemcpyAsync(base + u.off, u.src, u.n, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return set_error(HADROS_E_CUDA, std::string("upload: ") + cudaGetErrorString(e));
    }
    e = cudaMemsetAsync(base + kOffCounters, 0, 4 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return set_error(HADROS_E_CUDA, std::string("counter reset: ") + cudaGetErrorString(e));

    TraceArgs A{};
    A.cams = reinterpret_cast<const DevCam*>(base + kOffCam);
    A.n_cams = 1;
    A.max_bins = nb;
    A.total_items = P;
    A.pixel_ids = nullptr;
    A.bins = reinterpret_cast<const DevBin*>(base + kOffBins);
    A.sig.n = n_sig;
    A.sig.E_min = h.E.front();
    A.sig.E_max = h.E.back();
    A.sig.sigma_scale = h.sigma_scale;
    A.sig.uniform = h.uniform;
    A.sig.lx0 = h.lx0;
    A.sig.inv_dlx = h.inv_dlx;
    A.sig.E = reinterpret_cast<const double*>(base + kOffE);
    A.sig.S = reinterpret_cast<const double*>(base + kOffS);
    A.sig.lnE = reinterpret_cast<const double*>(base + kOffLnE);
    A.sig.lnS = reinterpret_cast<const double*>(base + kOffLnS);
    A.sig.lx = reinterpret_cast<const float*>(base + kOffLx);
    A.sig.seg = reinterpret_cast<const float*>(base + kOffSeg);
    A.tau = dev_out->tau;
    A.P_surv = dev_out->P_surv;
    A.I_obs = dev_out->I_obs;
    A.fate = dev_out->fate;
    A.steps = dev_out->steps;
    A.attempts = dev_out->attempts;
    A.tau_E = dev_out->tau_E;
    A.I_E = static_cast<double*>(dev_out->I_E);
    A.tau_mev = dev_out->tau_mev;
    A.P_surv_mev = dev_out->P_surv_mev;
    A.I_obs_mev = dev_out->I_obs_mev;
    A.r_nu = dev_out->r_nu;
    A.leakage = dev_out->leakage;
    A.mev = p->mev_channel ? 1 : 0;
    A.counters = reinterpret_cast<unsigned long long*>(base + kOffCounters);
    A.attempt_budget = static_cast<int64_t>(p->max_steps) * 51 + 1;
    A.fast_geodesic = 0;
    if (P > 0) {
        std::string lerr;
        rc = launch_variant<0>(A, p->precision, n_sm, st, lerr);
        if (rc) return set_error(rc, lerr);
    }
    unsigned long long c[4] = {0, 0, 0, 0};
    e = cudaMemcpyAsync(c, base + kOffCounters, sizeof(c), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_error(HADROS_E_CUDA, std::string("trace kernel: ") + cudaGetErrorString(e));
    if (c[3] > 0) return set_error(HADROS_E_TIMEOUT, "rays exceeded the attempt budget");
    return set_error(HADROS_OK, "");
}
