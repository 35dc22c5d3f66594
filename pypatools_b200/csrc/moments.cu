// Bunch moments in float64 on the device: the ParticleDistribution
// statistics of the reference (src/PyPATools/particles.py:693-719 centroid
// and standard deviations, :761-788 emittances, :507-525 kinetic energy,
// :600-605 mean |p|), computed from (n,3) positions and velocities after the
// reference's per-component v -> beta*gamma -> v round trip
// (particles.py:71-117, :393-402, :440-457; relativistic settings).
//
// Two passes (means, then centred second moments), each a fixed-shape
// two-level reduction: every block reduces a grid-stride slice into a row of
// block partials in the scratch buffer, one block then sums the rows in a
// fixed order, so results are deterministic run to run.
#include <cmath>

#include "ppt_internal.cuh"

namespace ppt {

constexpr int kMomBlocks = 592;      // 4 x 148 SMs
constexpr int kMomThreads = 256;
constexpr int kNSum = 11;

struct MomDerived {
    double x[3];
    double xp[3];
    double p[3];
    double pabs;
    double ek;
};

// Per-particle derived quantities (reference conversions, float64).
__device__ __forceinline__ MomDerived derive(const double* r, const double* v, int64_t i, double mass_mev) {
    MomDerived d;
    double vv[3];
    for (int c = 0; c < 3; ++c) {
        d.x[c] = r[3 * i + c];
        const double vc = v[3 * i + c];
        double vsq = vc * vc;
        if (vsq >= kClight * kClight) vsq = 0.99999 * kClight * kClight;
        d.p[c] = vc / sqrt(kClight * kClight - vsq);                 // particles.py:94-103
        vv[c] = kClight * d.p[c] / sqrt(d.p[c] * d.p[c] + 1.0);       // particles.py:71-77
    }
    const double vz = fabs(vv[2]) < 1e-10 ? 1e-10 : vv[2];          // particles.py:462-467
    for (int c = 0; c < 3; ++c) d.xp[c] = vv[c] / vz;
    const double p2 = d.p[0] * d.p[0] + d.p[1] * d.p[1] + d.p[2] * d.p[2];
    d.pabs = sqrt(p2);
    // sqrt((p m)^2 + m^2) - m written without the cancellation: m p^2 / (1 + sqrt(1 + p^2))
    d.ek = mass_mev * p2 / (1.0 + sqrt(1.0 + p2));
    return d;
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    return t;
}

// pass 0: sums of x, xp, p, |p|, Ekin.  pass 1: centred second moments.
__global__ void __launch_bounds__(kMomThreads) moments_pass(int pass, int64_t n, const double* __restrict__ r,
                                                            const double* __restrict__ v, double mass_mev,
                                                            const double* __restrict__ mean,
                                                            double* __restrict__ partial) {
    __shared__ double sh[32];
    double acc[kNSum];
    for (int q = 0; q < kNSum; ++q) acc[q] = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        MomDerived d = derive(r, v, i, mass_mev);
        if (pass == 0) {
            for (int c = 0; c < 3; ++c) {
                acc[c] += d.x[c];
                acc[3 + c] += d.xp[c];
                acc[6 + c] += d.p[c];
            }
            acc[9] += d.pabs;
            acc[10] += d.ek;
        } else {
            double dx[3], dxp[3];
            for (int c = 0; c < 3; ++c) {
                dx[c] = d.x[c] - mean[c];
                dxp[c] = d.xp[c] - mean[3 + c];
                acc[c] += dx[c] * dx[c];
                acc[3 + c] += dxp[c] * dxp[c];
            }
            acc[6] += dx[0] * dxp[0];
            acc[7] += dx[1] * dxp[1];
            acc[8] += dx[0] * dxp[1];
            acc[9] += dx[1] * dxp[0];
            const double de = d.ek - mean[10];
            acc[10] += de * de;
        }
    }
    for (int q = 0; q < kNSum; ++q) {
        double t = block_sum(acc[q], sh);
        if (threadIdx.x == 0) partial[(int64_t)q * gridDim.x + blockIdx.x] = t;
    }
}

// One block: sum the partial rows in a fixed order and divide by n.
__global__ void moments_finish(int pass, int nblocks, int64_t n, const double* __restrict__ partial,
                               double* __restrict__ mean, double* __restrict__ out) {
    __shared__ double sh[32];
    for (int q = 0; q < kNSum; ++q) {
        double t = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) t += partial[(int64_t)q * nblocks + b];
        t = block_sum(t, sh);
        if (threadIdx.x == 0) {
            const double m = t / (double)n;
            if (pass == 0) {
                mean[q] = m;
            } else {
                // store the finished moments
                if (q < 3) out[3 + q] = sqrt(m);                 // x_std
                else if (q < 6) out[6 + (q - 3)] = sqrt(m);      // xp_std
                else if (q < 10) out[12 + (q - 6)] = m;          // xxp yyp xyp yxp
                else out[21] = sqrt(m);                          // Ekin std
            }
        }
    }
    __syncthreads();
    if (pass == 0 && threadIdx.x == 0) {
        for (int c = 0; c < 3; ++c) {
            out[c] = mean[c];            // centroid
            out[9 + c] = mean[3 + c];    // xp mean
            out[17 + c] = mean[6 + c];   // mean p
        }
        out[16] = mean[9];
        out[20] = mean[10];
    }
}

int64_t moments_scratch_doubles() { return (int64_t)kNSum * kMomBlocks + 16; }

int moments_launch(int64_t n, const double* r, const double* v, double mass_mev, double* out, double* scratch,
                   cudaStream_t s) {
    int nb = (int)((n + kMomThreads - 1) / kMomThreads);
    nb = nb < 1 ? 1 : (nb > kMomBlocks ? kMomBlocks : nb);
    double* partial = scratch;
    double* mean = scratch + (int64_t)kNSum * kMomBlocks;
    for (int pass = 0; pass < 2; ++pass) {
        moments_pass<<<nb, kMomThreads, 0, s>>>(pass, n, r, v, mass_mev, mean, partial);
        moments_finish<<<1, 256, 0, s>>>(pass, nb, n, partial, mean, out);
    }
    PPT_CUDA_TRY(cudaGetLastError());
    return PPT_OK;
}

}  // namespace ppt

using namespace ppt;

extern "C" int64_t ppt_moments_scratch_bytes(int64_t n) {
    (void)n;
    return moments_scratch_doubles() * (int64_t)sizeof(double);
}

extern "C" int ppt_moments(int64_t n, const double* r, const double* v, double mass_mev, double* out,
                           void* scratch, void* stream) {
    if (n <= 0) return fail(PPT_ERR_ARG, "moments need n >= 1");
    if (!r || !v || !out || !scratch) return fail(PPT_ERR_ARG, "r, v, out and scratch must not be NULL");
    return moments_launch(n, r, v, mass_mev, out, static_cast<double*>(scratch), static_cast<cudaStream_t>(stream));
}

// ---------------------------------------------------------------------------
// Moments without any device allocation by the library or the caller.
//
// For callers that must not allocate device memory while they run: a host
// application whose GPU memory is all handed to another allocator's pool, or
// an analysis hook inside a latency-bound tracking loop, where cudaMalloc /
// cudaFree (which can synchronise the device) are not allowed.  The scratch
// lives in a file-scope __device__ array instead; every GPU that loads this
// library holds it (52 KB) until the process exits.
// ---------------------------------------------------------------------------
#include <mutex>

#include <cudaTypedefs.h>   // CUcontext and the cuCtxGetCurrent signature (called through the runtime)

namespace ppt {

// 11 partial sums for each of up to kMomBlocks blocks, then 16 means.
constexpr int64_t kNoAllocScratchDoubles = (int64_t)kNSum * kMomBlocks + 16;
static __device__ __align__(256) double g_moments_scratch[kNoAllocScratchDoubles];

constexpr int kMaxDevices = 64;
static std::mutex g_scratch_mutex;
static double* g_scratch_addr[kMaxDevices] = {};
static CUcontext g_scratch_ctx[kMaxDevices] = {};

// The calling thread's current context (the runtime's entry-point query
// gives the driver function without linking the driver library).
static int current_context(CUcontext* ctx) {
    static PFN_cuCtxGetCurrent_v4000 get = nullptr;
    if (!get) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetDriverEntryPoint(cuCtxGetCurrent)");
        if (q != cudaDriverEntryPointSuccess || !fn) return fail(PPT_ERR_CUDA, "cuCtxGetCurrent is not available");
        get = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(fn);
    }
    if (get(ctx) != CUDA_SUCCESS) return fail(PPT_ERR_CUDA, "cuCtxGetCurrent failed");
    return PPT_OK;
}

// Device address of g_moments_scratch in the current device's context,
// looked up once per device and context (host code only has a host-side
// stand-in for the symbol).  The module, and with it the array, is loaded
// anew in a new context -- after cudaDeviceReset, or in a context the caller
// made current itself -- so the address is looked up again when the context
// differs from the one it was taken in.
static int noalloc_scratch(double** out) {
    int dev = 0;
    PPT_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(PPT_ERR_UNSUPPORTED, "device ordinal above 63");
    CUcontext ctx = nullptr;
    int rc = current_context(&ctx);
    if (rc) return rc;
    if (!ctx) {
        // no context current on this thread yet: the device's primary context
        // (cudaSetDevice initialises and binds it; it allocates nothing)
        PPT_CUDA_TRY(cudaSetDevice(dev));
        rc = current_context(&ctx);
        if (rc) return rc;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_moments_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(moments scratch)");
        g_scratch_addr[dev] = static_cast<double*>(p);
        g_scratch_ctx[dev] = ctx;
    }
    *out = g_scratch_addr[dev];
    return PPT_OK;
}

}  // namespace ppt

extern "C" int ppt_moments_noalloc(int64_t n, const double* r, const double* v, double mass_mev, double* out,
                                   void* stream) {
    if (n <= 0) return fail(PPT_ERR_ARG, "moments need n >= 1");
    if (n > (1LL << 53))
        return fail(PPT_ERR_ARG, "ppt_moments_noalloc handles at most 2^53 particles (the float64 count limit)");
    if (!r || !v || !out) return fail(PPT_ERR_ARG, "r, v and out must not be NULL");
    if (moments_scratch_doubles() > kNoAllocScratchDoubles)
        return fail(PPT_ERR_UNSUPPORTED, "moments scratch larger than the static array");
    double* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    // every partial row and mean the reduction reads is written earlier in the
    // same call, so nothing in the shared array needs clearing first
    return moments_launch(n, r, v, mass_mev, out, scratch, static_cast<cudaStream_t>(stream));
}
