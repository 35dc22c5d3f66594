// Space-charge potential and field on the Poisson solver's mesh.
//
// Reference: PyAMGPoissonSolver (src/PyPATools/poisson_amg.py).  Its mesh has
// n[a] cells of size h = extent / n centred at -extent/2 + (i + 1/2) h
// (:227-239); the operator is the 7-point Laplacian assembled at :293-443,
// which without conductor cells is, per axis, 2 / (h h) on the diagonal and
// -2 / (h (h + h)) for each neighbour inside the box (a neighbour beyond the
// box is a zero potential one cell away); the right-hand side is rho / eps0
// (:913-921).  The reference solves with GMRES preconditioned by an AMG
// V-cycle to a relative residual (1e-6 by default, :70); here the operator is
// applied matrix-free and the system, symmetric positive definite, is solved
// by conjugate gradients to the requested relative residual.  E = -grad phi by
// central differences at the cells whose three indices are all interior,
// zero on the outer layer (compute_field_from_potential_numba, :98-130).
//
// Every reduction sums per-block partials in a fixed order (no atomics), and
// the iteration stops on the device at the first iterate meeting the
// tolerance: a solve gives the same bits however its launches are batched.
#include <cmath>

#include "ppt_internal.cuh"

namespace ppt {

struct PoissonOp {
    int64_t n[3];
    double off[3];   // the neighbour coefficients, -2 / (h (h + h)) per axis
    double diag;     // 2/(hx hx) + 2/(hy hy) + 2/(hz hz), summed in that order from 0
};

// Scalars the kernels share, in device memory.
enum { kRR = 0, kALPHA, kBETA, kDONE, kITERS, kTOL2, kBB, kNumScalars };

constexpr int kBlock = 256;

__device__ __forceinline__ double apply_op(const PoissonOp& A, const double* __restrict__ x, int64_t c, int64_t i,
                                           int64_t j, int64_t k) {
    const int64_t sy = A.n[2], sx = A.n[1] * A.n[2];
    double s = A.diag * x[c];
    // x, y, z neighbours as the reference's rows list them
    if (i + 1 < A.n[0]) s += A.off[0] * x[c + sx];
    if (i > 0) s += A.off[0] * x[c - sx];
    if (j + 1 < A.n[1]) s += A.off[1] * x[c + sy];
    if (j > 0) s += A.off[1] * x[c - sy];
    if (k + 1 < A.n[2]) s += A.off[2] * x[c + 1];
    if (k > 0) s += A.off[2] * x[c - 1];
    return s;
}

// Block sum of v into partial[blockIdx.x] (fixed shuffle / shared order).
__device__ __forceinline__ void block_partial(double v, double* partial) {
    __shared__ double warp_sums[kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) s += warp_sums[w];
        partial[blockIdx.x] = s;
    }
}

__device__ __forceinline__ void cell_ijk(const PoissonOp& A, int64_t c, int64_t& i, int64_t& j, int64_t& k) {
    k = c % A.n[2];
    const int64_t t = c / A.n[2];
    j = t % A.n[1];
    i = t / A.n[1];
}

// r = b - A x, p = r; partial sums of r.r and b.b
__global__ void __launch_bounds__(kBlock) cg_start(const __grid_constant__ PoissonOp A, int64_t m,
                                                   const double* __restrict__ b, const double* __restrict__ x,
                                                   double* __restrict__ r, double* __restrict__ p,
                                                   double* __restrict__ part_rr, double* __restrict__ part_bb) {
    const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
    double rr = 0.0, bb = 0.0;
    if (c < m) {
        int64_t i, j, k;
        cell_ijk(A, c, i, j, k);
        const double rc = b[c] - apply_op(A, x, c, i, j, k);
        r[c] = rc;
        p[c] = rc;
        rr = rc * rc;
        bb = b[c] * b[c];
    }
    block_partial(rr, part_rr);
    __syncthreads();
    block_partial(bb, part_bb);
}

// q = A p; partial sums of p.q
__global__ void __launch_bounds__(kBlock) cg_apply(const __grid_constant__ PoissonOp A, int64_t m,
                                                   const double* __restrict__ p, double* __restrict__ q,
                                                   double* __restrict__ part, const double* __restrict__ S) {
    if (S[kDONE] != 0.0) return;
    const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
    double s = 0.0;
    if (c < m) {
        int64_t i, j, k;
        cell_ijk(A, c, i, j, k);
        const double qc = apply_op(A, p, c, i, j, k);
        q[c] = qc;
        s = p[c] * qc;
    }
    block_partial(s, part);
}

// x += alpha p, r -= alpha q; partial sums of r.r
__global__ void __launch_bounds__(kBlock) cg_step(int64_t m, double* __restrict__ x, double* __restrict__ r,
                                                  const double* __restrict__ p, const double* __restrict__ q,
                                                  double* __restrict__ part, const double* __restrict__ S) {
    if (S[kDONE] != 0.0) return;
    const double alpha = S[kALPHA];
    const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
    double s = 0.0;
    if (c < m) {
        x[c] += alpha * p[c];
        const double rc = r[c] - alpha * q[c];
        r[c] = rc;
        s = rc * rc;
    }
    block_partial(s, part);
}

// p = r + beta p
__global__ void __launch_bounds__(kBlock) cg_direction(int64_t m, const double* __restrict__ r, double* __restrict__ p,
                                                       const double* __restrict__ S) {
    if (S[kDONE] != 0.0) return;
    const double beta = S[kBETA];
    const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
    if (c < m) p[c] = r[c] + beta * p[c];
}

__device__ double sum_partials(const double* part, int nb) {
    __shared__ double s[kBlock];
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += kBlock) v += part[b];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int w = kBlock / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    return s[0];
}

// One block.  mode 0: start (rr, bb -> tolerance); 1: alpha = rr / p.q;
// 2: rr' and beta = rr' / rr, stop once rr' <= tol^2 bb or rr' = 0.
__global__ void __launch_bounds__(kBlock) cg_scalars(int mode, const double* __restrict__ part,
                                                     const double* __restrict__ part2, int nb, double* S,
                                                     double rel_tol, int64_t max_iter) {
    if (mode != 0 && S[kDONE] != 0.0) return;
    const double v = sum_partials(part, nb);
    __syncthreads();
    if (mode == 0) {
        const double bb = sum_partials(part2, nb);
        if (threadIdx.x == 0) {
            S[kRR] = v;
            S[kBB] = bb;
            S[kTOL2] = rel_tol * rel_tol * bb;
            S[kITERS] = 0.0;
            S[kDONE] = (v <= S[kTOL2] || v == 0.0 || max_iter <= 0) ? 1.0 : 0.0;
        }
        return;
    }
    if (threadIdx.x != 0) return;
    if (mode == 1) {
        S[kALPHA] = S[kRR] / v;
    } else {
        S[kBETA] = v / S[kRR];
        S[kRR] = v;
        S[kITERS] += 1.0;
        if (v <= S[kTOL2] || v == 0.0 || S[kITERS] >= (double)max_iter) S[kDONE] = 1.0;
    }
}

__global__ void __launch_bounds__(kBlock) field_from_potential(int64_t nx, int64_t ny, int64_t nz,
                                                               const double* __restrict__ phi, double hx, double hy,
                                                               double hz, double* __restrict__ ex,
                                                               double* __restrict__ ey, double* __restrict__ ez) {
    const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
    if (c >= nx * ny * nz) return;
    const int64_t k = c % nz, t = c / nz, j = t % ny, i = t / ny;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1) {
        const int64_t sy = nz, sx = ny * nz;
        fx = -(phi[c + sx] - phi[c - sx]) / (2 * hx);
        fy = -(phi[c + sy] - phi[c - sy]) / (2 * hy);
        fz = -(phi[c + 1] - phi[c - 1]) / (2 * hz);
    }
    if (ex) ex[c] = fx;
    if (ey) ey[c] = fy;
    if (ez) ez[c] = fz;
}

// ---------------------------------------------------------------------------
// Operator with per-cell coefficients (conductor cells, Shortley-Weller rows):
// coef[7 c .. 7 c + 6] = diagonal, +x, -x, +y, -y, +z, -z couplings (0 for a
// neighbour outside the box or in a conductor; a conductor cell's row is the
// identity).  Not symmetric in general: BiCGSTAB (H. A. van der Vorst, SIAM J.
// Sci. Stat. Comput. 13(2), 1992).
// ---------------------------------------------------------------------------
struct CoefOp {
    int64_t n[3];
    const double* coef;
};

enum { bRR = 0, bBB, bTOL2, bRHO, bALPHA, bOMEGA, bBETA, bDONE, bITERS, bNumScalars };

__device__ __forceinline__ double apply_coef(const CoefOp& A, const double* __restrict__ x, int64_t c) {
    const int64_t nz = A.n[2], sy = nz, sx = A.n[1] * nz;
    const int64_t k = c % nz, t = c / nz, j = t % A.n[1], i = t / A.n[1];
    const double* w = A.coef + 7 * c;
    double s = w[0] * x[c];
    if (i + 1 < A.n[0]) s += w[1] * x[c + sx];
    if (i > 0) s += w[2] * x[c - sx];
    if (j + 1 < A.n[1]) s += w[3] * x[c + sy];
    if (j > 0) s += w[4] * x[c - sy];
    if (k + 1 < A.n[2]) s += w[5] * x[c + 1];
    if (k > 0) s += w[6] * x[c - 1];
    return s;
}

// r = b - A x, rhat = r, p = v = 0; partial sums of r.r and b.b
__global__ void __launch_bounds__(kBlock) bi_start(const __grid_constant__ CoefOp A, int64_t m,
                                                   const double* __restrict__ b, const double* __restrict__ x,
                                                   double* __restrict__ r, double* __restrict__ rhat,
                                                   double* __restrict__ p, double* __restrict__ v,
                                                   double* __restrict__ part, double* __restrict__ part2) {
    const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
    double rr = 0.0, bb = 0.0;
    if (c < m) {
        const double rc = b[c] - apply_coef(A, x, c);
        r[c] = rc;
        rhat[c] = rc;
        p[c] = 0.0;
        v[c] = 0.0;
        rr = rc * rc;
        bb = b[c] * b[c];
    }
    block_partial(rr, part);
    __syncthreads();
    block_partial(bb, part2);
}

// p = r + beta (p - omega v)
__global__ void __launch_bounds__(kBlock) bi_direction(int64_t m, const double* __restrict__ r, double* __restrict__ p,
                                                       const double* __restrict__ v, const double* __restrict__ S) {
    if (S[bDONE] != 0.0) return;
    const double beta = S[bBETA], omega = S[bOMEGA];
    const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
    if (c < m) p[c] = r[c] + beta * (p[c] - omega * v[c]);
}

// y = A z; partial sums of a.y (and of y.y when part2 is set)
__global__ void __launch_bounds__(kBlock) bi_apply(const __grid_constant__ CoefOp A, int64_t m,
                                                   const double* __restrict__ z, double* __restrict__ y,
                                                   const double* __restrict__ a, double* __restrict__ part,
                                                   double* __restrict__ part2, const double* __restrict__ S) {
    if (S[bDONE] != 0.0) return;
    const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
    double d1 = 0.0, d2 = 0.0;
    if (c < m) {
        const double yc = apply_coef(A, z, c);
        y[c] = yc;
        d1 = a[c] * yc;
        d2 = yc * yc;
    }
    block_partial(d1, part);
    if (part2) {
        __syncthreads();
        block_partial(d2, part2);
    }
}

// s = r - alpha v
__global__ void __launch_bounds__(kBlock) bi_half(int64_t m, const double* __restrict__ r, const double* __restrict__ v,
                                                  double* __restrict__ sv, const double* __restrict__ S) {
    if (S[bDONE] != 0.0) return;
    const double alpha = S[bALPHA];
    const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
    if (c < m) sv[c] = r[c] - alpha * v[c];
}

// x += alpha p + omega s, r = s - omega t; partial sums of rhat.r and r.r
__global__ void __launch_bounds__(kBlock) bi_update(int64_t m, double* __restrict__ x, double* __restrict__ r,
                                                    const double* __restrict__ rhat, const double* __restrict__ p,
                                                    const double* __restrict__ sv, const double* __restrict__ t,
                                                    double* __restrict__ part, double* __restrict__ part2,
                                                    const double* __restrict__ S) {
    if (S[bDONE] != 0.0) return;
    const double alpha = S[bALPHA], omega = S[bOMEGA];
    const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
    double d1 = 0.0, d2 = 0.0;
    if (c < m) {
        x[c] += alpha * p[c] + omega * sv[c];
        const double rc = sv[c] - omega * t[c];
        r[c] = rc;
        d1 = rhat[c] * rc;
        d2 = rc * rc;
    }
    block_partial(d1, part);
    __syncthreads();
    block_partial(d2, part2);
}

// One block.  mode 0: start; 1: alpha = rho / rhat.v; 2: omega = t.s / t.t;
// 3: rho', beta, residual and the stopping test.
__global__ void __launch_bounds__(kBlock) bi_scalars(int mode, const double* __restrict__ part,
                                                     const double* __restrict__ part2, int nb, double* S,
                                                     double rel_tol, int64_t max_iter) {
    if (mode != 0 && S[bDONE] != 0.0) return;
    const double a = sum_partials(part, nb);
    __syncthreads();
    const double b = part2 ? sum_partials(part2, nb) : 0.0;
    if (threadIdx.x != 0) return;
    if (mode == 0) {
        S[bRR] = a;
        S[bBB] = b;
        S[bTOL2] = rel_tol * rel_tol * b;
        S[bRHO] = a;          // rhat = r
        S[bALPHA] = 1.0;
        S[bOMEGA] = 1.0;
        S[bBETA] = 0.0;       // first direction p = r
        S[bITERS] = 0.0;
        S[bDONE] = (a <= S[bTOL2] || a == 0.0 || max_iter <= 0) ? 1.0 : 0.0;
    } else if (mode == 1) {
        S[bALPHA] = a != 0.0 ? S[bRHO] / a : 0.0;
        if (a == 0.0) S[bDONE] = 1.0;                       // breakdown
    } else if (mode == 2) {
        S[bOMEGA] = b > 0.0 ? a / b : 0.0;                  // a = t.s, b = t.t
    } else {
        S[bITERS] += 1.0;
        S[bRR] = b;
        const double rho = a;
        S[bBETA] = (S[bRHO] != 0.0 && S[bOMEGA] != 0.0) ? (rho / S[bRHO]) * (S[bALPHA] / S[bOMEGA]) : 0.0;
        S[bRHO] = rho;
        if (b <= S[bTOL2] || b == 0.0 || S[bITERS] >= (double)max_iter || rho == 0.0 || S[bOMEGA] == 0.0)
            S[bDONE] = 1.0;
    }
}

// Iterations of a solve: kIterPerGraph of them captured once as a CUDA graph
// on a private stream (the caller's may be the legacy default stream, which
// cannot be captured) and replayed until the device-side stop flag is set;
// one host check per replay.  The kernels and their order are those of plain
// launches, so the results are the same bits, with a fraction of the launch
// cost (a solve is thousands of short launches on L2-resident vectors).
constexpr int kIterPerGraph = 16;

template <typename Enqueue>
static int run_iterations(cudaStream_t caller, const double* S, int done_slot, int n_scalars, int64_t max_iter,
                          double* host, Enqueue enqueue_iteration) {
    cudaStream_t side = nullptr;
    cudaEvent_t ready = nullptr, finished = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&finished, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ready, caller);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(side, ready, 0);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(side, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        for (int it = 0; it < kIterPerGraph; ++it) enqueue_iteration(side);
        e = cudaStreamEndCapture(side, &graph);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    for (int64_t done = 0; e == cudaSuccess;) {
        e = cudaGraphLaunch(exec, side);
        if (e == cudaSuccess) e = cudaMemcpyAsync(host, S, n_scalars * sizeof(double), cudaMemcpyDeviceToHost, side);
        if (e == cudaSuccess) e = cudaStreamSynchronize(side);
        done += kIterPerGraph;
        if (e != cudaSuccess || host[done_slot] != 0.0 || done >= max_iter) break;
    }
    // the caller's stream continues after the solve
    if (e == cudaSuccess) e = cudaEventRecord(finished, side);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(caller, finished, 0);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (ready) cudaEventDestroy(ready);
    if (finished) cudaEventDestroy(finished);
    if (side) cudaStreamDestroy(side);
    if (e != cudaSuccess) return cuda_fail(e, "solver iterations");
    return PPT_OK;
}

static int mesh_geom(const ppt_mesh_desc* mesh, int64_t n[3], double h[3]) {
    if (!mesh) return fail(PPT_ERR_ARG, "mesh must not be NULL");
    int64_t total = 1;
    for (int a = 0; a < 3; ++a) {
        if (mesh->cells[a] < 1) return fail(PPT_ERR_ARG, "every mesh axis needs at least 1 cell");
        if (!(mesh->extent[a] > 0.0)) return fail(PPT_ERR_ARG, "mesh extents must be positive");
        n[a] = mesh->cells[a];
        h[a] = mesh->extent[a] / (double)mesh->cells[a];
        total *= n[a];
        if (total > (1LL << 34)) return fail(PPT_ERR_ARG, "mesh too large");
    }
    return PPT_OK;
}

}  // namespace ppt

using namespace ppt;

extern "C" int64_t ppt_poisson_scratch_bytes(const ppt_mesh_desc* mesh) {
    int64_t n[3];
    double h[3];
    if (mesh_geom(mesh, n, h)) return -1;
    const int64_t m = n[0] * n[1] * n[2];
    const int64_t nb = (m + kBlock - 1) / kBlock;
    return (3 * m + 2 * nb + kNumScalars) * (int64_t)sizeof(double);
}

extern "C" int ppt_poisson_solve(const ppt_mesh_desc* mesh, const double* rhs, double* phi, void* scratch,
                                 double rel_tol, int64_t max_iter, int64_t* iterations, double* rel_residual,
                                 void* stream) {
    int64_t n[3];
    double h[3];
    int rc = mesh_geom(mesh, n, h);
    if (rc) return rc;
    if (!rhs || !phi || !scratch) return fail(PPT_ERR_ARG, "rhs, phi and scratch must not be NULL");
    if (!(rel_tol >= 0.0)) return fail(PPT_ERR_ARG, "rel_tol must be >= 0");
    PoissonOp A;
    A.diag = 0.0;
    for (int a = 0; a < 3; ++a) {
        A.n[a] = n[a];
        A.off[a] = -2.0 / (h[a] * (h[a] + h[a]));
        A.diag += 2.0 / (h[a] * h[a]);
    }
    const int64_t m = n[0] * n[1] * n[2];
    const int nb = (int)((m + kBlock - 1) / kBlock);
    double* r = static_cast<double*>(scratch);
    double* p = r + m;
    double* q = p + m;
    double* part = q + m;
    double* part2 = part + nb;
    double* S = part2 + nb;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cg_start<<<nb, kBlock, 0, s>>>(A, m, rhs, phi, r, p, part, part2);
    cg_scalars<<<1, kBlock, 0, s>>>(0, part, part2, nb, S, rel_tol, max_iter);
    PPT_CUDA_TRY(cudaGetLastError());
    // Graph replays of kIterPerGraph iterations between host checks; a
    // finished solve turns the remaining launches of a replay into no-ops.
    double host[kNumScalars];
    rc = run_iterations(s, S, kDONE, kNumScalars, max_iter, host, [&](cudaStream_t st) {
        cg_apply<<<nb, kBlock, 0, st>>>(A, m, p, q, part, S);
        cg_scalars<<<1, kBlock, 0, st>>>(1, part, nullptr, nb, S, rel_tol, max_iter);
        cg_step<<<nb, kBlock, 0, st>>>(m, phi, r, p, q, part, S);
        cg_scalars<<<1, kBlock, 0, st>>>(2, part, nullptr, nb, S, rel_tol, max_iter);
        cg_direction<<<nb, kBlock, 0, st>>>(m, r, p, S);
    });
    if (rc) return rc;
    if (iterations) *iterations = (int64_t)host[kITERS];
    if (rel_residual) *rel_residual = host[kBB] > 0.0 ? std::sqrt(host[kRR] / host[kBB]) : 0.0;
    return PPT_OK;
}

extern "C" int ppt_field_from_potential(const ppt_mesh_desc* mesh, const double* phi, double* ex, double* ey,
                                        double* ez, void* stream) {
    int64_t n[3];
    double h[3];
    int rc = mesh_geom(mesh, n, h);
    if (rc) return rc;
    if (!phi) return fail(PPT_ERR_ARG, "phi must not be NULL");
    const int64_t m = n[0] * n[1] * n[2];
    field_from_potential<<<(unsigned)((m + kBlock - 1) / kBlock), kBlock, 0, static_cast<cudaStream_t>(stream)>>>(
        n[0], n[1], n[2], phi, h[0], h[1], h[2], ex, ey, ez);
    PPT_CUDA_TRY(cudaGetLastError());
    return PPT_OK;
}

extern "C" int64_t ppt_poisson_coef_scratch_bytes(const ppt_mesh_desc* mesh) {
    int64_t n[3];
    double h[3];
    if (mesh_geom(mesh, n, h)) return -1;
    const int64_t m = n[0] * n[1] * n[2];
    const int64_t nb = (m + kBlock - 1) / kBlock;
    return (6 * m + 2 * nb + bNumScalars) * (int64_t)sizeof(double);
}

extern "C" int ppt_poisson_solve_coef(const ppt_mesh_desc* mesh, const double* coef, const double* rhs, double* phi,
                                      void* scratch, double rel_tol, int64_t max_iter, int64_t* iterations,
                                      double* rel_residual, void* stream) {
    int64_t n[3];
    double h[3];
    int rc = mesh_geom(mesh, n, h);
    if (rc) return rc;
    if (!coef || !rhs || !phi || !scratch) return fail(PPT_ERR_ARG, "coef, rhs, phi and scratch must not be NULL");
    if (!(rel_tol >= 0.0)) return fail(PPT_ERR_ARG, "rel_tol must be >= 0");
    CoefOp A;
    for (int a = 0; a < 3; ++a) A.n[a] = n[a];
    A.coef = coef;
    const int64_t m = n[0] * n[1] * n[2];
    const int nb = (int)((m + kBlock - 1) / kBlock);
    double* r = static_cast<double*>(scratch);
    double* rhat = r + m;
    double* p = rhat + m;
    double* v = p + m;
    double* sv = v + m;
    double* t = sv + m;
    double* part = t + m;
    double* part2 = part + nb;
    double* S = part2 + nb;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    bi_start<<<nb, kBlock, 0, st>>>(A, m, rhs, phi, r, rhat, p, v, part, part2);
    bi_scalars<<<1, kBlock, 0, st>>>(0, part, part2, nb, S, rel_tol, max_iter);
    PPT_CUDA_TRY(cudaGetLastError());
    double host[bNumScalars];
    rc = run_iterations(st, S, bDONE, bNumScalars, max_iter, host, [&](cudaStream_t ss) {
        bi_direction<<<nb, kBlock, 0, ss>>>(m, r, p, v, S);
        bi_apply<<<nb, kBlock, 0, ss>>>(A, m, p, v, rhat, part, nullptr, S);
        bi_scalars<<<1, kBlock, 0, ss>>>(1, part, nullptr, nb, S, rel_tol, max_iter);
        bi_half<<<nb, kBlock, 0, ss>>>(m, r, v, sv, S);
        bi_apply<<<nb, kBlock, 0, ss>>>(A, m, sv, t, sv, part, part2, S);
        bi_scalars<<<1, kBlock, 0, ss>>>(2, part, part2, nb, S, rel_tol, max_iter);
        bi_update<<<nb, kBlock, 0, ss>>>(m, phi, r, rhat, p, sv, t, part, part2, S);
        bi_scalars<<<1, kBlock, 0, ss>>>(3, part, part2, nb, S, rel_tol, max_iter);
    });
    if (rc) return rc;
    if (iterations) *iterations = (int64_t)host[bITERS];
    if (rel_residual) *rel_residual = host[bBB] > 0.0 ? std::sqrt(host[bRR] / host[bBB]) : 0.0;
    return PPT_OK;
}
