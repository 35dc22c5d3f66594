// Cloud-in-cell charge deposition onto a Poisson mesh: the particle -> grid
// step that feeds a space-charge solve, next to the push.
//
// Reference: PyAMGPoissonSolver._bin_particles_cic_cpu and its kernel
// _cic_deposit_numba (src/PyPATools/poisson_amg.py:849-911).  The mesh has
// cells[d] nodes per axis, spaced h = extent / cells from -extent / 2
// (:178-185); rho is indexed [i][j][k], k fastest.  Per particle, in float64
// as there:
//   p = clip((x + extent/2) / h, 0, cells - 1)      (position in node units)
//   i = floor(p);  f = p - i;  i = clip(i, 0, cells - 2)
//   rho[corner] += q * wx * wy * wz  over the 8 corners, w = 1 - f or f
// and finally rho /= hx hy hz.  Because f is taken before i is clipped, a
// particle at p = cells - 1 (exactly on the last node, or clamped onto it from
// beyond) puts all its charge on the node before the last; that is kept.
//
// Float64 atomics into rho; for a cell-sorted bunch, warps keep running sums
// per cell (deposit_cic_kernel below).  The summation order differs from the
// reference's sequential loop, so results agree to rounding.
// A particle with a NaN coordinate deposits nothing (the reference's cast of
// NaN to an index is undefined).
#include <cmath>

#include "ppt_internal.cuh"

namespace ppt {

struct MeshGeom {
    double half[3];   // extent / 2
    double h[3];      // extent / cells
    int64_t n[3];     // nodes per axis (the reference's mesh_cells)
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One particle's position and charge (a particle past n reads nothing).
struct Loaded {
    double x[3];
    double q;
    bool in;
};

__device__ __forceinline__ Loaded load_particle(int64_t s, int64_t n, const double* __restrict__ r,
                                                const double* __restrict__ q) {
    Loaded L;
    L.in = s < n;
    if (L.in) {
#pragma unroll
        for (int a = 0; a < 3; ++a) L.x[a] = r[3 * s + a];
        L.q = q[s];
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) L.x[a] = 0.0;
        L.q = 0.0;
    }
    return L;
}

// One particle's cell (linear index of its lower corner) and corner charges;
// an invalid particle (past n, or a NaN position) gets cell -1 and no charge.
__device__ __forceinline__ int64_t particle_corners(const Loaded& L, const MeshGeom& G, const int64_t strides[3],
                                                    double w[8]) {
    bool valid = L.in;
    int64_t idx[3] = {0, 0, 0};
    double f[3] = {0.0, 0.0, 0.0};
    if (valid) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double p = (L.x[a] + G.half[a]) / G.h[a];
            valid = valid && !isnan(p);                        // a NaN position deposits nothing
            const double top = (double)(G.n[a] - 1);
            p = p < 0.0 ? 0.0 : (p > top ? top : p);          // np.clip
            p = isnan(p) ? 0.0 : p;
            double i = floor(p);
            f[a] = p - i;
            const double itop = (double)(G.n[a] - 2);
            i = i < 0.0 ? 0.0 : (i > itop ? itop : i);
            idx[a] = (int64_t)i;
        }
    }
    const double qs = valid ? L.q : 0.0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int di = (c >> 2) & 1, dj = (c >> 1) & 1, dk = c & 1;
        const double wx = di ? f[0] : 1.0 - f[0];
        const double wy = dj ? f[1] : 1.0 - f[1];
        const double wz = dk ? f[2] : 1.0 - f[2];
        w[c] = valid ? qs * (wx * wy * wz) : 0.0;
    }
    return valid ? idx[0] * strides[0] + idx[1] * strides[1] + idx[2] : -1;
}

__device__ __forceinline__ void add_corners(double* rho, int64_t base, const int64_t strides[3], const double w[8]) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int di = (c >> 2) & 1, dj = (c >> 1) & 1, dk = c & 1;
        atomicAdd(rho + base + di * strides[0] + dj * strides[1] + dk, w[c]);
    }
}

// Each warp takes kRounds rounds of 32 consecutive particles.  While all 32
// particles of a round are valid and in the same cell as the warp's running
// sums, each lane just adds its corner charges to its own running sums; when
// the cell changes (or at the end) the warp reduces them with shuffles and
// lane 0 issues 8 atomics.  A round whose particles are not all in one cell
// adds per lane.  A cell-sorted bunch thus costs 8 atomics per cell and warp
// instead of 8 per particle.  The next round's particle is loaded before the
// current one is processed, so its memory latency overlaps the arithmetic.
constexpr int kRounds = 8;

__global__ void __launch_bounds__(256) deposit_cic_kernel(int64_t n, const double* __restrict__ r,
                                                          const double* __restrict__ q, MeshGeom G,
                                                          double* __restrict__ rho) {
    const int64_t strides[3] = {G.n[1] * G.n[2], G.n[2], 1};
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t first = warp * (32 * kRounds);
    int64_t cur = -1;                 // cell of the running sums (warp-uniform), -1: none
    double acc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = 0.0;
    Loaded next = load_particle(first + lane, n, r, q);
    for (int round = 0; round < kRounds; ++round) {
        if (first + round * 32 >= n) break;          // warp-uniform
        const Loaded part = next;
        if (round + 1 < kRounds) next = load_particle(first + (round + 1) * 32 + lane, n, r, q);
        double w[8];
        const int64_t base = particle_corners(part, G, strides, w);
        const unsigned peers = __match_any_sync(0xffffffffu, (unsigned long long)base);
        const bool uniform = peers == 0xffffffffu && base >= 0;   // the same for every lane
        if (uniform && base == cur) {
#pragma unroll
            for (int c = 0; c < 8; ++c) acc[c] += w[c];
            continue;
        }
        if (cur >= 0) {                               // flush the running sums
#pragma unroll
            for (int c = 0; c < 8; ++c) acc[c] = warp_sum(acc[c]);
            if (lane == 0) add_corners(rho, cur, strides, acc);
            cur = -1;
        }
        if (uniform) {
            cur = base;
#pragma unroll
            for (int c = 0; c < 8; ++c) acc[c] = w[c];
        } else if (base >= 0) {
            add_corners(rho, base, strides, w);
        }
    }
    if (cur >= 0) {
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[c] = warp_sum(acc[c]);
        if (lane == 0) add_corners(rho, cur, strides, acc);
    }
}

__global__ void mesh_divide_kernel(int64_t m, double* __restrict__ rho, double volume) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        rho[i] = rho[i] / volume;
}

}  // namespace ppt

using namespace ppt;

extern "C" int ppt_deposit_cic(int64_t n, const double* r, const double* q, const ppt_mesh_desc* mesh, double* rho,
                               void* stream) {
    if (!mesh || !rho) return fail(PPT_ERR_ARG, "mesh and rho must not be NULL");
    if (n < 0) return fail(PPT_ERR_ARG, "n must be >= 0");
    if (n > 0 && (!r || !q)) return fail(PPT_ERR_ARG, "r and q must not be NULL");
    MeshGeom G;
    int64_t nodes = 1;
    for (int a = 0; a < 3; ++a) {
        if (mesh->cells[a] < 2) return fail(PPT_ERR_ARG, "every mesh axis needs at least 2 nodes");
        if (!(mesh->extent[a] > 0.0)) return fail(PPT_ERR_ARG, "mesh extents must be positive");
        G.n[a] = mesh->cells[a];
        G.half[a] = mesh->extent[a] / 2.0;
        G.h[a] = mesh->extent[a] / (double)mesh->cells[a];
        nodes *= mesh->cells[a];
        if (nodes > (1LL << 40)) return fail(PPT_ERR_ARG, "mesh too large");
    }
    const double volume = G.h[0] * G.h[1] * G.h[2];
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    PPT_CUDA_TRY(cudaMemsetAsync(rho, 0, (size_t)nodes * sizeof(double), s));
    if (n > 0) {
        const int block = 256;
        const int64_t per_block = (int64_t)block * kRounds;
        deposit_cic_kernel<<<(int)((n + per_block - 1) / per_block), block, 0, s>>>(n, r, q, G, rho);
        PPT_CUDA_TRY(cudaGetLastError());
    }
    const int block = 256;
    int64_t g = (nodes + block - 1) / block;
    mesh_divide_kernel<<<(int)(g > 148 * 16 ? 148 * 16 : g), block, 0, s>>>(nodes, rho, volume);
    PPT_CUDA_TRY(cudaGetLastError());
    return PPT_OK;
}
