// Electrode surfaces: upload of a triangle mesh with its cell grid, and the
// standalone segment test (the call the reference makes each step,
// PyElectrodeAssembly.segment_intersects_surface, src/PyPATools/pusher.py:984).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "surface.cuh"

namespace ppt {

__global__ void segments_hit_kernel(const __grid_constant__ SurfaceDev S, int64_t n, const double* __restrict__ p0,
                                    const double* __restrict__ p1, uint8_t* __restrict__ hit) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3 a = v3(p0[3 * i], p0[3 * i + 1], p0[3 * i + 2]);
    const V3 b = v3(p1[3 * i], p1[3 * i + 1], p1[3 * i + 2]);
    hit[i] = segment_hits_surface(S, a, b) ? 1 : 0;
}

// Cell grid over the mesh's bounding box: about two cells per triangle, cells
// as close to cubes as the box allows, at most 256 per axis.
static void grid_for_mesh(const double lo_in[3], const double hi_in[3], int64_t n_tri, double lo[3],
                          double h[3], int dims[3]) {
    double ext[3], big = 0.0;
    for (int a = 0; a < 3; ++a) big = std::max(big, hi_in[a] - lo_in[a]);
    const double pad = std::max(big * 1e-9, 1e-30);
    double vol = 1.0;
    for (int a = 0; a < 3; ++a) {
        lo[a] = lo_in[a] - pad;
        ext[a] = (hi_in[a] + pad) - lo[a];
        vol *= ext[a];
    }
    const double target = std::max<double>(1.0, 2.0 * (double)n_tri);
    const double side = std::cbrt(vol / target);
    for (int a = 0; a < 3; ++a) {
        double d = std::ceil(ext[a] / side);
        d = d < 1.0 ? 1.0 : (d > 256.0 ? 256.0 : d);
        dims[a] = (int)d;
        h[a] = ext[a] / (double)dims[a];
    }
}

}  // namespace ppt

using namespace ppt;

extern "C" int ppt_surface_create(int64_t n_vertices, const double* vertices, int64_t n_triangles,
                                  const int64_t* triangles, ppt_surface** out) {
    if (!out) return fail(PPT_ERR_ARG, "out must not be NULL");
    *out = nullptr;
    if (n_vertices < 3 || n_triangles < 1) return fail(PPT_ERR_ARG, "a surface needs >= 3 vertices and >= 1 triangle");
    if (!vertices || !triangles) return fail(PPT_ERR_ARG, "vertices and triangles must not be NULL");
    if (n_triangles > (1LL << 30)) return fail(PPT_ERR_ARG, "too many triangles");
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    std::vector<double> tri((size_t)n_triangles * 9);
    for (int64_t t = 0; t < n_triangles; ++t) {
        const double* v[3];
        for (int c = 0; c < 3; ++c) {
            const int64_t idx = triangles[3 * t + c];
            if (idx < 0 || idx >= n_vertices) return fail(PPT_ERR_ARG, "triangle vertex index out of range");
            v[c] = vertices + 3 * idx;
        }
        for (int a = 0; a < 3; ++a) {
            for (int c = 0; c < 3; ++c) {
                if (!std::isfinite(v[c][a])) return fail(PPT_ERR_ARG, "vertex coordinates must be finite");
                lo[a] = std::min(lo[a], v[c][a]);
                hi[a] = std::max(hi[a], v[c][a]);
            }
            tri[9 * t + a] = v[0][a];
            tri[9 * t + 3 + a] = v[1][a] - v[0][a];
            tri[9 * t + 6 + a] = v[2][a] - v[0][a];
        }
    }
    ppt_surface S;
    std::memset(&S, 0, sizeof(S));
    double h[3];
    grid_for_mesh(lo, hi, n_triangles, S.dev.lo, h, S.dev.dims);
    for (int a = 0; a < 3; ++a) S.dev.inv_h[a] = 1.0 / h[a];
    const int64_t cells = (int64_t)S.dev.dims[0] * S.dev.dims[1] * S.dev.dims[2];
    // bin each triangle into the cells its bounding box overlaps (count, then fill).
    // The box is padded by 1e-7 of a cell: the segment and ray tests work on
    // v0, e1 = v1 - v0, e2 = v2 - v0 rounded, whose hits can lie an ulp or so
    // outside the vertices' box; a triangle within the pad of a cell face is
    // listed on both sides of it, so no such hit falls in a cell that does not
    // list the triangle (the tests stay the same as testing every triangle).
    auto cell_range = [&](int64_t t, int a, int* c0, int* c1) {
        double mn = INFINITY, mx = -INFINITY;
        for (int c = 0; c < 3; ++c) {
            const double x = vertices[3 * triangles[3 * t + c] + a];
            mn = std::min(mn, x);
            mx = std::max(mx, x);
        }
        const double pad = 1e-7 / S.dev.inv_h[a];
        const double u0 = (mn - pad - S.dev.lo[a]) * S.dev.inv_h[a], u1 = (mx + pad - S.dev.lo[a]) * S.dev.inv_h[a];
        *c0 = std::min(std::max((int)std::floor(u0), 0), S.dev.dims[a] - 1);
        *c1 = std::min(std::max((int)std::floor(u1), 0), S.dev.dims[a] - 1);
    };
    std::vector<int64_t> count(cells + 1, 0);
    std::vector<int32_t> trange((size_t)n_triangles * 6);
    for (int64_t t = 0; t < n_triangles; ++t) {
        int r0[3], r1[3];
        for (int a = 0; a < 3; ++a) {
            cell_range(t, a, &r0[a], &r1[a]);
            trange[6 * t + 2 * a] = r0[a];
            trange[6 * t + 2 * a + 1] = r1[a];
        }
        for (int i = r0[0]; i <= r1[0]; ++i)
            for (int j = r0[1]; j <= r1[1]; ++j)
                for (int k = r0[2]; k <= r1[2]; ++k) ++count[(i * (int64_t)S.dev.dims[1] + j) * S.dev.dims[2] + k + 1];
    }
    for (int64_t c = 0; c < cells; ++c) count[c + 1] += count[c];
    if (count[cells] > 0x7fffffffLL) return fail(PPT_ERR_UNSUPPORTED, "surface cell lists exceed 2^31 entries");
    std::vector<int32_t> start(count.begin(), count.end());
    std::vector<int32_t> list((size_t)count[cells]);
    std::vector<int32_t> fill(start.begin(), start.end() - 1);
    for (int64_t t = 0; t < n_triangles; ++t) {
        int r0[3], r1[3];
        for (int a = 0; a < 3; ++a) cell_range(t, a, &r0[a], &r1[a]);
        for (int i = r0[0]; i <= r1[0]; ++i)
            for (int j = r0[1]; j <= r1[1]; ++j)
                for (int k = r0[2]; k <= r1[2]; ++k)
                    list[fill[(i * (int64_t)S.dev.dims[1] + j) * S.dev.dims[2] + k]++] = (int32_t)t;
    }
    const size_t b_tri = tri.size() * sizeof(double);
    const size_t b_start = start.size() * sizeof(int32_t);
    const size_t b_list = std::max<size_t>(list.size(), 1) * sizeof(int32_t);
    const size_t b_range = trange.size() * sizeof(int32_t);
    S.bytes = b_tri + b_start + b_list + b_range;
    PPT_CUDA_TRY(cudaGetDevice(&S.device));
    cudaError_t e = cudaMalloc(&S.buf, S.bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(PPT_ERR_OOM, "cudaMalloc of the surface failed");
    }
    char* base = static_cast<char*>(S.buf);
    e = cudaMemcpy(base, tri.data(), b_tri, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(base + b_tri, start.data(), b_start, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !list.empty())
        e = cudaMemcpy(base + b_tri + b_start, list.data(), list.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(base + b_tri + b_start + b_list, trange.data(), b_range, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(S.buf);
        return cuda_fail(e, "surface upload");
    }
    S.dev.tri = reinterpret_cast<const double*>(base);
    S.dev.cell_start = reinterpret_cast<const int32_t*>(base + b_tri);
    S.dev.cell_tri = reinterpret_cast<const int32_t*>(base + b_tri + b_start);
    S.dev.trange = reinterpret_cast<const int32_t*>(base + b_tri + b_start + b_list);
    S.dev.n_tri = (int32_t)n_triangles;
    *out = new ppt_surface(S);
    return PPT_OK;
}

__global__ void axis_rays_kernel(const __grid_constant__ SurfaceDev S, int64_t n, const double* __restrict__ pts,
                                 double* __restrict__ dist, int32_t* __restrict__ hits) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n * 6) return;
    const int64_t row = i / 6;
    const int dir = (int)(i - row * 6);
    int c;
    double d;
    axis_ray_hits(S, v3(pts[3 * row], pts[3 * row + 1], pts[3 * row + 2]), dir, c, d);
    dist[i] = d;
    hits[i] = c;
}

extern "C" int ppt_surface_axis_rays(const ppt_surface* s, int64_t n, const double* points, double* min_dist,
                                     int32_t* hits, void* stream) {
    if (!s) return fail(PPT_ERR_ARG, "surface is NULL");
    if (n < 0) return fail(PPT_ERR_ARG, "n must be >= 0");
    if (n == 0) return PPT_OK;
    if (!points || !min_dist || !hits) return fail(PPT_ERR_ARG, "points, min_dist and hits must not be NULL");
    const int block = 128;
    axis_rays_kernel<<<grid_for(n * 6, block), block, 0, static_cast<cudaStream_t>(stream)>>>(s->dev, n, points,
                                                                                              min_dist, hits);
    PPT_CUDA_TRY(cudaGetLastError());
    return PPT_OK;
}

extern "C" int ppt_surface_destroy(ppt_surface* s) {
    if (!s) return PPT_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    cudaError_t e = cudaFree(s->buf);
    cudaSetDevice(prev);
    delete s;
    if (e != cudaSuccess) return cuda_fail(e, "cudaFree(surface)");
    return PPT_OK;
}

extern "C" int ppt_surface_info(const ppt_surface* s, int64_t* bytes, int32_t dims[3]) {
    if (!s) return fail(PPT_ERR_ARG, "surface is NULL");
    if (bytes) *bytes = (int64_t)s->bytes;
    if (dims)
        for (int a = 0; a < 3; ++a) dims[a] = s->dev.dims[a];
    return PPT_OK;
}

extern "C" int ppt_surface_segments_hit(const ppt_surface* s, int64_t n, const double* p0, const double* p1,
                                        uint8_t* hit, void* stream) {
    if (!s) return fail(PPT_ERR_ARG, "surface is NULL");
    if (n < 0) return fail(PPT_ERR_ARG, "n must be >= 0");
    if (n == 0) return PPT_OK;
    if (!p0 || !p1 || !hit) return fail(PPT_ERR_ARG, "p0, p1 and hit must not be NULL");
    const int block = 128;
    segments_hit_kernel<<<grid_for(n, block), block, 0, static_cast<cudaStream_t>(stream)>>>(s->dev, n, p0, p1,
                                                                                             hit);
    PPT_CUDA_TRY(cudaGetLastError());
    return PPT_OK;
}
