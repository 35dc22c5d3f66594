// Field maps: upload/accumulate of node values into the interleaved device
// layout (records storing only the components that are not identically
// zero), and standalone E/B evaluation at arbitrary points.
//
// Reference behaviour restated here:
//   Field.from_arrays builds one NumbaInterpolator per component on the
//   shared grid, values copied to contiguous float64
//   (src/PyPATools/field.py:345-387, field_src/interpolators.py:299-347);
//   Field.__call__ -> _get_field_3d evaluates the three components and
//   multiplies by the field's scaling (field.py:213-244, :491-504).
#include <cmath>
#include <cstring>
#include <vector>

#include "ppt_internal.cuh"

namespace ppt {

int grid_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    return (int)(g < 1 ? 1 : g);
}

// Small particle counts (the 4096-particle case) would put all blocks on a
// handful of SMs; narrower blocks spread them over the 148 SMs.
int pick_block(int64_t n) {
    if (n <= 148LL * 32) return 32;
    if (n <= 148LL * 64 * 2) return 64;
    return 128;
}

// Layout storing a component mask: the smallest compiled layout containing it.
int layout_for(uint32_t comp_mask) {
    if (comp_mask == 0 || comp_mask > 0x3F) return -1;
    const int order[] = {kLayBz, kLayEzBz, kLayE, kLayB, kLayExEyBz, kLayFull};   // by size
    for (int layout : order)
        if ((comp_mask & ~(uint32_t)layout) == 0) return layout;
    return kLayFull;
}

// Record slot of component c (0..5) in a layout, or -1 when not stored.
int layout_slot(int layout, int c) {
    if (!(layout & (1 << c))) return -1;
    if (layout == kLayFull) return c < 3 ? c : c + 1;
    int slot = 0;
    for (int k = 0; k < c; ++k) slot += (layout >> k) & 1;
    return slot;
}

// ---------------------------------------------------------------------------
// accumulate kernel: map[node][slot] += scale * src[node]
// ---------------------------------------------------------------------------
template <typename Dst, typename Src>
__global__ void map_add_kernel(Dst* __restrict__ dst, int stride, int slot,
                               const Src* __restrict__ src, double scale, int64_t nodes) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t step = (int64_t)gridDim.x * blockDim.x;
    for (; i < nodes; i += step) {
        Dst* p = dst + i * stride + slot;
        *p = (Dst)((double)*p + scale * (double)src[i]);
    }
}

// The same for a map with axes it does not vary along: stored node (I, J, K)
// reads the caller's node (i, j, k), i = 0 on such an axis (both stored
// layers get the one source value).
struct FlatIndex {
    int64_t n1, n2;         // stored node layers of y and z
    int64_t src1, src2;     // caller's node counts of y and z
    int flat[3];
};

template <typename Dst, typename Src>
__global__ void map_add_flat_kernel(Dst* __restrict__ dst, int stride, int slot, const Src* __restrict__ src,
                                    double scale, int64_t nodes, FlatIndex X) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t step = (int64_t)gridDim.x * blockDim.x;
    for (; p < nodes; p += step) {
        const int64_t K = p % X.n2, J = (p / X.n2) % X.n1, I = p / (X.n1 * X.n2);
        const int64_t i = X.flat[0] ? 0 : I, j = X.flat[1] ? 0 : J, k = X.flat[2] ? 0 : K;
        Dst* q = dst + p * stride + slot;
        *q = (Dst)((double)*q + scale * (double)src[(i * X.src1 + j) * X.src2 + k]);
    }
}

int build_fields(const ppt_fields* f, FieldsDev* out) {
    if (!f) return fail(PPT_ERR_ARG, "fields is NULL");
    if (f->n_maps < 0 || f->n_maps > PPT_MAX_MAPS)
        return fail(PPT_ERR_ARG, "n_maps must be in [0, PPT_MAX_MAPS]");
    std::memset(out, 0, sizeof(*out));
    out->n_maps = f->n_maps;
    for (int i = 0; i < f->n_maps; ++i) {
        if (!f->maps[i]) return fail(PPT_ERR_ARG, "fields->maps[i] is NULL");
        out->maps[i] = f->maps[i]->dev;
        out->e_maps += out->maps[i].has_e;
        out->b_maps += out->maps[i].has_b;
    }
    for (int a = 0; a < 3; ++a) {
        out->box_lo[a] = f->n_maps ? out->maps[0].ax[a].lo : 0.0;
        out->box_hi[a] = f->n_maps ? out->maps[0].ax[a].hi : 0.0;
        for (int i = 1; i < f->n_maps; ++i) {
            out->box_lo[a] = std::min(out->box_lo[a], out->maps[i].ax[a].lo);
            out->box_hi[a] = std::max(out->box_hi[a], out->maps[i].ax[a].hi);
        }
    }
    for (int c = 0; c < 3; ++c) {
        out->e_const[c] = f->e_const[c];
        out->b_const[c] = f->b_const[c];
        out->e_const_nz |= (f->e_const[c] != 0.0);
        out->b_const_nz |= (f->b_const[c] != 0.0);
    }
    return PPT_OK;
}

// ---------------------------------------------------------------------------
// point evaluation kernel (the 'cuda' interpolator backend)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float tri_f(float c000, float c100, float c010, float c110, float c001,
                                       float c101, float c011, float c111, float tx, float ty, float tz);

__global__ void field_eval_kernel(const __grid_constant__ FieldsDev F, int64_t n,
                                  const double* __restrict__ pts, double* __restrict__ e_out,
                                  double* __restrict__ b_out) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= n) return;
    V3 r = v3(pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]);
    V3 E = v3(F.e_const[0], F.e_const[1], F.e_const[2]);
    V3 B = v3(F.b_const[0], F.b_const[1], F.b_const[2]);
    for (int mi = 0; mi < F.n_maps; ++mi) {
        const MapDev& m = F.maps[mi];
        Cell c;
        if (!locate(m, r, c)) continue;
        if (m.dtype == PPT_DTYPE_F64) {
            gather_map_f64(m, c, E, B);
        } else {
            // float32 records: every stored slot, then by layout
            const float* base = static_cast<const float*>(m.data);
            const float tx = (float)c.tx, ty = (float)c.ty, tz = (float)c.tz;
            float val[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int k = 0; k < m.stride; ++k) {
                float q[8];
                for (int corner = 0; corner < 8; ++corner) {
                    const int di = (corner >> 2) & 1, dj = (corner >> 1) & 1, dk = corner & 1;
                    const int64_t node = c.base + di * m.sx + dj * m.sy + dk;
                    q[corner] = __ldg(base + node * m.stride + k);
                }
                val[k] = tri_f(q[0], q[4], q[2], q[6], q[1], q[5], q[3], q[7], tx, ty, tz);
            }
            double comp[6];
            for (int cc = 0; cc < 6; ++cc) {
                int slot = -1;
                if (m.layout & (1 << cc)) {
                    if (m.layout == kLayFull) slot = cc < 3 ? cc : cc + 1;
                    else { slot = 0; for (int k = 0; k < cc; ++k) slot += (m.layout >> k) & 1; }
                }
                comp[cc] = slot >= 0 ? (double)val[slot] : 0.0;
            }
            if (m.has_e) E = E + v3(comp[0], comp[1], comp[2]);
            if (m.has_b) B = B + v3(comp[3], comp[4], comp[5]);
        }
    }
    if (e_out) { e_out[3 * p] = E.x; e_out[3 * p + 1] = E.y; e_out[3 * p + 2] = E.z; }
    if (b_out) { b_out[3 * p] = B.x; b_out[3 * p + 1] = B.y; b_out[3 * p + 2] = B.z; }
}

__device__ __forceinline__ float tri_f(float c000, float c100, float c010, float c110, float c001,
                                       float c101, float c011, float c111, float tx, float ty, float tz) {
    float c00 = fmaf(c100 - c000, tx, c000);
    float c01 = fmaf(c101 - c001, tx, c001);
    float c10 = fmaf(c110 - c010, tx, c010);
    float c11 = fmaf(c111 - c011, tx, c011);
    float c0 = fmaf(c10 - c00, ty, c00);
    float c1 = fmaf(c11 - c01, ty, c01);
    return fmaf(c1 - c0, tz, c0);
}

template <typename Dst, typename Src>
void launch_map_add(const ppt_fieldmap* map, Dst* dst, int slot, const Src* src, double scale, cudaStream_t s) {
    const int64_t nodes = map->n[0] * map->n[1] * map->n[2];
    const int block = 256;
    const int64_t g = (nodes + block - 1) / block;
    const int grid = (int)(g > 148 * 32 ? 148 * 32 : g);
    FlatIndex X;
    bool any_flat = false;
    for (int d = 0; d < 3; ++d) {
        X.flat[d] = map->src_n[d] == 1 && map->n[d] == 2;
        any_flat |= X.flat[d] != 0;
    }
    if (!any_flat) {
        map_add_kernel<<<grid, block, 0, s>>>(dst, map->dev.stride, slot, src, scale, nodes);
        return;
    }
    X.n1 = map->n[1];
    X.n2 = map->n[2];
    X.src1 = map->src_n[1];
    X.src2 = map->src_n[2];
    map_add_flat_kernel<<<grid, block, 0, s>>>(dst, map->dev.stride, slot, src, scale, nodes, X);
}

}  // namespace ppt

using namespace ppt;

extern "C" int ppt_fieldmap_layout(uint32_t comp_mask) {
    const int layout = layout_for(comp_mask);
    if (layout < 0) return fail(PPT_ERR_ARG, "comp_mask must be in [1, 0x3F]");
    return layout;
}

extern "C" int ppt_fieldmap_create(const ppt_grid_desc* grid, int has_e, int has_b, int store_dtype,
                                   ppt_fieldmap** out) {
    if (!has_e && !has_b) {
        if (out) *out = nullptr;
        return fail(PPT_ERR_ARG, "a map must store E, B or both");
    }
    return ppt_fieldmap_create_masked(grid, (has_e ? 0x07u : 0u) | (has_b ? 0x38u : 0u), store_dtype, out);
}

extern "C" int ppt_fieldmap_create_masked(const ppt_grid_desc* grid, uint32_t comp_mask, int store_dtype,
                                          ppt_fieldmap** out) {
    if (!grid || !out) return fail(PPT_ERR_ARG, "grid and out must not be NULL");
    *out = nullptr;
    const int layout = layout_for(comp_mask);
    if (layout < 0) return fail(PPT_ERR_ARG, "comp_mask must be in [1, 0x3F]");
    if (store_dtype != PPT_DTYPE_F64 && store_dtype != PPT_DTYPE_F32)
        return fail(PPT_ERR_ARG, "store_dtype must be PPT_DTYPE_F64 or PPT_DTYPE_F32");
    ppt_fieldmap m;
    std::memset(&m, 0, sizeof(m));
    int64_t total_nodes = 1;
    int flat_axes = 0;
    std::vector<double> axes;
    for (int d = 0; d < 3; ++d) {
        int64_t n = grid->n[d];
        if (n < 1) return fail(PPT_ERR_ARG, "every axis needs at least 1 node");
        if (n > (1LL << 30)) return fail(PPT_ERR_ARG, "axis too long");
        m.src_n[d] = n;
        if (n == 1) {
            // the map does not vary along this axis (a 1D or 2D field)
            AxisDev& a = m.dev.ax[d];
            a.n = 2;
            a.lo = -kFlatHalf;
            a.hi = kFlatHalf;
            a.d = 2.0 * kFlatHalf;
            a.inv_d = 0.5 / kFlatHalf;
            a.uniform = 1;
            m.n[d] = 2;
            total_nodes *= 2;
            axes.push_back(a.lo);
            axes.push_back(a.hi);
            ++flat_axes;
            continue;
        }
        if (!grid->axis[d]) return fail(PPT_ERR_ARG, "grid axis pointer is NULL");
        const double* g = grid->axis[d];
        for (int64_t i = 1; i < n; ++i)
            if (!(g[i] > g[i - 1])) return fail(PPT_ERR_ARG, "grid axes must be strictly increasing");
        AxisDev& a = m.dev.ax[d];
        a.n = (int)n;
        a.lo = g[0];
        a.hi = g[n - 1];
        a.d = (a.hi - a.lo) / (double)(n - 1);
        a.inv_d = (double)(n - 1) / (a.hi - a.lo);
        // Uniform when every node sits within 1e-12 cell widths of lo + i d:
        // the weights then differ from the bisection ones by rounding only.
        double worst = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            double dev = std::fabs(g[i] - (a.lo + (double)i * a.d));
            worst = dev > worst ? dev : worst;
        }
        a.uniform = worst <= 1e-12 * a.d;
        m.n[d] = n;
        total_nodes *= n;
        axes.insert(axes.end(), g, g + n);
    }
    if (flat_axes == 3) return fail(PPT_ERR_ARG, "a map needs an axis with at least 2 nodes (use constants)");
    m.dev.all_uniform = m.dev.ax[0].uniform && m.dev.ax[1].uniform && m.dev.ax[2].uniform;
    if (store_dtype == PPT_DTYPE_F32 && !m.dev.all_uniform)
        return fail(PPT_ERR_UNSUPPORTED, "float32 (mixed-precision) maps need uniform grid axes");
    m.dev.layout = layout;
    m.dev.has_e = layout_has_e(layout) ? 1 : 0;
    m.dev.has_b = layout_has_b(layout) ? 1 : 0;
    m.dev.stride = layout_width(layout);
    m.dev.b_off = layout == kLayFull ? 4 : 0;
    m.dev.dtype = store_dtype;
    m.dev.sy = m.n[2];
    m.dev.sx = m.n[1] * m.n[2];
    m.dev.idx32 = total_nodes * m.dev.stride < (1LL << 31) ? 1 : 0;
    size_t elem = store_dtype == PPT_DTYPE_F64 ? 8 : 4;
    m.bytes = (size_t)total_nodes * m.dev.stride * elem;
    PPT_CUDA_TRY(cudaGetDevice(&m.device));
    cudaError_t e = cudaMalloc(&m.data, m.bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(PPT_ERR_OOM, "cudaMalloc of the field map failed");
    }
    e = cudaMalloc(&m.axis_buf, axes.size() * sizeof(double));
    if (e != cudaSuccess) {
        cudaFree(m.data);
        cudaGetLastError();
        return fail(PPT_ERR_OOM, "cudaMalloc of the grid axes failed");
    }
    e = cudaMemcpy(m.axis_buf, axes.data(), axes.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m.data, 0, m.bytes);
    if (e != cudaSuccess) {
        cudaFree(m.data);
        cudaFree(m.axis_buf);
        return cuda_fail(e, "field map initialisation");
    }
    m.dev.data = m.data;
    m.dev.ax[0].nodes = m.axis_buf;
    m.dev.ax[1].nodes = m.axis_buf + m.n[0];
    m.dev.ax[2].nodes = m.axis_buf + m.n[0] + m.n[1];
    *out = new ppt_fieldmap(m);
    return PPT_OK;
}

extern "C" int ppt_fieldmap_add(ppt_fieldmap* map, const void* const comp[6], const double scale[6],
                                int src_dtype, void* stream) {
    if (!map || !comp || !scale) return fail(PPT_ERR_ARG, "map, comp and scale must not be NULL");
    if (src_dtype != PPT_DTYPE_F64 && src_dtype != PPT_DTYPE_F32)
        return fail(PPT_ERR_ARG, "src_dtype must be PPT_DTYPE_F64 or PPT_DTYPE_F32");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (int c = 0; c < 6; ++c) {
        if (!comp[c]) continue;
        const int slot = layout_slot(map->dev.layout, c);
        if (slot < 0) {
            static const char* names[6] = {"Ex", "Ey", "Ez", "Bx", "By", "Bz"};
            return fail(PPT_ERR_ARG, std::string("the map's layout does not store ") + names[c]);
        }
        const bool f64_dst = map->dev.dtype == PPT_DTYPE_F64, f64_src = src_dtype == PPT_DTYPE_F64;
        double* d64 = static_cast<double*>(map->data);
        float* d32 = static_cast<float*>(map->data);
        const double* s64 = static_cast<const double*>(comp[c]);
        const float* s32 = static_cast<const float*>(comp[c]);
        if (f64_dst && f64_src) launch_map_add(map, d64, slot, s64, scale[c], s);
        else if (f64_dst) launch_map_add(map, d64, slot, s32, scale[c], s);
        else if (f64_src) launch_map_add(map, d32, slot, s64, scale[c], s);
        else launch_map_add(map, d32, slot, s32, scale[c], s);
        PPT_CUDA_TRY(cudaGetLastError());
    }
    return PPT_OK;
}

extern "C" int ppt_fieldmap_destroy(ppt_fieldmap* map) {
    if (!map) return PPT_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(map->device);
    cudaError_t e1 = cudaFree(map->data);
    cudaError_t e2 = cudaFree(map->axis_buf);
    cudaSetDevice(prev);
    delete map;
    if (e1 != cudaSuccess) return cuda_fail(e1, "cudaFree(field map)");
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaFree(grid axes)");
    return PPT_OK;
}

extern "C" int ppt_fieldmap_info(const ppt_fieldmap* map, int64_t* bytes, int* flags) {
    if (!map) return fail(PPT_ERR_ARG, "map is NULL");
    if (bytes) *bytes = (int64_t)map->bytes;
    if (flags)
        *flags = map->dev.has_e | (map->dev.has_b << 1) | (map->dev.all_uniform << 2) |
                 ((map->dev.dtype == PPT_DTYPE_F32) << 3) | (map->dev.layout << 8);
    return PPT_OK;
}

extern "C" int ppt_field_eval(const ppt_fields* fields, int64_t n, const double* pts, double* e_out,
                              double* b_out, void* stream) {
    if (n < 0) return fail(PPT_ERR_ARG, "n must be >= 0");
    if (n == 0) return PPT_OK;
    if (!pts) return fail(PPT_ERR_ARG, "pts is NULL");
    FieldsDev F;
    int rc = build_fields(fields, &F);
    if (rc) return rc;
    const int block = 128;
    field_eval_kernel<<<grid_for(n, block), block, 0, static_cast<cudaStream_t>(stream)>>>(F, n, pts, e_out,
                                                                                           b_out);
    PPT_CUDA_TRY(cudaGetLastError());
    return PPT_OK;
}
