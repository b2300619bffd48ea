// dem_costmap.cu — KE collision costmap of the ice field (the planner's map).
//
// Restates medea_ice_ship/jax_costmap.py:build_costmap_jax (:179-331) on the
// GPU, as the reference runs it (float64 mode):
//   * per-element KE constant in double, clipped, then float (:256-268);
//   * rasterisation: every cell is the maximum over elements of
//     ke * max(0, (eff_r^2 - d^2) / eff_r^2) in float (:99-139); each element
//     paints only its bounding box of cells (one warp per element) with an
//     atomicMax on the float bits, exact because maxima do not depend on order;
//   * an element whose contribution the reference would make NaN everywhere
//     (NaN centroid, non-finite radius, NaN constant) makes the grid NaN, as
//     jnp.max over the stacked contributions does;
//   * the SIC modulation grid * SIC^weight when ice_resistance_weight > 0
//     (:271-284), SIC a float64 box mean of the ice-covered cells;
//   * the open-water floor max(grid, base_cost) (:286);
//   * the ship-footprint dilation: a (2h+1)^2 max window over the edge-padded
//     grid (:142-176), as a row pass and a column pass (exact for a max).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "dem_b200.h"
#include "dem_math.cuh"

namespace {

constexpr int kCmThreads = 256;

// the reference's float32 rasteriser arguments, rounded as the weak scalars are
struct CmArgs {
    int n, rows, cols;
    float x0, y0, res;    // grid origin and cell size
    float buf1, half_res; // float(1 + buffer factor), float(0.5 * resolution)
    double ccv2, ship_m, ke_scale;  // collision_cost * v * v, ship mass, ke_cost_scale
    int has_masses;
};

template <typename T>
__device__ __forceinline__ double mass_of(const T* masses, const T* radii, const T* thick, int has, int e) {
    if (has) return (double)masses[e];
    const double r = (double)radii[e];
    return 3.141592653589793 * (r * r) * (double)thick[e] * 920.0;  // jax_costmap.py:259
}

// KE constant of element e (jax_costmap.py:261-268): float64, clip to [0, 1e8], float.
__device__ __forceinline__ float ke_constant(const CmArgs& c, double m) {
    const double M = c.ship_m;
    double ke = c.ccv2 * m * M * (m + 2.0 * M) / (2.0 * ((M + m) * (M + m))) * c.ke_scale;
    ke = dem::jclip(ke, 0.0, 1e8);
    return (float)ke;
}

template <typename T>
__global__ void __launch_bounds__(kCmThreads) cm_paint_kernel(CmArgs c, const T* cents, const T* radii,
                                                               const T* thick, const T* masses,
                                                               unsigned* grid, int* poison) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int e = warp; e < c.n; e += nwarps) {
        const float cx = (float)cents[2 * e], cy = (float)cents[2 * e + 1];
        const float r = (float)radii[e];
        const float kw = ke_constant(c, mass_of(masses, radii, thick, c.has_masses, e));
        const float eff = r * c.buf1 + c.half_res;
        const float eff2 = eff * eff;
        if (isnan(cx) || isnan(cy) || !isfinite(eff2) || isnan(kw)) {
            if (lane == 0) atomicExch(poison, 1);
            continue;
        }
        // cells whose centre lies within eff of the centroid, with one cell of slack
        const double lo_x = ((double)cx - (double)eff - (double)c.x0) / (double)c.res - 0.5;
        const double hi_x = ((double)cx + (double)eff - (double)c.x0) / (double)c.res - 0.5;
        const double lo_y = ((double)cy - (double)eff - (double)c.y0) / (double)c.res - 0.5;
        const double hi_y = ((double)cy + (double)eff - (double)c.y0) / (double)c.res - 0.5;
        if (!(hi_x >= -1.0 && lo_x <= (double)c.cols && hi_y >= -1.0 && lo_y <= (double)c.rows)) continue;
        const int c0 = (int)fmax(floor(lo_x) - 1.0, 0.0), c1 = (int)fmin(ceil(hi_x) + 1.0, (double)(c.cols - 1));
        const int r0 = (int)fmax(floor(lo_y) - 1.0, 0.0), r1 = (int)fmin(ceil(hi_y) + 1.0, (double)(c.rows - 1));
        if (c1 < c0 || r1 < r0) continue;
        const int w = c1 - c0 + 1;
        const int cells = w * (r1 - r0 + 1);
        for (int t = lane; t < cells; t += 32) {
            const int row = r0 + t / w, col = c0 + t % w;
            const float xc = c.x0 + ((float)col + 0.5f) * c.res;
            const float yc = c.y0 + ((float)row + 0.5f) * c.res;
            const float dx = xc - cx, dy = yc - cy;
            const float dsq = dx * dx + dy * dy;
            const float fall = dem::jmax(0.0f, (eff2 - dsq) / eff2);
            const float v = kw * fall;
            if (v > 0.0f) atomicMax(&grid[(size_t)row * c.cols + col], __float_as_uint(v));
        }
    }
}

// SIC modulation (jax_costmap.py:271-284): SIC = box mean of the ice-covered
// cells (grid > 0) over a k x k window with mirror padding, as SciPy's
// uniform_filter computes it in float64 (along axis 0, then axis 1, each a
// running sum: the first window summed in order, then + (entering - leaving)),
// then grid *= max(float(clip(SIC, 0, 1)), 1e-6f)^weight.  One thread per
// column for the first pass, one per row for the second (which also scales).
__device__ __forceinline__ int mirror(int p, int len) { return p < 0 ? -p - 1 : (p >= len ? 2 * len - p - 1 : p); }

__global__ void cm_sic_cols_kernel(const float* __restrict__ grid, double* __restrict__ a, int rows, int cols, int k) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    const int s1 = k / 2;
    auto occ = [&](int p) -> double { return grid[(size_t)mirror(p, rows) * cols + c] > 0.0f ? 1.0 : 0.0; };
    double tmp = 0.0;
    for (int l = 0; l < k; ++l) tmp += occ(l - s1);
    a[c] = tmp / (double)k;
    for (int i = 1; i < rows; ++i) {
        tmp += occ(i + k - 1 - s1) - occ(i - 1 - s1);
        a[(size_t)i * cols + c] = tmp / (double)k;
    }
}

__global__ void cm_sic_rows_kernel(float* __restrict__ grid, const double* __restrict__ a, int rows, int cols, int k,
                                   double weight) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const int s1 = k / 2;
    const double* line = a + (size_t)r * cols;
    float* g = grid + (size_t)r * cols;
    auto scale = [&](int i, double s) {
        const float sf = (float)dem::jclip(s, 0.0, 1.0);
        const float safe = dem::jmax(sf, 1e-6f);
        // the power in double, rounded once (exact for weight 1)
        const float pw = (weight == 1.0) ? safe : (float)pow((double)safe, weight);
        g[i] = g[i] * pw;
    };
    double tmp = 0.0;
    for (int l = 0; l < k; ++l) tmp += line[mirror(l - s1, cols)];
    // the sums read the separate array `a`, so the grid row is scaled in place
    scale(0, tmp / (double)k);
    for (int i = 1; i < cols; ++i) {
        tmp += line[mirror(i + k - 1 - s1, cols)] - line[mirror(i - 1 - s1, cols)];
        scale(i, tmp / (double)k);
    }
}

// NaN poisoning, then the open-water floor (a NaN-propagating maximum); with
// no element at all, the open-water cost itself (jax_costmap.py:288-289)
__global__ void cm_floor_kernel(float* grid, size_t cells, float base, const int* poison, int empty) {
    const bool p = *poison != 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x)
        grid[i] = p ? __int_as_float(0x7fc00000) : (empty ? base : dem::jmax(grid[i], base));
}

// one pass of the square max window: along columns (dir 0) or rows (dir 1),
// indices clamped to the grid (edge padding)
__global__ void cm_dilate_kernel(const float* in, float* out, int rows, int cols, int half, int dir) {
    const size_t cells = (size_t)rows * cols;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols), c = (int)(i % cols);
        float m = -INFINITY;
        for (int d = -half; d <= half; ++d) {
            const int rr = dir ? min(max(r + d, 0), rows - 1) : r;
            const int cc = dir ? c : min(max(c + d, 0), cols - 1);
            m = dem::jmax(m, in[(size_t)rr * cols + cc]);
        }
        out[i] = m;
    }
}

template <typename T>
int launch_costmap(int32_t n, const void* cents, const void* radii, const void* thick, const void* masses,
                   const DemCostmapParams* p, float* grid, float* tmp, int32_t* poison, cudaStream_t st) {
    const size_t cells = (size_t)p->rows * p->cols;
    CmArgs c;
    c.n = n;
    c.rows = p->rows;
    c.cols = p->cols;
    c.x0 = (float)p->x_origin;
    c.y0 = (float)p->y_origin;
    c.res = (float)p->resolution;
    c.buf1 = (float)(1.0 + p->obs_cost_buffer_factor);
    c.half_res = (float)(0.5 * p->resolution);
    const double v = std::fmax(p->ship_speed, 1e-6);
    c.ccv2 = p->collision_cost * v * v;
    c.ship_m = p->ship_mass;
    c.ke_scale = p->ke_cost_scale;
    c.has_masses = p->has_masses;
    if (cudaMemsetAsync(poison, 0, sizeof(int32_t), st) != cudaSuccess) return DEM_ERR_CUDA;
    // grid = +0.0 everywhere (all contributions are >= +0)
    if (cudaMemsetAsync(grid, 0, sizeof(float) * cells, st) != cudaSuccess) return DEM_ERR_CUDA;
    if (n > 0) {
        const int blocks = (int)std::min<long long>(((long long)n * 32 + kCmThreads - 1) / kCmThreads, 65535LL);
        cm_paint_kernel<T><<<blocks, kCmThreads, 0, st>>>(c, (const T*)cents, (const T*)radii, (const T*)thick,
                                                          (const T*)masses, (unsigned*)grid, (int*)poison);
        if (cudaGetLastError() != cudaSuccess) return DEM_ERR_CUDA;
    }
    if (n > 0 && p->ice_resistance_weight > 0.0) {
        const int k = std::min(31, (std::min(p->rows, p->cols) / 4) | 1);  // odd (jax_costmap.py:274-276)
        double* a = reinterpret_cast<double*>(p->sic_scratch);
        cm_sic_cols_kernel<<<(p->cols + 127) / 128, 128, 0, st>>>(grid, a, p->rows, p->cols, k);
        cm_sic_rows_kernel<<<(p->rows + 127) / 128, 128, 0, st>>>(grid, a, p->rows, p->cols, k,
                                                                 p->ice_resistance_weight);
        if (cudaGetLastError() != cudaSuccess) return DEM_ERR_CUDA;
    }
    const int eblocks = (int)std::min<size_t>((cells + kCmThreads - 1) / kCmThreads, (size_t)65535);
    cm_floor_kernel<<<eblocks, kCmThreads, 0, st>>>(grid, cells, (float)p->base_cost, (const int*)poison, n == 0);
    if (cudaGetLastError() != cudaSuccess) return DEM_ERR_CUDA;
    if (p->dilate_half > 0) {
        cm_dilate_kernel<<<eblocks, kCmThreads, 0, st>>>(grid, tmp, p->rows, p->cols, p->dilate_half, 0);
        cm_dilate_kernel<<<eblocks, kCmThreads, 0, st>>>(tmp, grid, p->rows, p->cols, p->dilate_half, 1);
        if (cudaGetLastError() != cudaSuccess) return DEM_ERR_CUDA;
    }
    return DEM_OK;
}

}  // namespace

extern "C" int dem_ke_costmap(int32_t dtype, int32_t n, const void* centroids, const void* radii,
                              const void* thicknesses, const void* masses, const DemCostmapParams* p, float* grid,
                              float* tmp, int32_t* flag, void* stream) {
    if (!p || !grid || !flag || (dtype != DEM_F32 && dtype != DEM_F64) || n < 0) return DEM_ERR_INVALID;
    if (p->rows < 1 || p->cols < 1 || !(p->resolution > 0.0) || p->dilate_half < 0) return DEM_ERR_INVALID;
    if ((long long)p->rows * p->cols >= (1LL << 31)) return DEM_ERR_INVALID;
    if (p->dilate_half > 0 && !tmp) return DEM_ERR_INVALID;
    if (!(p->ice_resistance_weight >= 0.0) || (p->ice_resistance_weight > 0.0 && !p->sic_scratch))
        return DEM_ERR_INVALID;
    if (n > 0 && (!centroids || !radii || (p->has_masses ? !masses : !thicknesses))) return DEM_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == DEM_F32) return launch_costmap<float>(n, centroids, radii, thicknesses, masses, p, grid, tmp, flag, st);
    return launch_costmap<double>(n, centroids, radii, thicknesses, masses, p, grid, tmp, flag, st);
}
