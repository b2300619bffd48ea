// dem_rollout.cu — per-rollout costs of a batch of planner rollouts.
//
// One CTA per rollout q, after dem_rollout_segment has stepped every rollout's
// ship and ice window:
//   * the reference planner's four unweighted cost components
//     (medea_ice_ship/jax_mbd_planner.py:_make_raw_components_fn, :569-665) of
//     the pose path eta0, eta_1 .. eta_H, in float32 as the planner runs them:
//     costmap integral (bilinear query :128-168 at the hull centre and four
//     box corners, maximum, trapezoid rule over segment lengths), path length,
//     exponentially discounted goal distance, and jerk of the normalised
//     controls; the optional goal-line truncation (:621-637) masks waypoints
//     after the first crossing;
//   * the kinetic energy the rollout transferred to its ice window,
//     sum_e 0.5 m_e (|v_e(H)|^2 - |v_e(0)|^2) over the window's elements, in
//     double with a fixed summation order (run to run identical).
// Waypoint terms are computed one thread per waypoint into shared memory; the
// sums over waypoints run in waypoint order on one thread.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "dem_b200.h"

namespace {

constexpr int kRcThreads = 128;
constexpr int kRcMaxHorizon = 2000;  // 6 (H + 1) floats of shared memory stay under 48 KB

struct RcArgs {
    int Q, H, rows, cols, use_hull, has_truncate, has_jerk, has_ke;
    float xo, yo, res, oob, hl, hw, gx, gy, trunc_y, tau;
    float ac[3], as[3];
};

// jnp.max semantics: NaN wins
__device__ __forceinline__ float max_nan(float a, float b) { return (a > b || a != a) ? a : b; }

// _make_query (jax_mbd_planner.py:128-168) in float32
__device__ __forceinline__ float query(const RcArgs& c, const float* __restrict__ g, float x, float y) {
    const float cf = (x - c.xo) / c.res - 0.5f;
    const float rf = (y - c.yo) / c.res - 0.5f;
    const int r0 = (int)floorf(rf), c0 = (int)floorf(cf);
    const float fr = rf - (float)r0, fc = cf - (float)c0;
    const int r0c = min(max(r0, 0), c.rows - 1), r1c = min(max(r0 + 1, 0), c.rows - 1);
    const int c0c = min(max(c0, 0), c.cols - 1), c1c = min(max(c0 + 1, 0), c.cols - 1);
    const float oob = (c0 < 0 || c0 + 1 >= c.cols) ? c.oob : 0.0f;
    const float g00 = __ldg(g + (size_t)r0c * c.cols + c0c), g01 = __ldg(g + (size_t)r0c * c.cols + c1c);
    const float g10 = __ldg(g + (size_t)r1c * c.cols + c0c), g11 = __ldg(g + (size_t)r1c * c.cols + c1c);
    const float val = g00 * (1.0f - fr) * (1.0f - fc) + g01 * (1.0f - fr) * fc + g10 * fr * (1.0f - fc) + g11 * fr * fc;
    return val + oob;
}

// a waypoint's cost: the query at the hull centre and its four box corners,
// maximum (NaN wins), or at the centre alone without a hull
__device__ __forceinline__ float waypoint_cost(const RcArgs& c, const float* __restrict__ grid, float x, float y,
                                               float psi) {
    if (!c.use_hull) return query(c, grid, x, y);
    const float cs = cosf(psi), sn = sinf(psi);
    const float dxb[5] = {0.0f, c.hl, c.hl, -c.hl, -c.hl};
    const float dyb[5] = {0.0f, c.hw, -c.hw, c.hw, -c.hw};
    float w = 0.0f;
    for (int k = 0; k < 5; ++k) {
        const float wx = x + cs * dxb[k] - sn * dyb[k];
        const float wy = y + sn * dxb[k] + cs * dyb[k];
        const float v = query(c, grid, wx, wy);
        w = (k == 0) ? v : max_nan(w, v);
    }
    return w;
}

template <typename T>
__global__ void __launch_bounds__(kRcThreads) rollout_cost_kernel(RcArgs c, const int* __restrict__ sys_start,
                                                                  const T* __restrict__ eta0,
                                                                  const T* __restrict__ eta_hist,
                                                                  const T* __restrict__ u, const float* __restrict__ grid,
                                                                  const T* __restrict__ masses,
                                                                  const T* __restrict__ v0, const T* __restrict__ v1,
                                                                  double* __restrict__ out) {
    extern __shared__ float sm[];
    const int H = c.H, W = H + 1, q = blockIdx.x;
    float* wp = sm;            // (W) waypoint cost
    float* tx = wp + W;        // (W) path x
    float* ty = tx + W;        // (W) path y
    float* dsc = ty + W;       // (W) undiscounted weights exp(-t / tau)
    float* dd = dsc + W;       // (W) goal distance
    float* jk = dd + W;        // (H) squared jerk of step t, summed over the 3 controls
    __shared__ double s_ke[kRcThreads];
    for (int t = threadIdx.x; t < W; t += blockDim.x) {
        const T* p = (t == 0) ? eta0 + 3 * (size_t)q : eta_hist + 3 * ((size_t)(t - 1) * c.Q + q);
        const float x = (float)p[0], y = (float)p[1], psi = (float)p[2];
        wp[t] = waypoint_cost(c, grid, x, y, psi);
        tx[t] = x;
        ty[t] = y;
        dsc[t] = expf(-(float)t / c.tau);
        const float gdx = x - c.gx, gdy = y - c.gy;
        dd[t] = sqrtf(gdx * gdx + gdy * gdy + 1e-4f);
        if (t < H) {
            float j = 0.0f;
            if (c.has_jerk) {
                for (int k = 0; k < 3; ++k) {
                    const float a = ((float)u[3 * ((size_t)t * c.Q + q) + k] - c.ac[k]) / c.as[k];
                    const float b = ((float)u[3 * ((size_t)(t + 1 < H ? t + 1 : t) * c.Q + q) + k] - c.ac[k]) / c.as[k];
                    const float du = b - a;
                    j = j + du * du;
                }
            }
            jk[t] = j;
        }
    }
    // kinetic energy transferred to the window (double, fixed order)
    double ke = 0.0;
    if (c.has_ke) {
        const int e0 = sys_start[q], e1 = sys_start[q + 1];
        for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
            const double m = (double)masses[e];
            const double a0 = (double)v0[2 * (size_t)e], b0 = (double)v0[2 * (size_t)e + 1];
            const double a1 = (double)v1[2 * (size_t)e], b1 = (double)v1[2 * (size_t)e + 1];
            ke += 0.5 * m * ((a1 * a1 + b1 * b1) - (a0 * a0 + b0 * b0));
        }
    }
    s_ke[threadIdx.x] = ke;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) s_ke[threadIdx.x] += s_ke[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    // goal-line truncation: waypoint t counts while max(y_0 .. y_{t-1}) < truncate_y
    float cum = -1e9f, cost = 0.0f, len = 0.0f;
    float mprev = (-1e9f < c.trunc_y) ? 1.0f : 0.0f;  // mask of waypoint 0
    for (int t = 0; t < H; ++t) {
        float m0 = 1.0f, m1 = 1.0f;
        if (c.has_truncate) {
            m0 = mprev;
            cum = (t == 0) ? ty[0] : max_nan(cum, ty[t]);
            m1 = (cum < c.trunc_y) ? 1.0f : 0.0f;  // mask of waypoint t + 1
            mprev = m1;
        }
        const float dx = tx[t + 1] - tx[t], dy = ty[t + 1] - ty[t];
        const float seg = sqrtf(dx * dx + dy * dy + 1e-8f);
        len = len + seg * m0;
        cost = cost + 0.5f * (wp[t] * m0 + wp[t + 1] * m1) * seg;
    }
    float dsum = 0.0f;
    for (int t = 0; t < W; ++t) dsum = dsum + dsc[t];
    float goal = 0.0f;
    for (int t = 0; t < W; ++t) goal = goal + (dsc[t] / dsum) * dd[t];
    float jsum = 0.0f;
    for (int t = 0; t + 1 < H; ++t) jsum = jsum + jk[t];
    const float jerk = c.has_jerk ? jsum / (float)(3 * (H - 1)) : 0.0f;
    double* o = out + 5 * (size_t)q;
    o[0] = (double)cost;
    o[1] = (double)len;
    o[2] = (double)goal;
    o[3] = (double)jerk;
    o[4] = s_ke[0];
}

// one thread per (step, rollout): out[q, t] = the cost of the pose after step t
template <typename T>
__global__ void __launch_bounds__(kRcThreads) waypoint_cost_kernel(RcArgs c, const T* __restrict__ eta_hist,
                                                                   const float* __restrict__ grid,
                                                                   float* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)c.Q * c.H) return;
    const int t = (int)(i / c.Q), q = (int)(i % c.Q);
    const T* p = eta_hist + 3 * (size_t)i;
    out[(size_t)q * c.H + t] = waypoint_cost(c, grid, (float)p[0], (float)p[1], (float)p[2]);
}

// the costmap geometry of the cost arguments, as the planner's float32 query sees it
bool grid_args(const DemRolloutCostParams* p, RcArgs& c) {
    if (p->rows < 1 || p->cols < 1 || (long long)p->rows * p->cols >= (1LL << 31) || !(p->resolution > 0.0))
        return false;
    c.rows = p->rows;
    c.cols = p->cols;
    c.use_hull = (p->ship_length > 0.0 && p->ship_beam > 0.0) ? 1 : 0;
    // the planner's Python scalars meet float32 arrays: each is rounded to float
    c.xo = (float)p->x_origin;
    c.yo = (float)p->y_origin;
    c.res = (float)p->resolution;
    c.oob = (float)p->oob_penalty;
    c.hl = (float)(p->ship_length / 2.0);
    c.hw = (float)(p->ship_beam / 2.0);
    return true;
}

template <typename T>
int launch_costs(const RcArgs& c, const int32_t* sys_start, const void* eta0, const void* eta_hist,
                 const void* u, const float* grid, const void* masses, const void* v0, const void* v1, double* out,
                 cudaStream_t st) {
    const size_t smem = sizeof(float) * (6 * (size_t)(c.H + 1));
    rollout_cost_kernel<T><<<c.Q, kRcThreads, smem, st>>>(c, sys_start, (const T*)eta0, (const T*)eta_hist,
                                                          (const T*)u, grid, (const T*)masses, (const T*)v0,
                                                          (const T*)v1, out);
    return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

}  // namespace

extern "C" int dem_rollout_costs(int32_t dtype, int32_t n_systems, int32_t horizon, const int32_t* system_start,
                                 const void* eta0, const void* eta_hist, const void* controls, const float* grid,
                                 const DemRolloutCostParams* p, const void* masses, const void* vel0,
                                 const void* vel1, double* out, void* stream) {
    if (!p || !out || !eta0 || !eta_hist || !grid || (dtype != DEM_F32 && dtype != DEM_F64)) return DEM_ERR_INVALID;
    if (n_systems < 1 || horizon < 1 || horizon > kRcMaxHorizon) return DEM_ERR_INVALID;
    RcArgs c{};
    if (!grid_args(p, c)) return DEM_ERR_INVALID;
    const bool has_ke = masses || vel0 || vel1;
    if (has_ke && (!masses || !vel0 || !vel1 || !system_start)) return DEM_ERR_INVALID;
    if (controls)
        for (int k = 0; k < 3; ++k)
            if (!(p->action_scale[k] != 0.0) || !std::isfinite(p->action_scale[k])) return DEM_ERR_INVALID;
    c.Q = n_systems;
    c.H = horizon;
    c.has_truncate = p->has_truncate ? 1 : 0;
    c.has_jerk = controls ? 1 : 0;
    c.has_ke = has_ke ? 1 : 0;
    c.gx = (float)p->goal_x;
    c.gy = (float)p->goal_y;
    c.trunc_y = (float)p->truncate_y;
    c.tau = (float)((double)(horizon + 1) / 3.0);
    for (int k = 0; k < 3; ++k) {
        c.ac[k] = (float)p->action_center[k];
        c.as[k] = (float)p->action_scale[k];
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == DEM_F32)
        return launch_costs<float>(c, system_start, eta0, eta_hist, controls, grid, masses, vel0, vel1, out, st);
    return launch_costs<double>(c, system_start, eta0, eta_hist, controls, grid, masses, vel0, vel1, out, st);
}

extern "C" int dem_rollout_waypoint_costs(int32_t dtype, int32_t n_systems, int32_t horizon, const void* eta_hist,
                                          const float* grid, const DemRolloutCostParams* p, float* out,
                                          void* stream) {
    if (!p || !out || !eta_hist || !grid || (dtype != DEM_F32 && dtype != DEM_F64)) return DEM_ERR_INVALID;
    if (n_systems < 1 || horizon < 1 || horizon > kRcMaxHorizon) return DEM_ERR_INVALID;
    RcArgs c{};
    if (!grid_args(p, c)) return DEM_ERR_INVALID;
    c.Q = n_systems;
    c.H = horizon;
    const long long total = (long long)n_systems * horizon;
    const unsigned blocks = (unsigned)((total + kRcThreads - 1) / kRcThreads);
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == DEM_F32)
        waypoint_cost_kernel<float><<<blocks, kRcThreads, 0, st>>>(c, (const float*)eta_hist, grid, out);
    else
        waypoint_cost_kernel<double><<<blocks, kRcThreads, 0, st>>>(c, (const double*)eta_hist, grid, out);
    return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

// ════════════════════════════════════════════════════════════════════════════
// dem_rollout_ice_terms: per rollout, the hull impulse (sum over the steps of
// the frame's J_cumul_incr = |F_ice_on_ship| dt, jax_simulation.py:692-697)
// and the bonds its ship broke (intact at the start, broken at the end), one
// CTA per rollout with fixed-order sums.
// ════════════════════════════════════════════════════════════════════════════
namespace {

template <typename T>
__global__ void __launch_bounds__(kRcThreads) ice_terms_kernel(int Q, int H, const T* __restrict__ J_hist,
                                                               const int* __restrict__ bond_start,
                                                               const uint8_t* __restrict__ intact0,
                                                               const uint8_t* __restrict__ intact1,
                                                               double* __restrict__ out) {
    __shared__ double s_imp[kRcThreads];
    __shared__ long long s_brk[kRcThreads];
    const int q = blockIdx.x;
    double imp = 0.0;
    for (int t = threadIdx.x; t < H; t += blockDim.x) imp += (double)J_hist[(size_t)t * Q + q];
    long long brk = 0;
    if (bond_start) {
        for (int b = bond_start[q] + threadIdx.x; b < bond_start[q + 1]; b += blockDim.x)
            brk += (intact0[b] != 0 && intact1[b] == 0) ? 1 : 0;
    }
    s_imp[threadIdx.x] = imp;
    s_brk[threadIdx.x] = brk;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            s_imp[threadIdx.x] += s_imp[threadIdx.x + w];
            s_brk[threadIdx.x] += s_brk[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[2 * q] = s_imp[0];
        out[2 * q + 1] = (double)s_brk[0];
    }
}

}  // namespace

extern "C" int dem_rollout_ice_terms(int32_t dtype, int32_t n_systems, int32_t horizon, const void* J_hist,
                                     const int32_t* bond_start, const uint8_t* intact0, const uint8_t* intact1,
                                     double* out, void* stream) {
    if ((dtype != DEM_F32 && dtype != DEM_F64) || n_systems < 1 || horizon < 1 || !J_hist || !out)
        return DEM_ERR_INVALID;
    if (bond_start && (!intact0 || !intact1)) return DEM_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == DEM_F32)
        ice_terms_kernel<float><<<n_systems, kRcThreads, 0, st>>>(n_systems, horizon, (const float*)J_hist, bond_start,
                                                                  intact0, intact1, out);
    else
        ice_terms_kernel<double><<<n_systems, kRcThreads, 0, st>>>(n_systems, horizon, (const double*)J_hist,
                                                                   bond_start, intact0, intact1, out);
    return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

// ════════════════════════════════════════════════════════════════════════════
// dem_rollout_sweep_features: what a candidate's rigid-ship path sweeps
// through the plan's ice window, one CTA per candidate.  No counterpart in the
// reference.  An element is hit at the first pose t (0..H) at which its
// centroid, in the frame of that pose, lies inside the hull box grown by the
// element's radius r: |x| < half_len + r and |y| < half_beam + r.  The hit's
// ship velocity is the path's step velocity (pose t - pose t-1) / dt (the
// first step's for t = 0), and v_n its component towards the element's
// centroid, clamped at 0.  Per candidate, in double with fixed-order sums (run
// to run identical):
//   [0] elements hit, [1] their mass, [2] sum 0.5 m |v|^2, [3] sum m v_n,
//   [4] sum m (H + 1 - t) / (H + 1) (early hits weigh more), [5] sum 0.5 m v_n^2,
//   [6] bonds with exactly one end hit, [7] bonds with both ends hit.
// The geometry runs in float32 (cos and sin of the heading rounded from
// double), unfused, as a NumPy float32 evaluation of the same expressions.
// ════════════════════════════════════════════════════════════════════════════
namespace {

constexpr int kSwThreads = 256;
constexpr int kSwFeatures = DEM_SWEEP_FEATURES;
constexpr int kSwMaxElements = DEM_SWEEP_MAX_ELEMENTS;  // hit bits in shared memory: 8 KB
constexpr int kSwMaxHorizon = DEM_SWEEP_MAX_HORIZON;

struct SwArgs {
    int Q, H, n, nb;
    float hl, hw, inv_dt;
};

template <typename T>
__global__ void __launch_bounds__(kSwThreads) sweep_kernel(const SwArgs c, const T* __restrict__ eta0,
                                                           const T* __restrict__ hist, const T* __restrict__ pos,
                                                           const T* __restrict__ radii, const T* __restrict__ mass,
                                                           const int* __restrict__ bi, const int* __restrict__ bj,
                                                           float* __restrict__ out) {
    __shared__ float4 pose[kSwMaxHorizon + 1];  // x, y, cos, sin
    __shared__ float2 pvel[kSwMaxHorizon + 1];
    __shared__ unsigned hit[kSwMaxElements / 32];
    __shared__ double red[kSwThreads];
    const int q = blockIdx.x;
    const int H = c.H;
    for (int t = threadIdx.x; t <= H; t += blockDim.x) {
        const T* p = (t == 0) ? eta0 + 3 * (size_t)q : hist + ((size_t)(t - 1) * c.Q + q) * 3;
        const double psi = (double)p[2];
        pose[t] = make_float4((float)p[0], (float)p[1], (float)cos(psi), (float)sin(psi));
    }
    for (int w = threadIdx.x; w < (c.n + 31) / 32; w += blockDim.x) hit[w] = 0u;
    __syncthreads();
    for (int t = threadIdx.x; t <= H; t += blockDim.x) {
        const int a = (t == 0) ? 1 : t;  // the first step's velocity at the start pose
        pvel[t] = make_float2((pose[a].x - pose[a - 1].x) * c.inv_dt, (pose[a].y - pose[a - 1].y) * c.inv_dt);
    }
    __syncthreads();
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int e = threadIdx.x; e < c.n; e += blockDim.x) {
        const float ex = (float)pos[2 * (size_t)e], ey = (float)pos[2 * (size_t)e + 1];
        const float r = (float)radii[e];
        // a centroid inside the grown box lies within its half-diagonal of the
        // pose (the margin covers the rounding of the rotation): a cheaper
        // first test that rejects no hit
        const float gl = c.hl + r, gw = c.hw + r;
        const float lim2 = (gl * gl + gw * gw) * 1.001f + 1e-3f;
        for (int t = 0; t <= H; ++t) {
            const float4 p = pose[t];
            const float dx = ex - p.x, dy = ey - p.y;
            if (dx * dx + dy * dy > lim2) continue;
            const float bx = p.z * dx + p.w * dy;
            const float by = p.z * dy - p.w * dx;
            if (!(fabsf(bx) < gl && fabsf(by) < gw)) continue;
            const double m = (double)mass[e];
            const double vx = (double)pvel[t].x, vy = (double)pvel[t].y;
            const double dd = sqrt((double)dx * (double)dx + (double)dy * (double)dy);
            const double vn = fmax(0.0, (vx * (double)dx + vy * (double)dy) / fmax(dd, 1e-6));
            acc[0] += 1.0;
            acc[1] += m;
            acc[2] += 0.5 * m * (vx * vx + vy * vy);
            acc[3] += m * vn;
            acc[4] += m * (double)(H + 1 - t) / (double)(H + 1);
            acc[5] += 0.5 * m * vn * vn;
            atomicOr(&hit[e >> 5], 1u << (e & 31));
            break;
        }
    }
    __syncthreads();
    double b1 = 0.0, b2 = 0.0;
    for (int b = threadIdx.x; b < c.nb; b += blockDim.x) {
        const int i = bi[b], j = bj[b];
        if (i < 0 || i >= c.n || j < 0 || j >= c.n) continue;
        const bool hi = (hit[i >> 5] >> (i & 31)) & 1u, hj = (hit[j >> 5] >> (j & 31)) & 1u;
        b1 += (hi != hj) ? 1.0 : 0.0;
        b2 += (hi && hj) ? 1.0 : 0.0;
    }
    const double v[kSwFeatures] = {acc[0], acc[1], acc[2], acc[3], acc[4], acc[5], b1, b2};
    for (int k = 0; k < kSwFeatures; ++k) {
        red[threadIdx.x] = v[k];
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[(size_t)q * kSwFeatures + k] = (float)red[0];
        __syncthreads();
    }
}

}  // namespace

extern "C" int dem_rollout_sweep_features(int32_t dtype, int32_t n_rollouts, int32_t horizon, const void* eta0,
                                          const void* eta_hist, int32_t n, const void* positions, const void* radii,
                                          const void* masses, int32_t n_bonds, const int32_t* bond_i,
                                          const int32_t* bond_j, double half_len, double half_beam, double dt,
                                          float* out, void* stream) {
    if ((dtype != DEM_F32 && dtype != DEM_F64) || n_rollouts < 1 || horizon < 1 || horizon > kSwMaxHorizon)
        return DEM_ERR_INVALID;
    if (n < 0 || n > kSwMaxElements || n_bonds < 0 || !(dt > 0.0) || !(half_len >= 0.0) || !(half_beam >= 0.0))
        return DEM_ERR_INVALID;
    if (!eta0 || !eta_hist || !out || (n > 0 && (!positions || !radii || !masses)) ||
        (n_bonds > 0 && (!bond_i || !bond_j)))
        return DEM_ERR_INVALID;
    SwArgs c{};
    c.Q = n_rollouts;
    c.H = horizon;
    c.n = n;
    c.nb = n_bonds;
    c.hl = (float)half_len;
    c.hw = (float)half_beam;
    c.inv_dt = (float)(1.0 / dt);
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == DEM_F32)
        sweep_kernel<float><<<n_rollouts, kSwThreads, 0, st>>>(c, (const float*)eta0, (const float*)eta_hist,
                                                                (const float*)positions, (const float*)radii,
                                                                (const float*)masses, bond_i, bond_j, out);
    else
        sweep_kernel<double><<<n_rollouts, kSwThreads, 0, st>>>(c, (const double*)eta0, (const double*)eta_hist,
                                                                 (const double*)positions, (const double*)radii,
                                                                 (const double*)masses, bond_i, bond_j, out);
    return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}
