// dem_kernels.cuh — device code of the DPDEM frame step for sm_100a.
//
// One templated kernel (T = float or double) runs the phases of one or more
// frames.  Launched cooperatively with one CTA per resident slot, it runs every
// phase of every frame with bounded grid barriers in between (persistent mode);
// launched once per phase it needs no barrier (phased mode).  Both modes
// execute the same device functions, so they give identical results.
//
// Phases of a frame (reference: medea_ice_ship/jax_simulation.py:397-699)
//   P_CONTACT  ship contact (jax_geometry.py:515-594), contact force, side push,
//              submergence + buoyancy (jax_simulation.py:431-496), floe
//              collision flags, crack-front flags, grid insert for the
//              neighbour list, per-chunk partial sums for the thrust cap
//   P_REDUCE   fixed-order reduction of the partials -> thrust scale, reaction
//              on the ship, vessel step (jax_vessel_dynamics.py:246-348),
//              floe activation and DPDEM eligibility (jax_simulation.py:498-524),
//              neighbour-list build
//   per substep s (jax_simulation.py:363-395, 527-532):
//     P_INSERT / P_NBR   neighbour-list rebuild (skipped while the Verlet skin holds)
//     P_FORCE   fused bond forces + ice-ice contact + drag + rotational drag +
//               semi-implicit integration, one thread per element, gather form
//               (no atomics: each element sums its own bond and contact terms in
//               the reference's scatter order)
//   P_FRACTURE crack front, DPDEM damage, collision breaks (jax_simulation.py:534-653)
//              and history rows
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dem_b200.h"
#include "dem_math.cuh"

namespace dem {

constexpr int kThreads = 256;          // threads per CTA (chunk size of the fixed-order sums)
constexpr int kMaxNbLocal = 64;        // upper bound of DemParams.max_neighbors
constexpr int kMaxV = 32;              // upper bound of max_v (padded vertices per element)
constexpr int kMaxHull = 256;          // upper bound of hull outline points
constexpr int kMaxEdgeSamples = 16;
constexpr unsigned long long kBarrierLimitNs = 2000000000ull;  // 2 s per barrier wait

template <typename T>
struct IcePtrs {
    T *pos, *vel, *rot, *avel, *sub;
    uint8_t* intact;
    T *dmg, *dm0, *dmmax, *ds;
    uint8_t *active, *elig;
};

template <typename T>
struct ShipPtrs {
    T *eta, *nu, *na, *ei;
};

template <typename T>
struct KArgs {
    DemParams P;
    int n, V, nb, nf, S, K, k_sub, nchunks;
    int n_buckets, bucket_cap, max_nb, mode;
    T k_n, k_s, min_bstr, cell, skin, hull_r;
    T t_samp[kMaxEdgeSamples];
    // static data (caller-owned)
    const T* polys;
    const uint8_t* pmask;
    const T *mass, *inertia, *radii, *areas, *thick, *rest, *bstr, *sbar, *hull;
    const int *bi, *bj, *floe_of;
    // derived at create
    const int* boff;    // (n+1) CSR offsets of per-element bond slots
    const int2* bslot;  // (2 nb) {bond | role<<31, partner}; role 0: element is bond_i
    const T* bstiff;    // (nb) E * mean(h) * factor
    const T* vert_r;    // (n) max local vertex radius, rounded up
    // scratch
    int* bcnt;          // (n_buckets) grid-hash bucket fill
    int* bitems;        // (n_buckets * bucket_cap)
    int2* ecell;        // (n) grid cell of each element at the last build
    int* ncnt;          // (n) neighbour count
    int* nbr;           // (max_nb * n) neighbour lists, slot-major
    T* pos_ref;         // (n,2) positions at the last build
    T* soi;             // (n,2) ship force on ice (with buoyancy), constant over substeps
    T* fraw;            // (n) contact force magnitude before the thrust cap
    uint8_t* crack;     // (n) element touches a broken bond
    int* fcoll;         // (nf) floe touched by the ship this frame
    unsigned long long* fmax;  // (nf) max force magnitude per floe (ordered bits)
    double* part;       // (nchunks * 3) per-chunk sums: soi_x, soi_y, moment
    unsigned* gdisp;    // (k_sub + 2) max squared displacement since the last build, per substep
    T *sp_pos[2], *sp_vel[2], *sp_rot[2], *sp_avel[2];  // substep ping-pong
    // call arguments
    IcePtrs<T> in, out, tmp;
    ShipPtrs<T> ship_in, ship_out, ship_tmp[2];
    const T* setpoints;   // (K,6)
    const T* vw;          // (K,n,2)
    const T* vws;         // (K,2) or null
    const uint8_t* elig0; // dpdem_eligible argument of frame 0
    T *d_pen, *d_fmag, *d_F, *d_J;
    T *h_pos, *h_rot, *h_eta, *h_sub, *h_J, *h_F;
    uint8_t* h_intact;
    unsigned* bar;        // [count, generation]
    int* status;
    long long* stats;     // [rebuilds, max_nb_count, max_bucket_count]
};

// ─── per-frame pointer bundle ───────────────────────────────────────────────
template <typename T>
struct Frame {
    int f;
    IcePtrs<T> src, dst;
    ShipPtrs<T> ship_src, ship_dst;
    const uint8_t* elig_in;
    const T* vw;
    T sp[6];
    T vws[2];
};

template <typename T>
__device__ __forceinline__ Frame<T> make_frame(const KArgs<T>& a, int f) {
    Frame<T> F;
    F.f = f;
    const int K = a.K;
    F.dst = (((K - 1 - f) & 1) == 0) ? a.out : a.tmp;
    F.src = (f == 0) ? a.in : ((((K - f) & 1) == 0) ? a.out : a.tmp);
    F.ship_dst = (f == K - 1) ? a.ship_out : a.ship_tmp[f & 1];
    F.ship_src = (f == 0) ? a.ship_in : a.ship_tmp[(f - 1) & 1];
    F.elig_in = (f == 0) ? a.elig0 : F.src.elig;
    F.vw = a.vw + (size_t)f * a.n * 2;
    for (int i = 0; i < 6; ++i) F.sp[i] = a.setpoints[f * 6 + i];
    F.vws[0] = a.vws ? a.vws[f * 2 + 0] : T(0);
    F.vws[1] = a.vws ? a.vws[f * 2 + 1] : T(0);
    return F;
}

// ─── grid barrier (bounded) ──────────────────────────────────────────────────
// Returns false (and records DEM_ERR_TIMEOUT) if the wait exceeds its limit or
// another CTA already recorded a timeout; callers then return.
template <typename T>
__device__ bool grid_barrier(const KArgs<T>& a) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned* count = a.bar;
        unsigned* gen = a.bar + 1;
        unsigned g = ld_acquire_u32(gen);
        __threadfence();
        unsigned arrived = atomicAdd(count, 1u) + 1u;
        int ok = 1;
        if (arrived == gridDim.x) {
            atomicExch(count, 0u);
            __threadfence();
            st_release_u32(gen, g + 1u);
        } else {
            unsigned long long t0 = globaltimer_ns();
            while (ld_acquire_u32(gen) == g) {
                __nanosleep(40);
                if (globaltimer_ns() - t0 > kBarrierLimitNs) {
                    atomicMax(a.status, DEM_ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (*((volatile int*)a.status) == DEM_ERR_TIMEOUT) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ─── grid hash ──────────────────────────────────────────────────────────────
template <typename T>
__device__ __forceinline__ int2 cell_of(const KArgs<T>& a, T x, T y) {
    const double lim = 1073741823.0;  // keep cell indices inside int range
    double cx = fmin(fmax(floor((double)x / (double)a.cell), -lim), lim);
    double cy = fmin(fmax(floor((double)y / (double)a.cell), -lim), lim);
    return make_int2((int)cx, (int)cy);
}
__device__ __forceinline__ int bucket_of(int2 c, int n_buckets) {
    unsigned h = (unsigned)c.x * 73856093u ^ (unsigned)c.y * 19349663u;
    return (int)(h & (unsigned)(n_buckets - 1));
}

// insert element e (position p) into the grid; record its cell and reference position
template <typename T>
__device__ __forceinline__ void grid_insert(const KArgs<T>& a, int e, T px, T py) {
    a.pos_ref[2 * e] = px;
    a.pos_ref[2 * e + 1] = py;
    if (!(jfinite(px) && jfinite(py))) {
        a.ecell[e] = make_int2(INT_MIN, INT_MIN);
        return;
    }
    int2 c = cell_of(a, px, py);
    a.ecell[e] = c;
    int b = bucket_of(c, a.n_buckets);
    int slot = atomicAdd(&a.bcnt[b], 1);
    if (slot < a.bucket_cap) {
        a.bitems[(size_t)b * a.bucket_cap + slot] = e;
    } else {
        atomicMax(a.status, DEM_ERR_CAPACITY);
    }
    if (slot + 1 > a.bucket_cap / 2) atomicMax((unsigned long long*)&a.stats[2], (unsigned long long)(slot + 1));
}

// Build element e's candidate list: every element within r_e + r_o + skin at the
// positions of the last insert, sorted so that indices above e come first
// (ascending), then indices below e (ascending) — the order in which the
// reference's scatter-adds reach e (pairs (e, j>e) through pair_i, then pairs
// (i<e, e) through pair_j; jax_simulation.py:152-162).
template <typename T>
__device__ void build_neighbors(const KArgs<T>& a, int e) {
    T px = a.pos_ref[2 * e], py = a.pos_ref[2 * e + 1];
    int2 c = a.ecell[e];
    int cnt = 0;
    int loc[kMaxNbLocal];
    if (c.x != INT_MIN) {
        const T re = a.radii[e];
        for (int dy = -1; dy <= 1; ++dy) {
            for (int dx = -1; dx <= 1; ++dx) {
                int2 cc = make_int2(c.x + dx, c.y + dy);
                int b = bucket_of(cc, a.n_buckets);
                int m = min(a.bcnt[b], a.bucket_cap);
                for (int k = 0; k < m; ++k) {
                    int o = a.bitems[(size_t)b * a.bucket_cap + k];
                    if (o == e) continue;
                    int2 oc = a.ecell[o];
                    if (oc.x != cc.x || oc.y != cc.y) continue;  // hash collision
                    T ox = a.pos_ref[2 * o] - px, oy = a.pos_ref[2 * o + 1] - py;
                    double d2 = (double)ox * ox + (double)oy * oy;
                    double lim = ((double)re + (double)a.radii[o] + (double)a.skin) * (1.0 + 1e-5) + 1e-6;
                    if (d2 < lim * lim) {
                        if (cnt < a.max_nb) loc[cnt] = o;
                        ++cnt;
                    }
                }
            }
        }
    }
    if (cnt > a.max_nb) {
        atomicMax(a.status, DEM_ERR_CAPACITY);
    }
    {
        unsigned am = __activemask();
        int wmax = __reduce_max_sync(am, cnt);
        if ((threadIdx.x & 31) == (__ffs(am) - 1) && wmax > 0)
            atomicMax((unsigned long long*)&a.stats[1], (unsigned long long)wmax);
    }
    int m = min(cnt, a.max_nb);
    // insertion sort (lists are short)
    for (int i = 1; i < m; ++i) {
        int v = loc[i];
        int j = i - 1;
        while (j >= 0 && loc[j] > v) {
            loc[j + 1] = loc[j];
            --j;
        }
        loc[j + 1] = v;
    }
    int split = 0;
    while (split < m && loc[split] < e) ++split;
    int w = 0;
    for (int i = split; i < m; ++i) a.nbr[(size_t)(w++) * a.n + e] = loc[i];
    for (int i = 0; i < split; ++i) a.nbr[(size_t)(w++) * a.n + e] = loc[i];
    a.ncnt[e] = m;
}

// ─── ship contact (jax_geometry.py) ─────────────────────────────────────────
// Analytic tapered hull test of one point (jax_geometry.py:42-134).
template <typename T>
struct HullPose {
    T sx, sy, c_neg, s_neg, c_h, s_h, hl, hb, hb005;
};

template <typename T>
__device__ __forceinline__ void hull_point(const HullPose<T>& H, T px, T py, T& pen, T& nx, T& ny) {
    const T bts = T(0.6);
    const T one_m_bts = T(1.0 - 0.6);
    T dx = px - H.sx;
    T dy = py - H.sy;
    T rel_x = H.c_neg * dx - H.s_neg * dy;
    T rel_y = H.s_neg * dx + H.c_neg * dy;
    T x_rel = rel_x / H.hl;
    bool in_bow = x_rel < -bts;
    T t_bow = jclip((-x_rel - bts) / one_m_bts, T(0), T(1));
    T hb_bow = H.hb * (T(1) - T(0.9) * jpow(t_bow, T(1.5)));
    hb_bow = jmax(hb_bow, H.hb005);
    T hb_loc = in_bow ? hb_bow : H.hb;
    T arel_y = fabs(rel_y);
    bool inside = (rel_x >= -H.hl) && (rel_x <= H.hl) && (arel_y <= hb_loc);
    if (!inside) {
        pen = T(0);
        nx = T(0);
        ny = T(0);
        return;
    }
    T d_bow = rel_x + H.hl;
    T d_side = hb_loc - arel_y;
    T nxb, nyb, praw;
    if (in_bow) {
        T ang = T(0.3) + T(0.5) * t_bow;
        nxb = -jcos(ang);
        nyb = jsign(rel_y) * jsin(ang);
        praw = jmin(d_bow, d_side) + T(0.5);
    } else {
        bool side = d_side <= d_bow;
        nxb = side ? T(0) : T(-1);
        nyb = side ? jsign(rel_y) : T(0);
        praw = side ? d_side : d_bow;
    }
    nx = H.c_h * nxb - H.s_h * nyb;
    ny = H.s_h * nxb + H.c_h * nyb;
    pen = jmax(praw, T(0));
}

// Per-element maximum-penetration contact: pass 1 (ice vertices + edge samples
// vs the analytic hull), pass 2 (hull outline points inside the ice polygon),
// element-wise max (jax_geometry.py:515-594).  hullw: hull outline in world frame.
template <typename T>
__device__ void element_contact(const KArgs<T>& a, int e, const HullPose<T>& H, const T* hullw,
                                T px, T py, T rot, T& pen_o, T& nx_o, T& ny_o) {
    const int V = a.V;
    const int E = a.P.n_edge_samples;
    T c, s;
    jsincos(rot, &s, &c);
    T wx[kMaxV], wy[kMaxV];
    bool mk[kMaxV];
    const T* lp = a.polys + (size_t)e * V * 2;
    for (int k = 0; k < V; ++k) {
        T lx = lp[2 * k], ly = lp[2 * k + 1];
        wx[k] = c * lx - s * ly + px;
        wy[k] = s * lx + c * ly + py;
        mk[k] = a.pmask[(size_t)e * V + k] != 0;
    }
    // pass 1: points ordered vertex k, then its E edge samples (jax_geometry.py:190-211)
    T best1 = T(0), bnx1 = T(0), bny1 = T(0);
    bool first = true;
    for (int k = 0; k < V; ++k) {
        int k1 = (k + 1 == V) ? 0 : k + 1;
        for (int j = 0; j <= E; ++j) {
            T qx, qy;
            if (j == 0) {
                qx = wx[k];
                qy = wy[k];
            } else {
                T t = a.t_samp[j - 1];
                T omt = T(1) - t;
                qx = wx[k] * omt + wx[k1] * t;
                qy = wy[k] * omt + wy[k1] * t;
            }
            T p, nx, ny;
            hull_point(H, qx, qy, p, nx, ny);
            if (!mk[k]) p = T(0);
            // argmax, first index wins
            if (first || p > best1) {
                best1 = p;
                bnx1 = nx;
                bny1 = ny;
                first = false;
            }
        }
    }
    // pass 2 (jax_geometry.py:300-510)
    T best2 = T(0), bnx2 = T(0), bny2 = T(0);
    {
        T mx[kMaxV], my[kMaxV], mc[kMaxV];
        for (int k = 0; k < V; ++k) {
            mx[k] = mk[k] ? wx[k] : T(0);
            my[k] = mk[k] ? wy[k] : T(0);
            mc[k] = mk[k] ? T(1) : T(0);
        }
        T n_real = jmax(np_pairwise_sum(mc, V), T(1));
        T cxc = np_pairwise_sum(mx, V) / n_real;
        T cyc = np_pairwise_sum(my, V) / n_real;
        T enx[kMaxV], eny[kMaxV];
        for (int k = 0; k < V; ++k) {
            int k1 = (k + 1 == V) ? 0 : k + 1;
            T ex = wx[k1] - wx[k], ey = wy[k1] - wy[k];
            T nxe = ey, nye = -ex;
            T nlen = jsqrt(nxe * nxe + nye * nye + T(1e-20));
            nxe = nxe / nlen;
            nye = nye / nlen;
            T midx = (wx[k] + wx[k1]) / T(2), midy = (wy[k] + wy[k1]) / T(2);
            T dotc = (midx - cxc) * nxe + (midy - cyc) * nye;
            if (dotc < T(0)) {
                nxe = -nxe;
                nye = -nye;
            }
            enx[k] = nxe;
            eny[k] = nye;
        }
        bool firsts = true;
        for (int si = 0; si < a.S; ++si) {
            T hx = hullw[2 * si], hy = hullw[2 * si + 1];
            int crossings = 0;
            T dmin = T(0);
            int kbest = 0;
            for (int k = 0; k < V; ++k) {
                int k1 = (k + 1 == V) ? 0 : k + 1;
                T xi = wx[k], yi = wy[k], xj = wx[k1], yj = wy[k1];
                bool cond_y = (yi > hy) != (yj > hy);
                T x_int = (xj - xi) * (hy - yi) / (yj - yi + T(1e-10)) + xi;
                if (cond_y && (hx < x_int)) ++crossings;
                T vx = xj - xi, vy = yj - yi;
                T wx_ = hx - xi, wy_ = hy - yi;
                T c1 = wx_ * vx + wy_ * vy;
                T c2 = vx * vx + vy * vy + T(1e-20);
                T t = jclip(c1 / c2, T(0), T(1));
                T qx = xi + t * vx, qy = yi + t * vy;
                T ddx = hx - qx, ddy = hy - qy;
                T d = jsqrt(ddx * ddx + ddy * ddy + T(1e-20));
                if (k == 0 || d < dmin) {  // argmin, first index wins
                    dmin = d;
                    kbest = k;
                }
            }
            bool inside = (crossings % 2) == 1;
            T p = inside ? dmin : T(0);
            T nx = inside ? enx[kbest] : T(0);
            T ny = inside ? eny[kbest] : T(0);
            if (firsts || p > best2) {  // argmax over hull points
                best2 = p;
                bnx2 = nx;
                bny2 = ny;
                firsts = false;
            }
        }
        if (!(best2 > T(0))) {
            best2 = T(0);
            bnx2 = T(0);
            bny2 = T(0);
        }
    }
    if (best2 > best1) {
        pen_o = best2;
        nx_o = bnx2;
        ny_o = bny2;
    } else {
        pen_o = best1;
        nx_o = bnx1;
        ny_o = bny1;
    }
}

// ─── fixed-order block sum (deterministic, independent of the grid size) ────
template <int N>
__device__ __forceinline__ void block_sum3(double v0, double v1, double v2, double* out3) {
    __shared__ double sh[3][N];
    sh[0][threadIdx.x] = v0;
    sh[1][threadIdx.x] = v1;
    sh[2][threadIdx.x] = v2;
    __syncthreads();
    for (int w = N / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
            sh[2][threadIdx.x] += sh[2][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out3[0] = sh[0][0];
        out3[1] = sh[1][0];
        out3[2] = sh[2][0];
    }
    __syncthreads();
}

// ─── P_CONTACT ──────────────────────────────────────────────────────────────
template <typename T>
__device__ void phase_contact(const KArgs<T>& a, const Frame<T>& F, T* hullw_sh) {
    const DemParams& P = a.P;
    const T sx = F.ship_src.eta[0], sy = F.ship_src.eta[1], spsi = F.ship_src.eta[2];
    HullPose<T> H;
    H.sx = sx;
    H.sy = sy;
    jsincos(-spsi, &H.s_neg, &H.c_neg);
    jsincos(spsi, &H.s_h, &H.c_h);
    H.hl = T(P.half_len);
    H.hb = T(P.half_beam);
    H.hb005 = T(P.half_beam * 0.05);
    // hull outline in world frame: ship_hull_local @ R.T + [x, y] (jax_geometry.py:568-572)
    for (int i = threadIdx.x; i < a.S; i += blockDim.x) {
        T lx = a.hull[2 * i], ly = a.hull[2 * i + 1];
        hullw_sh[2 * i] = lx * H.c_h + ly * (-H.s_h) + sx;
        hullw_sh[2 * i + 1] = lx * H.s_h + ly * H.c_h + sy;
    }
    __syncthreads();
    const T reach_base = a.hull_r;
    const T wcf = T(P.w_contact_radius_factor), wcap = T(P.w_contact_cap);
    const T flex = T(P.flexural_strength_base);
    const T pcr = T(P.pen_crit_ref), pct = T(P.pen_crit_thickness_ref);
    const T spf = T(P.side_push_factor);
    const T srate = T(P.submergence_rate), scap = T(P.submergence_pen_cap);
    const T inv_rise = T(1.0 / P.rise_time_const);
    const T dt = T(P.dt);
    const T rho_g = T(P.water_density * 9.81);
    for (int chunk = blockIdx.x; chunk < a.nchunks; chunk += gridDim.x) {
        int e = chunk * kThreads + threadIdx.x;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        if (e < a.n) {
            typename vec2_of<T>::type p = ld2(F.src.pos, e);
            T rot = F.src.rot[e];
            T pen = T(0), nx = T(0), ny = T(0);
            T ddx = p.x - sx, ddy = p.y - sy;
            double dist = sqrt((double)ddx * ddx + (double)ddy * ddy);
            if (!(dist > (double)reach_base + (double)a.vert_r[e] + 1e-3)) {
                element_contact(a, e, H, hullw_sh, p.x, p.y, rot, pen, nx, ny);
            }
            bool has = pen > T(0);
            T h = a.thick[e];
            T w_contact = jmin(wcf * a.radii[e], wcap);
            T sigma_f = flex * jsqrt(h);
            T f_break = sigma_f * w_contact * (h * h);
            T pen_crit = pcr * (h / pct);
            T fm = has ? f_break * jmin(pen / jmax(pen_crit, T(1e-10)), T(1)) : T(0);
            T so_x = fm * nx;
            T so_y = fm * ny;
            T rel_y = p.y - sy;
            so_y = so_y + spf * fm * jsign(rel_y);
            // moment on the ship uses the force before the thrust cap (jax_simulation.py:474-477)
            T rx = p.x - sx, ry = p.y - sy;
            T mom = has ? (rx * (-so_y) - ry * (-so_x)) : T(0);
            s0 = (double)so_x;
            s1 = (double)so_y;
            s2 = (double)mom;
            // submergence and buoyancy (jax_simulation.py:480-496)
            T sub = F.src.sub[e];
            T pen_c = jmin(pen, scap);
            T new_sub = has ? jmin(sub + srate * pen_c * dt, h)
                            : jmax(T(0), sub - inv_rise * sub * dt);
            T z_sub = jmin(new_sub, h);
            T f_buoy = rho_g * a.areas[e] * z_sub;
            if (has) {
                so_x = so_x + f_buoy * nx;
                so_y = so_y + f_buoy * ny;
            }
            st2(a.soi, e, so_x, so_y);
            a.fraw[e] = fm;
            F.dst.sub[e] = new_sub;
            if (a.d_pen) a.d_pen[e] = pen;
            int fl = a.floe_of[e];
            if (has) atomicMax(&a.fcoll[fl], 1);
            if (fm > T(0)) {
                if (sizeof(T) == 4)
                    atomicMax(&a.fmax[fl], (unsigned long long)f2ord((float)fm));
                else
                    atomicMax(&a.fmax[fl], d2ord((double)fm));
            }
            // crack front: element touches a bond that is broken at frame start
            uint8_t ck = 0;
            for (int sl = a.boff[e]; sl < a.boff[e + 1]; ++sl) {
                int b = a.bslot[sl].x & 0x7fffffff;
                if (!F.src.intact[b]) {
                    ck = 1;
                    break;
                }
            }
            a.crack[e] = ck;
            grid_insert(a, e, p.x, p.y);
        }
        double r3[3];
        block_sum3<kThreads>(s0, s1, s2, r3);
        if (threadIdx.x == 0) {
            a.part[3 * chunk + 0] = r3[0];
            a.part[3 * chunk + 1] = r3[1];
            a.part[3 * chunk + 2] = r3[2];
        }
    }
}

// ─── vessel step (jax_vessel_dynamics.py:246-348) ───────────────────────────
template <typename T>
__device__ void ship_step(const DemParams& P, const T* eta, const T* nu, const T* na, const T* ei,
                          const T* sp, const T* spn, const T* tau_ice, const T* vws, T* eta_o,
                          T* nu_o, T* na_o, T* ei_o) {
    const T pi = T(M_PI), two_pi = T(2.0 * M_PI);
    const T dtf = T(P.dt);
    T c = jcos(eta[2]), s = jsin(eta[2]);
    // R = [[c,-s,0],[s,c,0],[0,0,1]]; R^T v with the full 3x3 product of the
    // reference (the zero terms add exactly)
    T nu_c[3];
    nu_c[0] = (c * vws[0] + s * vws[1]) + T(0) * T(0);
    nu_c[1] = ((-s) * vws[0] + c * vws[1]) + T(0) * T(0);
    nu_c[2] = (T(0) * vws[0] + T(0) * vws[1]) + T(1) * T(0);
    T tib[3];
    tib[0] = (c * tau_ice[0] + s * tau_ice[1]) + T(0) * tau_ice[2];
    tib[1] = ((-s) * tau_ice[0] + c * tau_ice[1]) + T(0) * tau_ice[2];
    tib[2] = (T(0) * tau_ice[0] + T(0) * tau_ice[1]) + T(1) * tau_ice[2];
    T dpsi_d = pymod(spn[2] - sp[2] + pi, two_pi) - pi;
    T v_d[3] = {(spn[0] - sp[0]) / dtf, (spn[1] - sp[1]) / dtf, dpsi_d / dtf};
    T nu_d[3];
    nu_d[0] = (c * v_d[0] + s * v_d[1]) + T(0) * v_d[2];
    nu_d[1] = ((-s) * v_d[0] + c * v_d[1]) + T(0) * v_d[2];
    nu_d[2] = (T(0) * v_d[0] + T(0) * v_d[1]) + T(1) * v_d[2];
    T tau_ff[3];
    {
        T DKt[9];
        for (int i = 0; i < 9; ++i) DKt[i] = T(P.D3[i]) + T(P.Kd[i]);
        for (int i = 0; i < 3; ++i)
            tau_ff[i] = (DKt[3 * i] * nu_d[0] + DKt[3 * i + 1] * nu_d[1]) + DKt[3 * i + 2] * nu_d[2];
    }
    // dp_control (jax_vessel_dynamics.py:127-184): tau = -(R^T Kp) e - Kd nu - (R^T Ki) e_int
    T e[3];
    e[0] = eta[0] - sp[0];
    e[1] = eta[1] - sp[1];
    e[2] = pymod(eta[2] - sp[2] + pi, two_pi) - pi;
    T Rt[9] = {c, s, T(0), -s, c, T(0), T(0), T(0), T(1)};
    T RKp[9], RKi[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            RKp[3 * i + j] = (Rt[3 * i] * T(P.Kp[j]) + Rt[3 * i + 1] * T(P.Kp[3 + j])) + Rt[3 * i + 2] * T(P.Kp[6 + j]);
            RKi[3 * i + j] = (Rt[3 * i] * T(P.Ki[j]) + Rt[3 * i + 1] * T(P.Ki[3 + j])) + Rt[3 * i + 2] * T(P.Ki[6 + j]);
        }
    T a1[3], a2[3], a3[3];
    for (int i = 0; i < 3; ++i) {
        a1[i] = (RKp[3 * i] * e[0] + RKp[3 * i + 1] * e[1]) + RKp[3 * i + 2] * e[2];
        a2[i] = (T(P.Kd[3 * i]) * nu[0] + T(P.Kd[3 * i + 1]) * nu[1]) + T(P.Kd[3 * i + 2]) * nu[2];
        a3[i] = (RKi[3 * i] * ei[0] + RKi[3 * i + 1] * ei[1]) + RKi[3 * i + 2] * ei[2];
    }
    T tau_c[3];
    for (int i = 0; i < 3; ++i) {
        tau_c[i] = (-a1[i] - a2[i]) - a3[i];
        ei_o[i] = ei[i] + dtf * e[i];
    }
    T tau_act[3];
    if (P.use_auto_icenav) {
        T tc[3] = {tau_c[0] + tau_ff[0], tau_c[1] + tau_ff[1], tau_c[2] + tau_ff[2]};
        T ncmd[6];
        for (int i = 0; i < 6; ++i) {
            T u = (T(P.B_pinv[3 * i]) * tc[0] + T(P.B_pinv[3 * i + 1]) * tc[1]) + T(P.B_pinv[3 * i + 2]) * tc[2];
            T n_ = jsign(u) * jsqrt(fabs(u) + T(1e-12));
            ncmd[i] = jclip(n_, -T(P.n_max[i]), T(P.n_max[i]));
            na_o[i] = na[i] + dtf * (ncmd[i] - na[i]) / T(P.T_n);
        }
        T q[6];
        for (int i = 0; i < 6; ++i) q[i] = fabs(na_o[i]) * na_o[i];
        for (int i = 0; i < 3; ++i) {
            T acc = T(P.B_mat[6 * i]) * q[0];
            for (int j = 1; j < 6; ++j) acc = acc + T(P.B_mat[6 * i + j]) * q[j];
            tau_act[i] = acc;
        }
    } else {
        for (int i = 0; i < 3; ++i) tau_act[i] = tau_c[i] + tau_ff[i];
        for (int i = 0; i < 6; ++i) na_o[i] = na[i];
    }
    T tau_tot[3] = {tau_act[0] + tib[0], tau_act[1] + tib[1], tau_act[2] + tib[2]};
    // ship_euler_step_jax (jax_vessel_dynamics.py:54-84)
    T nu_r[3] = {nu[0] - nu_c[0], nu[1] - nu_c[1], nu[2] - nu_c[2]};
    T dnr[3];
    for (int i = 0; i < 3; ++i) dnr[i] = (T(P.D3[3 * i]) * nu_r[0] + T(P.D3[3 * i + 1]) * nu_r[1]) + T(P.D3[3 * i + 2]) * nu_r[2];
    T rhs[3] = {tau_tot[0] - dnr[0], tau_tot[1] - dnr[1], tau_tot[2] - dnr[2]};
    T nu_new[3];
    for (int i = 0; i < 3; ++i) {
        T nd = (T(P.M3inv[3 * i]) * rhs[0] + T(P.M3inv[3 * i + 1]) * rhs[1]) + T(P.M3inv[3 * i + 2]) * rhs[2];
        nu_new[i] = nu[i] + dtf * nd;
    }
    T vx = c * nu_new[0] - s * nu_new[1];
    T vy = s * nu_new[0] + c * nu_new[1];
    T psi_new = pymod(eta[2] + dtf * nu_new[2] + pi, two_pi) - pi;
    eta_o[0] = eta[0] + dtf * vx;
    eta_o[1] = eta[1] + dtf * vy;
    eta_o[2] = psi_new;
    nu_o[0] = jclip(nu_new[0], -T(P.vc_surge), T(P.vc_surge));
    nu_o[1] = jclip(nu_new[1], -T(P.vc_sway), T(P.vc_sway));
    nu_o[2] = jclip(nu_new[2], -T(P.vc_yaw), T(P.vc_yaw));
}

// ─── P_REDUCE ───────────────────────────────────────────────────────────────
template <typename T>
__device__ void frame_totals(const KArgs<T>& a, double* tot3) {
    // every CTA reduces the partials in the same fixed order
    double v0 = 0.0, v1 = 0.0, v2 = 0.0;
    for (int i = threadIdx.x; i < a.nchunks; i += blockDim.x) {
        v0 += a.part[3 * i];
        v1 += a.part[3 * i + 1];
        v2 += a.part[3 * i + 2];
    }
    block_sum3<kThreads>(v0, v1, v2, tot3);
}

template <typename T>
__device__ __forceinline__ T thrust_scale_of(const KArgs<T>& a, const double* tot3) {
    if (!a.P.has_max_ship_ice_force) return T(1);
    T fx = T(tot3[0]), fy = T(tot3[1]);
    T mag = jsqrt(fx * fx + fy * fy);
    T mx = T(a.P.max_ship_ice_force);
    return (mag > mx) ? mx / jmax(mag, T(1e-6)) : T(1);
}

template <typename T>
__device__ void phase_reduce(const KArgs<T>& a, const Frame<T>& F, T* scale_out) {
    __shared__ double tot3[3];
    double r[3];
    frame_totals(a, r);
    if (threadIdx.x == 0) {
        tot3[0] = r[0];
        tot3[1] = r[1];
        tot3[2] = r[2];
    }
    __syncthreads();
    const T scale = thrust_scale_of(a, tot3);
    *scale_out = scale;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // reaction on the ship (jax_simulation.py:470-478)
        T Fx = -(T(tot3[0]) * scale), Fy = -(T(tot3[1]) * scale), M = T(tot3[2]);
        T tau[3] = {Fx, Fy, M};
        T J = jsqrt(Fx * Fx + Fy * Fy) * T(a.P.dt);
        T sp[3] = {F.sp[0], F.sp[1], F.sp[2]};
        const T* eta = F.ship_src.eta;
        if (a.P.ice_brake_threshold > 0.0) {  // jax_simulation.py:658-669
            T thr = T(a.P.ice_brake_threshold);
            T bf = jclip(thr / jmax(fabs(tau[0]), thr), T(0.1), T(1));
            sp[0] = eta[0] + bf * (F.sp[0] - eta[0]);
            sp[1] = eta[1] + bf * (F.sp[1] - eta[1]);
        }
        T eta_o[3], nu_o[3], na_o[6], ei_o[3];
        ship_step<T>(a.P, eta, F.ship_src.nu, F.ship_src.na, F.ship_src.ei, sp, F.sp + 3, tau, F.vws,
                     eta_o, nu_o, na_o, ei_o);
        for (int i = 0; i < 3; ++i) {
            F.ship_dst.eta[i] = eta_o[i];
            F.ship_dst.nu[i] = nu_o[i];
            F.ship_dst.ei[i] = ei_o[i];
        }
        for (int i = 0; i < 6; ++i) F.ship_dst.na[i] = na_o[i];
        if (a.d_F) {
            a.d_F[0] = Fx;
            a.d_F[1] = Fy;
        }
        if (a.d_J) a.d_J[0] = J;
        if (a.h_eta)
            for (int i = 0; i < 3; ++i) a.h_eta[F.f * 3 + i] = eta_o[i];
        if (a.h_J) a.h_J[F.f] = J;
        if (a.h_F) {
            a.h_F[F.f * 2] = Fx;
            a.h_F[F.f * 2 + 1] = Fy;
        }
    }
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gsz = gridDim.x * blockDim.x;
    // floe eligibility (jax_simulation.py:513-524)
    const T thr = a.min_bstr * T(a.P.effective_strength_collision);
    for (int fl = gtid; fl < a.nf; fl += gsz) {
        uint8_t el = F.elig_in[fl];
        if (a.nb > 0 && a.fcoll[fl]) {
            unsigned long long bits = a.fmax[fl];
            T fmx = (sizeof(T) == 4) ? T(__uint_as_float((unsigned)bits)) : T(__longlong_as_double((long long)bits));
            // max(force * scale) == max(force) * scale: rounding is monotone
            if (fmx * scale > thr) el = 1;
        }
        F.dst.elig[fl] = el;
    }
    // activation, diag force and neighbour lists
    for (int e = gtid; e < a.n; e += gsz) {
        F.dst.active[e] = (F.src.active[e] || a.fcoll[a.floe_of[e]]) ? 1 : 0;
        if (a.d_fmag) a.d_fmag[e] = a.fraw[e] * scale;
        build_neighbors(a, e);
    }
}

// ─── P_INSERT (mid-frame rebuild) ───────────────────────────────────────────
template <typename T>
__device__ void phase_insert(const KArgs<T>& a, const T* pos) {
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gsz = gridDim.x * blockDim.x;
    for (int e = gtid; e < a.n; e += gsz) {
        typename vec2_of<T>::type p = ld2(pos, e);
        grid_insert(a, e, p.x, p.y);
    }
}

template <typename T>
__device__ void phase_nbr(const KArgs<T>& a) {
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gsz = gridDim.x * blockDim.x;
    for (int e = gtid; e < a.n; e += gsz) build_neighbors(a, e);
}

// ─── P_FORCE: one substep (jax_simulation.py:63-268, 363-395) ───────────────
template <typename T>
__device__ void phase_force(const KArgs<T>& a, const Frame<T>& F, int s, bool clear_buckets,
                            unsigned* gdisp_slot) {
    const DemParams& P = a.P;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gsz = gridDim.x * blockDim.x;
    const int k = a.k_sub;
    const T* pin = (s == 0) ? F.src.pos : a.sp_pos[(s - 1) & 1];
    const T* vin = (s == 0) ? F.src.vel : a.sp_vel[(s - 1) & 1];
    const T* rin = (s == 0) ? F.src.rot : a.sp_rot[(s - 1) & 1];
    const T* ain = (s == 0) ? F.src.avel : a.sp_avel[(s - 1) & 1];
    T* pout = (s == k - 1) ? F.dst.pos : a.sp_pos[s & 1];
    T* vout = (s == k - 1) ? F.dst.vel : a.sp_vel[s & 1];
    T* rout = (s == k - 1) ? F.dst.rot : a.sp_rot[s & 1];
    T* aout = (s == k - 1) ? F.dst.avel : a.sp_avel[s & 1];
    const uint8_t* act = F.dst.active;
    const T hf = T(P.hertz_factor), hexp = T(P.hertz_exponent);
    const T mu = T(P.ice_ice_friction), fcap = T(P.friction_cap);
    const T c_drag = T(0.5 * P.water_density * P.c_d_drag);
    const T href = T(P.drag_ref_thickness);
    const T lin = T(P.linear_drag_factor);
    const T c_rot = T(-0.5 * P.drag_coefficient_moment * P.water_density);
    const T dti = T(P.dt_ice);
    const T damp = T(P.angular_damping), alo = T(P.angular_cap_lo), ahi = T(P.angular_cap_hi);
    const T vclip = T(P.velocity_clip), pclip = T(P.position_clip);
    float dmax2 = 0.0f;
    if (clear_buckets)
        for (int b = gtid; b < a.n_buckets; b += gsz) a.bcnt[b] = 0;
    for (int e = gtid; e < a.n; e += gsz) {
        typename vec2_of<T>::type pe = ld2(pin, e);
        typename vec2_of<T>::type ve = ld2(vin, e);
        const bool ae = act[e] != 0;
        // bond forces (jax_simulation.py:63-108): slots with e == bond_i first, then e == bond_j
        T fbx = T(0), fby = T(0), mb = T(0);
        const int s0 = a.boff[e], s1 = a.boff[e + 1];
        for (int sl = s0; sl < s1; ++sl) {
            int2 ent = a.bslot[sl];
            int b = ent.x & 0x7fffffff;
            bool role_j = (ent.x < 0);
            int o = ent.y;
            if (!F.src.intact[b]) continue;
            if ((act[o] != 0) != ae) continue;  // endpoints must share the active state
            typename vec2_of<T>::type po = ld2(pin, o);
            T dx, dy;
            if (!role_j) {
                dx = po.x - pe.x;
                dy = po.y - pe.y;
            } else {
                dx = pe.x - po.x;
                dy = pe.y - po.y;
            }
            T dist = jsqrt(dx * dx + dy * dy);
            T dsafe = jmax(dist, T(1e-10));
            T bx = dx / dsafe, by = dy / dsafe;
            T stretch = dist - a.rest[b];
            T fmag = a.bstiff[b] * stretch * (T(1) - F.src.dmg[b]);
            T fx = bx * fmag, fy = by * fmag;
            T cr = T(0.5) * (dx * fy - dy * fx);
            if (!role_j) {
                fbx += fx;
                fby += fy;
                mb += cr;
            } else {
                fbx += -fx;
                fby += -fy;
                mb += -cr;
            }
        }
        // ice-ice contact (jax_simulation.py:111-164)
        T fix = T(0), fiy = T(0), mi = T(0);
        const T re = a.radii[e];
        const int nc = a.ncnt[e];
        for (int q = 0; q < nc; ++q) {
            int o = a.nbr[(size_t)q * a.n + e];
            typename vec2_of<T>::type po = ld2(pin, o);
            const bool e_is_i = e < o;
            T dx = e_is_i ? po.x - pe.x : pe.x - po.x;
            T dy = e_is_i ? po.y - pe.y : pe.y - po.y;
            T dist = jsqrt(dx * dx + dy * dy);
            T ro = a.radii[o];
            T min_dist = e_is_i ? re + ro : ro + re;
            T overlap = jmax(min_dist - dist, T(0));
            if (!(dist > T(1e-6))) overlap = T(0);
            if (!(overlap > T(0))) continue;  // non-overlapping pairs add exact zeros
            T dsafe = jmax(dist, T(1e-10));
            T ux = dx / dsafe, uy = dy / dsafe;
            T fn = hf * jpow(overlap, hexp);
            T fnx = ux * fn, fny = uy * fn;
            typename vec2_of<T>::type vo = ld2(vin, o);
            T vrx = e_is_i ? vo.x - ve.x : ve.x - vo.x;
            T vry = e_is_i ? vo.y - ve.y : ve.y - vo.y;
            T vdot = vrx * ux + vry * uy;
            T vtx = vrx - vdot * ux, vty = vry - vdot * uy;
            T vtm = jsqrt(vtx * vtx + vty * vty);
            T vts = jmax(vtm, T(1e-10));
            T thx = -vtx / vts, thy = -vty / vts;
            T ftm = jmin(mu * fn, fcap);
            T ftx = T(0), fty = T(0);
            if (vtm > T(1e-6)) {
                ftx = thx * ftm;
                fty = thy * ftm;
            }
            T oix = -fnx - ftx, oiy = -fny - fty;
            T cr = -(dx * oiy - dy * oix);
            if (e_is_i) {
                fix += -fnx + ftx;
                fiy += -fny + fty;
                mi += T(0.5) * cr;
            } else {
                fix += fnx - ftx;
                fiy += fny - fty;
                mi += T(-0.5) * cr;
            }
        }
        // drag (jax_simulation.py:167-192)
        T h = a.thick[e], A = a.areas[e];
        T a_drag = A * (h / href);
        typename vec2_of<T>::type w = ld2(F.vw, e);
        T vrx = ve.x - w.x, vry = ve.y - w.y;
        T vm = jsqrt(vrx * vrx + vry * vry);
        T vms = jmax(vm, T(1e-12));
        T fdx, fdy;
        if (vm > T(1e-6)) {
            T mag = c_drag * a_drag * (vms * vms);
            fdx = (vrx / vms) * mag;
            fdy = (vry / vms) * mag;
        } else {
            T cl = c_drag * a_drag * lin;
            fdx = cl * vrx;
            fdy = cl * vry;
        }
        // rotational drag (jax_simulation.py:195-212)
        T av = ain[e];
        T sub = F.dst.sub[e];
        T a_sub = A * jmin(sub / jmax(h, T(1e-10)), T(1));
        T r3 = jpow(re, T(3));
        T md = c_rot * r3 * av * fabs(av) * a_sub;
        typename vec2_of<T>::type so = ld2(a.soi, e);
        T Fx = ((fbx + fix) - fdx) + so.x;
        T Fy = ((fby + fiy) - fdy) + so.y;
        T Mz = (mb + mi) + md;
        // semi-implicit Euler (jax_simulation.py:215-268)
        T m = a.mass[e];
        T nvx = jclip(ve.x + (Fx / m) * dti, -vclip, vclip);
        T nvy = jclip(ve.y + (Fy / m) * dti, -vclip, vclip);
        T npx = pe.x + nvx * dti, npy = pe.y + nvy * dti;
        T alpha = Mz / a.inertia[e];
        T nav = jclip(av * damp + alpha * dti, alo, ahi);
        T rot = rin[e];
        T nrot = rot + nav * dti;
        if (!jfinite(nvx)) nvx = T(0);
        if (!jfinite(nvy)) nvy = T(0);
        if (!jfinite(npx)) npx = pe.x;
        if (!jfinite(npy)) npy = pe.y;
        npx = jclip(npx, -pclip, pclip);
        npy = jclip(npy, -pclip, pclip);
        if (!ae) {
            nvx = ve.x;
            nvy = ve.y;
            npx = pe.x;
            npy = pe.y;
            nav = av;
            nrot = rot;
        }
        st2(pout, e, npx, npy);
        st2(vout, e, nvx, nvy);
        rout[e] = nrot;
        aout[e] = nav;
        // displacement since the last neighbour-list build
        T ddx = npx - a.pos_ref[2 * e], ddy = npy - a.pos_ref[2 * e + 1];
        float d2 = (float)((double)ddx * ddx + (double)ddy * ddy);
        if (!(d2 <= 3.0e38f)) d2 = 3.0e38f;
        dmax2 = fmaxf(dmax2, d2);
    }
    // CTA max, one atomic per CTA
    __shared__ float shm[kThreads / 32];
    for (int off = 16; off > 0; off >>= 1) dmax2 = fmaxf(dmax2, __shfl_xor_sync(0xffffffffu, dmax2, off));
    if ((threadIdx.x & 31) == 0) shm[threadIdx.x >> 5] = dmax2;
    __syncthreads();
    if (threadIdx.x == 0) {
        float m = shm[0];
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i) m = fmaxf(m, shm[i]);
        if (m > 0.0f) atomicMax(gdisp_slot, f2ord(m));
    }
    __syncthreads();
}

// ─── bond damage (jax_bond_fracture.py:133-208) ─────────────────────────────
template <typename T>
__device__ void bond_damage(const DemParams& P, T delta_n, T delta_s, T sigma_n, T sigma_t, T sigma_bar,
                            T cur_d, T cur_max, T cur_0, bool intact, T& nd, T& nmax, T& n0, bool& nint) {
    const T SC = T(1e12);
    delta_n = jclip(delta_n, T(-1e3), T(1e3));
    delta_s = jclip(delta_s, T(-1e3), T(1e3));
    sigma_bar = jclip(sigma_bar, T(1e-10), SC);
    // equivalent deformation (:69-77)
    T dn = jclip(delta_n, T(-1e3), T(1e3));
    T dsa = jclip(fabs(delta_s), T(0), T(1e3));
    T dnp = jmax(dn, T(0));
    T delta_m = jsqrt(jclip(dnp * dnp + dsa * dsa + T(1e-20), T(0), T(1e12)));
    nmax = jmax(cur_max, delta_m);
    // Mohr-Coulomb shear strength (:60-66)
    T tau_bar = jmax(T(P.bond_cohesion) - T(P.bond_internal_friction) * sigma_n, T(1e-6));
    // strength criterion (:35-57)
    T s_pos = jmax(jclip(sigma_n, -SC, SC), T(0));
    T tau = jclip(sigma_t, -SC, SC);
    T sb = jmax(jclip(sigma_bar, T(1e-10), SC), T(1e-10));
    T tb = jmax(jclip(tau_bar, T(1e-10), SC), T(1e-10));
    T q1 = s_pos / sb, q2 = tau / tb;
    T crit = jclip(q1 * q1 + q2 * q2, T(0), T(1e10));
    bool initiating = (crit >= T(1)) && (cur_0 <= T(0)) && (delta_m > T(1e-5));
    n0 = initiating ? delta_m : cur_0;
    // fracture-energy ratio and Benzeggagh-Kenane energy (:103-121)
    T dnp2 = jmax(delta_n, T(0));
    T g_ratio = (delta_s * delta_s) / (dnp2 * dnp2 + T(1e-10));
    T g_I = T(1) / (T(1) + g_ratio + T(1e-10));
    T g_II = g_ratio / (T(1) + g_ratio + T(1e-10));
    T g_tot = g_I + g_II + T(1e-10);
    T ratio = g_II / g_tot;
    T g_c = T(P.bond_G_c_I) + T(P.bond_G_c_II - P.bond_G_c_I) * jpow(ratio, T(P.bond_eta_bk));
    T snc = jclip(sigma_n, -SC, SC), stc = jclip(sigma_t, -SC, SC);
    T snp = jmax(snc, T(0));
    T sm0_raw = jsqrt(jclip(snp * snp + stc * stc + T(1e-20), T(0), T(1e24)));
    T sm0 = jmax(sm0_raw, T(1e-10));
    T dm_f = (T(2) * g_c) / (fabs(sm0) + T(1e-10));
    bool meaningful = sm0_raw >= T(1e4);
    bool has_dmg = (n0 > T(0)) && meaningful;
    // damage variable (:80-100)
    T comp = cur_d;
    if (has_dmg) {
        T d0c = jclip(n0, T(0), T(1e6));
        T dfc = jmax(jclip(dm_f, T(1e-10), T(1e6)), T(1e-10));
        T dmaxc = jmax(jclip(nmax, T(0), T(1e6)), d0c + T(1e-10));
        T denom = jmax(dmaxc * (dfc - d0c + T(1e-10)), T(1e-20));
        comp = jclip(dfc * (dmaxc - d0c) / denom, T(0), T(1));
    }
    T d = meaningful ? jmax(comp, cur_d) : cur_d;
    nd = jmin(d, cur_d + T(0.15));
    nint = intact && (nd < T(1));
}

// ─── P_FRACTURE (jax_simulation.py:534-653) + history ───────────────────────
template <typename T>
__device__ void phase_fracture(const KArgs<T>& a, const Frame<T>& F, T scale) {
    const DemParams& P = a.P;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gsz = gridDim.x * blockDim.x;
    const T mft = T(P.max_fracture_thickness);
    const T esc = T(P.effective_strength_collision);
    const T dti = T(P.dt_ice);
    const T kn = a.k_n, ks = a.k_s;
    for (int b = gtid; b < a.nb; b += gsz) {
        int i = a.bi[b], j = a.bj[b];
        typename vec2_of<T>::type pi_ = ld2(F.dst.pos, i), pj = ld2(F.dst.pos, j);
        T dx = pj.x - pi_.x, dy = pj.y - pi_.y;
        T dist = jsqrt(dx * dx + dy * dy);
        T dsafe = jmax(dist, T(1e-10));
        T bx = dx / dsafe, by = dy / dsafe;
        bool both_act = F.dst.active[i] && F.dst.active[j];
        bool floe_ok = F.dst.elig[a.floe_of[i]] && F.dst.elig[a.floe_of[j]];
        bool breakable = (a.thick[i] <= mft) && (a.thick[j] <= mft);
        T fmi = a.fraw[i] * scale, fmj = a.fraw[j] * scale;
        bool near = (fmi > T(0)) || (fmj > T(0));
        bool at_crack = a.crack[i] || a.crack[j];
        bool dpdem_ok = both_act && floe_ok && (near || at_crack) && breakable;
        typename vec2_of<T>::type vi = ld2(F.dst.vel, i), vj = ld2(F.dst.vel, j);
        T vrx = vj.x - vi.x, vry = vj.y - vi.y;
        T vn = vrx * bx + vry * by;
        T vtx = vrx - vn * bx, vty = vry - vn * by;
        T ds_incr = jsqrt(vtx * vtx + vty * vty) * dti;
        bool ds_gate = near && both_act && floe_ok && breakable;
        T new_ds = F.src.ds[b] + (ds_gate ? ds_incr : T(0));
        T rest = a.rest[b];
        T L0 = jmax(rest, T(1e-10));
        T delta_n = dist - rest;
        T dn_d = near ? delta_n : T(0);
        T cur_d = F.src.dmg[b];
        T sn = (kn * (dn_d / L0)) * (T(1) - cur_d);
        T st = (ks * (new_ds / L0)) * (T(1) - cur_d);
        bool intact = F.src.intact[b] != 0;
        T nd, nmax, n0;
        bool nint;
        bond_damage<T>(P, delta_n, new_ds, sn, st, a.sbar[b], cur_d, F.src.dmmax[b], F.src.dm0[b], intact,
                       nd, nmax, n0, nint);
        T od = cur_d, omax = F.src.dmmax[b], o0 = F.src.dm0[b];
        if (dpdem_ok) {
            od = nd;
            omax = nmax;
            o0 = n0;
        }
        bool fin = (dpdem_ok && breakable) ? nint : intact;
        // direct collision breaking (jax_simulation.py:629-637)
        bool coll_on = (fmi > T(0)) || (fmj > T(0));
        T coll_f = jmax(fmi, fmj);
        bool brk = intact && coll_on && (coll_f > a.bstr[b] * esc) && breakable;
        fin = fin && !brk;
        F.dst.dmg[b] = od;
        F.dst.dmmax[b] = omax;
        F.dst.dm0[b] = o0;
        F.dst.ds[b] = new_ds;
        F.dst.intact[b] = fin ? 1 : 0;
        if (a.h_intact) a.h_intact[(size_t)F.f * a.nb + b] = fin ? 1 : 0;
    }
    for (int e = gtid; e < a.n; e += gsz) {
        if (a.h_pos) {
            typename vec2_of<T>::type p = ld2(F.dst.pos, e);
            st2(a.h_pos + (size_t)F.f * a.n * 2, e, p.x, p.y);
        }
        if (a.h_rot) a.h_rot[(size_t)F.f * a.n + e] = F.dst.rot[e];
        if (a.h_sub) a.h_sub[(size_t)F.f * a.n + e] = F.dst.sub[e];
    }
    // per-frame scratch for the next frame
    for (int fl = gtid; fl < a.nf; fl += gsz) {
        a.fcoll[fl] = 0;
        a.fmax[fl] = 0ull;
    }
    for (int i = gtid; i < a.k_sub + 2; i += gsz) a.gdisp[i] = 0u;
}

// ─── the kernel ─────────────────────────────────────────────────────────────
// Phase numbering inside a frame: 0 contact, 1 reduce, then for substep s:
// 2+3s insert, 3+3s neighbour build, 4+3s force; last: 2+3k fracture.
template <typename T>
__global__ void __launch_bounds__(kThreads) dem_frames_kernel(KArgs<T> a, int ph_lo, int ph_hi) {
    extern __shared__ unsigned char smem_raw[];
    T* hullw = reinterpret_cast<T*>(smem_raw);
    const int k = a.k_sub;
    const int per_frame = 3 + 3 * k;
    const bool persistent = (a.mode == DEM_LAUNCH_PERSISTENT);
    // persistent-mode state (uniform across CTAs)
    bool dirty = false;
    bool need_rebuild = false;
    for (int ph = ph_lo; ph < ph_hi; ++ph) {
        const int f = ph / per_frame;
        const int p = ph % per_frame;
        Frame<T> F = make_frame(a, f);
        if (p == 0) {
            phase_contact(a, F, hullw);
            dirty = true;
        } else if (p == 1) {
            T sc;
            phase_reduce(a, F, &sc);
        } else if (p == per_frame - 1) {
            // recompute the frame's thrust scale (phased launches keep no state)
            __shared__ double tot3[3];
            double r[3];
            frame_totals(a, r);
            if (threadIdx.x == 0) {
                tot3[0] = r[0];
                tot3[1] = r[1];
                tot3[2] = r[2];
            }
            __syncthreads();
            T sc = thrust_scale_of(a, tot3);
            phase_fracture(a, F, sc);
        } else {
            const int s = (p - 2) / 3;
            const int sub = (p - 2) % 3;
            if (sub == 0 || sub == 1) {
                // neighbour-list rebuild before substep s (s >= 1 only: frame start built in P0/P1)
                bool run;
                if (persistent) {
                    run = (s >= 1) && need_rebuild;
                } else {
                    run = (s >= 1);
                }
                if (!run) continue;  // uniform across CTAs: no barrier for skipped phases
                if (sub == 0) {
                    const T* pos = a.sp_pos[(s - 1) & 1];
                    phase_insert(a, pos);
                    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd((unsigned long long*)&a.stats[0], 1ull);
                } else {
                    phase_nbr(a);
                    dirty = true;
                }
            } else {
                bool clear = persistent ? dirty : true;
                // substep s owns slot s: it is written only in this phase and read only
                // after the following barrier, so every CTA reads the same value
                phase_force(a, F, s, clear, &a.gdisp[s]);
                dirty = false;
            }
        }
        if (persistent && ph + 1 < ph_hi) {
            if (!grid_barrier(a)) return;
            // decide on a rebuild after each force phase (all CTAs read the same word)
            if (p >= 2 && p < per_frame - 1 && ((p - 2) % 3) == 2) {
                unsigned bits = *((volatile unsigned*)&a.gdisp[(p - 2) / 3]);
                float d2 = __uint_as_float(bits);
                double lim = 0.45 * (double)a.skin;
                need_rebuild = !(a.skin > T(0)) || !((double)d2 < lim * lim);
            }
        }
    }
}

// bond stiffness E * ((h_i + h_j) * 0.5) * factor, in the dtype (jax_simulation.py:81-82)
template <typename T>
__global__ void bond_stiffness_kernel(const T* thick, const int* bi, const int* bj, int nb, double E,
                                      double factor, T* out) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    T avg = (thick[bi[b]] + thick[bj[b]]) * T(0.5);
    out[b] = T(E) * avg * T(factor);
}

}  // namespace dem
