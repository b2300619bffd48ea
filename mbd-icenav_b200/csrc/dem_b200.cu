// dem_b200.cu — C ABI of the DPDEM frame step (see include/dem_b200.h).
//
// Host side: validates arguments, builds the per-element bond lists once,
// owns the scratch, and launches dem_frames_kernel either as one cooperative
// persistent launch per call or one launch per phase.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "dem_b200.h"
#include "dem_kernels.cuh"

using dem::IcePtrs;
using dem::KArgs;
using dem::ShipPtrs;

struct DemHandle {
    int dtype = DEM_F32;
    int device = 0;
    int mode = DEM_LAUNCH_PERSISTENT;
    int force_split = DEM_SPLIT_AUTO, mark_split = DEM_SPLIT_AUTO;
    DemParams P{};
    DemStatic S{};
    size_t esz = 4;
    int n = 0, V = 0, nb = 0, nf = 0, nh = 0;
    double r_max = 0.0, hull_r = 0.0, k_n = 0.0, k_s = 0.0, min_bstr = 0.0;
    double t_samp[dem::kMaxEdgeSamples] = {0};
    int n_buckets = 0;
    int grid_blocks = 0;
    int sm_count = 0;
    size_t smem = 0;
    // derived
    int* boff = nullptr;
    int2* bslot = nullptr;
    void* slot_rest = nullptr;
    void* slot_stiff = nullptr;
    void* vert_r = nullptr;
    // broad phase (persists across calls)
    int* bcnt = nullptr;
    int* bitems = nullptr;
    int2* ecell = nullptr;
    int* ncnt = nullptr;
    int* nbr = nullptr;
    void* pos_ref = nullptr;
    unsigned* dirty = nullptr;
    int fail_phase = -1;      // one-shot barrier fault for the next persistent call (test hook)
    int capacity_flags = 0;   // what overflowed at the last DEM_ERR_CAPACITY (1 bucket, 2 list)
    unsigned round_base = 0;  // dirty stamps issued so far (since the last clear)
    int* bflag = nullptr;
    int* comp_list = nullptr;
    int* comp_cnt = nullptr;
    int* esc_list = nullptr;
    int* dirty_list = nullptr;
    int* dirty_cnt = nullptr;
    int* work_cnt = nullptr;
    int* act_list = nullptr;
    int* lazy_list = nullptr;
    int* lazy_cnt = nullptr;
    int* counters = nullptr;  // block holding the per-call counters below
    size_t counters_bytes = 0;
    unsigned* bstamp = nullptr;  // (nb) frame stamps of bonds with an active end
    int* fb_list = nullptr;      // (nb) the frame's bonds with an active end
    int* fb_cnt = nullptr;
    int* act_cnt = nullptr;
    int* slot_owner = nullptr;
    unsigned* esc_cnt = nullptr;
    int* near_list = nullptr;
    int* near_cnt = nullptr;
    void* cpen = nullptr;
    void* cnx = nullptr;
    void* cny = nullptr;
    void* soi = nullptr;
    void* fraw = nullptr;
    uint8_t* crack = nullptr;
    int* fcoll = nullptr;
    unsigned long long* fmax = nullptr;
    double* part = nullptr;
    // per force chunk: warm (an element in contact or submerged at the last
    // cforce) and the stamp of the last frame with a near element
    uint8_t* cwarm = nullptr;
    unsigned* cnear = nullptr;
    void* kin[2] = {nullptr, nullptr};
    void* kvel[2] = {nullptr, nullptr};
    void* sp_rot[2] = {nullptr, nullptr};
    void* sp_avel[2] = {nullptr, nullptr};
    // frame ping-pong state for scans
    void* slotrec = nullptr;
    void* r3 = nullptr;
    void* econ = nullptr;
    double* fscal = nullptr;
    unsigned long long* ptimes = nullptr;
    bool profiling = false;
    void* ship_tmp = nullptr;  // 2 x 15 x nsys
    // independent systems (ice windows with their own ships)
    int nsys = 1;
    int nchunks = 0;
    int* sys_of = nullptr;
    int* floe_sys = nullptr;
    int2* chunk_info = nullptr;
    int* sys_end = nullptr;
    int* part_base = nullptr;
    std::vector<int> sys_start_h;  // (nsys + 1) element offsets
    void* sprow = nullptr;     // (6,) setpoint row of dem_frame_step
    unsigned* bar = nullptr;
    unsigned* bar_groups = nullptr;
    int bar_group_cap = 0;  // group words allocated
    // contact-set recording (dem_debug_record_contacts; caller-owned device arrays)
    int2* crec = nullptr;
    unsigned* crec_cnt = nullptr;
    int crec_cap = 0, crec_max_marks = 0;
    int* crec_marks = nullptr;
    int* status = nullptr;
    long long* stats = nullptr;
    int* host_status = nullptr;  // pinned
    std::vector<void*> allocs;
    std::string err;
};

namespace {

int set_err(DemHandle* h, int code, const char* fmt, ...) {
    if (h) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        h->err = buf;
    }
    return code;
}

#define CUDA_TRY(h, call)                                                                        \
    do {                                                                                         \
        cudaError_t _e = (call);                                                                 \
        if (_e != cudaSuccess)                                                                   \
            return set_err((h), DEM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e));  \
    } while (0)

template <typename P>
int dev_alloc(DemHandle* h, P** ptr, size_t bytes) {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) return set_err(h, DEM_ERR_CUDA, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    h->allocs.push_back(p);
    *ptr = reinterpret_cast<P*>(p);
    return DEM_OK;
}

void dev_free(DemHandle* h, void* p) {
    if (!p) return;
    auto it = std::find(h->allocs.begin(), h->allocs.end(), p);
    if (it != h->allocs.end()) {
        cudaFree(p);
        h->allocs.erase(it);
    }
}

// numpy.linspace(start, stop, num) with endpoint=True, in float64
void np_linspace(double start, double stop, int num, double* out) {
    if (num <= 0) return;
    if (num == 1) {
        out[0] = start;
        return;
    }
    const int div = num - 1;
    const double step = (stop - start) / div;
    for (int i = 0; i < num; ++i) out[i] = (double)i * step + start;
    out[num - 1] = stop;
}

int next_pow2(long long v) {
    int p = 1;
    while (p < v && p < (1 << 30)) p <<= 1;
    return p;
}

template <typename T>
std::vector<double> to_host_f64(const void* dptr, size_t count) {
    std::vector<T> tmp(count);
    std::vector<double> out(count);
    if (count) cudaMemcpy(tmp.data(), dptr, count * sizeof(T), cudaMemcpyDeviceToHost);
    for (size_t i = 0; i < count; ++i) out[i] = (double)tmp[i];
    return out;
}

std::vector<double> fetch(DemHandle* h, const void* dptr, size_t count) {
    return h->dtype == DEM_F32 ? to_host_f64<float>(dptr, count) : to_host_f64<double>(dptr, count);
}

int alloc_neighbors(DemHandle* h) {
    dev_free(h, h->nbr);
    dev_free(h, h->bitems);
    h->nbr = nullptr;
    h->bitems = nullptr;
    int rc;
    if ((rc = dev_alloc(h, &h->nbr, sizeof(int) * (size_t)h->P.max_neighbors * std::max(h->n, 1)))) return rc;
    if ((rc = dev_alloc(h, &h->bitems, sizeof(int) * (size_t)h->P.bucket_capacity * h->n_buckets))) return rc;
    return DEM_OK;
}

// Forget the persistent broad-phase state: reference positions become NaN so the
// next call rebuilds every list (after a capacity change or a device error).
int reset_broad_phase(DemHandle* h, cudaStream_t st) {
    CUDA_TRY(h, cudaMemsetAsync(h->bcnt, 0, sizeof(int) * (size_t)h->n_buckets, st));
    CUDA_TRY(h, cudaMemsetAsync(h->bitems, 0xFF, sizeof(int) * (size_t)h->n_buckets * h->P.bucket_capacity, st));
    CUDA_TRY(h, cudaMemsetAsync(h->comp_cnt, 0, sizeof(int), st));
    CUDA_TRY(h, cudaMemsetAsync(h->pos_ref, 0xFF, h->esz * 2 * (size_t)h->n, st));
    CUDA_TRY(h, cudaMemsetAsync(h->dirty, 0, sizeof(unsigned) * (size_t)h->n, st));
    CUDA_TRY(h, cudaMemsetAsync(h->bstamp, 0, sizeof(unsigned) * (size_t)std::max(h->nb, 1), st));
    CUDA_TRY(h, cudaMemsetAsync(h->bflag, 0, sizeof(int) * (size_t)h->n_buckets, st));
    CUDA_TRY(h, cudaMemsetAsync(h->ncnt, 0, sizeof(int) * (size_t)h->n, st));
    return DEM_OK;
}

template <typename T>
int occupancy_grid(DemHandle* h) {
    int per_sm = 0;
    CUDA_TRY(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dem::dem_frames_kernel<T>, dem::kThreads,
                                                              h->smem));
    if (per_sm < 1) return set_err(h, DEM_ERR_CUDA, "persistent kernel cannot be resident");
    h->grid_blocks = per_sm * h->sm_count;
    return DEM_OK;
}

template <typename T>
IcePtrs<T> ice_ptrs(const DemIceState* s) {
    IcePtrs<T> p;
    p.pos = (T*)s->positions;
    p.vel = (T*)s->velocities;
    p.rot = (T*)s->rotations;
    p.avel = (T*)s->angular_vels;
    p.sub = (T*)s->submergence;
    p.intact = s->bond_intact;
    p.dmg = (T*)s->bond_damage;
    p.dm0 = (T*)s->bond_delta_m_0;
    p.dmmax = (T*)s->bond_delta_m_max;
    p.ds = (T*)s->bond_delta_s;
    p.active = s->elem_active;
    p.elig = s->dpdem_floe_eligible;
    return p;
}

template <typename T>
ShipPtrs<T> ship_ptrs(const DemShipState* s) {
    ShipPtrs<T> p;
    p.eta = (T*)s->eta;
    p.nu = (T*)s->nu;
    p.na = (T*)s->n_actual;
    p.ei = (T*)s->e_int;
    return p;
}

int check_state(DemHandle* h, const DemIceState* s, const char* what) {
    if (!s) return set_err(h, DEM_ERR_INVALID, "%s state is NULL", what);
    if (!s->positions || !s->velocities || !s->rotations || !s->angular_vels || !s->submergence ||
        !s->elem_active || !s->dpdem_floe_eligible)
        return set_err(h, DEM_ERR_INVALID, "%s state has a NULL element field", what);
    if (h->nb > 0 && (!s->bond_intact || !s->bond_damage || !s->bond_delta_m_0 || !s->bond_delta_m_max ||
                      !s->bond_delta_s))
        return set_err(h, DEM_ERR_INVALID, "%s state has a NULL bond field", what);
    return DEM_OK;
}

int check_ship(DemHandle* h, const DemShipState* s, const char* what) {
    if (!s || !s->eta || !s->nu || !s->n_actual || !s->e_int)
        return set_err(h, DEM_ERR_INVALID, "%s ship state has a NULL field", what);
    return DEM_OK;
}

template <typename T>
int launch(DemHandle* h, const DemIceState* in, DemIceState* out, const DemShipState* ship_in,
           DemShipState* ship_out, int K, const void* setpoints, const void* vw, const void* vws,
           const uint8_t* elig0, DemDiag* diag, DemHistory* hist, cudaStream_t stream,
           const void* u_ctrl = nullptr) {
    KArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.u_ctrl = (const T*)u_ctrl;
    a.P = h->P;
    a.n = h->n;
    a.V = h->V;
    a.nb = h->nb;
    a.nf = h->nf;
    a.S = h->nh;
    a.K = K;
    a.k_sub = h->P.n_ice_steps;
    a.nchunks = h->nchunks;
    a.nsys = h->nsys;
    a.sys_of = h->sys_of;
    a.floe_sys = h->floe_sys;
    a.chunk_info = h->chunk_info;
    a.sys_end = h->sys_end;
    a.part_base = h->part_base;
    a.n_buckets = h->n_buckets;
    a.bucket_cap = h->P.bucket_capacity;
    a.max_nb = h->P.max_neighbors;
    a.mode = h->mode;
    a.force_split = h->force_split;
    a.mark_split = h->mark_split;
    a.k_n = (T)h->k_n;
    a.k_s = (T)h->k_s;
    a.min_bstr = (T)h->min_bstr;
    double cell = (2.0 * h->r_max + h->P.skin) * 1.0001;
    a.cell = (T)(cell > 1e-6 ? cell : 1.0);  // zero radii and skin: no pair can touch
    a.skin = (T)h->P.skin;
    {
        // escape period and thresholds (see the Verlet-list notes in dem_kernels.cuh)
        const double S = h->P.skin;
        const double dmax = std::sqrt(2.0) * std::fabs(h->P.velocity_clip) * h->P.dt_ice;
        const double h_urgent = 0.45 * 0.99 * S;
        const double h_two = 0.99 * (0.5 * S - dmax);
        const bool two = std::isfinite(dmax) && h_two >= 0.25 * S;
        a.esc_period = two ? 2 : 1;
        // lazy escapes replace the every-second-substep processing
        a.lazy = (two && h->P.n_ice_steps >= 2) ? 1 : 0;
        a.esc_h_check = (T)(two ? std::min(h_two, h_urgent) : h_urgent);
        a.esc_h_urgent = (T)h_urgent;
    }
    a.hull_r = (T)h->hull_r;
    for (int i = 0; i < dem::kMaxEdgeSamples; ++i) a.t_samp[i] = (T)h->t_samp[i];
    a.polys = (const T*)h->S.local_polys_padded;
    a.pmask = h->S.poly_mask;
    a.mass = (const T*)h->S.masses;
    a.inertia = (const T*)h->S.inertia;
    a.radii = (const T*)h->S.radii;
    a.areas = (const T*)h->S.areas;
    a.thick = (const T*)h->S.thicknesses;
    a.rest = (const T*)h->S.rest_lengths;
    a.bstr = (const T*)h->S.bond_strengths;
    a.sbar = (const T*)h->S.sigma_bar_bond;
    a.hull = (const T*)h->S.ship_hull_local;
    a.bi = h->S.bond_i;
    a.bj = h->S.bond_j;
    a.floe_of = h->S.initial_floe_of;
    a.boff = h->boff;
    a.bslot = h->bslot;
    a.slot_rest = (const T*)h->slot_rest;
    a.slot_stiff = (const T*)h->slot_stiff;
    a.vert_r = (const T*)h->vert_r;
    a.bcnt = h->bcnt;
    a.bitems = h->bitems;
    a.near_list = h->near_list;
    a.near_cnt = h->near_cnt;
    a.cpen = (T*)h->cpen;
    a.cnx = (T*)h->cnx;
    a.cny = (T*)h->cny;
    a.ecell = h->ecell;
    a.ncnt = h->ncnt;
    a.nbr = h->nbr;
    a.pos_ref = (T*)h->pos_ref;
    a.dirty = h->dirty;
    a.bflag = h->bflag;
    a.comp_list = h->comp_list;
    a.comp_cnt = h->comp_cnt;
    a.esc_list = h->esc_list;
    a.dirty_list = h->dirty_list;
    a.dirty_cnt = h->dirty_cnt;
    a.work_cnt = h->work_cnt;
    a.act_list = h->act_list;
    a.lazy_list = h->lazy_list;
    a.lazy_cnt = h->lazy_cnt;
    a.bstamp = h->bstamp;
    a.fb_list = h->fb_list;
    a.fb_cnt = h->fb_cnt;
    a.act_cnt = h->act_cnt;
    a.slot_owner = h->slot_owner;
    a.esc_cnt = h->esc_cnt;
    a.soi = (T*)h->soi;
    a.fraw = (T*)h->fraw;
    a.crack = h->crack;
    a.fcoll = h->fcoll;
    a.fmax = h->fmax;
    a.part = h->part;
    a.cwarm = h->cwarm;
    a.cnear = h->cnear;
    for (int i = 0; i < 2; ++i) {
        a.kin[i] = (T*)h->kin[i];
        a.kvel[i] = (T*)h->kvel[i];
        a.sp_rot[i] = (T*)h->sp_rot[i];
        a.sp_avel[i] = (T*)h->sp_avel[i];
    }
    a.slotrec = h->slotrec;
    a.r3 = (const T*)h->r3;
    {
        const DemParams& P = h->P;
        a.fc.hf = (T)P.hertz_factor;
        a.fc.hexp = (T)P.hertz_exponent;
        a.fc.h15 = (P.hertz_exponent == 1.5) ? 1 : 0;
        a.fc.mu = (T)P.ice_ice_friction;
        a.fc.fcap = (T)P.friction_cap;
        a.fc.c_drag = (T)(0.5 * P.water_density * P.c_d_drag);
        a.fc.href = (T)P.drag_ref_thickness;
        a.fc.lin = (T)P.linear_drag_factor;
        a.fc.c_rot = (T)(-0.5 * P.drag_coefficient_moment * P.water_density);
        a.fc.dti = (T)P.dt_ice;
        a.fc.damp = (T)P.angular_damping;
        a.fc.alo = (T)P.angular_cap_lo;
        a.fc.ahi = (T)P.angular_cap_hi;
        a.fc.vclip = (T)P.velocity_clip;
        a.fc.pclip = (T)P.position_clip;
    }
    a.econ = (const T*)h->econ;
    a.fscal = h->fscal;
    a.ptimes = h->profiling ? h->ptimes : nullptr;
    a.in = ice_ptrs<T>(in);
    a.out = ice_ptrs<T>(out);
    a.ship_in = ship_ptrs<T>(ship_in);
    a.ship_out = ship_ptrs<T>(ship_out);
    T* st = (T*)h->ship_tmp;
    for (int i = 0; i < 2; ++i) {
        const int q = h->nsys;  // per buffer: eta (3q), nu (3q), n_actual (6q), e_int (3q)
        a.ship_tmp[i].eta = st + 15 * q * i;
        a.ship_tmp[i].nu = st + 15 * q * i + 3 * q;
        a.ship_tmp[i].na = st + 15 * q * i + 6 * q;
        a.ship_tmp[i].ei = st + 15 * q * i + 12 * q;
    }
    a.setpoints = (const T*)setpoints;
    a.vw = (const T*)vw;
    a.vws = (const T*)vws;
    a.elig0 = elig0;
    if (diag) {
        a.d_pen = (T*)diag->pen_max;
        a.d_fmag = (T*)diag->force_mag;
        a.d_F = (T*)diag->F_ice_on_ship;
        a.d_J = (T*)diag->J_cumul_incr;
    }
    if (hist) {
        a.h_pos = (T*)hist->positions;
        a.h_rot = (T*)hist->rotations;
        a.h_intact = hist->bond_intact;
        a.h_eta = (T*)hist->eta;
        a.h_sub = (T*)hist->submergence;
        a.h_J = (T*)hist->J_cumul_incr;
        a.h_F = (T*)hist->F_ice_on_ship;
    }
    a.bar = h->bar;
    a.bar_groups = h->bar_groups;
    a.status = h->status;
    a.stats = h->stats;
    a.crec = h->crec;
    a.crec_cnt = h->crec_cnt;
    a.crec_cap = h->crec_cap;
    a.crec_marks = h->crec_marks;
    a.crec_max_marks = h->crec_max_marks;
    if (h->crec) CUDA_TRY(h, cudaMemsetAsync(h->crec_cnt, 0, sizeof(unsigned), stream));

    // per-call scratch reset (the kernel keeps it clean between frames)
    // per-call counters (escapes, rebuilds, work, lazy escapes, barrier, near
    // count) in one memset; the per-floe flags are cleared by each frame's cull
    CUDA_TRY(h, cudaMemsetAsync(h->counters, 0, h->counters_bytes, stream));
    {
        // every rebuild round of every call gets its own dirty stamp; clear the
        // stamps before the counter would wrap
        const unsigned need = (unsigned)K * (unsigned)h->P.n_ice_steps + 1u;
        if (h->round_base > 0xFFFFFFFFu - need) {
            CUDA_TRY(h, cudaMemsetAsync(h->dirty, 0, sizeof(unsigned) * (size_t)h->n, stream));
            CUDA_TRY(h, cudaMemsetAsync(h->bstamp, 0, sizeof(unsigned) * (size_t)std::max(h->nb, 1), stream));
            h->round_base = 0;
        }
        a.round_base = h->round_base;
        a.fail_phase = (h->mode == DEM_LAUNCH_PERSISTENT) ? h->fail_phase : -1;
        h->fail_phase = -1;
        h->round_base += need;
    }
    if (h->profiling) CUDA_TRY(h, cudaMemsetAsync(h->ptimes, 0, sizeof(unsigned long long) * 2, stream));

    const int k = h->P.n_ice_steps;
    const int per_frame = dem::phases_per_frame(k);
    if (h->mode == DEM_LAUNCH_PERSISTENT) {
        if (dem::kBarGroup > 0 && (h->grid_blocks + dem::kBarGroup - 1) / dem::kBarGroup > h->bar_group_cap)
            return set_err(h, DEM_ERR_INVALID, "persistent grid exceeds the barrier's group words");
        int lo = 0, hi = K * per_frame;
        void* args[] = {(void*)&a, (void*)&lo, (void*)&hi};
        CUDA_TRY(h, cudaLaunchCooperativeKernel((const void*)dem::dem_frames_kernel<T>, dim3(h->grid_blocks),
                                                dim3(dem::kThreads), args, h->smem, stream));
    } else {
        long long work = std::max<long long>(std::max(h->n, h->nb), 1);
        int blocks = (int)std::min<long long>((work + dem::kThreads - 1) / dem::kThreads, (long long)h->sm_count * 16);
        blocks = std::max(blocks, 1);
        for (int f = 0; f < K; ++f) {
            for (int p = 0; p < per_frame; ++p) {
                int ph = f * per_frame + p;
                dem::dem_frames_kernel<T><<<blocks, dem::kThreads, h->smem, stream>>>(a, ph, ph + 1);
                CUDA_TRY(h, cudaGetLastError());
            }
        }
    }
    return DEM_OK;
}

}  // namespace

namespace {

// The planners' rigid-ship rollout (jax_mbd_planner.py:51-122 rolls the
// 3-DOF ship out alone): per candidate, H steps of the frame step's vessel
// update driven by its body-frame control with no ice load, exactly the ship
// part of a dem_rollout_segment frame whose ice exerts nothing.
template <typename T>
__global__ void ship_rollout_kernel(const DemParams P, int Q, int H, const T* __restrict__ eta0,
                                    const T* __restrict__ nu0, const T* __restrict__ u,
                                    const T* __restrict__ vws, T* __restrict__ eta_hist, T* __restrict__ nu_out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Q) return;
    T eta[3], nu[3], na[6] = {T(0), T(0), T(0), T(0), T(0), T(0)}, ei[3] = {T(0), T(0), T(0)};
    for (int i = 0; i < 3; ++i) {
        eta[i] = eta0[3 * q + i];
        nu[i] = nu0[3 * q + i];
    }
    const T zero3[3] = {T(0), T(0), T(0)};
    const T zero2[2] = {T(0), T(0)};
    for (int t = 0; t < H; ++t) {
        T eo[3], no[3], nao[6], eio[3];
        const T* w = vws ? vws + ((size_t)t * Q + q) * 2 : zero2;
        dem::ship_step<T>(P, eta, nu, na, ei, zero3, zero3, zero3, w, eo, no, nao, eio, u + ((size_t)t * Q + q) * 3);
        for (int i = 0; i < 3; ++i) {
            eta[i] = eo[i];
            nu[i] = no[i];
            eta_hist[((size_t)t * Q + q) * 3 + i] = eo[i];
        }
    }
    if (nu_out)
        for (int i = 0; i < 3; ++i) nu_out[3 * q + i] = nu[i];
}

}  // namespace

extern "C" {

const char* dem_version(void) { return "dem_b200 0.1 sm_100a"; }

int dem_create(const DemParams* params, const DemStatic* s, int dtype, int device, DemHandle** out) {
    if (!params || !s || !out) return DEM_ERR_INVALID;
    *out = nullptr;
    DemHandle* h = new DemHandle();
    h->dtype = dtype;
    h->device = device;
    h->P = *params;
    h->S = *s;
    h->esz = dtype == DEM_F64 ? 8 : 4;
    h->n = s->n;
    h->V = s->max_v;
    h->nb = s->n_bonds;
    h->nf = s->n_floes;
    h->nh = s->n_hull;
    auto fail = [&](int rc) {
        *out = h;  // keep the handle so dem_get_error can report; caller destroys it
        return rc;
    };
    if (dtype != DEM_F32 && dtype != DEM_F64) return fail(set_err(h, DEM_ERR_INVALID, "dtype must be DEM_F32 or DEM_F64"));
    if (h->n < 1) return fail(set_err(h, DEM_ERR_INVALID, "n must be >= 1"));
    if (h->V < 1 || h->V > dem::kMaxV) return fail(set_err(h, DEM_ERR_INVALID, "max_v=%d outside [1,%d]", h->V, dem::kMaxV));
    if (h->nb < 0 || h->nf < 1) return fail(set_err(h, DEM_ERR_INVALID, "bad n_bonds/n_floes"));
    if (h->nh < 1 || h->nh > dem::kMaxHull) return fail(set_err(h, DEM_ERR_INVALID, "n_hull=%d outside [1,%d]", h->nh, dem::kMaxHull));
    if (h->P.n_ice_steps < 1) return fail(set_err(h, DEM_ERR_INVALID, "n_ice_steps must be >= 1"));
    if (h->P.n_edge_samples < 0 || h->P.n_edge_samples > dem::kMaxEdgeSamples)
        return fail(set_err(h, DEM_ERR_INVALID, "n_edge_samples outside [0,%d]", dem::kMaxEdgeSamples));
    if (h->P.max_neighbors < 1 || h->P.max_neighbors > dem::kMaxNbLocal)
        return fail(set_err(h, DEM_ERR_INVALID, "max_neighbors outside [1,%d]", dem::kMaxNbLocal));
    if (h->P.bucket_capacity < 1) return fail(set_err(h, DEM_ERR_INVALID, "bucket_capacity must be >= 1"));
    if (!(h->P.skin >= 0.0)) return fail(set_err(h, DEM_ERR_INVALID, "skin must be >= 0"));
    if (!s->local_polys_padded || !s->poly_mask || !s->masses || !s->inertia || !s->radii || !s->areas ||
        !s->thicknesses || !s->initial_floe_of || !s->ship_hull_local)
        return fail(set_err(h, DEM_ERR_INVALID, "static data has a NULL array"));
    if (h->nb > 0 && (!s->bond_i || !s->bond_j || !s->rest_lengths || !s->bond_strengths || !s->sigma_bar_bond))
        return fail(set_err(h, DEM_ERR_INVALID, "static data has a NULL bond array"));

    cudaError_t ce = cudaSetDevice(device);
    if (ce != cudaSuccess) return fail(set_err(h, DEM_ERR_CUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(ce)));
    cudaDeviceProp prop;
    ce = cudaGetDeviceProperties(&prop, device);
    if (ce != cudaSuccess) return fail(set_err(h, DEM_ERR_CUDA, "cudaGetDeviceProperties: %s", cudaGetErrorString(ce)));
    h->sm_count = prop.multiProcessorCount;
    if (!prop.cooperativeLaunch) h->mode = DEM_LAUNCH_PHASED;

    // host copies of the static data the set-up needs (one-time)
    const int n = h->n, nb = h->nb, nf = h->nf;
    std::vector<double> radii = fetch(h, s->radii, n);
    std::vector<double> polys = fetch(h, s->local_polys_padded, (size_t)n * h->V * 2);
    std::vector<double> hull = fetch(h, s->ship_hull_local, (size_t)h->nh * 2);
    std::vector<int> floe((size_t)n);
    cudaMemcpy(floe.data(), s->initial_floe_of, sizeof(int) * n, cudaMemcpyDeviceToHost);
    std::vector<int> bi(nb), bj(nb);
    std::vector<double> bstr;
    if (nb) {
        cudaMemcpy(bi.data(), s->bond_i, sizeof(int) * nb, cudaMemcpyDeviceToHost);
        cudaMemcpy(bj.data(), s->bond_j, sizeof(int) * nb, cudaMemcpyDeviceToHost);
        bstr = fetch(h, s->bond_strengths, nb);
    }
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return fail(set_err(h, DEM_ERR_CUDA, "copying static data: %s", cudaGetErrorString(ce)));
    for (int e = 0; e < n; ++e)
        if (floe[e] < 0 || floe[e] >= nf) return fail(set_err(h, DEM_ERR_INVALID, "initial_floe_of[%d]=%d outside [0,%d)", e, floe[e], nf));
    for (int b = 0; b < nb; ++b)
        if (bi[b] < 0 || bi[b] >= n || bj[b] < 0 || bj[b] >= n || bi[b] == bj[b])
            return fail(set_err(h, DEM_ERR_INVALID, "bond %d=(%d,%d) invalid", b, bi[b], bj[b]));
    // systems: contiguous element ranges; floes and bonds may not span two
    h->nsys = s->n_systems > 1 ? s->n_systems : 1;
    h->sys_start_h.assign(h->nsys + 1, 0);
    h->sys_start_h[h->nsys] = n;
    if (h->nsys > 1) {
        if (!s->system_start) return fail(set_err(h, DEM_ERR_INVALID, "n_systems > 1 needs system_start"));
        for (int q = 0; q <= h->nsys; ++q) h->sys_start_h[q] = s->system_start[q];
        if (h->sys_start_h[0] != 0 || h->sys_start_h[h->nsys] != n)
            return fail(set_err(h, DEM_ERR_INVALID, "system_start must run from 0 to n"));
        for (int q = 0; q < h->nsys; ++q)
            if (h->sys_start_h[q + 1] <= h->sys_start_h[q])
                return fail(set_err(h, DEM_ERR_INVALID, "system %d has no element", q));
    }
    std::vector<int> sys_of(n), floe_sys(nf, -1);
    for (int q = 0; q < h->nsys; ++q)
        for (int e = h->sys_start_h[q]; e < h->sys_start_h[q + 1]; ++e) sys_of[e] = q;
    for (int e = 0; e < n; ++e) {
        if (floe_sys[floe[e]] >= 0 && floe_sys[floe[e]] != sys_of[e])
            return fail(set_err(h, DEM_ERR_INVALID, "floe %d spans two systems", floe[e]));
        floe_sys[floe[e]] = sys_of[e];
    }
    for (int& v : floe_sys) v = std::max(v, 0);
    for (int b = 0; b < nb; ++b)
        if (sys_of[bi[b]] != sys_of[bj[b]]) return fail(set_err(h, DEM_ERR_INVALID, "bond %d spans two systems", b));
    // force chunks of kThreads elements, aligned to each system's first element
    std::vector<int2> chunks;
    std::vector<int> part_base(h->nsys + 1, 0), sys_end(h->nsys);
    for (int q = 0; q < h->nsys; ++q) {
        part_base[q] = (int)chunks.size();
        sys_end[q] = h->sys_start_h[q + 1];
        for (int e0 = h->sys_start_h[q]; e0 < h->sys_start_h[q + 1]; e0 += dem::kThreads) chunks.push_back(make_int2(q, e0));
    }
    part_base[h->nsys] = (int)chunks.size();
    h->nchunks = (int)chunks.size();
    h->r_max = 0.0;
    for (double r : radii) {
        if (!(r >= 0.0) || !std::isfinite(r)) return fail(set_err(h, DEM_ERR_INVALID, "radii must be finite and >= 0"));
        h->r_max = std::max(h->r_max, r);
    }
    std::vector<double> vr(n, 0.0);
    for (int e = 0; e < n; ++e)
        for (int k = 0; k < h->V; ++k) {
            double x = polys[((size_t)e * h->V + k) * 2], y = polys[((size_t)e * h->V + k) * 2 + 1];
            vr[e] = std::max(vr[e], std::sqrt(x * x + y * y));
        }
    for (int e = 0; e < n; ++e) vr[e] = vr[e] * (1.0 + 1e-5) + 1e-4;  // conservative (rounded up)
    // reach of the ship: its outline points (pass 2) and the corners of the
    // analytic hull box |x| <= half_len, |y| <= half_beam (pass 1)
    h->hull_r = std::hypot(h->P.half_len, h->P.half_beam);
    for (int i = 0; i < h->nh; ++i) h->hull_r = std::max(h->hull_r, std::hypot(hull[2 * i], hull[2 * i + 1]));
    h->hull_r = h->hull_r * (1.0 + 1e-5) + 1e-4;
    h->k_n = s->k_n;
    h->k_s = s->k_s;
    h->min_bstr = 0.0;
    if (nb) {
        h->min_bstr = bstr[0];
        for (double v : bstr) h->min_bstr = std::min(h->min_bstr, v);
    }
    np_linspace(1.0 / (h->P.n_edge_samples + 1), (double)h->P.n_edge_samples / (h->P.n_edge_samples + 1),
                h->P.n_edge_samples, h->t_samp);

    // per-element bond slots: bonds with e == bond_i (ascending), then e == bond_j (ascending)
    std::vector<int> ci(n, 0), cj(n, 0), off(n + 1, 0);
    for (int b = 0; b < nb; ++b) {
        ci[bi[b]]++;
        cj[bj[b]]++;
    }
    for (int e = 0; e < n; ++e) off[e + 1] = off[e] + ci[e] + cj[e];
    std::vector<int> pi(n), pj(n);
    for (int e = 0; e < n; ++e) {
        pi[e] = off[e];
        pj[e] = off[e] + ci[e];
    }
    std::vector<int2> slots((size_t)std::max(2 * nb, 1));
    for (int b = 0; b < nb; ++b) {
        slots[pi[bi[b]]++] = make_int2(b, bj[b]);
        slots[pj[bj[b]]++] = make_int2((int)((unsigned)b | 0x80000000u), bi[b]);
    }

    int rc;
    const size_t es = h->esz;
    h->n_buckets = std::max(1024, next_pow2(2LL * n));
    if ((rc = dev_alloc(h, &h->boff, sizeof(int) * (n + 1)))) return fail(rc);
    if ((rc = dev_alloc(h, &h->bslot, sizeof(int2) * slots.size()))) return fail(rc);
    if ((rc = dev_alloc(h, &h->slot_rest, es * slots.size()))) return fail(rc);
    if ((rc = dev_alloc(h, &h->slot_stiff, es * slots.size()))) return fail(rc);
    if ((rc = dev_alloc(h, &h->vert_r, es * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->bcnt, sizeof(int) * (size_t)h->n_buckets))) return fail(rc);
    if ((rc = dev_alloc(h, &h->near_list, sizeof(int) * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->cpen, es * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->cnx, es * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->cny, es * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->ecell, sizeof(int2) * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->ncnt, sizeof(int) * n))) return fail(rc);
    if ((rc = alloc_neighbors(h))) return fail(rc);
    if ((rc = dev_alloc(h, &h->pos_ref, es * 2 * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->dirty, sizeof(unsigned) * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->bflag, sizeof(int) * (size_t)h->n_buckets))) return fail(rc);
    if ((rc = dev_alloc(h, &h->comp_list, sizeof(int) * (size_t)h->n_buckets))) return fail(rc);
    if ((rc = dev_alloc(h, &h->comp_cnt, sizeof(int)))) return fail(rc);
    if ((rc = dev_alloc(h, &h->esc_list, sizeof(int) * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->dirty_list, sizeof(int) * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->act_list, sizeof(int) * (size_t)dem::kActLists * std::max(n, 1)))) return fail(rc);
    if ((rc = dev_alloc(h, &h->lazy_list, sizeof(int) * std::max(n, 1)))) return fail(rc);
    if ((rc = dev_alloc(h, &h->bstamp, sizeof(unsigned) * std::max(nb, 1)))) return fail(rc);
    if ((rc = dev_alloc(h, &h->fb_list, sizeof(int) * std::max(nb, 1)))) return fail(rc);
    if ((rc = dev_alloc(h, &h->fb_cnt, sizeof(int)))) return fail(rc);
    if ((rc = dev_alloc(h, &h->act_cnt, sizeof(int) * dem::kActLists))) return fail(rc);
    if ((rc = dev_alloc(h, &h->slot_owner, sizeof(int) * slots.size()))) return fail(rc);
    {
        // the per-call counters in one block, cleared by one memset per call:
        // esc_cnt, dirty_cnt, work_cnt, lazy_cnt (k + 2 each), bar (2), near_cnt
        // (1), then, from the next 128-byte line, the grid barrier's group words
        // (one line each)
        const size_t k2 = (size_t)h->P.n_ice_steps + 2;
        const size_t stride = (size_t)dem::kBarGroupStride;
        const size_t groups_at = ((4 * k2 + 3 + stride - 1) / stride) * stride;
        // enough groups for the largest persistent grid: every SM full of CTAs
        // of kThreads threads (the grid is sized by occupancy later)
        const size_t max_grid = (size_t)h->sm_count * (2048 / dem::kThreads);
        const size_t n_groups = dem::kBarGroup > 0 ? (max_grid + dem::kBarGroup - 1) / dem::kBarGroup : 0;
        h->bar_group_cap = (int)n_groups;
        const size_t words = groups_at + n_groups * stride;
        if ((rc = dev_alloc(h, &h->counters, sizeof(int) * words))) return fail(rc);
        h->counters_bytes = sizeof(int) * words;
        h->esc_cnt = reinterpret_cast<unsigned*>(h->counters);
        h->dirty_cnt = h->counters + k2;
        h->work_cnt = h->counters + 2 * k2;
        h->lazy_cnt = h->counters + 3 * k2;
        h->bar = reinterpret_cast<unsigned*>(h->counters + 4 * k2);
        h->near_cnt = h->counters + 4 * k2 + 2;
        h->bar_groups = reinterpret_cast<unsigned*>(h->counters + groups_at);
    }
    if ((rc = dev_alloc(h, &h->soi, es * 2 * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->fraw, es * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->crack, n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->fcoll, sizeof(int) * nf))) return fail(rc);
    if ((rc = dev_alloc(h, &h->fmax, sizeof(unsigned long long) * nf))) return fail(rc);
    if ((rc = dev_alloc(h, &h->part, sizeof(double) * 3 * std::max(h->nchunks, 1)))) return fail(rc);
    {
        const size_t nc = (size_t)std::max(h->nchunks, 1);
        if ((rc = dev_alloc(h, &h->cwarm, nc))) return fail(rc);
        if ((rc = dev_alloc(h, &h->cnear, sizeof(unsigned) * nc))) return fail(rc);
    }
    if ((rc = dev_alloc(h, &h->sys_of, sizeof(int) * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->floe_sys, sizeof(int) * nf))) return fail(rc);
    if ((rc = dev_alloc(h, &h->chunk_info, sizeof(int2) * std::max(h->nchunks, 1)))) return fail(rc);
    if ((rc = dev_alloc(h, &h->sys_end, sizeof(int) * h->nsys))) return fail(rc);
    if ((rc = dev_alloc(h, &h->part_base, sizeof(int) * (h->nsys + 1)))) return fail(rc);
    for (int i = 0; i < 2; ++i) {
        if ((rc = dev_alloc(h, &h->kin[i], es * 4 * n))) return fail(rc);
        if ((rc = dev_alloc(h, &h->kvel[i], es * 2 * n))) return fail(rc);
        if ((rc = dev_alloc(h, &h->sp_rot[i], es * n))) return fail(rc);
        if ((rc = dev_alloc(h, &h->sp_avel[i], es * n))) return fail(rc);
    }
    if ((rc = dev_alloc(h, &h->ship_tmp, es * 30 * h->nsys))) return fail(rc);
    if ((rc = dev_alloc(h, &h->slotrec, (es == 4 ? 16 : 32) * slots.size()))) return fail(rc);
    if ((rc = dev_alloc(h, &h->r3, es * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->econ, es * 4 * n))) return fail(rc);
    if ((rc = dev_alloc(h, &h->fscal, sizeof(double) * 4 * h->nsys))) return fail(rc);
    if ((rc = dev_alloc(h, &h->ptimes, sizeof(unsigned long long) * (2 + 2 * dem::kMaxPhaseTimes)))) return fail(rc);
    if ((rc = dev_alloc(h, &h->sprow, es * 6))) return fail(rc);
    if ((rc = dev_alloc(h, &h->status, sizeof(int)))) return fail(rc);
    if ((rc = dev_alloc(h, &h->stats, sizeof(long long) * 8))) return fail(rc);
    ce = cudaMallocHost(&h->host_status, sizeof(int));
    if (ce != cudaSuccess) return fail(set_err(h, DEM_ERR_CUDA, "cudaMallocHost: %s", cudaGetErrorString(ce)));

#define CREATE_TRY(call)                                                                                  \
    do {                                                                                                  \
        cudaError_t _e = (call);                                                                          \
        if (_e != cudaSuccess) return fail(set_err(h, DEM_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e))); \
    } while (0)
    CREATE_TRY(cudaMemcpy(h->boff, off.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    CREATE_TRY(cudaMemcpy(h->sys_of, sys_of.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    CREATE_TRY(cudaMemcpy(h->floe_sys, floe_sys.data(), sizeof(int) * nf, cudaMemcpyHostToDevice));
    CREATE_TRY(cudaMemcpy(h->chunk_info, chunks.data(), sizeof(int2) * chunks.size(), cudaMemcpyHostToDevice));
    CREATE_TRY(cudaMemcpy(h->sys_end, sys_end.data(), sizeof(int) * h->nsys, cudaMemcpyHostToDevice));
    CREATE_TRY(cudaMemcpy(h->part_base, part_base.data(), sizeof(int) * (h->nsys + 1), cudaMemcpyHostToDevice));
    {
        // every first frame of a call sets the chunk flags; start from "warm"
        const size_t nc = (size_t)std::max(h->nchunks, 1);
        CREATE_TRY(cudaMemset(h->cwarm, 1, nc));
        CREATE_TRY(cudaMemset(h->cnear, 0, sizeof(unsigned) * nc));
    }
    CREATE_TRY(cudaMemcpy(h->bslot, slots.data(), sizeof(int2) * slots.size(), cudaMemcpyHostToDevice));
    {
        std::vector<int> owner(slots.size(), 0);
        for (int e = 0; e < n; ++e)
            for (int sl = off[e]; sl < off[e + 1]; ++sl) owner[sl] = e;
        CREATE_TRY(cudaMemcpy(h->slot_owner, owner.data(), sizeof(int) * owner.size(), cudaMemcpyHostToDevice));
    }
    if (h->dtype == DEM_F32) {
        std::vector<float> v(n);
        for (int e = 0; e < n; ++e) v[e] = std::nextafter((float)vr[e], INFINITY);
        CREATE_TRY(cudaMemcpy(h->vert_r, v.data(), 4 * n, cudaMemcpyHostToDevice));
    } else {
        CREATE_TRY(cudaMemcpy(h->vert_r, vr.data(), 8 * n, cudaMemcpyHostToDevice));
    }
    if ((rc = reset_broad_phase(h, 0))) return fail(rc);
    CREATE_TRY(cudaMemset(h->status, 0, sizeof(int)));
    CREATE_TRY(cudaMemset(h->stats, 0, sizeof(long long) * 8));
    CREATE_TRY(cudaMemset(h->counters, 0, h->counters_bytes));
    if (nb) {
        int n_slots = 2 * nb;
        int blocks = (n_slots + 255) / 256;
        if (h->dtype == DEM_F32)
            dem::slot_setup_kernel<float><<<blocks, 256>>>((const float*)s->thicknesses, (const float*)s->rest_lengths,
                                                           s->bond_i, s->bond_j, h->bslot, n_slots, h->P.youngs_modulus,
                                                           h->P.bond_stiffness_factor, (float*)h->slot_rest,
                                                           (float*)h->slot_stiff);
        else
            dem::slot_setup_kernel<double><<<blocks, 256>>>((const double*)s->thicknesses,
                                                            (const double*)s->rest_lengths, s->bond_i, s->bond_j,
                                                            h->bslot, n_slots, h->P.youngs_modulus,
                                                            h->P.bond_stiffness_factor, (double*)h->slot_rest,
                                                            (double*)h->slot_stiff);
        CREATE_TRY(cudaGetLastError());
    }
    {
        int blocks = (n + 255) / 256;
        if (h->dtype == DEM_F32)
            dem::cube_kernel<float><<<blocks, 256>>>((const float*)s->radii, n, (float*)h->r3);
        else
            dem::cube_kernel<double><<<blocks, 256>>>((const double*)s->radii, n, (double*)h->r3);
        CREATE_TRY(cudaGetLastError());
        if (h->dtype == DEM_F32)
            dem::econ_kernel<float><<<blocks, 256>>>((const float*)s->masses, (const float*)s->inertia,
                                                     (const float*)s->thicknesses, (const float*)s->areas, n,
                                                     (float*)h->econ);
        else
            dem::econ_kernel<double><<<blocks, 256>>>((const double*)s->masses, (const double*)s->inertia,
                                                      (const double*)s->thicknesses, (const double*)s->areas, n,
                                                      (double*)h->econ);
        CREATE_TRY(cudaGetLastError());
    }
    h->smem = (size_t)h->nh * 2 * es + 16;
    if ((rc = (h->dtype == DEM_F32 ? occupancy_grid<float>(h) : occupancy_grid<double>(h)))) return fail(rc);
    CREATE_TRY(cudaDeviceSynchronize());
#undef CREATE_TRY
    *out = h;
    return DEM_OK;
}

int dem_frame_step(DemHandle* h, const DemIceState* in, DemIceState* out, const DemShipState* ship_in,
                   DemShipState* ship_out, const void* setpoint, const void* setpoint_next, const void* v_water,
                   const uint8_t* dpdem_eligible, const void* v_water_ship, DemDiag* diag, void* stream) {
    if (!h) return DEM_ERR_INVALID;
    int rc;
    if ((rc = check_state(h, in, "input"))) return rc;
    if ((rc = check_state(h, out, "output"))) return rc;
    if ((rc = check_ship(h, ship_in, "input"))) return rc;
    if ((rc = check_ship(h, ship_out, "output"))) return rc;
    if (!setpoint || !setpoint_next || !v_water || !dpdem_eligible)
        return set_err(h, DEM_ERR_INVALID, "setpoint / setpoint_next / v_water / dpdem_eligible is NULL");
    if (out->positions == in->positions || out->velocities == in->velocities || out->rotations == in->rotations ||
        out->angular_vels == in->angular_vels)
        return set_err(h, DEM_ERR_ALIAS, "output element kinematics alias the input");
    if (h->nsys > 1)
        return set_err(h, DEM_ERR_INVALID, "a handle with several systems steps through dem_scan_segment");
    CUDA_TRY(h, cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    // pack [setpoint, setpoint_next] into the (1,6) row the kernel reads
    const size_t es = h->esz;
    void* sprow = h->sprow;
    CUDA_TRY(h, cudaMemcpyAsync(sprow, setpoint, es * 3, cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync((char*)sprow + es * 3, setpoint_next, es * 3, cudaMemcpyDeviceToDevice, st));
    if (h->dtype == DEM_F32)
        rc = launch<float>(h, in, out, ship_in, ship_out, 1, sprow, v_water, v_water_ship, dpdem_eligible, diag,
                           nullptr, st);
    else
        rc = launch<double>(h, in, out, ship_in, ship_out, 1, sprow, v_water, v_water_ship, dpdem_eligible, diag,
                            nullptr, st);
    return rc;
}

int dem_scan_segment(DemHandle* h, const DemIceState* in, DemIceState* out, const DemShipState* ship_in,
                     DemShipState* ship_out, int32_t K, const void* setpoints_K6, const void* v_water_Kn2,
                     const void* v_water_ship_K2, DemHistory* hist, void* stream) {
    if (!h) return DEM_ERR_INVALID;
    int rc;
    if (K < 1) return set_err(h, DEM_ERR_INVALID, "K must be >= 1");
    if ((long long)K * dem::phases_per_frame(h->P.n_ice_steps) > (long long)INT_MAX / 2)
        return set_err(h, DEM_ERR_INVALID, "K = %d frames is too many for one call", (int)K);
    if ((rc = check_state(h, in, "input"))) return rc;
    if ((rc = check_state(h, out, "output"))) return rc;
    if ((rc = check_ship(h, ship_in, "input"))) return rc;
    if ((rc = check_ship(h, ship_out, "output"))) return rc;
    if (!setpoints_K6 || !v_water_Kn2) return set_err(h, DEM_ERR_INVALID, "setpoints / v_water is NULL");
    if (out->positions == in->positions || out->velocities == in->velocities || out->rotations == in->rotations ||
        out->angular_vels == in->angular_vels)
        return set_err(h, DEM_ERR_ALIAS, "output element kinematics alias the input");
    CUDA_TRY(h, cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    if (h->dtype == DEM_F32)
        return launch<float>(h, in, out, ship_in, ship_out, K, setpoints_K6, v_water_Kn2, v_water_ship_K2,
                             in->dpdem_floe_eligible, nullptr, hist, st);
    return launch<double>(h, in, out, ship_in, ship_out, K, setpoints_K6, v_water_Kn2, v_water_ship_K2,
                          in->dpdem_floe_eligible, nullptr, hist, st);
}

int dem_rollout_segment(DemHandle* h, const DemIceState* in, DemIceState* out, const DemShipState* ship_in,
                        DemShipState* ship_out, int32_t K, const void* controls_KQ3, const void* v_water_Kn2,
                        const void* v_water_ship_KQ2, DemHistory* hist, void* stream) {
    if (!h) return DEM_ERR_INVALID;
    int rc;
    if (K < 1) return set_err(h, DEM_ERR_INVALID, "K must be >= 1");
    if ((long long)K * dem::phases_per_frame(h->P.n_ice_steps) > (long long)INT_MAX / 2)
        return set_err(h, DEM_ERR_INVALID, "K = %d frames is too many for one call", (int)K);
    if ((rc = check_state(h, in, "input"))) return rc;
    if ((rc = check_state(h, out, "output"))) return rc;
    if ((rc = check_ship(h, ship_in, "input"))) return rc;
    if ((rc = check_ship(h, ship_out, "output"))) return rc;
    if (!controls_KQ3 || !v_water_Kn2) return set_err(h, DEM_ERR_INVALID, "controls / v_water is NULL");
    if (out->positions == in->positions || out->velocities == in->velocities || out->rotations == in->rotations ||
        out->angular_vels == in->angular_vels)
        return set_err(h, DEM_ERR_ALIAS, "output element kinematics alias the input");
    CUDA_TRY(h, cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    if (h->dtype == DEM_F32)
        return launch<float>(h, in, out, ship_in, ship_out, K, nullptr, v_water_Kn2, v_water_ship_KQ2,
                             in->dpdem_floe_eligible, nullptr, hist, st, controls_KQ3);
    return launch<double>(h, in, out, ship_in, ship_out, K, nullptr, v_water_Kn2, v_water_ship_KQ2,
                          in->dpdem_floe_eligible, nullptr, hist, st, controls_KQ3);
}

int dem_sync_status(DemHandle* h, void* stream) {
    if (!h) return DEM_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(h, cudaMemcpyAsync(h->host_status, h->status, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    int v = *h->host_status;
    if (v != 0) {
        CUDA_TRY(h, cudaMemsetAsync(h->status, 0, sizeof(int), st));
        int rc = reset_broad_phase(h, st);
        if (rc) return rc;
        CUDA_TRY(h, cudaStreamSynchronize(st));
        if (v == DEM_ERR_CAPACITY) {
            long long flags = 0;
            CUDA_TRY(h, cudaMemcpy(&flags, h->stats + 5, sizeof(flags), cudaMemcpyDeviceToHost));
            CUDA_TRY(h, cudaMemset(h->stats + 5, 0, sizeof(flags)));
            h->capacity_flags = (int)flags;
            return set_err(h, DEM_ERR_CAPACITY, "%s%s%s capacity exceeded (max_neighbors=%d, bucket_capacity=%d)",
                           (flags & 2) ? "neighbour-list" : "", (flags & 3) == 3 ? " and " : "",
                           (flags & 1) ? "grid-bucket" : "", h->P.max_neighbors, h->P.bucket_capacity);
        }
        if (v == DEM_ERR_TIMEOUT) return set_err(h, DEM_ERR_TIMEOUT, "grid barrier wait exceeded its limit");
        return set_err(h, v, "device status %d", v);
    }
    return DEM_OK;
}

int dem_set_capacity(DemHandle* h, int32_t max_neighbors, int32_t bucket_capacity) {
    if (!h) return DEM_ERR_INVALID;
    if (max_neighbors < 1 || max_neighbors > dem::kMaxNbLocal)
        return set_err(h, DEM_ERR_INVALID, "max_neighbors outside [1,%d]", dem::kMaxNbLocal);
    if (bucket_capacity < 1) return set_err(h, DEM_ERR_INVALID, "bucket_capacity must be >= 1");
    CUDA_TRY(h, cudaSetDevice(h->device));
    CUDA_TRY(h, cudaDeviceSynchronize());
    h->P.max_neighbors = max_neighbors;
    h->P.bucket_capacity = bucket_capacity;
    int rc = alloc_neighbors(h);
    if (rc) return rc;
    rc = reset_broad_phase(h, 0);
    if (rc) return rc;
    CUDA_TRY(h, cudaDeviceSynchronize());
    return DEM_OK;
}

int dem_set_launch_mode(DemHandle* h, int32_t mode) {
    if (!h) return DEM_ERR_INVALID;
    if (mode != DEM_LAUNCH_PERSISTENT && mode != DEM_LAUNCH_PHASED) return set_err(h, DEM_ERR_INVALID, "bad launch mode");
    h->mode = mode;
    return DEM_OK;
}

int dem_set_work_split(DemHandle* h, int32_t force_split, int32_t mark_split) {
    if (!h) return DEM_ERR_INVALID;
    if (force_split < DEM_SPLIT_AUTO || force_split > DEM_SPLIT_WARP || mark_split < DEM_SPLIT_AUTO ||
        mark_split > DEM_SPLIT_WARP)
        return set_err(h, DEM_ERR_INVALID, "bad work split");
    h->force_split = force_split;
    h->mark_split = mark_split;
    return DEM_OK;
}

int dem_get_info(DemHandle* h, DemInfo* info) {
    if (!h || !info) return DEM_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->device));
    long long st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    CUDA_TRY(h, cudaMemcpy(st, h->stats, sizeof(st), cudaMemcpyDeviceToHost));
    info->grid_blocks = h->grid_blocks;
    info->threads_per_block = dem::kThreads;
    info->neighbor_rebuilds = st[0];
    info->max_neighbor_count = (int)st[1];
    info->max_bucket_count = (int)st[2];
    info->hash_buckets = h->n_buckets;
    info->cell_size = 2.0 * h->r_max + h->P.skin;
    info->escaped_total = st[3];
    info->rebuilt_lists_total = st[4];
    info->capacity_flags = h->capacity_flags;
    return DEM_OK;
}

int dem_set_profiling(DemHandle* h, int32_t on) {
    if (!h) return DEM_ERR_INVALID;
    h->profiling = on != 0;
    return DEM_OK;
}

int dem_get_phase_times(DemHandle* h, int64_t* pairs, int32_t max_pairs, int32_t* count, int64_t* start_ns) {
    if (!h || !count) return DEM_ERR_INVALID;
    CUDA_TRY(h, cudaSetDevice(h->device));
    std::vector<unsigned long long> buf(2 + 2 * (size_t)dem::kMaxPhaseTimes);
    CUDA_TRY(h, cudaDeviceSynchronize());
    CUDA_TRY(h, cudaMemcpy(buf.data(), h->ptimes, sizeof(unsigned long long) * buf.size(), cudaMemcpyDeviceToHost));
    int c = (int)std::min<unsigned long long>(buf[0], (unsigned long long)dem::kMaxPhaseTimes);
    c = std::min(c, std::max(max_pairs, 0));
    for (int i = 0; i < c && pairs; ++i) {
        pairs[2 * i] = (int64_t)buf[2 + 2 * i];
        pairs[2 * i + 1] = (int64_t)buf[3 + 2 * i];
    }
    *count = c;
    if (start_ns) *start_ns = (int64_t)buf[1];
    return DEM_OK;
}

int dem_debug_fail_barrier(DemHandle* h, int32_t phase) {
    if (!h || phase < 0) return DEM_ERR_INVALID;
    if (h->mode != DEM_LAUNCH_PERSISTENT)
        return set_err(h, DEM_ERR_INVALID, "barrier faults apply to persistent launches only");
    h->fail_phase = phase;
    return DEM_OK;
}

int dem_get_error(DemHandle* h, char* buf, size_t len) {
    if (!h || !buf || len == 0) return DEM_ERR_INVALID;
    std::snprintf(buf, len, "%s", h->err.c_str());
    return DEM_OK;
}

int dem_ship_rollout(const DemParams* params, int32_t dtype, int32_t n_rollouts, int32_t horizon, const void* eta0,
                     const void* nu0, const void* controls, const void* v_water_ship, void* eta_hist, void* nu_out,
                     void* stream) {
    if (!params || (dtype != DEM_F32 && dtype != DEM_F64) || n_rollouts < 1 || horizon < 1 || !eta0 || !nu0 ||
        !controls || !eta_hist)
        return DEM_ERR_INVALID;
    const int blocks = (n_rollouts + 127) / 128;
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == DEM_F32)
        ship_rollout_kernel<float><<<blocks, 128, 0, st>>>(*params, n_rollouts, horizon, (const float*)eta0,
                                                           (const float*)nu0, (const float*)controls,
                                                           (const float*)v_water_ship, (float*)eta_hist,
                                                           (float*)nu_out);
    else
        ship_rollout_kernel<double><<<blocks, 128, 0, st>>>(*params, n_rollouts, horizon, (const double*)eta0,
                                                            (const double*)nu0, (const double*)controls,
                                                            (const double*)v_water_ship, (double*)eta_hist,
                                                            (double*)nu_out);
    return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

int dem_debug_record_contacts(DemHandle* h, int32_t* pairs, int32_t capacity, int32_t* marks, int32_t max_marks,
                              uint32_t* count) {
    if (!h) return DEM_ERR_INVALID;
    if (!pairs) {
        h->crec = nullptr;
        h->crec_cnt = nullptr;
        h->crec_marks = nullptr;
        h->crec_cap = h->crec_max_marks = 0;
        return DEM_OK;
    }
    if (capacity < 0 || max_marks < 0 || !count || (max_marks > 0 && !marks))
        return set_err(h, DEM_ERR_INVALID, "dem_debug_record_contacts: bad arguments");
    h->crec = reinterpret_cast<int2*>(pairs);
    h->crec_cnt = count;
    h->crec_cap = capacity;
    h->crec_marks = marks;
    h->crec_max_marks = max_marks;
    return DEM_OK;
}

int dem_destroy(DemHandle* h) {
    if (!h) return DEM_OK;
    cudaSetDevice(h->device);
    cudaDeviceSynchronize();
    for (void* p : h->allocs) cudaFree(p);
    h->allocs.clear();
    if (h->host_status) cudaFreeHost(h->host_status);
    delete h;
    return DEM_OK;
}

}  // extern "C"

// ════════════════════════════════════════════════════════════════════════════
// dem_ship_contact_noalloc: the frame step's ship-contact test with its
// near-element list in a static device array instead of handle scratch.
// ════════════════════════════════════════════════════════════════════════════
namespace {

constexpr int kNoAllocMax = DEM_CONTACT_NOALLOC_MAX_ELEMENTS;
// bytes [0, 4): near-element count; from byte 256: the near-element list
constexpr size_t kNoAllocListOffset = 256;
constexpr size_t kNoAllocBytes = kNoAllocListOffset + sizeof(int) * (size_t)kNoAllocMax;
static __device__ __align__(256) unsigned char g_contact_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocDevice {
    unsigned char* scratch = nullptr;  // device address of g_contact_scratch
    int sm_count = 0;
};
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];

template <typename T>
struct ContactArgs {
    int n, V, S, E;
    const T* polys;
    const uint8_t* pmask;
    const T* pos;
    const T* rot;
    const T* hull;
    const T* eta;
    double half_len, half_beam;
    T t_samp[dem::kMaxEdgeSamples];
    T* pen;
    T* nrm;
    int* near_cnt;
    int* near_list;
};

// Elements whose bounding circle reaches the ship go to the near list; the
// rest get pen = 0 and a zero normal, which is what all of their point tests
// return (every query point lies within the element's vertex radius of its
// centroid, every hull point within the hull reach of the ship).
template <typename T>
__global__ void __launch_bounds__(dem::kThreads) noalloc_cull_kernel(const __grid_constant__ ContactArgs<T> c) {
    __shared__ double s_part[dem::kThreads / 32];
    double r = 0.0;
    for (int i = threadIdx.x; i < c.S; i += blockDim.x)
        r = fmax(r, hypot((double)c.hull[2 * i], (double)c.hull[2 * i + 1]));
    for (int off = 16; off > 0; off >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, off));
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = r;
    __syncthreads();
    double reach = hypot(c.half_len, c.half_beam);  // corners of the analytic hull box
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) reach = fmax(reach, s_part[w]);
    reach = reach * (1.0 + 1e-5) + 1e-3;
    const double sx = (double)c.eta[0], sy = (double)c.eta[1];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < c.n; e += gridDim.x * blockDim.x) {
        const T* lp = c.polys + (size_t)e * c.V * 2;
        double vr = 0.0;
        for (int k = 0; k < c.V; ++k) vr = fmax(vr, hypot((double)lp[2 * k], (double)lp[2 * k + 1]));
        const double lim = reach + vr * (1.0 + 1e-5) + 1e-4;
        const double dx = (double)c.pos[2 * e] - sx, dy = (double)c.pos[2 * e + 1] - sy;
        // NaN positions stay on the exact path (the comparison is false)
        if (!(dx * dx + dy * dy > lim * lim * 1.0001)) {
            c.near_list[atomicAdd(c.near_cnt, 1)] = e;
        } else {
            c.pen[e] = T(0);
            if (c.nrm) {
                c.nrm[2 * e] = T(0);
                c.nrm[2 * e + 1] = T(0);
            }
        }
    }
}

// One warp per near element: pass 1 (the element's vertices and edge samples
// against the analytic hull), pass 2 (hull outline points inside the
// element's polygon), element-wise deepest with the reference's first-index
// ties (jax_geometry.py:515-594).
template <typename T>
__global__ void __launch_bounds__(dem::kThreads) noalloc_near_kernel(const __grid_constant__ ContactArgs<T> c) {
    extern __shared__ double noalloc_smem[];
    T* hullw = reinterpret_cast<T*>(noalloc_smem);
    dem::HullPose<T> H;
    H.sx = c.eta[0];
    H.sy = c.eta[1];
    const T spsi = c.eta[2];
    dem::jsincos(-spsi, &H.s_neg, &H.c_neg);
    dem::jsincos(spsi, &H.s_h, &H.c_h);
    H.hl = T(c.half_len);
    H.hb = T(c.half_beam);
    H.hb005 = T(c.half_beam * 0.05);
    for (int i = threadIdx.x; i < c.S; i += blockDim.x) {
        const T lx = c.hull[2 * i], ly = c.hull[2 * i + 1];
        hullw[2 * i] = lx * H.c_h + ly * (-H.s_h) + H.sx;
        hullw[2 * i + 1] = lx * H.s_h + ly * H.c_h + H.sy;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nnear = *((volatile int*)c.near_cnt);
    const int V = c.V, E = c.E, P1 = V * (1 + E);
    for (int q = warp; q < nnear; q += nwarps) {
        const int e = c.near_list[q];
        const T px = c.pos[2 * e], py = c.pos[2 * e + 1];
        T cs, sn;
        dem::jsincos(c.rot[e], &sn, &cs);
        const T* lp = c.polys + (size_t)e * V * 2;
        const uint8_t* mk = c.pmask + (size_t)e * V;
        auto wv = [&](int k, T& x, T& y) {
            const T lx = lp[2 * k], ly = lp[2 * k + 1];
            x = cs * lx - sn * ly + px;
            y = sn * lx + cs * ly + py;
        };
        dem::Best<T> b1 = {T(0), T(0), T(0), INT_MAX};
        for (int pt = lane; pt < P1; pt += 32) {
            const int k = pt / (1 + E), j = pt % (1 + E);
            T qx, qy;
            wv(k, qx, qy);
            if (j > 0) {
                T x1, y1;
                wv((k + 1 == V) ? 0 : k + 1, x1, y1);
                const T t = c.t_samp[j - 1];
                const T omt = T(1) - t;
                qx = qx * omt + x1 * t;
                qy = qy * omt + y1 * t;
            }
            T p, nx, ny;
            dem::hull_point(H, qx, qy, p, nx, ny);
            if (!mk[k]) p = T(0);
            dem::better(b1, p, nx, ny, pt);
        }
        b1 = dem::warp_best(b1);
        T wx[dem::kMaxV], wy[dem::kMaxV], mx[dem::kMaxV], my[dem::kMaxV], mc[dem::kMaxV];
        for (int k = 0; k < V; ++k) {
            wv(k, wx[k], wy[k]);
            const bool m = mk[k] != 0;
            mx[k] = m ? wx[k] : T(0);
            my[k] = m ? wy[k] : T(0);
            mc[k] = m ? T(1) : T(0);
        }
        const T n_real = dem::jmax(dem::np_pairwise_sum(mc, V), T(1));
        const T cxc = dem::np_pairwise_sum(mx, V) / n_real;
        const T cyc = dem::np_pairwise_sum(my, V) / n_real;
        dem::Best<T> b2 = {T(0), T(0), T(0), INT_MAX};
        for (int si = lane; si < c.S; si += 32) {
            const T hx = hullw[2 * si], hy = hullw[2 * si + 1];
            int crossings = 0;
            T dmin = T(0);
            int kbest = 0;
            for (int k = 0; k < V; ++k) {
                const int k1 = (k + 1 == V) ? 0 : k + 1;
                const T xi = wx[k], yi = wy[k], xj = wx[k1], yj = wy[k1];
                const bool cond_y = (yi > hy) != (yj > hy);
                const T x_int = (xj - xi) * (hy - yi) / (yj - yi + T(1e-10)) + xi;
                if (cond_y && (hx < x_int)) ++crossings;
                const T vx = xj - xi, vy = yj - yi;
                const T c1 = (hx - xi) * vx + (hy - yi) * vy;
                const T c2 = vx * vx + vy * vy + T(1e-20);
                const T t = dem::jclip(c1 / c2, T(0), T(1));
                const T ddx = hx - (xi + t * vx), ddy = hy - (yi + t * vy);
                const T d = dem::jsqrt(ddx * ddx + ddy * ddy + T(1e-20));
                if (k == 0 || d < dmin) {
                    dmin = d;
                    kbest = k;
                }
            }
            T p = T(0), nx = T(0), ny = T(0);
            if ((crossings % 2) == 1) {
                const int k = kbest, k1 = (k + 1 == V) ? 0 : k + 1;
                const T ex = wx[k1] - wx[k], ey = wy[k1] - wy[k];
                T nxe = ey, nye = -ex;
                const T nlen = dem::jsqrt(nxe * nxe + nye * nye + T(1e-20));
                nxe = nxe / nlen;
                nye = nye / nlen;
                const T midx = (wx[k] + wx[k1]) / T(2), midy = (wy[k] + wy[k1]) / T(2);
                if ((midx - cxc) * nxe + (midy - cyc) * nye < T(0)) {
                    nxe = -nxe;
                    nye = -nye;
                }
                p = dmin;
                nx = nxe;
                ny = nye;
            }
            dem::better(b2, p, nx, ny, si);
        }
        b2 = dem::warp_best(b2);
        if (lane == 0) {
            const bool use2 = (b2.p > T(0)) && (b2.p > b1.p);
            c.pen[e] = use2 ? b2.p : b1.p;
            if (c.nrm) {
                c.nrm[2 * e] = use2 ? b2.nx : b1.nx;
                c.nrm[2 * e + 1] = use2 ? b2.ny : b1.ny;
            }
        }
    }
}

template <typename T>
int noalloc_contact(const NoAllocDevice& d, ContactArgs<T>& c, const double* t_samp, cudaStream_t st) {
    for (int i = 0; i < dem::kMaxEdgeSamples; ++i) c.t_samp[i] = (T)t_samp[i];
    // the count must start at zero; the list keeps the previous call's entries
    // but only the first `count` are read
    if (cudaMemsetAsync(c.near_cnt, 0, sizeof(int), st) != cudaSuccess) return DEM_ERR_CUDA;
    const int blocks = (int)std::min<long long>(((long long)c.n + dem::kThreads - 1) / dem::kThreads,
                                                (long long)d.sm_count * 8);
    noalloc_cull_kernel<T><<<blocks, dem::kThreads, 0, st>>>(c);
    if (cudaGetLastError() != cudaSuccess) return DEM_ERR_CUDA;
    const size_t smem = (size_t)c.S * 2 * sizeof(T) + 16;
    noalloc_near_kernel<T><<<d.sm_count * 4, dem::kThreads, smem, st>>>(c);
    if (cudaGetLastError() != cudaSuccess) return DEM_ERR_CUDA;
    return DEM_OK;
}

}  // namespace

extern "C" int dem_ship_contact_noalloc(int32_t dtype, int32_t n, int32_t max_v, const void* local_polys_padded,
                                        const uint8_t* poly_mask, const void* positions, const void* rotations,
                                        int32_t n_hull, const void* ship_hull_local, double half_len,
                                        double half_beam, int32_t n_edge_samples, const void* ship_eta,
                                        void* pen_max, void* normals, void* stream) {
    if (dtype != DEM_F32 && dtype != DEM_F64) return DEM_ERR_INVALID;
    if (n < 0) return DEM_ERR_INVALID;
    if (n > kNoAllocMax) return DEM_ERR_CAPACITY;  // the static scratch holds at most kNoAllocMax elements
    if (max_v < 1 || max_v > dem::kMaxV || n_hull < 0 || n_hull > dem::kMaxHull || n_edge_samples < 0 ||
        n_edge_samples > dem::kMaxEdgeSamples)
        return DEM_ERR_INVALID;
    if (!local_polys_padded || !poly_mask || !positions || !rotations || !ship_eta || !pen_max ||
        (n_hull > 0 && !ship_hull_local))
        return DEM_ERR_INVALID;
    if (n == 0) return DEM_OK;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return DEM_ERR_CUDA;
    if (dev < 0 || dev >= kNoAllocMaxDevices) return DEM_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    // Outside stream capture the address is looked up again on every call, so
    // a device reset (which reloads the module at a new address) leaves no
    // stale pointer; under capture, where the lookup may load the module, the
    // address of the last call outside capture on this device is used.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) return DEM_ERR_CUDA;
    NoAllocDevice d;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        NoAllocDevice& slot = g_noalloc_dev[dev];
        if (cap == cudaStreamCaptureStatusNone) {
            // with this device current: the address of its copy of the static scratch array
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_contact_scratch) != cudaSuccess || !p) return DEM_ERR_CUDA;
            slot.scratch = static_cast<unsigned char*>(p);
        }
        if (!slot.scratch) return DEM_ERR_INVALID;  // first call on this device inside a capture
        if (slot.sm_count == 0) {
            int sm = 0;
            if (cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sm < 1)
                return DEM_ERR_CUDA;
            slot.sm_count = sm;
        }
        d = slot;
    }
    double t_samp[dem::kMaxEdgeSamples] = {0};
    np_linspace(1.0 / (n_edge_samples + 1), (double)n_edge_samples / (n_edge_samples + 1), n_edge_samples, t_samp);
    int* near_cnt = reinterpret_cast<int*>(d.scratch);
    int* near_list = reinterpret_cast<int*>(d.scratch + kNoAllocListOffset);
    if (dtype == DEM_F32) {
        ContactArgs<float> c{};
        c.n = n, c.V = max_v, c.S = n_hull, c.E = n_edge_samples;
        c.polys = (const float*)local_polys_padded, c.pmask = poly_mask, c.pos = (const float*)positions;
        c.rot = (const float*)rotations, c.hull = (const float*)ship_hull_local, c.eta = (const float*)ship_eta;
        c.half_len = half_len, c.half_beam = half_beam;
        c.pen = (float*)pen_max, c.nrm = (float*)normals, c.near_cnt = near_cnt, c.near_list = near_list;
        return noalloc_contact<float>(d, c, t_samp, st);
    }
    ContactArgs<double> c{};
    c.n = n, c.V = max_v, c.S = n_hull, c.E = n_edge_samples;
    c.polys = (const double*)local_polys_padded, c.pmask = poly_mask, c.pos = (const double*)positions;
    c.rot = (const double*)rotations, c.hull = (const double*)ship_hull_local, c.eta = (const double*)ship_eta;
    c.half_len = half_len, c.half_beam = half_beam;
    c.pen = (double*)pen_max, c.nrm = (double*)normals, c.near_cnt = near_cnt, c.near_list = near_list;
    return noalloc_contact<double>(d, c, t_samp, st);
}
