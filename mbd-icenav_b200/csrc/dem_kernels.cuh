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
constexpr int kMaxPhaseTimes = 4096;

// Phases of one frame: cull, near contact, contact forces, reduce, then per
// substep escape round, all-lists rebuild and force, and last fracture.
__host__ __device__ constexpr int phases_per_frame(int k_sub) { return 5 + 3 * k_sub; }
// work items per thread and step whose loads are issued together in the
// per-frame bond-record build and in the fracture update (more than one adds
// registers that the force loop then spills)
#ifndef DEM_SLOT_BATCH
#define DEM_SLOT_BATCH 1
#endif
#ifndef DEM_MIN_BLOCKS
#define DEM_MIN_BLOCKS 2  // resident CTAs per SM the register allocation targets
#endif

// Per-frame record of one bond slot (see phase_reduce): partner index with the
// slot's role in the sign bit, rest length, stiffness E*mean(h)*factor, and
// (1 - damage), or -1 when the bond adds no force this frame (broken, or its
// endpoints differ in active state; jax_simulation.py:86-96).
template <typename T> struct SlotRec;
template <> struct __align__(16) SlotRec<float> {
    int o;
    float rest, stiff, omd;
};
template <> struct __align__(16) SlotRec<double> {
    int o, pad;
    double rest, stiff, omd;
};

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

// Force-phase constants in the kernel's dtype, converted once on the host and
// read from the kernel parameter (constant bank) rather than held in registers.
template <typename T>
struct ForceConst {
    T hf, hexp, mu, fcap, c_drag, href, lin, c_rot, dti, damp, alo, ahi, vclip, pclip;
    int h15;  // hertz_exponent == 1.5: overlap * sqrt(overlap) instead of pow
};

template <typename T>
struct KArgs {
    DemParams P;
    int n, V, nb, nf, S, K, k_sub, nchunks;
    // independent systems (an ice window with its own ship) advanced together;
    // 1 for a plain field.  Elements of system s are [sys_start_s, sys_end[s]),
    // its force chunks [part_base[s], part_base[s + 1]).
    int nsys;
    const int* sys_of;        // (n) system of each element (read when nsys > 1)
    const int* floe_sys;      // (nf) system of each floe (read when nsys > 1)
    const int2* chunk_info;   // (nchunks) {system, first element} of each chunk of kThreads elements
    const int* sys_end;       // (nsys) one past each system's last element
    const int* part_base;     // (nsys + 1) first chunk of each system
    const T* u_ctrl;          // (K, nsys, 3) body-frame ship controls of planner rollouts, or NULL
    int n_buckets, bucket_cap, max_nb, mode;
    int force_split, mark_split;  // DEM_SPLIT_*: how substep work is split (tests and tuning)
    T k_n, k_s, min_bstr, cell, skin, hull_r;
    // escape thresholds: a substep whose successor is a check substep (s + 1 a
    // multiple of esc_period) tests against esc_h_check, every other one
    // against esc_h_urgent (the limit of an element's next use)
    T esc_h_check, esc_h_urgent;
    int esc_period;
    // lazy escapes (with esc_period 2): before an even substep s (s + 1 < k_sub)
    // an element beyond esc_h_check but within esc_h_urgent goes to lazy_list[s];
    // the force phase of s re-references it and marks its neighbourhood for a
    // rebuild at s + 1, beside the force work, instead of an escape phase
    int lazy;
    int* lazy_list;     // (n) lazily escaped elements of the current detection
    int* lazy_cnt;      // (k_sub + 2) per substep
    T t_samp[kMaxEdgeSamples];
    // static data (caller-owned)
    const T* polys;
    const uint8_t* pmask;
    const T *mass, *inertia, *radii, *areas, *thick, *rest, *bstr, *sbar, *hull;
    const int *bi, *bj, *floe_of;
    // derived at create
    const int* boff;    // (n+1) CSR offsets of per-element bond slots
    const int2* bslot;  // (2 nb) {bond | role<<31, partner}; role 0: element is bond_i
    const T* slot_rest; // (2 nb) rest length of each slot's bond
    const T* slot_stiff;// (2 nb) E * mean(h) * factor of each slot's bond
    const T* vert_r;    // (n) max local vertex radius, rounded up
    // broad phase: grids, reference positions and lists persist across calls
    int* bcnt;          // (n_buckets) grid-hash bucket fill
    int* bitems;        // (n_buckets * bucket_cap) entries; stale ones are filtered by home cell
    int2* ecell;        // (n) home cell of each reference position
    int* ncnt;          // (n) neighbour count
    int* nbr;           // (max_nb * n) neighbour lists, slot-major
    T* pos_ref;         // (n,2) reference positions (NaN before the first build)
    unsigned* dirty;    // (n) stamp of the round whose list rebuild the element needs
    int* bflag;         // (n_buckets) bucket queued for compaction
    int* comp_list;     // (n_buckets) buckets to compact at the next frame start
    int* comp_cnt;      // (1) queued buckets
    unsigned* esc_cnt;  // (k_sub + 2) escaped elements found before substep s
    // per-frame scratch
    int* near_list;     // (n) elements whose bounding circle reaches the hull
    int* near_cnt;      // (1)
    T *cpen, *cnx, *cny;  // (n) max penetration contact per element
    T* soi;             // (n,2) ship force on ice (with buoyancy), constant over substeps
    T* fraw;            // (n) contact force magnitude before the thrust cap
    uint8_t* crack;     // (n) element touches a broken bond
    int* fcoll;         // (nf) floe touched by the ship this frame
    unsigned long long* fmax;  // (nf) max force magnitude per floe (ordered bits)
    double* part;       // (nchunks * 3) per-chunk sums: soi_x, soi_y, moment
    // per force chunk, for phase_cforce in a call's later frames
    uint8_t* cwarm;     // (nchunks) an element in contact or submerged at the last cforce
    unsigned* cnear;    // (nchunks) frame stamp of the last frame with a near element
    T* kin[2];          // (n,4) {x, y, radius, radius^3} of the substep being read / written
    T* kvel[2];         // (n,2) {vx, vy} of the substep being read / written
    int* esc_list;      // (n) escaped elements of the current detection
    int* dirty_list;    // (n) elements whose list is rebuilt
    int* dirty_cnt;     // (k_sub + 2) lists to rebuild, per substep
    int* work_cnt;      // (k_sub + 2) element chunks handed out dynamically, per substep
    int* act_list;      // (kActLists * n) elements active this frame, then by work bin (built by phase_reduce)
    unsigned* bstamp;   // (nb) frame stamp of the bonds with an active end (set by phase_reduce)
    int* fb_list;       // (nb) the frame's bonds with an active end, each once (phase_reduce)
    int* fb_cnt;        // (1) entries of fb_list
    int* act_cnt;       // (kActLists) entries of the list and of each bin
    unsigned round_base;  // first dirty stamp of this call minus one (advanced by the host)
    int fail_phase;       // test hook: the last CTA skips the barrier after this phase (-1: off)
    ForceConst<T> fc;     // force-phase constants
    const int* slot_owner;  // (2 nb) element that owns each bond slot
    T *sp_rot[2], *sp_avel[2];  // substep ping-pong of own-element angles
    void* slotrec;      // (2 nb) SlotRec<T>: per-frame bond slot records
    const T* r3;        // (n) radius^3 (dtype pow, once at create)
    const T* econ;      // (n,4) {mass, inertia, thickness, area}, packed once at create
    double* fscal;      // (4) frame scalars: thrust scale, F_x, F_y, M
    unsigned long long* ptimes;  // (2 * kMaxPhaseTimes) [phase, globaltimer ns] or null
    // call arguments
    IcePtrs<T> in, out;  // frame 0 reads in; every frame writes out (in place after frame 0)
    ShipPtrs<T> ship_in, ship_out, ship_tmp[2];
    const T* setpoints;   // (K,6)
    const T* vw;          // (K,n,2)
    const T* vws;         // (K,2) or null
    const uint8_t* elig0; // dpdem_eligible argument of frame 0
    T *d_pen, *d_fmag, *d_F, *d_J;
    T *h_pos, *h_rot, *h_eta, *h_sub, *h_J, *h_F;
    uint8_t* h_intact;
    unsigned* bar;        // top arrival word of the grid barrier
    unsigned* bar_groups; // group arrival words, kBarGroupStride apart (kBarGroup > 0)
    // contact-set recording (parity aid, off when crec is null): every pair
    // whose contact term a force phase computes goes to crec as {e, o}, seen
    // from the active element e; crec_marks[f * k_sub + s] = pairs recorded
    // up to the end of substep s of frame f
    int2* crec;
    unsigned* crec_cnt;
    int crec_cap, crec_max_marks;
    int* crec_marks;
    int* status;
    long long* stats;     // [rounds, max list, max bucket, re-referenced, lists rebuilt, overflow flags]
};

template <typename T> struct vec4_of;
template <> struct vec4_of<float> { typedef float4 type; };
template <> struct vec4_of<double> { typedef double4 type; };

template <typename T>
__device__ __forceinline__ typename vec4_of<T>::type ld4(const T* p, int i) {
    return reinterpret_cast<const typename vec4_of<T>::type*>(p)[i];
}

// ─── per-frame pointer bundle ───────────────────────────────────────────────
template <typename T>
struct Frame {
    int f;
    IcePtrs<T> src, dst;
    ShipPtrs<T> ship_src, ship_dst;
    const uint8_t* elig_in;
    const T* vw;
    const T* sp;   // (nsys, 6) [setpoint, setpoint_next] of this frame
    const T* vws;  // (nsys, 2) current at the ships, or NULL (none)
};

template <typename T>
__device__ __forceinline__ Frame<T> make_frame(const KArgs<T>& a, int f) {
    Frame<T> F;
    F.f = f;
    const int K = a.K;
    // frame 0 reads the call's input and writes all of `out`; later frames update
    // `out` in place (every phase reads and writes only its own element or bond,
    // or reads a partner's flag that only turns on), so state that does not
    // change (frozen elements, bonds between them) is not copied frame to frame
    F.dst = a.out;
    F.src = (f == 0) ? a.in : a.out;
    F.ship_dst = (f == K - 1) ? a.ship_out : a.ship_tmp[f & 1];
    F.ship_src = (f == 0) ? a.ship_in : a.ship_tmp[(f - 1) & 1];
    F.elig_in = (f == 0) ? a.elig0 : F.src.elig;
    F.vw = a.vw + (size_t)f * a.n * 2;
    F.sp = a.setpoints ? a.setpoints + (size_t)f * a.nsys * 6 : nullptr;
    F.vws = a.vws ? a.vws + (size_t)f * a.nsys * 2 : nullptr;
    return F;
}

// Stamp of frame f of this call: the dirty stamp of its first rebuild round,
// unique since the stamps were last cleared (never 0)
template <typename T>
__device__ __forceinline__ unsigned frame_stamp(const KArgs<T>& a, const Frame<T>& F) {
    return a.round_base + (unsigned)(F.f * a.k_sub) + 1u;
}

// ─── grid barrier (bounded) ──────────────────────────────────────────────────
// Returns false (and records DEM_ERR_TIMEOUT) if the wait exceeds its limit;
// callers then return.
//
// Arrival counts use flip words: of the n arrivals at a word, the first CTA of
// the set adds 2^31 - (n - 1) and every other one adds 1, so the arrivals of
// one barrier sum to 2^31, bit 31 of the word flips exactly at the last
// arrival (the one whose add carries into bit 31), and no word needs a reset
// between barriers.  With DEM_BAR_GROUP = g > 0 the CTAs arrive in groups of g
// consecutive CTAs, each group on a word of its own 128-byte line
// (a.bar_groups); the last arrival of a group carries it to the top word
// a.bar, and every CTA polls a.bar.  The hottest word then takes
// ceil(grid / g) atomics per barrier instead of one per CTA.
#ifndef DEM_BAR_GROUP
#define DEM_BAR_GROUP 0
#endif
constexpr int kBarGroup = DEM_BAR_GROUP;
constexpr int kBarGroupStride = 32;  // words between group counters (128 bytes)

template <typename T>
__device__ bool grid_barrier(const KArgs<T>& a) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        // the arrivals are releases at GPU scope, cumulative over the CTA's
        // writes ordered before them by __syncthreads; a group arrival is an
        // acquire too, so that the group's last arrival, which reads every
        // earlier arrival of its group, carries their writes into its release
        // on the top word; the polls are acquires: the pattern orders every
        // CTA's phase writes before every CTA's next phase
        unsigned old;
        if (kBarGroup > 0) {
            const unsigned g = blockIdx.x / (unsigned)kBarGroup;
            const unsigned first = g * (unsigned)kBarGroup;
            const unsigned size = min((unsigned)kBarGroup, gridDim.x - first);
            const unsigned ginc = (blockIdx.x == first) ? 0x80000000u - (size - 1u) : 1u;
            const unsigned gold = atom_add_acqrel_u32(a.bar_groups + (size_t)g * kBarGroupStride, ginc);
            const unsigned n_groups = (gridDim.x + (unsigned)kBarGroup - 1u) / (unsigned)kBarGroup;
            if (((gold + ginc) ^ gold) & 0x80000000u) {
                // this group's last arrival: carry the group to the top word
                const unsigned tinc = (g == 0u) ? 0x80000000u - (n_groups - 1u) : 1u;
                atom_add_release_u32(a.bar, tinc);
            }
            // every word flips once per barrier, so the group word's bit 31
            // before this arrival is the top word's before the barrier
            old = gold;
        } else {
            const unsigned inc = (blockIdx.x == 0) ? 0x80000000u - (gridDim.x - 1u) : 1u;
            old = atom_add_release_u32(a.bar, inc);
        }
        int ok = 1;
        unsigned long long t0 = 0;
        for (unsigned it = 0; ((ld_acquire_u32(a.bar) ^ old) & 0x80000000u) == 0u; ++it) {
            if ((it & 63u) != 0u) continue;  // the time limit is read every 64 polls
            const unsigned long long t = globaltimer_ns();
            if (it == 0) {
                t0 = t;
            } else if (t - t0 > kBarrierLimitNs) {
                // a CTA that gives up returns; every other CTA's wait then ends
                // at its own limit, so the launch always finishes
                atomicMax(a.status, DEM_ERR_TIMEOUT);
                ok = 0;
                break;
            }
        }
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
// The system id is part of the key: systems that occupy the same space (planner
// rollouts on overlapping windows) hash their cells to different buckets, so a
// neighbourhood scan reads its own system's entries only.
__device__ __forceinline__ int bucket_of(int2 c, int sys, int n_buckets) {
    unsigned h = (unsigned)c.x * 73856093u ^ (unsigned)c.y * 19349663u ^ (unsigned)sys * 83492791u;
    return (int)(h & (unsigned)(n_buckets - 1));
}
template <typename T>
__device__ __forceinline__ int sys_id(const KArgs<T>& a, int e) {
    return a.nsys > 1 ? a.sys_of[e] : 0;
}

// Neighbour lists are Verlet lists over reference positions: list(e) holds every
// o with |ref_e - ref_o| < r_e + r_o + skin.  An element whose position leaves the
// ball of radius h around its reference "escapes": it takes its current
// position as new reference, and every element within reach of that new
// reference rebuilds its list.  With |p - ref| < skin/2 for every element at
// every use of the lists, any pair closer than r_e + r_o is in both lists, so the
// contact set equals the all-pairs one of the reference (jax_ice_state.py:212-214).
//
// Escapes are processed only before check substeps (s a multiple of the escape
// period P, 1 or 2).  Before a check substep the test uses h = esc_h_check,
// chosen so that h + (one substep's largest move, sqrt(2) vclip dt_ice) stays
// below skin/2: the element is then safe through the next, unchecked substep.
// Before any other substep the test uses h = esc_h_urgent = 0.4455 skin, the
// limit for the very next use; only a move larger than that bound (an input
// position outside the clip box) can trip it, and then the escape is processed
// at once.  P = 1 (the default skin) tests every substep at 0.4455 skin.

template <typename T>
__device__ __forceinline__ bool escaped_from(T px, T py, T rx, T ry, T h) {
    const bool fp = jfinite(px) && jfinite(py);
    const bool fr = jfinite(rx) && jfinite(ry);
    if (fp != fr) return true;
    if (!fp) return false;
    // |p - ref| > h; h carries a 1 % margin so rounding of the test can only make
    // an element escape early, never late
    const T dx = px - rx, dy = py - ry;
    return dx * dx + dy * dy > h * h;
}
template <typename T>
__device__ __forceinline__ bool escaped(const KArgs<T>& a, int e, T px, T py, T h) {
    return escaped_from(px, py, a.pos_ref[2 * e], a.pos_ref[2 * e + 1], h);
}

// one atomic per CTA: add the CTA's count of `v` to *ctr (all threads must call)
__device__ __forceinline__ void cta_count_add(unsigned* ctr, int v) {
    __shared__ int s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&s_cnt, v);
    __syncthreads();
    if (threadIdx.x == 0 && s_cnt) atomicAdd(ctr, (unsigned)s_cnt);
    __syncthreads();
}

// Grid-hash buckets of fixed capacity.  An element that escapes is appended to
// the bucket of its new home cell; its old entry goes stale and is ignored
// (its home cell no longer matches) until the next compaction drops it.
template <typename T>
__device__ __forceinline__ void grid_put(const KArgs<T>& a, int e, T px, T py) {
    if (!(jfinite(px) && jfinite(py))) {
        a.ecell[e] = make_int2(INT_MIN, INT_MIN);
        return;
    }
    int2 c = cell_of(a, px, py);
    a.ecell[e] = c;
    int b = bucket_of(c, sys_id(a, e), a.n_buckets);
    int slot = atomicAdd(&a.bcnt[b], 1);
    if (slot < a.bucket_cap) {
        a.bitems[(size_t)b * a.bucket_cap + slot] = e;
    } else {
        atomicMax(a.status, DEM_ERR_CAPACITY);
        atomicOr((unsigned long long*)&a.stats[5], 1ull);  // a grid bucket overflowed
    }
    if (slot + 1 > a.bucket_cap / 2) atomicMax((unsigned long long*)&a.stats[2], (unsigned long long)(slot + 1));
}

// Warp-cooperative neighbourhood scan: the 9 stencil buckets' entries are
// spread over the lanes; `fn(o)` runs on the lane that found o.  Every element
// within r_e + r_o + skin of ref_e (double test with a margin) is visited; an
// element can be visited twice (stale + current entry in one bucket).
template <typename T, typename Fn>
__device__ __forceinline__ void warp_near_at(const KArgs<T>& a, int e, T px, T py, int2 c, Fn fn) {
    const int lane = threadIdx.x & 31;
    if (c.x == INT_MIN) return;
    const double re = (double)a.radii[e] + (double)a.skin;
    // lanes 0..8 own one stencil bucket each; warp prefix of their fills
    const int se = sys_id(a, e);
    int b = 0, m = 0;
    if (lane < 9) {
        const int2 cc = make_int2(c.x + (lane % 3) - 1, c.y + (lane / 3) - 1);
        b = bucket_of(cc, se, a.n_buckets);
        m = min(a.bcnt[b], a.bucket_cap);
    }
    int incl = m;
    for (int off = 1; off < 32; off <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int excl = incl - m;
    // uniform trip count: every lane executes every shuffle
    for (int t0 = 0; t0 < total; t0 += 32) {
        const int t = t0 + lane;
        // bucket j holding entry t: the last stencil lane whose prefix start <= t
        int q = 0, qb = 0, qe = 0;
        for (int j = 0; j < 9; ++j) {
            const int ej = __shfl_sync(0xffffffffu, excl, j);
            const int bj = __shfl_sync(0xffffffffu, b, j);
            if (t >= ej) {
                q = j;
                qb = bj;
                qe = ej;
            }
        }
        if (t >= total) continue;
        // entries are written after their slot is claimed: a concurrent insertion
        // can show an old value (-1 or a valid stale index), never an invalid one
        const int o = ((volatile const int*)a.bitems)[(size_t)qb * a.bucket_cap + (t - qe)];
        if (o < 0 || o >= a.n || o == e) continue;
        if (a.nsys > 1 && a.sys_of[o] != se) continue;  // systems never interact
        const int2 cc = make_int2(c.x + (q % 3) - 1, c.y + (q / 3) - 1);
        const int2 oc = a.ecell[o];
        if (oc.x != cc.x || oc.y != cc.y) continue;  // stale entry or hash collision
        const double ddx = (double)a.pos_ref[2 * o] - (double)px, ddy = (double)a.pos_ref[2 * o + 1] - (double)py;
        const double lim = (re + (double)a.radii[o]) * (1.0 + 1e-5) + 1e-6;
        if (ddx * ddx + ddy * ddy < lim * lim) fn(o);
    }
}

// The same neighbourhood scan by a whole CTA (every thread must call it with
// the same e): the stencil entries are spread over all threads, so the scan
// takes one or two dependent load rounds instead of the warp's several.
template <typename T, typename Fn>
__device__ __forceinline__ void block_near_at(const KArgs<T>& a, int e, T px, T py, int2 c, Fn fn) {
    __shared__ int s_b[9];
    __shared__ int s_start[10];
    if (c.x == INT_MIN) return;  // depends on e only: uniform over the CTA
    if (threadIdx.x < 9) {
        const int2 cc = make_int2(c.x + ((int)threadIdx.x % 3) - 1, c.y + ((int)threadIdx.x / 3) - 1);
        const int b = bucket_of(cc, sys_id(a, e), a.n_buckets);
        s_b[threadIdx.x] = b;
        s_start[threadIdx.x + 1] = min(a.bcnt[b], a.bucket_cap);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        s_start[0] = 0;
        for (int j = 0; j < 9; ++j) s_start[j + 1] += s_start[j];
    }
    __syncthreads();
    const int total = s_start[9];
    const double re = (double)a.radii[e] + (double)a.skin;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int q = 0;
        while (q < 8 && t >= s_start[q + 1]) ++q;
        // entries are written after their slot is claimed: a concurrent insertion
        // can show an old value (-1 or a valid stale index), never an invalid one
        const int o = ((volatile const int*)a.bitems)[(size_t)s_b[q] * a.bucket_cap + (t - s_start[q])];
        if (o < 0 || o >= a.n || o == e) continue;
        if (a.nsys > 1 && a.sys_of[o] != a.sys_of[e]) continue;  // systems never interact
        const int2 cc = make_int2(c.x + (q % 3) - 1, c.y + (q / 3) - 1);
        const int2 oc = a.ecell[o];
        if (oc.x != cc.x || oc.y != cc.y) continue;  // stale entry or hash collision
        const double ddx = (double)a.pos_ref[2 * o] - (double)px, ddy = (double)a.pos_ref[2 * o + 1] - (double)py;
        const double lim = (re + (double)a.radii[o]) * (1.0 + 1e-5) + 1e-6;
        if (ddx * ddx + ddy * ddy < lim * lim) fn(o);
    }
    __syncthreads();  // s_b / s_start are reused by the next call
}

template <typename T, typename Fn>
__device__ __forceinline__ void warp_near(const KArgs<T>& a, int e, Fn fn) {
    warp_near_at(a, e, a.pos_ref[2 * e], a.pos_ref[2 * e + 1], a.ecell[e], fn);
}

// Append `flag`-set lanes' values to list[atomicAdd(cnt)] with one atomic per warp.
__device__ __forceinline__ void warp_append(int* list, int* cnt, bool flag, int v) {
    const unsigned am = __activemask();
    const unsigned bal = __ballot_sync(am, flag);
    if (!bal) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(am) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(cnt, __popc(bal));
    base = __shfl_sync(am, base, leader);
    if (flag) list[base + __popc(bal & ((1u << lane) - 1u))] = v;
}

// Two flagged values per lane, appended with one atomic per warp (the
// frame's bond list: up to two slots per lane and step).
__device__ __forceinline__ void warp_append2(int* list, int* cnt, bool f0, int v0, bool f1, int v1) {
    const unsigned am = __activemask();
    const unsigned bal0 = __ballot_sync(am, f0), bal1 = __ballot_sync(am, f1);
    const int n0 = __popc(bal0), n = n0 + __popc(bal1);
    if (!n) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(am) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(cnt, n);
    base = __shfl_sync(am, base, leader);
    const unsigned lt = (1u << lane) - 1u;
    if (f0) list[base + __popc(bal0 & lt)] = v0;
    if (f1) list[base + n0 + __popc(bal1 & lt)] = v1;
}

// Build element e's list (one warp): candidates are gathered in shared memory,
// sorted and deduplicated, then stored so that indices above e come first
// (ascending), then indices below e (ascending) — the order in which the
// reference's scatter-adds reach e: pairs (e, j>e) through pair_i, then pairs
// (i<e, e) through pair_j (jax_simulation.py:152-162).
template <typename T>
__device__ void warp_build(const KArgs<T>& a, int e, int* sbuf, int* scnt) {
    const int lane = threadIdx.x & 31;
    if (lane == 0) *scnt = 0;
    __syncwarp();
    const int cap = 2 * kMaxNbLocal;
    warp_near(a, e, [&](int o) {
        const int slot = atomicAdd(scnt, 1);
        if (slot < cap) sbuf[slot] = o;
    });
    __syncwarp();
    const int found = *scnt;
    const int cnt = min(found, cap);
    // drop repeats (a stale and a current entry of one element), in parallel:
    // entry i stays if no earlier entry holds the same index.  All lanes walk
    // the buffer together (broadcast reads, no early exit, so the reads
    // pipeline); a lane holds entries lane, lane + 32, ...
    constexpr int kPer = (2 * kMaxNbLocal + 31) / 32;
    int v[kPer];
    bool keep[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int i = lane + 32 * k;
        v[k] = (i < cnt) ? sbuf[i] : -1;
        keep[k] = i < cnt;
    }
    if (cnt <= 64) {
#pragma unroll 4
        for (int j = 0; j < cnt; ++j) {
            const int u = sbuf[j];
            keep[0] = keep[0] && !(j < lane && u == v[0]);
            keep[1] = keep[1] && !(j < lane + 32 && u == v[1]);
        }
    } else {
#pragma unroll 2
        for (int j = 0; j < cnt; ++j) {
            const int u = sbuf[j];
#pragma unroll
            for (int k = 0; k < kPer; ++k) keep[k] = keep[k] && !(j < lane + 32 * k && u == v[k]);
        }
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < kPer; ++k)
        if (lane + 32 * k < cnt && !keep[k]) sbuf[lane + 32 * k] = -1;
    __syncwarp();
    int nk = 0, nlow = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        nk += keep[k] ? 1 : 0;
        nlow += (keep[k] && v[k] < e) ? 1 : 0;
    }
    const int w = __reduce_add_sync(0xffffffffu, nk);
    const int split = __reduce_add_sync(0xffffffffu, nlow);  // kept indices below e
    if (lane == 0) {
        if (found > cap || w > a.max_nb) {
            atomicMax(a.status, DEM_ERR_CAPACITY);
            atomicOr((unsigned long long*)&a.stats[5], 2ull);  // a neighbour list overflowed
        }
        if (w > 16) atomicMax((unsigned long long*)&a.stats[1], (unsigned long long)w);
    }
    const int m = min(w, a.max_nb);
    // slot of a kept index = its rank among the kept ones, indices above e first
    int r[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) r[k] = 0;
    if (cnt <= 64) {
#pragma unroll 4
        for (int j = 0; j < cnt; ++j) {
            const int u = sbuf[j];
            r[0] += (u >= 0 && u < v[0]) ? 1 : 0;
            r[1] += (u >= 0 && u < v[1]) ? 1 : 0;
        }
    } else {
#pragma unroll 2
        for (int j = 0; j < cnt; ++j) {
            const int u = sbuf[j];
#pragma unroll
            for (int k = 0; k < kPer; ++k) r[k] += (u >= 0 && u < v[k]) ? 1 : 0;
        }
    }
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        if (!keep[k]) continue;
        const int pos = (v[k] > e) ? r[k] - split : (w - split) + r[k];
        if (pos < m) a.nbr[(size_t)pos * a.n + e] = v[k];
    }
    if (lane == 0) a.ncnt[e] = m;
    __syncwarp();
}

// The same list build by a whole CTA (every thread must call it with the same
// e): the stencil entries are scanned in one load round (block_near_at), and
// thread t checks gathered candidate t (at most 2 kMaxNbLocal <= kThreads).
// The list equals warp_build's: the same candidates, repeats dropped, the
// same order and the same capacity flags.
template <typename T>
__device__ void block_build(const KArgs<T>& a, int e) {
    constexpr int cap = 2 * kMaxNbLocal;
    static_assert(cap <= kThreads, "one candidate per thread");
    __shared__ int s_c[cap];
    __shared__ int s_n;
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    block_near_at(a, e, a.pos_ref[2 * e], a.pos_ref[2 * e + 1], a.ecell[e], [&](int o) {
        const int slot = atomicAdd(&s_n, 1);
        if (slot < cap) s_c[slot] = o;
    });  // ends with __syncthreads (or returns at once, before any, for an element without a cell)
    __syncthreads();
    const int found = s_n;
    const int cnt = min(found, cap);
    const int t = threadIdx.x;
    const int v = (t < cnt) ? s_c[t] : -1;
    bool keep = t < cnt;
    if ((t & ~31) < cnt) {  // warp-uniform: warps holding candidates
#pragma unroll 4
        for (int j = 0; j < cnt; ++j) {
            const int u = s_c[j];
            keep = keep && !(j < t && u == v);
        }
    }
    const int w = __syncthreads_count(keep);
    const int split = __syncthreads_count(keep && v < e);  // kept indices below e
    if (t < cnt && !keep) s_c[t] = -1;
    __syncthreads();
    if (t == 0) {
        if (found > cap || w > a.max_nb) {
            atomicMax(a.status, DEM_ERR_CAPACITY);
            atomicOr((unsigned long long*)&a.stats[5], 2ull);  // a neighbour list overflowed
        }
        if (w > 16) atomicMax((unsigned long long*)&a.stats[1], (unsigned long long)w);
    }
    const int m = min(w, a.max_nb);
    if (keep) {
        int r = 0;
#pragma unroll 4
        for (int j = 0; j < cnt; ++j) {
            const int u = s_c[j];
            r += (u >= 0 && u < v) ? 1 : 0;
        }
        const int pos = (v > e) ? r - split : (w - split) + r;
        if (pos < m) a.nbr[(size_t)pos * a.n + e] = v;
    }
    if (t == 0) a.ncnt[e] = m;
    __syncthreads();  // the list is complete for the CTA; s_c / s_n are reused by the next call
}

// Queue bucket b for compaction at the next frame start.
template <typename T>
__device__ __forceinline__ void queue_bucket(const KArgs<T>& a, int b) {
    if (atomicExch(&a.bflag[b], 1) == 0) a.comp_list[atomicAdd(a.comp_cnt, 1)] = b;
}

// Stamp o dirty for this round; the first stamper lists it.
template <typename T>
__device__ __forceinline__ void mark_dirty(const KArgs<T>& a, int o, int s, unsigned round) {
    if (atomicExch(&a.dirty[o], round) != round) a.dirty_list[atomicAdd(&a.dirty_cnt[s], 1)] = o;
}

// Move escaped element e to its new reference (px, py) and home bucket; old and
// new buckets are queued for compaction at the next frame start, the
// independent atomics of each level issued together.
template <typename T>
__device__ __forceinline__ void rereference(const KArgs<T>& a, int e, T px, T py, int2 c) {
    const int2 old = a.ecell[e];
    a.pos_ref[2 * e] = px;
    a.pos_ref[2 * e + 1] = py;
    a.ecell[e] = c;
    const int se = sys_id(a, e);
    const int bo = (old.x != INT_MIN) ? bucket_of(old, se, a.n_buckets) : -1;
    const int bn = (c.x != INT_MIN) ? bucket_of(c, se, a.n_buckets) : -1;
    const int slot = (bn >= 0) ? atomicAdd(&a.bcnt[bn], 1) : 0;
    const int fo = (bo >= 0) ? atomicExch(&a.bflag[bo], 1) : 1;
    const int fn = (bn >= 0 && bn != bo) ? atomicExch(&a.bflag[bn], 1) : 1;
    if (bn >= 0) {
        if (slot < a.bucket_cap) {
            a.bitems[(size_t)bn * a.bucket_cap + slot] = e;
        } else {
            atomicMax(a.status, DEM_ERR_CAPACITY);
            atomicOr((unsigned long long*)&a.stats[5], 1ull);  // a grid bucket overflowed
        }
        if (slot + 1 > a.bucket_cap / 2) atomicMax((unsigned long long*)&a.stats[2], (unsigned long long)(slot + 1));
    }
    if (fo == 0) a.comp_list[atomicAdd(a.comp_cnt, 1)] = bo;
    if (fn == 0) a.comp_list[atomicAdd(a.comp_cnt, 1)] = bn;
}

// Whether o's list already holds e, whose reference was (rx, ry): o's list
// was built with e's reference there, and it takes every element within
// (r_o + skin + r_e)(1 + 1e-5) + 1e-6 of its own reference (warp_near_at, seen
// from o).  The test is made a little stricter than the builder's, so rounding
// can only send o to a needless rebuild.
template <typename T>
__device__ __forceinline__ bool list_holds(const KArgs<T>& a, int o, int e, double rx, double ry) {
    const double dx = rx - (double)a.pos_ref[2 * o], dy = ry - (double)a.pos_ref[2 * o + 1];
    const double lim = ((double)a.radii[o] + (double)a.skin + (double)a.radii[e]) * (1.0 + 1e-5) + 1e-6;
    return dx * dx + dy * dy < lim * lim * (1.0 - 1e-9);
}

// One rebuild round before substep s.  For each escaped element e (a CTA each
// when they fit one per CTA, else a warp each): e is stamped dirty, and so is
// every element o within reach of e's new reference whose list does not hold e
// yet (e was out of o's reach at its old reference).  An o whose list holds e
// keeps it, and keeps an entry of an e that moved out of reach: such an entry is
// a candidate that does not touch, whose terms are exact zeros, and it goes at
// o's next rebuild.  The same unit then re-references e, after reading e's old
// reference.  Candidates' references are read concurrently with other escaped
// elements' re-referencing; those elements rebuild their own lists anyway.
// When most elements escaped, every list is rebuilt instead (no marking).
template <typename T>
__device__ void phase_escape(const KArgs<T>& a, const T* kin, unsigned cnt, int n_lazy, int s, unsigned round,
                             bool all) {
    // items: the escaped elements, then (lazy mode) this substep's lazily escaped ones
    const int n_esc = (int)cnt + (all ? 0 : n_lazy);
    auto item = [&](int q) { return q < (int)cnt ? a.esc_list[q] : a.lazy_list[q - (int)cnt]; };
    if (all) {
        const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
        const int gsz = gridDim.x * blockDim.x;
        for (int q = gtid; q < n_esc; q += gsz) {
            const int e = item(q);
            const T px = kin[4 * (size_t)e], py = kin[4 * (size_t)e + 1];
            const int2 c = (jfinite(px) && jfinite(py)) ? cell_of(a, px, py) : make_int2(INT_MIN, INT_MIN);
            rereference(a, e, px, py, c);
        }
    } else if (a.mark_split == DEM_SPLIT_CTA || (a.mark_split == DEM_SPLIT_AUTO && n_esc <= (int)gridDim.x)) {
        // few escapes: a CTA per element, its stencil entries in one load round
        for (int q = blockIdx.x; q < n_esc; q += gridDim.x) {
            const int e = item(q);
            const T px = kin[4 * (size_t)e], py = kin[4 * (size_t)e + 1];
            const int2 c = (jfinite(px) && jfinite(py)) ? cell_of(a, px, py) : make_int2(INT_MIN, INT_MIN);
            const double rx = (double)a.pos_ref[2 * e], ry = (double)a.pos_ref[2 * e + 1];
            const bool had = isfinite(rx) && isfinite(ry) && a.ecell[e].x != INT_MIN;
            block_near_at(a, e, px, py, c, [&](int o) {
                if (!(had && list_holds(a, o, e, rx, ry))) mark_dirty(a, o, s, round);
            });  // ends with __syncthreads: every read of e's old reference is done
            if (threadIdx.x == 0) {
                mark_dirty(a, e, s, round);
                rereference(a, e, px, py, c);
            }
        }
    } else {
        // many escapes (batched windows): a warp per element
        const int lane = threadIdx.x & 31;
        const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const int nwarps = (gridDim.x * blockDim.x) >> 5;
        for (int q = warp; q < n_esc; q += nwarps) {
            const int e = item(q);
            const T px = kin[4 * (size_t)e], py = kin[4 * (size_t)e + 1];
            const int2 c = (jfinite(px) && jfinite(py)) ? cell_of(a, px, py) : make_int2(INT_MIN, INT_MIN);
            const double rx = (double)a.pos_ref[2 * e], ry = (double)a.pos_ref[2 * e + 1];
            const bool had = isfinite(rx) && isfinite(ry) && a.ecell[e].x != INT_MIN;
            warp_near_at(a, e, px, py, c, [&](int o) {
                if (!(had && list_holds(a, o, e, rx, ry))) mark_dirty(a, o, s, round);
            });
            __syncwarp();  // every lane is done with e's old reference
            if (lane == 0) {
                mark_dirty(a, e, s, round);
                rereference(a, e, px, py, c);
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd((unsigned long long*)&a.stats[0], 1ull);
        atomicAdd((unsigned long long*)&a.stats[3], (unsigned long long)n_esc);
    }
}

// Lazy escape of element e during the force phase of substep s (warp-wide):
// the neighbours its move brings into reach, and e itself, are stamped dirty for
// the rebuild at substep s + 1; then e takes its position at substep s as new
// reference.  Nothing else in the force phase reads references, buckets or
// dirty stamps; e's own force this substep uses its current list, which is
// valid (e is within the urgent limit of its old reference).
template <typename T>
__device__ __forceinline__ void lazy_escape_warp(const KArgs<T>& a, const T* kin, int e, int s_next,
                                                 unsigned round_next) {
    const int lane = threadIdx.x & 31;
    const T px = kin[4 * (size_t)e], py = kin[4 * (size_t)e + 1];
    const int2 c = (jfinite(px) && jfinite(py)) ? cell_of(a, px, py) : make_int2(INT_MIN, INT_MIN);
    const double rx = (double)a.pos_ref[2 * e], ry = (double)a.pos_ref[2 * e + 1];
    const bool had = isfinite(rx) && isfinite(ry) && a.ecell[e].x != INT_MIN;
    warp_near_at(a, e, px, py, c, [&](int o) {
        if (!(had && list_holds(a, o, e, rx, ry))) mark_dirty(a, o, s_next, round_next);
    });
    __syncwarp();
    if (lane == 0) {
        mark_dirty(a, e, s_next, round_next);
        rereference(a, e, px, py, c);
    }
}

// The same lazy escape by a whole CTA (every thread must call it with the same
// e), its stencil entries in one load round.
template <typename T>
__device__ __forceinline__ void lazy_escape_block(const KArgs<T>& a, const T* kin, int e, int s_next,
                                                  unsigned round_next) {
    const T px = kin[4 * (size_t)e], py = kin[4 * (size_t)e + 1];
    const int2 c = (jfinite(px) && jfinite(py)) ? cell_of(a, px, py) : make_int2(INT_MIN, INT_MIN);
    const double rx = (double)a.pos_ref[2 * e], ry = (double)a.pos_ref[2 * e + 1];
    const bool had = isfinite(rx) && isfinite(ry) && a.ecell[e].x != INT_MIN;
    block_near_at(a, e, px, py, c, [&](int o) {
        if (!(had && list_holds(a, o, e, rx, ry))) mark_dirty(a, o, s_next, round_next);
    });
    __syncthreads();  // every thread is done with e's old reference
    if (threadIdx.x == 0) {
        mark_dirty(a, e, s_next, round_next);
        rereference(a, e, px, py, c);
    }
}

// Rebuild every list (when most elements escaped at once).
template <typename T>
__device__ void phase_build_all(const KArgs<T>& a) {
    __shared__ int sbuf[kThreads / 32][2 * kMaxNbLocal];
    __shared__ int scnt[kThreads / 32];
    const int wl = threadIdx.x >> 5;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int e = warp; e < a.n; e += nwarps) warp_build(a, e, sbuf[wl], &scnt[wl]);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd((unsigned long long*)&a.stats[4], (unsigned long long)a.n);
}

// Drop stale and duplicate entries of the queued buckets (run while nothing
// reads or writes the grid).
template <typename T>
__device__ void compact_buckets(const KArgs<T>& a) {
    // one warp per queued bucket: lanes test 32 entries at a time; an entry
    // stays if it is current (its home cell hashes here) and no earlier entry
    // holds the same element; kept entries move to the front in their order
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nq = *((volatile int*)a.comp_cnt);
    for (int i = warp; i < nq; i += nwarps) {
        const int b = a.comp_list[i];
        const int m = min(a.bcnt[b], a.bucket_cap);
        int* it = a.bitems + (size_t)b * a.bucket_cap;
        int w = 0;
        for (int k0 = 0; k0 < m; k0 += 32) {
            const int k = k0 + lane;
            const int o = (k < m) ? it[k] : -1;
            bool keep = false;
            if (o >= 0 && o < a.n) {
                const int2 c = a.ecell[o];
                keep = c.x != INT_MIN && bucket_of(c, sys_id(a, o), a.n_buckets) == b;
            }
            for (int q = 0; keep && q < w; ++q)  // kept in earlier chunks
                if (it[q] == o) keep = false;
            for (int j = 0; j < 32; ++j) {       // earlier lanes of this chunk
                const int oj = __shfl_sync(0xffffffffu, o, j);
                const bool kj = __shfl_sync(0xffffffffu, keep, j);
                if (j < lane && kj && oj == o) keep = false;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            __syncwarp();  // every lane has read its entry before any is overwritten
            if (keep) it[w + __popc(bal & ((1u << lane) - 1u))] = o;
            w += __popc(bal);
            __syncwarp();
        }
        for (int k = w + lane; k < m; k += 32) it[k] = -1;
        if (lane == 0) {
            a.bcnt[b] = w;
            a.bflag[b] = 0;
        }
    }
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

// ─── fixed-order sums (deterministic, independent of the grid size) ─────────
// lane 0 receives the warp's sum (shuffle-down tree)
__device__ __forceinline__ double warp_sum_lane0(double v) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

// thread 0 receives the block's sums: a tree in each warp, then over the warps
template <int N>
__device__ __forceinline__ void block_sum3(double v0, double v1, double v2, double* out3) {
    constexpr int kW = N / 32;
    __shared__ double sh[3][kW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v0 = warp_sum_lane0(v0);
    v1 = warp_sum_lane0(v1);
    v2 = warp_sum_lane0(v2);
    if (lane == 0) {
        sh[0][w] = v0;
        sh[1][w] = v1;
        sh[2][w] = v2;
    }
    __syncthreads();
    if (w == 0) {
        double u0 = lane < kW ? sh[0][lane] : 0.0, u1 = lane < kW ? sh[1][lane] : 0.0;
        double u2 = lane < kW ? sh[2][lane] : 0.0;
        u0 = warp_sum_lane0(u0);
        u1 = warp_sum_lane0(u1);
        u2 = warp_sum_lane0(u2);
        if (lane == 0) {
            out3[0] = u0;
            out3[1] = u1;
            out3[2] = u2;
        }
    }
    __syncthreads();  // sh is reused by the next call
}

template <typename T>
__device__ __forceinline__ HullPose<T> hull_pose(const KArgs<T>& a, const T* eta) {
    HullPose<T> H;
    H.sx = eta[0];
    H.sy = eta[1];
    const T spsi = eta[2];
    jsincos(-spsi, &H.s_neg, &H.c_neg);
    jsincos(spsi, &H.s_h, &H.c_h);
    H.hl = T(a.P.half_len);
    H.hb = T(a.P.half_beam);
    H.hb005 = T(a.P.half_beam * 0.05);
    return H;
}

// Force chunk of element e: chunks of kThreads elements from each system's
// first element.
template <typename T>
__device__ __forceinline__ int chunk_of(const KArgs<T>& a, int e) {
    if (a.nsys == 1) return e / kThreads;
    const int s = a.sys_of[e];
    return a.part_base[s] + (e - (s > 0 ? a.sys_end[s - 1] : 0)) / kThreads;
}

// ─── active list, binned by work ────────────────────────────────────────────
// phase_reduce lists the frame's active elements in act_list (n entries,
// counted by act_cnt[0]).  With kActBins > 1 it also lists them in kActBins
// bins of n entries each (act_list + (1 + b) * n, counted by act_cnt[1 + b])
// by their work in a substep: the larger of their bond slot and candidate
// counts, in bins [0, 6), [6, 9), [9, 12) and from 12 with four bins.  The
// thread-per-element path of the force phases takes the bins one after
// another as one list, so the lanes of a warp hold elements of like work; the
// warp-per-element path, which a frame with few active elements takes, reads
// the plain list.  The order of the elements does not change any result: each
// element sums its own terms.
#ifndef DEM_ACT_BINS
#define DEM_ACT_BINS 1
#endif
constexpr int kActBins = DEM_ACT_BINS;
constexpr int kActLists = kActBins > 1 ? 1 + kActBins : 1;

__device__ __forceinline__ int act_bin(int work) { return min(max((work - 3) / 3, 0), kActBins - 1); }

// ─── P_CULL: elements whose bounding circle reaches the hull; escapes ───────
template <typename T>
__device__ void phase_cull(const KArgs<T>& a, const Frame<T>& F) {
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gsz = gridDim.x * blockDim.x;
    const T reach = a.hull_r * T(1.0001) + T(1e-3);
    // nothing reads the grid in this phase: drop stale entries queued last frame
    compact_buckets(a);
    if (gtid == 0) {
        for (int b = 0; b < kActLists; ++b) a.act_cnt[b] = 0;  // read last by the previous frame's force phases
        *a.fb_cnt = 0;   // read last by the previous frame's fracture
    }
    // per-floe scratch of this frame (read last by the previous frame's fracture)
    for (int fl = gtid; fl < a.nf; fl += gsz) {
        a.fcoll[fl] = 0;
        a.fmax[fl] = 0ull;
    }
    const unsigned fstamp = frame_stamp(a, F);
    for (int e = gtid; e < a.n; e += gsz) {
        typename vec2_of<T>::type p = ld2(F.src.pos, e);
        const T* eta = F.ship_src.eta + 3 * (a.nsys > 1 ? a.sys_of[e] : 0);  // this element's ship
        const T ddx = p.x - eta[0], ddy = p.y - eta[1];
        const T lim = reach + a.vert_r[e];
        // every query point of e lies within vert_r of its centroid and every hull
        // point within hull_r of the ship: farther elements get pen = 0, which is
        // what all of their point tests return (jax_geometry.py:104-134, :359-368);
        // the test keeps NaN positions (comparison false) on the exact path
        if (!(ddx * ddx + ddy * ddy > lim * lim * T(1.0001))) {
            const int slot = atomicAdd(a.near_cnt, 1);
            a.near_list[slot] = e;
            a.cnear[chunk_of(a, e)] = fstamp;  // phase_cforce runs this chunk
        } else {
            a.cpen[e] = T(0);
            a.cnx[e] = T(0);
            a.cny[e] = T(0);
        }
        a.crack[e] = 0;  // set by phase_reduce for elements touching a broken bond
        const bool urg = escaped(a, e, p.x, p.y, a.lazy ? a.esc_h_urgent : a.esc_h_check);
        warp_append(a.esc_list, (int*)&a.esc_cnt[0], urg, e);
        if (a.lazy) warp_append(a.lazy_list, &a.lazy_cnt[0], !urg && escaped(a, e, p.x, p.y, a.esc_h_check), e);
    }
}

// ─── P_NEAR: one warp per near element (jax_geometry.py:515-594) ────────────
// Pass 1: the element's vertices and edge samples vs the analytic hull; pass 2:
// the hull outline points inside the element's polygon; element-wise max.  Lanes
// split the points; argmax/argmin keep the reference's first-index ties.
template <typename T>
struct Best {
    T p, nx, ny;
    int i;
};

template <typename T>
__device__ __forceinline__ void better(Best<T>& b, T p, T nx, T ny, int i) {
    if (p > b.p || (p == b.p && i < b.i)) {
        b.p = p;
        b.nx = nx;
        b.ny = ny;
        b.i = i;
    }
}

template <typename T>
__device__ __forceinline__ Best<T> warp_best(Best<T> b) {
    for (int off = 16; off > 0; off >>= 1) {
        Best<T> o;
        o.p = __shfl_xor_sync(0xffffffffu, b.p, off);
        o.nx = __shfl_xor_sync(0xffffffffu, b.nx, off);
        o.ny = __shfl_xor_sync(0xffffffffu, b.ny, off);
        o.i = __shfl_xor_sync(0xffffffffu, b.i, off);
        better(b, o.p, o.nx, o.ny, o.i);
    }
    return b;
}

template <typename T>
__device__ void phase_near(const KArgs<T>& a, const Frame<T>& F, T* hullw) {
    // hull outline in world frame: ship_hull_local @ R.T + [x, y] (jax_geometry.py:568-572),
    // staged once per CTA for a single ship; with several ships each element
    // transforms its own ship's outline point by point (the same expression)
    const bool one_ship = a.nsys == 1;
    HullPose<T> H1 = hull_pose(a, F.ship_src.eta);
    if (one_ship) {
        for (int i = threadIdx.x; i < a.S; i += blockDim.x) {
            T lx = a.hull[2 * i], ly = a.hull[2 * i + 1];
            hullw[2 * i] = lx * H1.c_h + ly * (-H1.s_h) + H1.sx;
            hullw[2 * i + 1] = lx * H1.s_h + ly * H1.c_h + H1.sy;
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nnear = *((volatile int*)a.near_cnt);
    const int V = a.V;
    const int E = a.P.n_edge_samples;
    const int P1 = V * (1 + E);
    for (int q = warp; q < nnear; q += nwarps) {
        const int e = a.near_list[q];
        const HullPose<T> H = one_ship ? H1 : hull_pose(a, F.ship_src.eta + 3 * a.sys_of[e]);
        typename vec2_of<T>::type pe = ld2(F.src.pos, e);
        T c, sn;
        jsincos(F.src.rot[e], &sn, &c);
        const T* lp = a.polys + (size_t)e * V * 2;
        const uint8_t* mk = a.pmask + (size_t)e * V;
        // world vertex k (jax_geometry.py:176-180)
        auto wv = [&](int k, T& x, T& y) {
            T lx = lp[2 * k], ly = lp[2 * k + 1];
            x = c * lx - sn * ly + pe.x;
            y = sn * lx + c * ly + pe.y;
        };
        // pass 1: point index = vertex * (1 + E) + sample (jax_geometry.py:190-211)
        Best<T> b1 = {T(0), T(0), T(0), INT_MAX};
        for (int pt = lane; pt < P1; pt += 32) {
            const int k = pt / (1 + E), j = pt % (1 + E);
            T qx, qy;
            wv(k, qx, qy);
            if (j > 0) {
                T x1, y1;
                wv((k + 1 == V) ? 0 : k + 1, x1, y1);
                T t = a.t_samp[j - 1];
                T omt = T(1) - t;
                qx = qx * omt + x1 * t;
                qy = qy * omt + y1 * t;
            }
            T p, nx, ny;
            hull_point(H, qx, qy, p, nx, ny);
            if (!mk[k]) p = T(0);
            better(b1, p, nx, ny, pt);
        }
        b1 = warp_best(b1);
        // pass 2 (jax_geometry.py:300-510)
        T wx[kMaxV], wy[kMaxV], mx[kMaxV], my[kMaxV], mc[kMaxV];
        for (int k = 0; k < V; ++k) {
            wv(k, wx[k], wy[k]);
            const bool m = mk[k] != 0;
            mx[k] = m ? wx[k] : T(0);
            my[k] = m ? wy[k] : T(0);
            mc[k] = m ? T(1) : T(0);
        }
        const T n_real = jmax(np_pairwise_sum(mc, V), T(1));
        const T cxc = np_pairwise_sum(mx, V) / n_real;
        const T cyc = np_pairwise_sum(my, V) / n_real;
        Best<T> b2 = {T(0), T(0), T(0), INT_MAX};
        for (int si = lane; si < a.S; si += 32) {
            T hx, hy;
            if (one_ship) {
                hx = hullw[2 * si];
                hy = hullw[2 * si + 1];
            } else {
                const T lx = a.hull[2 * si], ly = a.hull[2 * si + 1];
                hx = lx * H.c_h + ly * (-H.s_h) + H.sx;
                hy = lx * H.s_h + ly * H.c_h + H.sy;
            }
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
                const T t = jclip(c1 / c2, T(0), T(1));
                const T ddx = hx - (xi + t * vx), ddy = hy - (yi + t * vy);
                const T d = jsqrt(ddx * ddx + ddy * ddy + T(1e-20));
                if (k == 0 || d < dmin) {  // argmin, first index wins
                    dmin = d;
                    kbest = k;
                }
            }
            T p = T(0), nx = T(0), ny = T(0);
            if ((crossings % 2) == 1) {
                // outward normal of the closest edge (jax_geometry.py:389-405)
                const int k = kbest, k1 = (k + 1 == V) ? 0 : k + 1;
                const T ex = wx[k1] - wx[k], ey = wy[k1] - wy[k];
                T nxe = ey, nye = -ex;
                const T nlen = jsqrt(nxe * nxe + nye * nye + T(1e-20));
                nxe = nxe / nlen;
                nye = nye / nlen;
                const T midx = (wx[k] + wx[k1]) / T(2), midy = (wy[k] + wy[k1]) / T(2);
                const T dotc = (midx - cxc) * nxe + (midy - cyc) * nye;
                if (dotc < T(0)) {
                    nxe = -nxe;
                    nye = -nye;
                }
                p = dmin;
                nx = nxe;
                ny = nye;
            }
            better(b2, p, nx, ny, si);
        }
        b2 = warp_best(b2);
        if (lane == 0) {
            // pass 2 replaces pass 1 only where strictly deeper (jax_geometry.py:585-590)
            const bool use2 = (b2.p > T(0)) && (b2.p > b1.p);
            a.cpen[e] = use2 ? b2.p : b1.p;
            a.cnx[e] = use2 ? b2.nx : b1.nx;
            a.cny[e] = use2 ? b2.ny : b1.ny;
        }
    }
}

// ─── P_CFORCE: ship force on ice, submergence, reductions (jax_simulation.py:431-496)
template <typename T>
__device__ void phase_cforce(const KArgs<T>& a, const Frame<T>& F) {
    const DemParams& P = a.P;
    const T wcf = T(P.w_contact_radius_factor), wcap = T(P.w_contact_cap);
    const T flex = T(P.flexural_strength_base);
    const T pcr = T(P.pen_crit_ref), pct = T(P.pen_crit_thickness_ref);
    const T spf = T(P.side_push_factor);
    const T srate = T(P.submergence_rate), scap = T(P.submergence_pen_cap);
    const T inv_rise = T(1.0 / P.rise_time_const);
    const T dt = T(P.dt);
    const T rho_g = T(P.water_density * 9.81);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *a.near_cnt = 0;   // P_NEAR is done with it
        *a.comp_cnt = 0;   // P_CULL compacted the queue
    }
    const unsigned fstamp = frame_stamp(a, F);
    for (int chunk = blockIdx.x; chunk < a.nchunks; chunk += gridDim.x) {
        // in a call's later frames (state in place) a chunk with no element
        // near the hull now and none in contact or submerged at the last
        // cforce is skipped: every one of its elements would store what it
        // holds (no ship force, no contact force, submergence 0) and its sums
        // are the zeros it holds
        if (F.f >= 1 && !a.cwarm[chunk] && a.cnear[chunk] != fstamp) continue;  // uniform over the CTA
        // chunks of kThreads elements start at each system's first element, so a
        // system's sums are grouped as they would be if it were simulated alone
        const int2 ci = a.chunk_info[chunk];
        const int e = ci.y + threadIdx.x;
        const T sx = F.ship_src.eta[3 * ci.x], sy = F.ship_src.eta[3 * ci.x + 1];
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        bool warm = false;
        if (e < a.sys_end[ci.x]) {
            typename vec2_of<T>::type p = ld2(F.src.pos, e);
            const T pen = a.cpen[e], nx = a.cnx[e], ny = a.cny[e];
            const bool has = pen > T(0);
            const T h = a.thick[e];
            const T w_contact = jmin(wcf * a.radii[e], wcap);
            const T sigma_f = flex * jsqrt(h);
            const T f_break = sigma_f * w_contact * (h * h);
            const T pen_crit = pcr * (h / pct);
            const T fm = has ? f_break * jmin(pen / jmax(pen_crit, T(1e-10)), T(1)) : T(0);
            T so_x = fm * nx;
            T so_y = fm * ny;
            so_y = so_y + spf * fm * jsign(p.y - sy);
            // moment on the ship uses the force before the thrust cap (jax_simulation.py:474-477)
            const T rx = p.x - sx, ry = p.y - sy;
            const T mom = has ? (rx * (-so_y) - ry * (-so_x)) : T(0);
            s0 = (double)so_x;
            s1 = (double)so_y;
            s2 = (double)mom;
            // submergence and buoyancy (jax_simulation.py:480-496)
            const T sub = F.src.sub[e];
            const T pen_c = jmin(pen, scap);
            const T new_sub = has ? jmin(sub + srate * pen_c * dt, h) : jmax(T(0), sub - inv_rise * sub * dt);
            const T z_sub = jmin(new_sub, h);
            const T f_buoy = rho_g * a.areas[e] * z_sub;
            if (has) {
                so_x = so_x + f_buoy * nx;
                so_y = so_y + f_buoy * ny;
            }
            st2(a.soi, e, so_x, so_y);
            a.fraw[e] = fm;
            F.dst.sub[e] = new_sub;
            warm = has || new_sub != T(0);
            if (a.d_pen) a.d_pen[e] = pen;
            const int fl = a.floe_of[e];
            if (has) atomicMax(&a.fcoll[fl], 1);
            if (fm > T(0)) {
                if (sizeof(T) == 4)
                    atomicMax(&a.fmax[fl], (unsigned long long)f2ord((float)fm));
                else
                    atomicMax(&a.fmax[fl], d2ord((double)fm));
            }
        }
        double r3[3];
        block_sum3<kThreads>(s0, s1, s2, r3);
        const int any_warm = __syncthreads_or(warm ? 1 : 0);
        if (threadIdx.x == 0) {
            a.part[3 * chunk + 0] = r3[0];
            a.part[3 * chunk + 1] = r3[1];
            a.part[3 * chunk + 2] = r3[2];
            a.cwarm[chunk] = any_warm ? 1 : 0;
        }
    }
}

// ─── vessel step (jax_vessel_dynamics.py:246-348) ───────────────────────────
template <typename T>
__device__ void ship_step(const DemParams& P, const T* eta, const T* nu, const T* na, const T* ei,
                          const T* sp, const T* spn, const T* tau_ice, const T* vws, T* eta_o,
                          T* nu_o, T* na_o, T* ei_o, const T* u_ctrl = nullptr) {
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
    T tau_act[3];
    if (u_ctrl) {
        // planner rollouts: the body-frame control replaces the DP controller
        // and the thrust allocation (RPMs and integral error stay as they are)
        for (int i = 0; i < 3; ++i) {
            tau_act[i] = u_ctrl[i];
            ei_o[i] = ei[i];
        }
        for (int i = 0; i < 6; ++i) na_o[i] = na[i];
    } else {
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
// A warp reduces one system's chunk partials in a fixed order (lane 0 gets them).
template <typename T>
__device__ void frame_totals(const KArgs<T>& a, int sys, double* tot3) {
    const int lane = threadIdx.x & 31;
    double v0 = 0.0, v1 = 0.0, v2 = 0.0;
    for (int i = a.part_base[sys] + lane; i < a.part_base[sys + 1]; i += 32) {
        v0 += a.part[3 * i];
        v1 += a.part[3 * i + 1];
        v2 += a.part[3 * i + 2];
    }
    tot3[0] = warp_sum_lane0(v0);
    tot3[1] = warp_sum_lane0(v1);
    tot3[2] = warp_sum_lane0(v2);
}

template <typename T>
__device__ __forceinline__ T thrust_scale_of(const KArgs<T>& a, const double* tot3) {
    if (!a.P.has_max_ship_ice_force) return T(1);
    T fx = T(tot3[0]), fy = T(tot3[1]);
    T mag = jsqrt(fx * fx + fy * fy);
    T mx = T(a.P.max_ship_ice_force);
    return (mag > mx) ? mx / jmax(mag, T(1e-6)) : T(1);
}

// Warps with at most this many active elements share each one's slots among
// their lanes in phase_reduce.
constexpr int kCoopSlots = 3;

// The bond slot records of active element e by one lane: two slots per step,
// their loads issued level by level (slot -> partner -> floe flag).  The bond
// has an active end this frame; it is listed once, by its active end of lower
// index (e, unless the partner is active and lower).
template <typename T>
__device__ __forceinline__ void slot_records_lane(const KArgs<T>& a, const Frame<T>& F, SlotRec<T>* rec, int e,
                                                  unsigned fstamp) {
    const int s0 = a.boff[e], s1 = a.boff[e + 1];
    for (int sl = s0; sl < s1; sl += 2) {
        const bool two = sl + 1 < s1;
        const int2 ent0 = a.bslot[sl];
        const int2 ent1 = two ? a.bslot[sl + 1] : ent0;
        const int b0 = ent0.x & 0x7fffffff, b1 = ent1.x & 0x7fffffff;
        const bool in0 = F.src.intact[b0] != 0, in1 = F.src.intact[b1] != 0;
        const bool sa0 = F.src.active[ent0.y] != 0, sa1 = F.src.active[ent1.y] != 0;
        const int fo0 = a.floe_of[ent0.y], fo1 = a.floe_of[ent1.y];
        const T d0 = F.src.dmg[b0], d1 = F.src.dmg[b1];
        const T r0 = a.slot_rest[sl], r1 = two ? a.slot_rest[sl + 1] : r0;
        const T k0 = a.slot_stiff[sl], k1 = two ? a.slot_stiff[sl + 1] : k0;
        const bool ao0 = sa0 || a.fcoll[fo0];
        const bool ao1 = sa1 || a.fcoll[fo1];
        a.bstamp[b0] = fstamp;
        a.bstamp[b1] = fstamp;
        warp_append2(a.fb_list, a.fb_cnt, !(ao0 && ent0.y < e), b0, two && !(ao1 && ent1.y < e), b1);
        if (!in0 || (two && !in1)) a.crack[e] = 1;
        SlotRec<T> q;
        q.o = (ent0.x < 0) ? (int)((unsigned)ent0.y | 0x80000000u) : ent0.y;
        q.rest = r0;
        q.stiff = k0;
        q.omd = (in0 && ao0) ? T(1) - d0 : T(-1);  // e is active: both ends must be
        rec[sl] = q;
        if (two) {
            q.o = (ent1.x < 0) ? (int)((unsigned)ent1.y | 0x80000000u) : ent1.y;
            q.rest = r1;
            q.stiff = k1;
            q.omd = (in1 && ao1) ? T(1) - d1 : T(-1);
            rec[sl + 1] = q;
        }
    }
}

template <typename T>
__device__ void phase_reduce(const KArgs<T>& a, const Frame<T>& F) {
    typedef typename vec2_of<T>::type V2;
    // one warp per system: totals, thrust cap and the vessel step (warp 0 of
    // CTA 0 for a single system)
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int ngwarp = (gridDim.x * blockDim.x) >> 5;
    for (int sys = gwarp; sys < a.nsys; sys += ngwarp) {
        double tot3[3];
        frame_totals(a, sys, tot3);
        if ((threadIdx.x & 31) == 0) {
            const T scale = thrust_scale_of(a, tot3);
            // reaction on the ship (jax_simulation.py:470-478)
            T Fx = -(T(tot3[0]) * scale), Fy = -(T(tot3[1]) * scale), M = T(tot3[2]);
            double* fs = a.fscal + 4 * sys;
            fs[0] = (double)scale;
            fs[1] = (double)Fx;
            fs[2] = (double)Fy;
            fs[3] = (double)M;
            T tau[3] = {Fx, Fy, M};
            T J = jsqrt(Fx * Fx + Fy * Fy) * T(a.P.dt);
            // rollouts drive the ship by controls (no setpoints, no ice brake)
            const T* u = a.u_ctrl ? a.u_ctrl + ((size_t)F.f * a.nsys + sys) * 3 : nullptr;
            const T zero6[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
            const T* spf = u ? zero6 : F.sp + 6 * sys;
            T sp[3] = {spf[0], spf[1], spf[2]};
            const T* eta = F.ship_src.eta + 3 * sys;
            if (!u && a.P.ice_brake_threshold > 0.0) {  // jax_simulation.py:658-669
                T thr = T(a.P.ice_brake_threshold);
                T bf = jclip(thr / jmax(fabs(tau[0]), thr), T(0.1), T(1));
                sp[0] = eta[0] + bf * (spf[0] - eta[0]);
                sp[1] = eta[1] + bf * (spf[1] - eta[1]);
            }
            const T vzero[2] = {T(0), T(0)};
            const T* vws = F.vws ? F.vws + 2 * sys : vzero;
            T eta_o[3], nu_o[3], na_o[6], ei_o[3];
            ship_step<T>(a.P, eta, F.ship_src.nu + 3 * sys, F.ship_src.na + 6 * sys, F.ship_src.ei + 3 * sys, sp,
                         spf + 3, tau, vws, eta_o, nu_o, na_o, ei_o, u);
            for (int i = 0; i < 3; ++i) {
                F.ship_dst.eta[3 * sys + i] = eta_o[i];
                F.ship_dst.nu[3 * sys + i] = nu_o[i];
                F.ship_dst.ei[3 * sys + i] = ei_o[i];
            }
            for (int i = 0; i < 6; ++i) F.ship_dst.na[6 * sys + i] = na_o[i];
            if (a.d_F) {
                a.d_F[2 * sys] = Fx;
                a.d_F[2 * sys + 1] = Fy;
            }
            if (a.d_J) a.d_J[sys] = J;
            const size_t fs_i = (size_t)F.f * a.nsys + sys;
            if (a.h_eta)
                for (int i = 0; i < 3; ++i) a.h_eta[fs_i * 3 + i] = eta_o[i];
            if (a.h_J) a.h_J[fs_i] = J;
            if (a.h_F) {
                a.h_F[fs_i * 2] = Fx;
                a.h_F[fs_i * 2 + 1] = Fy;
            }
        }
    }
    // With one system, CTA 0 runs the vessel step above and the other CTAs share
    // the element and slot work (all CTAs when the grid has one); with several
    // systems every CTA takes part in both.
    const int c0 = (gridDim.x > 1 && a.nsys == 1) ? 1 : 0;
    if ((int)blockIdx.x < c0) return;
    const int gtid = (blockIdx.x - c0) * blockDim.x + threadIdx.x;
    const int gsz = (gridDim.x - c0) * blockDim.x;
    SlotRec<T>* rec = reinterpret_cast<SlotRec<T>*>(a.slotrec);
    typedef typename vec4_of<T>::type V4;
    const unsigned fstamp = frame_stamp(a, F);
    // lanes take consecutive elements; the loop bound is uniform over the warp,
    // so that the warp can share the slot work of the active elements it finds
    const int lane = threadIdx.x & 31;
    for (int w0 = gtid - lane; w0 < a.n; w0 += gsz) {
        const int e = w0 + lane;
        bool ae = false;
        if (e < a.n) {
            // activation (jax_simulation.py:498-509)
            const bool was = F.src.active[e] != 0;
            ae = was || a.fcoll[a.floe_of[e]];
            // after the first frame of a call, an element frozen before and
            // after this frame's activation has its state, substep buffers and
            // frame output in place already (the previous frame wrote them)
            if (F.f == 0 || ae) {
                F.dst.active[e] = ae ? 1 : 0;
                // packed kinematics read by substep 0
                const V2 p = ld2(F.src.pos, e), v = ld2(F.src.vel, e);
                V4 k4;
                k4.x = p.x;
                k4.y = p.y;
                k4.z = a.radii[e];
                k4.w = a.r3[e];
                reinterpret_cast<V4*>(a.kin[0])[e] = k4;
                st2(a.kvel[0], e, v.x, v.y);
                if (!ae) {
                    // frozen for the whole frame, it keeps its state
                    // (jax_simulation.py:257-262): both substep buffers and the
                    // frame's output hold it now, and the substeps skip it
                    reinterpret_cast<V4*>(a.kin[1])[e] = k4;
                    st2(a.kvel[1], e, v.x, v.y);
                    st2(F.dst.pos, e, p.x, p.y);
                    st2(F.dst.vel, e, v.x, v.y);
                    F.dst.rot[e] = F.src.rot[e];
                    F.dst.avel[e] = F.src.avel[e];
                }
            }
        }
        {
            // the frame's active list, binned by the element's work in a
            // substep (bond slots and candidates, of which the thread path
            // walks the longer), so that the lanes of a warp end together
            warp_append(a.act_list, a.act_cnt, ae, e);
            if (kActBins > 1) {
                int bin = 0;
                if (ae) bin = act_bin(max(a.boff[e + 1] - a.boff[e], a.ncnt[e]));
#pragma unroll
                for (int b = 0; b < kActBins; ++b)
                    warp_append(a.act_list + (size_t)(1 + b) * a.n, &a.act_cnt[1 + b], ae && bin == b, e);
            }
        }
        // the bond slot records of the active elements for this frame (only
        // active elements read them); crack front = the element touches a bond
        // broken at frame start (read for bonds between two active elements).
        // A warp with few active elements takes them one after another, each
        // element's slots spread over the lanes; with more, every lane takes
        // its own element's slots.
        unsigned m = __ballot_sync(0xffffffffu, ae);
        if (__popc(m) > kCoopSlots) {
            if (ae) slot_records_lane(a, F, rec, e, fstamp);
            continue;
        }
        while (m) {
            const int ee = w0 + __ffs(m) - 1;
            m &= m - 1;
            const int s0 = a.boff[ee], s1 = a.boff[ee + 1];
            for (int sl = s0 + lane; sl < s1; sl += 32) {
                const int2 ent = a.bslot[sl];
                const int b = ent.x & 0x7fffffff;
                const bool in = F.src.intact[b] != 0;
                const bool sa = F.src.active[ent.y] != 0;
                const int fo = a.floe_of[ent.y];
                const T d = F.src.dmg[b];
                const T r = a.slot_rest[sl], k = a.slot_stiff[sl];
                const bool ao = sa || a.fcoll[fo];
                // the bond has an active end this frame; it is listed once, by
                // its active end of lower index (ee, unless the partner is
                // active and lower)
                a.bstamp[b] = fstamp;
                warp_append(a.fb_list, a.fb_cnt, !(ao && ent.y < ee), b);
                if (!in) a.crack[ee] = 1;
                SlotRec<T> q;
                q.o = (ent.x < 0) ? (int)((unsigned)ent.y | 0x80000000u) : ent.y;
                q.rest = r;
                q.stiff = k;
                q.omd = (in && ao) ? T(1) - d : T(-1);  // ee is active: both ends must be
                rec[sl] = q;
            }
        }
    }
}

// ─── P_FORCE: one substep (jax_simulation.py:63-268, 363-395) ───────────────
// One thread per element, gather form: each element sums its own bond and
// contact terms in the reference's scatter order, so no atomics are needed.
// Positions are packed with radii as {x, y, r} (one 16-byte load per neighbour,
// velocities only for overlapping pairs) and bond slots are 16-byte records;
// the loads of a batch are issued before any of them is used.
// Every operation is unfused (-fmad=false) and in the reference's order, with
// divisions where it divides, so that fp32 forces round as NumPy's fp32
// evaluation of the same expressions does.
#ifndef DEM_KBATCH
#define DEM_KBATCH 2
#endif
constexpr int kBatch = DEM_KBATCH;  // bond slots / contact candidates whose loads are issued together


// overlap^1.5 of the Hertz law, as the reference's power of an fp32 array: in
// float the product o * sqrt(o) is formed in double and rounded once, which
// gives the correctly rounded power (the value the C library's powf returns
// but for its rare last-place misses); in double as is
__device__ __forceinline__ float hertz15(float o) {
    const double od = (double)o;
    return (float)(od * sqrt(od));
}
__device__ __forceinline__ double hertz15(double o) { return o * sqrt(o); }

// Constants and substep buffers of one force phase.
template <typename T>
struct ForceCtx {
    const T *kin, *kvin, *rin, *ain;
    T *kout, *kvout, *rout, *aout;
    const uint8_t* act;
    T esc_h;  // escape threshold of this substep's test (urgent in lazy mode)
    T h_lazy;           // lazy threshold of this substep's test
    bool lazy_detect;   // the next substep processes lazy escapes
    const SlotRec<T>* rec;
    bool last;
};

template <typename T>
__device__ __forceinline__ ForceCtx<T> force_ctx(const KArgs<T>& a, const Frame<T>& F, int s) {
    ForceCtx<T> c;
    const int k = a.k_sub;
    c.kin = a.kin[s & 1];
    c.kout = a.kin[(s + 1) & 1];
    c.kvin = a.kvel[s & 1];
    c.kvout = a.kvel[(s + 1) & 1];
    c.rin = (s == 0) ? F.src.rot : a.sp_rot[(s - 1) & 1];
    c.ain = (s == 0) ? F.src.avel : a.sp_avel[(s - 1) & 1];
    c.last = (s == k - 1);
    c.rout = c.last ? F.dst.rot : a.sp_rot[s & 1];
    c.aout = c.last ? F.dst.avel : a.sp_avel[s & 1];
    c.act = F.dst.active;
    c.esc_h = ((s + 1) % a.esc_period == 0) ? a.esc_h_check : a.esc_h_urgent;
    c.h_lazy = a.esc_h_check;
    c.lazy_detect = false;
    if (a.lazy) {
        c.esc_h = a.esc_h_urgent;
        c.lazy_detect = ((s + 1) % 2 == 0) && (s + 2 < a.k_sub);
    }
    c.rec = reinterpret_cast<const SlotRec<T>*>(a.slotrec);
    return c;
}

// Bond slot term (jax_simulation.py:63-108) of a slot record with omd >= 0:
// the force and half-moment that the slot's role adds to (role i) or
// subtracts from (role j) the element's bond sums.
template <typename T>
__device__ __forceinline__ void bond_term(const SlotRec<T>& r, typename vec2_of<T>::type kb, T ex, T ey, T& fx,
                                          T& fy, T& cr) {
    const bool role_j = r.o < 0;
    const T dx = role_j ? ex - kb.x : kb.x - ex;
    const T dy = role_j ? ey - kb.y : kb.y - ey;
    const T dist = jsqrt(dx * dx + dy * dy);
    const T dsafe = jmax(dist, T(1e-10));
    const T fmag = r.stiff * (dist - r.rest) * r.omd;
    fx = (dx / dsafe) * fmag;  // bond_dir * f_mag (jax_simulation.py:76-96)
    fy = (dy / dsafe) * fmag;
    cr = T(0.5) * (dx * fy - dy * fx);
}

// Ice-ice contact term (jax_simulation.py:111-164) of element e (kinematics
// ke, ve) with candidate o (ko, vo); e_is_i = e < o.  Returns false when the
// pair does not touch; else e adds (tx, ty) to its contact force and adds
// (e_is_i) or subtracts hm from its contact moment.
template <typename T>
__device__ __forceinline__ bool contact_term(const ForceConst<T>& fc, bool h15, typename vec4_of<T>::type ke,
                                             typename vec2_of<T>::type ve, typename vec4_of<T>::type ko,
                                             typename vec2_of<T>::type vo, bool e_is_i, T& tx, T& ty, T& hm) {
    const T dx = e_is_i ? ko.x - ke.x : ke.x - ko.x;
    const T dy = e_is_i ? ko.y - ke.y : ke.y - ko.y;
    const T d2 = dx * dx + dy * dy;
    const T min_dist = e_is_i ? ke.z + ko.z : ko.z + ke.z;
    // d2 > (min_dist (1 + 1e-5))^2, all roundings included, puts the rounded
    // square root above min_dist, where the reference's overlap is exactly
    // 0: such candidates skip the square root (NaN falls through)
    const T mdm = min_dist * T(1.00001);
    if (d2 > mdm * mdm) return false;
    // the contact predicate, unfused as in the reference (jax_simulation.py:127-131)
    const T dist = jsqrt(d2);
    const T overlap = jmax(min_dist - dist, T(0));
    if (!((dist > T(1e-6)) && (overlap > T(0)))) return false;
    // direction = d / max(dist, 1e-10); here dist > 1e-6 (jax_simulation.py:133-136)
    const T ux = dx / dist, uy = dy / dist;
    const T fn = fc.hf * (h15 ? hertz15(overlap) : jpow(overlap, fc.hexp));
    const T fnx = ux * fn, fny = uy * fn;
    const T vrx = e_is_i ? vo.x - ve.x : ve.x - vo.x;
    const T vry = e_is_i ? vo.y - ve.y : ve.y - vo.y;
    // tangential relative velocity and kinetic friction (jax_simulation.py:139-149)
    const T vdot = vrx * ux + vry * uy;
    const T vtx = vrx - vdot * ux, vty = vry - vdot * uy;
    const T vtm = jsqrt(vtx * vtx + vty * vty);
    T ftx = T(0), fty = T(0);
    if (vtm > T(1e-6)) {
        const T ftm = jmin(fc.mu * fn, fc.fcap);
        ftx = (-vtx / vtm) * ftm;  // t_hat * f_t_mag
        fty = (-vty / vtm) * ftm;
    }
    const T oix = -fnx - ftx, oiy = -fny - fty;
    const T cr = -(dx * oiy - dy * oix);
    tx = e_is_i ? ftx - fnx : fnx - ftx;
    ty = e_is_i ? fty - fny : fny - fty;
    hm = T(0.5) * cr;
    return true;
}

// Contact-set recording (only when a.crec is set): one pair {e, o} whose
// contact term element e's force computation added.
template <typename T>
__device__ __forceinline__ void record_contact(const KArgs<T>& a, int e, int o) {
    const unsigned i = atomicAdd(a.crec_cnt, 1u);
    if (i < (unsigned)a.crec_cap) a.crec[i] = make_int2(e, o);
}

// Escape code of element e at its new position: 2 = escaped past this substep's
// threshold (processed before the next substep), 1 = lazily escaped (re-referenced
// during the next force phase), 0 = neither.
template <typename T>
__device__ __forceinline__ int esc_code(const KArgs<T>& a, const ForceCtx<T>& cx, int e, T px, T py) {
    if (cx.last) return 0;
    const T rx = a.pos_ref[2 * e], ry = a.pos_ref[2 * e + 1];
    if (escaped_from(px, py, rx, ry, cx.esc_h)) return 2;
    return (cx.lazy_detect && escaped_from(px, py, rx, ry, cx.h_lazy)) ? 1 : 0;
}

// Drag, rotational drag and the semi-implicit update of an active element
// from its bond and contact sums; stores the substep's output and returns
// its escape code (esc_code).
template <typename T>
__device__ __forceinline__ int integrate_element(const KArgs<T>& a, const Frame<T>& F, const ForceCtx<T>& cx, int e,
                                                  typename vec4_of<T>::type ke, typename vec2_of<T>::type ve,
                                                  typename vec4_of<T>::type ec, typename vec2_of<T>::type w, T sub,
                                                  typename vec2_of<T>::type so, T av, T rot, T fbx, T fby, T mb,
                                                  T fix, T fiy, T mi) {
    typedef typename vec4_of<T>::type V4;
    // drag (jax_simulation.py:167-192)
    const T m = ec.x, inertia = ec.y, h = ec.z, A = ec.w;
    const T a_drag = A * (h / a.fc.href);
    const T vrx = ve.x - w.x, vry = ve.y - w.y;
    const T vm = jsqrt(vrx * vrx + vry * vry);
    T fdx, fdy;
    if (vm > T(1e-6)) {
        // (v / |v|) * (c A |v|^2), evaluated as the reference writes it
        const T q = (a.fc.c_drag * a_drag) * (vm * vm);
        fdx = (vrx / vm) * q;
        fdy = (vry / vm) * q;
    } else {
        const T cl = a.fc.c_drag * a_drag * a.fc.lin;
        fdx = cl * vrx;
        fdy = cl * vry;
    }
    // rotational drag (jax_simulation.py:195-212)
    const T a_sub = A * jmin(sub / jmax(h, T(1e-10)), T(1));
    const T md = a.fc.c_rot * ke.w * av * fabs(av) * a_sub;
    const T Fx = ((fbx + fix) - fdx) + so.x;
    const T Fy = ((fby + fiy) - fdy) + so.y;
    const T Mz = (mb + mi) + md;
    // semi-implicit Euler (jax_simulation.py:215-268)
    const T dti = a.fc.dti, vclip = a.fc.vclip, pclip = a.fc.pclip;
    T nvx = jclip(ve.x + (Fx / m) * dti, -vclip, vclip);
    T nvy = jclip(ve.y + (Fy / m) * dti, -vclip, vclip);
    T npx = ke.x + nvx * dti, npy = ke.y + nvy * dti;
    const T alpha = Mz / inertia;
    const T nav = jclip(av * a.fc.damp + alpha * dti, a.fc.alo, a.fc.ahi);
    const T nrot = rot + nav * dti;
    if (!jfinite(nvx)) nvx = T(0);
    if (!jfinite(nvy)) nvy = T(0);
    if (!jfinite(npx)) npx = ke.x;
    if (!jfinite(npy)) npy = ke.y;
    npx = jclip(npx, -pclip, pclip);
    npy = jclip(npy, -pclip, pclip);
    if (cx.last) {
        st2(F.dst.pos, e, npx, npy);
        st2(F.dst.vel, e, nvx, nvy);
    } else {
        V4 v4;
        v4.x = npx;
        v4.y = npy;
        v4.z = ke.z;
        v4.w = ke.w;
        reinterpret_cast<V4*>(cx.kout)[e] = v4;
        st2(cx.kvout, e, nvx, nvy);
    }
    cx.rout[e] = nrot;
    cx.aout[e] = nav;
    return esc_code(a, cx, e, npx, npy);
}

// Forces, torque and the semi-implicit update of element e for one substep,
// one thread per element; returns e's escape code (esc_code).
//
// Latency layout: every load that depends only on e is issued first; then one
// loop walks the bond slots and the contact candidates together, kBatch of
// each per iteration, issuing the slot records and candidate indices of a
// batch at once, then all partner gathers at once.  Bond and contact sums keep
// separate accumulators, each in the reference's order (bond slots with
// e == bond_i first, then e == bond_j; candidates above e ascending, then
// below e ascending), so the interleaving does not change any rounding.
template <typename T>
__device__ __forceinline__ int force_element(const KArgs<T>& a, const Frame<T>& F, const ForceCtx<T>& cx,
                                              int e) {
    typedef typename vec2_of<T>::type V2;
    typedef typename vec4_of<T>::type V4;
    const T *kin = cx.kin, *kvin = cx.kvin;
    const SlotRec<T>* rec = cx.rec;
    const bool h15 = a.fc.h15 != 0;
    // loads that depend on e only
    const V4 ke = ld4(kin, e);  // x, y, radius, radius^3
    const V2 ve = ld2(kvin, e);
    if (!(cx.act[e] != 0)) {
        // a frozen element keeps its state (jax_simulation.py:257-262) whatever its
        // forces are, and no other element reads them (each element sums its own
        // bond and contact forces): carry the state over, compute nothing
        const T av0 = cx.ain[e], rot0 = cx.rin[e];
        if (cx.last) {
            st2(F.dst.pos, e, ke.x, ke.y);
            st2(F.dst.vel, e, ve.x, ve.y);
        } else {
            reinterpret_cast<V4*>(cx.kout)[e] = ke;
            st2(cx.kvout, e, ve.x, ve.y);
        }
        cx.rout[e] = rot0;
        cx.aout[e] = av0;
        return esc_code(a, cx, e, ke.x, ke.y);
    }
    const int s0 = a.boff[e], s1 = a.boff[e + 1];
    const int nc = a.ncnt[e];
    const V4 ec = ld4(a.econ, e);  // mass, inertia, thickness, area
    const V2 w = ld2(F.vw, e);
    const T sub = F.dst.sub[e];
    const V2 so = ld2(a.soi, e);
    const T av = cx.ain[e];
    const T rot = cx.rin[e];
    // bonds (jax_simulation.py:63-108) and ice-ice contacts (:111-164)
    T fbx = T(0), fby = T(0), mb = T(0);
    T fix = T(0), fiy = T(0), mi = T(0);
    const int nbe = s1 - s0;
    const int iters = max((nbe + kBatch - 1) / kBatch, (nc + kBatch - 1) / kBatch);
    for (int it = 0; it < iters; ++it) {
        const int bb = s0 + it * kBatch, cb = it * kBatch;
        SlotRec<T> r[kBatch];
        int idx[kBatch];
#pragma unroll
        for (int j = 0; j < kBatch; ++j) {
            if (bb + j < s1) {
                r[j] = rec[bb + j];
            } else {
                r[j].o = 0;
                r[j].omd = T(-1);
            }
            idx[j] = (cb + j < nc) ? a.nbr[(size_t)(cb + j) * a.n + e] : -1;
        }
        V2 kb[kBatch];
        V4 ko[kBatch];
        V2 vo[kBatch];
#pragma unroll
        for (int j = 0; j < kBatch; ++j) {
            if (r[j].omd >= T(0)) kb[j] = reinterpret_cast<const V2*>(kin)[2 * (r[j].o & 0x7fffffff)];
            if (idx[j] >= 0) {
                ko[j] = ld4(kin, idx[j]);
                vo[j] = ld2(kvin, idx[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < kBatch; ++j) {
            if (r[j].omd < T(0)) continue;  // no slot, broken, or active/frozen endpoints
            T fx, fy, cr;
            bond_term(r[j], kb[j], ke.x, ke.y, fx, fy, cr);
            if (!(r[j].o < 0)) {
                fbx += fx;
                fby += fy;
                mb += cr;
            } else {
                fbx -= fx;
                fby -= fy;
                mb -= cr;
            }
        }
#pragma unroll
        for (int j = 0; j < kBatch; ++j) {
            const int o = idx[j];
            if (o < 0) continue;
            const bool e_is_i = e < o;
            T tx, ty, hm;
            if (!contact_term(a.fc, h15, ke, ve, ko[j], vo[j], e_is_i, tx, ty, hm)) continue;
            if (a.crec) record_contact(a, e, o);
            fix += tx;
            fiy += ty;
            mi = e_is_i ? mi + hm : mi - hm;
        }
    }
    return integrate_element(a, F, cx, e, ke, ve, ec, w, sub, so, av, rot, fbx, fby, mb, fix, fiy, mi);
}

// The same substep for one active element computed by a whole warp: lane j
// takes bond slot j and contact candidate j (32 at a time), so all partner
// gathers are in flight at once; the terms then go through the warp's slice of
// shared memory, and every lane sums them in slot / candidate order, exactly as
// force_element adds them (a select keeps the sum unchanged for a slot without
// a term, so the loop has no branch and its reads pipeline).  The element's own
// loads for the integration are issued first, beside the gathers.  For
// substeps with few active elements, where one element's chain of dependent
// loads decides the phase's length.  Every lane returns the escape code.
template <typename T>
__device__ __forceinline__ int force_element_warp(const KArgs<T>& a, const Frame<T>& F, const ForceCtx<T>& cx,
                                                   int e) {
    typedef typename vec2_of<T>::type V2;
    typedef typename vec4_of<T>::type V4;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const T *kin = cx.kin, *kvin = cx.kvin;
    const bool h15 = a.fc.h15 != 0;
    __shared__ T s_terms[kThreads / 32][6 * 32];
    T* wt = s_terms[threadIdx.x >> 5];
    const V4 ke = ld4(kin, e);
    const V2 ve = ld2(kvin, e);
    const int s0 = a.boff[e], s1 = a.boff[e + 1];
    const int nc = a.ncnt[e];
    // the integration's own loads (no other warp writes these during the phase)
    const V4 ec = ld4(a.econ, e);
    const V2 w = ld2(F.vw, e);
    const T sub = F.dst.sub[e];
    const V2 so = ld2(a.soi, e);
    const T av = cx.ain[e], rot = cx.rin[e];
    const int nbe = s1 - s0;
    const int m = max(nbe, nc);
    T fbx = T(0), fby = T(0), mb = T(0);
    T fix = T(0), fiy = T(0), mi = T(0);
    for (int j0 = 0; j0 < m; j0 += 32) {
        const int j = j0 + lane;
        SlotRec<T> r;
        r.o = 0;
        r.omd = T(-1);
        if (j < nbe) r = cx.rec[s0 + j];
        const int o = (j < nc) ? a.nbr[(size_t)j * a.n + e] : -1;
        const bool bv = r.omd >= T(0);
        V2 kb;
        V4 ko;
        V2 vo;
        if (bv) kb = reinterpret_cast<const V2*>(kin)[2 * (r.o & 0x7fffffff)];
        if (o >= 0) {
            ko = ld4(kin, o);
            vo = ld2(kvin, o);
        }
        T bfx = T(0), bfy = T(0), bcr = T(0);
        if (bv) bond_term(r, kb, ke.x, ke.y, bfx, bfy, bcr);
        T tx = T(0), ty = T(0), hm = T(0);
        const bool eis = e < o;
        const bool cv = (o >= 0) && contact_term(a.fc, h15, ke, ve, ko, vo, eis, tx, ty, hm);
        if (cv && a.crec) record_contact(a, e, o);
        const unsigned bm = __ballot_sync(full, bv);
        const unsigned rm = __ballot_sync(full, bv && r.o < 0);
        const unsigned cm = __ballot_sync(full, cv);
        const unsigned em = __ballot_sync(full, cv && eis);
        wt[lane] = bfx;
        wt[32 + lane] = bfy;
        wt[64 + lane] = bcr;
        wt[96 + lane] = tx;
        wt[128 + lane] = ty;
        wt[160 + lane] = hm;
        __syncwarp();
        const int nbp = min(32, nbe - j0), ncp = min(32, nc - j0);  // warp-uniform
        // four terms per step: their twelve reads first, then the four sums in order
        for (int l0 = 0; l0 < nbp; l0 += 4) {
            T x[4], y[4], c[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int l = min(l0 + u, 31);
                x[u] = wt[l];
                y[u] = wt[32 + l];
                c[u] = wt[64 + l];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int l = (l0 + u) & 31;
                const bool on = (l0 + u < nbp) && ((bm >> l) & 1u), neg = (rm >> l) & 1u;
                const T sx = neg ? fbx - x[u] : fbx + x[u];
                const T sy = neg ? fby - y[u] : fby + y[u];
                const T sc = neg ? mb - c[u] : mb + c[u];
                fbx = on ? sx : fbx;
                fby = on ? sy : fby;
                mb = on ? sc : mb;
            }
        }
        for (int l0 = 0; l0 < ncp; l0 += 4) {
            T x[4], y[4], h[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int l = min(l0 + u, 31);
                x[u] = wt[96 + l];
                y[u] = wt[128 + l];
                h[u] = wt[160 + l];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int l = (l0 + u) & 31;
                const bool on = (l0 + u < ncp) && ((cm >> l) & 1u);
                const T sx = fix + x[u], sy = fiy + y[u];
                const T sm = ((em >> l) & 1u) ? mi + h[u] : mi - h[u];
                fix = on ? sx : fix;
                fiy = on ? sy : fiy;
                mi = on ? sm : mi;
            }
        }
        __syncwarp();  // the next pass overwrites the terms
    }
    int esc = 0;
    if (lane == 0) esc = integrate_element(a, F, cx, e, ke, ve, ec, w, sub, so, av, rot, fbx, fby, mb, fix, fiy, mi);
    return __shfl_sync(full, esc, 0);
}

template <typename T>
__device__ __forceinline__ void copy4(const T* __restrict__ s, T* __restrict__ d, bool plus_zero);

// Out of place (a frame that writes the caller's separate output), the state of
// every bond is copied to the output during the substeps, a slice of the bond
// groups of four per substep, by warps that have no element work there (the
// substeps of a frame with few active elements leave most warps idle).  A
// bond keeps its state unless it has an active end (jax_simulation.py:534-653:
// with both ends frozen no gate opens and no collision breaks it), and the
// fracture phase overwrites the copies of the bonds that have one.  The shear
// displacement is copied as x + 0 and the intact flag as 0/1, as the update
// itself would write them.  Warp `cw` of `ncw` copiers takes its share.
template <typename T>
__device__ __forceinline__ void copy_bond_slice(const KArgs<T>& a, const Frame<T>& F, int s, int cw, int ncw) {
    const int ng = (a.nb + 3) >> 2;
    const int g_lo = (int)((long long)ng * s / a.k_sub), g_hi = (int)((long long)ng * (s + 1) / a.k_sub);
    auto al16 = [](const void* p) { return ((size_t)p & 15u) == 0; };
    const bool vec = al16(F.src.ds) && al16(F.dst.ds) && al16(F.src.dmg) && al16(F.dst.dmg) && al16(F.src.dm0) &&
                     al16(F.dst.dm0) && al16(F.src.dmmax) && al16(F.dst.dmmax) &&
                     ((size_t)F.src.intact & 3u) == 0 && ((size_t)F.dst.intact & 3u) == 0;
    for (int g = g_lo + cw * 32 + (threadIdx.x & 31); g < g_hi; g += ncw * 32) {
        const int b0 = 4 * g;
        const int cnt = min(4, a.nb - b0);
        if (vec && cnt == 4) {
            copy4<T>(F.src.ds + b0, F.dst.ds + b0, true);
            copy4<T>(F.src.dmg + b0, F.dst.dmg + b0, false);
            copy4<T>(F.src.dm0 + b0, F.dst.dm0 + b0, false);
            copy4<T>(F.src.dmmax + b0, F.dst.dmmax + b0, false);
            const unsigned raw = *reinterpret_cast<const unsigned*>(F.src.intact + b0);
            unsigned in4 = 0u;
            for (int k = 0; k < 4; ++k)
                if ((raw >> (8 * k)) & 0xffu) in4 |= 1u << (8 * k);
            *reinterpret_cast<unsigned*>(F.dst.intact + b0) = in4;
        } else {
            for (int k = 0; k < cnt; ++k) {
                const int b = b0 + k;
                F.dst.ds[b] = F.src.ds[b] + T(0);
                F.dst.dmg[b] = F.src.dmg[b];
                F.dst.dm0[b] = F.src.dm0[b];
                F.dst.dmmax[b] = F.src.dmmax[b];
                F.dst.intact[b] = F.src.intact[b] != 0 ? 1 : 0;
            }
        }
    }
}

template <typename T>
__device__ void phase_force(const KArgs<T>& a, const Frame<T>& F, int s, unsigned round, int nd, int n_lazy,
                            int na) {
    const ForceCtx<T> cx = force_ctx(a, F, s);
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gsz = gridDim.x * blockDim.x;
    int* esc_ctr = (int*)&a.esc_cnt[s + 1];
    int* lazy_ctr = &a.lazy_cnt[s + 1];
    const int warp = gtid >> 5, nwarps = gsz >> 5, lane = threadIdx.x & 31;
    const bool has_dirty = nd > 0;
    if (has_dirty && gtid == 0) atomicAdd((unsigned long long*)&a.stats[4], (unsigned long long)nd);
    // The special items of this substep: elements whose list this round
    // invalidated (rebuilt, then computed, here; the element loop below skips
    // them), or the lazy escapes.  A few take a CTA each, so that a stencil scan
    // is one load round, on CTAs that then take no element work; many take a
    // warp each.
    const int nspecial = has_dirty ? nd : n_lazy;
    const bool cta_items = nspecial > 0 && a.mark_split != DEM_SPLIT_WARP &&
                           nspecial <= (int)gridDim.x / (a.mark_split == DEM_SPLIT_CTA ? 2 : 4);
    if (cta_items) {
        if ((int)blockIdx.x < nspecial) {  // uniform over the CTA
            if (has_dirty) {
                const int e = a.dirty_list[blockIdx.x];
                block_build(a, e);
                if (threadIdx.x < 32) {
                    // a frozen element's substep buffers and output are written for the frame
                    const int code = cx.act[e] ? force_element_warp(a, F, cx, e) : 0;
                    if (lane == 0 && code == 2) a.esc_list[atomicAdd(esc_ctr, 1)] = e;
                    if (lane == 0 && code == 1) a.lazy_list[atomicAdd(lazy_ctr, 1)] = e;
                }
            } else {
                lazy_escape_block(a, cx.kin, a.lazy_list[blockIdx.x], s + 1, round + 1u);
            }
            return;
        }
    } else if (has_dirty) {
        // one warp rebuilds the list, then computes the element
        __shared__ int sbuf[kThreads / 32][2 * kMaxNbLocal];
        __shared__ int scnt[kThreads / 32];
        const int wl = threadIdx.x >> 5;
        for (int q = warp; q < nd; q += nwarps) {
            const int e = a.dirty_list[q];
            warp_build(a, e, sbuf[wl], &scnt[wl]);
            // a frozen element's substep buffers and output are written for the frame
            const int code = cx.act[e] ? force_element_warp(a, F, cx, e) : 0;
            if (lane == 0 && code == 2) a.esc_list[atomicAdd(esc_ctr, 1)] = e;
            if (lane == 0 && code == 1) a.lazy_list[atomicAdd(lazy_ctr, 1)] = e;
            __syncwarp();
        }
    } else if (n_lazy > 0) {
        // lazy escapes of this substep: a warp each, beside the force work
        for (int q = warp; q < n_lazy; q += nwarps) lazy_escape_warp(a, cx.kin, a.lazy_list[q], s + 1, round + 1u);
    }
    // The warps that rebuilt a list (or took a lazy escape) above take no share
    // of the element loop (while enough warps remain), so they do not finish
    // the phase last; with a CTA per item, those CTAs' warps.
    const int skip = cta_items ? nspecial * (kThreads / 32) : ((nspecial < nwarps / 2) ? nspecial : 0);
    if (warp < skip) return;
    // Only active elements move (frozen ones were carried over by phase_reduce).
    // Chunks of 32 active elements: every warp starts with one chunk of its own,
    // then takes further chunks from a counter (the next grab is issued before
    // the current chunk is computed), so uneven chunks do not leave warps idle.
    const int nw2 = nwarps - skip;
    const bool copy_bonds = a.nb > 0 && F.src.ds != F.dst.ds;
    if (a.force_split == DEM_SPLIT_WARP || (a.force_split == DEM_SPLIT_AUTO && na <= 2 * nw2)) {
        // at most two active elements per warp: a warp per element
        for (int i = warp - skip; i < na; i += nw2) {
            const int e = a.act_list[i];
            if (has_dirty && a.dirty[e] == round) continue;
            const int code = force_element_warp(a, F, cx, e);
            if (lane == 0 && code == 2) a.esc_list[atomicAdd(esc_ctr, 1)] = e;
            if (lane == 0 && code == 1) a.lazy_list[atomicAdd(lazy_ctr, 1)] = e;
        }
        if (copy_bonds) {
            // the warps without an element copy this substep's slice; when every
            // warp has one, all of them copy after it
            const int busy = min(na, nw2);
            if (busy < nw2) {
                if (warp - skip >= busy) copy_bond_slice(a, F, s, warp - skip - busy, nw2 - busy);
            } else {
                copy_bond_slice(a, F, s, warp - skip, nw2);
            }
        }
        return;
    }
    const int nchunks = (na + 31) >> 5;
    int c = warp - skip;
    int* ctr = &a.work_cnt[s];
    // with work bins: lane k < kActBins holds the entries of bin k
    int bcnt = 0;
    if (kActBins > 1 && lane < kActBins) bcnt = *((volatile int*)&a.act_cnt[1 + lane]);
    while (c < nchunks) {
        int next = 0;
        if (lane == 0) next = nw2 + atomicAdd(ctr, 1);
        const int i = c * 32 + lane;
        int e = -1;
        if (kActBins > 1) {
            // entry i of the bins taken one after another (the warp is converged here)
            int off = i, b = 0;
#pragma unroll
            for (int k = 0; k < kActBins - 1; ++k) {
                const int ck = __shfl_sync(0xffffffffu, bcnt, k);
                if (b == k && off >= ck) {
                    off -= ck;
                    b = k + 1;
                }
            }
            if (i < na) e = a.act_list[(size_t)(1 + b) * a.n + off];
        } else if (i < na) {
            e = a.act_list[i];
        }
        if (e >= 0 && !(has_dirty && a.dirty[e] == round)) {
            const int code = force_element(a, F, cx, e);
            if (!cx.last) {
                warp_append(a.esc_list, esc_ctr, code == 2, e);
                warp_append(a.lazy_list, lazy_ctr, code == 1, e);
            }
        }
        c = __shfl_sync(0xffffffffu, next, 0);
    }
    if (copy_bonds) copy_bond_slice(a, F, s, warp - skip, nw2);
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
    const T dG = T(P.bond_G_c_II - P.bond_G_c_I);
    // (G_c^II - G_c^I) * ratio^eta with ratio in [0, 1]: exactly 0 when the energies are equal
    T g_c = T(P.bond_G_c_I) + ((dG != T(0)) ? dG * jpow(ratio, T(P.bond_eta_bk)) : dG * T(0));
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

// DPDEM floe eligibility after this frame's contact (jax_simulation.py:511-524):
// max(force * scale) == max(force) * scale because rounding is monotone.
template <typename T>
__device__ __forceinline__ bool new_elig(const KArgs<T>& a, const Frame<T>& F, int fl, T scale) {
    if (F.elig_in[fl]) return true;
    if (a.nb == 0 || !a.fcoll[fl]) return false;
    const unsigned long long bits = a.fmax[fl];
    const T fmx = (sizeof(T) == 4) ? T(__uint_as_float((unsigned)bits)) : T(__longlong_as_double((long long)bits));
    return fmx * scale > a.min_bstr * T(a.P.effective_strength_collision);
}

// ─── P_FRACTURE (jax_simulation.py:534-653) + history ───────────────────────
// thrust-cap scale of system `sys` for this frame (one value when nsys == 1)
template <typename T>
__device__ __forceinline__ T sys_scale(const KArgs<T>& a, T scale1, int sys) {
    return a.nsys == 1 ? scale1 : T(*((volatile double*)&a.fscal[4 * sys]));
}

// The full fracture update of bond b (jax_simulation.py:534-653), for a bond
// with an active end.
template <typename T>
__device__ __forceinline__ void fracture_bond(const KArgs<T>& a, const Frame<T>& F, T scale, int b) {
    typedef typename vec2_of<T>::type V2;
    const DemParams& P = a.P;
    const T mft = T(P.max_fracture_thickness);
    const T esc = T(P.effective_strength_collision);
    const T dti = T(P.dt_ice);
    const T kn = a.k_n, ks = a.k_s;
    const int i = a.bi[b], j = a.bj[b];
    const T ds0 = F.src.ds[b], cur_d = F.src.dmg[b], dmmax0 = F.src.dmmax[b], dm00 = F.src.dm0[b];
    const bool intact = F.src.intact[b] != 0;
    const T rest = a.rest[b], sbar = a.sbar[b], bstr = a.bstr[b];
    const V2 pi = ld2(F.dst.pos, i), pj = ld2(F.dst.pos, j);
    const V2 vi = ld2(F.dst.vel, i), vj = ld2(F.dst.vel, j);
    const bool both_act = F.dst.active[i] && F.dst.active[j];
    const int fli = a.floe_of[i], flj = a.floe_of[j];
    const bool breakable = (a.thick[i] <= mft) && (a.thick[j] <= mft);
    const T sc = sys_scale(a, scale, a.nsys > 1 ? a.sys_of[i] : 0);  // i and j share a system
    const T fmi = a.fraw[i] * sc, fmj = a.fraw[j] * sc;
    const bool at_crack = a.crack[i] || a.crack[j];
    const T scf = sys_scale(a, scale, a.nsys > 1 ? a.floe_sys[fli] : 0);
    const bool floe_ok = new_elig(a, F, fli, scf) && new_elig(a, F, flj, scf);
    T dx = pj.x - pi.x, dy = pj.y - pi.y;
    T dist = jsqrt(dx * dx + dy * dy);
    T dsafe = jmax(dist, T(1e-10));
    T bx = dx / dsafe, by = dy / dsafe;
    bool near = (fmi > T(0)) || (fmj > T(0));
    bool dpdem_ok = both_act && floe_ok && (near || at_crack) && breakable;
    T vrx = vj.x - vi.x, vry = vj.y - vi.y;
    T vn = vrx * bx + vry * by;
    T vtx = vrx - vn * bx, vty = vry - vn * by;
    T ds_incr = jsqrt(vtx * vtx + vty * vty) * dti;
    bool ds_gate = near && both_act && floe_ok && breakable;
    T new_ds = ds0 + (ds_gate ? ds_incr : T(0));
    T L0 = jmax(rest, T(1e-10));
    T delta_n = dist - rest;
    T dn_d = near ? delta_n : T(0);
    T sn = (kn * (dn_d / L0)) * (T(1) - cur_d);
    T st = (ks * (new_ds / L0)) * (T(1) - cur_d);
    T od = cur_d, omax = dmmax0, o0 = dm00;
    bool fin = intact;
    if (dpdem_ok) {
        // the damage law's result is only selected for DPDEM-eligible bonds
        // (jnp.where at jax_simulation.py:620-623); elsewhere the old state stays
        T nd, nmax, n0;
        bool nint;
        bond_damage<T>(P, delta_n, new_ds, sn, st, sbar, cur_d, omax, o0, intact, nd, nmax, n0, nint);
        od = nd;
        omax = nmax;
        o0 = n0;
        if (breakable) fin = nint;
    }
    // direct collision breaking (jax_simulation.py:629-637)
    bool coll_on = (fmi > T(0)) || (fmj > T(0));
    T coll_f = jmax(fmi, fmj);
    bool brk = intact && coll_on && (coll_f > bstr * esc) && breakable;
    fin = fin && !brk;
    F.dst.dmg[b] = od;
    F.dst.dmmax[b] = omax;
    F.dst.dm0[b] = o0;
    F.dst.ds[b] = new_ds;
    F.dst.intact[b] = fin ? 1 : 0;
    if (a.h_intact) a.h_intact[(size_t)F.f * a.nb + b] = fin ? 1 : 0;
}

template <typename T>
__device__ __forceinline__ void copy4(const T* __restrict__ s, T* __restrict__ d, bool plus_zero);
template <>
__device__ __forceinline__ void copy4<float>(const float* __restrict__ s, float* __restrict__ d, bool plus_zero) {
    float4 v = *reinterpret_cast<const float4*>(s);
    if (plus_zero) {
        v.x = v.x + 0.0f;
        v.y = v.y + 0.0f;
        v.z = v.z + 0.0f;
        v.w = v.w + 0.0f;
    }
    *reinterpret_cast<float4*>(d) = v;
}
template <>
__device__ __forceinline__ void copy4<double>(const double* __restrict__ s, double* __restrict__ d, bool plus_zero) {
    double2 v = reinterpret_cast<const double2*>(s)[0], w = reinterpret_cast<const double2*>(s)[1];
    if (plus_zero) {
        v.x = v.x + 0.0;
        v.y = v.y + 0.0;
        w.x = w.x + 0.0;
        w.y = w.y + 0.0;
    }
    reinterpret_cast<double2*>(d)[0] = v;
    reinterpret_cast<double2*>(d)[1] = w;
}

template <typename T>
__device__ void phase_fracture(const KArgs<T>& a, const Frame<T>& F, T scale) {
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gsz = gridDim.x * blockDim.x;
    const unsigned fstamp = frame_stamp(a, F);
    // the bonds with an active end (listed by phase_reduce) take the full
    // update; every other bond keeps its state, which the force phases have
    // copied already when the frame writes a separate output, or which is in
    // place; its history row is that state
    const int nfb = *((volatile int*)a.fb_cnt);
    if ((long long)nfb * 4 > (long long)a.nb) {
        // most bonds are listed: visit them in index order by their stamps,
        // with coalesced bond loads (the list's order is the append order)
        for (int b = gtid; b < a.nb; b += gsz)
            if (a.bstamp[b] == fstamp) fracture_bond(a, F, scale, b);
    } else {
        for (int i = gtid; i < nfb; i += gsz) fracture_bond(a, F, scale, a.fb_list[i]);
    }
    if (a.h_intact)
        for (int b = gtid; b < a.nb; b += gsz)
            if (a.bstamp[b] != fstamp) a.h_intact[(size_t)F.f * a.nb + b] = F.src.intact[b] != 0 ? 1 : 0;
    for (int e = gtid; e < a.n; e += gsz) {
        if (a.h_pos) {
            typename vec2_of<T>::type p = ld2(F.dst.pos, e);
            st2(a.h_pos + (size_t)F.f * a.n * 2, e, p.x, p.y);
        }
        if (a.h_rot) a.h_rot[(size_t)F.f * a.n + e] = F.dst.rot[e];
        if (a.h_sub) a.h_sub[(size_t)F.f * a.n + e] = F.dst.sub[e];
    }
    for (int fl = gtid; fl < a.nf; fl += gsz)
        F.dst.elig[fl] = new_elig(a, F, fl, sys_scale(a, scale, a.nsys > 1 ? a.floe_sys[fl] : 0)) ? 1 : 0;
    if (a.d_fmag)
        for (int e = gtid; e < a.n; e += gsz)
            a.d_fmag[e] = a.fraw[e] * sys_scale(a, scale, a.nsys > 1 ? a.sys_of[e] : 0);
    for (int i = gtid; i < a.k_sub + 2; i += gsz) {
        a.esc_cnt[i] = 0u;
        a.lazy_cnt[i] = 0;
        a.dirty_cnt[i] = 0;
        a.work_cnt[i] = 0;
    }
}

// ─── the kernel ─────────────────────────────────────────────────────────────
// Phase numbering inside a frame: 0 cull (+ grid compaction), 1 near-element
// contact, 2 contact forces, 3 reduce + vessel, then for substep s: 4+3s
// escape round (re-reference + mark), 5+3s rebuild of every list (only when
// most elements escaped), 6+3s force (rebuilding marked lists first); last:
// 4+3k fracture.  Whether a list phase runs is decided by every CTA from the
// same word after a barrier, so skipped phases skip their barrier too.
template <typename T>
__global__ void __launch_bounds__(kThreads, DEM_MIN_BLOCKS) dem_frames_kernel(const __grid_constant__ KArgs<T> a, int ph_lo, int ph_hi) {
    extern __shared__ unsigned char smem_raw[];
    T* hullw = reinterpret_cast<T*>(smem_raw);
    const int k = a.k_sub;
    const int per_frame = phases_per_frame(k);
    if (ph_hi > a.K * per_frame) ph_hi = a.K * per_frame;  // uniform over the grid
    const bool persistent = (a.mode == DEM_LAUNCH_PERSISTENT);
    if (persistent && a.ptimes && blockIdx.x == 0 && threadIdx.x == 0) a.ptimes[1] = globaltimer_ns();
    for (int ph = ph_lo; ph < ph_hi; ++ph) {
        const int f = ph / per_frame;
        const int p = ph % per_frame;
        if (a.crec && p >= 7 && (p - 7) % 3 == 0 && blockIdx.x == 0 && threadIdx.x == 0) {
            // the force phase of substep (p - 7) / 3 has ended (barrier or launch boundary)
            const int m = f * k + (p - 7) / 3;
            if (m < a.crec_max_marks) a.crec_marks[m] = (int)*((volatile unsigned*)a.crec_cnt);
        }
        Frame<T> F = make_frame(a, f);
        if (p == 0) {
            phase_cull(a, F);
        } else if (p == 1) {
            phase_near(a, F, hullw);
        } else if (p == 2) {
            phase_cforce(a, F);
        } else if (p == 3) {
            phase_reduce(a, F);
        } else if (p == per_frame - 1) {
            phase_fracture(a, F, T(*((volatile double*)&a.fscal[0])));
        } else {
            const int s = (p - 4) / 3;
            const int sub = (p - 4) % 3;
            const unsigned cnt = *((volatile unsigned*)&a.esc_cnt[s]);
            const bool all = (unsigned long long)cnt * 8ull > (unsigned long long)a.n;
            // lazily escaped elements are taken at even substeps with a successor
            const bool lazy_sub = a.lazy && (s % 2 == 0) && (s + 1 < k);
            const int n_lazy = lazy_sub ? *((volatile int*)&a.lazy_cnt[s]) : 0;
            // stamp of this rebuild round, unique since the dirty stamps were last cleared
            const unsigned round = a.round_base + (unsigned)(f * k + s) + 1u;
            if (sub == 0) {
                if (cnt == 0u) continue;  // uniform: no barrier either
                // with escapes to process now, the lazy ones of this substep join them
                phase_escape(a, a.kin[s & 1], cnt, n_lazy, s, round, all);
            } else if (sub == 1) {
                if (cnt == 0u || !all) continue;
                phase_build_all(a);
            } else {
                // lists to rebuild: this round's marks (escape phase, or the lazy
                // escapes of the previous substep); the counters are read
                // together, before any branch on them
                const int nd = *((volatile int*)&a.dirty_cnt[s]);
                const int na = *((volatile int*)a.act_cnt);
                phase_force(a, F, s, round, all ? 0 : nd, (cnt == 0u) ? n_lazy : 0, na);
            }
        }
        // a barrier after every phase but the last; with profiling on, after the
        // last one too, so that its end time is recorded
        if (persistent && (ph + 1 < ph_hi || a.ptimes)) {
            // failure-detection test: one CTA leaves, every other CTA's barrier
            // wait ends at its time limit with DEM_ERR_TIMEOUT
            if (ph == a.fail_phase && blockIdx.x == gridDim.x - 1) return;
            if (!grid_barrier(a)) return;
            if (a.ptimes && blockIdx.x == 0 && threadIdx.x == 0) {
                // phase end times (debug/profiling): entry i = [phase, globaltimer]
                const unsigned long long i = atomicAdd(a.ptimes, 1ull);
                if (i < (unsigned long long)kMaxPhaseTimes) {
                    a.ptimes[2 + 2 * i] = (unsigned long long)ph;
                    a.ptimes[3 + 2 * i] = globaltimer_ns();
                }
            }
        }
    }
}

// per-element constants packed for one vector load per substep
template <typename T>
__global__ void econ_kernel(const T* mass, const T* inertia, const T* thick, const T* area, int n, T* out) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    out[4 * (size_t)e + 0] = mass[e];
    out[4 * (size_t)e + 1] = inertia[e];
    out[4 * (size_t)e + 2] = thick[e];
    out[4 * (size_t)e + 3] = area[e];
}

// r^3 per element in the dtype (radii ** 3, jax_simulation.py:205)
template <typename T>
__global__ void cube_kernel(const T* r, int n, T* out) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) out[e] = jpow(r[e], T(3));
}

// per-slot bond constants: rest length and E * ((h_i + h_j) * 0.5) * factor in
// the dtype (jax_simulation.py:81-82)
template <typename T>
__global__ void slot_setup_kernel(const T* thick, const T* rest, const int* bi, const int* bj,
                                  const int2* slots, int n_slots, double E, double factor, T* slot_rest,
                                  T* slot_stiff) {
    int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= n_slots) return;
    int b = slots[sl].x & 0x7fffffff;
    T avg = (thick[bi[b]] + thick[bj[b]]) * T(0.5);
    slot_stiff[sl] = T(E) * avg * T(factor);
    slot_rest[sl] = rest[b];
}

}  // namespace dem
