// dem_math.cuh — scalar helpers with the NumPy/JAX semantics the frame step relies on.
//
// The reference computes with jnp (XLA) ops whose NaN and rounding semantics
// differ from C's fmin/fmax: jnp.maximum/minimum/clip propagate NaN, jnp.sign(0)
// is 0, float `%` is a floor-mod whose result takes the divisor's sign.  The
// kernels are compiled with -fmad=false so that a*b+c rounds twice, as NumPy
// and XLA-CPU do, which keeps contact and fracture predicates computed from
// identical inputs identical.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace dem {

template <typename T> struct vec2_of;
template <> struct vec2_of<float> { typedef float2 type; };
template <> struct vec2_of<double> { typedef double2 type; };

template <typename T>
__device__ __forceinline__ typename vec2_of<T>::type ld2(const T* p, int i) {
    return reinterpret_cast<const typename vec2_of<T>::type*>(p)[i];
}
template <typename T>
__device__ __forceinline__ void st2(T* p, int i, T x, T y) {
    typename vec2_of<T>::type v;
    v.x = x;
    v.y = y;
    reinterpret_cast<typename vec2_of<T>::type*>(p)[i] = v;
}

// jnp.maximum / jnp.minimum: NaN in either operand gives NaN.
template <typename T> __device__ __forceinline__ T jmax(T a, T b) {
    return (a != a) ? a : ((b != b) ? b : (a > b ? a : b));
}
template <typename T> __device__ __forceinline__ T jmin(T a, T b) {
    return (a != a) ? a : ((b != b) ? b : (a < b ? a : b));
}
// jnp.clip(x, lo, hi) == minimum(maximum(x, lo), hi)
template <typename T> __device__ __forceinline__ T jclip(T x, T lo, T hi) {
    return jmin(jmax(x, lo), hi);
}
template <typename T> __device__ __forceinline__ T jsign(T x) {
    return (x > T(0)) ? T(1) : ((x < T(0)) ? T(-1) : x);  // 0 -> 0, NaN -> NaN
}
// Python / NumPy float remainder: result in [0, m) for m > 0.
template <typename T> __device__ __forceinline__ T pymod(T x, T m) {
    T r = fmod(x, m);
    if (r != T(0)) {
        if ((m < T(0)) != (r < T(0))) r += m;
    } else {
        r = copysign(T(0), m);
    }
    return r;
}
template <typename T> __device__ __forceinline__ bool jfinite(T x) { return isfinite(x); }

__device__ __forceinline__ float jpow(float a, float b) { return powf(a, b); }
__device__ __forceinline__ double jpow(double a, double b) { return pow(a, b); }
__device__ __forceinline__ float jsqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ double jsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ void jsincos(float a, float* s, float* c) { sincosf(a, s, c); }
__device__ __forceinline__ void jsincos(double a, double* s, double* c) { sincos(a, s, c); }
__device__ __forceinline__ float jcos(float a) { return cosf(a); }
__device__ __forceinline__ double jcos(double a) { return cos(a); }
__device__ __forceinline__ float jsin(float a) { return sinf(a); }
__device__ __forceinline__ double jsin(double a) { return sin(a); }

// NumPy's pairwise summation for a contiguous reduction of n <= 128 items
// (numpy/_core/src/umath/loops_utils.h): sequential below 8 items, otherwise
// eight interleaved partial sums combined as ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7))
// followed by the tail.  Used for the masked vertex mean of ship-contact pass 2.
template <typename T>
__device__ __forceinline__ T np_pairwise_sum(const T* a, int n) {
    if (n < 8) {
        T res = T(0);
        // NumPy starts from -0.0 for n < 8 and adds in order
        res = -T(0);
        for (int i = 0; i < n; ++i) res += a[i];
        return res;
    }
    T r[8];
    for (int j = 0; j < 8; ++j) r[j] = a[j];
    int i = 8;
    for (; i < n - (n % 8); i += 8)
        for (int j = 0; j < 8; ++j) r[j] += a[i + j];
    T res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; ++i) res += a[i];
    return res;
}

// Monotone bit patterns of non-negative floats for atomicMax.
__device__ __forceinline__ unsigned f2ord(float x) { return __float_as_uint(x); }
__device__ __forceinline__ unsigned long long d2ord(double x) {
    return (unsigned long long)__double_as_longlong(x);
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned atom_add_release_u32(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned atom_add_acqrel_u32(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

}  // namespace dem
