// sg_kernels.cu — device kernels of the screening surrogate (include/surrogate_b200.h).
//
// The GEMM is the Blackwell tensor-core path: a 128 x BN output tile per CTA
// (BN = 64, 128 or 256), K consumed 64 bf16 at a time through a ring of
// shared-memory buffers (8, 6 or 4 deep, under 200 KB) that TMA fills (128-byte swizzled, the layout tcgen05 reads), one
// elected thread issuing tcgen05.mma into an fp32 accumulator in tensor
// memory, and all four warps reading it back (tcgen05.ld) for the fused
// epilogue (bias, ReLU, ReLU-derivative mask, fp32 or bf16 store).
// The other kernels are the surrogate's memory-bound glue: patch gathers for
// the convolutions and their adjoint, transposes, column sums, Adam and the loss.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "sg_tc.cuh"
#include "surrogate_b200.h"

namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;  // bf16 per 128-byte swizzled row
// stages of the operand ring: enough 64-deep K slices in flight to cover a
// TMA round trip behind the MMAs of the slices before it (32 KB a stage at
// BN = 128, 24 KB at BN = 64; both rings stay under 200 KB of shared memory)
template <int BN>
__host__ __device__ constexpr int stages_of() { return BN >= 256 ? 4 : BN >= 128 ? 6 : 8; }

struct GemmArgs {
    int M, N, K;
    void* D;
    int ldd, d_bf16;
    const float* bias;
    int relu;
    const __nv_bfloat16* mask;
    int ldm;
    int* err;
};

template <int BN>
constexpr size_t gemm_smem_bytes() {
    return 1024 + (size_t)stages_of<BN>() * (kBM * kBK * 2 + BN * kBK * 2) + 256;
}

static_assert(gemm_smem_bytes<64>() <= 232448 && gemm_smem_bytes<128>() <= 232448 &&
                  gemm_smem_bytes<256>() <= 232448,
              "operand ring above the 227 KB of shared memory a CTA may use");

template <int BN>
__global__ void __launch_bounds__(128, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, const GemmArgs g) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                           ~static_cast<uintptr_t>(1023));
    constexpr int kStages = stages_of<BN>();
    constexpr uint32_t kABytes = kBM * kBK * 2, kBBytes = BN * kBK * 2, kStage = kABytes + kBBytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + kStages * kStage);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 1);
    const uint32_t sbase = sg::smem_addr(base);
    const uint32_t bar0 = sg::smem_addr(bars);
    auto full = [&](int s) { return bar0 + 8u * (uint32_t)s; };
    auto empty = [&](int s) { return bar0 + 8u * (uint32_t)(kStages + s); };
    const uint32_t done = bar0 + 8u * (uint32_t)(2 * kStages);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;  // M tiles on x: no 65535 limit on M
    const int nk = (g.K + kBK - 1) / kBK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            sg::mbar_init(full(s), 1);
            sg::mbar_init(empty(s), 1);
        }
        sg::mbar_init(done, 1);
        sg::mbar_fence_init();
        sg::tma_prefetch(&ta);
        sg::tma_prefetch(&tb);
    }
    if (warp == 0) {
        sg::tmem_alloc(sg::smem_addr(tmem_slot), (uint32_t)BN);
        sg::tmem_relinquish();
    }
    sg::tc_fence_before();
    __syncthreads();
    sg::tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);

    bool ok = true;
    if (warp == 0 && lane == 0) {
        // TMA producer: stage s is refilled once the MMAs that read it have completed
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kStages;
            const uint32_t ph = (uint32_t)(kb / kStages) & 1u;
            if (!sg::mbar_wait(empty(s), ph ^ 1u)) {
                ok = false;
                break;
            }
            sg::mbar_expect_tx(full(s), kStage);
            sg::tma_load_2d(sbase + (uint32_t)s * kStage, &ta, full(s), kb * kBK, m0);
            sg::tma_load_2d(sbase + (uint32_t)s * kStage + kABytes, &tb, full(s), kb * kBK, n0);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: four K=16 steps per stage, advancing 32 bytes inside the swizzle atom
        constexpr uint32_t idesc = sg::idesc_bf16_f32(kBM, BN);
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kStages;
            const uint32_t ph = (uint32_t)(kb / kStages) & 1u;
            if (!sg::mbar_wait(full(s), ph)) {
                ok = false;
                break;
            }
            sg::tc_fence_after();
            const uint32_t a = sbase + (uint32_t)s * kStage, b = a + kABytes;
#pragma unroll
            for (int k = 0; k < kBK / 16; ++k)
                sg::mma_bf16(tmem, sg::desc_kmajor_sw128(a + 32u * k), sg::desc_kmajor_sw128(b + 32u * k), idesc,
                             (kb > 0 || k > 0) ? 1u : 0u);
            sg::mma_commit(empty(s));
        }
        // arrives once every MMA issued above has completed (also after a failed wait)
        sg::mma_commit(done);
    }
    __syncwarp();

    // epilogue: thread t owns accumulator row t (TMEM lane t)
    const bool got = sg::mbar_wait(done, 0);
    sg::tc_fence_after();
    if ((!ok || !got) && lane == 0) atomicExch(g.err, 1);
    const int row = warp * 32 + lane;
    const int gm = m0 + row;
    const bool row_ok = got && gm < g.M;
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
        float v[16];
        sg::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
        if (!row_ok) continue;
        const int n_here = min(16, g.N - (n0 + c));
        if (n_here <= 0) continue;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int col = n0 + c + j;
            float x = v[j];
            if (j < n_here) {
                if (g.bias) x += g.bias[col];
                if (g.relu) x = fmaxf(x, 0.0f);
                if (g.mask && !(__bfloat162float(g.mask[(size_t)gm * g.ldm + col]) > 0.0f)) x = 0.0f;
            }
            v[j] = x;
        }
        if (g.d_bf16) {
            __nv_bfloat16* d = reinterpret_cast<__nv_bfloat16*>(g.D) + (size_t)gm * g.ldd + n0 + c;
            if (n_here == 16 && (g.ldd % 8) == 0) {
                uint4 w[2];
                uint32_t* wp = reinterpret_cast<uint32_t*>(w);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                    wp[j] = *reinterpret_cast<uint32_t*>(&h);
                }
                reinterpret_cast<uint4*>(d)[0] = w[0];
                reinterpret_cast<uint4*>(d)[1] = w[1];
            } else {
                for (int j = 0; j < n_here; ++j) d[j] = __float2bfloat16_rn(v[j]);
            }
        } else {
            float* d = reinterpret_cast<float*>(g.D) + (size_t)gm * g.ldd + n0 + c;
            if (n_here == 16 && (g.ldd % 4) == 0) {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    reinterpret_cast<float4*>(d)[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
            } else {
                for (int j = 0; j < n_here; ++j) d[j] = v[j];
            }
        }
    }
    sg::tc_fence_before();
    __syncthreads();
    if (warp == 0) sg::tmem_dealloc(tmem, (uint32_t)BN);
}

// ─── tensor maps ────────────────────────────────────────────────────────────
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// Row-major bf16 (rows, cols) with row stride ld (elements), boxes of box_rows x 64.
bool make_map(CUtensorMap* map, const void* ptr, int rows, int cols, int ld, int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN>
int launch_gemm(const GemmArgs& g, const void* A, int lda, const void* B, int ldb, cudaStream_t st) {
    CUtensorMap ta, tb;
    if (!make_map(&ta, A, g.M, g.K, lda, kBM) || !make_map(&tb, B, g.N, g.K, ldb, BN)) return SG_ERR_CUDA;
    constexpr size_t smem = gemm_smem_bytes<BN>();
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(gemm_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
    if (attr != cudaSuccess) return SG_ERR_CUDA;
    dim3 grid((g.M + kBM - 1) / kBM, (g.N + BN - 1) / BN);
    gemm_kernel<BN><<<grid, 128, smem, st>>>(ta, tb, g);
    return cudaGetLastError() == cudaSuccess ? SG_OK : SG_ERR_CUDA;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// ─── glue kernels ───────────────────────────────────────────────────────────
__global__ void im2col_kernel(int B, int H, int W, int C, const __nv_bfloat16* __restrict__ X, int kpad,
                              __nv_bfloat16* __restrict__ cols) {
    const int Ho = H / 2, Wo = W / 2;
    const long long total = (long long)B * Ho * Wo * kpad;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i % kpad);
        const long long r = i / kpad;
        __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
        if (k < 9 * C) {
            const int c = k % C, t = k / C, kx = t % 3, ky = t / 3;
            const int ox = (int)(r % Wo), oy = (int)((r / Wo) % Ho), b = (int)(r / ((long long)Wo * Ho));
            const int iy = 2 * oy - 1 + ky, ix = 2 * ox - 1 + kx;
            if (iy >= 0 && iy < H && ix >= 0 && ix < W) v = X[(((long long)b * H + iy) * W + ix) * C + c];
        }
        cols[i] = v;
    }
}

__global__ void col2im_kernel(int B, int H, int W, int C, const float* __restrict__ dcols, int kpad,
                              const __nv_bfloat16* __restrict__ act, __nv_bfloat16* __restrict__ dX) {
    const int Ho = H / 2, Wo = W / 2;
    const long long total = (long long)B * H * W * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long long p = i / C;
        const int ix = (int)(p % W), iy = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
        float s = 0.0f;
        // patches (oy, ox) with iy = 2 oy - 1 + ky, ix = 2 ox - 1 + kx, in (ky, kx) order
        for (int ky = 0; ky < 3; ++ky) {
            const int ty = iy + 1 - ky;
            if (ty < 0 || (ty & 1) || (ty >> 1) >= Ho) continue;
            for (int kx = 0; kx < 3; ++kx) {
                const int tx = ix + 1 - kx;
                if (tx < 0 || (tx & 1) || (tx >> 1) >= Wo) continue;
                const long long row = ((long long)b * Ho + (ty >> 1)) * Wo + (tx >> 1);
                s += dcols[row * kpad + (ky * 3 + kx) * C + c];
            }
        }
        if (act && !(__bfloat162float(act[i]) > 0.0f)) s = 0.0f;
        dX[i] = __float2bfloat16_rn(s);
    }
}

__global__ void transpose_kernel(int rows, int cols, const __nv_bfloat16* __restrict__ in, int ld_in,
                                 __nv_bfloat16* __restrict__ out, int ld_out) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = by + j, c = bx + threadIdx.x;
        if (r < rows && c < cols) tile[j][threadIdx.x] = in[(size_t)r * ld_in + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int c = bx + j, r = by + threadIdx.x;
        if (r < rows && c < cols) out[(size_t)c * ld_out + r] = tile[threadIdx.x][j];
    }
}

// column sums: block (x) = 32 columns, threads (32, 8) walk the rows in a
// fixed interleave, then the 8 partial sums of a column are added in order
__global__ void colsum_kernel(int rows, int cols, const void* __restrict__ in, int ld, int in_bf16,
                              float* __restrict__ out) {
    __shared__ float part[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    float s = 0.0f;
    if (c < cols) {
        for (int r = threadIdx.y; r < rows; r += 8) {
            const size_t o = (size_t)r * ld + c;
            s += in_bf16 ? __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(in)[o])
                         : reinterpret_cast<const float*>(in)[o];
        }
    }
    part[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && c < cols) {
        float t = 0.0f;
        for (int j = 0; j < 8; ++j) t += part[j][threadIdx.x];
        out[c] = t;
    }
}

__global__ void adam_kernel(int rows, int cols, float* __restrict__ p, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps,
                            float c1, float c2, __nv_bfloat16* __restrict__ w, int ldw, __nv_bfloat16* __restrict__ wt,
                            int ldwt) {
    const long long n = (long long)rows * cols;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        const int r = (int)(i / cols), c = (int)(i % cols);
        const __nv_bfloat16 h = __float2bfloat16_rn(pi);
        w[(size_t)r * ldw + c] = h;
        if (wt) wt[(size_t)c * ldwt + r] = h;
    }
}

// one block: each thread sums a strided share, then a fixed-order tree
__global__ void mse_kernel(int rows, int n_out, const float* __restrict__ pred, int ldp,
                           const float* __restrict__ target, int ldt, __nv_bfloat16* __restrict__ grad, int ldg,
                           float* __restrict__ loss) {
    __shared__ float red[1024];
    const float inv = 1.0f / ((float)rows * (float)n_out);
    float s = 0.0f;
    const long long total = (long long)rows * ldg;
    for (long long i = threadIdx.x; i < total; i += blockDim.x) {
        const int r = (int)(i / ldg), c = (int)(i % ldg);
        float gv = 0.0f;
        if (c < n_out) {
            const float d = pred[(size_t)r * ldp + c] - target[(size_t)r * ldt + c];
            s += d * d;
            gv = 2.0f * d * inv;
        }
        grad[i] = __float2bfloat16_rn(gv);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss[0] = red[0] * inv;
}

__global__ void pack_rows_kernel(int rows, int enc_dim, const __nv_bfloat16* __restrict__ enc, int ld_enc,
                                 const int* __restrict__ enc_row, int n_extra, const float* __restrict__ extra,
                                 int ld_extra, __nv_bfloat16* __restrict__ x, int ldx) {
    const long long total = (long long)rows * ldx;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / ldx), c = (int)(i % ldx);
        __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
        if (c < enc_dim) {
            const int er = enc_row ? enc_row[r] : r;
            v = enc[(size_t)er * ld_enc + c];
        } else if (c < enc_dim + n_extra) {
            v = __float2bfloat16_rn(extra[(size_t)r * ld_extra + (c - enc_dim)]);
        }
        x[i] = v;
    }
}

__global__ void unpack_grad_kernel(int rows, int enc_dim, const __nv_bfloat16* __restrict__ dx, int ldx,
                                   const __nv_bfloat16* __restrict__ act, __nv_bfloat16* __restrict__ d_enc) {
    const long long total = (long long)rows * enc_dim;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / enc_dim), c = (int)(i % enc_dim);
        __nv_bfloat16 v = dx[(size_t)r * ldx + c];
        if (act && !(__bfloat162float(act[i]) > 0.0f)) v = __float2bfloat16_rn(0.0f);
        d_enc[i] = v;
    }
}

// out[r, :] = in[idx[r], :], rows of `bytes` bytes (16-byte units when aligned)
__global__ void gather_rows_kernel(int rows, long long bytes, const unsigned char* __restrict__ in, long long ld_in,
                                   const int* __restrict__ idx, unsigned char* __restrict__ out, long long ld_out,
                                   int vec16) {
    const long long per = vec16 ? bytes / 16 : bytes;
    const long long total = (long long)rows * per;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / per);
        const long long o = i % per;
        const unsigned char* src = in + (long long)idx[r] * ld_in;
        unsigned char* dst = out + (long long)r * ld_out;
        if (vec16)
            reinterpret_cast<uint4*>(dst)[o] = reinterpret_cast<const uint4*>(src)[o];
        else
            dst[o] = src[o];
    }
}

__global__ void to_bf16_kernel(long long n, const float* __restrict__ in, __nv_bfloat16* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = __float2bfloat16_rn(in[i]);
}

int grid_for(long long work, int threads = 256) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms < 1) sms = 148;
    }
    const long long b = (work + threads - 1) / threads;
    return (int)std::max<long long>(1, std::min<long long>(b, (long long)sms * 16));
}

int launched() { return cudaGetLastError() == cudaSuccess ? SG_OK : SG_ERR_CUDA; }

}  // namespace

extern "C" {

int sg_gemm(int32_t M, int32_t N, int32_t K, const void* A, int32_t lda, const void* B, int32_t ldb, void* D,
            int32_t ldd, int32_t d_dtype, const float* bias, int32_t relu, const void* mask, int32_t ldm, int32_t* err,
            void* stream) {
    if (M < 1 || N < 1 || K < 1 || !A || !B || !D || !err) return SG_ERR_INVALID;
    if (lda < K || ldb < K || (lda % 8) || (ldb % 8) || !aligned16(A) || !aligned16(B)) return SG_ERR_INVALID;
    if (ldd < N || (d_dtype != SG_OUT_F32 && d_dtype != SG_OUT_BF16)) return SG_ERR_INVALID;
    if (mask && ldm < N) return SG_ERR_INVALID;
    if ((N + 63) / 64 > 65535) return SG_ERR_INVALID;
    GemmArgs g{M, N, K, D, ldd, d_dtype == SG_OUT_BF16 ? 1 : 0, bias, relu ? 1 : 0,
               reinterpret_cast<const __nv_bfloat16*>(mask), ldm, err};
    cudaStream_t st = (cudaStream_t)stream;
    if (N <= 64) return launch_gemm<64>(g, A, lda, B, ldb, st);
    // 128 x 256 tiles halve the re-reads of A where they still fill a wave of
    // the 148 SMs (measured: 8192 x 512 x 2304 in 36.5 us against 48.9 us with
    // 128 x 128 tiles; with fewer tiles the narrower ones win)
    const long long tiles256 = (long long)((M + kBM - 1) / kBM) * ((N + 255) / 256);
    if (N >= 512 && tiles256 >= 128) return launch_gemm<256>(g, A, lda, B, ldb, st);
    return launch_gemm<128>(g, A, lda, B, ldb, st);
}

int sg_im2col(int32_t B, int32_t H, int32_t W, int32_t C, const void* X, int32_t kpad, void* cols, void* stream) {
    if (B < 1 || H < 2 || W < 2 || (H & 1) || (W & 1) || C < 1 || kpad < 9 * C || !X || !cols) return SG_ERR_INVALID;
    const long long work = (long long)B * (H / 2) * (W / 2) * kpad;
    im2col_kernel<<<grid_for(work), 256, 0, (cudaStream_t)stream>>>(
        B, H, W, C, reinterpret_cast<const __nv_bfloat16*>(X), kpad, reinterpret_cast<__nv_bfloat16*>(cols));
    return launched();
}

int sg_col2im(int32_t B, int32_t H, int32_t W, int32_t C, const float* dcols, int32_t kpad, const void* act,
              void* dX, void* stream) {
    if (B < 1 || H < 2 || W < 2 || (H & 1) || (W & 1) || C < 1 || kpad < 9 * C || !dcols || !dX) return SG_ERR_INVALID;
    const long long work = (long long)B * H * W * C;
    col2im_kernel<<<grid_for(work), 256, 0, (cudaStream_t)stream>>>(
        B, H, W, C, dcols, kpad, reinterpret_cast<const __nv_bfloat16*>(act), reinterpret_cast<__nv_bfloat16*>(dX));
    return launched();
}

int sg_transpose(int32_t rows, int32_t cols, const void* in, int32_t ld_in, void* out, int32_t ld_out,
                 void* stream) {
    if (rows < 1 || cols < 1 || !in || !out || ld_in < cols || ld_out < rows) return SG_ERR_INVALID;
    if ((cols + 31) / 32 > 2147483647 || (rows + 31) / 32 > 65535) return SG_ERR_INVALID;
    dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    transpose_kernel<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(
        rows, cols, reinterpret_cast<const __nv_bfloat16*>(in), ld_in, reinterpret_cast<__nv_bfloat16*>(out), ld_out);
    return launched();
}

int sg_colsum(int32_t rows, int32_t cols, const void* in, int32_t ld, int32_t in_bf16, float* out, void* stream) {
    if (rows < 1 || cols < 1 || !in || !out || ld < cols) return SG_ERR_INVALID;
    colsum_kernel<<<(cols + 31) / 32, dim3(32, 8), 0, (cudaStream_t)stream>>>(rows, cols, in, ld, in_bf16 ? 1 : 0,
                                                                              out);
    return launched();
}

int sg_adam(int32_t rows, int32_t cols, float* p, const float* g, float* m, float* v, float lr, float beta1,
            float beta2, float eps, int32_t t, void* w, int32_t ldw, void* wt, int32_t ldwt, void* stream) {
    if (rows < 1 || cols < 1 || !p || !g || !m || !v || !w || t < 1 || ldw < cols || (wt && ldwt < rows))
        return SG_ERR_INVALID;
    const float c1 = 1.0f - powf(beta1, (float)t), c2 = 1.0f - powf(beta2, (float)t);
    adam_kernel<<<grid_for((long long)rows * cols), 256, 0, (cudaStream_t)stream>>>(
        rows, cols, p, g, m, v, lr, beta1, beta2, eps, c1, c2, reinterpret_cast<__nv_bfloat16*>(w), ldw,
        reinterpret_cast<__nv_bfloat16*>(wt), ldwt);
    return launched();
}

int sg_mse(int32_t rows, int32_t n_out, const float* pred, int32_t ldp, const float* target, int32_t ldt,
           void* grad, int32_t ldg, float* loss, void* stream) {
    if (rows < 1 || n_out < 1 || !pred || !target || !grad || !loss || ldp < n_out || ldt < n_out || ldg < n_out)
        return SG_ERR_INVALID;
    mse_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(rows, n_out, pred, ldp, target, ldt,
                                                     reinterpret_cast<__nv_bfloat16*>(grad), ldg, loss);
    return launched();
}

int sg_pack_rows(int32_t rows, int32_t enc_dim, const void* enc, int32_t ld_enc, const int32_t* enc_row,
                 int32_t n_extra, const float* extra, int32_t ld_extra, void* x, int32_t ldx, void* stream) {
    if (rows < 1 || enc_dim < 0 || n_extra < 0 || ldx < enc_dim + n_extra || !x) return SG_ERR_INVALID;
    if ((enc_dim > 0 && (!enc || ld_enc < enc_dim)) || (n_extra > 0 && (!extra || ld_extra < n_extra)))
        return SG_ERR_INVALID;
    pack_rows_kernel<<<grid_for((long long)rows * ldx), 256, 0, (cudaStream_t)stream>>>(
        rows, enc_dim, reinterpret_cast<const __nv_bfloat16*>(enc), ld_enc, enc_row, n_extra, extra, ld_extra,
        reinterpret_cast<__nv_bfloat16*>(x), ldx);
    return launched();
}

int sg_unpack_grad(int32_t rows, int32_t enc_dim, const void* dx, int32_t ldx, const void* act, void* d_enc,
                   void* stream) {
    if (rows < 1 || enc_dim < 1 || !dx || !d_enc || ldx < enc_dim) return SG_ERR_INVALID;
    unpack_grad_kernel<<<grid_for((long long)rows * enc_dim), 256, 0, (cudaStream_t)stream>>>(
        rows, enc_dim, reinterpret_cast<const __nv_bfloat16*>(dx), ldx, reinterpret_cast<const __nv_bfloat16*>(act),
        reinterpret_cast<__nv_bfloat16*>(d_enc));
    return launched();
}

int sg_gather_rows(int32_t rows, int64_t row_bytes, const void* in, int64_t ld_in_bytes, const int32_t* idx,
                   void* out, int64_t ld_out_bytes, void* stream) {
    if (rows < 1 || row_bytes < 1 || !in || !idx || !out || ld_in_bytes < row_bytes || ld_out_bytes < row_bytes)
        return SG_ERR_INVALID;
    const bool v16 = (row_bytes % 16) == 0 && (ld_in_bytes % 16) == 0 && (ld_out_bytes % 16) == 0 && aligned16(in) &&
                     aligned16(out);
    const long long work = (long long)rows * (v16 ? row_bytes / 16 : row_bytes);
    gather_rows_kernel<<<grid_for(work), 256, 0, (cudaStream_t)stream>>>(
        rows, row_bytes, reinterpret_cast<const unsigned char*>(in), ld_in_bytes, idx,
        reinterpret_cast<unsigned char*>(out), ld_out_bytes, v16 ? 1 : 0);
    return launched();
}

int sg_to_bf16(int64_t n, const float* in, void* out, void* stream) {
    if (n < 0 || (n > 0 && (!in || !out))) return SG_ERR_INVALID;
    if (n == 0) return SG_OK;
    to_bf16_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(n, in, reinterpret_cast<__nv_bfloat16*>(out));
    return launched();
}

}  // extern "C"
