// lcb_mlp.cu — the light-curve surrogate: a small MLP trained and evaluated
// with hand-written sm_100a BF16 tensor-core kernels.
//
// The network maps the five physical parameters of a binary (q, iangle, r1,
// t1, t2, normalised by the caller) to a light curve on a fixed phase grid
// (standardised log fluxes): n_in -> width x n_hidden (GELU) -> n_out.  It is
// the cheap first stage of delayed-acceptance MCMC; the light-curve engine
// stays the second stage that decides every move.
//
// GEMM kernel (k_gemm): C[M x N] = A[M x K] . B[N x K]^T, both operands BF16
// row-major (K contiguous), FP32 accumulation in tensor memory:
//   - one CTA per 128 x TBN output tile (TBN = 256 when N >= 256, else 128),
//     sixteen warps; a K-split grid (blockIdx.z) for FP32 outputs;
//   - warp 0 lane 0 streams 64-wide K-slices of A and B into shared memory
//     with TMA (cp.async.bulk.tensor, 128-byte swizzle), four stages on
//     mbarriers;
//   - warp 1 lane 0 issues tcgen05.mma (kind::f16, M=128, N=TBN, K=16) from
//     shared-memory descriptors into a TBN-column TMEM accumulator, and
//     releases each stage with tcgen05.commit;
//   - every warp reads the accumulator back with tcgen05.ld (warp w: TMEM
//     lanes 32 (w % 4) .. + 31 = tile rows, every fourth 32-column chunk from
//     w / 4), applies the fused epilogue and stages each 32 x 32 chunk in the
//     idle operand buffers so the global stores are row-contiguous:
//       EPI_F32        out = acc                                  (weight gradients)
//       EPI_BIAS_GELU  z = acc + bias; out = bf16(gelu(z)); out2 = z  (hidden layers)
//       EPI_BIAS_F32   out = acc + bias                           (output layer)
//       EPI_DGELU      out = bf16(acc * gelu'(aux))               (backward through GELU)
//     the two BF16 modes optionally also write out transposed (outT).
// Every mbarrier wait is bounded; a time-out sets the error word and the CTA
// still releases its tensor memory.
//
// Training runs forward (keeping each hidden activation transposed as well),
// backward (weight gradients dZ^T . X over K = batch split across the SMs and
// summed in a fixed order; bias gradients as row sums of dZ^T; input gradients
// dZ . W^T through the dGELU epilogue, which also writes dZ^T for the next
// layer) and Adam on FP32 master weights; every step is a fixed launch
// sequence on the network's stream.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/lcurve_b200.h"
#include "../../include/lcurve_b200_surrogate.h"

namespace {

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
// Tiles: 128 rows x TBN columns (TBN = 256 when N allows: half the CTAs, the
// widest single-CTA MMA; 128 otherwise), K-slices of 64.
// 16 warps: warp 0 lane 0 issues the TMA copies, warp 1 lane 0 the MMAs; in the epilogue warp w
// reads TMEM lanes 32 (w % 4) .. + 31 (the quarter its warp id may access) and the column
// chunks w / 4, w / 4 + 4, ... of 32.
constexpr int BM = 128, BK = 64, STAGES = 4, GEMM_THREADS = 512, EPI_GROUPS = GEMM_THREADS / 128;
constexpr uint32_t TILE_A = BM * BK * 2;
template <int TBN>
__host__ __device__ constexpr uint32_t tile_b() { return (uint32_t)TBN * BK * 2; }

enum { EPI_F32 = 0, EPI_BIAS_GELU = 1, EPI_BIAS_F32 = 2, EPI_DGELU = 3 };

template <int TBN>
struct GemmSmem {
    uint8_t a[STAGES][TILE_A];  // 1024-byte aligned slices (128-byte swizzle atoms)
    uint8_t b[STAGES][tile_b<TBN>()];
    uint64_t full[STAGES], empty[STAGES], done;
    uint32_t tmem_base;
    int abort;
};
// the epilogue's per-warp staging (6 KB a warp) reuses a[] and b[]
static_assert((GEMM_THREADS / 32) * 6144 <= STAGES * (TILE_A + tile_b<128>()), "epilogue staging");

struct GemmArgs {
    int M, N, K;
    int kchunks;      // BK-chunks of K per split (blockIdx.z); all of K when not split
    int64_t zstride;  // elements between the FP32 outputs of consecutive splits
    const float* bias;
    const float* aux;
    void* out;
    void* out2;
    void* outT;       // optional (EPI_BIAS_GELU, EPI_DGELU): bf16 copy of out, transposed (N x M)
    int* err;
};

__device__ __forceinline__ uint32_t s_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* b) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(s_u32(b)));
}
__device__ __forceinline__ void bar_expect(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_test(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(s_u32(b)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// Bounded wait (about 2 s of SM clock).
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity) {
    if (bar_test(b, parity)) return true;
    long long t0 = clock64();
    while (!bar_test(b, parity)) {
        __nanosleep(32);
        if (clock64() - t0 > 4000000000LL) return false;
    }
    return true;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* b) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            s_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(s_u32(b))
        : "memory");
}
// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), descriptor version 1, base offset 0.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;             // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;   // stride byte offset
    d |= (uint64_t)1 << 46;             // version
    d |= (uint64_t)2 << 61;             // SWIZZLE_128B
    return d;
}
// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, both K-major, M = 128, N = TBN.
template <int TBN>
__host__ __device__ constexpr uint32_t idesc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TBN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(id), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t* b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(s_u32(b)) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

#define LCB_R8(i) "=r"(v[i]), "=r"(v[i + 1]), "=r"(v[i + 2]), "=r"(v[i + 3]), "=r"(v[i + 4]), "=r"(v[i + 5]), "=r"(v[i + 6]), "=r"(v[i + 7])
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : LCB_R8(0), LCB_R8(8), LCB_R8(16), LCB_R8(24)
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
#undef LCB_R8

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float dgelu(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// ---------------------------------------------------------------------------
// k_gemm
// ---------------------------------------------------------------------------
template <int MODE, int TBN>
__global__ void __launch_bounds__(GEMM_THREADS, 1)
    k_gemm(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmArgs g) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = s_u32(smem_raw);
    GemmSmem<TBN>& S = *reinterpret_cast<GemmSmem<TBN>*>(smem_raw + (((raw + 1023u) & ~1023u) - raw));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * TBN;
    const int kb = blockIdx.z * g.kchunks;                           // first K-chunk of this split
    const int nk = min((g.K + BK - 1) / BK - kb, g.kchunks);         // >= 1: the host makes no empty split

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            bar_init(&S.full[s]);
            bar_init(&S.empty[s]);
        }
        bar_init(&S.done);
        S.abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_u32(&S.tmem_base)),
                     "r"(TBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem_base;

    int issued = 0;  // TMA stages issued by the producer
    if (warp == 0 && lane == 0) {
        for (int kc = 0; kc < nk; ++kc) {
            const int s = kc % STAGES;
            if (kc >= STAGES && !bar_wait(&S.empty[s], ((kc / STAGES) - 1) & 1)) {
                S.abort = 1;
                break;
            }
            bar_expect(&S.full[s], TILE_A + tile_b<TBN>());
            tma_load_2d(S.a[s], &ta, (kb + kc) * BK, m0, &S.full[s]);
            tma_load_2d(S.b[s], &tb, (kb + kc) * BK, n0, &S.full[s]);
            issued = kc + 1;
        }
    } else if (warp == 1 && lane == 0) {
        for (int kc = 0; kc < nk; ++kc) {
            const int s = kc % STAGES;
            if (!bar_wait(&S.full[s], (kc / STAGES) & 1)) {
                S.abort = 1;
                break;
            }
            tc_fence_after();
            const uint64_t da = sw128_desc(s_u32(S.a[s])), db = sw128_desc(s_u32(S.b[s]));
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) umma(tmem, da + 2 * kk, db + 2 * kk, idesc<TBN>(), (kc | kk) != 0);
            umma_commit(&S.empty[s]);
        }
        umma_commit(&S.done);  // arrives once every MMA issued above has completed
    }
    __syncwarp();

    const bool ok = __all_sync(0xffffffffu, bar_wait(&S.done, 0));
    tc_fence_after();
    const int quarter = warp & 3;
    const int rbase = m0 + quarter * 32;          // first output row of this warp's TMEM lanes
    const int rows = min(32, g.M - rbase);        // rows in range (even when M is)
    // Per-warp staging, 32 rows x 32 columns as FP32 (4 KB) and as BF16 (2 KB), in the operand
    // buffers (idle once S.done has fired: every copy has landed and every MMA has read it).
    // 16-byte chunks are XOR-swizzled by row so the row-per-lane accesses (TMEM layout) and the
    // row-contiguous accesses of the global copies both spread over all banks.
    uint8_t* stage = &S.a[0][0] + warp * 6144;
    float* stf = reinterpret_cast<float*>(stage);
    uint8_t* stb = stage + 4096;
    auto f32_at = [&](int i, int c) { return reinterpret_cast<float4*>(stf + i * 32 + ((c ^ (i & 7)) << 2)); };
    auto b16_at = [&](int i, int c) { return reinterpret_cast<uint4*>(stb + i * 64 + ((c ^ ((i >> 1) & 3)) << 4)); };
    if (ok && rows > 0) {
        for (int c0 = (warp >> 2) * 32; c0 < TBN && n0 + c0 < g.N; c0 += 32 * EPI_GROUPS) {
            uint32_t v[32];
            tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0, v);
            const int nb = n0 + c0;
            const int nv = min(32, g.N - nb);  // multiple of 8 (N % 8 == 0)
            if (MODE == EPI_DGELU) {  // pre-activations in, row-contiguous
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int i = k * 4 + (lane >> 3), c = lane & 7;
                    if (i < rows && c * 4 < nv)
                        *f32_at(i, c) = __ldg(reinterpret_cast<const float4*>(g.aux + (size_t)(rbase + i) * g.N + nb + c * 4));
                }
                __syncwarp();
            }
            // lane = row: epilogue arithmetic into the staging tiles
            if (MODE == EPI_F32 || MODE == EPI_BIAS_F32) {
                for (int j = 0; j < nv; j += 4) {
                    float4 q;
                    q.x = __uint_as_float(v[j]) + (MODE == EPI_BIAS_F32 ? __ldg(g.bias + nb + j) : 0.f);
                    q.y = __uint_as_float(v[j + 1]) + (MODE == EPI_BIAS_F32 ? __ldg(g.bias + nb + j + 1) : 0.f);
                    q.z = __uint_as_float(v[j + 2]) + (MODE == EPI_BIAS_F32 ? __ldg(g.bias + nb + j + 2) : 0.f);
                    q.w = __uint_as_float(v[j + 3]) + (MODE == EPI_BIAS_F32 ? __ldg(g.bias + nb + j + 3) : 0.f);
                    *f32_at(lane, j >> 2) = q;
                }
            } else {
                for (int j = 0; j < nv; j += 8) {
                    float y[8];
                    if (MODE == EPI_BIAS_GELU) {
                        float z[8];
#pragma unroll
                        for (int t = 0; t < 8; ++t) {
                            z[t] = __uint_as_float(v[j + t]) + __ldg(g.bias + nb + j + t);
                            y[t] = gelu(z[t]);
                        }
                        *f32_at(lane, j >> 2) = make_float4(z[0], z[1], z[2], z[3]);
                        *f32_at(lane, (j >> 2) + 1) = make_float4(z[4], z[5], z[6], z[7]);
                    } else {  // EPI_DGELU
                        const float4 a0 = *f32_at(lane, j >> 2), a1 = *f32_at(lane, (j >> 2) + 1);
                        const float zz[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
                        for (int t = 0; t < 8; ++t) y[t] = __uint_as_float(v[j + t]) * dgelu(zz[t]);
                    }
                    __align__(16) __nv_bfloat162 h[4];
#pragma unroll
                    for (int t = 0; t < 4; ++t) h[t] = __floats2bfloat162_rn(y[2 * t], y[2 * t + 1]);
                    *b16_at(lane, j >> 3) = *reinterpret_cast<const uint4*>(h);
                    if (g.outT) {
                        // Transposed copy: rows r and r^1 (lanes l and l^1; rows is even) packed per
                        // column, the even lane storing column c and the odd lane column c + 1.
                        uint16_t* ot = reinterpret_cast<uint16_t*>(g.outT);
                        const int r = rbase + lane;
#pragma unroll
                        for (int t = 0; t < 4; ++t) {
                            const uint32_t w = *reinterpret_cast<const uint32_t*>(&h[t]);
                            const uint32_t other = __shfl_xor_sync(0xffffffffu, (lane & 1) ? (w & 0xffffu) : (w >> 16), 1);
                            const size_t c = (size_t)(nb + j + 2 * t);
                            if (lane < rows) {
                                if (lane & 1)
                                    *reinterpret_cast<uint32_t*>(ot + (c + 1) * g.M + r - 1) = other | (w & 0xffff0000u);
                                else
                                    *reinterpret_cast<uint32_t*>(ot + c * g.M + r) = (w & 0xffffu) | (other << 16);
                            }
                        }
                    }
                }
            }
            __syncwarp();
            // staging -> global, row-contiguous (8 lanes per 128-byte FP32 row, 4 per 64-byte BF16 row)
            if (MODE != EPI_DGELU) {
                float* dst = MODE == EPI_BIAS_GELU ? reinterpret_cast<float*>(g.out2)
                                                   : reinterpret_cast<float*>(g.out) + (size_t)blockIdx.z * g.zstride;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int i = k * 4 + (lane >> 3), c = lane & 7;
                    if (i < rows && c * 4 < nv)
                        *reinterpret_cast<float4*>(dst + (size_t)(rbase + i) * g.N + nb + c * 4) = *f32_at(i, c);
                }
            }
            if (MODE == EPI_BIAS_GELU || MODE == EPI_DGELU) {
                __nv_bfloat16* dst = reinterpret_cast<__nv_bfloat16*>(g.out);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int i = k * 8 + (lane >> 2), c = lane & 3;
                    if (i < rows && c * 8 < nv)
                        *reinterpret_cast<uint4*>(dst + (size_t)(rbase + i) * g.N + nb + c * 8) = *b16_at(i, c);
                }
            }
            __syncwarp();  // the staging tiles are rewritten by the next chunk
        }
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && (S.abort || !ok)) {
        // let copies still in flight land before the CTA's shared memory is released
        for (int kc = max(0, issued - STAGES); kc < issued; ++kc) (void)bar_wait(&S.full[kc % STAGES], (kc / STAGES) & 1);
        atomicExch(g.err, 1);
    }
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TBN));
    }
}

// ---------------------------------------------------------------------------
// element-wise / reduction kernels
// ---------------------------------------------------------------------------
// out[c][r] = in[r][c] (bf16), 32 x 32 tiles through shared memory.
__global__ void k_transpose(int rows, int cols, const uint16_t* __restrict__ in, uint16_t* __restrict__ out) {
    __shared__ uint16_t t[32][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = blockIdx.y * 32 + k;
        t[k][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * cols + c] : 0;
    }
    __syncthreads();
    const int r2 = blockIdx.y * 32 + threadIdx.x;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c2 = blockIdx.x * 32 + k;
        if (c2 < cols && r2 < rows) out[(size_t)c2 * rows + r2] = t[threadIdx.x][k];
    }
}

// out[i] = part[0][i] + part[1][i] + ... in that order: the FP32 partial products of a K-split GEMM
// (n a multiple of 4; the order is fixed, so the sum is the same on every run).
__global__ void k_sum_splits(int64_t n4, int splits, const float4* __restrict__ part, float4* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
        float4 s = __ldcs(part + i);
        for (int z = 1; z < splits; ++z) {
            const float4 t = __ldcs(part + (int64_t)z * n4 + i);
            s.x += t.x; s.y += t.y; s.z += t.z; s.w += t.w;
        }
        out[i] = s;
    }
}

// out[r] = sum over the columns of in[r][c] (bf16 in, fp32 out; cols a multiple of 8): one 256-thread
// block per row, 16-byte loads, a fixed summation order.
__global__ void __launch_bounds__(256) k_rowsum(int cols, const __nv_bfloat16* __restrict__ in, float* __restrict__ out) {
    __shared__ float red[8];
    const uint4* row = reinterpret_cast<const uint4*>(in + (size_t)blockIdx.x * cols);
    float s = 0.f;
#pragma unroll 4
    for (int c = threadIdx.x; c < cols / 8; c += 256) {
        const uint4 q = __ldg(row + c);
        const __nv_bfloat162* b = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const float2 f = __bfloat1622float2(b[t]);
            s += f.x + f.y;
        }
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < 8; ++w) t += red[w];
        out[blockIdx.x] = t;
    }
}

// Input rows (fp32, n_in wide) -> bf16 rows padded with zeros to ld columns.
__global__ void k_pack_input(int rows, int n_in, int ld, const float* __restrict__ x, __nv_bfloat16* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)rows * ld) return;
    const int r = (int)(i / ld), c = (int)(i % ld);
    out[i] = __float2bfloat16_rn(c < n_in ? x[(size_t)r * n_in + c] : 0.f);
}

// Mean-squared-error gradient: g = 2 (pred - target) / (rows * cols) as bf16;
// loss accumulates sum (pred - target)^2 / (rows * cols).
__global__ void k_mse_grad(int64_t n, float inv, const float* __restrict__ pred, const float* __restrict__ target,
                           __nv_bfloat16* __restrict__ g, double* loss) {
    __shared__ float red[32];
    float acc = 0.f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float d = pred[i] - target[i];
        g[i] = __float2bfloat16_rn(2.f * d * inv);
        acc += d * d;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        float a = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
        for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (threadIdx.x == 0 && loss) atomicAdd(loss, (double)a * inv);
    }
}

struct LayerTab {
    int n;
    int64_t off[9];       // start of W_l in the flat parameter vector; off[n] = total
    int out[8], in[8];    // W_l is out x in (in padded); b_l follows W_l
    int64_t wbf[8];       // offset of layer l in the bf16 weight copies
};

// Adam with decoupled weight decay on the FP32 master parameters; refreshes
// the bf16 weights (out x in) and their transpose (in x out).
__global__ void k_adam(int64_t n, LayerTab T, float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, __nv_bfloat16* __restrict__ wbf, __nv_bfloat16* __restrict__ wtbf,
                       float lr, float b1, float b2, float eps, float wd, float c1, float c2) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        int l = 0;
        while (l + 1 < T.n && i >= T.off[l + 1]) ++l;
        const int64_t w = i - T.off[l];
        const int64_t nw = (int64_t)T.out[l] * T.in[l];
        const float decay = w < nw ? wd : 0.f;
        const float pi = p[i] - lr * ((mi * c1) / (sqrtf(vi * c2) + eps) + decay * p[i]);
        p[i] = pi;
        if (w < nw) {
            const int r = (int)(w / T.in[l]), c = (int)(w % T.in[l]);
            const __nv_bfloat16 h = __float2bfloat16_rn(pi);
            wbf[T.wbf[l] + w] = h;
            wtbf[T.wbf[l] + (int64_t)c * T.out[l] + r] = h;
        }
    }
}

// bf16 copies of the weights (after a parameter upload).
__global__ void k_cast_weights(int64_t n, LayerTab T, const float* __restrict__ p, __nv_bfloat16* __restrict__ wbf,
                               __nv_bfloat16* __restrict__ wtbf) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int l = 0;
        while (l + 1 < T.n && i >= T.off[l + 1]) ++l;
        const int64_t w = i - T.off[l];
        if (w < (int64_t)T.out[l] * T.in[l]) {
            const int r = (int)(w / T.in[l]), c = (int)(w % T.in[l]);
            const __nv_bfloat16 h = __float2bfloat16_rn(p[i]);
            wbf[T.wbf[l] + w] = h;
            wtbf[T.wbf[l] + (int64_t)c * T.out[l] + r] = h;
        }
    }
}

// Per-row chi-squared of a surrogate curve: flux_j = exp(pred_j * sd_j + mean_j),
// optionally scaled by the least-squares factor (orchestration.rs:361-401 re_scale).
__global__ void k_logflux_chisq(int rows, int n, const float* __restrict__ pred, const float* __restrict__ mean,
                                const float* __restrict__ sd, const double* __restrict__ flux,
                                const double* __restrict__ ferr, int scale, double* __restrict__ out) {
    __shared__ double red[3][8];
    const int r = blockIdx.x;
    if (r >= rows) return;
    double sff = 0, sfd = 0, sdd = 0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double f = exp((double)pred[(size_t)r * n + j] * sd[j] + mean[j]);
        const double w = 1.0 / (ferr[j] * ferr[j]);
        sff += w * f * f;
        sfd += w * f * flux[j];
        sdd += w * flux[j] * flux[j];
    }
    for (int o = 16; o; o >>= 1) {
        sff += __shfl_xor_sync(0xffffffffu, sff, o);
        sfd += __shfl_xor_sync(0xffffffffu, sfd, o);
        sdd += __shfl_xor_sync(0xffffffffu, sdd, o);
    }
    const int wid = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][wid] = sff;
        red[1][wid] = sfd;
        red[2][wid] = sdd;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, c = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            a += red[0][k];
            b += red[1][k];
            c += red[2][k];
        }
        const double s = scale ? (a > 0 ? b / a : 0.0) : 1.0;
        out[r] = c - 2 * s * b + s * s * a;  // sum w (d - s f)^2
    }
}

// ---------------------------------------------------------------------------
// surrogate sub-chain: stretch moves under the surrogate posterior, on device
// ---------------------------------------------------------------------------
constexpr int kMaxDim = 8;

enum { MOVE_STRETCH = 0, MOVE_KDE = 1 };

struct StretchArgs {
    int n, m, d, n_in;
    int move;              // MOVE_STRETCH or MOVE_KDE
    int rstride;           // random numbers per move: 3 (stretch) or 3 + d (KDE)
    double* y;             // n x d sub-chain positions (in/out)
    double* ls;            // n surrogate log probabilities (in/out)
    const double* comp;    // m x d complementary walkers (fixed)
    const double* rnd;     // K x n x rstride: uniform (z / component), uniform (partner), log uniform, d normals (KDE)
    double* yp;            // n x d proposals
    double* lz;            // n: log proposal-density ratio, or -inf outside the prior box
    double* lq;            // n: KDE log density at the current positions
    double* lqp;           // n: KDE log density at the proposals
    float* xin;            // n x n_in network inputs
    double lo[kMaxDim], hi[kMaxDim];
    float fmul[kMaxDim], fadd[kMaxDim];
    int frecip[kMaxDim];
    double a;
    const double* kde;     // device: chol[8 x 8] then prec[8 x 8] -- KDE kernel covariance h^2 S =
                           // chol chol^T (row-major, lower) and its inverse; a buffer, not a kernel
                           // parameter, so one captured graph serves every half-step
};

// log of the Gaussian KDE of the complementary walkers at v (up to a constant),
// log sum_j exp(-(v - c_j)^T prec (v - c_j) / 2), computed by one warp: each lane
// takes every 32nd component, then a log-sum-exp across the warp.  Every lane
// returns the value.
__device__ double kde_logq_warp(const StretchArgs& A, const double* v) {
    const int lane = threadIdx.x & 31;
    const double* prec = A.kde + kMaxDim * kMaxDim;
    double mx = -INFINITY, acc = 0.0;
    for (int j = lane; j < A.m; j += 32) {
        double dv[kMaxDim];
        for (int k = 0; k < A.d; ++k) dv[k] = v[k] - A.comp[(size_t)j * A.d + k];
        double qf = 0.0;
        for (int k = 0; k < A.d; ++k) {
            double t = 0.0;
            for (int l = 0; l < A.d; ++l) t += prec[k * kMaxDim + l] * dv[l];
            qf += dv[k] * t;
        }
        const double e = -0.5 * qf;
        if (e > mx) {
            acc = acc * exp(mx - e) + 1.0;
            mx = e;
        } else {
            acc += exp(e - mx);
        }
    }
    double wmx = mx;
    for (int o = 16; o > 0; o >>= 1) wmx = fmax(wmx, __shfl_xor_sync(0xffffffffu, wmx, o));
    double part = mx == -INFINITY ? 0.0 : acc * exp(mx - wmx);
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    return wmx + log(part);
}

constexpr int kWalkersPerBlock = 4;  // one warp per walker in the KDE kernels

__global__ void k_kde_logq(StretchArgs A) {
    const int i = blockIdx.x * kWalkersPerBlock + (threadIdx.x >> 5);
    if (i >= A.n || A.move != MOVE_KDE) return;  // uniform per warp
    double v[kMaxDim];
    for (int k = 0; k < A.d; ++k) v[k] = A.y[(size_t)i * A.d + k];
    const double lq = kde_logq_warp(A, v);
    if ((threadIdx.x & 31) == 0) A.lq[i] = lq;
}

// KDE move (emcee's KDEMove): an independence proposal from the Gaussian KDE
// of the complementary walkers, y' = c_j + chol eps, for walker i (one warp);
// writes y', its network inputs and the log density ratio log q(y) - log q(y'),
// or -inf outside the prior box.
__global__ void k_kde_propose(StretchArgs A, int step) {
    const int i = blockIdx.x * kWalkersPerBlock + (threadIdx.x >> 5);
    if (i >= A.n) return;  // uniform per warp
    const bool lead = (threadIdx.x & 31) == 0;
    const double* r = A.rnd + ((size_t)step * A.n + i) * A.rstride;
    const int j = min((int)(r[0] * A.m), A.m - 1);
    double v[kMaxDim];
    bool inside = true;
    for (int k = 0; k < A.d; ++k) {
        double t = 0.0;
        for (int l = 0; l <= k; ++l) t += A.kde[k * kMaxDim + l] * r[3 + l];
        v[k] = A.comp[(size_t)j * A.d + k] + t;
        inside = inside && v[k] >= A.lo[k] && v[k] <= A.hi[k];
        if (lead) {
            A.yp[(size_t)i * A.d + k] = v[k];
            const double f = A.frecip[k] ? 1.0 / v[k] : v[k];
            A.xin[(size_t)i * A.n_in + k] = (float)__dadd_rn((double)A.fadd[k], __dmul_rn((double)A.fmul[k], f));
        }
    }
    const double lqp = kde_logq_warp(A, v);
    if (lead) {
        A.lqp[i] = lqp;
        A.lz[i] = inside ? A.lq[i] - lqp : -INFINITY;
    }
}

// Goodman & Weare stretch proposal y' = c + z (y - c), z ~ g(z) on [1/a, a];
// the network input of y' is fadd + fmul * (y' or 1/y') per dimension.  (The
// KDE move, emcee's KDEMove, is k_kde_propose above.)
__global__ void k_stretch_propose(StretchArgs A, int step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const double* r = A.rnd + ((size_t)step * A.n + i) * A.rstride;
    // explicitly rounded operations (no contraction), so the moves are the
    // ones a host implementation of the same formulas makes
    double z = __dadd_rn(__dmul_rn(A.a - 1.0, r[0]), 1.0);
    z = __ddiv_rn(__dmul_rn(z, z), A.a);
    const int j = min((int)(r[1] * A.m), A.m - 1);
    bool inside = true;
    for (int k = 0; k < A.d; ++k) {
        const double c = A.comp[(size_t)j * A.d + k];
        const double v = __dadd_rn(c, __dmul_rn(z, __dsub_rn(A.y[(size_t)i * A.d + k], c)));
        A.yp[(size_t)i * A.d + k] = v;
        inside = inside && v >= A.lo[k] && v <= A.hi[k];
        const double f = A.frecip[k] ? 1.0 / v : v;
        // separate multiply and add (no contraction): the host computes the inputs the same way
        A.xin[(size_t)i * A.n_in + k] = (float)__dadd_rn((double)A.fadd[k], __dmul_rn((double)A.fmul[k], f));
    }
    A.lz[i] = inside ? (A.d - 1) * log(z) : -INFINITY;
}

// Metropolis step of the sub-chain: accept y' with min(1, z^(d-1) exp(l~(y') - l~(y))),
// l~ = -chisq / 2 inside the prior box.
__global__ void k_stretch_accept(StretchArgs A, const double* __restrict__ chi, int step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const double lz = A.lz[i];
    if (lz == -INFINITY) return;
    double lsp = -0.5 * chi[i];
    if (!(lsp == lsp)) lsp = -INFINITY;
    const double logu = A.rnd[((size_t)step * A.n + i) * A.rstride + 2];
    if (logu < lz + lsp - A.ls[i]) {
        for (int k = 0; k < A.d; ++k) A.y[(size_t)i * A.d + k] = A.yp[(size_t)i * A.d + k];
        A.ls[i] = lsp;
        if (A.move == MOVE_KDE) A.lq[i] = A.lqp[i];
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
thread_local std::string t_err;

struct Fail : std::runtime_error {
    int code;
    Fail(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(expr)                                                                                                   \
    do {                                                                                                           \
        cudaError_t e_ = (expr);                                                                                   \
        if (e_ != cudaSuccess) throw Fail(LCB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));       \
    } while (0)

template <class F>
int guard(F&& f) {
    try {
        f();
        return LCB_OK;
    } catch (const Fail& e) {
        t_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        t_err = e.what();
        return LCB_ERR_INVALID;
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    if (!fn) throw Fail(LCB_ERR_NO_DEVICE, "cuTensorMapEncodeTiled is not available from the driver");
    return fn;
}

// Tensor map of a row-major bf16 matrix (rows x cols), boxes of 64 columns x 128 rows, 128-byte swizzle.
CUtensorMap bf16_map(const void* ptr, int64_t rows, int64_t cols, uint32_t box_rows) {
    if (((uintptr_t)ptr & 15) || (cols % 8)) throw Fail(LCB_ERR_INVALID, "GEMM operand: 16-byte alignment and cols % 8 == 0 required");
    CUtensorMap m;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    cuuint32_t box[2] = {(cuuint32_t)BK, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Fail(LCB_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

template <int TBN>
constexpr size_t gemm_smem() { return sizeof(GemmSmem<TBN>) + 1024; }

template <int MODE, int TBN>
void launch_gemm_mode(const CUtensorMap& ta, const CUtensorMap& tb, const GemmArgs& g, cudaStream_t s) {
    static cudaError_t attr =
        cudaFuncSetAttribute(k_gemm<MODE, TBN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem<TBN>());
    CK(attr);
    dim3 grid((g.M + BM - 1) / BM, (g.N + TBN - 1) / TBN, (unsigned)(((g.K + BK - 1) / BK + g.kchunks - 1) / g.kchunks));
    k_gemm<MODE, TBN><<<grid, GEMM_THREADS, gemm_smem<TBN>(), s>>>(ta, tb, g);
    CK(cudaGetLastError());
}

// Sets the dynamic shared-memory limit of every GEMM variant (needed before a
// stream capture, during which the first launch of a variant cannot set it).
void prepare_gemm_attributes() {
#define LCB_SMEM_ATTR(M, T) \
    CK(cudaFuncSetAttribute(k_gemm<M, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem<T>()))
    LCB_SMEM_ATTR(EPI_F32, 128); LCB_SMEM_ATTR(EPI_BIAS_GELU, 128); LCB_SMEM_ATTR(EPI_BIAS_F32, 128);
    LCB_SMEM_ATTR(EPI_DGELU, 128);
    LCB_SMEM_ATTR(EPI_F32, 256); LCB_SMEM_ATTR(EPI_BIAS_GELU, 256); LCB_SMEM_ATTR(EPI_BIAS_F32, 256);
    LCB_SMEM_ATTR(EPI_DGELU, 256);
#undef LCB_SMEM_ATTR
}

int tile_n(int64_t N) { return N >= 256 ? 256 : 128; }  // 128 x 256 tiles where N allows

// Number of K-splits for an FP32-output GEMM: enough CTAs to cover `sms` SMs, none of them empty.
int split_count(int64_t M, int64_t N, int64_t K, int sms) {
    const int64_t tiles = ((M + BM - 1) / BM) * ((N + tile_n(N) - 1) / tile_n(N)), nk = (K + BK - 1) / BK;
    const int64_t s = std::max<int64_t>(1, std::min<int64_t>(sms / tiles, nk)), kc = (nk + s - 1) / s;
    return (int)((nk + kc - 1) / kc);
}

// Upper bound of split_count(M, N, K, sms) over every K.
int max_split_count(int64_t M, int64_t N, int sms) {
    const int64_t tiles = ((M + BM - 1) / BM) * ((N + tile_n(N) - 1) / tile_n(N));
    return (int)std::max<int64_t>(1, sms / tiles);
}

// splits > 1 (EPI_F32 only): split z writes its partial product to out + z * M * N.
void gemm(int mode, int64_t M, int64_t N, int64_t K, const void* A, const void* B, const float* bias, const float* aux,
          void* out, void* out2, int* err, cudaStream_t s, int splits = 1, void* outT = nullptr) {
    if (M <= 0 || N <= 0 || K <= 0 || N % 8 || K % 8 || M > INT32_MAX || N > 65535 * (int64_t)128)
        throw Fail(LCB_ERR_INVALID, "GEMM sizes: M, N, K > 0 and N, K multiples of 8 required");
    if (((uintptr_t)out & 15) || (out2 && ((uintptr_t)out2 & 15)) || (aux && ((uintptr_t)aux & 15)))
        throw Fail(LCB_ERR_INVALID, "GEMM outputs must be 16-byte aligned");
    if ((mode == EPI_BIAS_GELU || mode == EPI_BIAS_F32) && !bias) throw Fail(LCB_ERR_INVALID, "bias required");
    if (mode == EPI_BIAS_GELU && !out2) throw Fail(LCB_ERR_INVALID, "pre-activation output required");
    if (mode == EPI_DGELU && !aux) throw Fail(LCB_ERR_INVALID, "pre-activation input required");
    if (!err) throw Fail(LCB_ERR_INVALID, "error word required");
    if (outT && ((mode != EPI_BIAS_GELU && mode != EPI_DGELU) || M % 2 || ((uintptr_t)outT & 3)))
        throw Fail(LCB_ERR_INVALID, "transposed copy: bf16 modes, even M, 4-byte aligned");
    const int nk = (int)((K + BK - 1) / BK), kchunks = (nk + splits - 1) / std::max(splits, 1);
    if (splits < 1 || (splits > 1 && mode != EPI_F32) || (nk + kchunks - 1) / kchunks != splits)
        throw Fail(LCB_ERR_INVALID, "GEMM K-split must be an FP32-output split with no empty part");
    const bool wide = tile_n(N) == 256;
    const CUtensorMap ta = bf16_map(A, M, K, 128u), tb = bf16_map(B, N, K, wide ? 256u : 128u);
    GemmArgs g{(int)M, (int)N, (int)K, kchunks, M * N, bias, aux, out, out2, outT, err};
    switch (mode * 2 + (wide ? 1 : 0)) {
        case EPI_F32 * 2: launch_gemm_mode<EPI_F32, 128>(ta, tb, g, s); break;
        case EPI_F32 * 2 + 1: launch_gemm_mode<EPI_F32, 256>(ta, tb, g, s); break;
        case EPI_BIAS_GELU * 2: launch_gemm_mode<EPI_BIAS_GELU, 128>(ta, tb, g, s); break;
        case EPI_BIAS_GELU * 2 + 1: launch_gemm_mode<EPI_BIAS_GELU, 256>(ta, tb, g, s); break;
        case EPI_BIAS_F32 * 2: launch_gemm_mode<EPI_BIAS_F32, 128>(ta, tb, g, s); break;
        case EPI_BIAS_F32 * 2 + 1: launch_gemm_mode<EPI_BIAS_F32, 256>(ta, tb, g, s); break;
        case EPI_DGELU * 2: launch_gemm_mode<EPI_DGELU, 128>(ta, tb, g, s); break;
        case EPI_DGELU * 2 + 1: launch_gemm_mode<EPI_DGELU, 256>(ta, tb, g, s); break;
        default: throw Fail(LCB_ERR_INVALID, "unknown GEMM epilogue mode");
    }
}

void sum_splits(int64_t n, int splits, const float* part, float* out, cudaStream_t s) {
    const int64_t n4 = n / 4;
    k_sum_splits<<<(unsigned)std::min<int64_t>((n4 + 255) / 256, 1184), 256, 0, s>>>(
        n4, splits, reinterpret_cast<const float4*>(part), reinterpret_cast<float4*>(out));
    CK(cudaGetLastError());
}

void transpose(int64_t rows, int64_t cols, const void* in, void* out, cudaStream_t s) {
    dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
    k_transpose<<<grid, dim3(32, 8), 0, s>>>((int)rows, (int)cols, (const uint16_t*)in, (uint16_t*)out);
    CK(cudaGetLastError());
}

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        n = count;
        CK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
        CK(cudaMemset(p, 0, std::max<size_t>(count, 1) * sizeof(T)));
    }
    void free() {
        if (p) cudaFree(p);
        p = nullptr;
    }
};

}  // namespace

struct lcb_mlp {
    int device = 0;
    int n_in = 0, width = 0, n_hidden = 0, n_out = 0, nl = 0;
    int64_t max_batch = 0;
    int sms = 0;                      // SM count (sizes the K-splits of the weight-gradient GEMMs)
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<int> out, in;         // per layer (in padded to a multiple of 8)
    LayerTab tab{};
    int64_t nparam = 0, nwbf = 0;
    DBuf<float> p, m, v, g;           // flat FP32 parameters [W0 b0 W1 b1 ...], Adam moments, gradients
    DBuf<__nv_bfloat16> wbf, wtbf;    // bf16 weights and transposes
    DBuf<__nv_bfloat16> x0;           // packed input
    std::vector<DBuf<__nv_bfloat16>> y;  // hidden activations (bf16)
    std::vector<DBuf<float>> z;          // hidden pre-activations (fp32)
    std::vector<DBuf<__nv_bfloat16>> yT; // hidden activations transposed (training only)
    DBuf<float> pred;
    DBuf<__nv_bfloat16> dz[2], dzt, xt;
    DBuf<float> wsplit;               // FP32 partial products of the K-split weight-gradient GEMMs
    DBuf<int> err;
    DBuf<double> loss;
    DBuf<float> sub_x;                   // sub-chain: network inputs
    DBuf<double> sub_yp, sub_lz, sub_chi;  // proposals, log proposal ratio, chi-squared
    DBuf<double> sub_lq, sub_lqp;          // KDE log densities (current, proposed)
    DBuf<double> sub_kde;                  // KDE factors of the current call
    DBuf<double> sub_y, sub_ls, sub_comp, sub_rnd;  // fixed copies of the sub-chain's inputs (graph operands)
    DBuf<double> sub_stage;                // lcb_surrogate_subchain_host: device side of the staging
    double* sub_pinned = nullptr;          // ... and its page-locked host side
    size_t sub_pinned_n = 0;
    cudaGraphExec_t sub_graph = nullptr;   // the captured K-step sub-chain
    std::vector<unsigned char> sub_key;    // what the captured graph depends on
    int64_t steps = 0;

    const float* W(int l) const { return p.p + tab.off[l]; }
    const float* b(int l) const { return p.p + tab.off[l] + (int64_t)out[l] * in[l]; }
    float* gW(int l) { return g.p + tab.off[l]; }
    float* gb(int l) { return g.p + tab.off[l] + (int64_t)out[l] * in[l]; }

    void release() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        p.free(); m.free(); v.free(); g.free(); wbf.free(); wtbf.free(); x0.free(); pred.free(); dzt.free(); xt.free();
        wsplit.free();
        dz[0].free(); dz[1].free(); err.free(); loss.free();
        sub_x.free(); sub_yp.free(); sub_lz.free(); sub_chi.free(); sub_lq.free(); sub_lqp.free(); sub_kde.free();
        sub_y.free(); sub_ls.free(); sub_comp.free(); sub_rnd.free(); sub_stage.free();
        if (sub_pinned) cudaFreeHost(sub_pinned);
        sub_pinned = nullptr;
        sub_pinned_n = 0;
        if (sub_graph) cudaGraphExecDestroy(sub_graph);
        sub_graph = nullptr;
        for (auto& t : y) t.free();
        for (auto& t : z) t.free();
        for (auto& t : yT) t.free();
        if (own_stream && stream) cudaStreamDestroy(stream);
        stream = nullptr;
    }

    void check_err() {
        int h = 0;
        CK(cudaMemcpyAsync(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        if (h) throw Fail(LCB_ERR_DEVICE_CHECK, "a bounded wait in the surrogate GEMM timed out");
    }

    // keep_t: also store each hidden activation transposed (yT), for the weight gradients
    void forward(const float* x, int64_t B, float* y_out, bool keep_t = false) {
        if (B <= 0 || B > max_batch) throw Fail(LCB_ERR_INVALID, "batch size out of range");
        const int64_t nx = B * in[0];
        k_pack_input<<<(unsigned)((nx + 255) / 256), 256, 0, stream>>>((int)B, n_in, in[0], x, x0.p);
        CK(cudaGetLastError());
        const void* a = x0.p;
        for (int l = 0; l < nl; ++l) {
            if (l + 1 < nl) {
                gemm(EPI_BIAS_GELU, B, out[l], in[l], a, wbf.p + tab.wbf[l], b(l), nullptr, y[l].p, z[l].p, err.p, stream,
                     1, keep_t ? yT[l].p : nullptr);
                a = y[l].p;
            } else {
                gemm(EPI_BIAS_F32, B, out[l], in[l], a, wbf.p + tab.wbf[l], b(l), nullptr, y_out ? y_out : pred.p,
                     nullptr, err.p, stream);
            }
        }
    }

    void backward(const float* x, const float* target, int64_t B) {
        if (B % 8) throw Fail(LCB_ERR_INVALID, "training batch must be a multiple of 8");
        forward(x, B, nullptr, true);
        const int64_t npred = B * n_out;
        CK(cudaMemsetAsync(g.p, 0, nparam * sizeof(float), stream));
        k_mse_grad<<<(unsigned)std::min<int64_t>((npred + 255) / 256, 1184), 256, 0, stream>>>(
            npred, 1.0f / (float)npred, pred.p, target, dz[0].p, loss.p);
        CK(cudaGetLastError());
        // dzt holds the current layer's output gradient transposed: made here for the last layer, then by
        // the dGELU GEMM that produces each earlier layer's gradient
        transpose(B, n_out, dz[0].p, dzt.p, stream);
        int cur = 0;
        for (int l = nl - 1; l >= 0; --l) {
            const void* xlt = l > 0 ? (const void*)yT[l - 1].p : (const void*)xt.p;
            if (l == 0) transpose(B, in[0], x0.p, xt.p, stream);
            // dW = dz^T x: K = batch is long and the output small, so K is split across the SMs
            const int ns = split_count(out[l], in[l], B, sms);
            if (ns > 1) {
                if ((int64_t)ns * out[l] * in[l] > (int64_t)wsplit.n) throw Fail(LCB_ERR_INVALID, "weight-gradient split workspace too small");
                gemm(EPI_F32, out[l], in[l], B, dzt.p, xlt, nullptr, nullptr, wsplit.p, nullptr, err.p, stream, ns);
                sum_splits((int64_t)out[l] * in[l], ns, wsplit.p, gW(l), stream);
            } else {
                gemm(EPI_F32, out[l], in[l], B, dzt.p, xlt, nullptr, nullptr, gW(l), nullptr, err.p, stream);
            }
            // db = row sums of dz^T
            k_rowsum<<<(unsigned)out[l], 256, 0, stream>>>((int)B, dzt.p, gb(l));
            CK(cudaGetLastError());
            if (l > 0) {  // stream order: the GEMMs above have read dzt before this one rewrites it
                gemm(EPI_DGELU, B, in[l], out[l], dz[cur].p, wtbf.p + tab.wbf[l], nullptr, z[l - 1].p, dz[cur ^ 1].p,
                     nullptr, err.p, stream, 1, dzt.p);
                cur ^= 1;
            }
        }
    }

    void adam(float lr, float b1, float b2, float eps, float wd) {
        ++steps;
        const float c1 = 1.0f / (1.0f - std::pow(b1, (float)steps)), c2 = 1.0f / (1.0f - std::pow(b2, (float)steps));
        k_adam<<<(unsigned)std::min<int64_t>((nparam + 255) / 256, 2368), 256, 0, stream>>>(
            nparam, tab, p.p, m.p, v.p, g.p, wbf.p, wtbf.p, lr, b1, b2, eps, wd, c1, c2);
        CK(cudaGetLastError());
    }

    void refresh_bf16() {
        k_cast_weights<<<(unsigned)std::min<int64_t>((nparam + 255) / 256, 2368), 256, 0, stream>>>(nparam, tab, p.p,
                                                                                                   wbf.p, wtbf.p);
        CK(cudaGetLastError());
    }
};

extern "C" {

const char* lcb_mlp_last_error(void) { return t_err.c_str(); }

int lcb_mlp_create(int device, int n_in, int width, int n_hidden, int n_out, int64_t max_batch, uint64_t seed,
                   lcb_mlp** out) {
    if (!out) return LCB_ERR_INVALID;
    *out = nullptr;
    return guard([&] {
        if (n_in <= 0 || width <= 0 || width % 8 || n_hidden < 1 || n_hidden > 7 || n_out <= 0 || n_out % 8 ||
            max_batch <= 0 || max_batch > (1 << 24))
            throw Fail(LCB_ERR_INVALID, "bad network shape (width and n_out multiples of 8, 1..7 hidden layers)");
        auto N = std::make_unique<lcb_mlp>();
        N->device = device;
        CK(cudaSetDevice(device));
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, device));
        if (prop.major < 10) throw Fail(LCB_ERR_NO_DEVICE, "this library is built for sm_100a (B200)");
        N->n_in = n_in; N->width = width; N->n_hidden = n_hidden; N->n_out = n_out;
        N->sms = prop.multiProcessorCount;
        N->nl = n_hidden + 1;
        N->max_batch = (max_batch + 7) / 8 * 8;
        for (int l = 0; l < N->nl; ++l) {
            N->in.push_back(l == 0 ? (n_in + 7) / 8 * 8 : width);
            N->out.push_back(l + 1 < N->nl ? width : n_out);
        }
        LayerTab& T = N->tab;
        T.n = N->nl;
        int64_t off = 0, wo = 0;
        for (int l = 0; l < N->nl; ++l) {
            T.off[l] = off;
            T.out[l] = N->out[l];
            T.in[l] = N->in[l];
            T.wbf[l] = wo;
            off += (int64_t)N->out[l] * N->in[l] + N->out[l];
            wo += (int64_t)N->out[l] * N->in[l];
        }
        T.off[N->nl] = off;
        N->nparam = off;
        N->nwbf = wo;
        CK(cudaStreamCreateWithFlags(&N->stream, cudaStreamNonBlocking));
        N->own_stream = true;
        N->p.alloc(off); N->m.alloc(off); N->v.alloc(off); N->g.alloc(off);
        N->wbf.alloc(wo); N->wtbf.alloc(wo);
        const int64_t B = N->max_batch;
        N->x0.alloc(B * N->in[0]);
        N->y.resize(N->nl - 1);
        N->z.resize(N->nl - 1);
        N->yT.resize(N->nl - 1);
        for (int l = 0; l + 1 < N->nl; ++l) {
            N->y[l].alloc(B * width);
            N->z[l].alloc(B * width);
            N->yT[l].alloc(B * width);
        }
        const int wmax = std::max(width, n_out);
        N->pred.alloc(B * n_out);
        N->dz[0].alloc(B * wmax);
        N->dz[1].alloc(B * wmax);
        N->dzt.alloc(B * wmax);
        N->xt.alloc(B * N->in[0]);
        int64_t nsplit = 0;
        for (int l = 0; l < N->nl; ++l)
            nsplit = std::max(nsplit, (int64_t)max_split_count(N->out[l], N->in[l], N->sms) * N->out[l] * N->in[l]);
        N->wsplit.alloc(nsplit);
        N->err.alloc(1);
        N->loss.alloc(1);
        N->sub_x.alloc(B * N->in[0]);
        N->sub_yp.alloc(B * kMaxDim);
        N->sub_lz.alloc(B);
        N->sub_chi.alloc(B);
        N->sub_lq.alloc(B);
        N->sub_lqp.alloc(B);
        N->sub_kde.alloc(2 * kMaxDim * kMaxDim);
        N->sub_y.alloc(B * kMaxDim);
        N->sub_ls.alloc(B);
        N->sub_comp.alloc(B * kMaxDim);
        // He-uniform initial weights, zero biases (padding columns stay zero)
        std::vector<float> h(off, 0.f);
        std::mt19937_64 rng(seed);
        for (int l = 0; l < N->nl; ++l) {
            const int fan_in = l == 0 ? n_in : width;
            const float a = std::sqrt(6.0f / (float)fan_in);
            std::uniform_real_distribution<float> U(-a, a);
            for (int r = 0; r < N->out[l]; ++r)
                for (int c = 0; c < fan_in; ++c) h[T.off[l] + (int64_t)r * N->in[l] + c] = U(rng);
        }
        CK(cudaMemcpy(N->p.p, h.data(), off * sizeof(float), cudaMemcpyHostToDevice));
        N->refresh_bf16();
        CK(cudaStreamSynchronize(N->stream));
        *out = N.release();
    });
}

void lcb_mlp_destroy(lcb_mlp* net) {
    if (!net) return;
    net->release();
    delete net;
}

int lcb_mlp_set_stream(lcb_mlp* net, void* stream) {
    if (!net) return LCB_ERR_INVALID;
    return guard([&] {
        CK(cudaSetDevice(net->device));
        CK(cudaStreamSynchronize(net->stream));
        if (net->own_stream) CK(cudaStreamDestroy(net->stream));
        net->own_stream = stream == nullptr;
        if (stream) net->stream = (cudaStream_t)stream;
        else CK(cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking));
    });
}

int lcb_mlp_num_params(const lcb_mlp* net, int64_t* n) {
    if (!net || !n) return LCB_ERR_INVALID;
    int64_t t = 0;
    for (int l = 0; l < net->nl; ++l) t += (int64_t)net->out[l] * ((l == 0 ? net->n_in : net->width) + 1);
    *n = t;
    return LCB_OK;
}

// Copies between the unpadded host layout [W0 (out x n_in), b0, W1, b1, ...] and the device layout.
static void host_layout(const lcb_mlp* net, const float* dev_flat, float* host, bool to_host, std::vector<float>& dev) {
    int64_t h = 0;
    for (int l = 0; l < net->nl; ++l) {
        const int fan = l == 0 ? net->n_in : net->width;
        for (int r = 0; r < net->out[l]; ++r)
            for (int c = 0; c < fan; ++c, ++h) {
                float& d = dev[net->tab.off[l] + (int64_t)r * net->in[l] + c];
                if (to_host) host[h] = d;
                else d = host[h];
            }
        for (int r = 0; r < net->out[l]; ++r, ++h) {
            float& d = dev[net->tab.off[l] + (int64_t)net->out[l] * net->in[l] + r];
            if (to_host) host[h] = d;
            else d = host[h];
        }
    }
    (void)dev_flat;
}

static int fetch_flat(lcb_mlp* net, const float* src, float* host, int64_t n) {
    return guard([&] {
        int64_t want = 0;
        lcb_mlp_num_params(net, &want);
        if (n != want) throw Fail(LCB_ERR_INVALID, "parameter count mismatch");
        CK(cudaSetDevice(net->device));
        net->check_err();
        std::vector<float> dev(net->nparam);
        CK(cudaMemcpyAsync(dev.data(), src, net->nparam * sizeof(float), cudaMemcpyDeviceToHost, net->stream));
        CK(cudaStreamSynchronize(net->stream));
        host_layout(net, src, host, true, dev);
    });
}

int lcb_mlp_get_params(lcb_mlp* net, float* host, int64_t n) {
    if (!net || !host) return LCB_ERR_INVALID;
    return fetch_flat(net, net->p.p, host, n);
}

// Training state for checkpoints: the FP32 master parameters and both Adam
// moments in the device layout (3 x state_size floats) and the step count.
int lcb_mlp_state_size(const lcb_mlp* net, int64_t* n) {
    if (!net || !n) return LCB_ERR_INVALID;
    *n = net->nparam;
    return LCB_OK;
}

int lcb_mlp_get_state(lcb_mlp* net, float* host, int64_t n, int64_t* steps) {
    if (!net || !host || !steps) return LCB_ERR_INVALID;
    return guard([&] {
        if (n != 3 * net->nparam) throw Fail(LCB_ERR_INVALID, "state size mismatch");
        CK(cudaSetDevice(net->device));
        net->check_err();
        const size_t b = net->nparam * sizeof(float);
        CK(cudaMemcpyAsync(host, net->p.p, b, cudaMemcpyDeviceToHost, net->stream));
        CK(cudaMemcpyAsync(host + net->nparam, net->m.p, b, cudaMemcpyDeviceToHost, net->stream));
        CK(cudaMemcpyAsync(host + 2 * net->nparam, net->v.p, b, cudaMemcpyDeviceToHost, net->stream));
        CK(cudaStreamSynchronize(net->stream));
        *steps = net->steps;
    });
}

int lcb_mlp_set_state(lcb_mlp* net, const float* host, int64_t n, int64_t steps) {
    if (!net || !host || steps < 0) return LCB_ERR_INVALID;
    return guard([&] {
        if (n != 3 * net->nparam) throw Fail(LCB_ERR_INVALID, "state size mismatch");
        CK(cudaSetDevice(net->device));
        const size_t b = net->nparam * sizeof(float);
        CK(cudaMemcpyAsync(net->p.p, host, b, cudaMemcpyHostToDevice, net->stream));
        CK(cudaMemcpyAsync(net->m.p, host + net->nparam, b, cudaMemcpyHostToDevice, net->stream));
        CK(cudaMemcpyAsync(net->v.p, host + 2 * net->nparam, b, cudaMemcpyHostToDevice, net->stream));
        net->steps = steps;
        net->refresh_bf16();
        CK(cudaStreamSynchronize(net->stream));
    });
}

int lcb_mlp_get_grads(lcb_mlp* net, float* host, int64_t n) {
    if (!net || !host) return LCB_ERR_INVALID;
    return fetch_flat(net, net->g.p, host, n);
}

int lcb_mlp_set_params(lcb_mlp* net, const float* host, int64_t n) {
    if (!net || !host) return LCB_ERR_INVALID;
    return guard([&] {
        int64_t want = 0;
        lcb_mlp_num_params(net, &want);
        if (n != want) throw Fail(LCB_ERR_INVALID, "parameter count mismatch");
        CK(cudaSetDevice(net->device));
        std::vector<float> dev(net->nparam, 0.f);
        host_layout(net, nullptr, const_cast<float*>(host), false, dev);
        CK(cudaMemcpyAsync(net->p.p, dev.data(), net->nparam * sizeof(float), cudaMemcpyHostToDevice, net->stream));
        CK(cudaMemsetAsync(net->m.p, 0, net->nparam * sizeof(float), net->stream));
        CK(cudaMemsetAsync(net->v.p, 0, net->nparam * sizeof(float), net->stream));
        net->steps = 0;
        net->refresh_bf16();
        CK(cudaStreamSynchronize(net->stream));
    });
}

int lcb_mlp_forward(lcb_mlp* net, const float* x_dev, int64_t batch, float* y_dev) {
    if (!net || !x_dev || !y_dev) return LCB_ERR_INVALID;
    return guard([&] {
        CK(cudaSetDevice(net->device));
        net->forward(x_dev, batch, y_dev);
    });
}

int lcb_mlp_backward(lcb_mlp* net, const float* x_dev, const float* target_dev, int64_t batch) {
    if (!net || !x_dev || !target_dev) return LCB_ERR_INVALID;
    return guard([&] {
        CK(cudaSetDevice(net->device));
        net->backward(x_dev, target_dev, batch);
    });
}

int lcb_mlp_train_step(lcb_mlp* net, const float* x_dev, const float* target_dev, int64_t batch, float lr,
                       float beta1, float beta2, float eps, float weight_decay) {
    if (!net || !x_dev || !target_dev) return LCB_ERR_INVALID;
    return guard([&] {
        CK(cudaSetDevice(net->device));
        net->backward(x_dev, target_dev, batch);
        net->adam(lr, beta1, beta2, eps, weight_decay);
    });
}

int lcb_mlp_grads_device(lcb_mlp* net, float** grads_dev, int64_t* n) {
    if (!net || !grads_dev || !n) return LCB_ERR_INVALID;
    *grads_dev = net->g.p;
    *n = net->nparam;
    return LCB_OK;
}

int lcb_mlp_adam_step(lcb_mlp* net, float lr, float beta1, float beta2, float eps, float weight_decay) {
    if (!net) return LCB_ERR_INVALID;
    return guard([&] {
        CK(cudaSetDevice(net->device));
        net->adam(lr, beta1, beta2, eps, weight_decay);
    });
}

int lcb_mlp_take_loss(lcb_mlp* net, double* loss_sum) {
    if (!net || !loss_sum) return LCB_ERR_INVALID;
    return guard([&] {
        CK(cudaSetDevice(net->device));
        net->check_err();
        CK(cudaMemcpyAsync(loss_sum, net->loss.p, sizeof(double), cudaMemcpyDeviceToHost, net->stream));
        CK(cudaMemsetAsync(net->loss.p, 0, sizeof(double), net->stream));
        CK(cudaStreamSynchronize(net->stream));
    });
}

int lcb_mlp_sync(lcb_mlp* net) {
    if (!net) return LCB_ERR_INVALID;
    return guard([&] {
        CK(cudaSetDevice(net->device));
        net->check_err();
    });
}

int lcb_mlp_gemm(int mode, int64_t M, int64_t N, int64_t K, const void* a, const void* b, const float* bias,
                 const float* aux, void* out, void* out2, int* err_dev, void* stream) {
    return guard([&] { gemm(mode, M, N, K, a, b, bias, aux, out, out2, err_dev, (cudaStream_t)stream); });
}

int lcb_surrogate_subchain(lcb_mlp* net, int64_t n, int64_t m, int d, double* y_dev, double* ls_dev,
                           const double* comp_dev, const double* rnd_dev, int steps, double a, const double* lo,
                           const double* hi, const int* recip, const float* fmul, const float* fadd,
                           const float* mean_dev, const float* sd_dev, const double* flux_dev, const double* ferr_dev,
                           int scale, int move, const double* kde_chol, const double* kde_prec) {
    if (!net || !y_dev || !ls_dev || !comp_dev || !rnd_dev || !lo || !hi || !recip || !fmul || !fadd || !mean_dev ||
        !sd_dev || !flux_dev || !ferr_dev || (move == MOVE_KDE && (!kde_chol || !kde_prec)))
        return LCB_ERR_INVALID;
    return guard([&] {
        if (n <= 0 || n > net->max_batch || m <= 0 || m > INT32_MAX || d != net->n_in || d > kMaxDim || steps < 0 ||
            !(a > 1.0))
            throw Fail(LCB_ERR_INVALID, "sub-chain: 0 < n <= max_batch, d == n_in <= 8, a > 1 required");
        if (move != MOVE_STRETCH && move != MOVE_KDE) throw Fail(LCB_ERR_INVALID, "sub-chain: unknown move");
        if (m > net->max_batch) throw Fail(LCB_ERR_INVALID, "sub-chain: at most max_batch complementary walkers");
        CK(cudaSetDevice(net->device));
        if (steps == 0) return;
        cudaStream_t st = net->stream;
        const int rstride = move == MOVE_KDE ? 3 + d : 3;
        const size_t nrnd = (size_t)steps * n * rstride;
        if (net->sub_rnd.n < nrnd) {  // grow the random-number buffer (outside any capture)
            CK(cudaStreamSynchronize(st));
            net->sub_rnd.free();
            net->sub_rnd.alloc(nrnd);
            if (net->sub_graph) cudaGraphExecDestroy(net->sub_graph);
            net->sub_graph = nullptr;
        }
        StretchArgs A{};
        A.n = (int)n; A.m = (int)m; A.d = d; A.n_in = net->n_in;  // rows of lcb_mlp_forward input: n_in wide
        A.y = net->sub_y.p; A.ls = net->sub_ls.p; A.comp = net->sub_comp.p; A.rnd = net->sub_rnd.p;
        A.yp = net->sub_yp.p; A.lz = net->sub_lz.p; A.xin = net->sub_x.p;
        A.lq = net->sub_lq.p; A.lqp = net->sub_lqp.p;
        A.move = move; A.rstride = rstride;
        double kde[2 * kMaxDim * kMaxDim] = {};
        for (int k = 0; k < d; ++k) {
            A.lo[k] = lo[k]; A.hi[k] = hi[k]; A.frecip[k] = recip[k]; A.fmul[k] = fmul[k]; A.fadd[k] = fadd[k];
            if (move == MOVE_KDE)
                for (int l = 0; l < d; ++l) {
                    kde[k * kMaxDim + l] = l <= k ? kde_chol[k * d + l] : 0.0;
                    kde[kMaxDim * kMaxDim + k * kMaxDim + l] = kde_prec[k * d + l];
                }
        }
        A.kde = net->sub_kde.p;
        A.a = a;
        // the graph is valid while everything it was captured with is unchanged
        std::vector<unsigned char> key(sizeof(A) + 6 * sizeof(int64_t) + 4 * sizeof(void*));
        {
            unsigned char* q = key.data();
            auto put = [&](const void* v, size_t b) { std::memcpy(q, v, b); q += b; };
            put(&A, sizeof(A));
            const int64_t ints[6] = {n, m, d, steps, scale, (int64_t)net->sub_rnd.n};
            put(ints, sizeof(ints));
            const void* ptrs[4] = {mean_dev, sd_dev, flux_dev, ferr_dev};
            put(ptrs, sizeof(ptrs));
        }
        CK(cudaMemcpyAsync(net->sub_y.p, y_dev, n * d * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(net->sub_ls.p, ls_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(net->sub_comp.p, comp_dev, m * d * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(net->sub_rnd.p, rnd_dev, nrnd * sizeof(double), cudaMemcpyDeviceToDevice, st));
        if (move == MOVE_KDE) {  // pageable source: the copy is staged before this call returns
            CK(cudaMemcpyAsync(net->sub_kde.p, kde, sizeof(kde), cudaMemcpyHostToDevice, st));
        }
        auto enqueue = [&] {
            const unsigned g = (unsigned)((n + 127) / 128);
            const unsigned gw = (unsigned)((n + kWalkersPerBlock - 1) / kWalkersPerBlock);  // a warp per walker
            if (move == MOVE_KDE) {
                k_kde_logq<<<gw, 32 * kWalkersPerBlock, 0, st>>>(A);
                CK(cudaGetLastError());
            }
            for (int k = 0; k < steps; ++k) {
                if (move == MOVE_KDE) k_kde_propose<<<gw, 32 * kWalkersPerBlock, 0, st>>>(A, k);
                else k_stretch_propose<<<g, 128, 0, st>>>(A, k);
                CK(cudaGetLastError());
                net->forward(net->sub_x.p, n, nullptr);
                k_logflux_chisq<<<(unsigned)n, 128, 0, st>>>((int)n, net->n_out, net->pred.p, mean_dev, sd_dev,
                                                            flux_dev, ferr_dev, scale, net->sub_chi.p);
                CK(cudaGetLastError());
                k_stretch_accept<<<g, 128, 0, st>>>(A, net->sub_chi.p, k);
                CK(cudaGetLastError());
            }
        };
        if (!net->sub_graph || net->sub_key != key) {
            if (net->sub_graph) cudaGraphExecDestroy(net->sub_graph);
            net->sub_graph = nullptr;
            net->sub_key.clear();
            prepare_gemm_attributes();  // function attributes are set outside the capture
            cudaGraph_t graph;
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue();
            } catch (...) {
                if (cudaStreamEndCapture(st, &graph) == cudaSuccess && graph) cudaGraphDestroy(graph);
                throw;
            }
            CK(cudaStreamEndCapture(st, &graph));
            cudaError_t e = cudaGraphInstantiate(&net->sub_graph, graph, 0);
            cudaGraphDestroy(graph);
            CK(e);
            net->sub_key = key;
        }
        CK(cudaGraphLaunch(net->sub_graph, st));
        CK(cudaMemcpyAsync(y_dev, net->sub_y.p, n * d * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(ls_dev, net->sub_ls.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    });
}

int lcb_surrogate_subchain_host(lcb_mlp* net, int64_t n, int64_t m, int d, double* y, double* ls, const double* comp,
                                const double* rnd, int steps, double a, const double* lo, const double* hi,
                                const int* recip, const float* fmul, const float* fadd, const float* mean_dev,
                                const float* sd_dev, const double* flux_dev, const double* ferr_dev, int scale, int move,
                                const double* kde_chol, const double* kde_prec) {
    if (!net || !y || !ls || !comp || !rnd) return LCB_ERR_INVALID;
    if (n <= 0 || m <= 0 || d <= 0 || steps < 0 || n > net->max_batch || m > net->max_batch || d > kMaxDim)
        return LCB_ERR_INVALID;
    const int rstride = move == MOVE_KDE ? 3 + d : 3;
    const size_t ny = (size_t)n * d, nc = (size_t)m * d, nr = (size_t)steps * n * rstride;
    const size_t total = ny + n + nc + nr;  // [y | ls | comp | rnd], doubles
    int rc = guard([&] {
        CK(cudaSetDevice(net->device));
        if (net->sub_pinned_n < total) {  // grow both sides of the staging (outside any capture)
            const size_t want = std::max<size_t>(total, 2 * net->sub_pinned_n);
            CK(cudaStreamSynchronize(net->stream));
            if (net->sub_pinned) CK(cudaFreeHost(net->sub_pinned));
            net->sub_pinned = nullptr;
            net->sub_pinned_n = 0;
            net->sub_stage.free();
            CK(cudaMallocHost((void**)&net->sub_pinned, want * sizeof(double)));
            net->sub_pinned_n = want;
            net->sub_stage.alloc(want);
        }
        double* h = net->sub_pinned;
        std::memcpy(h, y, ny * sizeof(double));
        std::memcpy(h + ny, ls, n * sizeof(double));
        std::memcpy(h + ny + n, comp, nc * sizeof(double));
        std::memcpy(h + ny + n + nc, rnd, nr * sizeof(double));
        CK(cudaMemcpyAsync(net->sub_stage.p, h, total * sizeof(double), cudaMemcpyHostToDevice, net->stream));
    });
    if (rc != LCB_OK) return rc;
    double* dv = net->sub_stage.p;
    rc = lcb_surrogate_subchain(net, n, m, d, dv, dv + ny, dv + ny + n, dv + ny + n + nc, steps, a, lo, hi, recip,
                                fmul, fadd, mean_dev, sd_dev, flux_dev, ferr_dev, scale, move, kde_chol, kde_prec);
    if (rc != LCB_OK) {
        cudaStreamSynchronize(net->stream);  // the staging is reused by the next call
        return rc;
    }
    return guard([&] {
        double* h = net->sub_pinned;
        CK(cudaMemcpyAsync(h, dv, (ny + n) * sizeof(double), cudaMemcpyDeviceToHost, net->stream));
        CK(cudaStreamSynchronize(net->stream));
        std::memcpy(y, h, ny * sizeof(double));
        std::memcpy(ls, h + ny, n * sizeof(double));
    });
}

int lcb_logflux_chisq(int64_t rows, int n, const float* pred, const float* mean, const float* sd, const double* flux,
                      const double* ferr, int scale, double* chisq_out, void* stream) {
    if (rows <= 0 || n <= 0 || !pred || !mean || !sd || !flux || !ferr || !chisq_out) return LCB_ERR_INVALID;
    return guard([&] {
        k_logflux_chisq<<<(unsigned)rows, 128, 0, (cudaStream_t)stream>>>((int)rows, n, pred, mean, sd, flux, ferr,
                                                                          scale, chisq_out);
        CK(cudaGetLastError());
    });
}

}  // extern "C"
