// dtt_tc.cu — split-precision half-integer transforms on the tcgen05 tensor
// cores (sm_100a).
//
// Replaces the reference's FFTW REDFT11/RODFT11 plans
// (movefieldshydrolinlayersplit.cpp:389-427) and scales up its dense-matrix
// GPU attempt (surfaceFFT.cu:108-164, matrix table fft_matrix.cu:10-24):
// a 2-D transform is two passes of out_f = (in_f . A)^T with A the
// symmetric 2cos/2sin((j+1/2)(k+1/2)pi/n) matrix.
//
// Precision: FP32 data and FP64-built matrices are split into 2 or 3
// low-precision terms (BF16 or TF32), the products of the leading terms are
// accumulated in FP32 in TMEM:
//   BF16X3: a0b0 + a0b1 + a1b0      (~2^-16 relative)
//   TF32X3: a0b0 + a0b1 + a1b0      (~2^-22 relative, TF32 MMAs)
//   BF16X6: a0b0+a0b1+a1b0+a0b2+a1b1+a2b0   (~2^-24 relative)
//
// Kernel: one CTA of 4 warps per 128 x 64 output tile of one field.
//   warp 0 lane 0 : TMA producer (cp.async.bulk.tensor, 128B swizzle, no
//                   multicast) into a STAGES-deep smem ring
//   warp 1 lane 0 : issues tcgen05.mma (kind::f16 or kind::tf32) for every
//                   term pair, commits each stage back to the producer
//   warp 2        : allocates / frees the 64 TMEM columns of the accumulator
//   all 4 warps   : epilogue, tcgen05.ld 32x32b, transposed store: either
//                   FP32 (scaled) to the destination plane or the split
//                   terms of the next pass's operand.
// Every mbarrier wait is bounded; on a timeout the kernel raises
// DEV_ERR_TIMEOUT, drains its own TMA copies (bounded), frees TMEM, returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cmath>
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "dtt_tc.h"
#include "qs_common.cuh"
#include "split.cuh"
#include "pdl.cuh"

namespace qs {
namespace tcx {

constexpr int BM = 128;   // output rows per tile (matrix rows, MMA M)

constexpr uint32_t SPIN_LIMIT = 1u << 22;

struct Params {
    int R, K;              // data rows per field (output columns), transform size
    int data_rows;         // rows of one split term in the data map (nfmax * R)
    int mat_rows;          // rows of one split term in the matrix map (2 * K)
    int nfmax;             // field capacity of the split operand buffers
    unsigned long long kindmask;  // bit f: matrix kind (REDFT11 / RODFT11) of field f
    int promo;             // k-blocks accumulated in TMEM before an FP32 drain
    int out_split;         // 1: write split terms to out_base [term][nfmax][K][R]
    int out_contig;        // 1: field f writes to out[0] + f * R * K
    void* out_base;
    float* out[kMaxXfFields];
    float scale;
    int* err;
};

// ------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait: false on timeout or when another role aborted
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                          uint32_t limit = SPIN_LIMIT) {
    for (uint32_t i = 0; i < limit; i++) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 255u) == 255u && *abort_flag) return false;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(bar)
        : "memory");
}

__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    // tcgen05 shared-memory descriptor: K-major tile of 128 B rows,
    // 128B swizzle, 8-row atoms 1024 B apart (stride byte offset), version 1.
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFFu) >> 4);           // start address
    d |= (uint64_t)1 << 16;                            // leading byte offset (unused)
    d |= (uint64_t)(1024u >> 4) << 32;                 // stride byte offset
    d |= (uint64_t)1 << 46;                            // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                            // SWIZZLE_128B
    return d;
}

template <int KIND>
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                    uint32_t accum) {
    if (KIND == 0) {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accum));
    } else {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accum));
    }
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}

__device__ __forceinline__ void fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}


// ------------------------------------------------------------ the GEMM
// Product terms (matrix split index, data split index), small terms first.
template <int NSPLIT>
struct Terms;
template <>
struct Terms<2> {
    static constexpr int N = 3;
    __device__ static constexpr int a(int t) { return t == 0 ? 0 : (t == 1 ? 1 : 0); }
    __device__ static constexpr int b(int t) { return t == 0 ? 1 : 0; }
};
template <>
struct Terms<3> {
    static constexpr int N = 6;
    // (0,2) (1,1) (2,0) (0,1) (1,0) (0,0)
    __device__ static constexpr int a(int t) {
        return t == 0 ? 0 : t == 1 ? 1 : t == 2 ? 2 : t == 3 ? 0 : t == 4 ? 1 : 0;
    }
    __device__ static constexpr int b(int t) {
        return t == 0 ? 2 : t == 1 ? 1 : t == 2 ? 0 : t == 3 ? 1 : t == 4 ? 0 : 0;
    }
};

// Tile: 128 output rows n (rows of the symmetric matrix, the MMA's M side)
// x 64 output columns m (rows of one field's data, the MMA's N side):
//   D[n][m] = sum_k mat[n][k] * data_f[m][k] = (data_f . mat)^T [n][m]
// so TMEM lane = output row and every epilogue thread owns 64 contiguous
// outputs.  Warps: 0 = TMA producer, 1 = MMA issuer, 2..5 = epilogue (TMEM
// lane quarter = warp % 4).  The accumulator is double buffered in TMEM and
// drained every `promo` k-blocks into FP32 registers (partial sums of at most
// promo*BK products live in the tensor-core accumulator).
constexpr int EPI_WARPS = 8;   // two per TMEM lane quarter, 64 columns each
constexpr int THREADS_V2 = 32 * (2 + EPI_WARPS);

template <int KIND, int NSPLIT, int STAGES, int BN>
__global__ void __launch_bounds__(THREADS_V2, 1)
    dtt_tc_kernel(const __grid_constant__ CUtensorMap mapM,
                  const __grid_constant__ CUtensorMap mapD, const Params p) {
    constexpr int ELEM = (KIND == 0) ? 2 : 4;
    constexpr int BK = 128 / ELEM;                  // one 128-byte swizzle row
    constexpr uint32_t M_TILE = BM * 128;           // matrix tile, 16 KB
    constexpr uint32_t D_TILE = BN * 128;           // data tile, 8 KB
    constexpr uint32_t STAGE = NSPLIT * (M_TILE + D_TILE);
    constexpr int NT = Terms<NSPLIT>::N;
    constexpr uint32_t TCOLS = 2 * BN;              // two accumulator buffers

    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], accf[2], acce[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int f = blockIdx.z;
    const int n0 = blockIdx.x * BM, m0 = blockIdx.y * BN;
    const int nkb = p.K / BK;
    const int promo = p.promo;
    const int nchunks = nkb / promo;
    const int kind = (int)((p.kindmask >> f) & 1ull);

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(smem_u32(&full_bar[s]), 1);
            mbar_init(smem_u32(&empty_bar[s]), 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(smem_u32(&accf[b]), 1);
            mbar_init(smem_u32(&acce[b]), EPI_WARPS);
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;
    volatile int* abortp = &abort_flag;
    qs::pdl_wait();   // operands and outputs are the previous kernel's

    if (warp == 0) {
        if (lane != 0) qs::pdl_trigger();
        if (lane == 0) {
            // ---------------- TMA producer
            asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&mapM) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&mapD) : "memory");
            const int rowM = kind * p.K + n0;
            const int rowD = f * p.R + m0;
            int issued = 0;
            for (int kb = 0; kb < nkb; kb++) {
                const int s = kb % STAGES;
                const uint32_t use = kb / STAGES;
                if (kb >= STAGES &&
                    !mbar_wait(smem_u32(&empty_bar[s]), (use - 1) & 1, abortp)) {
                    *abortp = 1;
                    break;
                }
                const uint32_t fb = smem_u32(&full_bar[s]);
                mbar_expect_tx(fb, STAGE);
                uint8_t* st = smem + (size_t)s * STAGE;
#pragma unroll
                for (int t = 0; t < NSPLIT; t++)
                    tma_load_2d(smem_u32(st + t * M_TILE), &mapM, fb, kb * BK,
                                t * p.mat_rows + rowM);
#pragma unroll
                for (int t = 0; t < NSPLIT; t++)
                    tma_load_2d(smem_u32(st + NSPLIT * M_TILE + t * D_TILE), &mapD, fb, kb * BK,
                                t * p.data_rows + rowD);
                issued = kb + 1;
            }
            qs::pdl_trigger();
            if (*abortp) {
                for (int kb = (issued > STAGES ? issued - STAGES : 0); kb < issued; kb++)
                    mbar_wait(smem_u32(&full_bar[kb % STAGES]), (kb / STAGES) & 1, abortp);
            }
        }
    } else if (warp == 1) {
        if (lane != 0) qs::pdl_trigger();
        if (lane == 0) {
            // ---------------- MMA issuer
            const uint32_t idesc = (1u << 4) | ((KIND == 0 ? 1u : 2u) << 7) |
                                   ((KIND == 0 ? 1u : 2u) << 10) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)(BM >> 4) << 24);
            bool ok = true;
            int kb = 0;
            for (int c = 0; c < nchunks && ok; c++) {
                const int b = c & 1;
                if (c >= 2 && !mbar_wait(smem_u32(&acce[b]), ((c >> 1) - 1) & 1, abortp)) {
                    *abortp = 1;
                    ok = false;
                    break;
                }
                fence_after();
                const uint32_t dt = tmem + (uint32_t)(b * BN);
                for (int q = 0; q < promo; q++, kb++) {
                    const int s = kb % STAGES;
                    if (!mbar_wait(smem_u32(&full_bar[s]), (kb / STAGES) & 1, abortp)) {
                        *abortp = 1;
                        ok = false;
                        break;
                    }
                    fence_after();
                    const uint32_t st = smem_u32(smem + (size_t)s * STAGE);
                    const uint64_t dM = sw128_desc(st);
                    const uint64_t dD = sw128_desc(st + NSPLIT * M_TILE);
#pragma unroll
                    for (int t = 0; t < NT; t++) {
#pragma unroll
                        for (int kk = 0; kk < 4; kk++) {
                            // advance the start address (16-byte units) inside the row
                            const uint64_t a = dM + (uint64_t)((Terms<NSPLIT>::a(t) * M_TILE +
                                                                kk * 32) >> 4);
                            const uint64_t bb = dD + (uint64_t)((Terms<NSPLIT>::b(t) * D_TILE +
                                                                 kk * 32) >> 4);
                            mma<KIND>(dt, a, bb, idesc, (q | t | kk) != 0);
                        }
                    }
                    mma_commit(smem_u32(&empty_bar[s]));
                }
                if (ok) mma_commit(smem_u32(&accf[b]));
            }
            qs::pdl_trigger();
        }
    } else {
        // ---------------- epilogue: drain every chunk into FP32 registers
        const int e = warp - 2;                        // epilogue warp 0..7
        const int qtr = warp & 3;                      // TMEM lane quarter
        const int half = e >> 2;                       // column half of the tile
        const int rloc = qtr * 32 + lane;              // tile row owned by this thread
        constexpr int HC = BN / 2;                     // columns per epilogue warp
        float acc[HC];
#pragma unroll
        for (int i = 0; i < HC; i++) acc[i] = 0.f;
        bool have = true;
        for (int c = 0; c < nchunks; c++) {
            const int b = c & 1;
            if (!mbar_wait(smem_u32(&accf[b]), (c >> 1) & 1, abortp)) {
                have = false;
                *abortp = 1;
                break;
            }
            fence_after();
#pragma unroll
            for (int j = 0; j < HC; j += 16) {
                uint32_t v[16];
                tmem_ld16(tmem + ((uint32_t)(qtr * 32) << 16) + (uint32_t)(b * BN + half * HC + j),
                          v);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; i++) acc[j + i] += __uint_as_float(v[i]);
            }
            fence_before();
            __syncwarp();
            if (lane == 0) {
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acce[b]))
                             : "memory");
            }
        }
        qs::pdl_trigger();
        // every MMA has completed (the last chunk was committed after them),
        // so the pipeline smem is free: stage the tile there row-major
        constexpr int LD = BN + 4;
        float* tile = (float*)smem;
        if (have) {
            const float sc = p.scale;
            float4* trow = (float4*)(tile + (size_t)rloc * LD + half * HC);
#pragma unroll
            for (int i = 0; i < HC / 4; i++)
                trow[i] = make_float4(acc[4 * i] * sc, acc[4 * i + 1] * sc, acc[4 * i + 2] * sc,
                                      acc[4 * i + 3] * sc);
        }
        asm volatile("bar.sync 1, %0;" ::"r"(32 * EPI_WARPS) : "memory");
        if (have && !*abortp) {
            // each warp writes whole rows; a row is BN values, 4 per lane
            float* o = nullptr;
            if (p.out_contig) {
                o = p.out[0] + (size_t)f * p.R * p.K;
            } else {
#pragma unroll
                for (int i = 0; i < kMaxXfFields; i++)
                    if (i == f) o = p.out[i];
            }
            const size_t plane = (size_t)p.R * p.K;
            const size_t tstride = (size_t)p.nfmax * plane;
            constexpr int LPR = BN / 4;                // lanes per row
            constexpr int RPI = 32 / LPR;              // rows per warp instruction
            const int sub = lane / LPR, lc = lane % LPR;
            for (int rr = 0; rr < BM / EPI_WARPS; rr += RPI) {
                const int r = e * (BM / EPI_WARPS) + rr + sub;
                const float4 v = *(const float4*)(tile + (size_t)r * LD + lc * 4);
                const size_t g = (size_t)(n0 + r) * p.R + m0 + lc * 4;
                if (!p.out_split) {
                    *(float4*)(o + g) = v;
                } else {
                    const float vv[4] = {v.x, v.y, v.z, v.w};
                    float t[4][3];
#pragma unroll
                    for (int q = 0; q < 4; q++) split_value<KIND>(vv[q], NSPLIT, t[q]);
                    const size_t idx = (size_t)f * plane + g;
                    if (KIND == 0) {
                        __nv_bfloat16* ob = (__nv_bfloat16*)p.out_base;
#pragma unroll
                        for (int s = 0; s < NSPLIT; s++) {
                            __nv_bfloat162 h0 = __floats2bfloat162_rn(t[0][s], t[1][s]);
                            __nv_bfloat162 h1 = __floats2bfloat162_rn(t[2][s], t[3][s]);
                            *(uint2*)(ob + (size_t)s * tstride + idx) =
                                make_uint2(*(uint32_t*)&h0, *(uint32_t*)&h1);
                        }
                    } else {
                        float* of = (float*)p.out_base;
#pragma unroll
                        for (int s = 0; s < NSPLIT; s++)
                            *(float4*)(of + (size_t)s * tstride + idx) =
                                make_float4(t[0][s], t[1][s], t[2][s], t[3][s]);
                    }
                }
            }
        } else if (lane == 0 && e == 0) {
            atomicOr(p.err, DEV_ERR_TIMEOUT);
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 2) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TCOLS)
                     : "memory");
    }
}

// split nf FP32 planes stored from `in` with stride `stride` into the
// operand terms [term][8][plane]; 4 values per thread
template <int KIND, int NSPLIT>
__global__ void split_planes_kernel(const float* __restrict__ in, size_t stride, int nf,
                                    size_t plane, size_t tstride, void* __restrict__ out) {
    const size_t i4 = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
    const int f = blockIdx.y;
    if (i4 >= plane || f >= nf) return;
    qs::pdl_wait();
    const float4 v = *(const float4*)(in + (size_t)f * stride + i4);
    qs::pdl_trigger();
    const float vv[4] = {v.x, v.y, v.z, v.w};
    float t[4][3];
#pragma unroll
    for (int e = 0; e < 4; e++) split_value<KIND>(vv[e], NSPLIT, t[e]);
    const size_t idx = (size_t)f * plane + i4;
    if (KIND == 0) {
        __nv_bfloat16* o = (__nv_bfloat16*)out;
#pragma unroll
        for (int s = 0; s < NSPLIT; s++) {
            __nv_bfloat162 a = __floats2bfloat162_rn(t[0][s], t[1][s]);
            __nv_bfloat162 b = __floats2bfloat162_rn(t[2][s], t[3][s]);
            *(uint2*)(o + (size_t)s * tstride + idx) =
                make_uint2(*(uint32_t*)&a, *(uint32_t*)&b);
        }
    } else {
        float* o = (float*)out;
#pragma unroll
        for (int s = 0; s < NSPLIT; s++)
            *(float4*)(o + (size_t)s * tstride + idx) =
                make_float4(t[0][s], t[1][s], t[2][s], t[3][s]);
    }
}

// A self-test of the bounded waits: one thread initialises an mbarrier that
// nothing arrives at and waits on it through mbar_wait with `limit` tries;
// the wait gives up and the kernel sets DEV_ERR_TIMEOUT, as the roles of the
// transform kernel do.  No copy, TMEM or other CTA is involved, so the
// kernel ends after at most `limit` tries.
__global__ void wait_limit_probe_kernel(int* err, uint32_t limit) {
    __shared__ __align__(8) uint64_t bar;
    __shared__ int abort_flag;
    if (threadIdx.x == 0) {
        abort_flag = 0;
        mbar_init(smem_u32(&bar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0 && !mbar_wait(smem_u32(&bar), 0, &abort_flag, limit))
        atomicOr(err, DEV_ERR_TIMEOUT);
}

}  // namespace tcx

int launch_wait_limit_probe(int* err, unsigned limit, cudaStream_t st) {
    tcx::wait_limit_probe_kernel<<<1, 32, 0, st>>>(err, limit);
    return 1;
}

// ---------------------------------------------------------------- host side
namespace {

PFN_cuTensorMapEncodeTiled_v12000 get_encoder(std::string& why) {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (fn) return fn;
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !ptr) {
        why = "cuTensorMapEncodeTiled entry point unavailable";
        return nullptr;
    }
    fn = (PFN_cuTensorMapEncodeTiled_v12000)ptr;
    return fn;
}

bool encode_2d(CUtensorMap* map, void* base, bool bf16, uint64_t cols, uint64_t rows,
               uint32_t box_cols, uint32_t box_rows, std::string& why) {
    auto enc = get_encoder(why);
    if (!enc) return false;
    const int elem = bf16 ? 2 : 4;
    cuuint64_t dims[2] = {cols, rows};
    cuuint64_t strides[1] = {cols * elem};
    cuuint32_t box[2] = {box_cols, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                     2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        why = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
        return false;
    }
    return true;
}

// round a double to the split representation on the host
float round_term(double x, bool bf16) {
    float f = (float)x;
    if (bf16) return __bfloat162float(__float2bfloat16_rn(f));
    uint32_t u;
    memcpy(&u, &f, 4);
    // round to nearest, ties away, at 10 mantissa bits (cvt.rna.tf32.f32)
    u = (u + 0x1000u) & 0xFFFFE000u;
    memcpy(&f, &u, 4);
    return f;
}

class TcImpl : public TcTransformer {
public:
    int mode = 0, ny = 0, nz = 0, kind = 0, nsplit = 2;
    int nfmax = 64;
    void* splitA = nullptr;
    void* splitB = nullptr;
    void* matY = nullptr;
    void* matZ = nullptr;
    int* err = nullptr;
    // tensor maps: data (N side) for tile widths 64 / 128, matrix (M side)
    CUtensorMap mapD1[2], mapM1, mapD2[2], mapM2;
    size_t smem_bytes[2] = {0, 0};
    int chunk_k = 128;

    ~TcImpl() override {
        for (void* p : {splitA, splitB, matY, matZ})
            if (p) cudaFree(p);
    }

    // pipeline depth of each kernel instantiation (must match launch_gemm)
    int stages_for(int bnidx) const {
        if (nsplit == 3) return bnidx ? 2 : 3;
        return bnidx ? 3 : 4;
    }

    bool upload_matrix(int n, void** dst, std::string& why) {
        const bool bf16 = (kind == 0);
        const int elem = bf16 ? 2 : 4;
        const size_t nn = (size_t)n * n;
        std::vector<uint8_t> host((size_t)nsplit * 2 * nn * elem);
        for (int kd = 0; kd < 2; kd++)
            for (size_t r = 0; r < (size_t)n; r++)
                for (size_t c = 0; c < (size_t)n; c++) {
                    long long q = ((long long)(2 * c + 1) * (2 * r + 1)) % (8LL * n);
                    double a = M_PI * (double)q / (4.0 * n);
                    double v = 2.0 * (kd == 0 ? std::cos(a) : std::sin(a));
                    double rem = v;
                    for (int sp = 0; sp < nsplit; sp++) {
                        float t = round_term(rem, bf16);
                        rem -= (double)t;
                        size_t idx = (size_t)sp * 2 * nn + (size_t)kd * nn + r * n + c;
                        if (bf16) {
                            __nv_bfloat16 b = __float2bfloat16_rn(t);
                            memcpy(host.data() + idx * 2, &b, 2);
                        } else {
                            memcpy(host.data() + idx * 4, &t, 4);
                        }
                    }
                }
        if (cudaMalloc(dst, host.size()) != cudaSuccess) {
            why = "cudaMalloc of split matrices failed";
            return false;
        }
        if (cudaMemcpy(*dst, host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
            why = "upload of split matrices failed";
            return false;
        }
        return true;
    }

    bool init(std::string& why) {
        if (ny % 128 || nz % 128) {
            why = "ny and nz must be multiples of 128 for the tensor-core transforms";
            return false;
        }
        if (mode == QS_PREC_BF16X3) { kind = 0; nsplit = 2; }
        else if (mode == QS_PREC_TF32X3) { kind = 1; nsplit = 2; }
        else if (mode == QS_PREC_BF16X6) { kind = 0; nsplit = 3; }
        else { why = "not a tensor-core precision"; return false; }
        const bool bf16 = kind == 0;
        const int elem = bf16 ? 2 : 4;
        const size_t plane = (size_t)ny * nz;
        const size_t bytes = (size_t)nsplit * nfmax * plane * elem;
        if (cudaMalloc(&splitA, bytes) != cudaSuccess || cudaMalloc(&splitB, bytes) != cudaSuccess) {
            why = "cudaMalloc of split operands failed";
            return false;
        }
        cudaMemset(splitA, 0, bytes);
        cudaMemset(splitB, 0, bytes);
        if (!upload_matrix(ny, &matY, why)) return false;
        if (nz != ny && !upload_matrix(nz, &matZ, why)) return false;
        void* mz = matZ ? matZ : matY;
        const uint32_t bk = 128 / elem;
        for (int b = 0; b < 2; b++) {
            const uint32_t bn = b ? 128 : 64;
            // pass 1 (along y): data = splitA [term][nfmax][nz][ny]
            if (!encode_2d(&mapD1[b], splitA, bf16, ny, (uint64_t)nsplit * nfmax * nz, bk, bn, why))
                return false;
            // pass 2 (along z): data = splitB [term][nfmax][ny][nz]
            if (!encode_2d(&mapD2[b], splitB, bf16, nz, (uint64_t)nsplit * nfmax * ny, bk, bn, why))
                return false;
            smem_bytes[b] = (size_t)stages_for(b) * nsplit * (128 * 128 + bn * 128) + 1024;
        }
        if (!encode_2d(&mapM1, matY, bf16, ny, (uint64_t)nsplit * 2 * ny, bk, 128, why)) return false;
        if (!encode_2d(&mapM2, mz, bf16, nz, (uint64_t)nsplit * 2 * nz, bk, 128, why)) return false;
        chunk_k = 128;
        if (const char* e = getenv("QS_TC_CHUNK")) chunk_k = atoi(e);
        cudaError_t e = cudaSuccess;
#define QS_SET_SMEM(K, NS, ST, BN, B)                                                              \
    if (e == cudaSuccess)                                                                          \
        e = cudaFuncSetAttribute(tcx::dtt_tc_kernel<K, NS, ST, BN>,                                \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes[B]);
        if (mode == QS_PREC_BF16X3) { QS_SET_SMEM(0, 2, 4, 64, 0) QS_SET_SMEM(0, 2, 3, 128, 1) }
        else if (mode == QS_PREC_TF32X3) { QS_SET_SMEM(1, 2, 4, 64, 0) QS_SET_SMEM(1, 2, 3, 128, 1) }
        else { QS_SET_SMEM(0, 3, 3, 64, 0) QS_SET_SMEM(0, 3, 2, 128, 1) }
#undef QS_SET_SMEM
        if (e != cudaSuccess) {
            why = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
            return false;
        }
        return true;
    }

    int promo_for(int K) const {
        const int bk = (kind == 0) ? 64 : 32;
        const int nkb = K / bk;
        if (chunk_k <= 0) return nkb;
        int pr = chunk_k / bk;
        if (pr < 1) pr = 1;
        while (pr > 1 && nkb % pr) pr--;
        return pr;
    }

    // tile width: 128 when the batch fills the GPU with 128-wide tiles
    int bn_index(int nf, int R, int K) const { return nf * (R / 128) * (K / 128) >= 96 ? 1 : 0; }

    void launch_gemm(int pass, tcx::Params& p, int nf, cudaStream_t st) {
        const int b = bn_index(nf, p.R, p.K);
        const int bn = b ? 128 : 64;
        dim3 grid(p.K / tcx::BM, p.R / bn, nf);
        const CUtensorMap& D = pass == 1 ? mapD1[b] : mapD2[b];
        const CUtensorMap& M = pass == 1 ? mapM1 : mapM2;
        const int T = tcx::THREADS_V2;
        const size_t sm = smem_bytes[b];
        if (mode == QS_PREC_BF16X3) {
            if (b) qs::launch_pdl(tcx::dtt_tc_kernel<0, 2, 3, 128>, grid, dim3(T), sm, st, M, D, p);
            else qs::launch_pdl(tcx::dtt_tc_kernel<0, 2, 4, 64>, grid, dim3(T), sm, st, M, D, p);
        } else if (mode == QS_PREC_TF32X3) {
            if (b) qs::launch_pdl(tcx::dtt_tc_kernel<1, 2, 3, 128>, grid, dim3(T), sm, st, M, D, p);
            else qs::launch_pdl(tcx::dtt_tc_kernel<1, 2, 4, 64>, grid, dim3(T), sm, st, M, D, p);
        } else {
            if (b) qs::launch_pdl(tcx::dtt_tc_kernel<0, 3, 2, 128>, grid, dim3(T), sm, st, M, D, p);
            else qs::launch_pdl(tcx::dtt_tc_kernel<0, 3, 3, 64>, grid, dim3(T), sm, st, M, D, p);
        }
    }

    void launch_split(const float* base, int nf, cudaStream_t st) {
        const size_t plane = (size_t)ny * nz;
        const size_t ts = (size_t)nfmax * plane;
        dim3 sg((unsigned)((plane / 4 + 255) / 256), nf);
        if (kind == 0 && nsplit == 2)
            qs::launch_pdl(tcx::split_planes_kernel<0, 2>, sg, dim3(256), 0, st, base, plane, nf, plane, ts, splitA);
        else if (kind == 0)
            qs::launch_pdl(tcx::split_planes_kernel<0, 3>, sg, dim3(256), 0, st, base, plane, nf, plane, ts, splitA);
        else
            qs::launch_pdl(tcx::split_planes_kernel<1, 2>, sg, dim3(256), 0, st, base, plane, nf, plane, ts, splitA);
    }

    void pass_params(int stage, int nf, const int* kz, const int* ky, double scale,
                     tcx::Params& p) {
        p.err = err;
        p.nfmax = nfmax;
        unsigned long long mask = 0;
        if (stage == 1) {   // along y: splitA (nz rows of ny) -> splitB, transposed
            for (int f = 0; f < nf; f++) mask |= (unsigned long long)(ky ? (ky[f] & 1) : 0) << f;
            p.R = nz; p.K = ny;
            p.data_rows = nfmax * nz; p.mat_rows = 2 * ny;
            p.out_split = 1; p.out_base = splitB; p.scale = 1.0f;
        } else {            // along z: splitB (ny rows of nz) -> FP32 destination
            for (int f = 0; f < nf; f++) mask |= (unsigned long long)(kz ? (kz[f] & 1) : 0) << f;
            p.R = ny; p.K = nz;
            p.data_rows = nfmax * ny; p.mat_rows = 2 * nz;
            p.out_split = 0; p.out_base = nullptr; p.scale = (float)scale;
        }
        p.kindmask = mask;
        p.promo = promo_for(p.K);
    }

    int run_stage(int stage, int nf, const void* const* in, void* const* out, const int* kz,
                  const int* ky, double scale, cudaStream_t st) override {
        if (nf <= 0 || nf > kMaxXfFields) return 0;
        const size_t plane = (size_t)ny * nz;
        if (stage == 0) {
            const float* base = (const float*)in[0];
            for (int f = 1; f < nf; f++)
                if ((const float*)in[f] != base + (size_t)f * plane) return -1;
            launch_split(base, nf, st);
            return 1;
        }
        tcx::Params p{};
        pass_params(stage, nf, kz, ky, scale, p);
        if (stage == 2)
            for (int f = 0; f < nf; f++) p.out[f] = (float*)out[f];
        launch_gemm(stage, p, nf, st);
        return 1;
    }

    int run(int nf, const void* const* in, void* const* out, const int* kz, const int* ky,
            double scale, int elem_size, cudaStream_t st) override {
        if (elem_size != 4) return 0;
        int n = 0;
        for (int s = 0; s < 3; s++) n += run_stage(s, nf, in, out, kz, ky, scale, st);
        return n;
    }

    void split_target(void** base, int* ns, int* kd, size_t* term_stride) override {
        *base = splitA;
        *ns = nsplit;
        *kd = kind;
        *term_stride = (size_t)nfmax * ny * nz;
    }

    int run_batched(const float* in, float* out, int nplanes, double scale, int stage,
                    cudaStream_t st) override {
        int n = 0;
        const size_t plane = (size_t)ny * nz;
        for (int b0 = 0; b0 < nplanes; b0 += nfmax) {
            const int nf = std::min(nfmax, nplanes - b0);
            if (stage < 0 || stage == 0) { launch_split(in + (size_t)b0 * plane, nf, st); n++; }
            for (int ps = 1; ps <= 2; ps++) {
                if (stage >= 0 && stage != ps) continue;
                tcx::Params p{};
                pass_params(ps, nf, nullptr, nullptr, scale, p);
                if (ps == 2) {
                    p.out_contig = 1;
                    p.out[0] = out + (size_t)b0 * plane;
                }
                launch_gemm(ps, p, nf, st);
                n++;
            }
        }
        return n;
    }
};

}  // namespace


TcTransformer* TcTransformer::create(int mode, int ny, int nz, int* err_flag, std::string& why) {
    auto* t = new TcImpl();
    t->mode = mode;
    t->ny = ny;
    t->nz = nz;
    t->err = err_flag;
    if (!t->init(why)) {
        delete t;
        return nullptr;
    }
    return t;
}

}  // namespace qs
