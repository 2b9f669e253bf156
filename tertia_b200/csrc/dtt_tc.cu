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
#include <cstring>
#include <vector>

#include "dtt_tc.h"
#include "qs_common.cuh"

namespace qs {
namespace tcx {

constexpr int BM = 128;
constexpr int BN = 64;
constexpr int THREADS = 128;
constexpr int TMEM_COLS = 64;
constexpr uint32_t SPIN_LIMIT = 1u << 22;

struct Params {
    int R, K;              // rows per field, row length (= transform size)
    int nsplit;            // operand split terms
    int nterm;             // product terms
    int ta[6], tb[6];      // split index of A and B for each product term
    int kind[kMaxXfFields];
    int rowsA;             // rows of one split term in the A map (8 * R)
    int rowsB;             // rows of one split term in the B map (2 * K)
    int out_split;         // 1: write split planes to out_base
    void* out_base;        // [term][8][K][R]
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
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
    for (uint32_t i = 0; i < SPIN_LIMIT; i++) {
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

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// split an FP32 value into n terms of the low-precision type
template <int KIND>
__device__ __forceinline__ void split_value(float v, int n, float (&t)[3]) {
    float r = v;
#pragma unroll
    for (int s = 0; s < 3; s++) {
        if (s < n) {
            float h = (KIND == 0) ? __bfloat162float(__float2bfloat16_rn(r)) : tf32_rna(r);
            t[s] = h;
            r = r - h;
        } else {
            t[s] = 0.f;
        }
    }
}

// ------------------------------------------------------------ the GEMM
template <int KIND, int NSPLIT, int STAGES>
__global__ void __launch_bounds__(THREADS, 1)
    dtt_tc_kernel(const __grid_constant__ CUtensorMap mapA,
                  const __grid_constant__ CUtensorMap mapB, const Params p) {
    constexpr int ELEM = (KIND == 0) ? 2 : 4;
    constexpr int BK = 128 / ELEM;                  // one 128-byte swizzle row
    constexpr uint32_t A_TILE = BM * 128;           // 16 KB
    constexpr uint32_t B_TILE = BN * 128;           // 8 KB
    constexpr uint32_t STAGE = NSPLIT * (A_TILE + B_TILE);

    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], accum_bar;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int f = blockIdx.z;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int nkb = p.K / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(smem_u32(&full_bar[s]), 1);
            mbar_init(smem_u32(&empty_bar[s]), 1);
        }
        mbar_init(smem_u32(&accum_bar), 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;
    volatile int* abortp = &abort_flag;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer
        const int rowA = f * p.R + m0;
        const int rowB = p.kind[f] * p.K + n0;
        int issued = 0;
        for (int kb = 0; kb < nkb; kb++) {
            const int s = kb % STAGES;
            const uint32_t use = kb / STAGES;
            if (kb >= STAGES && !mbar_wait(smem_u32(&empty_bar[s]), (use - 1) & 1, abortp)) {
                *abortp = 1;
                break;
            }
            const uint32_t fb = smem_u32(&full_bar[s]);
            mbar_expect_tx(fb, STAGE);
            uint8_t* st = smem + (size_t)s * STAGE;
#pragma unroll
            for (int t = 0; t < NSPLIT; t++)
                tma_load_2d(smem_u32(st + t * A_TILE), &mapA, fb, kb * BK, t * p.rowsA + rowA);
#pragma unroll
            for (int t = 0; t < NSPLIT; t++)
                tma_load_2d(smem_u32(st + NSPLIT * A_TILE + t * B_TILE), &mapB, fb, kb * BK,
                            t * p.rowsB + rowB);
            issued = kb + 1;
        }
        if (*abortp) {
            // drain the copies this thread put in flight before leaving
            for (int kb = (issued > STAGES ? issued - STAGES : 0); kb < issued; kb++)
                mbar_wait(smem_u32(&full_bar[kb % STAGES]), (kb / STAGES) & 1, abortp);
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer
        const uint32_t idesc = (1u << 4) | ((KIND == 0 ? 1u : 2u) << 7) |
                               ((KIND == 0 ? 1u : 2u) << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(BM >> 4) << 24);
        bool ok = true;
        for (int kb = 0; kb < nkb && ok; kb++) {
            const int s = kb % STAGES;
            if (!mbar_wait(smem_u32(&full_bar[s]), (kb / STAGES) & 1, abortp)) {
                *abortp = 1;
                ok = false;
                break;
            }
            fence_after();
            const uint32_t st = smem_u32(smem + (size_t)s * STAGE);
            for (int t = 0; t < p.nterm; t++) {
                const uint32_t a = st + p.ta[t] * A_TILE;
                const uint32_t b = st + NSPLIT * A_TILE + p.tb[t] * B_TILE;
#pragma unroll
                for (int kk = 0; kk < 4; kk++) {
                    mma<KIND>(tmem, sw128_desc(a + kk * 32), sw128_desc(b + kk * 32), idesc,
                              (kb | t | kk) != 0);
                }
            }
            mma_commit(smem_u32(&empty_bar[s]));
        }
        if (ok) mma_commit(smem_u32(&accum_bar));
    }
    __syncwarp();

    // ---------------- epilogue (all 4 warps)
    const bool have = mbar_wait(smem_u32(&accum_bar), 0, abortp);
    fence_after();
    if (have) {
        const int m = m0 + warp * 32 + lane;    // TMEM lane = tile row
        const size_t plane = (size_t)p.R * p.K;
#pragma unroll
        for (int c = 0; c < BN; c += 16) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
            tmem_wait_ld();
            if (!p.out_split) {
                float* o = p.out[f];
#pragma unroll
                for (int jj = 0; jj < 16; jj++) {
                    const int n = n0 + c + jj;
                    o[(size_t)n * p.R + m] = __uint_as_float(v[jj]) * p.scale;
                }
            } else {
#pragma unroll
                for (int jj = 0; jj < 16; jj++) {
                    const int n = n0 + c + jj;
                    const size_t idx = (size_t)f * plane + (size_t)n * p.R + m;
                    float t[3];
                    split_value<KIND>(__uint_as_float(v[jj]) * p.scale, NSPLIT, t);
                    if (KIND == 0) {
                        __nv_bfloat16* ob = (__nv_bfloat16*)p.out_base;
#pragma unroll
                        for (int s = 0; s < NSPLIT; s++)
                            ob[(size_t)s * 8 * plane + idx] = __float2bfloat16_rn(t[s]);
                    } else {
                        float* of = (float*)p.out_base;
#pragma unroll
                        for (int s = 0; s < NSPLIT; s++) of[(size_t)s * 8 * plane + idx] = t[s];
                    }
                }
            }
        }
    } else if (threadIdx.x == 0) {
        atomicOr(p.err, DEV_ERR_TIMEOUT);
    }
    fence_before();
    __syncthreads();
    if (warp == 2) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TMEM_COLS)
                     : "memory");
    }
}

// split nf FP32 planes (R x K each) into the operand terms [term][8][R][K]
template <int KIND>
__global__ void split_planes_kernel(const float* const* __restrict__ in_ptrs, int nf, size_t plane,
                                    int nsplit, void* out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (i >= plane || f >= nf) return;
    const float v = in_ptrs[f][i];
    float t[3];
    split_value<KIND>(v, nsplit, t);
    const size_t idx = (size_t)f * plane + i;
    if (KIND == 0) {
        __nv_bfloat16* o = (__nv_bfloat16*)out;
        for (int s = 0; s < nsplit; s++) o[(size_t)s * 8 * plane + idx] = __float2bfloat16_rn(t[s]);
    } else {
        float* o = (float*)out;
        for (int s = 0; s < nsplit; s++) o[(size_t)s * 8 * plane + idx] = t[s];
    }
}

struct PtrPack {
    const float* p[kMaxXfFields];
};

template <int KIND>
__global__ void split_planes_kernel_v(PtrPack in, int nf, size_t plane, int nsplit, void* out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (i >= plane || f >= nf) return;
    const float v = in.p[f][i];
    float t[3];
    split_value<KIND>(v, nsplit, t);
    const size_t idx = (size_t)f * plane + i;
    if (KIND == 0) {
        __nv_bfloat16* o = (__nv_bfloat16*)out;
        for (int s = 0; s < nsplit; s++) o[(size_t)s * 8 * plane + idx] = __float2bfloat16_rn(t[s]);
    } else {
        float* o = (float*)out;
        for (int s = 0; s < nsplit; s++) o[(size_t)s * 8 * plane + idx] = t[s];
    }
}

}  // namespace tcx

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
    int mode = 0, ny = 0, nz = 0, kind = 0, nsplit = 2, nterm = 3, stages = 4;
    int ta[6] = {0, 0, 1, 0, 1, 2}, tb[6] = {0, 1, 0, 2, 1, 0};
    void* splitA = nullptr;
    void* splitB = nullptr;
    void* matY = nullptr;
    void* matZ = nullptr;
    int* err = nullptr;
    CUtensorMap mapA1, mapB1, mapA2, mapB2;
    size_t smem_bytes = 0;

    ~TcImpl() override {
        for (void* p : {splitA, splitB, matY, matZ})
            if (p) cudaFree(p);
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
                    for (int s = 0; s < nsplit; s++) {
                        float t = round_term(rem, bf16);
                        rem -= (double)t;
                        size_t idx = (size_t)s * 2 * nn + (size_t)kd * nn + r * n + c;
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
        if (ny % BM_ || nz % BM_) {
            why = "ny and nz must be multiples of 128 for the tensor-core transforms";
            return false;
        }
        if (mode == QS_PREC_BF16X3) { kind = 0; nsplit = 2; nterm = 3; stages = 4; }
        else if (mode == QS_PREC_TF32X3) { kind = 1; nsplit = 2; nterm = 3; stages = 4; }
        else if (mode == QS_PREC_BF16X6) { kind = 0; nsplit = 3; nterm = 6; stages = 3; }
        else { why = "not a tensor-core precision"; return false; }
        const bool bf16 = kind == 0;
        const int elem = bf16 ? 2 : 4;
        const size_t plane = (size_t)ny * nz;
        const size_t bytes = (size_t)nsplit * 8 * plane * elem;
        if (cudaMalloc(&splitA, bytes) != cudaSuccess || cudaMalloc(&splitB, bytes) != cudaSuccess) {
            why = "cudaMalloc of split operands failed";
            return false;
        }
        cudaMemset(splitA, 0, bytes);
        cudaMemset(splitB, 0, bytes);
        if (!upload_matrix(ny, &matY, why)) return false;
        if (nz == ny) matZ = nullptr;
        else if (!upload_matrix(nz, &matZ, why)) return false;
        void* mz = matZ ? matZ : matY;
        const uint32_t bk = 128 / elem;
        // pass 1: A = splitA [term][8][nz][ny], B = matY [term][2][ny][ny]
        if (!encode_2d(&mapA1, splitA, bf16, ny, (uint64_t)nsplit * 8 * nz, bk, 128, why)) return false;
        if (!encode_2d(&mapB1, matY, bf16, ny, (uint64_t)nsplit * 2 * ny, bk, 64, why)) return false;
        // pass 2: A = splitB [term][8][ny][nz], B = matZ [term][2][nz][nz]
        if (!encode_2d(&mapA2, splitB, bf16, nz, (uint64_t)nsplit * 8 * ny, bk, 128, why)) return false;
        if (!encode_2d(&mapB2, mz, bf16, nz, (uint64_t)nsplit * 2 * nz, bk, 64, why)) return false;
        smem_bytes = (size_t)stages * nsplit * (128 * 128 + 64 * 128) + 1024;
        cudaError_t e = cudaSuccess;
        if (mode == QS_PREC_BF16X3)
            e = cudaFuncSetAttribute(tcx::dtt_tc_kernel<0, 2, 4>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
        else if (mode == QS_PREC_TF32X3)
            e = cudaFuncSetAttribute(tcx::dtt_tc_kernel<1, 2, 4>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
        else
            e = cudaFuncSetAttribute(tcx::dtt_tc_kernel<0, 3, 3>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
        if (e != cudaSuccess) {
            why = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
            return false;
        }
        return true;
    }

    static constexpr int BM_ = 128;

    void launch_gemm(const CUtensorMap& A, const CUtensorMap& B, const tcx::Params& p, int nf,
                     cudaStream_t st) {
        dim3 grid(p.R / tcx::BM, p.K / tcx::BN, nf);
        if (mode == QS_PREC_BF16X3)
            tcx::dtt_tc_kernel<0, 2, 4><<<grid, tcx::THREADS, smem_bytes, st>>>(A, B, p);
        else if (mode == QS_PREC_TF32X3)
            tcx::dtt_tc_kernel<1, 2, 4><<<grid, tcx::THREADS, smem_bytes, st>>>(A, B, p);
        else
            tcx::dtt_tc_kernel<0, 3, 3><<<grid, tcx::THREADS, smem_bytes, st>>>(A, B, p);
    }

    int run_stage(int stage, int nf, const void* const* in, void* const* out, const int* kz,
                  const int* ky, double scale, cudaStream_t st) override {
        if (nf <= 0 || nf > kMaxXfFields) return 0;
        const size_t plane = (size_t)ny * nz;
        if (stage == 0) {
            tcx::PtrPack pk{};
            for (int f = 0; f < nf; f++) pk.p[f] = (const float*)in[f];
            dim3 sg((unsigned)((plane + 255) / 256), nf);
            if (kind == 0)
                tcx::split_planes_kernel_v<0><<<sg, 256, 0, st>>>(pk, nf, plane, nsplit, splitA);
            else
                tcx::split_planes_kernel_v<1><<<sg, 256, 0, st>>>(pk, nf, plane, nsplit, splitA);
            return 1;
        }
        tcx::Params p{};
        p.nsplit = nsplit;
        p.nterm = nterm;
        for (int t = 0; t < 6; t++) { p.ta[t] = ta[t]; p.tb[t] = tb[t]; }
        p.err = err;
        if (stage == 1) {   // along y: splitA (nz x ny rows) -> splitB, transposed
            p.R = nz; p.K = ny;
            for (int f = 0; f < nf; f++) p.kind[f] = ky[f];
            p.rowsA = 8 * nz; p.rowsB = 2 * ny;
            p.out_split = 1; p.out_base = splitB; p.scale = 1.0f;
            launch_gemm(mapA1, mapB1, p, nf, st);
        } else {            // along z: splitB (ny x nz rows) -> FP32 destination
            p.R = ny; p.K = nz;
            for (int f = 0; f < nf; f++) { p.kind[f] = kz[f]; p.out[f] = (float*)out[f]; }
            p.rowsA = 8 * ny; p.rowsB = 2 * nz;
            p.out_split = 0; p.out_base = nullptr; p.scale = (float)scale;
            launch_gemm(mapA2, mapB2, p, nf, st);
        }
        return 1;
    }

    int run(int nf, const void* const* in, void* const* out, const int* kz, const int* ky,
            double scale, int elem_size, cudaStream_t st) override {
        if (elem_size != 4) return 0;
        int n = 0;
        for (int s = 0; s < 3; s++) n += run_stage(s, nf, in, out, kz, ky, scale, st);
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
