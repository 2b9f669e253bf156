// sort.cu — keeping the FP32 CIC plasma grouped by cell.
//
// In CIC the plasma moves between cells (the reference relinks a particle to
// the cell it moves into on the full step, movepart_layer_CIC.cpp:449-496);
// at 512^2 with thermal spread nearly every particle has left its seeded cell
// by the tail of the box.  The CIC push stages each cell tile's fields and
// deposits in shared memory and pushes the particles of the tile, so the
// particle arrays are regrouped by cell after each full push: a counting sort
// whose histogram the full push itself builds (atomic count per new cell), an
// exclusive scan of the counts in one kernel (per 1024-cell block; the last
// block to finish scans the block totals), and a scatter whose within-cell
// rank is an atomic decrement of the count (so the counts end at zero, ready
// for the next full push).  Each particle carries its load-order id so that
// the host gets the plasma back in load order.
#include "qs_common.cuh"
#include "qs_internal.h"
#include "pdl.cuh"
#include "trace.cuh"

namespace qs {

namespace {

constexpr int kScanBlock = 1024;

__global__ void __launch_bounds__(256) count_cells_kernel(const int32_t* __restrict__ cell,
                                                          int64_t n, int ncell,
                                                          int* __restrict__ cnt,
                                                          int* __restrict__ err) {
    pdl_wait();
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    pdl_trigger();
    if (p >= n) return;
    const int c = cell[p];
    if (c < 0 || c >= ncell) atomicOr(err, DEV_ERR_INTERNAL);
    else atomicAdd(cnt + c, 1);
}

__device__ __forceinline__ int block_exclusive_scan(int v, int* wsum, int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;   // inclusive warp scan
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int s = wsum[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= d) s += y;
        }
        wsum[lane] = s;   // inclusive over warps
    }
    __syncthreads();
    total = wsum[31];
    return (warp > 0 ? wsum[warp - 1] : 0) + x - v;
}

// Exclusive scan of cnt within blocks of kScanBlock cells (loff); the last
// block to finish (ticket counter) scans the block totals into bpref
// (bpref[nb] = total) and resets the counter.  No block waits on another.
__global__ void __launch_bounds__(kScanBlock) scan_cells_kernel(int* __restrict__ cnt, int ncell,
                                                                int* __restrict__ loff,
                                                                int* __restrict__ bsum,
                                                                int* __restrict__ bpref,
                                                                unsigned* __restrict__ ticket,
                                                                int clear) {
    __shared__ int wsum[kScanBlock / 32];
    __shared__ bool last;
    QS_TRACE_ENTRY();
    pdl_wait();
    QS_TRACE_WAITED();
    const int c = blockIdx.x * kScanBlock + threadIdx.x;
    const int v = c < ncell ? cnt[c] : 0;
    if (clear && c < ncell) cnt[c] = 0;
    int total = 0;
    const int before = block_exclusive_scan(v, wsum, total);
    if (c < ncell) loff[c] = before;
    if (threadIdx.x == 0) {
        bsum[blockIdx.x] = total;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    QS_TRACE_END(trace::K_SCAN);
    if (!last) return;
    __threadfence();
    const int nb = gridDim.x;
    const int b = threadIdx.x;
    __syncthreads();
    const int bv = b < nb ? __ldcg(bsum + b) : 0;
    int all = 0;
    const int bex = block_exclusive_scan(bv, wsum, all);
    pdl_trigger();
    if (b < nb) bpref[b] = bex;
    if (b == 0) {
        bpref[nb] = all;
        *ticket = 0u;
    }
}

template <class T>
__global__ void __launch_bounds__(256) scatter_kernel(PlasmaSet<T> in, PlasmaSet<T> out, int64_t n,
                                                      int ncell, int* __restrict__ cnt,
                                                      const int* __restrict__ loff,
                                                      const int* __restrict__ bpref,
                                                      int* __restrict__ err) {
    QS_TRACE_ENTRY();
    pdl_wait();
    QS_TRACE_WAITED();
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int c = in.cell[p];
    if (c < 0 || c >= ncell) {   // a cell the counts never saw: record, skip
        atomicOr(err, DEV_ERR_INTERNAL);
        return;
    }
    const int r = atomicSub(cnt + c, 1) - 1;
    const int64_t q = (int64_t)loff[c] + bpref[c / kScanBlock] + r;
    if (r < 0 || q < 0 || q >= n) {   // counts out of step with the cells: record, skip
        atomicOr(err, DEV_ERR_INTERNAL);
        return;
    }
    const T y = in.y[p], z = in.z[p], px = in.px[p], py = in.py[p], pz = in.pz[p], w = in.w[p];
    const int32_t id = in.id[p];
    pdl_trigger();
    out.cell[q] = c;
    out.y[q] = y; out.z[q] = z; out.px[q] = px; out.py[q] = py; out.pz[q] = pz; out.w[q] = w;
    out.id[q] = id;
    QS_TRACE_END(trace::K_SCATTER);
}

__global__ void iota_kernel(int32_t* __restrict__ id, int64_t n) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) id[p] = (int32_t)p;
}

}  // namespace

int scan_blocks_count(int ncell) { return (ncell + kScanBlock - 1) / kScanBlock; }

int launch_count_cells(const int32_t* cell, int64_t n, int ncell, int* cnt, int* err,
                       cudaStream_t st) {
    if (n <= 0) return 0;
    launch_pdl(count_cells_kernel, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, st, cell, n,
               ncell, cnt, err);
    return 1;
}

int launch_cell_offsets(int* cnt, int ncell, int* loff, int* bsum, int* bpref,
                        unsigned* ticket, int clear, cudaStream_t st) {
    const int nb = scan_blocks_count(ncell);
    launch_pdl(scan_cells_kernel, dim3(nb), dim3(kScanBlock), 0, st, cnt, ncell, loff, bsum, bpref,
               ticket, clear);
    return 1;
}

template <class T>
int launch_scatter(const PlasmaSet<T>& in, const PlasmaSet<T>& out, int64_t n, int ncell,
                   int* cnt, const int* loff, const int* bpref, int* err, cudaStream_t st) {
    if (n <= 0) return 0;
    launch_pdl(scatter_kernel<T>, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, st, in, out, n,
               ncell, cnt, loff, bpref, err);
    return 1;
}

int launch_iota(int32_t* id, int64_t n, cudaStream_t st) {
    if (n <= 0) return 0;
    iota_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(id, n);
    return 1;
}

template int launch_scatter<float>(const PlasmaSet<float>&, const PlasmaSet<float>&, int64_t, int,
                                   int*, const int*, const int*, int*, cudaStream_t);
template int launch_scatter<double>(const PlasmaSet<double>&, const PlasmaSet<double>&, int64_t,
                                    int, int*, const int*, const int*, int*, cudaStream_t);

}  // namespace qs

QS_TRACE_UNIT(sort)
