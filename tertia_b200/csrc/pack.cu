// pack.cu — the particle blocks of the xi-pipeline hand-off buffer gathered on
// the device (PackLayer, para.cpp:135-146 of the reference): the plasma in
// flight ordered cell by cell (k outer, j inner, as the layer walk of
// paraCPUlayers.cu:76-113), load order within a cell, written as the 12
// double rows Px Py Pz X Y Z Q2m Weight i_X i_Y i_Z isort, so that the whole
// buffer leaves the device in one copy.
//
// Order: a counting sort by cell (count, one-block scan, placement with a
// per-cell atomic cursor), then one thread per cell puts its few particles
// back in load order (insertion sort on the load id; the ids are a
// permutation, so the order is unique), then one thread per output row entry
// gathers and widens the particle's values.  The unpack runs the same sort the
// other way: the buffer checked on the device, its particles ordered by cell
// (buffer order within a cell) and narrowed into the plasma arrays.
#include "qs_internal.h"

namespace qs {
namespace {

__global__ void pack_count_kernel(const int32_t* __restrict__ cell, int64_t m, int ncell,
                                  int* __restrict__ cnt, int* __restrict__ err) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m) return;
    const int c = cell[q];
    if (c < 0 || c >= ncell) {
        atomicOr(err, DEV_ERR_INTERNAL);
        return;
    }
    atomicAdd(cnt + c, 1);
}

// start[0..n] = exclusive prefix sums of cnt[0..n): each of the 1024 threads
// sums a contiguous chunk, the block scans the chunk sums in shared memory,
// and each thread writes the offsets of its chunk
__global__ void __launch_bounds__(1024) pack_scan_kernel(const int* __restrict__ cnt, int n,
                                                         int* __restrict__ start) {
    __shared__ int part[1024];
    const int t = threadIdx.x;
    const int chunk = (n + 1023) / 1024;
    const int b = min(n, t * chunk), e = min(n, b + chunk);
    int s = 0;
    for (int i = b; i < e; i++) s += cnt[i];
    part[t] = s;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {   // inclusive scan of the chunk sums
        const int v = t >= d ? part[t - d] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int off = part[t] - s;
    for (int i = b; i < e; i++) {
        start[i] = off;
        off += cnt[i];
    }
    if (t == 1023) start[n] = part[1023];
}

__global__ void pack_place_kernel(const int32_t* __restrict__ cell, int64_t m, int ncell,
                                  const int* __restrict__ start, int* __restrict__ fill,
                                  int32_t* __restrict__ ord) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m) return;
    const int c = cell[q];
    if (c < 0 || c >= ncell) return;   // counted as an error, not placed
    ord[start[c] + atomicAdd(fill + c, 1)] = (int32_t)q;
}

// one thread per cell: its particles in ascending load id (key[q], or q
// itself when the device order is the load order)
__global__ void pack_cell_order_kernel(const int* __restrict__ start, int ncell,
                                       const int32_t* __restrict__ key,
                                       int32_t* __restrict__ ord) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const int b = start[c], e = start[c + 1];
    for (int i = b + 1; i < e; i++) {
        const int32_t v = ord[i];
        const int32_t kv = key ? key[v] : v;
        int j = i - 1;
        while (j >= b) {
            const int32_t u = ord[j];
            if ((key ? key[u] : u) <= kv) break;
            ord[j + 1] = u;
            j--;
        }
        ord[j + 1] = v;
    }
}

template <class T>
__global__ void pack_rows_kernel(PackArgs<T> a) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t m = a.m;
    if (r >= m || r >= a.start[a.ncell]) return;   // rows past the placed particles stay unset
    const int32_t q = a.ord[r];
    if (q < 0 || q >= m) {
        atomicOr(a.err, DEV_ERR_INTERNAL);
        return;
    }
    const int c = a.cell[q];
    double* o = a.out;
    o[r] = (double)a.px[q];
    o[r + m] = (double)a.py[q];
    o[r + 2 * m] = (double)a.pz[q];
    o[r + 3 * m] = 0.0;                 // in-cell xi: plasma enters at x = 0
    o[r + 4 * m] = (double)a.y[q];
    o[r + 5 * m] = (double)a.z[q];
    o[r + 6 * m] = a.q2m;
    o[r + 7 * m] = (double)a.w[q];
    o[r + 8 * m] = 0.0;                 // the layer index i_X
    o[r + 9 * m] = (double)(c % a.My);
    o[r + 10 * m] = (double)(c / a.My);
    o[r + 11 * m] = 0.0;                // isort: the plasma electrons
}

// out = w0 a + w1 b in double, rounded as the separate products and sum
template <class T>
__global__ void pack_mix_kernel(const T* __restrict__ a, const T* __restrict__ b, double w0,
                                double w1, size_t n, double* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = __dadd_rn(__dmul_rn(w0, (double)a[i]), __dmul_rn(w1, (double)b[i]));
}

// ---- UnpackLayer (para.cpp:175-285) on the device: the buffer's particle
// blocks checked row by row, then ordered by cell (stable: buffer order within
// a cell) and gathered into the plasma arrays.

// a row's cell, or -1 and the lowest bad row recorded: the cell must be a
// whole (j, k) inside the layer, the in-cell position in [0, 1], the species
// the plasma electrons (Q2m, isort 0) - the host reports the row's reason
__global__ void unpack_check_kernel(const double* __restrict__ pb, int64_t m, int My, int Mz,
                                    double q2m, int32_t* __restrict__ key_cell,
                                    int* __restrict__ cnt, unsigned long long* __restrict__ bad) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    const double jd = pb[r + 9 * m], kd = pb[r + 10 * m];
    const double yy = pb[r + 4 * m], zz = pb[r + 5 * m];
    const bool cell_ok = jd >= 0 && jd < My && kd >= 0 && kd < Mz && jd == (double)(int)jd &&
                         kd == (double)(int)kd;
    const bool pos_ok = yy >= 0 && yy <= 1 && zz >= 0 && zz <= 1;
    const bool sort_ok = pb[r + 6 * m] == q2m && pb[r + 11 * m] == 0.0;
    if (!(cell_ok && pos_ok && sort_ok)) {
        atomicMin(bad, (unsigned long long)r);
        key_cell[r] = -1;
        return;
    }
    const int c = (int)jd + My * (int)kd;
    key_cell[r] = c;
    atomicAdd(cnt + c, 1);
}

__global__ void unpack_place_kernel(const int32_t* __restrict__ key_cell, int64_t m,
                                    const int* __restrict__ start, int* __restrict__ fill,
                                    int32_t* __restrict__ ord) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    const int c = key_cell[r];
    if (c < 0) return;
    ord[start[c] + atomicAdd(fill + c, 1)] = (int32_t)r;
}

template <class T>
__global__ void unpack_gather_kernel(UnpackArgs<T> a) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t m = a.m;
    if (r >= m) return;
    const int32_t q = a.ord[r];
    if (q < 0 || q >= m) {
        atomicOr(a.err, DEV_ERR_INTERNAL);
        return;
    }
    const double* pb = a.buf;
    const int c = a.key_cell[q];
    a.cell[r] = c;
    a.px[r] = (T)pb[q];
    a.py[r] = (T)pb[q + m];
    a.pz[r] = (T)pb[q + 2 * m];
    a.y[r] = (T)pb[q + 4 * m];
    a.z[r] = (T)pb[q + 5 * m];
    a.w[r] = (T)pb[q + 7 * m];
    if (a.ppc <= 0 || c != (int)(r / a.ppc)) atomicOr(a.nonuniform, 1);
}

}  // namespace

template <class T>
int launch_unpack_check(const UnpackArgs<T>& a, cudaStream_t st) {
    if (a.m <= 0) return 0;
    unpack_check_kernel<<<(unsigned)((a.m + 255) / 256), 256, 0, st>>>(
        a.buf, a.m, a.My, a.Mz, a.q2m, a.key_cell, a.cnt, a.bad);
    return 1;
}

template <class T>
int launch_unpack_order(const UnpackArgs<T>& a, cudaStream_t st) {
    if (a.m <= 0) return 0;
    const unsigned gm = (unsigned)((a.m + 255) / 256);
    const unsigned gc = (unsigned)((a.ncell + 255) / 256);
    pack_scan_kernel<<<1, 1024, 0, st>>>(a.cnt, a.ncell, a.start);
    unpack_place_kernel<<<gm, 256, 0, st>>>(a.key_cell, a.m, a.start, a.fill, a.ord);
    pack_cell_order_kernel<<<gc, 256, 0, st>>>(a.start, a.ncell, nullptr, a.ord);
    unpack_gather_kernel<T><<<gm, 256, 0, st>>>(a);
    return 4;
}

template <class T>
int launch_pack_particles(const PackArgs<T>& a, cudaStream_t st) {
    if (a.m <= 0) return 0;
    const unsigned gm = (unsigned)((a.m + 255) / 256);
    const unsigned gc = (unsigned)((a.ncell + 255) / 256);
    pack_count_kernel<<<gm, 256, 0, st>>>(a.cell, a.m, a.ncell, a.cnt, a.err);
    pack_scan_kernel<<<1, 1024, 0, st>>>(a.cnt, a.ncell, a.start);
    pack_place_kernel<<<gm, 256, 0, st>>>(a.cell, a.m, a.ncell, a.start, a.fill, a.ord);
    pack_cell_order_kernel<<<gc, 256, 0, st>>>(a.start, a.ncell, a.key, a.ord);
    pack_rows_kernel<T><<<gm, 256, 0, st>>>(a);
    return 5;
}

template <class T>
int launch_pack_mix(const T* a, const T* b, double w0, double w1, size_t n, double* out,
                    cudaStream_t st) {
    if (!n) return 0;
    pack_mix_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, b, w0, w1, n, out);
    return 1;
}

template int launch_pack_particles<float>(const PackArgs<float>&, cudaStream_t);
template int launch_pack_particles<double>(const PackArgs<double>&, cudaStream_t);
template int launch_unpack_check<float>(const UnpackArgs<float>&, cudaStream_t);
template int launch_unpack_check<double>(const UnpackArgs<double>&, cudaStream_t);
template int launch_unpack_order<float>(const UnpackArgs<float>&, cudaStream_t);
template int launch_unpack_order<double>(const UnpackArgs<double>&, cudaStream_t);
template int launch_pack_mix<float>(const float*, const float*, double, double, size_t, double*,
                                    cudaStream_t);
template int launch_pack_mix<double>(const double*, const double*, double, double, size_t,
                                     double*, cudaStream_t);

}  // namespace qs
