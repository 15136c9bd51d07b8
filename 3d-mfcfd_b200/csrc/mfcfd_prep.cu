/*
 * mfcfd_prep.cu - the set-up's graph passes on the GPU (mfcfd_params
 * .gpu_setup): split stencils, the alias breadth-first search and the sweep
 * levels.  Each gives exactly the host path's result (mfcfd_setup.cpp):
 *
 *  - split stencils (generate_connectivity.f90:38-246): one thread per point
 *    evaluates the same projections (same operand order, no fused
 *    multiply-add) and sign tests.  The reference stores each list in 22
 *    entries and lets longer ones run into the next point's column, which
 *    depends on the order points are visited; when any list is longer than
 *    the capacity, the caller redoes the pass on the host.
 *  - alias (implicit_aliasing.f90:21-42) is a FIFO breadth-first search.
 *    It is run level by level: every parent of the current level offers
 *    each unvisited neighbour the key (parent position, slot j); the
 *    smallest key is the first discovery of the sequential search, and the
 *    keys' order is the order of discovery, which a prefix sum over the key
 *    space turns into alias numbers.  Point 1's first neighbour takes alias
 *    1 and is never a parent, as in the reference.
 *  - levels: the longest-path depth over a sweep's dependencies, by Kahn's
 *    layering (a point joins level L+1 when its last dependency leaves
 *    level L), with one kernel per level queued without host round trips.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "mfcfd_internal.h"

namespace mfcfd {
namespace {

constexpr int PREP_THREADS = 256;

// Device buffers of one pass, freed on every return path.
struct DevBufs {
    std::vector<void *> ptrs;
    ~DevBufs() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <typename T>
    cudaError_t alloc(T **p, size_t count) {
        void *v = nullptr;
        cudaError_t e = cudaMalloc(&v, sizeof(T) * (count > 0 ? count : 1));
        if (e == cudaSuccess) ptrs.push_back(v);
        *p = (T *)v;
        return e;
    }
};

struct Stream {
    cudaStream_t s = nullptr;
    ~Stream() {
        if (s) cudaStreamDestroy(s);
    }
};

#define PREP_CK(call)                                                      \
    do {                                                                   \
        cudaError_t e_ = (call);                                           \
        if (e_ != cudaSuccess) {                                           \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);      \
            return MFCFD_ERR_CUDA;                                         \
        }                                                                  \
    } while (0)

// ---------------------------------------------------------------- split stencils

__global__ void k_split(int n, int cap, const int8_t *cls, const double *x, const double *y, const double *z,
                        const double *tan1, const double *tan2, const double *nor, const int32_t *nbhs,
                        const int32_t *conn, int32_t *split, int32_t *cnt, int *overflow) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = cls[i];
    int cn[NDIR] = {0, 0, 0, 0, 0, 0};
    if (c == CLS_INTERIOR || c == CLS_WALL || c == CLS_OUTER) {
        const double xi = x[i], yi = y[i], zi = z[i];
        const double *t1 = tan1 + 3 * (size_t)i, *t2 = tan2 + 3 * (size_t)i, *nn = nor + 3 * (size_t)i;
        auto push = [&](int d, int k) {
            const int j = cn[d]++;
            if (j < cap) split[(size_t)d * n * cap + (size_t)i * cap + j] = k;
        };
        for (int r = 0; r < nbhs[i]; ++r) {
            const int k = conn[(size_t)i * MAX_CONN + r];
            const double delx = x[k - 1] - xi, dely = y[k - 1] - yi, delz = z[k - 1] - zi;
            const double dels = delx * t1[0] + dely * t1[1] + delz * t1[2];
            const double delt = delx * t2[0] + dely * t2[1] + delz * t2[2];
            if (c == CLS_INTERIOR) {
                const double deln = delx * nn[0] + dely * nn[1] + delz * nn[2];
                if (dels <= 0.0) push(0, k);
                if (dels > 0.0) push(1, k);
                if (delt <= 0.0) push(2, k);
                if (delt > 0.0) push(3, k);
                if (deln <= 0.0) push(4, k);
                if (deln > 0.0) push(5, k);
            } else {
                if (dels <= 0.0) push(0, k);
                if (dels >= 0.0) push(1, k);
                if (delt <= 0.0) push(2, k);
                if (delt >= 0.0) push(3, k);
                push(c == CLS_WALL ? 5 : 4, k);
            }
        }
    }
    bool over = false;
#pragma unroll
    for (int d = 0; d < NDIR; ++d) {
        cnt[(size_t)d * n + i] = cn[d];
        over = over || cn[d] > cap;
    }
    if (over) atomicExch(overflow, 1);
}

// ---------------------------------------------------------------- prefix sum

// Exclusive scan of `len` ints in blocks of 1024: per-block scans and sums,
// one block scans the sums (carrying across chunks), then offsets are added.
__device__ __forceinline__ int block_exclusive_scan(int v, int *warp_sums, int *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
        int si = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += t;
        }
        warp_sums[lane] = si - s;   // exclusive over warps
        if (lane == 31) *total = si;
    }
    __syncthreads();
    return inc - v + warp_sums[warp];
}

__global__ void __launch_bounds__(1024) k_scan_blocks(const int *in, int *out, int *block_sums, int len) {
    __shared__ int ws[32];
    __shared__ int tot;
    const int i = blockIdx.x * 1024 + threadIdx.x;
    const int v = i < len ? in[i] : 0;
    const int ex = block_exclusive_scan(v, ws, &tot);
    if (i < len) out[i] = ex;
    if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) k_scan_sums(int *block_sums, int nblocks, int *total) {
    __shared__ int ws[32];
    __shared__ int tot;
    int carry = 0;
    for (int base = 0; base < nblocks; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < nblocks ? block_sums[i] : 0;
        const int ex = block_exclusive_scan(v, ws, &tot);
        if (i < nblocks) block_sums[i] = ex + carry;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(1024) k_scan_add(int *out, const int *block_sums, int len) {
    const int i = blockIdx.x * 1024 + threadIdx.x;
    if (i < len) out[i] += block_sums[blockIdx.x];
}

// ---------------------------------------------------------------- alias search

constexpr unsigned NO_KEY = 0xffffffffu;

// key space: (frontier position f, neighbour slot j) -> f * MAX_CONN + j
__global__ void k_bfs_offer(const int32_t *front, int m, const int32_t *nbhs, const int32_t *conn,
                            const int32_t *alias, unsigned *key) {
    const size_t len = (size_t)m * MAX_CONN;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < len; t += (size_t)gridDim.x * blockDim.x) {
        const int f = (int)(t / MAX_CONN), j = (int)(t % MAX_CONN);
        const int p = front[f];
        if (j >= nbhs[p]) continue;
        const int k = conn[(size_t)p * MAX_CONN + j] - 1;
        if (alias[k] == 0) atomicMin(&key[k], (unsigned)t);
    }
}

__global__ void k_bfs_winners(const int32_t *front, int m, const int32_t *nbhs, const int32_t *conn,
                              const int32_t *alias, const unsigned *key, int *flag) {
    const size_t len = (size_t)m * MAX_CONN;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < len; t += (size_t)gridDim.x * blockDim.x) {
        const int f = (int)(t / MAX_CONN), j = (int)(t % MAX_CONN);
        const int p = front[f];
        int win = 0;
        if (j < nbhs[p]) {
            const int k = conn[(size_t)p * MAX_CONN + j] - 1;
            win = alias[k] == 0 && key[k] == (unsigned)t;
        }
        flag[t] = win;
    }
}

__global__ void k_bfs_emit(const int32_t *front, int m, const int32_t *conn, const int *flag, const int *pos,
                           int base, int32_t *alias, int32_t *pwa, int32_t *next, unsigned *key) {
    const size_t len = (size_t)m * MAX_CONN;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < len; t += (size_t)gridDim.x * blockDim.x) {
        if (!flag[t]) continue;
        const int f = (int)(t / MAX_CONN), j = (int)(t % MAX_CONN);
        const int k = conn[(size_t)front[f] * MAX_CONN + j] - 1;
        const int a = base + pos[t] + 1;          // alias number (count after this discovery)
        next[pos[t]] = k;
        alias[k] = a;
        pwa[a - 1] = k + 1;
        key[k] = NO_KEY;
    }
}

// ---------------------------------------------------------------- levels

__global__ void k_lv_count(const int32_t *order, int nsw, const int32_t *doff, const int32_t *deps,
                           int32_t *indeg, int32_t *rcnt) {
    const int oi = blockIdx.x * blockDim.x + threadIdx.x;
    if (oi >= nsw) return;
    const int p = order[oi];
    indeg[p] = doff[p + 1] - doff[p];
    for (int e = doff[p]; e < doff[p + 1]; ++e) atomicAdd(&rcnt[deps[e]], 1);
}

__global__ void k_lv_fill(const int32_t *order, int nsw, const int32_t *doff, const int32_t *deps,
                          const int32_t *roff, int32_t *rcur, int32_t *rlist) {
    const int oi = blockIdx.x * blockDim.x + threadIdx.x;
    if (oi >= nsw) return;
    const int p = order[oi];
    for (int e = doff[p]; e < doff[p + 1]; ++e) {
        const int k = deps[e];
        rlist[roff[k] + atomicAdd(&rcur[k], 1)] = p;
    }
}

__global__ void k_lv_roots(const int32_t *order, int nsw, const int32_t *indeg, int32_t *level, int32_t *front,
                           int32_t *count) {
    const int oi = blockIdx.x * blockDim.x + threadIdx.x;
    if (oi >= nsw) return;
    const int p = order[oi];
    if (indeg[p] == 0) {
        level[p] = 0;
        front[atomicAdd(count, 1)] = p;
    }
}

// Level L: the points of front (count[L]) release their dependents.
__global__ void k_lv_step(int L, const int32_t *front, const int32_t *count, const int32_t *roff,
                          const int32_t *rlist, int32_t *indeg, int32_t *level, int32_t *next) {
    const int m = count[L];
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m; f += gridDim.x * blockDim.x) {
        const int p = front[f];
        for (int e = roff[p]; e < roff[p + 1]; ++e) {
            const int q = rlist[e];
            if (atomicSub(&indeg[q], 1) == 1) {
                level[q] = L + 1;
                next[atomicAdd((int32_t *)&count[L + 1], 1)] = q;
            }
        }
    }
}

int exclusive_scan(const int *in, int *out, int len, int *d_sums, int *d_total, cudaStream_t s, std::string &err) {
    const int nb = (len + 1023) / 1024;
    if (len > 0) {
        k_scan_blocks<<<nb, 1024, 0, s>>>(in, out, d_sums, len);
        k_scan_sums<<<1, 1024, 0, s>>>(d_sums, nb, d_total);
        k_scan_add<<<nb, 1024, 0, s>>>(out, d_sums, len);
    } else {
        PREP_CK(cudaMemsetAsync(d_total, 0, sizeof(int), s));
    }
    PREP_CK(cudaGetLastError());
    return MFCFD_OK;
}

}  // namespace

int prep_split_gpu(int device, int n, int cap, const std::vector<int8_t> &cls, const double *x, const double *y,
                   const double *z, const double *tan1, const double *tan2, const double *nor, const int32_t *nbhs,
                   const int32_t *conn, Topology &T, bool *overflow, std::string &err) {
    PREP_CK(cudaSetDevice(device));
    Stream st;
    PREP_CK(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
    DevBufs b;
    int8_t *d_cls;
    double *d_x, *d_y, *d_z, *d_t1, *d_t2, *d_nn;
    int32_t *d_nb, *d_conn, *d_split, *d_cnt;
    int *d_over;
    const size_t n3 = 3 * (size_t)n;
    PREP_CK(b.alloc(&d_cls, n));
    PREP_CK(b.alloc(&d_x, n)); PREP_CK(b.alloc(&d_y, n)); PREP_CK(b.alloc(&d_z, n));
    PREP_CK(b.alloc(&d_t1, n3)); PREP_CK(b.alloc(&d_t2, n3)); PREP_CK(b.alloc(&d_nn, n3));
    PREP_CK(b.alloc(&d_nb, n)); PREP_CK(b.alloc(&d_conn, (size_t)n * MAX_CONN));
    PREP_CK(b.alloc(&d_split, (size_t)NDIR * n * cap)); PREP_CK(b.alloc(&d_cnt, (size_t)NDIR * n));
    PREP_CK(b.alloc(&d_over, 1));
    cudaStream_t s = st.s;
    PREP_CK(cudaMemcpyAsync(d_cls, cls.data(), n, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_x, x, 8 * (size_t)n, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_y, y, 8 * (size_t)n, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_z, z, 8 * (size_t)n, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_t1, tan1, 8 * n3, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_t2, tan2, 8 * n3, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_nn, nor, 8 * n3, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_nb, nbhs, 4 * (size_t)n, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_conn, conn, 4 * (size_t)n * MAX_CONN, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemsetAsync(d_split, 0, 4 * (size_t)NDIR * n * cap, s));
    PREP_CK(cudaMemsetAsync(d_over, 0, sizeof(int), s));
    k_split<<<(n + PREP_THREADS - 1) / PREP_THREADS, PREP_THREADS, 0, s>>>(n, cap, d_cls, d_x, d_y, d_z, d_t1, d_t2,
                                                                        d_nn, d_nb, d_conn, d_split, d_cnt, d_over);
    PREP_CK(cudaGetLastError());
    int over = 0;
    PREP_CK(cudaMemcpyAsync(&over, d_over, sizeof(int), cudaMemcpyDeviceToHost, s));
    PREP_CK(cudaStreamSynchronize(s));
    *overflow = over != 0;
    if (over) return MFCFD_OK;   // the caller runs the reference's sequential storage
    for (int d = 0; d < NDIR; ++d) {
        T.split[d].assign((size_t)n * cap + 64, 0);
        T.split_cnt[d].assign(n, 0);
        PREP_CK(cudaMemcpyAsync(T.split[d].data(), d_split + (size_t)d * n * cap, 4 * (size_t)n * cap,
                                cudaMemcpyDeviceToHost, s));
        PREP_CK(cudaMemcpyAsync(T.split_cnt[d].data(), d_cnt + (size_t)d * n, 4 * (size_t)n, cudaMemcpyDeviceToHost,
                                s));
    }
    PREP_CK(cudaStreamSynchronize(s));
    T.split_overflows = 0;
    return MFCFD_OK;
}

int prep_alias_gpu(int device, int n, const int32_t *nbhs, const int32_t *conn, std::vector<int32_t> &alias,
                   std::vector<int32_t> &pwa, std::string &err) {
    PREP_CK(cudaSetDevice(device));
    Stream st;
    PREP_CK(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
    cudaStream_t s = st.s;
    DevBufs b;
    int32_t *d_nb, *d_conn, *d_alias, *d_pwa, *d_fa, *d_fb;
    unsigned *d_key;
    int *d_flag, *d_pos, *d_sums, *d_total;
    const size_t kspace = (size_t)n * MAX_CONN;
    if (kspace >= 0x7fffffffull) {
        err = "cloud too large for the GPU alias search";
        return MFCFD_ERR_UNSUPPORTED;
    }
    PREP_CK(b.alloc(&d_nb, n)); PREP_CK(b.alloc(&d_conn, kspace));
    PREP_CK(b.alloc(&d_alias, n)); PREP_CK(b.alloc(&d_pwa, n));
    PREP_CK(b.alloc(&d_fa, n)); PREP_CK(b.alloc(&d_fb, n));
    PREP_CK(b.alloc(&d_key, n)); PREP_CK(b.alloc(&d_flag, kspace)); PREP_CK(b.alloc(&d_pos, kspace));
    PREP_CK(b.alloc(&d_sums, (kspace + 1023) / 1024)); PREP_CK(b.alloc(&d_total, 1));
    PREP_CK(cudaMemcpyAsync(d_nb, nbhs, 4 * (size_t)n, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_conn, conn, 4 * kspace, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemsetAsync(d_alias, 0, 4 * (size_t)n, s));
    PREP_CK(cudaMemsetAsync(d_pwa, 0, 4 * (size_t)n, s));
    PREP_CK(cudaMemsetAsync(d_key, 0xff, 4 * (size_t)n, s));
    // point 1 is alias 1 and the first parent (implicit_aliasing.f90:17-19)
    const int one = 1, zero = 0;
    PREP_CK(cudaMemcpyAsync(d_alias, &one, sizeof(int), cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_pwa, &one, sizeof(int), cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_fa, &zero, sizeof(int), cudaMemcpyHostToDevice, s));
    int m = 1, count = 0, skip = 0;
    int32_t *front = d_fa, *next = d_fb;
    while (m > 0) {
        const size_t len = (size_t)m * MAX_CONN;
        const int grid = (int)std::min<size_t>((len + PREP_THREADS - 1) / PREP_THREADS, (size_t)device_sms(device) * 16);
        k_bfs_offer<<<grid, PREP_THREADS, 0, s>>>(front + skip, m, d_nb, d_conn, d_alias, d_key);
        k_bfs_winners<<<grid, PREP_THREADS, 0, s>>>(front + skip, m, d_nb, d_conn, d_alias, d_key, d_flag);
        int rc = exclusive_scan(d_flag, d_pos, (int)len, d_sums, d_total, s, err);
        if (rc) return rc;
        k_bfs_emit<<<grid, PREP_THREADS, 0, s>>>(front + skip, m, d_conn, d_flag, d_pos, count, d_alias, d_pwa, next,
                                               d_key);
        PREP_CK(cudaGetLastError());
        int found = 0;
        PREP_CK(cudaMemcpyAsync(&found, d_total, sizeof(int), cudaMemcpyDeviceToHost, s));
        PREP_CK(cudaStreamSynchronize(s));
        // the first point found from point 1 shares its alias slot and is
        // never a parent (implicit_aliasing.f90:27-40 with pwa(1) overwritten)
        skip = count == 0 ? 1 : 0;
        m = found - skip;
        count += found;
        std::swap(front, next);
    }
    alias.assign(n, 0);
    pwa.assign(n, 0);
    PREP_CK(cudaMemcpyAsync(alias.data(), d_alias, 4 * (size_t)n, cudaMemcpyDeviceToHost, s));
    PREP_CK(cudaMemcpyAsync(pwa.data(), d_pwa, 4 * (size_t)n, cudaMemcpyDeviceToHost, s));
    PREP_CK(cudaStreamSynchronize(s));
    return MFCFD_OK;
}

int prep_levels_gpu(int device, int n, const std::vector<int> &order, const std::vector<int32_t> &doff,
                    const std::vector<int32_t> &deps, std::vector<int32_t> &level, std::string &err) {
    PREP_CK(cudaSetDevice(device));
    Stream st;
    PREP_CK(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
    cudaStream_t s = st.s;
    const int nsw = (int)order.size();
    const int ne = (int)deps.size();
    DevBufs b;
    int32_t *d_order, *d_doff, *d_deps, *d_indeg, *d_rcnt, *d_roff, *d_rcur, *d_rlist, *d_level, *d_fa, *d_fb,
        *d_count;
    int *d_sums, *d_total;
    PREP_CK(b.alloc(&d_order, nsw)); PREP_CK(b.alloc(&d_doff, (size_t)n + 1)); PREP_CK(b.alloc(&d_deps, ne));
    PREP_CK(b.alloc(&d_indeg, n)); PREP_CK(b.alloc(&d_rcnt, (size_t)n + 1)); PREP_CK(b.alloc(&d_roff, (size_t)n + 1));
    PREP_CK(b.alloc(&d_rcur, n)); PREP_CK(b.alloc(&d_rlist, ne)); PREP_CK(b.alloc(&d_level, n));
    PREP_CK(b.alloc(&d_fa, nsw)); PREP_CK(b.alloc(&d_fb, nsw)); PREP_CK(b.alloc(&d_count, (size_t)nsw + 2));
    PREP_CK(b.alloc(&d_sums, ((size_t)n + 1 + 1023) / 1024)); PREP_CK(b.alloc(&d_total, 1));
    PREP_CK(cudaMemcpyAsync(d_order, order.data(), 4 * (size_t)nsw, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_doff, doff.data(), 4 * ((size_t)n + 1), cudaMemcpyHostToDevice, s));
    if (ne > 0) PREP_CK(cudaMemcpyAsync(d_deps, deps.data(), 4 * (size_t)ne, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemsetAsync(d_rcnt, 0, 4 * ((size_t)n + 1), s));
    PREP_CK(cudaMemsetAsync(d_rcur, 0, 4 * (size_t)n, s));
    PREP_CK(cudaMemsetAsync(d_level, 0xff, 4 * (size_t)n, s));
    PREP_CK(cudaMemsetAsync(d_count, 0, 4 * ((size_t)nsw + 2), s));
    const int g = (nsw + PREP_THREADS - 1) / PREP_THREADS;
    if (nsw > 0) {
        k_lv_count<<<g, PREP_THREADS, 0, s>>>(d_order, nsw, d_doff, d_deps, d_indeg, d_rcnt);
        int rc = exclusive_scan(d_rcnt, d_roff, n + 1, d_sums, d_total, s, err);
        if (rc) return rc;
        k_lv_fill<<<g, PREP_THREADS, 0, s>>>(d_order, nsw, d_doff, d_deps, d_roff, d_rcur, d_rlist);
        k_lv_roots<<<g, PREP_THREADS, 0, s>>>(d_order, nsw, d_indeg, d_level, d_fa, d_count);
        PREP_CK(cudaGetLastError());
    }
    // level L reads count[L] and front, writes count[L+1] and next; batches
    // of levels are queued before the host looks whether the last was empty
    int L = 0;
    int32_t *front = d_fa, *next = d_fb;
    constexpr int BATCH = 256;
    while (L < nsw) {
        const int stop = std::min(nsw, L + BATCH);
        for (; L < stop; ++L) {
            k_lv_step<<<64, PREP_THREADS, 0, s>>>(L, front, d_count, d_roff, d_rlist, d_indeg, d_level, next);
            std::swap(front, next);
        }
        PREP_CK(cudaGetLastError());
        int last = 0;
        PREP_CK(cudaMemcpyAsync(&last, d_count + L, sizeof(int), cudaMemcpyDeviceToHost, s));
        PREP_CK(cudaStreamSynchronize(s));
        if (last == 0) break;
    }
    level.assign(n, -1);
    PREP_CK(cudaMemcpyAsync(level.data(), d_level, 4 * (size_t)n, cudaMemcpyDeviceToHost, s));
    PREP_CK(cudaStreamSynchronize(s));
    for (int p : order)
        if (level[p] < 0) {
            err = "sweep dependencies contain a cycle";
            return MFCFD_ERR_STENCIL;
        }
    return MFCFD_OK;
}

}  // namespace mfcfd
