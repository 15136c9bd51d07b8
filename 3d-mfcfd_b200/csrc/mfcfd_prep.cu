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
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <type_traits>
#include <string>
#include <thread>
#include <vector>

#include "mfcfd_internal.h"

namespace mfcfd {
namespace {

constexpr int PREP_THREADS = 256;

// Device buffers of one pass, freed on every return path.  With a stream
// they are stream-ordered (allocated and freed on it), so a set-up running
// beside other work never waits for the whole device to drain.
struct DevBufs {
    std::vector<void *> ptrs;
    cudaStream_t stream = nullptr;
    DevBufs() = default;
    explicit DevBufs(cudaStream_t s) : stream(s) {}
    ~DevBufs() {
        for (void *p : ptrs) {
            if (stream) cudaFreeAsync(p, stream);
            else cudaFree(p);
        }
    }
    template <typename T>
    cudaError_t alloc(T **p, size_t count) {
        void *v = nullptr;
        const size_t bytes = sizeof(T) * (count > 0 ? count : 1);
        cudaError_t e = stream ? cudaMallocAsync(&v, bytes, stream) : cudaMalloc(&v, bytes);
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

namespace {

// The breadth-first search on device arrays (nbhs, 1-based conn): alias and
// point_with_alias, both n long, are written on stream s.
int alias_search(int device, int n, const int32_t *d_nb, const int32_t *d_conn, int32_t *d_alias, int32_t *d_pwa,
                 cudaStream_t s, std::string &err) {
    DevBufs b(s);
    int32_t *d_fa, *d_fb;
    unsigned *d_key;
    int *d_flag, *d_pos, *d_sums, *d_total;
    const size_t kspace = (size_t)n * MAX_CONN;
    if (kspace >= 0x7fffffffull) {
        err = "cloud too large for the GPU alias search";
        return MFCFD_ERR_UNSUPPORTED;
    }
    PREP_CK(b.alloc(&d_fa, n)); PREP_CK(b.alloc(&d_fb, n));
    PREP_CK(b.alloc(&d_key, n)); PREP_CK(b.alloc(&d_flag, kspace)); PREP_CK(b.alloc(&d_pos, kspace));
    PREP_CK(b.alloc(&d_sums, (kspace + 1023) / 1024)); PREP_CK(b.alloc(&d_total, 1));
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
    return MFCFD_OK;
}

}  // namespace

int prep_alias_gpu(int device, int n, const int32_t *nbhs, const int32_t *conn, std::vector<int32_t> &alias,
                   std::vector<int32_t> &pwa, std::string &err) {
    PREP_CK(cudaSetDevice(device));
    Stream st;
    PREP_CK(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
    cudaStream_t s = st.s;
    DevBufs b;
    int32_t *d_nb, *d_conn, *d_alias, *d_pwa;
    const size_t kspace = (size_t)n * MAX_CONN;
    PREP_CK(b.alloc(&d_nb, n)); PREP_CK(b.alloc(&d_conn, kspace));
    PREP_CK(b.alloc(&d_alias, n)); PREP_CK(b.alloc(&d_pwa, n));
    PREP_CK(cudaMemcpyAsync(d_nb, nbhs, 4 * (size_t)n, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(d_conn, conn, 4 * kspace, cudaMemcpyHostToDevice, s));
    if (int rc = alias_search(device, n, d_nb, d_conn, d_alias, d_pwa, s, err)) return rc;
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

// ================================================================ device-resident set-up
//
// The passes of build_topology (mfcfd_setup.cpp) on device arrays, in the
// storage order of the handle: a point p of storage is the reference's point
// inv[p], and every point id a kernel writes is a storage index.  Each pass
// evaluates what the host's does for that point, with the same operations in
// the same order (this file is compiled without contraction), so the arrays
// equal those build_topology + permute_topology give.

namespace {

struct SplitPtrs {
    int32_t *p[NDIR];
};

__device__ __forceinline__ int map_id(const int32_t *perm, int i) { return perm ? perm[i] : i; }

inline int grid_for(int device, size_t len) {
    const size_t g = (len + PREP_THREADS - 1) / PREP_THREADS;
    return (int)std::max<size_t>(1, std::min<size_t>(g, (size_t)device_sms(device) * 16));
}

#define GRID_STRIDE(t, len) \
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (len); t += (size_t)gridDim.x * blockDim.x)

// storage-order copies of the cloud: coordinates, frames (tan1, tan2, nor per
// point), classes, neighbour counts and conn with 0-based storage ids (an id
// past nbhs that is not a point reads 0, like a zero pad)
__global__ void k_stage_cloud(int n, const int32_t *perm, const double *x, const double *y, const double *z,
                              const double *t1, const double *t2, const double *nn, const int8_t *cls,
                              const int32_t *nbhs, const int32_t *conn, double *sx, double *sy, double *sz,
                              double *frame, int8_t *scls, int32_t *snb, int32_t *sconn) {
    GRID_STRIDE(t, (size_t)n) {
        const int i = (int)t, p = map_id(perm, i);
        sx[p] = x[i];
        sy[p] = y[i];
        sz[p] = z[i];
        for (int r = 0; r < 3; ++r) {
            frame[9 * (size_t)p + r] = t1[3 * (size_t)i + r];
            frame[9 * (size_t)p + 3 + r] = t2[3 * (size_t)i + r];
            frame[9 * (size_t)p + 6 + r] = nn[3 * (size_t)i + r];
        }
        scls[p] = cls[i];
        snb[p] = nbhs[i];
        for (int r = 0; r < MAX_CONN; ++r) {
            const int k = conn[(size_t)i * MAX_CONN + r];
            sconn[(size_t)p * MAX_CONN + r] = (k > 0 && k <= n) ? map_id(perm, k - 1) : 0;
        }
    }
}

// split stencils in the reference's storage (logical): own cells only; the
// counts are the lists' full lengths
__global__ void k_split_own(int n, int cap, const int8_t *cls, const double *x, const double *y, const double *z,
                            const double *tan1, const double *tan2, const double *nor, const int32_t *nbhs,
                            const int32_t *conn, SplitPtrs split, int32_t *cnt, int *overflow) {
    GRID_STRIDE(t, (size_t)n) {
        const int i = (int)t;
        const int c = cls[i];
        int cn[NDIR] = {0, 0, 0, 0, 0, 0};
        if (c == CLS_INTERIOR || c == CLS_WALL || c == CLS_OUTER) {
            const double xi = x[i], yi = y[i], zi = z[i];
            const double *t1 = tan1 + 3 * (size_t)i, *t2 = tan2 + 3 * (size_t)i, *nn = nor + 3 * (size_t)i;
            auto push = [&](int d, int k) {
                const int j = cn[d]++;
                if (j < cap) split.p[d][(size_t)i * cap + j] = k;
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
        for (int d = 0; d < NDIR; ++d) {
            cnt[(size_t)d * n + i] = cn[d];
            over = over || cn[d] > cap;
        }
        if (over) atomicExch(overflow, 1);
    }
}

__global__ void k_spill_apply(int m, const int *d, const long long *at, const int32_t *val, SplitPtrs split) {
    GRID_STRIDE(t, (size_t)m) split.p[d[t]][at[t]] = val[t];
}

// alias of every storage point (the sweeps compare aliases)
__global__ void k_alias_storage(int n, const int32_t *perm, const int32_t *alias, int32_t *salias) {
    GRID_STRIDE(t, (size_t)n) salias[map_id(perm, (int)t)] = alias[t];
}

enum { SLOT_OK = 0, SLOT_ZERO, SLOT_LONG, SLOT_WIDE };

// effective lists and neighbour slots (build_topology's "effective lists")
__global__ void k_slots(int n, int cap, const int32_t *perm, const int32_t *inv, const int8_t *cls,
                        const int32_t *nbhs, const int32_t *conn, SplitPtrs split, const int32_t *cnt,
                        int32_t *slot_nbr, uint8_t *nslot, uint8_t *slot_mask, uint8_t *list_cnt, uint8_t *list_ent,
                        uint8_t *code, int *bad) {
    GRID_STRIDE(t, (size_t)n) {
        const int p = (int)t, i = inv ? inv[p] : p;
        int32_t *slots = slot_nbr + (size_t)p * MAX_SLOTS;
        uint8_t *mask = slot_mask + (size_t)p * MAX_SLOTS;
        for (int s = 0; s < MAX_SLOTS; ++s) {
            slots[s] = -1;
            mask[s] = 0;
        }
        for (int e = 0; e < NDIR * LIST_STRIDE; ++e) list_ent[(size_t)p * NDIR * LIST_STRIDE + e] = 0;
        for (int d = 0; d < NDIR; ++d) list_cnt[(size_t)p * NDIR + d] = 0;
        int ns = 0;
        auto slot_of = [&](int k) -> int {
            for (int s = 0; s < ns; ++s)
                if (slots[s] == k) return s;
            if (ns == MAX_SLOTS) return -1;
            slots[ns] = k;
            return ns++;
        };
        const int nb = nbhs[i];
        for (int r = 0; r < nb; ++r) slot_of(map_id(perm, conn[(size_t)i * MAX_CONN + r] - 1));
        const int c = cls[i];
        int status = SLOT_OK;
        for (int d = 0; d < NDIR && status == SLOT_OK; ++d) {
            const bool unused = (c == CLS_WALL && d == 4) || (c == CLS_OUTER && d == 5) || c == CLS_SUPERSONIC;
            if (unused) continue;
            const bool use_conn = c == CLS_WALL && d == 5;
            const int len = use_conn ? nb : cnt[(size_t)d * n + i];
            if (!use_conn)
                for (int j = 0; j < len; ++j) {
                    const int k = split.p[d][(size_t)i * cap + j];
                    if (k < 1 || k > n) status = SLOT_ZERO;
                }
            if (status != SLOT_OK) break;
            if (len > MAX_CONN) { status = SLOT_LONG; break; }
            list_cnt[(size_t)p * NDIR + d] = (uint8_t)len;
            for (int j = 0; j < len; ++j) {
                const int k1 = use_conn ? conn[(size_t)i * MAX_CONN + j] : split.p[d][(size_t)i * cap + j];
                const int s = slot_of(map_id(perm, k1 - 1));
                if (s < 0) { status = SLOT_WIDE; break; }
                list_ent[((size_t)p * NDIR + d) * LIST_STRIDE + j] = (uint8_t)s;
                mask[s] |= (uint8_t)(1u << d);
            }
        }
        nslot[p] = (uint8_t)ns;
        code[i] = (uint8_t)status;
        if (status != SLOT_OK) atomicMin(bad, i);
    }
}

__device__ __forceinline__ double dev_det(double xx, double yy, double zz, double xy, double yz, double zx) {
    return xx * (yy * zz - yz * yz) - xy * (xy * zz - yz * zx) + zx * (xy * yz - yy * zx);
}

// Cramer numerators in the reference's operand order (implicit_D_inv_interior
// .f90:103-105, :225-227, :347-349), as the host set-up's numerator()
__device__ __forceinline__ double dev_numerator(int axis, double xx, double yy, double zz, double xy, double yz,
                                                double zx, double fx, double fy, double fz) {
    if (axis == 0)
        return fx * (yy * zz - yz * yz) - fy * (xy * zz - zx * yz) + fz * (xy * yz - zx * yy);
    if (axis == 1)
        return xx * (fy * zz - yz * fz) - xy * (fx * zz - zx * fz) + zx * (fx * yz - zx * fy);
    return xx * (yy * fz - fy * yz) - xy * (xy * fz - fx * yz) + zx * (xy * fy - fx * yy);
}

// least-squares moments, determinant and D_inv numerator per (point, list),
// weight 1 (power 0)
__global__ void k_geo(int n, const double *x, const double *y, const double *z, const double *frame,
                      const uint8_t *list_cnt, const uint8_t *list_ent, const int32_t *slot_nbr, double *geo) {
    GRID_STRIDE(t, (size_t)n) {
        const int i = (int)t;
        const double *t1 = frame + 9 * (size_t)i, *t2 = t1 + 3, *nn = t1 + 6;
        for (int d = 0; d < NDIR; ++d) {
            const int c = list_cnt[(size_t)i * NDIR + d];
            double xx = 0, yy = 0, zz = 0, xy = 0, yz = 0, zx = 0, sdx = 0, sdy = 0, sdz = 0;
            for (int j = 0; j < c; ++j) {
                const int s = list_ent[((size_t)i * NDIR + d) * LIST_STRIDE + j];
                const int k = slot_nbr[(size_t)i * MAX_SLOTS + s];
                const double delx = x[k] - x[i], dely = y[k] - y[i], delz = z[k] - z[i];
                const double dels = delx * t1[0] + dely * t1[1] + delz * t1[2];
                const double delt = delx * t2[0] + dely * t2[1] + delz * t2[2];
                const double deln = delx * nn[0] + dely * nn[1] + delz * nn[2];
                const double w = 1.0;
                const double ws = dels * w, wt = delt * w, wn = deln * w;
                xx = xx + dels * ws;
                yy = yy + delt * wt;
                zz = zz + deln * wn;
                xy = xy + dels * wt;
                yz = yz + delt * wn;
                zx = zx + deln * ws;
                sdx = sdx + ws;
                sdy = sdy + wt;
                sdz = sdz + wn;
            }
            double *g = geo + (size_t)i * GEO_STRIDE + d * 8;
            g[G_XX] = xx; g[G_YY] = yy; g[G_ZZ] = zz;
            g[G_XY] = xy; g[G_YZ] = yz; g[G_ZX] = zx;
            g[G_DET] = dev_det(xx, yy, zz, xy, yz, zx);
            g[G_DNUM] = dev_numerator(d / 2, xx, yy, zz, xy, yz, zx, sdx, sdy, sdz);
        }
    }
}

// sweep order: the points point_with_alias names that the sweeps update
__global__ void k_swept_flags(int n, const int32_t *pwa, const int8_t *cls, int *flag) {
    GRID_STRIDE(t, (size_t)n) {
        const int q = pwa[t];
        const int c = q > 0 ? cls[q - 1] : -1;
        flag[t] = (c == CLS_WALL || c == CLS_INTERIOR) ? 1 : 0;
    }
}

__global__ void k_swept_emit(int n, const int32_t *pwa, const int32_t *perm, const int *flag, const int *pos,
                             int32_t *order, uint8_t *swept) {
    GRID_STRIDE(t, (size_t)n) {
        if (!flag[t]) continue;
        const int p = map_id(perm, pwa[t] - 1);
        order[pos[t]] = p;
        swept[p] = 1;
    }
}

__global__ void k_reverse(int m, const int32_t *a, int32_t *b) {
    GRID_STRIDE(t, (size_t)m) b[t] = a[m - 1 - (int)t];
}

// sweep terms: count per point (then a scan gives the offsets), fill
__global__ void k_ent_count(int nsw, bool forward, const int32_t *order, const int32_t *salias,
                            const uint8_t *list_cnt, const uint8_t *list_ent, const int32_t *slot_nbr, uint8_t *cnt,
                            int *tot) {
    GRID_STRIDE(t, (size_t)nsw) {
        const int p = order[t];
        int all = 0;
        for (int d = 0; d < NDIR; ++d) {
            const int c = list_cnt[(size_t)p * NDIR + d];
            int taken = 0;
            for (int j = 0; j < c; ++j) {
                const int k = slot_nbr[(size_t)p * MAX_SLOTS + list_ent[((size_t)p * NDIR + d) * LIST_STRIDE + j]];
                if (forward ? salias[k] < salias[p] : salias[k] > salias[p]) ++taken;
            }
            cnt[(size_t)p * NDIR + d] = (uint8_t)taken;
            all += taken;
        }
        tot[p] = all;
    }
}

__global__ void k_ent_fill(int nsw, bool forward, const int32_t *order, const int32_t *salias, const double *x,
                           const double *y, const double *z, const double *frame, const uint8_t *list_cnt,
                           const uint8_t *list_ent, const int32_t *slot_nbr, const int32_t *off, SweepEntry *ent,
                           uint32_t *need, int *too_many) {
    GRID_STRIDE(t, (size_t)nsw) {
        const int p = order[t];
        const double *t1 = frame + 9 * (size_t)p, *t2 = t1 + 3, *nn = t1 + 6;
        int at = off[p];
        uint32_t nd = 0;
        for (int d = 0; d < NDIR; ++d) {
            const int c = list_cnt[(size_t)p * NDIR + d];
            for (int j = 0; j < c; ++j) {
                const int s = list_ent[((size_t)p * NDIR + d) * LIST_STRIDE + j];
                const int k = slot_nbr[(size_t)p * MAX_SLOTS + s];
                if (!(forward ? salias[k] < salias[p] : salias[k] > salias[p])) continue;
                const double delx = x[k] - x[p], dely = y[k] - y[p], delz = z[k] - z[p];
                const double dels = delx * t1[0] + dely * t1[1] + delz * t1[2];
                const double delt = delx * t2[0] + dely * t2[1] + delz * t2[2];
                const double deln = delx * nn[0] + dely * nn[1] + delz * nn[2];
                const double w = 1.0;
                SweepEntry &e = ent[at++];
                e.k = k;
                e.pad = d | (s << 8);
                e.w[0] = dels * w;
                e.w[1] = delt * w;
                e.w[2] = deln * w;
                nd |= 1u << s;
            }
        }
        need[p] = nd;
        if (at - off[p] > SWEEP_MAX_ENTRIES) atomicExch(too_many, 1);
    }
}

// levels by Kahn's layering over the sweep terms whose producer is swept
__global__ void k_dep_count(int nsw, const int32_t *order, const int32_t *off, const SweepEntry *ent,
                            const uint8_t *swept, int32_t *indeg, int32_t *rcnt) {
    GRID_STRIDE(t, (size_t)nsw) {
        const int p = order[t];
        int c = 0;
        for (int e = off[p]; e < off[p + 1]; ++e) {
            const int k = ent[e].k;
            if (!swept[k]) continue;
            ++c;
            atomicAdd(&rcnt[k], 1);
        }
        indeg[p] = c;
    }
}

__global__ void k_dep_fill(int nsw, const int32_t *order, const int32_t *off, const SweepEntry *ent,
                           const uint8_t *swept, const int32_t *roff, int32_t *rcur, int32_t *rlist) {
    GRID_STRIDE(t, (size_t)nsw) {
        const int p = order[t];
        for (int e = off[p]; e < off[p + 1]; ++e) {
            const int k = ent[e].k;
            if (swept[k]) rlist[roff[k] + atomicAdd(&rcur[k], 1)] = p;
        }
    }
}

__global__ void k_level_keys(int nsw, const int32_t *order, const int32_t *level, uint32_t *key, int32_t *hist,
                             int *cycle) {
    GRID_STRIDE(t, (size_t)nsw) {
        const int lv = level[order[t]];
        if (lv < 0) {
            atomicExch(cycle, 1);
            key[t] = 0;
            continue;
        }
        key[t] = (uint32_t)lv;
        atomicAdd(&hist[lv], 1);
    }
}

// Kahn's layering in one block: the frontier of level L (count0[0] points
// in front, from k_lv_roots) releases the dependents whose last producer it
// holds into level L+1; a warp takes a frontier point and its lanes its
// dependents.  The loop ends when a level releases nothing; it runs at most
// nsw levels.
__global__ void __launch_bounds__(1024) k_levels_block(int nsw, int32_t *front, int32_t *next, const int32_t *count0,
                                                       const int32_t *roff, const int32_t *rlist, int32_t *indeg,
                                                       int32_t *level) {
    __shared__ int m, m_next;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    if (threadIdx.x == 0) {
        m = count0[0];
        m_next = 0;
    }
    __syncthreads();
    for (int L = 0; L < nsw && m > 0; ++L) {
        for (int f = warp; f < m; f += warps) {
            const int p = front[f];
            const int e1 = roff[p + 1];
            for (int e = roff[p] + lane; e < e1; e += 32) {
                const int q = rlist[e];
                if (atomicSub(&indeg[q], 1) == 1) {
                    level[q] = L + 1;
                    next[atomicAdd(&m_next, 1)] = q;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            m = m_next;
            m_next = 0;
        }
        int32_t *t = front;
        front = next;
        next = t;
        __syncthreads();
    }
}

// a point's dependencies of the deepest level, in entry order (count, fill)
__global__ void k_cand(int nsw, const int32_t *order, const int32_t *off, const SweepEntry *ent,
                       const uint8_t *swept, const int32_t *level, const int32_t *coff, int32_t *cnt_or_cand,
                       bool fill) {
    GRID_STRIDE(t, (size_t)nsw) {
        const int p = order[t];
        int best = -1;
        for (int e = off[p]; e < off[p + 1]; ++e)
            if (swept[ent[e].k]) best = max(best, level[ent[e].k]);
        int c = 0;
        for (int e = off[p]; e < off[p + 1]; ++e) {
            const int k = ent[e].k;
            if (!swept[k] || level[k] != best) continue;
            if (fill) cnt_or_cand[coff[p] + c] = k;
            ++c;
        }
        if (!fill) cnt_or_cand[p] = c;
    }
}

// where each term's producer increment comes from (chain bits of the
// entries) and which points publish; terms[0..2] ring, same warp, cross warp
__global__ void k_chain_mark(int nsw, const int32_t *lpts, const int32_t *off, SweepEntry *ent,
                             const uint8_t *swept, const uint8_t *shared, const int32_t *owner, const int32_t *pos,
                             uint8_t *publish, unsigned long long *terms) {
    unsigned long long ring = 0, local = 0, cross = 0;
    GRID_STRIDE(t, (size_t)nsw) {
        const int p = lpts[t];
        const bool sh = shared[p] != 0;
        for (int e = off[p]; e < off[p + 1]; ++e) {
            SweepEntry &E = ent[e];
            E.pad &= ~ENT_CHAIN_BITS;
            if (E.pad & (ENT_COPY | ENT_OLD)) continue;
            const int k = E.k;
            if (!swept[k]) continue;
            const bool same = owner[k] == owner[p];
            if (!sh) continue;
            if (same && pos[p] - pos[k] <= CHAIN_RING) {
                E.pad |= ENT_RING | ((pos[k] % CHAIN_RING) << ENT_RING_SHIFT);
                ++ring;
            } else {
                publish[k] = 1;
                if (same) ++local;
                else ++cross;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        ring += __shfl_down_sync(0xffffffffu, ring, o);
        local += __shfl_down_sync(0xffffffffu, local, o);
        cross += __shfl_down_sync(0xffffffffu, cross, o);
    }
    if ((threadIdx.x & 31) == 0 && (ring | local | cross)) {
        atomicAdd(&terms[0], ring);
        atomicAdd(&terms[1], local);
        atomicAdd(&terms[2], cross);
    }
}

__global__ void k_chain_items(int m, const int32_t *pts, const int32_t *off, const uint8_t *cnt, const int8_t *cls,
                              const uint8_t *shared, const uint8_t *publish, const int32_t *g0_of, ChainItem *items) {
    GRID_STRIDE(t, (size_t)m) {
        const int p = pts[t];
        ChainItem it;
        it.p = p;
        it.off = off[p];
        it.cnt = 0;
        for (int e = 0; e < NDIR; ++e) it.cnt |= (uint32_t)cnt[(size_t)p * NDIR + e] << (5 * e);
        it.info = (cls[p] == CLS_WALL ? CI_WALL : 0u) | (shared[p] ? CI_SHARED : 0u) |
                  (publish[p] ? CI_PUBLISH : 0u) | (cls[p] == CLS_SUPERSONIC ? CI_COPY : 0u) |
                  (cls[p] == CLS_OUTER ? CI_OUTER : 0u);
        if (g0_of[p] >= 0) it.info |= CI_G0 | ((uint32_t)g0_of[p] << CI_G0_SHIFT);
        items[t] = it;
    }
}

__global__ void k_positions(int warps, const int32_t *ptr, const int32_t *pts, int32_t *pos) {
    GRID_STRIDE(t, (size_t)warps) {
        for (int i = ptr[t]; i < ptr[t + 1]; ++i) pos[pts[i]] = i - ptr[t];
    }
}

// consumers in the shared frame and the phase-A (k_g0) candidates, by
// logical index
__global__ void k_shared_g0(int n, const int32_t *perm, const uint8_t *swept, const int8_t *scls, int shared_frame,
                            uint8_t *shared, int *g0_flag) {
    GRID_STRIDE(t, (size_t)n) {
        const int p = map_id(perm, (int)t);
        const uint8_t sh = (swept[p] && scls[p] == CLS_INTERIOR && shared_frame) ? 1 : 0;
        shared[p] = sh;
        g0_flag[t] = (swept[p] && !sh && scls[p] != CLS_SUPERSONIC) ? 1 : 0;
    }
}

__global__ void k_g0_emit(int n, const int32_t *perm, const int *flag, const int *pos, int32_t *g0_pts,
                          int32_t *g0_of) {
    GRID_STRIDE(t, (size_t)n) {
        if (!flag[t]) continue;
        const int p = map_id(perm, (int)t);
        g0_pts[pos[t]] = p;
        if (g0_of) g0_of[p] = pos[t];
    }
}

// the fused flux kernel's visiting order: keys as build_pre_order's, sorted
// stably (ties in storage index order)
__global__ void k_pre_keys(int n, const uint8_t *swept, const int32_t *level, uint32_t *key, int32_t *idx) {
    GRID_STRIDE(t, (size_t)n) {
        key[t] = swept[t] ? 2u * (uint32_t)level[t] + 1u : 0xffffffffu;
        idx[t] = (int32_t)t;
    }
}

__global__ void k_pre_min(int nsw, const int32_t *order, const int32_t *off, const SweepEntry *ent,
                          const uint8_t *swept, const int32_t *level, uint32_t *key) {
    GRID_STRIDE(t, (size_t)nsw) {
        const int p = order[t];
        for (int e = off[p]; e < off[p + 1]; ++e) {
            if (ent[e].pad & (ENT_COPY | ENT_OLD)) continue;
            const int k = ent[e].k;
            if (!swept[k]) atomicMin(&key[k], 2u * (uint32_t)level[p]);
        }
    }
}

}  // namespace

#define DS_TMP(ptr, count)                                                              \
    do {                                                                                \
        cudaError_t e_ = tmp.alloc(&(ptr), (count));                                    \
        if (e_ != cudaSuccess) {                                                        \
            err = std::string("device set-up scratch: ") + cudaGetErrorString(e_);      \
            return e_ == cudaErrorMemoryAllocation ? MFCFD_ERR_NOMEM : MFCFD_ERR_CUDA;   \
        }                                                                               \
    } while (0)

#define DS_KEEP(ptr, count)                                                             \
    do {                                                                                \
        void *v_ = nullptr;                                                             \
        const size_t c_ = (size_t)(count);                                              \
        if (int rc_ = alloc(&v_, sizeof(*(ptr)) * (c_ > 0 ? c_ : 1))) {                 \
            if (err.empty()) err = "device memory allocation failed";                  \
            return rc_;                                                                 \
        }                                                                               \
        (ptr) = static_cast<std::remove_reference_t<decltype(ptr)>>(v_);                \
    } while (0)

bool device_setup_supported(const mfcfd_params &P, const Topology &T) {
    return P.device >= 0 && P.sweep_variant == MFCFD_SWEEPS_ALIAS && P.power == 0.0 && T.ss_inlet_idx.empty() &&
           T.ss_outlet_idx.empty() && T.n > 0 &&
           (size_t)T.n * MAX_CONN < 0x7fffffffull;
}

namespace {

// stable sort of (key, value) pairs by key on the device
template <typename K>
int sort_pairs(const K *key_in, K *key_out, const int32_t *val_in, int32_t *val_out, int m, cudaStream_t s,
               DevBufs &tmp, std::string &err) {
    if (m <= 0) return MFCFD_OK;
    size_t bytes = 0;
    const int bits = 8 * (int)sizeof(K);
    PREP_CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, key_in, key_out, val_in, val_out, m, 0, bits, s));
    uint8_t *scratch = nullptr;
    DS_TMP(scratch, bytes);
    PREP_CK(cub::DeviceRadixSort::SortPairs(scratch, bytes, key_in, key_out, val_in, val_out, m, 0, bits, s));
    return MFCFD_OK;
}

// the bits of v (21 of them) spread to every third bit, as morton_order's
__device__ __forceinline__ uint64_t dev_spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

struct Box {
    double lo[3], scale[3];
};

// morton_order's keys (the same quantisation), with the point index as value
__global__ void k_morton_keys(int n, const double *x, const double *y, const double *z, Box b, uint64_t *key,
                              int32_t *idx) {
    GRID_STRIDE(t, (size_t)n) {
        const double v[3] = {x[t], y[t], z[t]};
        uint64_t q[3];
        for (int a = 0; a < 3; ++a) {
            double u = (v[a] - b.lo[a]) * b.scale[a];
            u = u < 0.0 ? 0.0 : (u > 2097151.0 ? 2097151.0 : u);
            q[a] = (uint64_t)u;
        }
        key[t] = dev_spread3(q[0]) | (dev_spread3(q[1]) << 1) | (dev_spread3(q[2]) << 2);
        idx[t] = (int32_t)t;
    }
}

__global__ void k_invert(int n, const int32_t *inv, int32_t *perm) {
    GRID_STRIDE(t, (size_t)n) perm[inv[t]] = (int32_t)t;
}

template <typename V>
__global__ void k_scatter(int n, const int32_t *perm, const V *src, V *dst) {
    GRID_STRIDE(t, (size_t)n) dst[perm ? perm[t] : (int32_t)t] = src[t];
}

template <typename V>
int to_host(std::vector<V> &dst, const V *src, size_t count, cudaStream_t s, std::string &err) {
    dst.resize(count);
    if (count) PREP_CK(cudaMemcpyAsync(dst.data(), src, sizeof(V) * count, cudaMemcpyDeviceToHost, s));
    PREP_CK(cudaStreamSynchronize(s));
    return MFCFD_OK;
}

__global__ void k_g0_of(int m, const int32_t *g0_pts, int32_t *g0_of) {
    GRID_STRIDE(t, (size_t)m) g0_of[g0_pts[t]] = (int32_t)t;
}

}  // namespace

int device_setup(int device, const mfcfd_params &P, Topology &T, const double *x, const double *y,
                 const double *z, const double *tan1, const double *tan2, const double *nor, const int32_t *nbhs,
                 const int32_t *conn, const std::vector<double> &eps2, cudaStream_t s, const DevAlloc &alloc,
                 DevCloud &d, DevTopology &dt, std::string &err) {
    const int n = T.n, cap = T.cap;
    const size_t n3 = 3 * (size_t)n;
    const bool chains = P.sweep_mode == MFCFD_SWEEP_CHAINS;
    DevBufs tmp(s);
    // ---- the cloud, in the reference's order, and the permutation
    double *Lx, *Ly, *Lz, *Lt1, *Lt2, *Ln;
    int32_t *Lnb, *Lconn, *perm = nullptr, *inv = nullptr;
    int8_t *Lcls;
    DS_TMP(Lx, n); DS_TMP(Ly, n); DS_TMP(Lz, n);
    DS_TMP(Lt1, n3); DS_TMP(Lt2, n3); DS_TMP(Ln, n3);
    DS_TMP(Lnb, n); DS_TMP(Lconn, (size_t)n * MAX_CONN); DS_TMP(Lcls, n);
    PREP_CK(cudaMemcpyAsync(Lx, x, 8 * (size_t)n, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(Ly, y, 8 * (size_t)n, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(Lz, z, 8 * (size_t)n, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(Lt1, tan1, 8 * n3, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(Lt2, tan2, 8 * n3, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(Ln, nor, 8 * n3, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(Lnb, nbhs, 4 * (size_t)n, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(Lconn, conn, 4 * (size_t)n * MAX_CONN, cudaMemcpyHostToDevice, s));
    PREP_CK(cudaMemcpyAsync(Lcls, T.cls.data(), (size_t)n, cudaMemcpyHostToDevice, s));
    const int g = grid_for(device, (size_t)n);
    T.perm.clear();
    T.inv.clear();
    if (P.storage_order == MFCFD_ORDER_MORTON && n > 1) {
        // morton_order on the device: the bounding box (exact minima and
        // maxima) on the host, the keys and a stable sort on the device
        Box b;
        double hi[3] = {x[0], y[0], z[0]};
        b.lo[0] = x[0]; b.lo[1] = y[0]; b.lo[2] = z[0];
        for (int i = 1; i < n; ++i) {
            const double v[3] = {x[i], y[i], z[i]};
            for (int a = 0; a < 3; ++a) {
                b.lo[a] = std::min(b.lo[a], v[a]);
                hi[a] = std::max(hi[a], v[a]);
            }
        }
        for (int a = 0; a < 3; ++a) b.scale[a] = hi[a] > b.lo[a] ? 2097151.0 / (hi[a] - b.lo[a]) : 0.0;
        uint64_t *key, *key_sorted;
        int32_t *idx;
        DS_TMP(key, n); DS_TMP(key_sorted, n); DS_TMP(idx, n);
        DS_TMP(perm, n); DS_TMP(inv, n);
        k_morton_keys<<<g, PREP_THREADS, 0, s>>>(n, Lx, Ly, Lz, b, key, idx);
        if (int rc = sort_pairs(key, key_sorted, idx, inv, n, s, tmp, err)) return rc;
        k_invert<<<g, PREP_THREADS, 0, s>>>(n, inv, perm);
        PREP_CK(cudaGetLastError());
        if (int rc = to_host(T.perm, perm, (size_t)n, s, err)) return rc;
        if (int rc = to_host(T.inv, inv, (size_t)n, s, err)) return rc;
    }
    int *d_sums, *d_total, *flag, *fpos;
    DS_TMP(d_sums, ((size_t)n + 1 + 1023) / 1024 + 1); DS_TMP(d_total, 1);
    DS_TMP(flag, (size_t)n + 1); DS_TMP(fpos, (size_t)n + 1);
    auto scan = [&](const int *in, int *out, int len, int *total) -> int {
        if (int rc = exclusive_scan(in, out, len, d_sums, d_total, s, err)) return rc;
        int v = 0;
        PREP_CK(cudaMemcpyAsync(&v, d_total, sizeof(int), cudaMemcpyDeviceToHost, s));
        PREP_CK(cudaStreamSynchronize(s));
        *total = v;
        return MFCFD_OK;
    };

    // ---- storage-order cloud
    double *sx, *sy, *sz, *frame;
    int8_t *scls;
    int32_t *snb, *sconn;
    DS_KEEP(sx, n); DS_KEEP(sy, n); DS_KEEP(sz, n); DS_KEEP(frame, 9 * (size_t)n);
    DS_KEEP(scls, n); DS_KEEP(snb, n); DS_KEEP(sconn, (size_t)n * MAX_CONN);
    k_stage_cloud<<<g, PREP_THREADS, 0, s>>>(n, perm, Lx, Ly, Lz, Lt1, Lt2, Ln, Lcls, Lnb, Lconn, sx, sy, sz, frame,
                                             scls, snb, sconn);
    PREP_CK(cudaGetLastError());
    d.x = sx; d.y = sy; d.z = sz; d.frame = frame; d.cls = scls; d.nbhs = snb; d.conn = sconn;

    // ---- split stencils (generate_connectivity.f90:38-246), the reference's storage
    SplitPtrs sp;
    const size_t flat = (size_t)n * cap + 64;
    for (int k = 0; k < NDIR; ++k) {
        DS_KEEP(dt.split[k], flat);
        PREP_CK(cudaMemsetAsync(dt.split[k], 0, 4 * flat, s));
        sp.p[k] = dt.split[k];
    }
    DS_KEEP(dt.split_cnt, (size_t)NDIR * n);
    int *over;
    DS_TMP(over, 1);
    PREP_CK(cudaMemsetAsync(over, 0, sizeof(int), s));
    k_split_own<<<g, PREP_THREADS, 0, s>>>(n, cap, Lcls, Lx, Ly, Lz, Lt1, Lt2, Ln, Lnb, Lconn, sp, dt.split_cnt, over);
    PREP_CK(cudaGetLastError());
    int h_over = 0;
    PREP_CK(cudaMemcpyAsync(&h_over, over, sizeof(int), cudaMemcpyDeviceToHost, s));
    PREP_CK(cudaStreamSynchronize(s));
    dt.split_overflows = 0;
    if (h_over) {
        // spilled entries land in the next points' storage in the
        // reference's visiting order: resolved on the host from the counts
        std::vector<int32_t> hc;
        if (int rc = to_host(hc, dt.split_cnt, (size_t)NDIR * n, s, err)) return rc;
        const int32_t *cnt[NDIR];
        for (int k = 0; k < NDIR; ++k) {
            cnt[k] = hc.data() + (size_t)k * n;
            for (int i = 0; i < n; ++i) dt.split_overflows += std::max(0, cnt[k][i] - cap);
        }
        std::vector<SpillWrite> w;
        split_spill_writes(T, x, y, z, tan1, tan2, nor, nbhs, conn, cnt, w);
        const int m = (int)w.size();
        if (m > 0) {
            std::vector<int> wd(m);
            std::vector<long long> wat(m);
            std::vector<int32_t> wv(m);
            for (int j = 0; j < m; ++j) { wd[j] = w[j].d; wat[j] = (long long)w[j].at; wv[j] = w[j].value; }
            int *dd; long long *dat; int32_t *dv;
            DS_TMP(dd, m); DS_TMP(dat, m); DS_TMP(dv, m);
            PREP_CK(cudaMemcpyAsync(dd, wd.data(), sizeof(int) * m, cudaMemcpyHostToDevice, s));
            PREP_CK(cudaMemcpyAsync(dat, wat.data(), sizeof(long long) * m, cudaMemcpyHostToDevice, s));
            PREP_CK(cudaMemcpyAsync(dv, wv.data(), sizeof(int32_t) * m, cudaMemcpyHostToDevice, s));
            k_spill_apply<<<grid_for(device, m), PREP_THREADS, 0, s>>>(m, dd, dat, dv, sp);
            PREP_CK(cudaGetLastError());
            PREP_CK(cudaStreamSynchronize(s));   // the host vectors go out of scope
        }
    }

    // ---- alias breadth-first search (implicit_aliasing.f90:21-42)
    DS_KEEP(dt.alias, n);
    DS_KEEP(dt.pwa, n);
    if (int rc = alias_search(device, n, Lnb, Lconn, dt.alias, dt.pwa, s, err)) return rc;
    int32_t *salias;
    DS_TMP(salias, n);
    k_alias_storage<<<g, PREP_THREADS, 0, s>>>(n, perm, dt.alias, salias);

    // ---- effective lists and neighbour slots
    int32_t *slot_nbr;
    uint8_t *nslot, *slot_mask, *list_cnt, *list_ent, *code;
    DS_KEEP(slot_nbr, (size_t)n * MAX_SLOTS); DS_KEEP(nslot, n); DS_KEEP(slot_mask, (size_t)n * MAX_SLOTS);
    DS_KEEP(list_cnt, (size_t)n * NDIR); DS_KEEP(list_ent, (size_t)n * NDIR * LIST_STRIDE);
    DS_TMP(code, n);
    int *bad;
    DS_TMP(bad, 1);
    PREP_CK(cudaMemsetAsync(bad, 0x7f, sizeof(int), s));
    k_slots<<<g, PREP_THREADS, 0, s>>>(n, cap, perm, inv, Lcls, Lnb, Lconn, sp, dt.split_cnt, slot_nbr, nslot,
                                       slot_mask, list_cnt, list_ent, code, bad);
    PREP_CK(cudaGetLastError());
    int h_bad = 0;
    PREP_CK(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    PREP_CK(cudaStreamSynchronize(s));
    if (h_bad != 0x7f7f7f7f) {
        uint8_t c = 0;
        PREP_CK(cudaMemcpyAsync(&c, code + h_bad, 1, cudaMemcpyDeviceToHost, s));
        PREP_CK(cudaStreamSynchronize(s));
        const std::string at = std::to_string(h_bad + 1);
        if (c == SLOT_ZERO) err = "split list of point " + at + " names point 0";
        else if (c == SLOT_LONG) err = "split list longer than 27 at point " + at;
        else err = "more than 32 distinct stencil neighbours at point " + at;
        return MFCFD_ERR_STENCIL;
    }
    d.slot_nbr = slot_nbr; d.nslot = nslot; d.slot_mask = slot_mask; d.list_cnt = list_cnt; d.list_ent = list_ent;
    d.sweep_slot_mask = slot_mask;   // the alias driver's sweep terms use the same lists

    // ---- geometry per (point, list) and the limiter's epsilon
    double *geo, *e2;
    DS_KEEP(geo, (size_t)n * GEO_STRIDE);
    k_geo<<<g, PREP_THREADS, 0, s>>>(n, sx, sy, sz, frame, list_cnt, list_ent, slot_nbr, geo);
    PREP_CK(cudaGetLastError());
    DS_KEEP(e2, n);
    {
        double *le2;
        DS_TMP(le2, n);
        PREP_CK(cudaMemcpyAsync(le2, eps2.data(), 8 * (size_t)n, cudaMemcpyHostToDevice, s));
        k_scatter<<<g, PREP_THREADS, 0, s>>>(n, perm, le2, e2);
        PREP_CK(cudaGetLastError());
    }
    d.geo = geo; d.eps2 = e2; d.wq = nullptr; d.wf = nullptr; d.outer_delt = nullptr;

    // ---- sweep orders (implicit_forward_and_reverse_sweeps.f90:26-84)
    uint8_t *swept;
    DS_KEEP(swept, n);
    PREP_CK(cudaMemsetAsync(swept, 0, (size_t)n, s));
    int nsw = 0;
    int32_t *order[2];
    DS_TMP(order[0], n); DS_TMP(order[1], n);
    k_swept_flags<<<g, PREP_THREADS, 0, s>>>(n, dt.pwa, Lcls, flag);
    if (int rc = scan(flag, fpos, n, &nsw)) return rc;
    k_swept_emit<<<g, PREP_THREADS, 0, s>>>(n, dt.pwa, perm, flag, fpos, order[0], swept);
    if (nsw > 0) k_reverse<<<grid_for(device, nsw), PREP_THREADS, 0, s>>>(nsw, order[0], order[1]);
    PREP_CK(cudaGetLastError());
    d.swept = swept;
    d.n_swept = nsw;

    // ---- per direction: terms, levels, level-major points
    const int gs = grid_for(device, (size_t)std::max(nsw, 1));
    dt.max_width = 0;
    uint8_t *cnt_dir[2];
    int32_t *off_dir[2], *lpts_dir[2], *lptr_dir[2];
    uint32_t *need_dir[2], *old_dir[2];
    SweepEntry *ent_dir[2];
    int nlev[2] = {0, 0};
    for (int dir = 0; dir < 2; ++dir) {
        const bool fwd = dir == 0;
        DS_KEEP(cnt_dir[dir], (size_t)n * NDIR);
        PREP_CK(cudaMemsetAsync(cnt_dir[dir], 0, (size_t)n * NDIR, s));
        DS_KEEP(off_dir[dir], (size_t)n + 1);
        PREP_CK(cudaMemsetAsync(flag, 0, 4 * ((size_t)n + 1), s));
        if (nsw > 0)
            k_ent_count<<<gs, PREP_THREADS, 0, s>>>(nsw, fwd, order[dir], salias, list_cnt, list_ent, slot_nbr,
                                                    cnt_dir[dir], flag);
        int ne = 0;
        if (int rc = scan(flag, off_dir[dir], n + 1, &ne)) return rc;
        DS_KEEP(ent_dir[dir], ne);
        DS_KEEP(need_dir[dir], n);
        DS_KEEP(old_dir[dir], n);
        PREP_CK(cudaMemsetAsync(need_dir[dir], 0, 4 * (size_t)n, s));
        PREP_CK(cudaMemsetAsync(old_dir[dir], 0, 4 * (size_t)n, s));
        int *too_many;
        DS_TMP(too_many, 1);
        PREP_CK(cudaMemsetAsync(too_many, 0, sizeof(int), s));
        if (nsw > 0)
            k_ent_fill<<<gs, PREP_THREADS, 0, s>>>(nsw, fwd, order[dir], salias, sx, sy, sz, frame, list_cnt,
                                                   list_ent, slot_nbr, off_dir[dir], ent_dir[dir], need_dir[dir],
                                                   too_many);
        PREP_CK(cudaGetLastError());
        int h_many = 0;
        PREP_CK(cudaMemcpyAsync(&h_many, too_many, sizeof(int), cudaMemcpyDeviceToHost, s));
        PREP_CK(cudaStreamSynchronize(s));
        if (h_many) {
            err = "a point reads more than " + std::to_string(SWEEP_MAX_ENTRIES) + " sweep terms";
            return MFCFD_ERR_STENCIL;
        }
        dt.n_ent[dir] = ne;

        // levels: the longest path over swept producers (Kahn's layering)
        DS_KEEP(dt.level[dir], n);
        PREP_CK(cudaMemsetAsync(dt.level[dir], 0xff, 4 * (size_t)n, s));
        DS_KEEP(lpts_dir[dir], nsw);
        std::vector<int32_t> hist;
        if (nsw > 0) {
            int32_t *indeg, *rcnt, *roff, *rcur, *rlist, *fa, *fb, *count, *hcnt;
            uint32_t *key, *key_sorted;
            int *cycle;
            DS_TMP(indeg, n); DS_TMP(rcnt, (size_t)n + 1); DS_TMP(roff, (size_t)n + 1); DS_TMP(rcur, n);
            DS_TMP(rlist, ne); DS_TMP(fa, nsw); DS_TMP(fb, nsw); DS_TMP(count, (size_t)nsw + 2);
            DS_TMP(hcnt, (size_t)nsw + 1); DS_TMP(key, nsw); DS_TMP(key_sorted, nsw); DS_TMP(cycle, 1);
            PREP_CK(cudaMemsetAsync(rcnt, 0, 4 * ((size_t)n + 1), s));
            PREP_CK(cudaMemsetAsync(rcur, 0, 4 * (size_t)n, s));
            PREP_CK(cudaMemsetAsync(count, 0, 4 * ((size_t)nsw + 2), s));
            PREP_CK(cudaMemsetAsync(hcnt, 0, 4 * ((size_t)nsw + 1), s));
            PREP_CK(cudaMemsetAsync(cycle, 0, sizeof(int), s));
            k_dep_count<<<gs, PREP_THREADS, 0, s>>>(nsw, order[dir], off_dir[dir], ent_dir[dir], swept, indeg, rcnt);
            int ndep = 0;
            if (int rc = scan(rcnt, roff, n + 1, &ndep)) return rc;
            k_dep_fill<<<gs, PREP_THREADS, 0, s>>>(nsw, order[dir], off_dir[dir], ent_dir[dir], swept, roff, rcur,
                                                   rlist);
            // one thread per point of the order (k_lv_roots has no grid-stride loop)
            k_lv_roots<<<(nsw + PREP_THREADS - 1) / PREP_THREADS, PREP_THREADS, 0, s>>>(order[dir], nsw, indeg,
                                                                                     dt.level[dir], fa, count);
            // every level in one block: a barrier per level instead of a launch
            k_levels_block<<<1, 1024, 0, s>>>(nsw, fa, fb, count, roff, rlist, indeg, dt.level[dir]);
            PREP_CK(cudaGetLastError());
            k_level_keys<<<gs, PREP_THREADS, 0, s>>>(nsw, order[dir], dt.level[dir], key, hcnt, cycle);
            PREP_CK(cudaGetLastError());
            int h_cycle = 0;
            PREP_CK(cudaMemcpyAsync(&h_cycle, cycle, sizeof(int), cudaMemcpyDeviceToHost, s));
            PREP_CK(cudaStreamSynchronize(s));
            if (h_cycle) {
                err = "sweep dependencies contain a cycle";
                return MFCFD_ERR_STENCIL;
            }
            // points of each level in the sweep's order
            if (int rc = sort_pairs(key, key_sorted, order[dir], lpts_dir[dir], nsw, s, tmp, err)) return rc;
            if (int rc = to_host(hist, hcnt, (size_t)nsw + 1, s, err)) return rc;
        }
        int nl = 0;
        for (int l = 0; l < (int)hist.size(); ++l)
            if (hist[l] > 0) nl = l + 1;
        std::vector<int32_t> &lptr = dt.lvl_ptr[dir];
        lptr.assign(nl + 1, 0);
        for (int l = 0; l < nl; ++l) {
            lptr[l + 1] = lptr[l] + hist[l];
            dt.max_width = std::max(dt.max_width, hist[l]);
        }
        DS_KEEP(lptr_dir[dir], nl + 1);
        PREP_CK(cudaMemcpyAsync(lptr_dir[dir], lptr.data(), 4 * ((size_t)nl + 1), cudaMemcpyHostToDevice, s));
        PREP_CK(cudaStreamSynchronize(s));
        nlev[dir] = nl;

        // the chain schedule's inputs on the host: levels, level-major
        // points, each point's deepest dependencies in entry order
        if (chains) {
            if (int rc = to_host(dt.h_level[dir], dt.level[dir], (size_t)n, s, err)) return rc;
            if (int rc = to_host(dt.h_lpts[dir], lpts_dir[dir], (size_t)nsw, s, err)) return rc;
            int32_t *ccnt, *coff, *cand;
            DS_TMP(ccnt, (size_t)n + 1); DS_TMP(coff, (size_t)n + 1);
            PREP_CK(cudaMemsetAsync(ccnt, 0, 4 * ((size_t)n + 1), s));
            if (nsw > 0)
                k_cand<<<gs, PREP_THREADS, 0, s>>>(nsw, order[dir], off_dir[dir], ent_dir[dir], swept, dt.level[dir],
                                                   nullptr, ccnt, false);
            int nc = 0;
            if (int rc = scan(ccnt, coff, n + 1, &nc)) return rc;
            DS_TMP(cand, nc);
            if (nsw > 0)
                k_cand<<<gs, PREP_THREADS, 0, s>>>(nsw, order[dir], off_dir[dir], ent_dir[dir], swept, dt.level[dir],
                                                   coff, cand, true);
            PREP_CK(cudaGetLastError());
            if (int rc = to_host(dt.h_coff[dir], coff, (size_t)n + 1, s, err)) return rc;
            if (int rc = to_host(dt.h_cand[dir], cand, (size_t)nc, s, err)) return rc;
        }
    }
    d.fwd_cnt = cnt_dir[0]; d.bwd_cnt = cnt_dir[1];
    d.fwd_off = off_dir[0]; d.bwd_off = off_dir[1];
    d.fwd_ent = ent_dir[0]; d.bwd_ent = ent_dir[1];
    d.fwd_need = need_dir[0]; d.bwd_need = need_dir[1];
    d.fwd_old = old_dir[0]; d.bwd_old = old_dir[1];
    d.fwd_lvl_pts = lpts_dir[0]; d.bwd_lvl_pts = lpts_dir[1];
    d.fwd_lvl_ptr = lptr_dir[0]; d.bwd_lvl_ptr = lptr_dir[1];
    d.n_fwd_levels = nlev[0];
    d.n_bwd_levels = nlev[1];
    d.max_width = dt.max_width;

    // ---- the shared interior frame (every interior point's frame bit-equal
    // to the first's), its consumers, and the phase-A (k_g0) points
    d.shared_frame = 0;
    if (!T.interior_idx.empty()) {
        const int i0 = T.interior_idx[0];
        bool same = true;
        for (int i : T.interior_idx) {
            if (std::memcmp(tan1 + 3 * (size_t)i, tan1 + 3 * (size_t)i0, 24) ||
                std::memcmp(tan2 + 3 * (size_t)i, tan2 + 3 * (size_t)i0, 24) ||
                std::memcmp(nor + 3 * (size_t)i, nor + 3 * (size_t)i0, 24)) {
                same = false;
                break;
            }
        }
        if (same) {
            d.shared_frame = 1;
            for (int r = 0; r < 3; ++r) {
                d.frame0[r] = tan1[3 * (size_t)i0 + r];
                d.frame0[3 + r] = tan2[3 * (size_t)i0 + r];
                d.frame0[6 + r] = nor[3 * (size_t)i0 + r];
            }
        }
    }
    if (!d.shared_frame) std::memset(d.frame0, 0, sizeof d.frame0);
    uint8_t *shared;
    DS_KEEP(shared, n);
    k_shared_g0<<<g, PREP_THREADS, 0, s>>>(n, perm, swept, scls, d.shared_frame, shared, flag);
    int ng0 = 0;
    if (int rc = scan(flag, fpos, n, &ng0)) return rc;
    d.consumer_shared = shared;
    dt.g0_pts.clear();
    d.g0_pts = nullptr;
    d.n_g0 = 0;
    if (ng0 > std::max(4096, n / 8) || ng0 >= (1 << 24)) ng0 = 0;
    if (ng0 > 0) {
        int32_t *g0p;
        DS_TMP(g0p, ng0);
        k_g0_emit<<<g, PREP_THREADS, 0, s>>>(n, perm, flag, fpos, g0p, nullptr);
        PREP_CK(cudaGetLastError());
        if (int rc = to_host(dt.g0_pts, g0p, (size_t)ng0, s, err)) return rc;
        if (chains) {
            int32_t *kept;
            DS_KEEP(kept, ng0);
            PREP_CK(cudaMemcpyAsync(kept, g0p, 4 * (size_t)ng0, cudaMemcpyDeviceToDevice, s));
            d.g0_pts = kept;
            d.n_g0 = ng0;
        }
    }

    // ---- the residual's order: wall, then interior points, each in the
    // reference's index order (state_update_implicit.f90:28-61)
    {
        std::vector<int32_t> ro;
        ro.reserve(T.wall_idx.size() + T.interior_idx.size());
        for (int i : T.wall_idx) ro.push_back(T.perm.empty() ? i : T.perm[i]);
        for (int i : T.interior_idx) ro.push_back(T.perm.empty() ? i : T.perm[i]);
        int32_t *r;
        DS_KEEP(r, ro.size());
        if (!ro.empty()) PREP_CK(cudaMemcpyAsync(r, ro.data(), 4 * ro.size(), cudaMemcpyHostToDevice, s));
        PREP_CK(cudaStreamSynchronize(s));
        d.res_order = r;
        d.n_res = (int)ro.size();
        d.n_wall = (int)T.wall_idx.size();
    }

    // ---- the fused flux kernel's visiting order (build_pre_order)
    d.pre_order = nullptr;
    if (chains) {
        uint32_t *key, *key_sorted;
        int32_t *idx, *pre;
        DS_TMP(key, n); DS_TMP(key_sorted, n); DS_TMP(idx, n);
        DS_KEEP(pre, n);
        k_pre_keys<<<g, PREP_THREADS, 0, s>>>(n, swept, dt.level[0], key, idx);
        if (nsw > 0)
            k_pre_min<<<gs, PREP_THREADS, 0, s>>>(nsw, order[0], off_dir[0], ent_dir[0], swept, dt.level[0], key);
        PREP_CK(cudaGetLastError());
        if (int rc = sort_pairs(key, key_sorted, idx, pre, n, s, tmp, err)) return rc;
        d.pre_order = pre;
    }
    PREP_CK(cudaStreamSynchronize(s));
    return MFCFD_OK;
}

int device_chain_schedule(int device, DevTopology &dt, DevCloud &d, int warps, cudaStream_t s,
                          const DevAlloc &alloc, int64_t terms[3], std::string &err) {
    const int n = d.n;
    DevBufs tmp(s);
    terms[0] = terms[1] = terms[2] = 0;
    int32_t *g0_of, *pos;
    uint8_t *publish;
    unsigned long long *dterms;
    DS_TMP(g0_of, n); DS_TMP(pos, n); DS_TMP(publish, n); DS_TMP(dterms, 3);
    PREP_CK(cudaMemsetAsync(g0_of, 0xff, 4 * (size_t)n, s));
    if (d.n_g0 > 0) k_g0_of<<<grid_for(device, d.n_g0), PREP_THREADS, 0, s>>>(d.n_g0, d.g0_pts, g0_of);
    // the two directions' warp assignments are independent: the backward
    // one on a second host thread
    std::vector<int32_t> owners[2];
    std::vector<std::vector<int32_t>> lists_of[2];
    auto assign = [&](int dir) {
        chain_assign(dt.h_lpts[dir].data(), (int)dt.h_lpts[dir].size(), dt.h_level[dir].data(),
                     dt.h_coff[dir].data(), dt.h_cand[dir].data(), n, warps, owners[dir], lists_of[dir]);
    };
    {
        std::thread bwd;
        bool threaded = false;
        if (take_setup_threads(1) == 1) {
            try {
                bwd = std::thread([&] {
                    try {
                        assign(1);
                    } catch (...) {
                        owners[1].clear();
                    }
                });
                threaded = true;
            } catch (...) {
                give_setup_threads(1);
            }
        }
        std::exception_ptr e0;
        try {
            assign(0);
        } catch (...) {
            e0 = std::current_exception();
        }
        if (threaded) {
            bwd.join();
            give_setup_threads(1);
        }
        if (e0) std::rethrow_exception(e0);
        if (!threaded || owners[1].size() != (size_t)n) assign(1);
    }
    for (int dir = 0; dir < 2; ++dir) {
        const int nsw = (int)dt.h_lpts[dir].size();
        const std::vector<int32_t> &owner = owners[dir];
        const std::vector<std::vector<int32_t>> &lists = lists_of[dir];
        std::vector<int32_t> ptr(warps + 1, 0), pts;
        pts.reserve(nsw);
        for (int w = 0; w < warps; ++w) {
            ptr[w] = (int32_t)pts.size();
            pts.insert(pts.end(), lists[w].begin(), lists[w].end());
        }
        ptr[warps] = (int32_t)pts.size();
        int32_t *dptr, *dpts, *down;
        ChainItem *items;
        DS_KEEP(dptr, warps + 1); DS_KEEP(dpts, pts.size()); DS_KEEP(down, n); DS_KEEP(items, pts.size());
        PREP_CK(cudaMemcpyAsync(dptr, ptr.data(), 4 * ptr.size(), cudaMemcpyHostToDevice, s));
        if (!pts.empty()) PREP_CK(cudaMemcpyAsync(dpts, pts.data(), 4 * pts.size(), cudaMemcpyHostToDevice, s));
        PREP_CK(cudaMemcpyAsync(down, owner.data(), 4 * (size_t)n, cudaMemcpyHostToDevice, s));
        PREP_CK(cudaMemsetAsync(pos, 0xff, 4 * (size_t)n, s));
        PREP_CK(cudaMemsetAsync(publish, 0, (size_t)n, s));
        PREP_CK(cudaMemsetAsync(dterms, 0, 3 * sizeof(unsigned long long), s));
        k_positions<<<grid_for(device, warps), PREP_THREADS, 0, s>>>(warps, dptr, dpts, pos);
        const int32_t *lpts = dir == 0 ? d.fwd_lvl_pts : d.bwd_lvl_pts;
        const int32_t *off = dir == 0 ? d.fwd_off : d.bwd_off;
        SweepEntry *ent = const_cast<SweepEntry *>(dir == 0 ? d.fwd_ent : d.bwd_ent);
        const uint8_t *cnt = dir == 0 ? d.fwd_cnt : d.bwd_cnt;
        const int gs = grid_for(device, (size_t)std::max(nsw, 1));
        if (nsw > 0) {
            k_chain_mark<<<gs, PREP_THREADS, 0, s>>>(nsw, lpts, off, ent, d.swept, d.consumer_shared, down, pos,
                                                     publish, dterms);
            k_chain_items<<<gs, PREP_THREADS, 0, s>>>((int)pts.size(), dpts, off, cnt, d.cls, d.consumer_shared,
                                                      publish, g0_of, items);
        }
        PREP_CK(cudaGetLastError());
        unsigned long long h[3] = {0, 0, 0};
        PREP_CK(cudaMemcpyAsync(h, dterms, sizeof h, cudaMemcpyDeviceToHost, s));
        PREP_CK(cudaStreamSynchronize(s));
        for (int k = 0; k < 3; ++k) terms[k] += (int64_t)h[k];
        d.ch_ptr[dir] = dptr;
        d.ch_pts[dir] = dpts;
        d.ch_own[dir] = down;
        d.ch_items[dir] = items;
    }
    d.ch_warps = warps;
    return MFCFD_OK;
}

#undef DS_TMP
#undef DS_KEEP
#undef GRID_STRIDE

}  // namespace mfcfd
