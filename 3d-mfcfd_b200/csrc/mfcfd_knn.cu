/*
 * mfcfd_knn.cu - k nearest neighbours of every point of a cloud
 * (mfcfd_knn), the connectivity a cloud without one needs before the
 * reference's set-up can run (the reference reads conn from its input file,
 * point_preprocessor.f90:30-35; a request server must build it).
 *
 * The answer is defined exactly, so the GPU and the host give the same
 * arrays: the neighbours of point i are the k points j != i with the
 * smallest (d2, j), where d2 = dx*dx + dy*dy + dz*dz with dx = x[j] - x[i]
 * (evaluated in that order, without contraction), listed in that order;
 * min_dist is sqrt(d2) of the first.  Two points at distance 0 are an
 * error.
 *
 * Search structure: the points sorted along a Morton curve, cut into leaves
 * of KNN_LEAF consecutive points, with levels of nodes over KNN_FAN
 * consecutive children, each carrying its points' bounding box.  A query
 * first takes its own leaf, then walks the tree depth first, skipping every
 * node whose box lies farther than its current k-th distance (with a
 * relative margin far above rounding, so no candidate is ever skipped).
 * The walk is one function compiled for both the device (a thread per
 * query) and the host (a pool of threads).
 */
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "mfcfd_internal.h"

namespace mfcfd {
namespace {

constexpr int KNN_LEAF = 32;
constexpr int KNN_FAN = 8;
constexpr int KNN_MAX_LEVELS = 16;
constexpr int KNN_STACK = KNN_MAX_LEVELS * KNN_FAN;
constexpr double KNN_MARGIN = 1.0 + 1e-9;

struct Box6 {
    double lo[3], hi[3];
};

// The tree over the sorted points: level 0 are the leaves (KNN_LEAF points
// each), level l+1 groups KNN_FAN nodes of level l; node b of level l
// covers the sorted points [b * span_l, min(n, (b+1) * span_l)).
struct KnnTree {
    int n = 0, levels = 0;
    int count[KNN_MAX_LEVELS];
    long long span[KNN_MAX_LEVELS];
    const Box6 *box[KNN_MAX_LEVELS];
    const double *sx, *sy, *sz;   // coordinates in sorted order
    const int32_t *id;            // sorted position -> point index
};

__host__ __device__ inline int min_i(int a, int b) { return a < b ? a : b; }

__host__ __device__ inline double box_d2(const Box6 &b, double px, double py, double pz) {
    const double p[3] = {px, py, pz};
    double s = 0.0;
    for (int a = 0; a < 3; ++a) {
        const double d = p[a] < b.lo[a] ? b.lo[a] - p[a] : (p[a] > b.hi[a] ? p[a] - b.hi[a] : 0.0);
        s = s + d * d;
    }
    return s;
}

// insert (d2, j) into the ascending list (bd, bj) of length *m <= k
__host__ __device__ inline void knn_insert(double d2, int j, double *bd, int *bj, int *m, int k) {
    int at = *m;
    if (at == k) {
        if (!(d2 < bd[k - 1] || (d2 == bd[k - 1] && j < bj[k - 1]))) return;
        at = k - 1;
    } else {
        ++*m;
    }
    while (at > 0 && (d2 < bd[at - 1] || (d2 == bd[at - 1] && j < bj[at - 1]))) {
        bd[at] = bd[at - 1];
        bj[at] = bj[at - 1];
        --at;
    }
    bd[at] = d2;
    bj[at] = j;
}

// the k nearest neighbours of sorted point q (bd, bj ascending; returns how
// many were found, < k only when the cloud has fewer than k + 1 points);
// *dup is set when another point coincides with it
__host__ __device__ inline int knn_query(const KnnTree &t, int q, int k, double *bd, int *bj, int *dup) {
    const double px = t.sx[q], py = t.sy[q], pz = t.sz[q];
    const int self = t.id[q];
    int m = 0;
    auto scan_leaf = [&](int leaf) {
        const int a = leaf * KNN_LEAF, b = min_i(t.n, a + KNN_LEAF);
        for (int s = a; s < b; ++s) {
            const int j = t.id[s];
            if (j == self) continue;
            const double dx = t.sx[s] - px, dy = t.sy[s] - py, dz = t.sz[s] - pz;
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 == 0.0) *dup = 1;
            knn_insert(d2, j, bd, bj, &m, k);
        }
    };
    const int own = q / KNN_LEAF;
    scan_leaf(own);
    // depth-first over the tree from the root, nearer children first
    int stack_lvl[KNN_STACK], stack_node[KNN_STACK];
    int sp = 0;
    stack_lvl[sp] = t.levels - 1;
    stack_node[sp] = 0;
    ++sp;
    while (sp > 0) {
        --sp;
        const int l = stack_lvl[sp], b = stack_node[sp];
        const double lim = m == k ? bd[k - 1] * KNN_MARGIN : 1e300;
        if (box_d2(t.box[l][b], px, py, pz) > lim) continue;
        if (l == 0) {
            if (b != own) scan_leaf(b);
            continue;
        }
        // children of b at level l-1, pushed farthest first
        const int c0 = b * KNN_FAN, c1 = min_i(t.count[l - 1], c0 + KNN_FAN);
        double cd[KNN_FAN];
        int ci[KNN_FAN], nc = 0;
        for (int c = c0; c < c1; ++c) {
            const double dd = box_d2(t.box[l - 1][c], px, py, pz);
            if (dd > lim) continue;
            int at = nc++;
            while (at > 0 && cd[at - 1] < dd) {   // descending distance
                cd[at] = cd[at - 1];
                ci[at] = ci[at - 1];
                --at;
            }
            cd[at] = dd;
            ci[at] = c;
        }
        for (int c = 0; c < nc && sp < KNN_STACK; ++c) {
            stack_lvl[sp] = l - 1;
            stack_node[sp] = ci[c];
            ++sp;
        }
    }
    return m;
}


__host__ __device__ inline uint64_t knn_spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__host__ __device__ inline uint64_t knn_key(double x, double y, double z, const double *lo, const double *scale) {
    const double v[3] = {x, y, z};
    uint64_t q[3];
    for (int a = 0; a < 3; ++a) {
        double u = (v[a] - lo[a]) * scale[a];
        u = u < 0.0 ? 0.0 : (u > 2097151.0 ? 2097151.0 : u);
        q[a] = (uint64_t)u;
    }
    return knn_spread3(q[0]) | (knn_spread3(q[1]) << 1) | (knn_spread3(q[2]) << 2);
}

// the box of node b of a level from its range of sorted points (level 0) or
// its children's boxes
__host__ __device__ inline Box6 knn_leaf_box(int b, int n, const double *sx, const double *sy, const double *sz) {
    Box6 r;
    const int a = b * KNN_LEAF, e = min_i(n, a + KNN_LEAF);
    r.lo[0] = r.hi[0] = sx[a];
    r.lo[1] = r.hi[1] = sy[a];
    r.lo[2] = r.hi[2] = sz[a];
    for (int s = a + 1; s < e; ++s) {
        const double v[3] = {sx[s], sy[s], sz[s]};
        for (int k = 0; k < 3; ++k) {
            r.lo[k] = v[k] < r.lo[k] ? v[k] : r.lo[k];
            r.hi[k] = v[k] > r.hi[k] ? v[k] : r.hi[k];
        }
    }
    return r;
}

__host__ __device__ inline Box6 knn_node_box(int b, int nchild, const Box6 *child) {
    const int a = b * KNN_FAN, e = min_i(nchild, a + KNN_FAN);
    Box6 r = child[a];
    for (int c = a + 1; c < e; ++c)
        for (int k = 0; k < 3; ++k) {
            r.lo[k] = child[c].lo[k] < r.lo[k] ? child[c].lo[k] : r.lo[k];
            r.hi[k] = child[c].hi[k] > r.hi[k] ? child[c].hi[k] : r.hi[k];
        }
    return r;
}

// one query's output rows (conn 1-based, zero padded to MAX_CONN)
__host__ __device__ inline void knn_store(const KnnTree &t, int q, int k, int32_t *nbhs, int32_t *conn,
                                          double *min_dist, int *dup, int *short_) {
    double bd[MAX_CONN];
    int bj[MAX_CONN];
    const int m = knn_query(t, q, k, bd, bj, dup);
    const int i = t.id[q];
    if (m < k) *short_ = 1;
    nbhs[i] = m;
    for (int r = 0; r < MAX_CONN; ++r) conn[(size_t)i * MAX_CONN + r] = r < m ? bj[r] + 1 : 0;
    min_dist[i] = m > 0 ? sqrt(bd[0]) : 0.0;
}

__global__ void k_knn_keys(int n, const double *x, const double *y, const double *z, Box6 b, uint64_t *key,
                           int32_t *idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    key[i] = knn_key(x[i], y[i], z[i], b.lo, b.hi);   // hi carries the scale
    idx[i] = i;
}

__global__ void k_knn_gather(int n, const int32_t *id, const double *x, const double *y, const double *z,
                             double *sx, double *sy, double *sz) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    sx[s] = x[id[s]];
    sy[s] = y[id[s]];
    sz[s] = z[id[s]];
}

__global__ void k_knn_leaves(int count, int n, const double *sx, const double *sy, const double *sz, Box6 *box) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < count) box[b] = knn_leaf_box(b, n, sx, sy, sz);
}

__global__ void k_knn_nodes(int count, int nchild, const Box6 *child, Box6 *box) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < count) box[b] = knn_node_box(b, nchild, child);
}

__global__ void k_knn_query(KnnTree t, int k, int32_t *nbhs, int32_t *conn, double *min_dist, int *flags) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= t.n) return;
    int dup = 0, sh = 0;
    knn_store(t, q, k, nbhs, conn, min_dist, &dup, &sh);
    if (dup) atomicExch(&flags[0], 1);
    if (sh) atomicExch(&flags[1], 1);
}

// bounding box and Morton scale over the cloud (exact minima and maxima)
void knn_frame(int n, const double *x, const double *y, const double *z, double lo[3], double scale[3]) {
    double hi[3] = {x[0], y[0], z[0]};
    lo[0] = x[0]; lo[1] = y[0]; lo[2] = z[0];
    for (int i = 1; i < n; ++i) {
        const double v[3] = {x[i], y[i], z[i]};
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], v[a]);
            hi[a] = std::max(hi[a], v[a]);
        }
    }
    for (int a = 0; a < 3; ++a) scale[a] = hi[a] > lo[a] ? 2097151.0 / (hi[a] - lo[a]) : 0.0;
}

int level_counts(int n, int count[KNN_MAX_LEVELS], long long span[KNN_MAX_LEVELS]) {
    int levels = 0;
    long long sp = KNN_LEAF;
    int c = (n + KNN_LEAF - 1) / KNN_LEAF;
    while (true) {
        count[levels] = c;
        span[levels] = sp;
        ++levels;
        if (c == 1 || levels == KNN_MAX_LEVELS) break;
        c = (c + KNN_FAN - 1) / KNN_FAN;
        sp *= KNN_FAN;
    }
    return levels;
}

// stream-ordered scratch, so a search beside running solves does not wait
// for the whole device
struct KnnBufs {
    std::vector<void *> p;
    cudaStream_t s;
    explicit KnnBufs(cudaStream_t st) : s(st) {}
    ~KnnBufs() {
        for (void *v : p) cudaFreeAsync(v, s);
        cudaStreamSynchronize(s);
    }
    template <typename T>
    cudaError_t alloc(T **ptr, size_t count) {
        void *v = nullptr;
        cudaError_t e = cudaMallocAsync(&v, sizeof(T) * (count ? count : 1), s);
        if (e == cudaSuccess) p.push_back(v);
        *ptr = (T *)v;
        return e;
    }
};

#define KNN_CK(call)                                                   \
    do {                                                               \
        cudaError_t e_ = (call);                                       \
        if (e_ != cudaSuccess) {                                       \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);  \
            return e_ == cudaErrorMemoryAllocation ? MFCFD_ERR_NOMEM : MFCFD_ERR_CUDA; \
        }                                                              \
    } while (0)

int knn_device(int device, int n, const double *x, const double *y, const double *z, int k, int32_t *nbhs,
               int32_t *conn, double *min_dist, std::string &err) {
    KNN_CK(cudaSetDevice(device));
    cudaStream_t s = nullptr;
    KNN_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{s};
    KnnBufs b(s);
    double *dx, *dy, *dz, *sx, *sy, *sz, *dmd;
    uint64_t *key, *key2;
    int32_t *idx, *id, *dnb, *dconn;
    int *flags;
    KNN_CK(b.alloc(&dx, n)); KNN_CK(b.alloc(&dy, n)); KNN_CK(b.alloc(&dz, n));
    KNN_CK(b.alloc(&sx, n)); KNN_CK(b.alloc(&sy, n)); KNN_CK(b.alloc(&sz, n));
    KNN_CK(b.alloc(&key, n)); KNN_CK(b.alloc(&key2, n)); KNN_CK(b.alloc(&idx, n)); KNN_CK(b.alloc(&id, n));
    KNN_CK(b.alloc(&dnb, n)); KNN_CK(b.alloc(&dconn, (size_t)n * MAX_CONN)); KNN_CK(b.alloc(&dmd, n));
    KNN_CK(b.alloc(&flags, 2));
    KNN_CK(cudaMemcpyAsync(dx, x, 8 * (size_t)n, cudaMemcpyHostToDevice, s));
    KNN_CK(cudaMemcpyAsync(dy, y, 8 * (size_t)n, cudaMemcpyHostToDevice, s));
    KNN_CK(cudaMemcpyAsync(dz, z, 8 * (size_t)n, cudaMemcpyHostToDevice, s));
    KNN_CK(cudaMemsetAsync(flags, 0, 2 * sizeof(int), s));
    Box6 fr;
    knn_frame(n, x, y, z, fr.lo, fr.hi);
    const int T = 256, g = (n + T - 1) / T;
    k_knn_keys<<<g, T, 0, s>>>(n, dx, dy, dz, fr, key, idx);
    size_t bytes = 0;
    KNN_CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, key, key2, idx, id, n, 0, 64, s));
    uint8_t *scratch;
    KNN_CK(b.alloc(&scratch, bytes));
    KNN_CK(cub::DeviceRadixSort::SortPairs(scratch, bytes, key, key2, idx, id, n, 0, 64, s));
    k_knn_gather<<<g, T, 0, s>>>(n, id, dx, dy, dz, sx, sy, sz);
    KnnTree t;
    t.n = n;
    t.levels = level_counts(n, t.count, t.span);
    Box6 *boxes[KNN_MAX_LEVELS];
    for (int l = 0; l < t.levels; ++l) {
        KNN_CK(b.alloc(&boxes[l], t.count[l]));
        const int gl = (t.count[l] + T - 1) / T;
        if (l == 0) k_knn_leaves<<<gl, T, 0, s>>>(t.count[0], n, sx, sy, sz, boxes[0]);
        else k_knn_nodes<<<gl, T, 0, s>>>(t.count[l], t.count[l - 1], boxes[l - 1], boxes[l]);
        t.box[l] = boxes[l];
    }
    t.sx = sx; t.sy = sy; t.sz = sz; t.id = id;
    k_knn_query<<<(n + 127) / 128, 128, 0, s>>>(t, k, dnb, dconn, dmd, flags);
    KNN_CK(cudaGetLastError());
    int h_flags[2] = {0, 0};
    KNN_CK(cudaMemcpyAsync(h_flags, flags, sizeof h_flags, cudaMemcpyDeviceToHost, s));
    KNN_CK(cudaMemcpyAsync(nbhs, dnb, 4 * (size_t)n, cudaMemcpyDeviceToHost, s));
    KNN_CK(cudaMemcpyAsync(conn, dconn, 4 * (size_t)n * MAX_CONN, cudaMemcpyDeviceToHost, s));
    KNN_CK(cudaMemcpyAsync(min_dist, dmd, 8 * (size_t)n, cudaMemcpyDeviceToHost, s));
    KNN_CK(cudaStreamSynchronize(s));
    if (h_flags[0]) {
        err = "two points of the cloud coincide";
        return MFCFD_ERR_ARG;
    }
    if (h_flags[1]) {
        err = "the cloud has no more than k points";
        return MFCFD_ERR_ARG;
    }
    return MFCFD_OK;
}

int knn_host(int n, const double *x, const double *y, const double *z, int k, int32_t *nbhs, int32_t *conn,
             double *min_dist, std::string &err) {
    double lo[3], scale[3];
    knn_frame(n, x, y, z, lo, scale);
    std::vector<std::pair<uint64_t, int32_t>> key(n);
    for (int i = 0; i < n; ++i) key[i] = {knn_key(x[i], y[i], z[i], lo, scale), i};
    std::sort(key.begin(), key.end());
    std::vector<int32_t> id(n);
    std::vector<double> sx(n), sy(n), sz(n);
    for (int s = 0; s < n; ++s) {
        id[s] = key[s].second;
        sx[s] = x[id[s]];
        sy[s] = y[id[s]];
        sz[s] = z[id[s]];
    }
    KnnTree t;
    t.n = n;
    t.levels = level_counts(n, t.count, t.span);
    std::vector<Box6> boxes[KNN_MAX_LEVELS];
    for (int l = 0; l < t.levels; ++l) {
        boxes[l].resize(t.count[l]);
        for (int b = 0; b < t.count[l]; ++b)
            boxes[l][b] = l == 0 ? knn_leaf_box(b, n, sx.data(), sy.data(), sz.data())
                                 : knn_node_box(b, t.count[l - 1], boxes[l - 1].data());
        t.box[l] = boxes[l].data();
    }
    t.sx = sx.data(); t.sy = sy.data(); t.sz = sz.data(); t.id = id.data();
    // the queries on the calling thread and the set-up pool's threads
    const int want = std::min(31, n / 4096);
    const int extra = want > 0 ? take_setup_threads(want) : 0;
    const int nt = extra + 1;
    std::vector<int> dup(nt, 0), sh(nt, 0);
    auto run = [&](int w) {
        for (int q = w; q < n; q += nt) knn_store(t, q, k, nbhs, conn, min_dist, &dup[w], &sh[w]);
    };
    std::vector<std::thread> th;
    std::exception_ptr e0;
    try {
        for (int w = 1; w < nt; ++w) th.emplace_back(run, w);
    } catch (...) {
        e0 = std::current_exception();
    }
    if (!e0) run(0);
    for (auto &h : th) h.join();
    give_setup_threads(extra);
    if (e0) std::rethrow_exception(e0);
    for (int w = 0; w < nt; ++w) {
        if (dup[w]) {
            err = "two points of the cloud coincide";
            return MFCFD_ERR_ARG;
        }
        if (sh[w]) {
            err = "the cloud has no more than k points";
            return MFCFD_ERR_ARG;
        }
    }
    return MFCFD_OK;
}

}  // namespace

int knn_connectivity(int device, int n, const double *x, const double *y, const double *z, int k, int32_t *nbhs,
                     int32_t *conn, double *min_dist, std::string &err) {
    if (n < 1 || k < 1 || k > MAX_CONN) {
        err = "knn: need n >= 1 and 1 <= k <= 27";
        return MFCFD_ERR_ARG;
    }
    return device >= 0 ? knn_device(device, n, x, y, z, k, nbhs, conn, min_dist, err)
                       : knn_host(n, x, y, z, k, nbhs, conn, min_dist, err);
}

}  // namespace mfcfd
