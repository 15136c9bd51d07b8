/*
 * mfcfd_capi.cpp - the extern "C" boundary declared in include/mfcfd.h.
 *
 * Owns the device copy of one point cloud and its iteration state, and maps
 * each reference entry point (fpi_solver, the q_lskum loop, the setup
 * routines) onto kernel launches on the handle's stream.
 */
#include <algorithm>
#include <chrono>
#include <deque>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "mfcfd_internal.h"

using namespace mfcfd;

struct mfcfd_handle {
    mfcfd_params P;
    Topology T;
    DevCloud d;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;          // flux residual beside the chain forward sweep
    cudaEvent_t fork = nullptr, join = nullptr;
    double *U_buf[2] = {nullptr, nullptr};
    double *q_buf[2] = {nullptr, nullptr};
    int cur = 0;          // U/q buffer the next iteration reads
    int last = 0;         // U/q buffer the last iteration read
    std::vector<void *> allocs;
    std::string err;
    double res_old = 0.0, res_new = 0.0, residue = 0.0;
    int res_cap = 1024;
    int64_t bytes = 0;
    bool have_state = false;
    bool res_valid = false;                // res_sqr holds the terms of a completed iteration
    bool profiling = false;
    std::vector<cudaEvent_t> ev;          // (MFCFD_NPHASE+1) per iteration slot
    double phase_ms[MFCFD_NPHASE] = {0};
    int64_t prof_iters = 0;
    int64_t chain_terms[3] = {0, 0, 0};   // chain schedule: ring, same-warp, cross-warp terms
    double *wall_area = nullptr;           // per-point areas for mfcfd_forces (device), or null
    int32_t *perm_dev = nullptr;           // storage index of each point (device); null: index order
    double *xfer = nullptr;                // 5 doubles per point: index-order transfer buffer
    double *force_out = nullptr;           // 3 doubles (device)
    // host copies held between mfcfd_prepare and mfcfd_attach
    struct Staged {
        std::vector<double> x, y, z, frame;
        std::vector<int32_t> nbhs, conn, pre;
        ChainSchedule S;
        int ch_w = 0, ch_wpb = 0;
    };
    std::unique_ptr<Staged> staged;
    bool dry = false;                      // count device bytes, allocate and copy nothing
    // captured chunks of iterations: (chunk length, U/q buffer at its start)
    struct GraphSlot {
        int chunk = -1, parity = -1;
        cudaGraphExec_t exec = nullptr;
    };
    GraphSlot graphs[2];
    int graph_next = 0;
    cudaEvent_t batch_ev = nullptr;        // end of the handle's chunk in mfcfd_run_batch / mfcfd_launch
    int pending_chunk = 0;                 // mfcfd_launch: iterations not yet completed
    int32_t pending_t0 = 0;
    bool graphs_off = false;               // a capture failed: launch one by one
    // device-resident set-up (mfcfd_params.gpu_setup = 1): the topology was
    // computed on the device; the host keeps summaries and fetches the
    // query arrays (stencils, alias, levels) from dt on demand
    bool dev_setup = false;
    DevTopology dt;
    // mixed precision: sweep terms per direction, and (MIXED_DC) their
    // unfolded weights, which the switch to FP64 puts back
    int64_t n_ent[2] = {0, 0};
    double *w_saved[2] = {nullptr, nullptr};
};

namespace {

const char *kStrerr[] = {"ok", "bad argument", "CUDA error", "stencil too wide",
                         "singular least-squares system", "non-finite residual",
                         "unsupported input", "out of memory", "device wait timed out",
                         "file input/output error", "request not finished"};

int fail(mfcfd_handle *h, int code, const std::string &msg) {
    if (h) h->err = msg;
    return code;
}

int cuda_fail(mfcfd_handle *h, cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(h, e == cudaErrorMemoryAllocation ? MFCFD_ERR_NOMEM : MFCFD_ERR_CUDA, m);
}

#define CK(call)                                                        \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call);          \
    } while (0)

template <typename T>
int dalloc(mfcfd_handle *h, T **p, size_t count) {
    size_t bytes = sizeof(T) * (count > 0 ? count : 1);
    if (h->dry) {
        h->bytes += (int64_t)bytes;
        *p = nullptr;
        return MFCFD_OK;
    }
    // stream-ordered: freeing later does not synchronise the whole device
    void *v = nullptr;
    cudaError_t e = h->stream ? cudaMallocAsync(&v, bytes, h->stream) : cudaMalloc(&v, bytes);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaMalloc");
    h->allocs.push_back(v);
    h->bytes += (int64_t)bytes;
    *p = (T *)v;
    return MFCFD_OK;
}

template <typename T>
int upload(mfcfd_handle *h, const T **dst, const std::vector<T> &src) {
    T *p = nullptr;
    int rc = dalloc(h, &p, src.size());
    if (rc) return rc;
    if (!src.empty() && !h->dry) CK(cudaMemcpyAsync(p, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, h->stream));
    *dst = p;
    return MFCFD_OK;
}

// n rows of w doubles from host memory in the reference's index order to
// device memory in storage order, through the transfer buffer when the
// cloud is stored permuted (stream-ordered; the caller synchronises).
int rows_to_device(mfcfd_handle *h, double *dst, const double *src, int w) {
    const size_t n = (size_t)h->d.n;
    if (!h->perm_dev) {
        CK(cudaMemcpyAsync(dst, src, n * w * 8, cudaMemcpyHostToDevice, h->stream));
        return MFCFD_OK;
    }
    const size_t per = std::max<size_t>(1, n * 5 / (size_t)w);
    for (size_t a = 0; a < n; a += per) {
        const size_t rows = std::min(per, n - a);
        CK(cudaMemcpyAsync(h->xfer, src + a * w, rows * w * 8, cudaMemcpyHostToDevice, h->stream));
        CK(launch_rows(h->xfer, dst, h->perm_dev, (int)a, (int)rows, w, true, h->stream));
    }
    return MFCFD_OK;
}

// The reverse: n rows of w doubles of device memory in storage order to host
// memory in index order.
int rows_to_host(mfcfd_handle *h, double *dst, const double *src, int w) {
    const size_t n = (size_t)h->d.n;
    if (!h->perm_dev) {
        CK(cudaMemcpyAsync(dst, src, n * w * 8, cudaMemcpyDeviceToHost, h->stream));
        return MFCFD_OK;
    }
    const size_t per = std::max<size_t>(1, n * 5 / (size_t)w);
    for (size_t a = 0; a < n; a += per) {
        const size_t rows = std::min(per, n - a);
        CK(launch_rows(src, h->xfer, h->perm_dev, (int)a, (int)rows, w, false, h->stream));
        CK(cudaMemcpyAsync(dst + a * w, h->xfer, rows * w * 8, cudaMemcpyDeviceToHost, h->stream));
    }
    return MFCFD_OK;
}

// Free one device array of the handle.
void dfree(mfcfd_handle *h, const void *p) {
    for (size_t i = 0; i < h->allocs.size(); ++i)
        if (h->allocs[i] == p) {
            if (h->stream) cudaFreeAsync(h->allocs[i], h->stream);
            else cudaFree(h->allocs[i]);
            h->allocs.erase(h->allocs.begin() + (long)i);
            return;
        }
}

void drop_graphs(mfcfd_handle *h) {
    for (auto &g : h->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = mfcfd_handle::GraphSlot();
    }
}

void release(mfcfd_handle *h) {
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_graphs(h);
    if (h->side) cudaStreamSynchronize(h->side);
    for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
    h->ev.clear();
    for (void *p : h->allocs) {
        if (h->stream) cudaFreeAsync(p, h->stream);
        else cudaFree(p);
    }
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->allocs.clear();
    if (h->batch_ev) cudaEventDestroy(h->batch_ev);
    h->batch_ev = nullptr;
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->join) cudaEventDestroy(h->join);
    h->fork = h->join = nullptr;
    if (h->side) cudaStreamDestroy(h->side);
    h->side = nullptr;
    if (h->stream) cudaStreamDestroy(h->stream);
    h->stream = nullptr;
}

int finish_step(mfcfd_handle *h, int32_t t, double res_new) {
    h->res_new = res_new;
    if (t <= 2) {                      // fpi_solver.f90:38-40
        h->res_old = res_new;
        h->residue = 0.0;
    } else {
        h->residue = std::log10(res_new / h->res_old);
    }
    if (!std::isfinite(res_new)) return fail(h, MFCFD_ERR_NONFINITE, "res_new is not finite");
    return MFCFD_OK;
}

// Launch iteration j of the current chunk (iteration slot j of res_dev).
int launch_one(mfcfd_handle *h, int j) {
    DevCloud dc = h->d;
    dc.U = h->U_buf[h->cur];
    dc.q = h->q_buf[h->cur];
    cudaEvent_t *ev = h->profiling ? &h->ev[(size_t)j * (MFCFD_NPHASE + 1)] : nullptr;
    const IterStreams st{h->stream, h->side, h->fork, h->join};
    cudaError_t e = launch_iteration(dc, j, st, h->U_buf[1 - h->cur], h->q_buf[1 - h->cur], ev);
    if (e != cudaSuccess) return cuda_fail(h, e, "kernel launch");
    h->last = h->cur;
    h->cur = 1 - h->cur;
    return MFCFD_OK;
}

// Launch the iterations of one chunk (slots 0 .. chunk-1).  With graphs, the
// chunk is captured once per (length, starting U/q buffer) and replayed;
// the host-side buffer state then advances as the captured launches did.
int launch_chunk(mfcfd_handle *h, int chunk, bool batch) {
    h->res_valid = false;                  // valid again once the chunk has completed
    if (h->P.graphs < (batch ? 1 : 2) || h->graphs_off || h->profiling) {
        for (int j = 0; j < chunk; ++j) {
            int rc = launch_one(h, j);
            if (rc) return rc;
        }
        return MFCFD_OK;
    }
    const int c0 = h->cur;
    mfcfd_handle::GraphSlot *g = nullptr;
    for (auto &s : h->graphs)
        if (s.exec && s.chunk == chunk && s.parity == c0) g = &s;
    if (!g) {
        prepare_launches(h->P.device);
        mfcfd_handle::GraphSlot &slot = h->graphs[h->graph_next];
        h->graph_next ^= 1;
        if (slot.exec) cudaGraphExecDestroy(slot.exec);
        slot = mfcfd_handle::GraphSlot();
        const int last0 = h->last;
        cudaGraph_t graph = nullptr;
        int rc = MFCFD_OK;
        cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            for (int j = 0; j < chunk && rc == MFCFD_OK; ++j) rc = launch_one(h, j);
            e = cudaStreamEndCapture(h->stream, &graph);
        }
        h->cur = c0;
        h->last = last0;
        if (e == cudaSuccess && rc == MFCFD_OK) e = cudaGraphInstantiate(&slot.exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess || rc != MFCFD_OK || !slot.exec) {
            // no graph on this handle: launch one by one from now on
            (void)cudaGetLastError();
            slot = mfcfd_handle::GraphSlot();
            h->graphs_off = true;
            h->err.clear();
            for (int j = 0; j < chunk; ++j) {
                int rc2 = launch_one(h, j);
                if (rc2) return rc2;
            }
            return MFCFD_OK;
        }
        slot.chunk = chunk;
        slot.parity = c0;
        g = &slot;
    }
    CK(cudaGraphLaunch(g->exec, h->stream));
    h->last = (chunk & 1) ? c0 : 1 - c0;
    h->cur = (chunk & 1) ? 1 - c0 : c0;
    return MFCFD_OK;
}

// Wait for a chunk of `chunk` launched iterations (t = t0 ..) and do the
// host bookkeeping; res_hist (may be null) gets (res_new, residue) pairs.
int finish_chunk(mfcfd_handle *h, int32_t t0, int chunk, double *res_hist, int *status) {
    std::vector<double> res(chunk);
    int err_flag = 0;
    CK(cudaMemcpyAsync(res.data(), h->d.res_dev, sizeof(double) * chunk, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&err_flag, h->d.err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (err_flag) {
        CK(cudaMemsetAsync(h->d.err, 0, sizeof(int), h->stream));
        CK(cudaStreamSynchronize(h->stream));
        return fail(h, MFCFD_ERR_TIMEOUT, "a sweep wait ran out; the iteration results are invalid");
    }
    h->res_valid = true;
    if (h->profiling) {
        for (int j = 0; j < chunk; ++j) {
            const cudaEvent_t *ev = &h->ev[(size_t)j * (MFCFD_NPHASE + 1)];
            // event pairs per phase; under the chain schedule the flux
            // residual (ended by event 2, side stream) starts at event 3
            // and runs beside the forward sweep, after k_pending (1-3)
            static const int kSeq[MFCFD_NPHASE][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 4}, {4, 5}, {5, 6}, {6, 7}};
            static const int kFused[MFCFD_NPHASE][2] = {{0, 1}, {3, 2}, {1, 3}, {3, 4}, {4, 5}, {5, 6}, {6, 7}};
            const bool fused = h->d.sweep_mode == MFCFD_SWEEP_CHAINS;
            for (int ph = 0; ph < MFCFD_NPHASE; ++ph) {
                float ms = 0.f;
                const int *pr = fused ? kFused[ph] : kSeq[ph];
                CK(cudaEventElapsedTime(&ms, ev[pr[0]], ev[pr[1]]));
                h->phase_ms[ph] += ms;
            }
        }
        h->prof_iters += chunk;
    }
    for (int j = 0; j < chunk; ++j) {
        int rc = finish_step(h, t0 + j, res[j]);
        if (rc && *status == MFCFD_OK) *status = rc;
        if (res_hist) {
            res_hist[2 * (size_t)j] = h->res_new;
            res_hist[2 * (size_t)j + 1] = h->residue;
        }
    }
    return MFCFD_OK;
}

// Rebuild the chain schedule for about `want` warps on the handle's
// topology and replace its device copy (the term records are re-marked, so
// they are copied again); *warps receives the new schedule's warps.
int apply_chain_schedule(mfcfd_handle *h, int want, int *warps) {
    int wpb = 0, blocks = 0;
    const int w = chain_shape(h->P.device, want, h->P.chain_spread, &wpb, &blocks);
    if (w < 1) return fail(h, MFCFD_ERR_CUDA, "chain sweep kernel cannot be resident");
    if (h->dev_setup) {
        DevCloud &d = h->d;
        for (int dir = 0; dir < 2; ++dir) {
            dfree(h, d.ch_ptr[dir]);
            dfree(h, d.ch_pts[dir]);
            dfree(h, d.ch_own[dir]);
            dfree(h, d.ch_items[dir]);
        }
        const DevAlloc alloc = [h](void **ptr, size_t bytes) {
            uint8_t *p = nullptr;
            const int r = dalloc(h, &p, bytes);
            *ptr = p;
            return r;
        };
        std::string err;
        int64_t terms[3];
        if (int rc = device_chain_schedule(h->P.device, h->dt, d, w, h->stream, alloc, terms, err))
            return fail(h, rc, err.empty() ? h->err : err);
        d.ch_wpb = wpb;
        d.ch_spread = h->P.chain_spread;
        drop_graphs(h);
        for (int k = 0; k < 3; ++k) h->chain_terms[k] = terms[k];
        *warps = w;
        return MFCFD_OK;
    }
    ChainSchedule S;
    build_chain_schedule(h->T, w, S);
    DevCloud &d = h->d;
    int rc = MFCFD_OK;
    for (int dir = 0; dir < 2; ++dir) {
        dfree(h, d.ch_ptr[dir]);
        dfree(h, d.ch_pts[dir]);
        dfree(h, d.ch_own[dir]);
        dfree(h, d.ch_items[dir]);
        if ((rc = upload(h, &d.ch_ptr[dir], S.ptr[dir])) || (rc = upload(h, &d.ch_pts[dir], S.pts[dir])) ||
            (rc = upload(h, &d.ch_own[dir], S.owner[dir])) || (rc = upload(h, &d.ch_items[dir], S.items[dir])))
            return rc;
    }
    const std::vector<SweepEntry> *ents[2] = {&h->T.fwd_ent, &h->T.bwd_ent};
    const SweepEntry *dents[2] = {d.fwd_ent, d.bwd_ent};
    for (int dir = 0; dir < 2; ++dir)
        if (!ents[dir]->empty()) {
            cudaError_t e = cudaMemcpyAsync((void *)dents[dir], ents[dir]->data(), sizeof(SweepEntry) * ents[dir]->size(),
                                            cudaMemcpyHostToDevice, h->stream);
            if (e != cudaSuccess) return cuda_fail(h, e, "cudaMemcpyAsync");
        }
    // the host's terms carry the unfolded weights
    if (d.precision != MFCFD_PRECISION_FP64) CK(launch_fold_terms(d, h->w_saved, true, h->stream));
    d.ch_warps = w;
    d.ch_wpb = wpb;
    d.ch_spread = h->P.chain_spread;
    drop_graphs(h);                        // their launches name the old schedule
    h->chain_terms[0] = S.terms_ring;
    h->chain_terms[1] = S.terms_local;
    h->chain_terms[2] = S.terms_cross;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamSynchronize");
    *warps = w;
    return MFCFD_OK;
}

int run_iterations(mfcfd_handle *h, int32_t t0, int32_t iters, double *res_hist) {
    if (!h->have_state) return fail(h, MFCFD_ERR_ARG, "no state: call mfcfd_set_prim first");
    int status = MFCFD_OK;
    for (int32_t done = 0; done < iters;) {
        int chunk = std::min<int32_t>(iters - done, h->res_cap);
        int rc = launch_chunk(h, chunk, false);
        if (rc) return rc;
        rc = finish_chunk(h, t0 + done, chunk, res_hist ? res_hist + 2 * (size_t)done : nullptr, &status);
        if (rc) return rc;
        done += chunk;
    }
    return status;
}

}  // namespace

namespace {

int stage_host(mfcfd_handle *h, const double *x, const double *y, const double *z, const double *tan1,
               const double *tan2, const double *nor, const int32_t *nbhs, const int32_t *conn);
int attach_device(mfcfd_handle *h);
int attach_state(mfcfd_handle *h);
int create_on_device(mfcfd_handle *h, const double *x, const double *y, const double *z, const double *tan1,
                     const double *tan2, const double *nor, const int32_t *nbhs, const int32_t *conn,
                     const double *min_dist);

}  // namespace

extern "C" {

void mfcfd_params_init(mfcfd_params *p, double mach, double aoa_deg) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    const double pi = 4.0 * std::atan(1.0);         // parameter.f90:19
    const double theta = aoa_deg * pi / 180.0;      // parameter.f90:20
    p->power = 0.0;                                 // parameter.f90:21
    p->vl_const = 2.0;                              // parameter.f90:22
    p->cfl = 5.0;                                   // parameter.f90:23
    p->inner_iterations = 0;                        // parameter.f90:24
    p->rho_inf = 1.0;                               // parameter.f90:29
    p->u1_inf = mach * std::cos(theta);             // parameter.f90:30
    p->u2_inf = mach * std::sin(theta);             // parameter.f90:31
    p->u3_inf = 0.0;                                // parameter.f90:32
    p->pr_inf = 1.0 / 1.4;                          // parameter.f90:33
    p->split_capacity = 22;                         // data_structure.f90:83-88
    p->precision = MFCFD_PRECISION_FP64;
    p->device = 0;
    p->sweep_mode = MFCFD_SWEEP_CHAINS;
    p->graphs = 1;
    p->storage_order = MFCFD_ORDER_MORTON;
}

}  // extern "C"

namespace {

// mfcfd_create and mfcfd_prepare: validation and the host set-up; with
// `attach`, also the device copy.
int create_impl(const mfcfd_params *params, int32_t n, const int32_t *status, const double *x,
                const double *y, const double *z, const double *tan1, const double *tan2,
                const double *nor, const int32_t *nbhs, const int32_t *conn,
                const double *min_dist, mfcfd_handle **out, bool attach) {
    if (!out) return MFCFD_ERR_ARG;
    *out = nullptr;
    if (!params || n < 1 || !status || !x || !y || !z || !tan1 || !tan2 || !nor || !nbhs ||
        !conn || !min_dist)
        return MFCFD_ERR_ARG;
    mfcfd_handle *h = new (std::nothrow) mfcfd_handle();
    if (!h) return MFCFD_ERR_NOMEM;
    h->P = *params;
    const mfcfd_params &P = h->P;
    if (P.inner_iterations < 0 || P.inner_iterations > 1000) {
        h->err = "inner_iterations out of range [0, 1000]";
        *out = h;
        return MFCFD_ERR_ARG;
    }
    if (!(P.power >= 0.0 && P.power <= 16.0)) {
        h->err = "power out of range [0, 16]";
        *out = h;
        return MFCFD_ERR_ARG;
    }
    if (P.sweep_variant != MFCFD_SWEEPS_ALIAS && P.sweep_variant != MFCFD_SWEEPS_BACKUP) {
        h->err = "unknown sweep_variant";
        *out = h;
        return MFCFD_ERR_ARG;
    }
    if (P.update_variant != MFCFD_UPDATE_IMPLICIT && P.update_variant != MFCFD_UPDATE_EXPLICIT) {
        h->err = "unknown update_variant";
        *out = h;
        return MFCFD_ERR_ARG;
    }
    if (P.precision != MFCFD_PRECISION_FP64 && P.precision != MFCFD_PRECISION_MIXED &&
        P.precision != MFCFD_PRECISION_MIXED_DC) {
        h->err = "unknown precision";
        *out = h;
        return MFCFD_ERR_UNSUPPORTED;
    }
    if (P.precision != MFCFD_PRECISION_FP64 && P.sweep_mode != MFCFD_SWEEP_CHAINS) {
        h->err = "mixed precision requires the chain sweep schedule";
        *out = h;
        return MFCFD_ERR_UNSUPPORTED;
    }
    if (P.sweep_mode != MFCFD_SWEEP_DATAFLOW && P.sweep_mode != MFCFD_SWEEP_LEVELS &&
        P.sweep_mode != MFCFD_SWEEP_CHAINS) {
        h->err = "unknown sweep_mode";
        *out = h;
        return MFCFD_ERR_ARG;
    }
    if (P.split_capacity < 0 || P.split_capacity > 1000) {
        h->err = "split_capacity out of range";
        *out = h;
        return MFCFD_ERR_ARG;
    }
    if (P.flux_blocks_per_sm < 0 || P.flux_blocks_per_sm > 64) {
        h->err = "flux_blocks_per_sm out of range [0, 64]";
        *out = h;
        return MFCFD_ERR_ARG;
    }
    if (P.storage_order != MFCFD_ORDER_INDEX && P.storage_order != MFCFD_ORDER_MORTON) {
        h->err = "unknown storage_order";
        *out = h;
        return MFCFD_ERR_ARG;
    }
    *out = h;   // also on failure: it holds the message
    return host_guard(&h->err, [&]() -> int {
        if (attach && P.gpu_setup == 1 && P.device >= 0) {
            int rc = classify_points(P, n, status, nbhs, conn, h->T, h->err);
            if (rc) return rc;
            if (device_setup_supported(P, h->T))
                return create_on_device(h, x, y, z, tan1, tan2, nor, nbhs, conn, min_dist);
            h->T = Topology();   // the host set-up, with its GPU passes
        }
        int rc = build_topology(P, n, status, x, y, z, tan1, tan2, nor, nbhs, conn, min_dist, h->T, h->err);
        if (rc) return rc;
        if (P.device < 0) return MFCFD_OK;   // host-only handle: set-up results, no device state
        if (P.storage_order == MFCFD_ORDER_MORTON && n > 1) {
            // the device layout follows a space-filling curve; the set-up
            // above ran on the reference's indices and is relabelled
            std::vector<int32_t> perm;
            morton_order(n, x, y, z, perm);
            permute_topology(h->T, perm);
        }
        if ((rc = stage_host(h, x, y, z, tan1, tan2, nor, nbhs, conn))) return rc;
        if (attach) {
            if ((rc = attach_device(h))) return rc;
            h->staged.reset();
        }
        return MFCFD_OK;
    });
}

// Host copies of the inputs the device needs, in the device layout, and the
// chain schedule (the kernel's residency on P.device sets its warp count).
int stage_host(mfcfd_handle *h, const double *x, const double *y, const double *z, const double *tan1,
               const double *tan2, const double *nor, const int32_t *nbhs, const int32_t *conn) {
    const mfcfd_params &P = h->P;
    const int n = h->T.n;
    if (cudaSetDevice(P.device) != cudaSuccess) return fail(h, MFCFD_ERR_CUDA, "cudaSetDevice failed");
    auto st = std::make_unique<mfcfd_handle::Staged>();
    // in storage order (T.perm; the identity when it is empty)
    const std::vector<int32_t> &perm = h->T.perm;
    auto at = [&](int i) { return perm.empty() ? (size_t)i : (size_t)perm[i]; };
    st->x.resize(n);
    st->y.resize(n);
    st->z.resize(n);
    st->frame.resize((size_t)n * 9);
    st->nbhs.resize(n);
    st->conn.assign((size_t)n * MAX_CONN, 0);
    for (int i = 0; i < n; ++i) {
        const size_t s = at(i);
        st->x[s] = x[i];
        st->y[s] = y[i];
        st->z[s] = z[i];
        for (int r = 0; r < 3; ++r) {
            st->frame[9 * s + r] = tan1[3 * (size_t)i + r];
            st->frame[9 * s + 3 + r] = tan2[3 * (size_t)i + r];
            st->frame[9 * s + 6 + r] = nor[3 * (size_t)i + r];
        }
        st->nbhs[s] = nbhs[i];
        for (int r = 0; r < MAX_CONN; ++r) {
            const int32_t k = conn[(size_t)i * MAX_CONN + r];
            st->conn[s * MAX_CONN + r] = (k > 0 && k <= n) ? (int32_t)at(k - 1) : 0;
        }
    }
    if (P.sweep_mode == MFCFD_SWEEP_CHAINS) {
        // about twice the widest level in warps, all co-resident; the
        // schedule itself is built when first needed (attach_device), so a
        // warp count set before then costs one build
        if (P.chain_warps < 0) return fail(h, MFCFD_ERR_ARG, "chain_warps must not be negative");
        const int want = P.chain_warps > 0 ? P.chain_warps : std::max(1, 2 * h->T.max_level_width);
        int blocks = 0;
        if (P.chain_spread < 0 || P.chain_spread > 1) return fail(h, MFCFD_ERR_ARG, "chain_spread must be 0 or 1");
        st->ch_w = chain_shape(P.device, want, P.chain_spread, &st->ch_wpb, &blocks);
        if (st->ch_w < 1) return fail(h, MFCFD_ERR_CUDA, "chain sweep kernel cannot be resident");
    }
    h->staged = std::move(st);
    return MFCFD_OK;
}

// The device's default memory pool (every handle's stream-ordered memory)
// keeps what handles free for the next ones instead of unmapping it at the
// next synchronisation: a new handle's set-up then finds its memory mapped
// (1.1M points: 0.46 s, against up to 1.2 s when it had to be mapped again).
// cudaMemPoolTrimTo on the pool returns it.  Set once per device.
void keep_pool_memory(int device) {
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lk(mu);
    if (std::find(done.begin(), done.end(), device) != done.end()) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done.push_back(device);
}

// The handle's streams: the main stream outranks the side stream, so the
// chain sweep's blocks are placed before the concurrent flux kernel's.
int create_streams(mfcfd_handle *h) {
    if (cudaSetDevice(h->P.device) != cudaSuccess) return fail(h, MFCFD_ERR_CUDA, "cudaSetDevice failed");
    keep_pool_memory(h->P.device);
    int least = 0, greatest = 0;
    CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    CK(cudaStreamCreateWithPriority(&h->stream, cudaStreamNonBlocking, greatest));
    CK(cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, least));
    CK(cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming));
    return MFCFD_OK;
}

// DevCloud cleared, with the point count and the parameters the kernels read.
void init_devcloud(mfcfd_handle *h, int n) {
    const mfcfd_params &P = h->P;
    DevCloud &d = h->d;
    std::memset(&d, 0, sizeof d);
    d.n = n;
    d.power = P.power;
    d.inner_iterations = P.inner_iterations;
    d.update_variant = P.update_variant;
    d.sweep_variant = P.sweep_variant;
    d.cfl = P.cfl;
    d.rho_inf = P.rho_inf; d.u1_inf = P.u1_inf; d.u2_inf = P.u2_inf;
    d.u3_inf = P.u3_inf; d.pr_inf = P.pr_inf;
}

// Streams, device arrays and uploads from the staged copies (with h->dry:
// only the byte count).
int attach_device(mfcfd_handle *h) {
    const mfcfd_params &P = h->P;
    const Topology &T = h->T;
    const mfcfd_handle::Staged &st = *h->staged;
    const int n = T.n;
    int rc = MFCFD_OK;
    if (!h->dry && (rc = create_streams(h))) return rc;

    DevCloud &d = h->d;
    init_devcloud(h, n);
    d.shared_frame = T.shared_frame;
    std::memcpy(d.frame0, T.frame0, sizeof d.frame0);

    if (P.sweep_mode == MFCFD_SWEEP_CHAINS) {
        // the schedule marks the entry lists, so it precedes their upload
        mfcfd_handle::Staged &ms = *h->staged;
        if (ms.S.warps != ms.ch_w) {
            ms.S = ChainSchedule();
            build_chain_schedule(h->T, ms.ch_w, ms.S);
        }
        if (ms.pre.empty()) build_pre_order(h->T, ms.pre);
        const ChainSchedule &S = st.S;
        d.ch_warps = st.ch_w;
        d.ch_wpb = st.ch_wpb;
        d.ch_spread = P.chain_spread;
        d.flux_grid = P.flux_blocks_per_sm > 0 ? P.flux_blocks_per_sm * device_sms(P.device) : 0;
        if ((rc = upload(h, &d.pre_order, st.pre))) return rc;
        for (int dir = 0; dir < 2; ++dir) {
            if ((rc = upload(h, &d.ch_ptr[dir], S.ptr[dir]))) return rc;
            if ((rc = upload(h, &d.ch_pts[dir], S.pts[dir]))) return rc;
            if ((rc = upload(h, &d.ch_own[dir], S.owner[dir]))) return rc;
            if ((rc = upload(h, &d.ch_items[dir], S.items[dir]))) return rc;
        }
        h->chain_terms[0] = S.terms_ring;
        h->chain_terms[1] = S.terms_local;
        h->chain_terms[2] = S.terms_cross;
        if (!T.g0_pts.empty()) {
            if ((rc = upload(h, &d.g0_pts, T.g0_pts))) return rc;
            if ((rc = dalloc(h, &d.g0, T.g0_pts.size() * (size_t)G0_DOUBLES))) return rc;
            d.n_g0 = (int)T.g0_pts.size();
        }
    }
    std::vector<int32_t> order;
    order.insert(order.end(), T.wall_idx.begin(), T.wall_idx.end());
    order.insert(order.end(), T.interior_idx.begin(), T.interior_idx.end());
#define UP(field, vec) if ((rc = upload(h, &d.field, vec))) return rc
    UP(x, st.x); UP(y, st.y); UP(z, st.z); UP(frame, st.frame);
    UP(cls, T.cls); UP(nbhs, st.nbhs); UP(conn, st.conn); UP(eps2, T.eps2);
    UP(slot_nbr, T.slot_nbr); UP(nslot, T.nslot); UP(slot_mask, T.slot_mask);
    UP(list_cnt, T.list_cnt); UP(list_ent, T.list_ent); UP(geo, T.geo);
    if (!T.wq.empty()) { UP(wq, T.wq); UP(wf, T.wf); }
    UP(swept, T.swept); UP(consumer_shared, T.consumer_shared);
    UP(fwd_lvl_ptr, T.fwd_lvl_ptr); UP(fwd_lvl_pts, T.fwd_lvl_pts);
    UP(bwd_lvl_ptr, T.bwd_lvl_ptr); UP(bwd_lvl_pts, T.bwd_lvl_pts);
    UP(fwd_off, T.fwd_off); UP(bwd_off, T.bwd_off);
    UP(fwd_cnt, T.fwd_cnt); UP(bwd_cnt, T.bwd_cnt);
    UP(fwd_ent, T.fwd_ent); UP(bwd_ent, T.bwd_ent);
    UP(fwd_need, T.fwd_need); UP(bwd_need, T.bwd_need);
    UP(fwd_old, T.fwd_old); UP(bwd_old, T.bwd_old); UP(sweep_slot_mask, T.sweep_slot_mask);
    if (!T.outer_delt.empty()) UP(outer_delt, T.outer_delt);
    UP(res_order, order);
    if (!T.perm.empty()) {
        const int32_t *pd = nullptr;
        if ((rc = upload(h, &pd, T.perm))) return rc;
        h->perm_dev = const_cast<int32_t *>(pd);
        if ((rc = dalloc(h, &h->xfer, (size_t)n * 5))) return rc;
    }
#undef UP
    d.n_fwd_levels = (int)T.fwd_lvl_ptr.size() - 1;
    d.n_bwd_levels = (int)T.bwd_lvl_ptr.size() - 1;
    d.n_res = (int)order.size();
    d.n_wall = (int)T.wall_idx.size();
    d.n_swept = (int)T.fwd_lvl_pts.size();
    d.max_width = T.max_level_width;
    h->n_ent[0] = (int64_t)T.fwd_ent.size();
    h->n_ent[1] = (int64_t)T.bwd_ent.size();
    return attach_state(h);
}

// The iteration state and the work arrays of a handle whose topology is on
// the device (with h->dry: only their byte count).
int attach_state(mfcfd_handle *h) {
    const mfcfd_params &P = h->P;
    const Topology &T = h->T;
    DevCloud &d = h->d;
    const int n = d.n;
    int rc = MFCFD_OK;
    d.sweep_mode = P.sweep_mode;
    d.precision = P.precision;
    if ((rc = dalloc(h, &d.sweep_counter, 2))) return rc;
    if ((rc = dalloc(h, &d.err, 1))) return rc;
    size_t n5 = (size_t)n * 5;
#define AL(ptr, cnt) if ((rc = dalloc(h, &ptr, cnt))) return rc
    AL(d.prim, n5); AL(h->U_buf[0], n5); AL(h->U_buf[1], n5); AL(h->q_buf[0], n5);
    AL(h->q_buf[1], n5); AL(d.qm, (size_t)n * 10); AL(d.dq, (size_t)n * 15);
    AL(d.delt, n); AL(d.flux_res, n5); AL(d.dUp, n5); AL(d.dUn, n5); AL(d.dinv, n);
    AL(d.gold, (size_t)n * 30); AL(d.dgf, (size_t)n * DG_STRIDE); AL(d.dgb, (size_t)n * DG_STRIDE);
    AL(d.res_sqr, n); AL(d.partial, 1024); AL(d.res_dev, h->res_cap);
    if (P.inner_iterations > 0) AL(d.dq_tmp, (size_t)n * 15);
    if (P.sweep_variant == MFCFD_SWEEPS_BACKUP) AL(d.dg_old, (size_t)n * DG_STRIDE);
    if (!T.ss_pts.empty() || P.sweep_variant == MFCFD_SWEEPS_BACKUP) AL(d.dU_old, n5);
    if (!T.ss_pts.empty()) {
        d.n_ss = (int)T.ss_pts.size();
        if ((rc = upload(h, &d.ss_pts, T.ss_pts))) return rc;
        if ((rc = upload(h, &d.ss_src, T.ss_src))) return rc;
    }
    if (P.precision == MFCFD_PRECISION_MIXED_DC) {
        AL(h->w_saved[0], 3 * (size_t)std::max<int64_t>(h->n_ent[0], 1));
        AL(h->w_saved[1], 3 * (size_t)std::max<int64_t>(h->n_ent[1], 1));
    }
#undef AL
    d.U = h->U_buf[0];
    d.q = h->q_buf[0];
    if (h->dry) return MFCFD_OK;
    CK(cudaMemsetAsync(d.sweep_counter, 0, sizeof(int) * 2, h->stream));
    CK(cudaMemsetAsync(d.err, 0, sizeof(int), h->stream));
    CK(cudaMemsetAsync(d.dUp, 0, n5 * 8, h->stream));
    CK(cudaMemsetAsync(d.dUn, 0, n5 * 8, h->stream));
    CK(cudaMemsetAsync(d.flux_res, 0, n5 * 8, h->stream));
    CK(cudaMemsetAsync(d.dinv, 0, (size_t)n * 8, h->stream));
    CK(cudaMemsetAsync(d.res_sqr, 0, (size_t)n * 8, h->stream));
    if (P.precision != MFCFD_PRECISION_FP64 && P.sweep_mode == MFCFD_SWEEP_CHAINS)
        CK(launch_fold_terms(d, h->w_saved, true, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MFCFD_OK;
}

// mfcfd_create with gpu_setup = 1 where device_setup_supported(): the whole
// set-up on the device (T holds classify_points' result).
int create_on_device(mfcfd_handle *h, const double *x, const double *y, const double *z, const double *tan1,
                     const double *tan2, const double *nor, const int32_t *nbhs, const int32_t *conn,
                     const double *min_dist) {
    const mfcfd_params &P = h->P;
    Topology &T = h->T;
    const int n = T.n;
    int rc = MFCFD_OK;
    if (P.sweep_mode == MFCFD_SWEEP_CHAINS) {
        if (P.chain_warps < 0) return fail(h, MFCFD_ERR_ARG, "chain_warps must not be negative");
        if (P.chain_spread < 0 || P.chain_spread > 1) return fail(h, MFCFD_ERR_ARG, "chain_spread must be 0 or 1");
    }
    std::vector<double> eps2;
    limiter_eps2(P, n, min_dist, nullptr, eps2);
    if ((rc = create_streams(h))) return rc;
    init_devcloud(h, n);
    h->dev_setup = true;
    DevCloud &d = h->d;
    const DevAlloc alloc = [h](void **ptr, size_t bytes) {
        uint8_t *p = nullptr;
        const int r = dalloc(h, &p, bytes);
        *ptr = p;
        return r;
    };
    std::string err;
    if ((rc = device_setup(P.device, P, T, x, y, z, tan1, tan2, nor, nbhs, conn, eps2, h->stream, alloc, d, h->dt,
                           err)))
        return fail(h, rc, err.empty() ? h->err : err);
    // host summaries, in the host set-up's form
    T.fwd_lvl_ptr = h->dt.lvl_ptr[0];
    T.bwd_lvl_ptr = h->dt.lvl_ptr[1];
    T.max_level_width = h->dt.max_width;
    T.split_overflows = (int)h->dt.split_overflows;
    T.shared_frame = d.shared_frame;
    std::memcpy(T.frame0, d.frame0, sizeof T.frame0);
    T.g0_pts = h->dt.g0_pts;
    T.sweep_variant = P.sweep_variant;
    if (!T.perm.empty()) {
        std::vector<int8_t> cls(n);
        for (int i = 0; i < n; ++i) cls[T.perm[i]] = T.cls[i];
        T.cls.swap(cls);
        for (std::vector<int32_t> *a : {&T.wall_idx, &T.outer_idx, &T.interior_idx})
            for (int32_t &v : *a) v = T.perm[v];
    }
    if (P.sweep_mode == MFCFD_SWEEP_CHAINS) {
        const int want = P.chain_warps > 0 ? P.chain_warps : std::max(1, 2 * T.max_level_width);
        int wpb = 0, blocks = 0;
        const int w = chain_shape(P.device, want, P.chain_spread, &wpb, &blocks);
        if (w < 1) return fail(h, MFCFD_ERR_CUDA, "chain sweep kernel cannot be resident");
        int64_t terms[3];
        if ((rc = device_chain_schedule(P.device, h->dt, d, w, h->stream, alloc, terms, err)))
            return fail(h, rc, err.empty() ? h->err : err);
        d.ch_wpb = wpb;
        d.ch_spread = P.chain_spread;
        d.flux_grid = P.flux_blocks_per_sm > 0 ? P.flux_blocks_per_sm * device_sms(P.device) : 0;
        for (int k = 0; k < 3; ++k) h->chain_terms[k] = terms[k];
        if (d.n_g0 > 0 && (rc = dalloc(h, &d.g0, (size_t)d.n_g0 * G0_DOUBLES))) return rc;
    }
    if (!T.perm.empty()) {
        const int32_t *pd = nullptr;
        if ((rc = upload(h, &pd, T.perm))) return rc;
        h->perm_dev = const_cast<int32_t *>(pd);
        if ((rc = dalloc(h, &h->xfer, (size_t)n * 5))) return rc;
    }
    h->n_ent[0] = h->dt.n_ent[0];
    h->n_ent[1] = h->dt.n_ent[1];
    return attach_state(h);
}

// The topology arrays the queries read, fetched from a device set-up into
// the host copy the first time they are asked for.
int fetch_query_arrays(mfcfd_handle *h, bool stencils, bool alias, bool levels) {
    if (!h->dev_setup) return MFCFD_OK;
    Topology &T = h->T;
    const DevTopology &dt = h->dt;
    const int n = T.n;
    const size_t flat = (size_t)n * T.cap + 64;
    if (stencils && T.split[0].empty()) {
        std::vector<int32_t> cnt((size_t)NDIR * n);
        CK(cudaMemcpyAsync(cnt.data(), dt.split_cnt, 4 * cnt.size(), cudaMemcpyDeviceToHost, h->stream));
        for (int k = 0; k < NDIR; ++k) {
            T.split[k].resize(flat);
            CK(cudaMemcpyAsync(T.split[k].data(), dt.split[k], 4 * flat, cudaMemcpyDeviceToHost, h->stream));
        }
        CK(cudaStreamSynchronize(h->stream));
        for (int k = 0; k < NDIR; ++k) T.split_cnt[k].assign(cnt.begin() + (size_t)k * n, cnt.begin() + (size_t)(k + 1) * n);
    }
    if (alias && T.alias.empty()) {
        T.alias.resize(n);
        T.point_with_alias.resize(n);
        CK(cudaMemcpyAsync(T.alias.data(), dt.alias, 4 * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(T.point_with_alias.data(), dt.pwa, 4 * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (levels && T.fwd_level.empty()) {
        T.fwd_level.resize(n);
        T.bwd_level.resize(n);
        CK(cudaMemcpyAsync(T.fwd_level.data(), dt.level[0], 4 * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(T.bwd_level.data(), dt.level[1], 4 * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    return MFCFD_OK;
}

}  // namespace

extern "C" {

int mfcfd_create(const mfcfd_params *params, int32_t n, const int32_t *status, const double *x,
                 const double *y, const double *z, const double *tan1, const double *tan2,
                 const double *nor, const int32_t *nbhs, const int32_t *conn,
                 const double *min_dist, mfcfd_handle **out) {
    return host_guard(nullptr, [&]() -> int {
        return create_impl(params, n, status, x, y, z, tan1, tan2, nor, nbhs, conn, min_dist, out, true);
    });
}

int mfcfd_prepare(const mfcfd_params *params, int32_t n, const int32_t *status, const double *x,
                  const double *y, const double *z, const double *tan1, const double *tan2,
                  const double *nor, const int32_t *nbhs, const int32_t *conn,
                  const double *min_dist, mfcfd_handle **out) {
    return host_guard(nullptr, [&]() -> int {
        if (!out) return MFCFD_ERR_ARG;
        *out = nullptr;
        if (!params || params->device < 0) return MFCFD_ERR_ARG;
        return create_impl(params, n, status, x, y, z, tan1, tan2, nor, nbhs, conn, min_dist, out, false);
    });
}

int mfcfd_device_bytes(mfcfd_handle *h, int64_t *bytes) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !bytes) return MFCFD_ERR_ARG;
        if (h->stream) {
            *bytes = h->bytes;
            return MFCFD_OK;
        }
        if (!h->staged) return fail(h, MFCFD_ERR_ARG, "handle has no staged cloud");
        // the attach sequence with allocation counted, not performed
        h->dry = true;
        h->bytes = 0;
        const int rc = attach_device(h);
        *bytes = h->bytes;
        h->dry = false;
        h->bytes = 0;
        std::memset(&h->d, 0, sizeof h->d);
        h->allocs.clear();
        return rc;
    });
}

int mfcfd_attach(mfcfd_handle *h) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h) return MFCFD_ERR_ARG;
        if (h->stream) return MFCFD_OK;
        if (!h->staged) return fail(h, MFCFD_ERR_ARG, "handle has no staged cloud");
        const int rc = attach_device(h);
        if (rc) {
            release(h);
            return rc;
        }
        h->staged.reset();
        return MFCFD_OK;
    });
}

int mfcfd_set_prim(mfcfd_handle *h, const double *prim) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !prim) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle was not created successfully");
        size_t n5 = (size_t)h->d.n * 5;
        int rc = rows_to_device(h, h->d.prim, prim, 5);
        if (rc) return rc;
        CK(cudaMemsetAsync(h->d.dUp, 0, n5 * 8, h->stream));
        CK(cudaMemsetAsync(h->d.dUn, 0, n5 * 8, h->stream));
        DevCloud dc = h->d;
        dc.U = h->U_buf[h->cur];
        dc.q = h->q_buf[h->cur];
        CK(launch_conserved_q(dc, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        h->last = h->cur;
        h->res_old = h->res_new = h->residue = 0.0;
        h->have_state = true;
        h->res_valid = false;
        return MFCFD_OK;
    });
}

int mfcfd_fpi_step(mfcfd_handle *h, int32_t t, double *res_new, double *residue) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle was not created successfully");
        double hist[2];
        int rc = run_iterations(h, t, 1, hist);
        if (res_new) *res_new = hist[0];
        if (residue) *residue = hist[1];
        return rc;
    });
}

int mfcfd_launch(mfcfd_handle *h, int32_t t0, int32_t iters) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || iters < 1) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle was not created successfully");
        if (!h->have_state) return fail(h, MFCFD_ERR_ARG, "no state: call mfcfd_set_prim first");
        if (h->pending_chunk) return fail(h, MFCFD_ERR_ARG, "a launch is already pending on this handle");
        if (iters > h->res_cap) return fail(h, MFCFD_ERR_ARG, "at most 1024 iterations per launch");
        CK(cudaSetDevice(h->P.device));
        if (!h->batch_ev) CK(cudaEventCreateWithFlags(&h->batch_ev, cudaEventDisableTiming));
        int rc = launch_chunk(h, iters, true);
        if (rc) return rc;
        CK(cudaEventRecord(h->batch_ev, h->stream));
        h->pending_chunk = iters;
        h->pending_t0 = t0;
        return MFCFD_OK;
    });
}

int mfcfd_complete(mfcfd_handle *h, int32_t wait, double *res_hist, int32_t *done) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !done) return MFCFD_ERR_ARG;
        *done = 0;
        if (!h->pending_chunk) return fail(h, MFCFD_ERR_ARG, "no launch is pending on this handle");
        if (!wait) {
            const cudaError_t q = cudaEventQuery(h->batch_ev);
            if (q == cudaErrorNotReady) return MFCFD_OK;
            if (q != cudaSuccess) return cuda_fail(h, q, "cudaEventQuery");
        }
        int st = MFCFD_OK;
        const int chunk = h->pending_chunk;
        h->pending_chunk = 0;
        int rc = finish_chunk(h, h->pending_t0, chunk, res_hist, &st);
        *done = 1;
        return rc ? rc : st;
    });
}

int mfcfd_run(mfcfd_handle *h, int32_t t0, int32_t iters, double *res_hist) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || iters < 0) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle was not created successfully");
        return run_iterations(h, t0, iters, res_hist);
    });
}

int mfcfd_get(mfcfd_handle *h, int32_t field, double *out) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !out) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle was not created successfully");
        const DevCloud &d = h->d;
        size_t n = (size_t)d.n;
        const double *src = nullptr;
        size_t w = 0;
        switch (field) {
        case MFCFD_FIELD_PRIM: src = d.prim; w = 5; break;
        case MFCFD_FIELD_U: src = h->U_buf[h->last]; w = 5; break;
        case MFCFD_FIELD_Q: src = h->q_buf[h->last]; w = 5; break;
        case MFCFD_FIELD_QM: src = d.qm; w = 10; break;
        case MFCFD_FIELD_DQ: src = d.dq; w = 15; break;
        case MFCFD_FIELD_DELT: src = d.delt; w = 1; break;
        case MFCFD_FIELD_FLUX_RES: src = d.flux_res; w = 5; break;
        case MFCFD_FIELD_DELUP: src = d.dUp; w = 5; break;
        case MFCFD_FIELD_DELUN: src = d.dUn; w = 5; break;
        case MFCFD_FIELD_DINV: src = d.dinv; w = 1; break;
        default: return fail(h, MFCFD_ERR_ARG, "unknown field");
        }
        (void)n;
        int rc = rows_to_host(h, out, src, (int)w);
        if (rc) return rc;
        CK(cudaStreamSynchronize(h->stream));
        return MFCFD_OK;
    });
}

int mfcfd_get_state(mfcfd_handle *h, double *prim, double *delu, double *res_old) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !prim || !delu) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle was not created successfully");
        size_t n5 = (size_t)h->d.n * 5;
        (void)n5;
        int rc = rows_to_host(h, prim, h->d.prim, 5);
        if (!rc) rc = rows_to_host(h, delu, h->d.dUn, 5);
        if (rc) return rc;
        CK(cudaStreamSynchronize(h->stream));
        if (res_old) *res_old = h->res_old;
        return MFCFD_OK;
    });
}

int mfcfd_set_state(mfcfd_handle *h, const double *prim, const double *delu, double res_old) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !prim || !delu) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle was not created successfully");
        size_t n5 = (size_t)h->d.n * 5;
        int rc = rows_to_device(h, h->d.prim, prim, 5);
        if (!rc) rc = rows_to_device(h, h->d.dUn, delu, 5);
        if (rc) return rc;
        CK(cudaMemcpyAsync(h->d.dUp, h->d.dUn, n5 * 8, cudaMemcpyDeviceToDevice, h->stream));
        DevCloud dc = h->d;
        dc.U = h->U_buf[h->cur];
        dc.q = h->q_buf[h->cur];
        CK(launch_conserved_q(dc, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        h->last = h->cur;
        h->res_old = res_old;
        h->have_state = true;
        h->res_valid = false;
        return MFCFD_OK;
    });
}

int mfcfd_get_stencils(mfcfd_handle *h, int32_t *counts, int32_t *lists, int32_t width) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !counts || !lists || width < 1) return MFCFD_ERR_ARG;
        const Topology &T = h->T;
        if (T.n == 0) return fail(h, MFCFD_ERR_ARG, "handle was not created successfully");
        if (int rc = fetch_query_arrays(h, true, false, false)) return rc;
        for (int i = 0; i < T.n; ++i)
            for (int dd = 0; dd < NDIR; ++dd) {
                int c = T.split_cnt[dd][i];
                counts[(size_t)i * NDIR + dd] = c;
                for (int j = 0; j < width; ++j)
                    lists[((size_t)i * NDIR + dd) * width + j] =
                        j < c ? T.split[dd][(size_t)i * T.cap + j] : 0;
            }
        return MFCFD_OK;
    });
}

int mfcfd_get_alias(mfcfd_handle *h, int32_t *alias, int32_t *point_with_alias) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !alias || !point_with_alias) return MFCFD_ERR_ARG;
        const Topology &T = h->T;
        if (T.n == 0) return fail(h, MFCFD_ERR_ARG, "handle was not created successfully");
        if (int rc = fetch_query_arrays(h, false, true, false)) return rc;
        std::memcpy(alias, T.alias.data(), sizeof(int32_t) * T.n);
        std::memcpy(point_with_alias, T.point_with_alias.data(), sizeof(int32_t) * T.n);
        return MFCFD_OK;
    });
}

int mfcfd_get_levels(mfcfd_handle *h, int32_t dir, int32_t *level) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !level || (dir != 0 && dir != 1)) return MFCFD_ERR_ARG;
        const Topology &T = h->T;
        if (T.n == 0) return fail(h, MFCFD_ERR_ARG, "handle was not created successfully");
        if (int rc = fetch_query_arrays(h, false, false, true)) return rc;
        const std::vector<int32_t> &src = dir == 0 ? T.fwd_level : T.bwd_level;
        if (T.perm.empty()) std::memcpy(level, src.data(), sizeof(int32_t) * T.n);
        else
            for (int i = 0; i < T.n; ++i) level[i] = src[T.perm[i]];
        return MFCFD_OK;
    });
}

int mfcfd_knn(int32_t device, int32_t n, const double *x, const double *y, const double *z, int32_t k,
              int32_t *nbhs, int32_t *conn, double *min_dist) {
    return host_guard(&g_io_err, [&]() -> int {
        if (!x || !y || !z || !nbhs || !conn || !min_dist) return MFCFD_ERR_ARG;
        g_io_err.clear();
        return knn_connectivity(device, n, x, y, z, k, nbhs, conn, min_dist, g_io_err);
    });
}

int mfcfd_debug_digest(mfcfd_handle *h, const char *name, uint64_t *digest, int64_t *bytes) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !name || !digest || !bytes) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle has no device state");
        const DevCloud &d = h->d;
        const size_t n = (size_t)d.n;
        int32_t ends[2] = {0, 0};
        if (d.fwd_off) CK(cudaMemcpy(&ends[0], d.fwd_off + n, 4, cudaMemcpyDeviceToHost));
        if (d.bwd_off) CK(cudaMemcpy(&ends[1], d.bwd_off + n, 4, cudaMemcpyDeviceToHost));
        const size_t nsw = (size_t)d.n_swept, w1 = (size_t)d.ch_warps + 1;
        const bool ch = d.sweep_mode == MFCFD_SWEEP_CHAINS;
        const struct {
            const char *name;
            const void *p;
            size_t bytes;
        } arrays[] = {
            {"x", d.x, 8 * n}, {"y", d.y, 8 * n}, {"z", d.z, 8 * n}, {"frame", d.frame, 72 * n},
            {"cls", d.cls, n}, {"nbhs", d.nbhs, 4 * n}, {"conn", d.conn, 4 * n * MAX_CONN},
            {"eps2", d.eps2, 8 * n}, {"slot_nbr", d.slot_nbr, 4 * n * MAX_SLOTS}, {"nslot", d.nslot, n},
            {"slot_mask", d.slot_mask, n * MAX_SLOTS}, {"list_cnt", d.list_cnt, n * NDIR},
            {"list_ent", d.list_ent, n * NDIR * LIST_STRIDE}, {"geo", d.geo, 8 * n * GEO_STRIDE},
            {"swept", d.swept, n}, {"consumer_shared", d.consumer_shared, n},
            {"fwd_lvl_ptr", d.fwd_lvl_ptr, 4 * ((size_t)d.n_fwd_levels + 1)}, {"fwd_lvl_pts", d.fwd_lvl_pts, 4 * nsw},
            {"bwd_lvl_ptr", d.bwd_lvl_ptr, 4 * ((size_t)d.n_bwd_levels + 1)}, {"bwd_lvl_pts", d.bwd_lvl_pts, 4 * nsw},
            {"fwd_off", d.fwd_off, 4 * (n + 1)}, {"bwd_off", d.bwd_off, 4 * (n + 1)},
            {"fwd_cnt", d.fwd_cnt, n * NDIR}, {"bwd_cnt", d.bwd_cnt, n * NDIR},
            {"fwd_ent", d.fwd_ent, sizeof(SweepEntry) * (size_t)ends[0]},
            {"bwd_ent", d.bwd_ent, sizeof(SweepEntry) * (size_t)ends[1]},
            {"fwd_need", d.fwd_need, 4 * n}, {"bwd_need", d.bwd_need, 4 * n},
            {"fwd_old", d.fwd_old, 4 * n}, {"bwd_old", d.bwd_old, 4 * n},
            {"sweep_slot_mask", d.sweep_slot_mask, n * MAX_SLOTS}, {"res_order", d.res_order, 4 * (size_t)d.n_res},
            {"pre_order", d.pre_order, ch ? 4 * n : 0}, {"g0_pts", d.g0_pts, 4 * (size_t)d.n_g0},
            {"ch_ptr0", d.ch_ptr[0], ch ? 4 * w1 : 0}, {"ch_pts0", d.ch_pts[0], ch ? 4 * nsw : 0},
            {"ch_own0", d.ch_own[0], ch ? 4 * n : 0}, {"ch_items0", d.ch_items[0], ch ? sizeof(ChainItem) * nsw : 0},
            {"ch_ptr1", d.ch_ptr[1], ch ? 4 * w1 : 0}, {"ch_pts1", d.ch_pts[1], ch ? 4 * nsw : 0},
            {"ch_own1", d.ch_own[1], ch ? 4 * n : 0}, {"ch_items1", d.ch_items[1], ch ? sizeof(ChainItem) * nsw : 0},
        };
        for (const auto &a : arrays) {
            if (std::strcmp(a.name, name) != 0) continue;
            std::vector<uint8_t> buf(a.bytes);
            if (a.bytes && a.p) CK(cudaMemcpy(buf.data(), a.p, a.bytes, cudaMemcpyDeviceToHost));
            uint64_t hsh = 14695981039346656037ull;   // FNV-1a
            for (uint8_t b : buf) hsh = (hsh ^ b) * 1099511628211ull;
            *digest = hsh;
            *bytes = a.p ? (int64_t)a.bytes : -1;
            return MFCFD_OK;
        }
        return fail(h, MFCFD_ERR_ARG, std::string("unknown array ") + name);
    });
}

int mfcfd_get_info(mfcfd_handle *h, mfcfd_info *info) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !info) return MFCFD_ERR_ARG;
        const Topology &T = h->T;
        std::memset(info, 0, sizeof *info);
        info->n_points = T.n;
        info->n_wall = (int32_t)T.wall_idx.size();
        info->n_outer = (int32_t)T.outer_idx.size();
        info->n_interior = (int32_t)T.interior_idx.size();
        info->n_supersonic = (int32_t)(T.ss_inlet_idx.size() + T.ss_outlet_idx.size());
        info->n_levels_forward = T.fwd_lvl_ptr.empty() ? 0 : (int32_t)T.fwd_lvl_ptr.size() - 1;
        info->n_levels_backward = T.bwd_lvl_ptr.empty() ? 0 : (int32_t)T.bwd_lvl_ptr.size() - 1;
        info->max_level_width = T.max_level_width;
        info->split_overflows = T.split_overflows;
        info->shared_frame = T.shared_frame;
        info->device_bytes = h->bytes;
        info->sweep_mode = h->P.sweep_mode;
        info->chain_warps = h->d.ch_warps;
        info->chain_terms_ring = h->chain_terms[0];
        info->chain_terms_local = h->chain_terms[1];
        info->chain_terms_cross = h->chain_terms[2];
        if (h->P.sweep_mode == MFCFD_SWEEP_CHAINS && h->P.device >= 0) {
            const int wpb = h->stream ? h->d.ch_wpb : (h->staged ? h->staged->ch_wpb : 0);
            const int w = h->stream ? h->d.ch_warps : (h->staged ? h->staged->ch_w : 0);
            info->chain_slots =
                wpb > 0 ? (w + wpb - 1) / wpb * chain_block_slots(h->P.device, wpb, h->P.precision,
                                                      h->P.chain_spread)
                        : 0;
            info->chain_slot_capacity = chain_slot_capacity(h->P.device);
            info->chain_warps_per_block = wpb;
            if (!info->chain_warps) info->chain_warps = w;
            info->g0_points = (int32_t)h->T.g0_pts.size();
        }
        return MFCFD_OK;
    });
}

int mfcfd_get_stream(mfcfd_handle *h, void **stream) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !stream) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle has no device state");
        *stream = (void *)h->stream;
        return MFCFD_OK;
    });
}

int mfcfd_set_profiling(mfcfd_handle *h, int32_t on) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle has no device state");
        if (on && h->ev.empty()) {
            h->ev.resize((size_t)h->res_cap * (MFCFD_NPHASE + 1));
            for (auto &e : h->ev) CK(cudaEventCreate(&e));
        }
        h->profiling = on != 0;
        for (double &v : h->phase_ms) v = 0.0;
        h->prof_iters = 0;
        return MFCFD_OK;
    });
}

int mfcfd_get_phase_times(mfcfd_handle *h, double *ms, int64_t *iters) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !ms) return MFCFD_ERR_ARG;
        for (int p = 0; p < MFCFD_NPHASE; ++p) ms[p] = h->phase_ms[p];
        if (iters) *iters = h->prof_iters;
        return MFCFD_OK;
    });
}

int mfcfd_residual_noalloc(mfcfd_handle *h, double *res_new) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !res_new) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle has no device state");
        if (!h->res_valid)
            return fail(h, MFCFD_ERR_ARG,
                        "no completed iteration since the state was last set (or the last one timed out)");
        cudaError_t e = cudaSetDevice(h->P.device);
        if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
        return residual_noalloc(h->d, h->stream, res_new, h->err);
    });
}

int mfcfd_set_precision(mfcfd_handle *h, int32_t precision) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h) return MFCFD_ERR_ARG;
        if (precision != MFCFD_PRECISION_FP64 && precision != MFCFD_PRECISION_MIXED_DC)
            return fail(h, MFCFD_ERR_ARG, "only FP64 and MIXED_DC can be switched to");
        if (h->P.precision == MFCFD_PRECISION_MIXED)
            return fail(h, MFCFD_ERR_UNSUPPORTED, "a MIXED handle keeps only its folded sweep weights");
        if (precision == MFCFD_PRECISION_MIXED_DC && h->P.sweep_mode != MFCFD_SWEEP_CHAINS)
            return fail(h, MFCFD_ERR_UNSUPPORTED, "mixed precision requires the chain sweep schedule");
        if (h->pending_chunk) return fail(h, MFCFD_ERR_ARG, "a launch is pending on this handle");
        if (precision == h->P.precision) return MFCFD_OK;
        if (h->stream) {
            // MIXED_DC sweeps read folded weights, FP64 ones the three
            // weighted offsets: put back the saved ones, or save and fold
            if (precision == MFCFD_PRECISION_MIXED_DC)
                for (int dir = 0; dir < 2; ++dir)
                    if (!h->w_saved[dir]) {
                        int rc = dalloc(h, &h->w_saved[dir], 3 * (size_t)std::max<int64_t>(h->n_ent[dir], 1));
                        if (rc) return rc;
                    }
            CK(launch_fold_terms(h->d, h->w_saved, precision == MFCFD_PRECISION_MIXED_DC, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
        h->P.precision = precision;
        h->d.precision = precision;
        drop_graphs(h);                    // their launches name the other kernels
        return MFCFD_OK;
    });
}

int mfcfd_set_fault_hook(mfcfd_handle *h, int32_t point, int32_t wait_limit) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || point < 0 || wait_limit < 0) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle has no device state");
        if (point > h->d.n) return fail(h, MFCFD_ERR_ARG, "point out of range");
        if (h->pending_chunk) return fail(h, MFCFD_ERR_ARG, "a launch is pending on this handle");
        h->d.withhold1 = point;
        h->d.spin_limit = wait_limit;
        drop_graphs(h);                    // their launches carry the old settings
        return MFCFD_OK;
    });
}

int mfcfd_run_batch(mfcfd_handle *const *hs, int32_t count, const int32_t *t0, int32_t iters, double *res_hist,
                    int32_t *status) {
    return host_guard(hs && count > 0 && hs[0] ? &hs[0]->err : nullptr, [&]() -> int {
        if (!hs || count < 1 || !t0 || iters < 0) return MFCFD_ERR_ARG;
        const int dev = hs[0] ? hs[0]->P.device : -1;
        for (int32_t i = 0; i < count; ++i) {
            mfcfd_handle *h = hs[i];
            if (!h || !h->stream || !h->have_state || h->P.device != dev) return MFCFD_ERR_ARG;
            for (int32_t j = 0; j < i; ++j)
                if (hs[j] == h) return MFCFD_ERR_ARG;   // each handle once
            if (status) status[i] = MFCFD_OK;
        }
        if (cudaSetDevice(dev) != cudaSuccess) return MFCFD_ERR_CUDA;
        const int capacity = chain_slot_capacity(dev);
        int first_err = MFCFD_OK;
        // Continuous scheduling on SM slots: a handle's next chunk starts as
        // soon as its chain blocks fit beside the chunks running, and a chunk's
        // slots return when its completion event has fired.  So all running
        // chain blocks are always resident together (see k_sweep_chain), and no
        // handle waits for a whole group of others to finish.
        std::vector<int32_t> done(count, 0);
        std::vector<int> chunk_of(count, 0);
        std::deque<int32_t> ready;
        std::vector<int32_t> running;
        for (int32_t i = 0; i < count; ++i) {
            if (iters > 0) ready.push_back(i);
            if (!hs[i]->batch_ev && cudaEventCreateWithFlags(&hs[i]->batch_ev, cudaEventDisableTiming) != cudaSuccess)
                return cuda_fail(hs[i], cudaGetLastError(), "cudaEventCreateWithFlags");
        }
        auto slots_of = [&](int32_t i) {
            const DevCloud &d = hs[i]->d;
            return d.sweep_mode == MFCFD_SWEEP_CHAINS
                       ? (d.ch_warps + d.ch_wpb - 1) / d.ch_wpb *
                             chain_block_slots(hs[i]->P.device, d.ch_wpb, d.precision,
                                               d.ch_spread)
                       : 0;
        };
        int used = 0;
        while (!ready.empty() || !running.empty()) {
            while (!ready.empty()) {
                const int32_t i = ready.front();
                const int sl = slots_of(i);
                if (!running.empty() && used + sl > capacity) break;
                ready.pop_front();
                mfcfd_handle *h = hs[i];
                const int chunk = std::min<int32_t>(iters - done[i], std::max(h->res_cap, 1));
                int rc = launch_chunk(h, chunk, true);
                if (rc) return rc;
                cudaError_t e = cudaEventRecord(h->batch_ev, h->stream);
                if (e != cudaSuccess) return cuda_fail(h, e, "cudaEventRecord");
                chunk_of[i] = chunk;
                used += sl;
                running.push_back(i);
            }
            // wait for the first of the running chunks to complete
            int found = -1;
            while (found < 0) {
                for (size_t r = 0; r < running.size() && found < 0; ++r) {
                    const cudaError_t q = cudaEventQuery(hs[running[r]]->batch_ev);
                    if (q == cudaSuccess) found = (int)r;
                    else if (q != cudaErrorNotReady) return cuda_fail(hs[running[r]], q, "cudaEventQuery");
                }
                if (found < 0) std::this_thread::sleep_for(std::chrono::microseconds(20));
            }
            const int32_t i = running[found];
            running.erase(running.begin() + found);
            used -= slots_of(i);
            int st = MFCFD_OK;
            double *rh = res_hist ? res_hist + 2 * ((size_t)i * iters + done[i]) : nullptr;
            int rc = finish_chunk(hs[i], t0[i] + done[i], chunk_of[i], rh, &st);
            if (!rc) rc = st;
            if (status && rc && status[i] == MFCFD_OK) status[i] = rc;
            if (rc && first_err == MFCFD_OK) first_err = rc;
            done[i] += chunk_of[i];
            if (done[i] < iters) ready.push_back(i);
        }
        return first_err;
    });
}

namespace {

// Streams and events of one mfcfd_run_group call, released on every path.
struct GroupRun {
    cudaStream_t s = nullptr;
    cudaEvent_t start = nullptr, bwd = nullptr;
    struct Graph {
        int chunk;
        std::vector<int> cur;
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs;
    ~GroupRun() {
        if (s) cudaStreamSynchronize(s);
        for (auto &g : graphs) cudaGraphExecDestroy(g.exec);
        if (start) cudaEventDestroy(start);
        if (bwd) cudaEventDestroy(bwd);
        if (s) cudaStreamDestroy(s);
    }
};

// The launches of `chunk` lockstep iterations of a group on gr.s: per
// iteration every handle's ITER_PRE on its own streams, the group's forward
// sweep once all of them may start, its backward sweep once every flux
// residual has ended, then every handle's ITER_POST.  All the handles'
// streams join gr.s at the end.
cudaError_t launch_group_chunk(mfcfd_handle *const *hs, int count, int chunk, GroupRun &gr, ChainGroup &G) {
    const DevCloud &d0 = hs[0]->d;
    cudaError_t e = cudaEventRecord(gr.start, gr.s);
    for (int i = 0; i < count && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(hs[i]->stream, gr.start, 0);
    for (int j = 0; j < chunk && e == cudaSuccess; ++j) {
        for (int i = 0; i < count && e == cudaSuccess; ++i) {
            mfcfd_handle *h = hs[i];
            DevCloud &dc = G.cloud[i];
            dc = h->d;
            dc.U = h->U_buf[h->cur];
            dc.q = h->q_buf[h->cur];
            const IterStreams st{h->stream, h->side, h->fork, h->join};
            e = launch_iteration(dc, j, st, h->U_buf[1 - h->cur], h->q_buf[1 - h->cur], nullptr, ITER_PRE);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(gr.s, h->fork, 0);
        }
        if (e == cudaSuccess) e = launch_chain_group(G, d0.ch_wpb, d0.precision, d0.ch_spread, 1, gr.s);
        for (int i = 0; i < count && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(gr.s, hs[i]->join, 0);
        if (e == cudaSuccess) e = launch_chain_group(G, d0.ch_wpb, d0.precision, d0.ch_spread, 0, gr.s);
        if (e == cudaSuccess) e = cudaEventRecord(gr.bwd, gr.s);
        for (int i = 0; i < count && e == cudaSuccess; ++i) {
            mfcfd_handle *h = hs[i];
            const IterStreams st{h->stream, h->side, h->fork, h->join};
            e = cudaStreamWaitEvent(h->stream, gr.bwd, 0);
            if (e == cudaSuccess)
                e = launch_iteration(G.cloud[i], j, st, h->U_buf[1 - h->cur], h->q_buf[1 - h->cur], nullptr,
                                     ITER_POST);
            h->last = h->cur;
            h->cur = 1 - h->cur;
        }
    }
    for (int i = 0; i < count && e == cudaSuccess; ++i) {
        e = cudaEventRecord(hs[i]->batch_ev, hs[i]->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(gr.s, hs[i]->batch_ev, 0);
    }
    return e;
}

}  // namespace

int mfcfd_run_group(mfcfd_handle *const *hs, int32_t count, const int32_t *t0, int32_t iters, double *res_hist,
                    int32_t *status) {
    return host_guard(hs && count > 0 && hs[0] ? &hs[0]->err : nullptr, [&]() -> int {
        if (!hs || count < 1 || count > MFCFD_GROUP_MAX_CLOUDS || !t0 || iters < 0) return MFCFD_ERR_ARG;
        const int dev = hs[0] ? hs[0]->P.device : -1;
        for (int32_t i = 0; i < count; ++i) {
            mfcfd_handle *h = hs[i];
            if (!h || !h->stream || !h->have_state || h->P.device != dev || h->pending_chunk) return MFCFD_ERR_ARG;
            for (int32_t j = 0; j < i; ++j)
                if (hs[j] == h) return MFCFD_ERR_ARG;   // each handle once
            if (status) status[i] = MFCFD_OK;
        }
        mfcfd_handle *h0 = hs[0];
        const DevCloud &d0 = h0->d;
        int slots = 0;
        for (int32_t i = 0; i < count; ++i) {
            const mfcfd_handle *h = hs[i];
            const DevCloud &d = h->d;
            if (d.sweep_mode != MFCFD_SWEEP_CHAINS)
                return fail(h0, MFCFD_ERR_UNSUPPORTED, "a group runs chain-schedule handles only");
            if (d.ch_wpb != d0.ch_wpb || d.ch_spread != d0.ch_spread ||
                (d.precision == MFCFD_PRECISION_FP64) != (d0.precision == MFCFD_PRECISION_FP64))
                return fail(h0, MFCFD_ERR_UNSUPPORTED,
                            "a group's handles share one chain block shape, chain_spread and precision class");
            if (h->profiling) return fail(h0, MFCFD_ERR_UNSUPPORTED, "phase timing is per handle, not in a group");
            slots += (d.ch_warps + d.ch_wpb - 1) / d.ch_wpb * chain_block_slots(dev, d.ch_wpb, d.precision, d.ch_spread);
        }
        mfcfd_handle *const h = h0;        // errors of the group's own calls
        if (cudaSetDevice(dev) != cudaSuccess) return MFCFD_ERR_CUDA;
        if (slots > chain_slot_capacity(dev))
            return fail(h0, MFCFD_ERR_UNSUPPORTED,
                        "the group's chain sweeps (" + std::to_string(slots) + " slots) do not fit the device (" +
                            std::to_string(chain_slot_capacity(dev)) + ")");
        if (!chain_group_fits(dev, d0.ch_wpb, d0.precision, d0.ch_spread))
            return fail(h, MFCFD_ERR_UNSUPPORTED, "the group sweep kernel holds fewer blocks per SM than a handle's");
        for (int32_t i = 0; i < count; ++i)
            if (!hs[i]->batch_ev && cudaEventCreateWithFlags(&hs[i]->batch_ev, cudaEventDisableTiming) != cudaSuccess)
                return cuda_fail(hs[i], cudaGetLastError(), "cudaEventCreateWithFlags");
        prepare_launches(dev);
        auto G = std::make_unique<ChainGroup>();
        G->count = count;
        G->block_start[0] = 0;
        for (int32_t i = 0; i < count; ++i)
            G->block_start[i + 1] = G->block_start[i] + (hs[i]->d.ch_warps + d0.ch_wpb - 1) / d0.ch_wpb;
        GroupRun gr;
        int lo = 0, hi = 0;
        CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        CK(cudaStreamCreateWithPriority(&gr.s, cudaStreamNonBlocking, hi));
        CK(cudaEventCreateWithFlags(&gr.start, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&gr.bwd, cudaEventDisableTiming));
        int res_cap = 1 << 30;
        bool graphs = true;
        for (int32_t i = 0; i < count; ++i) {
            res_cap = std::min(res_cap, std::max(hs[i]->res_cap, 1));
            graphs = graphs && hs[i]->P.graphs >= 1 && !hs[i]->graphs_off;
        }
        int first_err = MFCFD_OK;
        for (int32_t done = 0; done < iters;) {
            const int chunk = std::min<int32_t>(iters - done, res_cap);
            for (int32_t i = 0; i < count; ++i) hs[i]->res_valid = false;
            std::vector<int> cur(count), last(count);
            for (int32_t i = 0; i < count; ++i) cur[i] = hs[i]->cur, last[i] = hs[i]->last;
            GroupRun::Graph *g = nullptr;
            for (auto &x : gr.graphs)
                if (x.chunk == chunk && x.cur == cur) g = &x;
            if (!g && graphs) {
                cudaGraph_t graph = nullptr;
                cudaGraphExec_t exec = nullptr;
                cudaError_t e = cudaStreamBeginCapture(gr.s, cudaStreamCaptureModeThreadLocal);
                if (e == cudaSuccess) {
                    const cudaError_t el = launch_group_chunk(hs, count, chunk, gr, *G);
                    e = cudaStreamEndCapture(gr.s, &graph);
                    if (e == cudaSuccess) e = el;
                }
                if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
                if (graph) cudaGraphDestroy(graph);
                for (int32_t i = 0; i < count; ++i) hs[i]->cur = cur[i], hs[i]->last = last[i];
                if (e == cudaSuccess && exec) {
                    gr.graphs.push_back({chunk, cur, exec});
                    g = &gr.graphs.back();
                } else {
                    (void)cudaGetLastError();   // launch one by one from here on
                    graphs = false;
                }
            }
            if (g) {
                CK(cudaGraphLaunch(g->exec, gr.s));
                for (int32_t i = 0; i < count; ++i) {
                    hs[i]->last = (chunk & 1) ? cur[i] : 1 - cur[i];
                    hs[i]->cur = (chunk & 1) ? 1 - cur[i] : cur[i];
                }
            } else {
                CK(launch_group_chunk(hs, count, chunk, gr, *G));
            }
            CK(cudaStreamSynchronize(gr.s));
            for (int32_t i = 0; i < count; ++i) {
                int st = MFCFD_OK;
                double *rh = res_hist ? res_hist + 2 * ((size_t)i * iters + done) : nullptr;
                int rc = finish_chunk(hs[i], t0[i] + done, chunk, rh, &st);
                if (!rc) rc = st;
                if (status && rc && status[i] == MFCFD_OK) status[i] = rc;
                if (rc && first_err == MFCFD_OK) first_err = rc;
            }
            done += chunk;
        }
        return first_err;
    });
}

int mfcfd_set_chain_warps(mfcfd_handle *h, int32_t warps, int32_t *actual) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || warps < 1) return MFCFD_ERR_ARG;
        if (h->P.sweep_mode != MFCFD_SWEEP_CHAINS) return fail(h, MFCFD_ERR_ARG, "the handle does not use the chain schedule");
        if (h->stream) {
            CK(cudaSetDevice(h->P.device));
            int w = 0;
            const int rc = apply_chain_schedule(h, warps, &w);
            if (rc) return rc;
            if (actual) *actual = w;
            return MFCFD_OK;
        }
        if (!h->staged) return fail(h, MFCFD_ERR_ARG, "handle has no device state");
        // a prepared handle: rebuild the staged schedule before it is attached
        mfcfd_handle::Staged &st = *h->staged;
        int blocks = 0;
        const int w = chain_shape(h->P.device, warps, h->P.chain_spread, &st.ch_wpb, &blocks);
        if (w < 1) return fail(h, MFCFD_ERR_CUDA, "chain sweep kernel cannot be resident");
        st.S = ChainSchedule();   // built for w at the next dry run or attach
        st.ch_w = w;
        if (actual) *actual = w;
        return MFCFD_OK;
    });
}

int mfcfd_tune_chain(mfcfd_handle *h, const int32_t *candidates, int32_t count, int32_t iters, int32_t *chosen,
                     double *ms) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !chosen || iters < 1 || iters > 1000 || count < 0 || (count > 0 && !candidates)) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle has no device state");
        if (!h->have_state) return fail(h, MFCFD_ERR_ARG, "no state: call mfcfd_set_prim first");
        if (h->d.sweep_mode != MFCFD_SWEEP_CHAINS) return fail(h, MFCFD_ERR_ARG, "tuning applies to the chain schedule");
        CK(cudaSetDevice(h->P.device));
        std::vector<int> wants;
        if (count == 0) {
            const int width = std::max(1, h->T.max_level_width);
            for (int num : {3, 4, 6, 8}) wants.push_back(std::max(1, num * width / 2));   // 1.5x .. 4x the widest level
        } else {
            for (int32_t i = 0; i < count; ++i) {
                if (candidates[i] < 1) return fail(h, MFCFD_ERR_ARG, "candidate warp counts must be positive");
                wants.push_back(candidates[i]);
            }
        }
        const size_t n5 = (size_t)h->d.n * 5;
        std::vector<double> prim(n5), delu(n5);
        double res_old = 0.0;
        int rc = mfcfd_get_state(h, prim.data(), delu.data(), &res_old);
        if (rc) return rc;
        const int start = h->d.ch_warps;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        double best_ms = 0.0;
        int best = start;
        for (size_t c = 0; c < wants.size() && rc == MFCFD_OK; ++c) {
            int w = 0;
            if ((rc = apply_chain_schedule(h, wants[c], &w))) break;
            // one untimed iteration, then `iters` timed ones, from the saved state
            if ((rc = mfcfd_set_state(h, prim.data(), delu.data(), res_old))) break;
            if ((rc = run_iterations(h, 3, 1, nullptr))) break;
            if ((rc = mfcfd_set_state(h, prim.data(), delu.data(), res_old))) break;
            cudaEventRecord(e0, h->stream);
            if ((rc = run_iterations(h, 3, iters, nullptr))) break;
            cudaEventRecord(e1, h->stream);
            cudaEventSynchronize(e1);
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            const double per = t / iters;
            if (ms) ms[c] = per;
            if (c == 0 || per < best_ms) {
                best_ms = per;
                best = w;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        // keep the fastest schedule (or the original one after a failure)
        int w = 0;
        const int ra = apply_chain_schedule(h, rc == MFCFD_OK ? best : start, &w);
        if (ra && rc == MFCFD_OK) rc = ra;
        const int rs = mfcfd_set_state(h, prim.data(), delu.data(), res_old);
        if (rc == MFCFD_OK) rc = rs;
        *chosen = h->d.ch_warps;
        return rc;
    });
}

int mfcfd_set_wall_areas(mfcfd_handle *h, const double *area) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle has no device state");
        CK(cudaSetDevice(h->P.device));
        if (!area) {
            h->wall_area = nullptr;   // the allocation stays with the handle
            return MFCFD_OK;
        }
        if (!h->wall_area) {
            int rc = dalloc(h, &h->wall_area, (size_t)h->d.n);
            if (rc) return rc;
        }
        int rc = rows_to_device(h, h->wall_area, area, 1);
        if (rc) return rc;
        CK(cudaStreamSynchronize(h->stream));
        return MFCFD_OK;
    });
}

int mfcfd_forces(mfcfd_handle *h, double wall_area, double ref_area, double *cl, double *cd, double *force) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle has no device state");
        if (!h->have_state) return fail(h, MFCFD_ERR_ARG, "no state: call mfcfd_set_prim first");
        if (!(ref_area > 0.0)) return fail(h, MFCFD_ERR_ARG, "ref_area must be positive");
        if (!h->wall_area && (h->d.n_wall < 1 || !(wall_area > 0.0)))
            return fail(h, MFCFD_ERR_ARG, "wall_area must be positive (or set per-point areas)");
        CK(cudaSetDevice(h->P.device));
        if (!h->force_out) {
            int rc = dalloc(h, &h->force_out, 3);
            if (rc) return rc;
        }
        const double each = h->d.n_wall > 0 ? wall_area / h->d.n_wall : 0.0;
        CK(launch_forces(h->d, h->stream, each, h->wall_area, h->force_out));
        double F[3];
        CK(cudaMemcpyAsync(F, h->force_out, sizeof F, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        const double u1 = h->P.u1_inf, u2 = h->P.u2_inf, u3 = h->P.u3_inf;
        const double v = std::sqrt(u1 * u1 + u2 * u2 + u3 * u3);
        const double sa = v > 0.0 ? u2 / v : 0.0, ca = v > 0.0 ? u1 / v : 1.0;
        const double q = 0.5 * h->P.rho_inf * v * v * ref_area;
        if (cl) *cl = (F[0] * (-sa) + F[1] * ca) / q;
        if (cd) *cd = (F[0] * ca + F[1] * sa) / q;
        if (force) { force[0] = F[0]; force[1] = F[1]; force[2] = F[2]; }
        return MFCFD_OK;
    });
}

int mfcfd_destroy(mfcfd_handle *h) {
    if (!h) return MFCFD_ERR_ARG;
    release(h);
    delete h;
    return MFCFD_OK;
}

const char *mfcfd_last_error(const mfcfd_handle *h) {
    if (!h) return g_io_err.c_str();
    return h->err.c_str();
}

const char *mfcfd_strerror(int code) {
    if (code < 0 || code > MFCFD_ERR_BUSY) return "unknown error";
    return kStrerr[code];
}

int mfcfd_count_input_points(const char *path, int32_t *n) {
    return host_guard(&g_io_err, [&]() -> int {
        if (!path || !n) return MFCFD_ERR_ARG;
        return io_count_input_points(path, n);
    });
}

int mfcfd_read_input_point_data(const char *path, int32_t n, int32_t *status, double *x, double *y,
                                double *z, double *tan1, double *tan2, double *nor, int32_t *nbhs,
                                int32_t *conn, double *min_dist) {
    return host_guard(&g_io_err, [&]() -> int {
        if (!path || n < 1 || !status || !x || !y || !z || !tan1 || !tan2 || !nor || !nbhs || !conn || !min_dist)
            return MFCFD_ERR_ARG;
        return io_read_input_point_data(path, n, status, x, y, z, tan1, tan2, nor, nbhs, conn, min_dist);
    });
}

int mfcfd_read_stored_solution(const char *path, int32_t n, double *prim) {
    return host_guard(&g_io_err, [&]() -> int {
        if (!path || n < 1 || !prim) return MFCFD_ERR_ARG;
        return io_read_stored_solution(path, n, prim);
    });
}

int mfcfd_print_primal_output(mfcfd_handle *h, const char *dir) {
    return host_guard(h ? &h->err : nullptr, [&]() -> int {
        if (!h || !dir) return MFCFD_ERR_ARG;
        if (!h->stream) return fail(h, MFCFD_ERR_ARG, "handle has no device state");
        const size_t n = (size_t)h->d.n;
        std::vector<double> x(n), y(n), z(n), prim(5 * n), flux(5 * n), dq(15 * n);
        int rc = rows_to_host(h, x.data(), h->d.x, 1);
        if (!rc) rc = rows_to_host(h, y.data(), h->d.y, 1);
        if (!rc) rc = rows_to_host(h, z.data(), h->d.z, 1);
        if (!rc) rc = rows_to_host(h, prim.data(), h->d.prim, 5);
        if (!rc) rc = rows_to_host(h, flux.data(), h->d.flux_res, 5);
        if (!rc) rc = rows_to_host(h, dq.data(), h->d.dq, 15);
        if (rc) return rc;
        CK(cudaStreamSynchronize(h->stream));
        std::vector<int32_t> status(n);
        const std::vector<int32_t> &perm = h->T.perm;   // statuses 0/1/2 are the classes
        for (size_t i = 0; i < n; ++i) status[i] = h->T.cls[perm.empty() ? i : (size_t)perm[i]];
        rc = io_write_primal_output(dir, (int32_t)n, status.data(), x.data(), y.data(), z.data(), prim.data(),
                                        flux.data(), dq.data());
        if (rc) return fail(h, rc, g_io_err);
        return MFCFD_OK;
    });
}

int mfcfd_write_residue(const char *path, int32_t t0, int32_t iters, const double *res_hist, int32_t append) {
    return host_guard(&g_io_err, [&]() -> int {
        if (!path || iters < 0 || (iters > 0 && !res_hist)) return MFCFD_ERR_ARG;
        return io_write_residue(path, t0, iters, res_hist, append);
    });
}

}  // extern "C"
