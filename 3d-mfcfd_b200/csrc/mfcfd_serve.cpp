/*
 * mfcfd_serve.cpp - the request server of include/mfcfd.h (continuous
 * batching of steady-state solves on one GPU), built on the public C ABI.
 *
 * Threads: `setup_threads` workers run the host set-up of submitted clouds
 * (mfcfd_prepare) and measure their device footprint (mfcfd_device_bytes);
 * one scheduler thread launches and polls.  It admits ready requests
 * (first ready, first admitted) while their bytes fit the budget beside the
 * live ones, launches the next `chunk` iterations of every idle live
 * request whose chain sweep fits beside the running ones (mfcfd_launch;
 * their streams overlap on the device), and as each chunk completes
 * (mfcfd_complete) lets the request go on, or hands it back for retirement
 * if it converged, reached max_iters or failed.  The workers also attach
 * admitted requests (uploads, allocation) and retire finished ones (state
 * copy-out, freeing), before any set-up, so the scheduler thread spends
 * its time on launches and completions.  No request waits for the others.  Every request iterates in whole chunks of `chunk` from
 * t = 1, so its arithmetic, and its result, do not depend on which other
 * requests share the device.
 */
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "mfcfd_internal.h"

namespace {

struct Request {
    int64_t id = 0;
    mfcfd_params P{};
    int32_t n = 0;
    std::vector<int32_t> status, nbhs, conn;
    std::vector<double> x, y, z, tan1, tan2, nor, min_dist, prim0;
    int32_t max_iters = 0;
    double target = 0.0, wall_area = 0.0, ref_area = 0.0;
    double polish = 0.0;              // MIXED_DC: residue at which it switches to FP64 (0: never)
    bool polished = false;
    mfcfd_handle *h = nullptr;
    int64_t bytes = 0;
    int32_t t = 1;                    // next iteration number
    mfcfd_result res{};
    std::vector<double> prim_out;
    std::string err;
    bool done = false;
    int slots = 0;                    // SM slots of its chain sweep (mfcfd_info)
    int slot_capacity = 0;            // the device's chain slots (mfcfd_info)
    bool running = false;             // a chunk is launched and not yet completed
    double t_launch = 0.0;            // server clock at its running chunk's launch
    bool retiring = false;            // finished: to be handed to the workers for retirement
    bool handed = false;              // queued for retirement (no longer live)
    int fail = MFCFD_OK;              // status it retires with
};
using RequestPtr = std::shared_ptr<Request>;

// A request's error message, kept if host memory allows.
void set_message(std::string &to, const char *msg) noexcept {
    try {
        to = msg;
    } catch (...) {
    }
}

}  // namespace

struct mfcfd_server {
    mfcfd_server_config cfg{};
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_setup, cv_sched, cv_done;
    std::deque<RequestPtr> to_prepare;   // submitted, not yet taken by a worker
    std::deque<RequestPtr> ready;        // prepared, in the order they became ready
    std::deque<RequestPtr> to_attach;    // admitted (memory reserved), for a worker to attach
    std::deque<RequestPtr> attached;     // attached, for the scheduler to take live
    std::deque<RequestPtr> to_retire;    // finished, for a worker to retire
    uint64_t events = 0;                 // bumped when the scheduler has something new to do
    std::map<int64_t, RequestPtr> all;   // every request not yet returned by wait
    std::vector<RequestPtr> live;        // scheduler thread only
    int64_t next_id = 1;
    int64_t preparing = 0, n_live = 0;
    bool stopping = false;
    mfcfd_server_stats st{};
    std::vector<std::thread> workers;
    std::thread scheduler;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    // Bookkeeping of a retired request (caller holds mu).
    void finish_locked(const RequestPtr &r, int status) {
        r->res.status = status;
        r->res.t_done = now();
        r->done = true;
        if (status == MFCFD_OK) ++st.completed;
        else ++st.failed;
        cv_done.notify_all();
    }

    void worker_loop();
    void scheduler_loop();
    int create_on_device(const RequestPtr &r);
    void retire(const RequestPtr &r, int status);
    int submit(const mfcfd_request *q, int64_t *id);
};

// device_setup: the request's handle made on the device when it is admitted
// (its inputs were kept); the reservation becomes the handle's own bytes.
int mfcfd_server::create_on_device(const RequestPtr &r) {
    mfcfd_params P = r->P;
    P.device = cfg.device;
    P.gpu_setup = 1;
    mfcfd_handle *h = nullptr;
    int rc = mfcfd_create(&P, r->n, r->status.data(), r->x.data(), r->y.data(), r->z.data(), r->tan1.data(),
                          r->tan2.data(), r->nor.data(), r->nbhs.data(), r->conn.data(), r->min_dist.data(), &h);
    if (!rc && cfg.chain_percent > 0 && P.sweep_mode == MFCFD_SWEEP_CHAINS) {
        mfcfd_info info;
        rc = mfcfd_get_info(h, &info);
        if (!rc)
            rc = mfcfd_set_chain_warps(h, std::max(4, (int)((int64_t)info.max_level_width * cfg.chain_percent / 100)),
                                       nullptr);
    }
    int64_t bytes = 0;
    if (!rc) rc = mfcfd_device_bytes(h, &bytes);
    if (rc && h) set_message(r->err, mfcfd_last_error(h));
    std::vector<int32_t>().swap(r->status);
    std::vector<int32_t>().swap(r->nbhs);
    std::vector<int32_t>().swap(r->conn);
    for (auto *v : {&r->x, &r->y, &r->z, &r->tan1, &r->tan2, &r->nor, &r->min_dist}) std::vector<double>().swap(*v);
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!rc) {
            st.bytes_live += bytes - r->bytes;
            st.peak_bytes_live = std::max(st.peak_bytes_live, st.bytes_live);
            r->bytes = bytes;
            r->res.device_bytes = bytes;
        }
    }
    r->h = h;   // destroyed with the request on failure too
    return rc;
}

void mfcfd_server::worker_loop() {
    for (;;) {
        RequestPtr r;
        enum { RETIRE, ATTACH, PREPARE } job;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_setup.wait(lk, [&] {
                return stopping || !to_retire.empty() || !to_attach.empty() || !to_prepare.empty();
            });
            if (stopping) return;
            // freeing memory first, then the requests already admitted
            std::deque<RequestPtr> &q = !to_retire.empty() ? to_retire : !to_attach.empty() ? to_attach : to_prepare;
            job = &q == &to_retire ? RETIRE : &q == &to_attach ? ATTACH : PREPARE;
            r = q.front();
            q.pop_front();
            if (job == PREPARE) ++preparing;
        }
        if (job == RETIRE) {
            retire(r, r->fail);
            continue;
        }
        if (job == ATTACH) {
            int rc = MFCFD_OK;
            if (cfg.device_setup) {
                rc = create_on_device(r);
            } else {
                rc = mfcfd_attach(r->h);
            }
            if (!rc) rc = mfcfd_set_prim(r->h, r->prim0.data());
            std::vector<double>().swap(r->prim0);
            mfcfd_info info;
            if (!rc) rc = mfcfd_get_info(r->h, &info);
            if (rc) {
                retire(r, rc);
                continue;
            }
            r->slots = info.chain_slots;
            r->slot_capacity = info.chain_slot_capacity;
            bool queued = false;
            {
                std::lock_guard<std::mutex> lk(mu);
                try {
                    attached.push_back(r);
                    queued = true;
                } catch (...) {
                }
                ++events;
                cv_sched.notify_one();
            }
            if (!queued) retire(r, MFCFD_ERR_NOMEM);
            continue;
        }
        if (cfg.device_setup) {
            // set up at admission: reserve an estimate of its device bytes
            const int64_t bytes = (int64_t)r->n * MFCFD_DEVICE_SETUP_BYTES_PER_POINT;
            std::lock_guard<std::mutex> lk(mu);
            --preparing;
            r->res.t_ready = now();
            r->res.device_bytes = bytes;
            int rc = MFCFD_OK;
            if (bytes > cfg.hbm_budget) {
                rc = MFCFD_ERR_NOMEM;
                set_message(r->err, "the request needs more device memory than the server's budget");
            } else {
                try {
                    ready.push_back(r);
                } catch (...) {
                    rc = MFCFD_ERR_NOMEM;
                }
            }
            if (rc) {
                finish_locked(r, rc);
            } else {
                r->bytes = bytes;
                ++events;
                cv_sched.notify_one();
            }
            continue;
        }
        mfcfd_params P = r->P;
        P.device = cfg.device;
        mfcfd_handle *h = nullptr;
        // this worker's own core counts against the set-up pool, so that the
        // passes of requests prepared at once share the host's cores
        const int own = mfcfd::take_setup_threads(1);
        int rc = mfcfd_prepare(&P, r->n, r->status.data(), r->x.data(), r->y.data(), r->z.data(), r->tan1.data(),
                               r->tan2.data(), r->nor.data(), r->nbhs.data(), r->conn.data(), r->min_dist.data(),
                               &h);
        mfcfd::give_setup_threads(own);
        if (!rc && cfg.chain_percent > 0 && P.sweep_mode == MFCFD_SWEEP_CHAINS) {
            mfcfd_info info;
            rc = mfcfd_get_info(h, &info);
            if (!rc)
                rc = mfcfd_set_chain_warps(h, std::max(4, (int)((int64_t)info.max_level_width * cfg.chain_percent / 100)),
                                           nullptr);
        }
        int64_t bytes = 0;
        if (!rc) rc = mfcfd_device_bytes(h, &bytes);
        if (rc && h) set_message(r->err, mfcfd_last_error(h));
        // the handle holds what the device needs; the request keeps prim0
        std::vector<int32_t>().swap(r->status);
        std::vector<int32_t>().swap(r->nbhs);
        std::vector<int32_t>().swap(r->conn);
        for (auto *v : {&r->x, &r->y, &r->z, &r->tan1, &r->tan2, &r->nor, &r->min_dist})
            std::vector<double>().swap(*v);
        if (!rc && bytes > cfg.hbm_budget) {
            rc = MFCFD_ERR_NOMEM;
            set_message(r->err, "the request needs more device memory than the server's budget");
        }
        std::lock_guard<std::mutex> lk(mu);
        --preparing;
        r->res.t_ready = now();
        r->res.device_bytes = bytes;
        if (!rc) {
            try {
                ready.push_back(r);
            } catch (...) {
                rc = MFCFD_ERR_NOMEM;
            }
        }
        if (rc && h) {
            mfcfd_destroy(h);
            h = nullptr;
        }
        if (rc) {
            finish_locked(r, rc);
        } else {
            r->h = h;
            r->bytes = bytes;
            ++events;
            cv_sched.notify_one();
        }
    }
}

// Copy out the state and forces of an admitted request, free its device
// memory and record the result (a worker; the scheduler thread when
// stopping).
void mfcfd_server::retire(const RequestPtr &r, int status) {
    if (r->h) {
        if (status == MFCFD_OK && r->wall_area > 0.0 && r->ref_area > 0.0) {
            const int rc = mfcfd_forces(r->h, r->wall_area, r->ref_area, &r->res.cl, &r->res.cd, nullptr);
            if (rc) status = rc;
        }
        if (status == MFCFD_OK) {
            int rc = mfcfd::host_guard(&r->err, [&]() -> int {
                r->prim_out.resize((size_t)r->n * 5);
                return MFCFD_OK;
            });
            if (!rc) rc = mfcfd_get(r->h, MFCFD_FIELD_PRIM, r->prim_out.data());
            if (rc) status = rc;
        }
        if (status != MFCFD_OK && r->err.empty()) set_message(r->err, mfcfd_last_error(r->h));
        mfcfd_destroy(r->h);
        r->h = nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    st.bytes_live -= r->bytes;
    --n_live;
    finish_locked(r, status);
    ++events;   // memory freed: waiting requests may fit
    cv_sched.notify_one();
}

void mfcfd_server::scheduler_loop() {
    cudaSetDevice(cfg.device);
    const int chunk = cfg.chunk;
    std::vector<double> hist(2 * (size_t)chunk);
    int used = 0, running = 0, capacity = 0;
    double t_acc = now();   // slot-seconds and busy time accumulated up to here
    auto account = [&] {
        const double t = now(), dt = t - t_acc;
        t_acc = t;
        std::lock_guard<std::mutex> lk(mu);
        if (running > 0) st.busy_s += dt;
        st.slot_s += used * dt;
        st.slot_capacity = capacity;
    };
    auto wait_running = [&] {   // let every launched chunk finish (stopping)
        for (const RequestPtr &r : live)
            if (r->running) {
                int32_t done = 0;
                mfcfd_complete(r->h, 1, nullptr, &done);
                r->running = false;
            }
    };
    // Every allocation of a pass comes before the state it would change, so
    // an exception (host memory exhausted) leaves each request in exactly one
    // place; the pass is then tried again.
    std::vector<RequestPtr> finished;
    for (;;) {
        try {
            account();
            finished.clear();
            finished.reserve(live.size());
            // admissions: ready requests in order while memory (and max_live)
            // allow, handed to the workers to attach; attached ones go live
            uint64_t seen = 0;
            bool progress = false;
            {
                std::unique_lock<std::mutex> lk(mu);
                if (stopping) break;
                seen = events;
                int admitted = 0;
                while (!ready.empty()) {
                    const RequestPtr &r = ready.front();
                    if (cfg.max_live > 0 && n_live >= cfg.max_live) break;
                    if (st.bytes_live + r->bytes > cfg.hbm_budget) break;
                    to_attach.push_back(r);
                    r->res.t_admit = now();
                    st.bytes_live += r->bytes;
                    ++n_live;
                    ready.pop_front();
                    ++admitted;
                }
                if (admitted) cv_setup.notify_all();
                st.peak_bytes_live = std::max(st.peak_bytes_live, st.bytes_live);
                st.peak_live = std::max(st.peak_live, n_live);
                live.reserve(live.size() + attached.size());
                finished.reserve(live.size() + attached.size());
                progress = !attached.empty();
                for (const RequestPtr &r : attached) {
                    if (r->slot_capacity > 0) capacity = r->slot_capacity;
                    live.push_back(r);
                }
                attached.clear();
            }

            // launches: the next chunk of every idle request whose chain sweeps
            // fit beside the running ones (one always may run)
            for (const RequestPtr &r : live) {
                if (r->running || r->retiring) continue;
                if (running > 0 && used + r->slots > capacity) continue;
                const int rc = mfcfd_launch(r->h, r->t, chunk);
                progress = true;
                if (rc) {
                    r->fail = rc;
                    r->retiring = true;
                    continue;
                }
                account();
                r->running = true;
                r->t_launch = now();
                used += r->slots;
                ++running;
            }

            // completions: each request goes on by itself, or is retired
            for (const RequestPtr &r : live) {
                if (!r->running) continue;
                int32_t done = 0;
                const int rc = mfcfd_complete(r->h, 0, hist.data(), &done);
                if (!done && rc == MFCFD_OK) continue;
                progress = true;
                account();
                r->res.run_s += now() - r->t_launch;
                r->running = false;
                used -= r->slots;
                --running;
                {
                    std::lock_guard<std::mutex> lk(mu);
                    ++st.rounds;
                    st.iterations += chunk;
                }
                r->t += chunk;
                r->res.iters += chunk;
                r->res.res_new = hist[2 * (size_t)(chunk - 1)];
                r->res.residue = hist[2 * (size_t)(chunk - 1) + 1];
                r->res.converged = rc == MFCFD_OK && r->t - 1 > 2 && r->res.residue <= r->target;
                if (rc != MFCFD_OK) r->fail = rc;
                if (rc != MFCFD_OK || r->res.converged || r->res.iters >= r->max_iters) r->retiring = true;
                if (!r->retiring && !r->polished && r->polish < 0.0 && r->P.precision == MFCFD_PRECISION_MIXED_DC &&
                    r->t - 1 > 2 && r->res.residue <= r->polish) {
                    // the last part of the solve in FP64 (its chain blocks may
                    // take other slots)
                    r->polished = true;
                    int prc = mfcfd_set_precision(r->h, MFCFD_PRECISION_FP64);
                    mfcfd_info info{};
                    if (prc == MFCFD_OK) prc = mfcfd_get_info(r->h, &info);
                    if (prc != MFCFD_OK) {
                        r->fail = prc;
                        r->retiring = true;
                    } else {
                        r->slots = info.chain_slots;
                    }
                }
            }

            // hand the finished requests to the workers; one that could not be
            // queued stays live (not launched) and is handed over next pass
            for (const RequestPtr &r : live)
                if (r->retiring) finished.push_back(r);
            if (!finished.empty()) {
                {
                    std::lock_guard<std::mutex> lk(mu);
                    try {
                        for (const RequestPtr &r : finished) {
                            to_retire.push_back(r);
                            r->handed = true;
                        }
                    } catch (...) {
                    }
                    cv_setup.notify_all();
                }
                live.erase(std::remove_if(live.begin(), live.end(), [](const RequestPtr &r) { return r->handed; }),
                           live.end());
            }
            if (!progress) {
                // nothing to do: poll the running chunks (or hand over finished
                // requests) again shortly, or sleep until a request is ready,
                // attached or retired
                std::unique_lock<std::mutex> lk(mu);
                auto changed = [&] { return stopping || events != seen; };
                if (running > 0 || !live.empty()) {
                    cv_sched.wait_for(lk, std::chrono::microseconds(50), changed);
                } else {
                    cv_sched.wait(lk, changed);
                    t_acc = now();   // idle, with nothing running
                }
            }
        } catch (...) {
            // host memory ran out in this pass: try again a little later
            std::this_thread::sleep_for(std::chrono::milliseconds(1));
        }
    }
    // stopping: running chunks finish, then every live request ends
    wait_running();
    for (const RequestPtr &r : live) retire(r, MFCFD_ERR_BUSY);
    live.clear();
}

extern "C" {

int mfcfd_server_create(const mfcfd_server_config *cfg, mfcfd_server **out) {
    if (!out) return MFCFD_ERR_ARG;
    *out = nullptr;
    if (!cfg || cfg->device < 0 || cfg->max_live < 0 || cfg->setup_threads < 1 || cfg->setup_threads > 64 ||
        cfg->chunk < 1 || cfg->chunk > 1024 || cfg->hbm_budget < 0 || cfg->chain_percent < 0 ||
        cfg->chain_percent > 1000 || cfg->device_setup < 0 || cfg->device_setup > 1)
        return MFCFD_ERR_ARG;
    if (cudaSetDevice(cfg->device) != cudaSuccess) return MFCFD_ERR_CUDA;
    auto *s = new (std::nothrow) mfcfd_server();
    if (!s) return MFCFD_ERR_NOMEM;
    s->cfg = *cfg;
    if (s->cfg.hbm_budget == 0) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            delete s;
            return MFCFD_ERR_CUDA;
        }
        s->cfg.hbm_budget = (int64_t)(0.9 * (double)free_b);
    }
    s->st.hbm_budget = s->cfg.hbm_budget;
    s->t0 = std::chrono::steady_clock::now();
    const int rc = mfcfd::host_guard(nullptr, [&]() -> int {
        s->workers.reserve((size_t)cfg->setup_threads);
        for (int i = 0; i < cfg->setup_threads; ++i) s->workers.emplace_back([s] { s->worker_loop(); });
        s->scheduler = std::thread([s] { s->scheduler_loop(); });
        return MFCFD_OK;
    });
    if (rc) {
        // a thread could not be started: stop the ones that were
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stopping = true;
        }
        s->cv_setup.notify_all();
        s->cv_sched.notify_all();
        for (std::thread &w : s->workers) w.join();
        if (s->scheduler.joinable()) s->scheduler.join();
        delete s;
        return rc;
    }
    *out = s;
    return MFCFD_OK;
}

int mfcfd_server_submit(mfcfd_server *s, const mfcfd_request *q, int64_t *id) {
    if (!s || !q || !id || q->n < 1 || !q->status || !q->x || !q->y || !q->z || !q->tan1 || !q->tan2 ||
        !q->nor || !q->nbhs || !q->conn || !q->min_dist || q->max_iters < 1)
        return MFCFD_ERR_ARG;
    return mfcfd::host_guard(nullptr, [&]() -> int { return s->submit(q, id); });
}

int mfcfd_server::submit(const mfcfd_request *q, int64_t *id) {
    auto r = std::make_shared<Request>();
    const size_t n = (size_t)q->n;
    r->P = q->params;
    r->n = q->n;
    r->status.assign(q->status, q->status + n);
    r->nbhs.assign(q->nbhs, q->nbhs + n);
    r->conn.assign(q->conn, q->conn + n * mfcfd::MAX_CONN);
    r->x.assign(q->x, q->x + n);
    r->y.assign(q->y, q->y + n);
    r->z.assign(q->z, q->z + n);
    r->tan1.assign(q->tan1, q->tan1 + 3 * n);
    r->tan2.assign(q->tan2, q->tan2 + 3 * n);
    r->nor.assign(q->nor, q->nor + 3 * n);
    r->min_dist.assign(q->min_dist, q->min_dist + n);
    if (q->prim) {
        r->prim0.assign(q->prim, q->prim + 5 * n);
    } else {
        // impulsive start: the freestream, without its normal component at
        // wall points (a uniform freestream is a fixed point of the scheme)
        const mfcfd_params &P = q->params;
        r->prim0.resize(5 * n);
        for (size_t i = 0; i < n; ++i) {
            double *p = &r->prim0[5 * i];
            p[0] = P.rho_inf; p[1] = P.u1_inf; p[2] = P.u2_inf; p[3] = P.u3_inf; p[4] = P.pr_inf;
            if (q->status[i] == 1) {
                const double *nr = q->nor + 3 * i;
                const double un = p[1] * nr[0] + p[2] * nr[1] + p[3] * nr[2];
                for (int k = 0; k < 3; ++k) p[1 + k] = p[1 + k] - un * nr[k];
            }
        }
    }
    const int32_t c = cfg.chunk;
    r->max_iters = (q->max_iters + c - 1) / c * c;
    r->target = q->residue_target;
    r->polish = q->polish_residue;
    r->wall_area = q->wall_area;
    r->ref_area = q->ref_area;
    r->res.n = q->n;
    std::lock_guard<std::mutex> lk(mu);
    if (stopping) return MFCFD_ERR_ARG;
    r->id = next_id++;
    r->res.id = r->id;
    r->res.t_submit = now();
    all[r->id] = r;
    try {
        to_prepare.push_back(r);
    } catch (...) {
        all.erase(r->id);   // leaves no trace of the request
        throw;
    }
    ++st.submitted;
    cv_setup.notify_one();
    *id = r->id;
    return MFCFD_OK;
}

int mfcfd_server_wait(mfcfd_server *s, int64_t id, double timeout_s, mfcfd_result *res, double *prim) {
    if (!s || !res) return MFCFD_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return MFCFD_ERR_ARG;
    RequestPtr r = it->second;
    auto pred = [&] { return r->done; };
    if (timeout_s < 0) s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) return MFCFD_ERR_BUSY;
    *res = r->res;
    if (prim && !r->prim_out.empty()) std::memcpy(prim, r->prim_out.data(), sizeof(double) * r->prim_out.size());
    s->all.erase(id);
    return MFCFD_OK;
}

int mfcfd_server_get_stats(mfcfd_server *s, mfcfd_server_stats *st) {
    if (!s || !st) return MFCFD_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    *st = s->st;
    st->preparing = s->preparing + (int64_t)s->to_prepare.size();
    st->waiting = (int64_t)s->ready.size();
    st->live = s->n_live;
    return MFCFD_OK;
}

int mfcfd_server_destroy(mfcfd_server *s) {
    if (!s) return MFCFD_ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_setup.notify_all();
    s->cv_sched.notify_all();
    for (std::thread &w : s->workers) w.join();
    s->scheduler.join();
    // requests between the threads when they stopped
    for (auto *q : {&s->ready, &s->to_attach, &s->attached, &s->to_retire})
        for (const RequestPtr &r : *q)
            if (r->h) mfcfd_destroy(r->h);
    delete s;
    return MFCFD_OK;
}

}  // extern "C"
