/*
 * mfcfd_setup.cpp - one-time host set-up of a point cloud.
 *
 * Builds, from the reference's input arrays:
 *   - the six split stencils of every point with the reference's storage
 *     (generate_connectivity.f90:12-246), including its fixed capacity of 22
 *     entries per list (data_structure.f90:83-88): a list that grows past the
 *     capacity continues into the next point's column of the same
 *     column-major array, as unchecked Fortran indexing does, and later reads
 *     see whatever that column holds after all writes;
 *   - the sweep order from the alias breadth-first search
 *     (implicit_aliasing.f90:13-44) with its quirks (the first neighbour of
 *     point 1 also receives alias 1; point_with_alias(N) stays 0);
 *   - the "effective" neighbour lists each routine actually reads (the wall
 *     z- terms use the full conn, wall_flux_dGzneg.f90:61-65,
 *     implicit_D_inv_wall.f90:309-310), compacted into at most 32 distinct
 *     neighbour slots per point for the warp-per-point flux kernel;
 *   - the per-list least-squares moments, determinant and D_inv numerator,
 *     which depend on geometry only (implicit_D_inv_interior.f90:63-105);
 *   - the level schedules of the forward and backward LU-SGS sweeps: a point's
 *     level is one more than the deepest level among the neighbours whose
 *     increments it reads (lower alias forward, higher alias backward), so
 *     every level can be processed in parallel and the result equals the
 *     reference's sequential sweep bit for bit.
 * All floating-point work here is compiled without contraction so the
 * values equal those the reference computes inline.
 */
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <thread>

#include "mfcfd_internal.h"

namespace mfcfd {

namespace {

struct Moments { double xx, yy, zz, xy, yz, zx; };

// at least this many indices per thread: starting a thread costs about as
// much as a few thousand of the cheapest passes' indices
constexpr int PAR_GRAIN = 4096;

// f(i) for i in [0, n) on the calling thread and up to 31 threads from the
// set-up pool; every i writes only its own outputs, so the result does not
// depend on the thread count.
//
// An exception in any chunk (host memory exhausted) reaches the caller after
// every thread has ended; a chunk whose thread cannot be started runs on the
// calling thread.
template <class F>
void parallel_for(int n, const F &f) {
    const int want = std::min(31, n / PAR_GRAIN - 1);
    const int extra = want > 0 ? take_setup_threads(want) : 0;
    if (extra == 0) {
        for (int i = 0; i < n; ++i) f(i);
        return;
    }
    struct Tokens {
        int k;
        ~Tokens() { give_setup_threads(k); }
    } tokens{extra};
    const int nt = extra + 1;
    const int chunk = (n + nt - 1) / nt;
    std::vector<std::exception_ptr> errs((size_t)nt);
    std::vector<std::thread> th;
    th.reserve((size_t)extra);
    int threaded = 1;   // chunks 1 .. threaded-1 run on their own threads
    for (int t = 1; t < nt; ++t) {
        const int a = t * chunk, b = std::min(n, a + chunk);
        if (a >= b) break;
        try {
            th.emplace_back([a, b, t, &f, &errs] {
                try {
                    for (int i = a; i < b; ++i) f(i);
                } catch (...) {
                    errs[(size_t)t] = std::current_exception();
                }
            });
        } catch (...) {
            break;
        }
        threaded = t + 1;
    }
    try {
        for (int i = 0; i < std::min(n, chunk); ++i) f(i);
        for (int i = threaded * chunk; i < n; ++i) f(i);
    } catch (...) {
        errs[0] = std::current_exception();
    }
    for (auto &t : th) t.join();
    for (const std::exception_ptr &e : errs)
        if (e) std::rethrow_exception(e);
}

inline double det_of(const Moments &m) {
    return m.xx * (m.yy * m.zz - m.yz * m.yz)
         - m.xy * (m.xy * m.zz - m.yz * m.zx)
         + m.zx * (m.xy * m.yz - m.yy * m.zx);
}

// Cramer numerators, in the reference's operand order
// (implicit_D_inv_interior.f90:103-105, :225-227, :347-349).
inline double numerator(int axis, const Moments &m, double fx, double fy, double fz) {
    if (axis == 0)
        return fx * (m.yy * m.zz - m.yz * m.yz) - fy * (m.xy * m.zz - m.zx * m.yz)
             + fz * (m.xy * m.yz - m.zx * m.yy);
    if (axis == 1)
        return m.xx * (fy * m.zz - m.yz * fz) - m.xy * (fx * m.zz - m.zx * fz)
             + m.zx * (fx * m.yz - m.zx * fy);
    return m.xx * (m.yy * fz - fy * m.yz) - m.xy * (m.xy * fz - fx * m.yz)
         + m.zx * (m.xy * fy - fx * m.yy);
}

// the host's cores less two: one for the calling thread, one for a thread
// that keeps a device busy meanwhile (the request server's scheduler); or
// MFCFD_SETUP_THREADS - 1 when that is set (1: every pass on its caller)
int initial_pool() {
    if (const char *v = std::getenv("MFCFD_SETUP_THREADS")) {
        const int t = std::atoi(v);
        if (t >= 1) return std::min(t, 256) - 1;
    }
    return std::max(0, (int)std::thread::hardware_concurrency() - 2);
}

std::atomic<int> &setup_pool() {
    static std::atomic<int> pool{initial_pool()};
    return pool;
}

}  // namespace

int take_setup_threads(int want) {
    std::atomic<int> &pool = setup_pool();
    int avail = pool.load(std::memory_order_relaxed);
    while (avail > 0) {
        const int got = std::min(avail, want);
        if (pool.compare_exchange_weak(avail, avail - got, std::memory_order_relaxed)) return got;
    }
    return 0;
}

void give_setup_threads(int k) {
    if (k > 0) setup_pool().fetch_add(k, std::memory_order_relaxed);
}

namespace {

// A point's neighbours in list order (generate_connectivity.f90:38-246):
// put(d, k) for each list d that takes neighbour k (1-based id); interior
// points split all three axes, wall and outer points put every neighbour in
// their one z list.
template <class F>
void split_point(int i, int cls, const double *x, const double *y, const double *z, const double *tan1,
                 const double *tan2, const double *nor, const int32_t *nbhs, const int32_t *conn, F &&put) {
    const double xi = x[i], yi = y[i], zi = z[i];
    const double *t1 = tan1 + 3 * (size_t)i, *t2 = tan2 + 3 * (size_t)i, *nn = nor + 3 * (size_t)i;
    for (int r = 0; r < nbhs[i]; ++r) {
        int k = conn[(size_t)i * MAX_CONN + r];
        double delx = x[k - 1] - xi, dely = y[k - 1] - yi, delz = z[k - 1] - zi;
        double dels = delx * t1[0] + dely * t1[1] + delz * t1[2];
        double delt = delx * t2[0] + dely * t2[1] + delz * t2[2];
        if (cls == CLS_INTERIOR) {
            double deln = delx * nn[0] + dely * nn[1] + delz * nn[2];
            if (dels <= 0.0) put(0, k);
            if (dels > 0.0) put(1, k);
            if (delt <= 0.0) put(2, k);
            if (delt > 0.0) put(3, k);
            if (deln <= 0.0) put(4, k);
            if (deln > 0.0) put(5, k);
        } else {
            if (dels <= 0.0) put(0, k);
            if (dels >= 0.0) put(1, k);
            if (delt <= 0.0) put(2, k);
            if (delt >= 0.0) put(3, k);
            put(cls == CLS_WALL ? 5 : 4, k);
        }
    }
}

}  // namespace

int classify_points(const mfcfd_params &P, int n, const int32_t *status, const int32_t *nbhs, const int32_t *conn,
                    Topology &T, std::string &err) {
    T.n = n;
    T.cap = P.split_capacity > 0 ? P.split_capacity : MAX_CONN;
    T.cls.assign(n, CLS_SUPERSONIC);
    for (int i = 0; i < n; ++i) {
        if (nbhs[i] < 0 || nbhs[i] > MAX_CONN) {
            err = "nbhs out of range [0,27] at point " + std::to_string(i + 1);
            return MFCFD_ERR_ARG;
        }
        for (int r = 0; r < nbhs[i]; ++r) {
            int k = conn[(size_t)i * MAX_CONN + r];
            if (k < 1 || k > n) {
                err = "conn entry out of range at point " + std::to_string(i + 1);
                return MFCFD_ERR_ARG;
            }
        }
        switch (status[i]) {
        case 0: T.cls[i] = CLS_INTERIOR; T.interior_idx.push_back(i); break;
        case 1: T.cls[i] = CLS_WALL; T.wall_idx.push_back(i); break;
        case 2: T.cls[i] = CLS_OUTER; T.outer_idx.push_back(i); break;
        case 5: T.cls[i] = CLS_SUPERSONIC; T.ss_inlet_idx.push_back(i); break;
        case 6: T.cls[i] = CLS_SUPERSONIC; T.ss_outlet_idx.push_back(i); break;
        default:
            err = "unknown point status " + std::to_string(status[i]);
            return MFCFD_ERR_ARG;
        }
    }
    return MFCFD_OK;
}

// The reference stores list d of point i at i*cap + j, and an entry past the
// capacity lands in the following points' storage; it visits the interior,
// then the wall, then the outer points, each once from zeroed counts, so a
// cell ends with the value of its last writer in that order.  Each point
// first fills its own cells; then the spilled entries, in that order,
// replace an owner's value that came earlier or was never written.  This
// gives those spilled writes, from every point's full list counts.
void split_spill_writes(const Topology &T, const double *x, const double *y, const double *z, const double *tan1,
                        const double *tan2, const double *nor, const int32_t *nbhs, const int32_t *conn,
                        const int32_t *const cnt[NDIR], std::vector<SpillWrite> &out) {
    const int n = T.n, cap = T.cap;
    out.clear();
    std::vector<int32_t> visit(n, -1);
    int at = 0;
    for (const std::vector<int32_t> *cl : {&T.interior_idx, &T.wall_idx, &T.outer_idx})
        for (int i : *cl) visit[i] = at++;
    for (const std::vector<int32_t> *cl : {&T.interior_idx, &T.wall_idx, &T.outer_idx})
        for (int s : *cl) {
            bool spills = false;
            for (int d = 0; d < NDIR; ++d) spills = spills || cnt[d][s] > cap;
            if (!spills) continue;
            int c[NDIR] = {0, 0, 0, 0, 0, 0};
            split_point(s, T.cls[s], x, y, z, tan1, tan2, nor, nbhs, conn, [&](int d, int k) {
                const int j = c[d]++;
                if (j < cap) return;
                const int t = s + j / cap, slot = j % cap;   // the cell's owner and its slot
                const bool owner_wrote = t < n && visit[t] >= 0 && cnt[d][t] > slot;
                if (!owner_wrote || visit[t] < visit[s]) out.push_back({d, (size_t)s * cap + j, k});
            });
        }
}

void limiter_eps2(const mfcfd_params &P, int n, const double *min_dist, const int32_t *perm, std::vector<double> &eps2) {
    eps2.resize(n);
    for (int i = 0; i < n; ++i) {
        double e = P.vl_const * min_dist[i];
        e = std::pow(e, 3.0);
        eps2[perm ? perm[i] : i] = e * e;
    }
}

int build_topology(const mfcfd_params &P, int n, const int32_t *status, const double *x,
                   const double *y, const double *z, const double *tan1, const double *tan2,
                   const double *nor, const int32_t *nbhs, const int32_t *conn,
                   const double *min_dist, Topology &T, std::string &err) {
    if (int rc = classify_points(P, n, status, nbhs, conn, T, err)) return rc;
    const int cap = T.cap;

    const bool gpu = P.gpu_setup != 0 && P.device >= 0;
    // ---- split stencils with the reference's storage (generate_connectivity.f90)
    bool split_done = false;
    if (gpu) {
        bool over = false;
        const int rc = prep_split_gpu(P.device, n, cap, T.cls, x, y, z, tan1, tan2, nor, nbhs, conn, T, &over, err);
        if (rc) return rc;
        split_done = !over;
    }
    const size_t flat = (size_t)n * cap + 64;
    for (int d = 0; d < NDIR && !split_done; ++d) {
        T.split[d].assign(flat, 0);
        T.split_cnt[d].assign(n, 0);
    }
    T.split_overflows = 0;
    if (!split_done) {
        // each point fills its own cells (in parallel), then the spilled
        // entries are written in the reference's visiting order
        parallel_for(n, [&](int i) {
            const int c = T.cls[i];
            if (c != CLS_INTERIOR && c != CLS_WALL && c != CLS_OUTER) return;
            split_point(i, c, x, y, z, tan1, tan2, nor, nbhs, conn, [&](int d, int k) {
                const int j = T.split_cnt[d][i]++;
                if (j < cap) T.split[d][(size_t)i * cap + j] = k;
            });
        });
        for (int d = 0; d < NDIR; ++d)
            for (int i = 0; i < n; ++i) T.split_overflows += std::max(0, T.split_cnt[d][i] - cap);
        if (T.split_overflows > 0) {
            const int32_t *cnt[NDIR];
            for (int d = 0; d < NDIR; ++d) cnt[d] = T.split_cnt[d].data();
            std::vector<SpillWrite> w;
            split_spill_writes(T, x, y, z, tan1, tan2, nor, nbhs, conn, cnt, w);
            for (const SpillWrite &e : w) T.split[e.d][e.at] = e.value;
        }
    }

    // ---- alias breadth-first search (implicit_aliasing.f90:21-42).
    // Index 0 of the 1-based arrays is a zero guard: point_with_alias(i) = 0
    // makes the inner loop run over nbhs(0) = 0 neighbours.
    if (gpu) {
        const int rc = prep_alias_gpu(P.device, n, nbhs, conn, T.alias, T.point_with_alias, err);
        if (rc) return rc;
    } else {
        std::vector<int32_t> alias1(n + 1, 0), pwa1(n + 1, 0);
        alias1[1] = 1;
        pwa1[1] = 1;
        int count = 0;
        for (int i = 1; i <= n; ++i) {
            int p = pwa1[i];
            int nb = p > 0 ? nbhs[p - 1] : 0;
            for (int j = 0; j < nb; ++j) {
                int k = conn[(size_t)(p - 1) * MAX_CONN + j];
                if (alias1[k] == 0) {
                    count = count + 1;
                    alias1[k] = count;
                    pwa1[count] = k;
                }
            }
        }
        T.alias.assign(alias1.begin() + 1, alias1.end());
        T.point_with_alias.assign(pwa1.begin() + 1, pwa1.end());
    }

    // ---- effective lists and neighbour slots
    T.slot_nbr.assign((size_t)n * MAX_SLOTS, -1);
    T.nslot.assign(n, 0);
    T.slot_mask.assign((size_t)n * MAX_SLOTS, 0);
    T.list_cnt.assign((size_t)n * NDIR, 0);
    T.list_ent.assign((size_t)n * NDIR * LIST_STRIDE, 0);
    auto effective = [&](int i, int d, std::vector<int> &out) {   // 0-based ids
        out.clear();
        int cls = T.cls[i];
        bool use_conn = (cls == CLS_WALL && d == 5);
        bool unused = (cls == CLS_WALL && d == 4) || (cls == CLS_OUTER && d == 5) || cls == CLS_SUPERSONIC;
        if (unused) return true;
        if (use_conn) {
            for (int r = 0; r < nbhs[i]; ++r) out.push_back(conn[(size_t)i * MAX_CONN + r] - 1);
            return true;
        }
        int c = T.split_cnt[d][i];
        for (int j = 0; j < c; ++j) {
            int k = T.split[d][(size_t)i * cap + j];
            if (k < 1 || k > n) return false;
            out.push_back(k - 1);
        }
        return true;
    };
    // per point: 0 ok, else the first problem found (reported for the
    // lowest such point, as a sequential pass would)
    enum { SLOT_OK = 0, SLOT_ZERO, SLOT_LONG, SLOT_WIDE };
    std::vector<uint8_t> slot_err(n, SLOT_OK);
    parallel_for(n, [&](int i) {
        std::vector<int> eff;
        int32_t *slots = &T.slot_nbr[(size_t)i * MAX_SLOTS];
        int ns = 0;
        auto slot_of = [&](int k) -> int {
            for (int s = 0; s < ns; ++s) if (slots[s] == k) return s;
            if (ns == MAX_SLOTS) return -1;
            slots[ns] = k;
            return ns++;
        };
        for (int r = 0; r < nbhs[i]; ++r) slot_of(conn[(size_t)i * MAX_CONN + r] - 1);
        for (int d = 0; d < NDIR; ++d) {
            if (!effective(i, d, eff)) { slot_err[i] = SLOT_ZERO; return; }
            if (eff.size() > (size_t)MAX_CONN) { slot_err[i] = SLOT_LONG; return; }
            T.list_cnt[(size_t)i * NDIR + d] = (uint8_t)eff.size();
            for (size_t j = 0; j < eff.size(); ++j) {
                int s = slot_of(eff[j]);
                if (s < 0) { slot_err[i] = SLOT_WIDE; return; }
                T.list_ent[((size_t)i * NDIR + d) * LIST_STRIDE + j] = (uint8_t)s;
                T.slot_mask[(size_t)i * MAX_SLOTS + s] |= (uint8_t)(1u << d);
            }
        }
        T.nslot[i] = (uint8_t)ns;
    });
    for (int i = 0; i < n; ++i) {
        if (slot_err[i] == SLOT_OK) continue;
        const std::string at = std::to_string(i + 1);
        if (slot_err[i] == SLOT_ZERO) err = "split list of point " + at + " names point 0";
        else if (slot_err[i] == SLOT_LONG) err = "split list longer than 27 at point " + at;
        else err = "more than 32 distinct stencil neighbours at point " + at;
        return MFCFD_ERR_STENCIL;
    }

    // ---- geometry per (point, list): moments, determinant, D_inv numerator
    T.geo.assign((size_t)n * GEO_STRIDE, 0.0);
    // least-squares weight 1/dist**power; dist**0 is exactly 1 for every dist
    auto weight = [&](double dels, double delt, double deln) {
        if (P.power == 0.0) return 1.0;
        const double dist = std::sqrt(dels * dels + delt * delt + deln * deln);
        return 1.0 / std::pow(dist, P.power);
    };
    const bool backup = P.sweep_variant == MFCFD_SWEEPS_BACKUP;
    T.sweep_variant = P.sweep_variant;
    // the backup driver's outer routines take z+ over the full conn
    // (implicit_D_inv_outer.f90:313-315): its moments go to the unused row 5
    auto conn_z = [&](int i, int d) { return backup && d == 5 && T.cls[i] == CLS_OUTER; };
    parallel_for(n, [&](int i) {
        const double *t1 = tan1 + 3 * (size_t)i, *t2 = tan2 + 3 * (size_t)i, *nn = nor + 3 * (size_t)i;
        for (int d = 0; d < NDIR; ++d) {
            const bool cz = conn_z(i, d);
            int c = cz ? nbhs[i] : T.list_cnt[(size_t)i * NDIR + d];
            Moments m = {0, 0, 0, 0, 0, 0};
            double sdx = 0, sdy = 0, sdz = 0;
            for (int j = 0; j < c; ++j) {
                int k;
                if (cz) {
                    k = conn[(size_t)i * MAX_CONN + j] - 1;
                } else {
                    int s = T.list_ent[((size_t)i * NDIR + d) * LIST_STRIDE + j];
                    k = T.slot_nbr[(size_t)i * MAX_SLOTS + s];
                }
                double delx = x[k] - x[i], dely = y[k] - y[i], delz = z[k] - z[i];
                double dels = delx * t1[0] + dely * t1[1] + delz * t1[2];
                double delt = delx * t2[0] + dely * t2[1] + delz * t2[2];
                double deln = delx * nn[0] + dely * nn[1] + delz * nn[2];
                double w = weight(dels, delt, deln);
                double ws = dels * w, wt = delt * w, wn = deln * w;
                m.xx = m.xx + dels * ws;
                m.yy = m.yy + delt * wt;
                m.zz = m.zz + deln * wn;
                m.xy = m.xy + dels * wt;
                m.yz = m.yz + delt * wn;
                m.zx = m.zx + deln * ws;
                sdx = sdx + ws;
                sdy = sdy + wt;
                sdz = sdz + wn;
            }
            double *g = &T.geo[(size_t)i * GEO_STRIDE + d * 8];
            g[G_XX] = m.xx; g[G_YY] = m.yy; g[G_ZZ] = m.zz;
            g[G_XY] = m.xy; g[G_YZ] = m.yz; g[G_ZX] = m.zx;
            g[G_DET] = det_of(m);
            g[G_DNUM] = numerator(d / 2, m, sdx, sdy, sdz);
        }
    });

    // weights of the q-derivative and flux least squares (q_derivatives.f90:
    // 44-45, interior_flux_dGxpos.f90:77-78): only for power != 0
    T.wq.clear();
    T.wf.clear();
    if (P.power != 0.0) {
        T.wq.assign((size_t)n * MAX_CONN, 0.0);
        T.wf.assign((size_t)n * MAX_SLOTS, 0.0);
        parallel_for(n, [&](int i) {
            for (int r = 0; r < nbhs[i]; ++r) {
                const int k = conn[(size_t)i * MAX_CONN + r] - 1;
                const double delx = x[k] - x[i], dely = y[k] - y[i], delz = z[k] - z[i];
                const double dist = std::sqrt(delx * delx + dely * dely + delz * delz);
                T.wq[(size_t)i * MAX_CONN + r] = 1.0 / std::pow(dist, P.power);
            }
            const double *t1 = tan1 + 3 * (size_t)i, *t2 = tan2 + 3 * (size_t)i, *nn = nor + 3 * (size_t)i;
            for (int s = 0; s < T.nslot[i]; ++s) {
                const int k = T.slot_nbr[(size_t)i * MAX_SLOTS + s];
                const double delx = x[k] - x[i], dely = y[k] - y[i], delz = z[k] - z[i];
                const double dels = delx * t1[0] + dely * t1[1] + delz * t1[2];
                const double delt = delx * t2[0] + dely * t2[1] + delz * t2[2];
                const double deln = delx * nn[0] + dely * nn[1] + delz * nn[2];
                T.wf[(size_t)i * MAX_SLOTS + s] = weight(dels, delt, deln);
            }
        });
    }

    // limiter epsilon: (VL_CONST*min_dist)**3 squared (limiters.f90:251-253)
    limiter_eps2(P, n, min_dist, nullptr, T.eps2);

    // ---- sweep schedules (implicit_forward_and_reverse_sweeps.f90:26-84, or
    // implicit_forward_and_reverse_sweeps_backup.f90:26-141)
    T.swept.assign(n, 0);
    std::vector<int> order_f, order_b;   // swept points in each sweep's order (0-based)
    if (!backup) {
        for (int i = 0; i < n; ++i) {
            int p = T.point_with_alias[i];
            if (p == 0) continue;   // the reference's out-of-range entry
            int cls = T.cls[p - 1];
            if (cls == CLS_WALL || cls == CLS_INTERIOR || cls == CLS_SUPERSONIC) {
                T.swept[p - 1] = 1;
                order_f.push_back(p - 1);
            }
        }
        order_b.assign(order_f.rbegin(), order_f.rend());
    } else {
        for (const std::vector<int32_t> *cl : {&T.wall_idx, &T.interior_idx, &T.outer_idx, &T.ss_inlet_idx,
                                               &T.ss_outlet_idx}) {
            for (int p : *cl) { T.swept[p] = 1; order_f.push_back(p); }
            for (auto it = cl->rbegin(); it != cl->rend(); ++it) order_b.push_back(*it);
        }
    }
    // nearest neighbour in conn order, first of equal distances, starting
    // from `start` (implicit_forward_and_reverse_sweeps.f90:39-50,
    // state_update_implicit.f90:63-94); -1 if none is closer than start
    auto nearest = [&](int p, bool skip_wall, double start) {
        double min_dist = start;
        int q = -1;
        for (int r = 0; r < nbhs[p]; ++r) {
            const int nbh = conn[(size_t)p * MAX_CONN + r] - 1;
            const double dx = x[nbh] - x[p], dy = y[nbh] - y[p], dz = z[nbh] - z[p];
            const double ds = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (ds < min_dist && (!skip_wall || T.cls[nbh] != CLS_WALL)) {
                min_dist = ds;
                q = nbh;
            }
        }
        return q;
    };
    T.copy_src.assign(n, -1);
    T.ss_pts.clear();
    T.ss_src.clear();
    for (int i = 0; i < n; ++i)
        if (T.cls[i] == CLS_SUPERSONIC)   // the backup driver skips walls, from 1e5
            T.copy_src[i] = backup ? nearest(i, true, 100000.0) : nearest(i, false, 1000000.0);
    // D_inv_outer's 1/delt operand: the tangential offset of the last conn
    // neighbour, which the direction loops leave in the time-step variable
    // (implicit_D_inv_outer.f90:47, :74); NaN: no neighbour, the time step
    T.outer_delt.clear();
    if (backup) {
        T.outer_delt.assign(n, std::nan(""));
        for (int i : T.outer_idx) {
            if (nbhs[i] < 1) continue;
            const int k = conn[(size_t)i * MAX_CONN + nbhs[i] - 1] - 1;
            const double *t2 = tan2 + 3 * (size_t)i;
            const double delx = x[k] - x[i], dely = y[k] - y[i], delz = z[k] - z[i];
            T.outer_delt[i] = delx * t2[0] + dely * t2[1] + delz * t2[2];
        }
    }
    // slot membership of the sweeps' term lists (outer z+ over conn under the
    // backup driver)
    T.sweep_slot_mask = T.slot_mask;
    if (backup)
        for (int i : T.outer_idx)
            for (int s = 0; s < MAX_SLOTS; ++s) {
                uint8_t &m = T.sweep_slot_mask[(size_t)i * MAX_SLOTS + s];
                m &= (uint8_t)~(1u << 4);
                if (s < T.nslot[i]) {
                    const int k = T.slot_nbr[(size_t)i * MAX_SLOTS + s];
                    for (int r = 0; r < nbhs[i]; ++r)
                        if (conn[(size_t)i * MAX_CONN + r] - 1 == k) { m |= 1u << 4; break; }
                }
            }
    // state_update_implicit.f90 skips wall sources; state_update.f90 does not
    const bool skip_wall = P.update_variant != MFCFD_UPDATE_EXPLICIT;
    for (int k : T.ss_outlet_idx) { T.ss_pts.push_back(k); T.ss_src.push_back(nearest(k, skip_wall, 100000.0)); }
    for (int k : T.ss_inlet_idx) { T.ss_pts.push_back(k); T.ss_src.push_back(nearest(k, skip_wall, 100000.0)); }
    auto al = [&](int k) { return T.alias[k]; };
    int gpu_rc = MFCFD_OK;
    std::vector<int32_t> pos(n, -1);
    // a point's sweep terms of list d in list order: (slot, neighbour)
    auto for_terms = [&](int p, int d, auto &&fn) {
        if (backup && d == 4 && T.cls[p] == CLS_OUTER) {   // z+ over conn
            for (int r = 0; r < nbhs[p]; ++r) {
                const int k = conn[(size_t)p * MAX_CONN + r] - 1;
                int s = 0;
                while (s < T.nslot[p] && T.slot_nbr[(size_t)p * MAX_SLOTS + s] != k) ++s;
                fn(s, k);
            }
            return;
        }
        if (T.cls[p] == CLS_OUTER && d == 5) return;
        const int c = T.list_cnt[(size_t)p * NDIR + d];
        for (int j = 0; j < c; ++j) {
            const int s = T.list_ent[((size_t)p * NDIR + d) * LIST_STRIDE + j];
            fn(s, (int)T.slot_nbr[(size_t)p * MAX_SLOTS + s]);
        }
    };
    auto build = [&](bool forward, const std::vector<int> &order, std::vector<int32_t> &level,
                     std::vector<int32_t> &lptr, std::vector<int32_t> &lpts, std::vector<int32_t> &off,
                     std::vector<uint8_t> &cnt, std::vector<SweepEntry> &ent, std::vector<uint32_t> &need,
                     std::vector<uint32_t> &old) {
        level.assign(n, -1);
        need.assign(n, 0u);
        old.assign(n, 0u);
        off.assign(n + 1, 0);
        cnt.assign((size_t)n * NDIR, 0);
        for (size_t i = 0; i < order.size(); ++i) pos[order[i]] = (int32_t)i;
        // the terms the reference's L/U routines take (alias test), and
        // whether the producer's increment is this sweep's (earlier in the
        // order) or from before it
        auto takes = [&](int p, int k) { return forward ? (al(k) < al(p)) : (al(k) > al(p)); };
        auto is_old = [&](int p, int k) { return backup && pos[k] > pos[p]; };
        // entries, in point index order of the offsets: count, then fill
        parallel_for((int)order.size(), [&](int oi) {
            const int p = order[oi];
            if (T.cls[p] == CLS_SUPERSONIC) {   // one copy entry
                cnt[(size_t)p * NDIR] = 1;
                off[p + 1] += 1;
                return;
            }
            for (int d = 0; d < NDIR; ++d) {
                int taken = 0;
                for_terms(p, d, [&](int, int k) { if (takes(p, k)) ++taken; });
                cnt[(size_t)p * NDIR + d] = (uint8_t)taken;
                off[p + 1] += taken;
            }
        });
        for (int p = 0; p < n; ++p) off[p + 1] += off[p];
        ent.clear();
        ent.resize((size_t)off[n]);
        parallel_for((int)order.size(), [&](int oi) {
            const int p = order[oi];
            if (T.cls[p] == CLS_SUPERSONIC) {
                const int q = T.copy_src[p];
                SweepEntry &e = ent[(size_t)off[p]];
                e.k = q;
                const bool fresh = q >= 0 && T.swept[q] && (backup ? pos[q] < pos[p] : takes(p, q));
                e.pad = ENT_COPY | (fresh ? ENT_COPY_NEW : 0);
                e.w[0] = e.w[1] = e.w[2] = 0.0;
                return;
            }
            const double *t1 = tan1 + 3 * (size_t)p, *t2 = tan2 + 3 * (size_t)p, *nn = nor + 3 * (size_t)p;
            size_t e_at = (size_t)off[p];
            for (int d = 0; d < NDIR; ++d) {
                for_terms(p, d, [&](int s, int k) {
                    if (!takes(p, k)) return;
                    double delx = x[k] - x[p], dely = y[k] - y[p], delz = z[k] - z[p];
                    double dels = delx * t1[0] + dely * t1[1] + delz * t1[2];
                    double delt = delx * t2[0] + dely * t2[1] + delz * t2[2];
                    double deln = delx * nn[0] + dely * nn[1] + delz * nn[2];
                    double w = weight(dels, delt, deln);
                    SweepEntry &e = ent[e_at++];
                    e.k = k;
                    e.pad = d | (s << 8) | (is_old(p, k) ? ENT_OLD : 0);   // list, neighbour slot
                    e.w[0] = dels * w; e.w[1] = delt * w; e.w[2] = deln * w;
                    need[p] |= 1u << s;
                    if (is_old(p, k)) old[p] |= 1u << s;
                });
            }
        });
        for (int p = 0; p < n; ++p)
            if (off[p + 1] - off[p] > SWEEP_MAX_ENTRIES) return false;
        // levels: longest path over swept dependencies, visited in the order
        int maxl = -1;
        auto is_dep = [&](const SweepEntry &E) { return entry_is_dependency(E) && T.swept[E.k]; };
        if (gpu) {
            std::vector<int32_t> doff(n + 1, 0), deps;
            parallel_for((int)order.size(), [&](int oi) {
                const int p = order[oi];
                int c = 0;
                for (int e = off[p]; e < off[p + 1]; ++e) c += is_dep(ent[e]) ? 1 : 0;
                doff[p + 1] = c;
            });
            for (int p = 0; p < n; ++p) doff[p + 1] += doff[p];
            deps.resize((size_t)doff[n]);
            parallel_for((int)order.size(), [&](int oi) {
                const int p = order[oi];
                int at = doff[p];
                for (int e = off[p]; e < off[p + 1]; ++e)
                    if (is_dep(ent[e])) deps[at++] = ent[e].k;
            });
            if ((gpu_rc = prep_levels_gpu(P.device, n, order, doff, deps, level, err))) return false;
            for (int p : order) maxl = std::max(maxl, (int)level[p]);
        } else {
            // the producers each point depends on, gathered in parallel and
            // laid out in the sweep order, so that the sequential
            // longest-path pass reads them front to back
            const int m = (int)order.size();
            std::vector<int32_t> doff((size_t)m + 1, 0), deps;
            parallel_for(m, [&](int oi) {
                const int p = order[oi];
                int c = 0;
                for (int e = off[p]; e < off[p + 1]; ++e) c += is_dep(ent[e]) ? 1 : 0;
                doff[(size_t)oi + 1] = c;
            });
            for (int oi = 0; oi < m; ++oi) doff[(size_t)oi + 1] += doff[oi];
            deps.resize((size_t)doff[m]);
            parallel_for(m, [&](int oi) {
                const int p = order[oi];
                int at = doff[oi];
                for (int e = off[p]; e < off[p + 1]; ++e)
                    if (is_dep(ent[e])) deps[at++] = ent[e].k;
            });
            for (int oi = 0; oi < m; ++oi) {
                int lv = 0;
                for (int j = doff[oi]; j < doff[(size_t)oi + 1]; ++j) {
                    const int k = deps[j];
                    if (level[k] + 1 > lv) lv = level[k] + 1;
                }
                level[order[oi]] = lv;
                maxl = std::max(maxl, lv);
            }
        }
        int nl = maxl + 1;
        lptr.assign(nl + 1, 0);
        for (int p : order) lptr[level[p] + 1]++;
        for (int l = 0; l < nl; ++l) {
            lptr[l + 1] += lptr[l];
            T.max_level_width = std::max(T.max_level_width, lptr[l + 1] - lptr[l]);
        }
        lpts.assign(order.size(), 0);
        std::vector<int32_t> fill(lptr.begin(), lptr.end() - 1);
        for (int p : order) lpts[fill[level[p]]++] = p;
        return true;
    };
    if (!build(true, order_f, T.fwd_level, T.fwd_lvl_ptr, T.fwd_lvl_pts, T.fwd_off, T.fwd_cnt, T.fwd_ent,
               T.fwd_need, T.fwd_old) ||
        !build(false, order_b, T.bwd_level, T.bwd_lvl_ptr, T.bwd_lvl_pts, T.bwd_off, T.bwd_cnt, T.bwd_ent,
               T.bwd_need, T.bwd_old)) {
        if (gpu_rc) return gpu_rc;
        err = "a point reads more than " + std::to_string(SWEEP_MAX_ENTRIES) + " sweep terms";
        return MFCFD_ERR_STENCIL;
    }

    // ---- shared interior frame: lets producers publish flux increments
    T.shared_frame = 0;
    if (!T.interior_idx.empty()) {
        int i0 = T.interior_idx[0];
        double f0[9];
        for (int r = 0; r < 3; ++r) {
            f0[r] = tan1[3 * (size_t)i0 + r];
            f0[3 + r] = tan2[3 * (size_t)i0 + r];
            f0[6 + r] = nor[3 * (size_t)i0 + r];
        }
        bool same = true;
        for (int i : T.interior_idx) {
            for (int r = 0; r < 3 && same; ++r) {
                if (std::memcmp(&tan1[3 * (size_t)i + r], &f0[r], 8) ||
                    std::memcmp(&tan2[3 * (size_t)i + r], &f0[3 + r], 8) ||
                    std::memcmp(&nor[3 * (size_t)i + r], &f0[6 + r], 8))
                    same = false;
            }
            if (!same) break;
        }
        if (same) {
            T.shared_frame = 1;
            std::memcpy(T.frame0, f0, sizeof f0);
        }
    }
    T.consumer_shared.assign(n, 0);
    for (int i = 0; i < n; ++i)
        T.consumer_shared[i] = (T.swept[i] && T.cls[i] == CLS_INTERIOR && T.shared_frame) ? 1 : 0;
    // points whose phase-A fluxes are computed before the sweeps: swept
    // points that evaluate their neighbours in their own frame
    T.g0_pts.clear();
    for (int i = 0; i < n; ++i)
        if (T.swept[i] && !T.consumer_shared[i] && T.cls[i] != CLS_SUPERSONIC) T.g0_pts.push_back(i);
    if (T.g0_pts.size() > (size_t)std::max(4096, n / 8) || T.g0_pts.size() >= (size_t)1 << 24)
        T.g0_pts.clear();
    return MFCFD_OK;
}

void chain_assign(const int32_t *lpts, int nsw, const int32_t *level, const int32_t *coff, const int32_t *cand, int n,
                  int warps, std::vector<int32_t> &owner, std::vector<std::vector<int32_t>> &lists) {
    owner.assign(n, -1);
    lists.assign(warps, {});
    std::vector<int32_t> last_point(warps, -1), last_level(warps, -1);
    // warps ordered by the level of their last point (lazy min-heap)
    std::vector<std::pair<int, int>> heap;
    auto cmp = [](const std::pair<int, int> &a, const std::pair<int, int> &b) {
        return a.first > b.first || (a.first == b.first && a.second > b.second);
    };
    for (int w = 0; w < warps; ++w) heap.push_back({-1, w});
    std::make_heap(heap.begin(), heap.end(), cmp);
    for (int li = 0; li < nsw; ++li) {   // level-major, a topological order
        const int p = lpts[li];
        // continue the warp of the last deepest dependency that is its
        // warp's latest point; otherwise the warp whose latest point is
        // shallowest
        int best = -1;
        for (int c = coff[p]; c < coff[p + 1]; ++c)
            if (last_point[owner[cand[c]]] == cand[c]) best = cand[c];
        int w = -1;
        if (best >= 0) {
            w = owner[best];
        } else {
            while (true) {     // pop stale heap entries
                std::pop_heap(heap.begin(), heap.end(), cmp);
                auto top = heap.back();
                heap.pop_back();
                if (top.first == last_level[top.second]) { w = top.second; break; }
            }
        }
        owner[p] = w;
        lists[w].push_back(p);
        last_point[w] = p;
        last_level[w] = level[p];
        heap.push_back({level[p], w});
        std::push_heap(heap.begin(), heap.end(), cmp);
    }
}

void build_chain_schedule(Topology &T, int warps, ChainSchedule &S) {
    S.warps = warps;
    const int n = T.n;
    std::vector<int32_t> g0_of(n, -1);
    for (size_t j = 0; j < T.g0_pts.size(); ++j) g0_of[T.g0_pts[j]] = (int32_t)j;
    for (int dir = 0; dir < 2; ++dir) {
        const bool fwd = dir == 0;
        const std::vector<int32_t> &lpts = fwd ? T.fwd_lvl_pts : T.bwd_lvl_pts;
        const std::vector<int32_t> &level = fwd ? T.fwd_level : T.bwd_level;
        const std::vector<int32_t> &off = fwd ? T.fwd_off : T.bwd_off;
        const std::vector<SweepEntry> &ent = fwd ? T.fwd_ent : T.bwd_ent;
        std::vector<int32_t> &owner = S.owner[dir];
        std::vector<std::vector<int32_t>> lists;
        // each point's dependencies of the deepest level, in entry order
        // (computed in parallel; the assignment below only reads them)
        std::vector<int32_t> coff(n + 1, 0), cand;
        parallel_for(n, [&](int p) {
            int best_level = -1, c = 0;
            for (int e = off[p]; e < off[p + 1]; ++e) {
                if (!entry_is_dependency(ent[e]) || !T.swept[ent[e].k]) continue;
                const int lv = level[ent[e].k];
                if (lv > best_level) { best_level = lv; c = 1; }
                else if (lv == best_level) ++c;
            }
            coff[p + 1] = c;
        });
        for (int p = 0; p < n; ++p) coff[p + 1] += coff[p];
        cand.resize((size_t)coff[n]);
        parallel_for(n, [&](int p) {
            // the deepest level first, so only its entries are written and
            // none lands past the point's own coff range
            int best_level = -1, at = coff[p];
            for (int e = off[p]; e < off[p + 1]; ++e)
                if (entry_is_dependency(ent[e]) && T.swept[ent[e].k]) best_level = std::max(best_level, level[ent[e].k]);
            for (int e = off[p]; e < off[p + 1]; ++e)
                if (entry_is_dependency(ent[e]) && T.swept[ent[e].k] && level[ent[e].k] == best_level)
                    cand[at++] = ent[e].k;
        });
        chain_assign(lpts.data(), (int)lpts.size(), level.data(), coff.data(), cand.data(), n, warps, owner,
                     lists);
        S.ptr[dir].assign(warps + 1, 0);
        S.pts[dir].clear();
        for (int w = 0; w < warps; ++w) {
            S.ptr[dir][w] = (int32_t)S.pts[dir].size();
            S.pts[dir].insert(S.pts[dir].end(), lists[w].begin(), lists[w].end());
        }
        S.ptr[dir][warps] = (int32_t)S.pts[dir].size();

        // where each term's producer increment comes from, and which points
        // must publish to global memory
        std::vector<int32_t> pos(n, -1);
        for (int w = 0; w < warps; ++w)
            for (int i = S.ptr[dir][w]; i < S.ptr[dir][w + 1]; ++i) pos[S.pts[dir][i]] = i - S.ptr[dir][w];
        std::vector<SweepEntry> &went = fwd ? T.fwd_ent : T.bwd_ent;
        std::vector<std::atomic<uint8_t>> publish(n);
        for (auto &v : publish) v.store(0, std::memory_order_relaxed);
        std::atomic<int64_t> n_ring{0}, n_local{0}, n_cross{0};
        parallel_for((int)lpts.size(), [&](int li) {
            const int p = lpts[li];
            const bool shared = T.consumer_shared[p] != 0;
            int64_t ring = 0, local = 0, cross = 0;
            for (int e = off[p]; e < off[p + 1]; ++e) {
                SweepEntry &E = went[e];
                E.pad &= ~ENT_CHAIN_BITS;
                if (E.pad & (ENT_COPY | ENT_OLD)) continue;   // dU or from before the sweep
                const int k = E.k;
                if (!T.swept[k]) continue;   // fixed increment written before the sweep
                const bool same = owner[k] == owner[p];
                if (!shared) continue;       // reads dU of its slots directly
                if (same && pos[p] - pos[k] <= CHAIN_RING) {
                    E.pad |= ENT_RING | ((pos[k] % CHAIN_RING) << ENT_RING_SHIFT);
                    ++ring;
                } else {
                    publish[k].store(1, std::memory_order_relaxed);
                    if (same) ++local;
                    else ++cross;
                }
            }
            n_ring += ring;
            n_local += local;
            n_cross += cross;
        });
        S.terms_ring += n_ring;
        S.terms_local += n_local;
        S.terms_cross += n_cross;
        const std::vector<uint8_t> &cnt = fwd ? T.fwd_cnt : T.bwd_cnt;
        std::vector<ChainItem> &items = S.items[dir];
        items.resize(S.pts[dir].size());
        for (size_t i = 0; i < items.size(); ++i) {
            const int p = S.pts[dir][i];
            ChainItem &it = items[i];
            it.p = p;
            it.off = off[p];
            it.cnt = 0;
            for (int e = 0; e < NDIR; ++e) it.cnt |= (uint32_t)cnt[(size_t)p * NDIR + e] << (5 * e);
            it.info = (T.cls[p] == CLS_WALL ? CI_WALL : 0u) | (T.consumer_shared[p] ? CI_SHARED : 0u) |
                      (publish[p].load(std::memory_order_relaxed) ? CI_PUBLISH : 0u) |
                      (T.cls[p] == CLS_SUPERSONIC ? CI_COPY : 0u) |
                      (T.cls[p] == CLS_OUTER ? CI_OUTER : 0u);
            if (g0_of[p] >= 0) it.info |= CI_G0 | ((uint32_t)g0_of[p] << CI_G0_SHIFT);
        }
    }
}

// Order in which the fused flux kernel visits the points: the forward
// sweep's levels, each preceded by the unswept points whose fixed increments
// that level reads first; points the forward sweep never reads come last.
void build_pre_order(const Topology &T, std::vector<int32_t> &order) {
    const int n = T.n;
    const int64_t last = INT64_MAX;
    std::vector<int64_t> key(n, last);
    for (int p = 0; p < n; ++p)
        if (T.swept[p]) key[p] = 2 * (int64_t)T.fwd_level[p] + 1;
    for (int p = 0; p < n; ++p) {
        if (!T.swept[p]) continue;
        for (int e = T.fwd_off[p]; e < T.fwd_off[p + 1]; ++e) {
            if (T.fwd_ent[e].pad & (ENT_COPY | ENT_OLD)) continue;   // not waiting on the flux kernel
            const int k = T.fwd_ent[e].k;
            if (!T.swept[k]) key[k] = std::min(key[k], 2 * (int64_t)T.fwd_level[p]);
        }
    }
    order.resize(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
}

// ---- storage order along a space-filling curve

namespace {

// the bits of v (21 of them) spread to every third bit
inline uint64_t spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// per-point rows of width w moved to their storage index
template <typename V>
void permute_rows(std::vector<V> &a, const std::vector<int32_t> &perm, size_t w) {
    if (a.empty()) return;
    std::vector<V> b(a.size());
    const int n = (int)perm.size();
    parallel_for(n, [&](int i) {
        std::copy(a.begin() + (size_t)i * w, a.begin() + (size_t)(i + 1) * w, b.begin() + (size_t)perm[i] * w);
    });
    a.swap(b);
}

// point ids (0-based; negative: none) mapped in place
void map_ids(std::vector<int32_t> &a, const std::vector<int32_t> &perm) {
    parallel_for((int)a.size(), [&](int j) {
        if (a[j] >= 0) a[j] = perm[a[j]];
    });
}

// a point's contiguous sweep entries, re-laid in storage order with mapped ids
void permute_entries(std::vector<int32_t> &off, std::vector<SweepEntry> &ent, const std::vector<int32_t> &perm,
                     const std::vector<int32_t> &inv) {
    const int n = (int)perm.size();
    std::vector<int32_t> noff(n + 1, 0);
    for (int q = 0; q < n; ++q) noff[q + 1] = noff[q] + (off[inv[q] + 1] - off[inv[q]]);
    std::vector<SweepEntry> nent(ent.size());
    parallel_for(n, [&](int q) {
        const int p = inv[q];
        int at = noff[q];
        for (int e = off[p]; e < off[p + 1]; ++e) {
            SweepEntry E = ent[e];
            if (E.k >= 0) E.k = perm[E.k];
            nent[at++] = E;
        }
    });
    off.swap(noff);
    ent.swap(nent);
}

}  // namespace

void morton_order(int n, const double *x, const double *y, const double *z, std::vector<int32_t> &perm) {
    double lo[3] = {x[0], y[0], z[0]}, hi[3] = {x[0], y[0], z[0]};
    for (int i = 1; i < n; ++i) {
        const double v[3] = {x[i], y[i], z[i]};
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], v[a]);
            hi[a] = std::max(hi[a], v[a]);
        }
    }
    double scale[3];
    for (int a = 0; a < 3; ++a) scale[a] = hi[a] > lo[a] ? 2097151.0 / (hi[a] - lo[a]) : 0.0;
    std::vector<std::pair<uint64_t, int32_t>> key(n);
    parallel_for(n, [&](int i) {
        const double v[3] = {x[i], y[i], z[i]};
        uint64_t q[3];
        for (int a = 0; a < 3; ++a) {
            double t = (v[a] - lo[a]) * scale[a];
            t = t < 0.0 ? 0.0 : (t > 2097151.0 ? 2097151.0 : t);
            q[a] = (uint64_t)t;
        }
        key[i] = {spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2), i};
    });
    std::sort(key.begin(), key.end());     // (key, index): ties in index order
    perm.assign(n, 0);
    for (int s = 0; s < n; ++s) perm[key[s].second] = s;
}

void permute_topology(Topology &T, const std::vector<int32_t> &perm) {
    const int n = T.n;
    T.perm = perm;
    T.inv.assign(n, 0);
    for (int i = 0; i < n; ++i) T.inv[perm[i]] = i;
    // per-point rows
    permute_rows(T.cls, perm, 1);
    permute_rows(T.slot_nbr, perm, MAX_SLOTS);
    map_ids(T.slot_nbr, perm);
    permute_rows(T.nslot, perm, 1);
    permute_rows(T.slot_mask, perm, MAX_SLOTS);
    permute_rows(T.list_cnt, perm, NDIR);
    permute_rows(T.list_ent, perm, (size_t)NDIR * LIST_STRIDE);
    permute_rows(T.geo, perm, GEO_STRIDE);
    permute_rows(T.eps2, perm, 1);
    permute_rows(T.wq, perm, MAX_CONN);
    permute_rows(T.wf, perm, MAX_SLOTS);
    permute_rows(T.fwd_level, perm, 1);
    permute_rows(T.bwd_level, perm, 1);
    permute_rows(T.fwd_cnt, perm, NDIR);
    permute_rows(T.bwd_cnt, perm, NDIR);
    permute_rows(T.fwd_need, perm, 1);
    permute_rows(T.bwd_need, perm, 1);
    permute_rows(T.fwd_old, perm, 1);
    permute_rows(T.bwd_old, perm, 1);
    permute_rows(T.sweep_slot_mask, perm, MAX_SLOTS);
    permute_rows(T.outer_delt, perm, 1);
    permute_rows(T.swept, perm, 1);
    permute_rows(T.consumer_shared, perm, 1);
    permute_rows(T.copy_src, perm, 1);
    map_ids(T.copy_src, perm);
    // entries of each sweep, contiguous per point in storage order
    permute_entries(T.fwd_off, T.fwd_ent, perm, T.inv);
    permute_entries(T.bwd_off, T.bwd_ent, perm, T.inv);
    // id lists, their order kept
    for (std::vector<int32_t> *a : {&T.fwd_lvl_pts, &T.bwd_lvl_pts, &T.wall_idx, &T.outer_idx, &T.interior_idx,
                                    &T.ss_inlet_idx, &T.ss_outlet_idx, &T.ss_pts, &T.ss_src, &T.g0_pts})
        map_ids(*a, perm);
}

}  // namespace mfcfd
