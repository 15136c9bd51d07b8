// Checks the invariants of the chain schedule (build_chain_schedule) that the
// sweep kernel relies on, for a cloud read from raw arrays in a directory:
//
//   status.bin x.bin y.bin z.bin tan1.bin tan2.bin nor.bin nbhs.bin conn.bin md.bin
//
// Usage: chain_schedule_check DIR N WARPS [sweep_variant]
// (WARPS < 0: -WARPS percent of the widest sweep level, as the library picks)
// Prints "ok <facts>" and exits 0, or prints the first violation and exits 1.
// Built by tests/test_chain_schedule.py together with csrc/mfcfd_setup.cpp.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "mfcfd_internal.h"

using namespace mfcfd;

namespace mfcfd {
// The GPU set-up passes are never requested here (device = -1).
int prep_split_gpu(int, int, int, const std::vector<int8_t> &, const double *, const double *, const double *,
                   const double *, const double *, const double *, const int32_t *, const int32_t *, Topology &,
                   bool *, std::string &) {
    return MFCFD_ERR_UNSUPPORTED;
}
int prep_alias_gpu(int, int, const int32_t *, const int32_t *, std::vector<int32_t> &, std::vector<int32_t> &,
                   std::string &) {
    return MFCFD_ERR_UNSUPPORTED;
}
int prep_levels_gpu(int, int, const std::vector<int> &, const std::vector<int32_t> &, const std::vector<int32_t> &,
                    std::vector<int32_t> &, std::string &) {
    return MFCFD_ERR_UNSUPPORTED;
}
}  // namespace mfcfd

namespace {

template <class T>
bool read_all(const std::string &path, std::vector<T> &v, size_t n) {
    v.resize(n);
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    const size_t got = std::fread(v.data(), sizeof(T), n, f);
    std::fclose(f);
    return got == n;
}

#define CHECK(cond, ...)                               \
    do {                                               \
        if (!(cond)) {                                 \
            std::printf("violation: " __VA_ARGS__);    \
            std::printf("\n");                         \
            return 1;                                  \
        }                                              \
    } while (0)

// FNV-1a over the bytes of a table
struct Hash {
    uint64_t h = 1469598103934665603ull;
    void bytes(const void *p, size_t n) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ull;
    }
    template <class T>
    void vec(const std::vector<T> &v) {
        const uint64_t n = v.size();
        bytes(&n, sizeof n);
        if (n) bytes(v.data(), sizeof(T) * n);
    }
};

bool same_items(const ChainSchedule &a, const ChainSchedule &b) {
    for (int d = 0; d < 2; ++d) {
        if (a.pts[d] != b.pts[d] || a.ptr[d] != b.ptr[d] || a.items[d].size() != b.items[d].size()) return false;
        for (size_t i = 0; i < a.items[d].size(); ++i) {
            const ChainItem &x = a.items[d][i], &y = b.items[d][i];
            if (x.p != y.p || x.off != y.off || x.cnt != y.cnt || x.info != y.info) return false;
        }
    }
    return true;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 4) {
        std::printf("usage: %s DIR N WARPS [sweep_variant]\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const int n = std::atoi(argv[2]);
    int warps = std::atoi(argv[3]);
    std::vector<int32_t> status, nbhs, conn;
    std::vector<double> x, y, z, t1, t2, nr, md;
    bool ok = read_all(dir + "/status.bin", status, n) && read_all(dir + "/x.bin", x, n) &&
              read_all(dir + "/y.bin", y, n) && read_all(dir + "/z.bin", z, n) &&
              read_all(dir + "/tan1.bin", t1, 3 * (size_t)n) && read_all(dir + "/tan2.bin", t2, 3 * (size_t)n) &&
              read_all(dir + "/nor.bin", nr, 3 * (size_t)n) && read_all(dir + "/nbhs.bin", nbhs, n) &&
              read_all(dir + "/conn.bin", conn, (size_t)MAX_CONN * n) && read_all(dir + "/md.bin", md, n);
    if (!ok) {
        std::printf("cannot read the cloud in %s\n", dir.c_str());
        return 2;
    }
    mfcfd_params P{};
    P.vl_const = 2.0;
    P.cfl = 5.0;
    P.split_capacity = 22;
    P.sweep_mode = MFCFD_SWEEP_CHAINS;
    P.sweep_variant = argc > 4 ? std::atoi(argv[4]) : MFCFD_SWEEPS_ALIAS;
    P.device = -1;
    Topology T;
    std::string err;
    const int rc = build_topology(P, n, status.data(), x.data(), y.data(), z.data(), t1.data(), t2.data(), nr.data(),
                                  nbhs.data(), conn.data(), md.data(), T, err);
    if (rc) {
        std::printf("set-up failed (%d): %s\n", rc, err.c_str());
        return 2;
    }
    if (warps < 0) warps = std::max(1, (int)((long)T.max_level_width * -warps / 100));
    ChainSchedule S, S2;
    build_chain_schedule(T, warps, S);
    build_chain_schedule(T, warps, S2);
    CHECK(same_items(S, S2), "two builds of the schedule differ");

    // the g0 points: swept points outside the shared frame, not copies
    std::vector<int32_t> g0_of(n, -1);
    {
        std::vector<int32_t> want;
        for (int i = 0; i < n; ++i)
            if (T.swept[i] && !T.consumer_shared[i] && T.cls[i] != CLS_SUPERSONIC) want.push_back(i);
        if (!T.g0_pts.empty()) CHECK(T.g0_pts == want, "g0 points are not the swept points outside the shared frame");
        else CHECK(want.size() > (size_t)std::max(4096, n / 8), "g0 table dropped below its size limit");
        for (size_t j = 0; j < T.g0_pts.size(); ++j) g0_of[T.g0_pts[j]] = (int32_t)j;
    }

    long ring_terms = 0, global_terms = 0;
    for (int d = 0; d < 2; ++d) {
        const bool fwd = d == 0;
        const std::vector<int32_t> &level = fwd ? T.fwd_level : T.bwd_level;
        const std::vector<int32_t> &lpts = fwd ? T.fwd_lvl_pts : T.bwd_lvl_pts;
        const std::vector<int32_t> &off = fwd ? T.fwd_off : T.bwd_off;
        const std::vector<uint8_t> &cnt = fwd ? T.fwd_cnt : T.bwd_cnt;
        const std::vector<SweepEntry> &ent = fwd ? T.fwd_ent : T.bwd_ent;
        const std::vector<int32_t> &ptr = S.ptr[d], &pts = S.pts[d], &owner = S.owner[d];
        const std::vector<ChainItem> &items = S.items[d];
        CHECK((int)ptr.size() == warps + 1 && ptr[0] == 0 && ptr[warps] == (int)pts.size(), "warp offsets");
        CHECK(pts.size() == lpts.size() && items.size() == pts.size(), "the schedule does not hold every swept point");
        std::vector<int32_t> seen(n, 0), pos(n, -1);
        for (int w = 0; w < warps; ++w) {
            CHECK(ptr[w] <= ptr[w + 1], "warp offsets decrease");
            for (int i = ptr[w]; i < ptr[w + 1]; ++i) {
                const int p = pts[i];
                CHECK(p >= 0 && p < n && T.swept[p], "a scheduled point is not swept");
                CHECK(++seen[p] == 1, "point %d is scheduled twice", p);
                CHECK(owner[p] == w, "owner of point %d", p);
                pos[p] = i - ptr[w];
                if (i > ptr[w]) CHECK(level[pts[i - 1]] <= level[p], "warp %d is not in level order", w);
            }
        }
        std::vector<uint8_t> publish(n, 0);
        for (size_t i = 0; i < items.size(); ++i) publish[items[i].p] = (items[i].info & CI_PUBLISH) ? 1 : 0;
        for (size_t i = 0; i < items.size(); ++i) {
            const ChainItem &it = items[i];
            const int p = it.p;
            CHECK(p == pts[i] && it.off == off[p], "item %zu does not describe point %d", i, p);
            for (int e = 0; e < NDIR; ++e)
                CHECK((int)((it.cnt >> (5 * e)) & 31u) == cnt[(size_t)p * NDIR + e], "item counts of point %d", p);
            CHECK(((it.info & CI_SHARED) != 0) == (T.consumer_shared[p] != 0), "shared flag of point %d", p);
            if (g0_of[p] >= 0)
                CHECK((it.info & CI_G0) && (int)(it.info >> CI_G0_SHIFT) == g0_of[p], "g0 mark of point %d", p);
            else
                CHECK(!(it.info & CI_G0) && (it.info >> CI_G0_SHIFT) == 0, "point %d marked g0", p);
            for (int e = off[p]; e < off[p + 1]; ++e) {
                const SweepEntry &E = ent[e];
                if (!entry_is_dependency(E) || !T.swept[E.k]) continue;
                const int k = E.k;
                CHECK(level[k] < level[p], "dependency %d of point %d is not on an earlier level", k, p);
                if (owner[k] == owner[p]) CHECK(pos[k] < pos[p], "dependency %d after point %d in its warp", k, p);
                if (!T.consumer_shared[p] || (E.pad & (ENT_COPY | ENT_OLD))) continue;
                if (E.pad & ENT_RING) {
                    ++ring_terms;
                    CHECK(owner[k] == owner[p] && pos[p] - pos[k] >= 1 && pos[p] - pos[k] <= CHAIN_RING,
                          "ring term %d -> %d outside the warp's last %d points", k, p, CHAIN_RING);
                    CHECK(((E.pad >> ENT_RING_SHIFT) & 15) == pos[k] % CHAIN_RING, "ring slot of %d -> %d", k, p);
                } else {
                    ++global_terms;
                    CHECK(publish[k], "point %d reads %d from global memory, which does not publish", p, k);
                }
            }
        }
    }
    Hash H;
    for (int d = 0; d < NDIR; ++d) {
        H.vec(T.split[d]);
        H.vec(T.split_cnt[d]);
    }
    H.vec(T.alias); H.vec(T.point_with_alias); H.vec(T.slot_nbr); H.vec(T.nslot); H.vec(T.slot_mask);
    H.vec(T.list_cnt); H.vec(T.list_ent); H.vec(T.geo); H.vec(T.eps2);
    H.vec(T.fwd_level); H.vec(T.bwd_level); H.vec(T.fwd_lvl_pts); H.vec(T.bwd_lvl_pts);
    H.vec(T.fwd_off); H.vec(T.bwd_off); H.vec(T.fwd_cnt); H.vec(T.bwd_cnt);
    H.vec(T.fwd_ent); H.vec(T.bwd_ent); H.vec(T.fwd_need); H.vec(T.bwd_need); H.vec(T.g0_pts);
    for (int d = 0; d < 2; ++d) {
        H.vec(S.ptr[d]);
        H.vec(S.pts[d]);
        H.vec(S.items[d]);
    }
    std::printf("ok ring %ld global %ld g0 %zu hash %016llx\n", ring_terms, global_terms, T.g0_pts.size(),
                (unsigned long long)H.h);
    return 0;
}
