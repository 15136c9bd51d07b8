/*
 * mfcfd_io.cpp - the reference program's file formats (host side).
 *
 * Readers follow Fortran list-directed input as the reference's READ
 * statements use it: each READ starts at a new record (line), takes values
 * separated by blanks, tabs, commas or line ends until its item list is
 * full, and discards the rest of the record it stopped in.  Values may carry
 * a repeat count (r*value); reals may use an E or D exponent.  Null values
 * and the slash terminator are rejected (the reference's files have none,
 * and they would leave items undefined).
 *
 *   3d_input_data        point_preprocessor.f90:25-36
 *   stored-solution.dat  initial_conditions.f90:18-29
 *
 * Writers produce the files of print_primal_output (post_processor.f90:13-44)
 * and the residue log (q_lskum.f90:22,31) in the layout of gfortran's
 * list-directed output: every record starts with a blank, an integer takes a
 * right-aligned field of 12, a real(8) is written with 17 significant digits
 * as by G25.17E3 (F form with five trailing blanks for 0.1 <= |x| < 1e17 and
 * zero, else E form with a three-digit exponent) after one blank.
 */
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mfcfd_internal.h"

namespace mfcfd {

thread_local std::string g_io_err;

namespace {

int io_fail(const std::string &msg) {
    g_io_err = msg;
    return MFCFD_ERR_IO;
}

bool read_file(const char *path, std::string &buf) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf.resize(sz > 0 ? (size_t)sz : 0);
    size_t got = sz > 0 ? std::fread(&buf[0], 1, (size_t)sz, f) : 0;
    std::fclose(f);
    buf.resize(got);
    return true;
}

// Fortran list-directed input over an in-memory file.
class ListInput {
public:
    explicit ListInput(const std::string &b) : buf_(b) {}

    // Start a READ statement: skip to the beginning of the next record
    // (the first READ starts at the first record).
    void begin() {
        if (started_) {
            while (pos_ < buf_.size() && buf_[pos_] != '\n') ++pos_;
            if (pos_ < buf_.size()) { ++pos_; ++line_; }
        }
        started_ = true;
        rep_left_ = 0;
    }

    // Next value token of the current READ (crossing record ends).
    // Returns false at end of file or on a null / slash (err set).
    bool next(std::string &tok, std::string &err) {
        if (rep_left_ > 0) {
            --rep_left_;
            tok = rep_tok_;
            return true;
        }
        for (;;) {
            while (pos_ < buf_.size() && (buf_[pos_] == ' ' || buf_[pos_] == '\t' || buf_[pos_] == '\r')) ++pos_;
            if (pos_ >= buf_.size()) { err = "unexpected end of file"; return false; }
            char ch = buf_[pos_];
            if (ch == '\n') { ++pos_; ++line_; continue; }
            if (ch == ',') { err = "null value (empty field) at line " + std::to_string(line_); return false; }
            if (ch == '/') { err = "slash terminator at line " + std::to_string(line_); return false; }
            size_t a = pos_;
            while (pos_ < buf_.size() && !std::strchr(" \t\r\n,/", buf_[pos_])) ++pos_;
            tok.assign(buf_, a, pos_ - a);
            // one value separator: blanks, then at most one comma
            while (pos_ < buf_.size() && (buf_[pos_] == ' ' || buf_[pos_] == '\t' || buf_[pos_] == '\r')) ++pos_;
            if (pos_ < buf_.size() && buf_[pos_] == ',') ++pos_;
            size_t star = tok.find('*');
            if (star != std::string::npos) {
                long r = 0;
                if (!parse_count(tok.substr(0, star), r) || r < 1) {
                    err = "bad repeat count '" + tok + "' at line " + std::to_string(line_);
                    return false;
                }
                if (star + 1 == tok.size()) { err = "null value (r*) at line " + std::to_string(line_); return false; }
                rep_tok_ = tok.substr(star + 1);
                rep_left_ = r - 1;
                tok = rep_tok_;
            }
            return true;
        }
    }

    int line() const { return line_; }

private:
    static bool parse_count(const std::string &s, long &v) {
        if (s.empty()) return false;
        for (char c : s) if (c < '0' || c > '9') return false;
        v = std::strtol(s.c_str(), nullptr, 10);
        return true;
    }
    const std::string &buf_;
    size_t pos_ = 0;
    int line_ = 1;
    bool started_ = false;
    long rep_left_ = 0;
    std::string rep_tok_;
};

bool parse_int(const std::string &t, int32_t &v) {
    size_t i = 0;
    if (i < t.size() && (t[i] == '+' || t[i] == '-')) ++i;
    if (i == t.size()) return false;
    for (size_t j = i; j < t.size(); ++j) if (t[j] < '0' || t[j] > '9') return false;
    errno = 0;
    long long x = std::strtoll(t.c_str(), nullptr, 10);
    if (errno || x < INT32_MIN || x > INT32_MAX) return false;
    v = (int32_t)x;
    return true;
}

// Fortran real input: [sign] digits [. digits] [exponent], the exponent
// letter E, D or Q (any case) or a bare signed exponent ("1.5-3").
bool parse_real(const std::string &t, double &v) {
    std::string s;
    s.reserve(t.size() + 1);
    size_t i = 0;
    if (i < t.size() && (t[i] == '+' || t[i] == '-')) s += t[i++];
    bool digits = false, dot = false;
    for (; i < t.size(); ++i) {
        char c = t[i];
        if (c >= '0' && c <= '9') { s += c; digits = true; }
        else if (c == '.' && !dot) { s += c; dot = true; }
        else break;
    }
    if (!digits) return false;
    if (i < t.size()) {
        char c = t[i];
        if (std::strchr("eEdDqQ", c)) ++i;
        else if (c != '+' && c != '-') return false;
        s += 'e';
        if (i < t.size() && (t[i] == '+' || t[i] == '-')) s += t[i++];
        const size_t d0 = i;
        for (; i < t.size() && t[i] >= '0' && t[i] <= '9'; ++i) s += t[i];
        if (i == d0 || i != t.size()) return false;
    }
    char *end = nullptr;
    v = std::strtod(s.c_str(), &end);
    return end && *end == '\0';
}

// gfortran-style list-directed output items.
void put_int(std::string &o, long long v) {
    char b[32];
    std::snprintf(b, sizeof b, "%12lld", v);
    o += b;
}

void put_real(std::string &o, double v) {
    char b[64];
    if (std::isnan(v) || std::isinf(v)) {
        std::snprintf(b, sizeof b, " %25s", std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity"));
        o += b;
        return;
    }
    // decimal exponent after rounding to 17 significant digits
    char e[64];
    std::snprintf(e, sizeof e, "%.16e", v);
    const char *ep = std::strchr(e, 'e');
    int x10 = ep ? std::atoi(ep + 1) : 0;
    if (v == 0.0 || (x10 >= -1 && x10 < 17)) {
        const int decimals = 16 - x10;   // 17 significant digits
        char f[64];
        std::snprintf(f, sizeof f, "%.*f", v == 0.0 ? 16 : decimals, v);
        std::string fs(f);
        if (v != 0.0 && decimals == 0) fs += '.';   // 17 digits before the point
        std::snprintf(b, sizeof b, " %20s     ", fs.c_str());
    } else {
        // mantissa d.dddddddddddddddd and a three-digit exponent: E-005
        std::string m(e, ep ? (size_t)(ep - e) : std::strlen(e));
        char ex[16];
        std::snprintf(ex, sizeof ex, "E%c%03d", x10 < 0 ? '-' : '+', x10 < 0 ? -x10 : x10);
        std::snprintf(b, sizeof b, " %25s", (m + ex).c_str());
    }
    o += b;
}

int write_text(const std::string &path, const std::string &text, bool append) {
    FILE *f = std::fopen(path.c_str(), append ? "ab" : "wb");
    if (!f) return io_fail("cannot open " + path + " for writing: " + std::strerror(errno));
    size_t w = std::fwrite(text.data(), 1, text.size(), f);
    int rc = std::fclose(f);
    if (w != text.size() || rc != 0) return io_fail("write to " + path + " failed");
    return MFCFD_OK;
}

}  // namespace

int io_count_input_points(const char *path, int32_t *n) {
    std::string buf;
    if (!read_file(path, buf)) return io_fail(std::string("cannot open ") + path + ": " + std::strerror(errno));
    ListInput in(buf);
    int32_t count = 0;
    std::string tok, err;
    for (;;) {
        in.begin();
        // a record is: idx status x y z tan1(3) tan2(3) nor(3) nbhs conn(nbhs) min_dist
        if (!in.next(tok, err)) {
            if (err == "unexpected end of file") break;
            return io_fail(err);
        }
        for (int i = 1; i < 14; ++i)
            if (!in.next(tok, err)) return io_fail("record " + std::to_string(count + 1) + ": " + err);
        int32_t nb = 0;
        if (!in.next(tok, err) || !parse_int(tok, nb) || nb < 0 || nb > MAX_CONN)
            return io_fail("record " + std::to_string(count + 1) + ": bad nbhs");
        for (int i = 0; i < nb + 1; ++i)
            if (!in.next(tok, err)) return io_fail("record " + std::to_string(count + 1) + ": " + err);
        ++count;
    }
    *n = count;
    return MFCFD_OK;
}

int io_read_input_point_data(const char *path, int32_t n, int32_t *status, double *x, double *y,
                             double *z, double *tan1, double *tan2, double *nor, int32_t *nbhs,
                             int32_t *conn, double *min_dist) {
    std::string buf;
    if (!read_file(path, buf)) return io_fail(std::string("cannot open ") + path + ": " + std::strerror(errno));
    ListInput in(buf);
    std::string tok, err;
    for (int32_t k = 0; k < n; ++k) {
        in.begin();
        const std::string where = " in record " + std::to_string(k + 1) + " (line " + std::to_string(in.line()) + ")";
        auto real = [&](double &v) {
            if (!in.next(tok, err)) return false;
            if (!parse_real(tok, v)) { err = "bad real '" + tok + "'"; return false; }
            return true;
        };
        auto integer = [&](int32_t &v) {
            if (!in.next(tok, err)) return false;
            if (!parse_int(tok, v)) { err = "bad integer '" + tok + "'"; return false; }
            return true;
        };
        int32_t counter = 0;
        bool ok = integer(counter) && integer(status[k]) && real(x[k]) && real(y[k]) && real(z[k]);
        for (int r = 0; ok && r < 3; ++r) ok = real(tan1[3 * (size_t)k + r]);
        for (int r = 0; ok && r < 3; ++r) ok = real(tan2[3 * (size_t)k + r]);
        for (int r = 0; ok && r < 3; ++r) ok = real(nor[3 * (size_t)k + r]);
        ok = ok && integer(nbhs[k]);
        if (ok && (nbhs[k] < 0 || nbhs[k] > MAX_CONN)) {
            ok = false;
            err = "nbhs " + std::to_string(nbhs[k]) + " outside [0, 27]";
        }
        for (int r = 0; ok && r < MAX_CONN; ++r) conn[(size_t)k * MAX_CONN + r] = 0;
        for (int r = 0; ok && r < nbhs[k]; ++r) ok = integer(conn[(size_t)k * MAX_CONN + r]);
        ok = ok && real(min_dist[k]);
        if (!ok) return io_fail(std::string(path) + where + ": " + err);
    }
    return MFCFD_OK;
}

int io_read_stored_solution(const char *path, int32_t n, double *prim) {
    std::string buf;
    if (!read_file(path, buf)) return io_fail(std::string("cannot open ") + path + ": " + std::strerror(errno));
    ListInput in(buf);
    std::string tok, err;
    for (int32_t k = 0; k < n; ++k) {
        in.begin();
        double v[8];
        for (int r = 0; r < 8; ++r) {
            if (!in.next(tok, err)) return io_fail(std::string(path) + " record " + std::to_string(k + 1) + ": " + err);
            if (!parse_real(tok, v[r]))
                return io_fail(std::string(path) + " record " + std::to_string(k + 1) + ": bad real '" + tok + "'");
        }
        for (int r = 0; r < 5; ++r) prim[5 * (size_t)k + r] = v[3 + r];   // x y z are read and dropped
    }
    return MFCFD_OK;
}

int io_write_primal_output(const std::string &dir, int32_t n, const int32_t *status, const double *x,
                           const double *y, const double *z, const double *prim, const double *flux_res,
                           const double *dq) {
    std::string a, b, c;
    a.reserve((size_t)n * 8 * 26 + 16);
    b.reserve((size_t)n * (24 + 5 * 26) + 16);
    c.reserve((size_t)n * (24 + 5 * 26) + 16);
    for (int32_t k = 0; k < n; ++k) {
        // primal-solution.dat: x y z prim(1:5)  (post_processor.f90:33)
        put_real(a, x[k]); put_real(a, y[k]); put_real(a, z[k]);
        for (int r = 0; r < 5; ++r) put_real(a, prim[5 * (size_t)k + r]);
        a += '\n';
        // qderivatives.dat: k status dq(3,1:5,k), the z-derivatives (:34)
        put_int(b, k + 1); put_int(b, status[k]);
        for (int r = 0; r < 5; ++r) put_real(b, dq[15 * (size_t)k + 3 * r + 2]);
        b += '\n';
        // flux-residual.dat: k status flux_res(1:5,k)  (:35)
        put_int(c, k + 1); put_int(c, status[k]);
        for (int r = 0; r < 5; ++r) put_real(c, flux_res[5 * (size_t)k + r]);
        c += '\n';
    }
    const std::string sep = dir.empty() || dir.back() == '/' ? "" : "/";
    int rc;
    if ((rc = write_text(dir + sep + "primal-solution.dat", a, false))) return rc;
    if ((rc = write_text(dir + sep + "normals.dat", "", false))) return rc;   // opened, never written
    if ((rc = write_text(dir + sep + "flux-residual.dat", c, false))) return rc;
    if ((rc = write_text(dir + sep + "qderivatives.dat", b, false))) return rc;
    return MFCFD_OK;
}

int io_write_residue(const char *path, int32_t t0, int32_t iters, const double *res_hist, int append) {
    std::string o;
    for (int32_t j = 0; j < iters; ++j) {
        put_int(o, t0 + j);
        put_real(o, res_hist[2 * (size_t)j]);
        put_real(o, res_hist[2 * (size_t)j + 1]);
        o += '\n';
    }
    return write_text(path, o, append != 0);
}

}  // namespace mfcfd
