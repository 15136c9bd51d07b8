/*
 * CPU oracle for the q-LSKUM implicit iteration -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, routine by routine, the reference's active build set
 * (the Fortran files named in each function's comment).  It exists to check
 * the CUDA library: only the tests, the smoke check and the CPU-baseline leg
 * of bench.py load it.  The product path never calls it.
 *
 * Parity pin: the reference has no tests, fixtures or data, and no Fortran
 * compiler exists on this machine.  The restatement is pinned instead against
 * a mechanical C translation of the reference's own Fortran sources
 * (oracle/f2c_ref.py -> oracle/_ref/libref.so) run on the same inputs; the
 * tests compare the two bit for bit.
 *
 * Semantics kept from the Fortran:
 *   - evaluation order left to right, no fused multiply-add (build with
 *     -ffp-contract=off), division where the source divides and
 *     multiplication by a reciprocal where it does (outer fluxes);
 *   - the single-precision literal 10e-6 in the limiter (limiters.f90:242)
 *     is (double)1.0e-5f;
 *   - arrays are 1-based with index 0 a zero guard, so the out-of-range
 *     entry point_with_alias(N)=0 of the alias quirk (implicit_aliasing.f90:
 *     276-291) reads zeros; the sweeps skip p=0 (it touches no real point);
 *   - the six split lists have the reference's capacity of 22 entries per
 *     point (data_structure.f90:83-88) stored column-major in one flat array,
 *     so an overflowing list spills into the next point's column exactly as
 *     unchecked Fortran indexing does; a tail pad stands in for the memory
 *     after the last column.
 * Transcendentals: glibc exp/log/erf/pow (what gfortran calls) by default;
 * libm mode 1 switches exp/log/erf to the solver's own mfmath.h functions.
 */
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../3d-mfcfd_b200/csrc/mfmath.h"

// Phase marks for the counting build (oracle_flops.cpp); nothing otherwise.
#ifndef ORACLE_PHASE
#define ORACLE_PHASE(k) ((void)0)
#endif

namespace {

struct OracleParams {
    double power, vl_const, cfl;
    double rho_inf, u1_inf, u2_inf, u3_inf, pr_inf;
    int inner_iterations;
    int split_capacity;   // 22 in the reference
    int update_variant;   // 0 state_update_implicit.f90, 1 state_update.f90
    int sweep_variant;    // 0 implicit_forward_and_reverse_sweeps.f90, 1 ..._backup.f90
};

const double PI = 3.141592653589793;           // 4*datan(1d0), parameter.f90:19
const double LIM_EPS = (double)1.0e-5f;        // 10e-6 (REAL*4), limiters.f90:242

int g_libm = 0;   // 0: glibc, 1: mfmath

inline double o_exp(double x) { return g_libm ? mf_exp(x) : std::exp(x); }
inline double o_log(double x) { return g_libm ? mf_log(x) : std::log(x); }
inline double o_erf(double x) { return g_libm ? mf_erf(x) : std::erf(x); }

struct Oracle {
    OracleParams P;
    int N;
    int cap;
    std::vector<double> x, y, z, tan1, tan2, nor, min_dist;
    std::vector<int> status, nbhs, conn;
    std::vector<int> xpos_nbhs, xneg_nbhs, ypos_nbhs, yneg_nbhs, zpos_nbhs, zneg_nbhs;
    std::vector<int> xpos_conn, xneg_conn, ypos_conn, yneg_conn, zpos_conn, zneg_conn;
    std::vector<double> U, delUp, delUn, prim, flux_res, q, qm, dq, temp_dq, delt, dinv;
    std::vector<double> delUp_fwd;   // delUp as the forward sweep left it (a diagnostic)
    std::vector<int> alias, point_with_alias;
    std::vector<int> interior_idx, wall_idx, outer_idx, ss_inlet_idx, ss_outlet_idx;
    double res_old = 0, res_new = 0, residue = 0, max_res = 0;
    int max_res_point = 0;

    // 1-based accessors (index 0 is a zero guard)
    double &TAN1(int r, int k) { return tan1[(size_t)k * 3 + r - 1]; }
    double &TAN2(int r, int k) { return tan2[(size_t)k * 3 + r - 1]; }
    double &NOR(int r, int k) { return nor[(size_t)k * 3 + r - 1]; }
    int &CONN(int r, int k) { return conn[(size_t)k * 27 + r - 1]; }
    double &V5(std::vector<double> &a, int r, int k) { return a[(size_t)k * 5 + r - 1]; }
    double &QM(int a, int r, int k) { return qm[(size_t)k * 10 + (size_t)(r - 1) * 2 + a - 1]; }
    double &DQ(int a, int r, int k) { return dq[(size_t)k * 15 + (size_t)(r - 1) * 3 + a - 1]; }
    double &TDQ(int a, int r, int k) { return temp_dq[(size_t)k * 15 + (size_t)(r - 1) * 3 + a - 1]; }
    // split lists: column-major (cap, N) without bounds checks, like Fortran
    int &SL(std::vector<int> &a, int j, int k) { return a[(size_t)(k - 1) * cap + (j - 1)]; }
};

// ---------------------------------------------------------------- setup

// point_preprocessor.f90:41-95: class counts and index lists.
void build_index_lists(Oracle &o) {
    for (int k = 1; k <= o.N; ++k) {
        int s = o.status[k];
        if (s == 0) o.interior_idx.push_back(k);
        else if (s == 1) o.wall_idx.push_back(k);
        else if (s == 2) o.outer_idx.push_back(k);
        else if (s == 6) o.ss_outlet_idx.push_back(k);
        else if (s == 5) o.ss_inlet_idx.push_back(k);
    }
}

// generate_connectivity.f90:38-111
void interior_neighbours(Oracle &o, int i) {
    double xi = o.x[i], yi = o.y[i], zi = o.z[i];
    o.xpos_nbhs[i] = 0; o.xneg_nbhs[i] = 0; o.ypos_nbhs[i] = 0;
    o.yneg_nbhs[i] = 0; o.zpos_nbhs[i] = 0; o.zneg_nbhs[i] = 0;
    for (int r = 1; r <= o.nbhs[i]; ++r) {
        int k = o.CONN(r, i);
        double delx = o.x[k] - xi, dely = o.y[k] - yi, delz = o.z[k] - zi;
        double dels = delx * o.TAN1(1, i) + dely * o.TAN1(2, i) + delz * o.TAN1(3, i);
        double delt = delx * o.TAN2(1, i) + dely * o.TAN2(2, i) + delz * o.TAN2(3, i);
        double deln = delx * o.NOR(1, i) + dely * o.NOR(2, i) + delz * o.NOR(3, i);
        if (dels <= 0.0) { o.SL(o.xpos_conn, ++o.xpos_nbhs[i], i) = k; }
        if (dels > 0.0) { o.SL(o.xneg_conn, ++o.xneg_nbhs[i], i) = k; }
        if (delt <= 0.0) { o.SL(o.ypos_conn, ++o.ypos_nbhs[i], i) = k; }
        if (delt > 0.0) { o.SL(o.yneg_conn, ++o.yneg_nbhs[i], i) = k; }
        if (deln <= 0.0) { o.SL(o.zpos_conn, ++o.zpos_nbhs[i], i) = k; }
        if (deln > 0.0) { o.SL(o.zneg_conn, ++o.zneg_nbhs[i], i) = k; }
    }
}

// generate_connectivity.f90:115-178 (zpos_nbhs is not touched)
void wall_neighbours(Oracle &o, int i) {
    double xi = o.x[i], yi = o.y[i], zi = o.z[i];
    o.xpos_nbhs[i] = 0; o.xneg_nbhs[i] = 0; o.ypos_nbhs[i] = 0;
    o.yneg_nbhs[i] = 0; o.zneg_nbhs[i] = 0;
    for (int r = 1; r <= o.nbhs[i]; ++r) {
        int k = o.CONN(r, i);
        double delx = o.x[k] - xi, dely = o.y[k] - yi, delz = o.z[k] - zi;
        double dels = delx * o.TAN1(1, i) + dely * o.TAN1(2, i) + delz * o.TAN1(3, i);
        double delt = delx * o.TAN2(1, i) + dely * o.TAN2(2, i) + delz * o.TAN2(3, i);
        if (dels <= 0.0) { o.SL(o.xpos_conn, ++o.xpos_nbhs[i], i) = k; }
        if (dels >= 0.0) { o.SL(o.xneg_conn, ++o.xneg_nbhs[i], i) = k; }
        if (delt <= 0.0) { o.SL(o.ypos_conn, ++o.ypos_nbhs[i], i) = k; }
        if (delt >= 0.0) { o.SL(o.yneg_conn, ++o.yneg_nbhs[i], i) = k; }
        o.SL(o.zneg_conn, ++o.zneg_nbhs[i], i) = k;
    }
}

// generate_connectivity.f90:182-246 (zpos_nbhs is not reset: starts from 0)
void outer_neighbours(Oracle &o, int i) {
    double xi = o.x[i], yi = o.y[i], zi = o.z[i];
    o.xpos_nbhs[i] = 0; o.xneg_nbhs[i] = 0; o.ypos_nbhs[i] = 0;
    o.yneg_nbhs[i] = 0; o.zneg_nbhs[i] = 0;
    for (int r = 1; r <= o.nbhs[i]; ++r) {
        int k = o.CONN(r, i);
        double delx = o.x[k] - xi, dely = o.y[k] - yi, delz = o.z[k] - zi;
        double dels = delx * o.TAN1(1, i) + dely * o.TAN1(2, i) + delz * o.TAN1(3, i);
        double delt = delx * o.TAN2(1, i) + dely * o.TAN2(2, i) + delz * o.TAN2(3, i);
        if (dels <= 0.0) { o.SL(o.xpos_conn, ++o.xpos_nbhs[i], i) = k; }
        if (dels >= 0.0) { o.SL(o.xneg_conn, ++o.xneg_nbhs[i], i) = k; }
        if (delt <= 0.0) { o.SL(o.ypos_conn, ++o.ypos_nbhs[i], i) = k; }
        if (delt >= 0.0) { o.SL(o.yneg_conn, ++o.yneg_nbhs[i], i) = k; }
        o.SL(o.zpos_conn, ++o.zpos_nbhs[i], i) = k;
    }
}

// generate_connectivity.f90:12-34
void generate_split_stencils(Oracle &o) {
    for (int i : o.interior_idx) interior_neighbours(o, i);
    for (int i : o.wall_idx) wall_neighbours(o, i);
    for (int i : o.outer_idx) outer_neighbours(o, i);
}

// implicit_aliasing.f90:13-44 (p = 0 reads the zero guard: nbhs(0) = 0)
void aliasing(Oracle &o) {
    for (int i = 1; i <= o.N; ++i) { o.alias[i] = 0; o.point_with_alias[i] = 0; }
    o.alias[1] = 1;
    o.point_with_alias[1] = 1;
    int count = 0;
    for (int i = 1; i <= o.N; ++i) {
        int p = o.point_with_alias[i];
        for (int j = 1; j <= o.nbhs[p]; ++j) {
            int k = o.CONN(j, p);
            if (o.alias[k] == 0) {
                count = count + 1;
                o.alias[k] = count;
                o.point_with_alias[count] = k;
            }
        }
    }
}

// ---------------------------------------------------------------- physics

// split_fluxes.f90:11-308
enum FluxKind { GXP, GXN, GYP, GYN, GZP, GZN, GWXP, GWXN, GWYP, GWYN, GOXP, GOXN, GOYP, GOYN };

void flux(int kind, double G[5], const double t1[3], const double t2[3], const double n[3],
          const double prim[5]) {
    double rho = prim[0], u1 = prim[1], u2 = prim[2], u3 = prim[3], pr = prim[4];
    double ut1 = t1[0] * u1 + t1[1] * u2 + t1[2] * u3;
    double ut2 = t2[0] * u1 + t2[1] * u2 + t2[2] * u3;
    double un = n[0] * u1 + n[1] * u2 + n[2] * u3;
    double beta = 0.5 * rho / pr;
    double u_sqr = ut1 * ut1 + ut2 * ut2 + un * un;
    double temp1;
    switch (kind) {
    case GXP: case GXN: {   // split_fluxes.f90:11-59, 63-109
        double S1 = ut1 * std::sqrt(beta);
        double B1 = 0.5 * o_exp(-(S1 * S1)) / std::sqrt(PI * beta);
        double A1 = (kind == GXP) ? 0.5 * (1.0 + o_erf(S1)) : 0.5 * (1.0 - o_erf(S1));
        temp1 = (kind == GXP) ? (ut1 * A1 + B1) : (ut1 * A1 - B1);
        G[0] = rho * temp1;
        G[1] = pr * A1 + rho * ut1 * temp1;
        G[2] = rho * ut2 * temp1;
        G[3] = rho * un * temp1;
        temp1 = 2.5 * pr + 0.5 * rho * u_sqr;
        G[4] = (kind == GXP) ? (temp1 + pr) * ut1 * A1 + (temp1 + 0.5 * pr) * B1
                             : (temp1 + pr) * ut1 * A1 - (temp1 + 0.5 * pr) * B1;
        return;
    }
    case GYP: case GYN: {   // split_fluxes.f90:112-158, 161-207
        double S2 = ut2 * std::sqrt(beta);
        double B2 = 0.5 * o_exp(-(S2 * S2)) / std::sqrt(PI * beta);
        double A2 = (kind == GYP) ? 0.5 * (1.0 + o_erf(S2)) : 0.5 * (1.0 - o_erf(S2));
        temp1 = (kind == GYP) ? (ut2 * A2 + B2) : (ut2 * A2 - B2);
        G[0] = rho * temp1;
        G[1] = rho * ut1 * temp1;
        G[2] = pr * A2 + rho * ut2 * temp1;
        G[3] = rho * un * temp1;
        temp1 = 2.5 * pr + 0.5 * rho * u_sqr;
        G[4] = (kind == GYP) ? (temp1 + pr) * ut2 * A2 + (temp1 + 0.5 * pr) * B2
                             : (temp1 + pr) * ut2 * A2 - (temp1 + 0.5 * pr) * B2;
        return;
    }
    case GZP: case GZN: {   // split_fluxes.f90:210-257, 260-308
        double S3 = un * std::sqrt(beta);
        double B3 = 0.5 * o_exp(-(S3 * S3)) / std::sqrt(PI * beta);
        double A3 = (kind == GZP) ? 0.5 * (1.0 + o_erf(S3)) : 0.5 * (1.0 - o_erf(S3));
        temp1 = (kind == GZP) ? (un * A3 + B3) : (un * A3 - B3);
        G[0] = rho * temp1;
        G[1] = rho * ut1 * temp1;
        G[2] = rho * ut2 * temp1;
        G[3] = pr * A3 + rho * un * temp1;
        temp1 = 2.5 * pr + 0.5 * rho * u_sqr;
        G[4] = (kind == GZP) ? (temp1 + pr) * un * A3 + (temp1 + 0.5 * pr) * B3
                             : (temp1 + pr) * un * A3 - (temp1 + 0.5 * pr) * B3;
        return;
    }
    default: break;
    }
    // octant_fluxes.f90:9-442.  x variants use (S1, S3); y variants (S2, S3).
    bool xdir = (kind == GWXP || kind == GWXN || kind == GOXP || kind == GOXN);
    bool tpos = (kind == GWXP || kind == GWYP || kind == GOXP || kind == GOYP);
    bool wall = (kind == GWXP || kind == GWXN || kind == GWYP || kind == GWYN);
    double ut = xdir ? ut1 : ut2;
    double S = ut * std::sqrt(beta);
    double S3 = un * std::sqrt(beta);
    double B = 0.5 * o_exp(-(S * S)) / std::sqrt(PI * beta);
    double B3 = 0.5 * o_exp(-(S3 * S3)) / std::sqrt(PI * beta);
    double A = tpos ? 0.5 * (1.0 + o_erf(S)) : 0.5 * (1.0 - o_erf(S));
    double A3 = wall ? 0.5 * (1.0 - o_erf(S3)) : 0.5 * (1.0 + o_erf(S3));
    temp1 = tpos ? (ut * A + B) : (ut * A - B);
    G[0] = rho * temp1 * A3;
    if (xdir) {
        G[1] = (pr * A + rho * ut1 * temp1) * A3;
        G[2] = rho * ut2 * temp1 * A3;
    } else {
        G[1] = rho * ut1 * temp1 * A3;
        G[2] = (pr * A + rho * ut2 * temp1) * A3;
    }
    G[3] = wall ? rho * temp1 * (un * A3 - B3) : rho * temp1 * (un * A3 + B3);
    double temp2 = 2.5 * pr + 0.5 * rho * u_sqr;
    double temp3 = tpos ? (temp2 + pr) * ut * A + (temp2 + 0.5 * pr) * B
                        : (temp2 + pr) * ut * A - (temp2 + 0.5 * pr) * B;
    G[4] = wall ? temp3 * A3 - 0.5 * rho * un * B3 * temp1
                : temp3 * A3 + 0.5 * rho * un * B3 * temp1;
}

// limiters.f90:12-52
void venkat_limiter(Oracle &o, const double qtilde[5], double phi[5], int k) {
    for (int r = 1; r <= 5; ++r) {
        double q = o.V5(o.q, r, k);
        double del_neg = qtilde[r - 1] - q;
        double del_pos = 0.0;
        if (std::fabs(del_neg) <= LIM_EPS) {
            phi[r - 1] = 1.0;
        } else if (std::fabs(del_neg) > LIM_EPS) {
            if (del_neg > 0.0) del_pos = o.QM(1, r, k) - q;
            else if (del_neg < 0.0) del_pos = o.QM(2, r, k) - q;
            double epsi = o.P.vl_const * o.min_dist[k];
            epsi = std::pow(epsi, 3.0);
            double num = (del_pos * del_pos) + (epsi * epsi);
            num = num * del_neg + 2.0 * del_neg * del_neg * del_pos;
            double den = del_pos * del_pos + 2.0 * del_neg * del_neg;
            den = den + del_neg * del_pos + epsi * epsi;
            den = den * del_neg;
            double temp = num / den;
            phi[r - 1] = (temp < 1.0) ? temp : 1.0;
        }
    }
}

// qvariables_to_primitive_variables.f90:9-31
void qtilde_to_primitive(const double q[5], double prim[5]) {
    double beta = -q[4] * 0.5;
    double temp = 0.5 / beta;
    prim[1] = q[1] * temp;
    prim[2] = q[2] * temp;
    prim[3] = q[3] * temp;
    double temp1 = q[0] + beta * (prim[1] * prim[1] + prim[2] * prim[2] + prim[3] * prim[3]);
    double temp2 = temp1 - (o_log(beta) * 2.5);
    prim[0] = o_exp(temp2);
    prim[4] = prim[0] * temp;
}

// get_primitive_vector.f90:10-41 (mutates U like the Fortran does)
void get_primitive_vector(Oracle &o, int k, double U[5], double prim[5]) {
    prim[0] = U[0];
    double temp = 1.0 / U[0];
    double U2r = U[1], U3r = U[2], U4r = U[3];
    U[1] = o.TAN1(1, k) * U2r + o.TAN2(1, k) * U3r + o.NOR(1, k) * U4r;
    U[2] = o.TAN1(2, k) * U2r + o.TAN2(2, k) * U3r + o.NOR(2, k) * U4r;
    U[3] = o.TAN1(3, k) * U2r + o.TAN2(3, k) * U3r + o.NOR(3, k) * U4r;
    prim[1] = temp * U[1];
    prim[2] = temp * U[2];
    prim[3] = temp * U[3];
    temp = prim[1] * prim[1] + prim[2] * prim[2] + prim[3] * prim[3];
    prim[4] = 0.4 * (U[4] - 0.5 * prim[0] * temp);
}

// conserved_to_primitive_vector.f90:10-42
void conserved_to_primitive(Oracle &o, int k, double U[5]) {
    double prim[5];
    get_primitive_vector(o, k, U, prim);   // identical arithmetic
    for (int r = 1; r <= 5; ++r) o.V5(o.prim, r, k) = prim[r - 1];
}

// conserved_vector_Ubar.f90:8-64
void conserved_vector_Ubar(Oracle &o, int k, double Ubar[5]) {
    const OracleParams &P = o.P;
    double u1_inf_rot = P.u1_inf * o.TAN1(1, k) + P.u2_inf * o.TAN1(2, k) + P.u3_inf * o.TAN1(3, k);
    double u2_inf_rot = P.u1_inf * o.TAN2(1, k) + P.u2_inf * o.TAN2(2, k) + P.u3_inf * o.TAN2(3, k);
    double u3_inf_rot = P.u1_inf * o.NOR(1, k) + P.u2_inf * o.NOR(2, k) + P.u3_inf * o.NOR(3, k);
    double rho_e_inf = P.pr_inf * 2.5 + 0.5 * P.rho_inf *
        (u1_inf_rot * u1_inf_rot + u2_inf_rot * u2_inf_rot + u3_inf_rot * u3_inf_rot);
    double beta = (0.5 * P.rho_inf) / P.pr_inf;
    double S3 = u3_inf_rot * std::sqrt(beta);
    double B3_inf = o_exp(-(S3 * S3)) / (2.0 * std::sqrt(PI * beta));
    double A3n_inf = 0.5 * (1.0 - o_erf(S3));
    double rho = o.V5(o.prim, 1, k), u1 = o.V5(o.prim, 2, k), u2 = o.V5(o.prim, 3, k);
    double u3 = o.V5(o.prim, 4, k), pr = o.V5(o.prim, 5, k);
    double u1_rot = u1 * o.TAN1(1, k) + u2 * o.TAN1(2, k) + u3 * o.TAN1(3, k);
    double u2_rot = u1 * o.TAN2(1, k) + u2 * o.TAN2(2, k) + u3 * o.TAN2(3, k);
    double u3_rot = u1 * o.NOR(1, k) + u2 * o.NOR(2, k) + u3 * o.NOR(3, k);
    double rho_e = pr * 2.5 + 0.5 * rho * (u1_rot * u1_rot + u2_rot * u2_rot + u3_rot * u3_rot);
    beta = (0.5 * rho) / pr;
    S3 = u3_rot * std::sqrt(beta);
    double B3 = o_exp(-(S3 * S3)) / (2.0 * std::sqrt(PI * beta));
    double A3p = 0.5 * (1.0 + o_erf(S3));
    Ubar[0] = (P.rho_inf * A3n_inf) + (rho * A3p);
    Ubar[1] = (P.rho_inf * u1_inf_rot * A3n_inf) + (rho * u1_rot * A3p);
    Ubar[2] = (P.rho_inf * u2_inf_rot * A3n_inf) + (rho * u2_rot * A3p);
    double temp1 = P.rho_inf * (u3_inf_rot * A3n_inf - B3_inf);
    double temp2 = rho * (u3_rot * A3p + B3);
    Ubar[3] = temp1 + temp2;
    temp1 = (rho_e_inf * A3n_inf - 0.5 * P.rho_inf * u3_inf_rot * B3_inf);
    temp2 = (rho_e * A3p + 0.5 * rho * u3_rot * B3);
    Ubar[4] = temp1 + temp2;
}

// ---------------------------------------------------------------- phases

// compute_conserved_vector.f90:13-34
void compute_conserved_vector(Oracle &o) {
    for (int k = 1; k <= o.N; ++k) {
        double *p = &o.V5(o.prim, 1, k);
        o.V5(o.U, 1, k) = p[0];
        double temp1 = p[0] * p[1], temp2 = p[0] * p[2], temp3 = p[0] * p[3];
        o.V5(o.U, 2, k) = temp1 * o.TAN1(1, k) + temp2 * o.TAN1(2, k) + temp3 * o.TAN1(3, k);
        o.V5(o.U, 3, k) = temp1 * o.TAN2(1, k) + temp2 * o.TAN2(2, k) + temp3 * o.TAN2(3, k);
        o.V5(o.U, 4, k) = temp1 * o.NOR(1, k) + temp2 * o.NOR(2, k) + temp3 * o.NOR(3, k);
        temp1 = p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
        o.V5(o.U, 5, k) = 2.5 * p[4] + 0.5 * o.V5(o.U, 1, k) * temp1;
    }
}

// q_variables.f90:10-40
void eval_q_variables(Oracle &o) {
    for (int k = 1; k <= o.N; ++k) {
        double rho = o.V5(o.prim, 1, k), u1 = o.V5(o.prim, 2, k), u2 = o.V5(o.prim, 3, k);
        double u3 = o.V5(o.prim, 4, k), pr = o.V5(o.prim, 5, k);
        double beta = 0.5 * rho / pr;
        o.V5(o.q, 1, k) = o_log(rho) + (o_log(beta) * 2.5) - beta * (u1 * u1 + u2 * u2 + u3 * u3);
        double two_times_beta = 2.0 * beta;
        o.V5(o.q, 2, k) = two_times_beta * u1;
        o.V5(o.q, 3, k) = two_times_beta * u2;
        o.V5(o.q, 4, k) = two_times_beta * u3;
        o.V5(o.q, 5, k) = -two_times_beta;
    }
}

inline double weight_of(const Oracle &o, double dist) {
    return 1.0 / std::pow(dist, o.P.power);
}

// Cramer numerators of the reference's 3x3 least-squares solves
// (q_derivatives.f90:85-107, *_flux_dG*.f90:114-122).
struct Moments { double xx, yy, zz, xy, yz, zx; };

inline double det_of(const Moments &m) {
    return m.xx * (m.yy * m.zz - m.yz * m.yz)
         - m.xy * (m.xy * m.zz - m.yz * m.zx)
         + m.zx * (m.xy * m.yz - m.yy * m.zx);
}
inline double num_x(const Moments &m, double fx, double fy, double fz) {
    return fx * (m.yy * m.zz - m.yz * m.yz)
         - fy * (m.xy * m.zz - m.zx * m.yz)
         + fz * (m.xy * m.yz - m.zx * m.yy);
}
inline double num_y(const Moments &m, double fx, double fy, double fz) {
    return m.xx * (fy * m.zz - m.yz * fz)
         - m.xy * (fx * m.zz - m.zx * fz)
         + m.zx * (fx * m.yz - m.zx * fy);
}
inline double num_z(const Moments &m, double fx, double fy, double fz) {
    return m.xx * (m.yy * fz - fy * m.yz)
         - m.xy * (m.xy * fz - fx * m.yz)
         + m.zx * (m.xy * fy - fx * m.yy);
}

// q_derivatives.f90:10-204
void eval_q_derivatives(Oracle &o) {
    for (int i = 1; i <= o.N; ++i) {
        double x_i = o.x[i], y_i = o.y[i], z_i = o.z[i];
        Moments m = {0, 0, 0, 0, 0, 0};
        double sx[5] = {0}, sy[5] = {0}, sz[5] = {0};
        for (int r = 1; r <= 5; ++r) { o.QM(1, r, i) = o.V5(o.q, r, i); o.QM(2, r, i) = o.V5(o.q, r, i); }
        for (int k = 1; k <= o.nbhs[i]; ++k) {
            int nbh = o.CONN(k, i);
            for (int r = 1; r <= 5; ++r) {
                if (o.V5(o.q, r, nbh) > o.QM(1, r, i)) o.QM(1, r, i) = o.V5(o.q, r, nbh);
                if (o.V5(o.q, r, nbh) < o.QM(2, r, i)) o.QM(2, r, i) = o.V5(o.q, r, nbh);
            }
            double delx = o.x[nbh] - x_i, dely = o.y[nbh] - y_i, delz = o.z[nbh] - z_i;
            double dist = std::sqrt(delx * delx + dely * dely + delz * delz);
            double weights = weight_of(o, dist);
            m.xx = m.xx + delx * delx * weights;
            m.yy = m.yy + dely * dely * weights;
            m.zz = m.zz + delz * delz * weights;
            m.xy = m.xy + delx * dely * weights;
            m.yz = m.yz + dely * delz * weights;
            m.zx = m.zx + delz * delx * weights;
            for (int r = 1; r <= 5; ++r) {
                double temp = (o.V5(o.q, r, nbh) - o.V5(o.q, r, i));
                sx[r - 1] = sx[r - 1] + weights * delx * temp;
                sy[r - 1] = sy[r - 1] + weights * dely * temp;
                sz[r - 1] = sz[r - 1] + weights * delz * temp;
            }
        }
        double det = det_of(m);
        double one_by_det = 1.0 / det;
        for (int r = 1; r <= 5; ++r) {
            o.DQ(1, r, i) = num_x(m, sx[r - 1], sy[r - 1], sz[r - 1]) * one_by_det;
            o.DQ(2, r, i) = num_y(m, sx[r - 1], sy[r - 1], sz[r - 1]) * one_by_det;
            o.DQ(3, r, i) = num_z(m, sx[r - 1], sy[r - 1], sz[r - 1]) * one_by_det;
        }
    }
    // inner iterations, q_derivatives.f90:116-201
    for (int j = 1; j <= o.P.inner_iterations; ++j) {
        for (int i = 1; i <= o.N; ++i) {
            double x_i = o.x[i], y_i = o.y[i], z_i = o.z[i];
            Moments m = {0, 0, 0, 0, 0, 0};
            double sx[5] = {0}, sy[5] = {0}, sz[5] = {0};
            for (int k = 1; k <= o.nbhs[i]; ++k) {
                int nbh = o.CONN(k, i);
                double delx = o.x[nbh] - x_i, dely = o.y[nbh] - y_i, delz = o.z[nbh] - z_i;
                double dist = std::sqrt(delx * delx + dely * dely + delz * delz);
                double weights = weight_of(o, dist);
                m.xx = m.xx + delx * delx * weights;
                m.yy = m.yy + dely * dely * weights;
                m.zz = m.zz + delz * delz * weights;
                m.xy = m.xy + delx * dely * weights;
                m.yz = m.yz + dely * delz * weights;
                m.zx = m.zx + delz * delx * weights;
                for (int r = 1; r <= 5; ++r) {
                    double qti = o.V5(o.q, r, i) - 0.5 * (delx * o.DQ(1, r, i) + dely * o.DQ(2, r, i) + delz * o.DQ(3, r, i));
                    double qtn = o.V5(o.q, r, nbh) - 0.5 * (delx * o.DQ(1, r, nbh) + dely * o.DQ(2, r, nbh) + delz * o.DQ(3, r, nbh));
                    double temp = qtn - qti;
                    sx[r - 1] = sx[r - 1] + weights * delx * temp;
                    sy[r - 1] = sy[r - 1] + weights * dely * temp;
                    sz[r - 1] = sz[r - 1] + weights * delz * temp;
                }
            }
            double det = det_of(m);
            double one_by_det = 1.0 / det;
            for (int r = 1; r <= 5; ++r) {
                o.TDQ(1, r, i) = num_x(m, sx[r - 1], sy[r - 1], sz[r - 1]) * one_by_det;
                o.TDQ(2, r, i) = num_y(m, sx[r - 1], sy[r - 1], sz[r - 1]) * one_by_det;
                o.TDQ(3, r, i) = num_z(m, sx[r - 1], sy[r - 1], sz[r - 1]) * one_by_det;
            }
        }
        for (int i = 1; i <= o.N; ++i)
            for (int c = 0; c < 15; ++c) o.dq[(size_t)i * 15 + c] = o.temp_dq[(size_t)i * 15 + c];
    }
}

// timestep_delt.f90:8-54
void timestep_delt(Oracle &o) {
    for (int i = 1; i <= o.N; ++i) {
        double min_delt = 1.0;
        for (int r = 1; r <= o.nbhs[i]; ++r) {
            int k = o.CONN(r, i);
            double rho = o.V5(o.prim, 1, k), u1 = o.V5(o.prim, 2, k), u2 = o.V5(o.prim, 3, k);
            double u3 = o.V5(o.prim, 4, k), pr = o.V5(o.prim, 5, k);
            double delx = o.x[k] - o.x[i], dely = o.y[k] - o.y[i], delz = o.z[k] - o.z[i];
            double dist = std::sqrt(delx * delx + dely * dely + delz * delz);
            double mod_u = std::sqrt(u1 * u1 + u2 * u2 + u3 * u3);
            double delt = o.P.cfl * dist / (mod_u + 3.0 * std::sqrt(pr / rho));
            if (delt < min_delt) min_delt = delt;
        }
        o.delt[i] = min_delt;
    }
}

// A list of one direction of one point: count and entry accessor.
struct ListRef {
    std::vector<int> *arr;   // null: the full conn
    int count;
};

inline int list_entry(Oracle &o, const ListRef &L, int j, int i) {
    return L.arr ? o.SL(*L.arr, j, i) : o.CONN(j, i);
}

enum Axis { AX_X = 0, AX_Y = 1, AX_Z = 2 };

// One direction of the flux residual: interior/wall/outer_flux_dG*.f90:20-126.
void dG(Oracle &o, double G[5], int i, const ListRef &L, int kind, int axis, bool by_reciprocal) {
    Moments m = {0, 0, 0, 0, 0, 0};
    double sx[5] = {0}, sy[5] = {0}, sz[5] = {0};
    double x_i = o.x[i], y_i = o.y[i], z_i = o.z[i];
    double tan1[3] = {o.TAN1(1, i), o.TAN1(2, i), o.TAN1(3, i)};
    double tan2[3] = {o.TAN2(1, i), o.TAN2(2, i), o.TAN2(3, i)};
    double nor[3] = {o.NOR(1, i), o.NOR(2, i), o.NOR(3, i)};
    for (int j = 1; j <= L.count; ++j) {
        int k = list_entry(o, L, j, i);
        double delx = o.x[k] - x_i, dely = o.y[k] - y_i, delz = o.z[k] - z_i;
        double dels = delx * tan1[0] + dely * tan1[1] + delz * tan1[2];
        double delt = delx * tan2[0] + dely * tan2[1] + delz * tan2[2];
        double deln = delx * nor[0] + dely * nor[1] + delz * nor[2];
        double dist = std::sqrt(dels * dels + delt * delt + deln * deln);
        double weights = weight_of(o, dist);
        double dels_w = dels * weights, delt_w = delt * weights, deln_w = deln * weights;
        m.xx = m.xx + dels * dels_w;
        m.yy = m.yy + delt * delt_w;
        m.zz = m.zz + deln * deln_w;
        m.xy = m.xy + dels * delt_w;
        m.yz = m.yz + delt * deln_w;
        m.zx = m.zx + deln * dels_w;
        double temp[5], qtilde[5], phi[5], prim[5], G_i[5], G_k[5];
        for (int r = 1; r <= 5; ++r)
            temp[r - 1] = delx * o.DQ(1, r, i) + dely * o.DQ(2, r, i) + delz * o.DQ(3, r, i);
        for (int r = 0; r < 5; ++r) qtilde[r] = o.V5(o.q, r + 1, i) - 0.5 * temp[r];
        venkat_limiter(o, qtilde, phi, i);
        for (int r = 0; r < 5; ++r) qtilde[r] = o.V5(o.q, r + 1, i) - 0.5 * phi[r] * temp[r];
        qtilde_to_primitive(qtilde, prim);
        flux(kind, G_i, tan1, tan2, nor, prim);
        for (int r = 1; r <= 5; ++r)
            temp[r - 1] = delx * o.DQ(1, r, k) + dely * o.DQ(2, r, k) + delz * o.DQ(3, r, k);
        for (int r = 0; r < 5; ++r) qtilde[r] = o.V5(o.q, r + 1, k) - 0.5 * temp[r];
        venkat_limiter(o, qtilde, phi, k);
        for (int r = 0; r < 5; ++r) qtilde[r] = o.V5(o.q, r + 1, k) - 0.5 * phi[r] * temp[r];
        qtilde_to_primitive(qtilde, prim);
        flux(kind, G_k, tan1, tan2, nor, prim);
        for (int r = 0; r < 5; ++r) {
            double t = G_k[r] - G_i[r];
            sx[r] = sx[r] + t * dels_w;
            sy[r] = sy[r] + t * delt_w;
            sz[r] = sz[r] + t * deln_w;
        }
    }
    double det = det_of(m);
    double one_by_det = by_reciprocal ? 1.0 / det : 0.0;
    for (int r = 0; r < 5; ++r) {
        double temp = axis == AX_X ? num_x(m, sx[r], sy[r], sz[r])
                    : axis == AX_Y ? num_y(m, sx[r], sy[r], sz[r])
                                   : num_z(m, sx[r], sy[r], sz[r]);
        G[r] = by_reciprocal ? temp * one_by_det : temp / det;
    }
}

// flux_residual.f90:30-84
void eval_flux_residual(Oracle &o) {
    double Gxp[5], Gxn[5], Gyp[5], Gyn[5], Gzp[5], Gzn[5];
    for (int k : o.wall_idx) {
        dG(o, Gxp, k, {&o.xpos_conn, o.xpos_nbhs[k]}, GWXP, AX_X, false);
        dG(o, Gxn, k, {&o.xneg_conn, o.xneg_nbhs[k]}, GWXN, AX_X, false);
        dG(o, Gyp, k, {&o.ypos_conn, o.ypos_nbhs[k]}, GWYP, AX_Y, false);
        dG(o, Gyn, k, {&o.yneg_conn, o.yneg_nbhs[k]}, GWYN, AX_Y, false);
        dG(o, Gzn, k, {nullptr, o.nbhs[k]}, GZN, AX_Z, false);   // wall_flux_dGzneg.f90:61-65
        for (int r = 0; r < 5; ++r)
            o.V5(o.flux_res, r + 1, k) = 2.0 * (Gxp[r] + Gxn[r] + Gyp[r] + Gyn[r] + Gzn[r]);
    }
    for (int k : o.outer_idx) {
        dG(o, Gxp, k, {&o.xpos_conn, o.xpos_nbhs[k]}, GOXP, AX_X, true);
        dG(o, Gxn, k, {&o.xneg_conn, o.xneg_nbhs[k]}, GOXN, AX_X, true);
        dG(o, Gyp, k, {&o.ypos_conn, o.ypos_nbhs[k]}, GOYP, AX_Y, true);
        dG(o, Gyn, k, {&o.yneg_conn, o.yneg_nbhs[k]}, GOYN, AX_Y, true);
        dG(o, Gzp, k, {&o.zpos_conn, o.zpos_nbhs[k]}, GZP, AX_Z, true);
        for (int r = 0; r < 5; ++r)
            o.V5(o.flux_res, r + 1, k) = (Gxp[r] + Gxn[r] + Gyp[r] + Gyn[r] + Gzp[r]);
    }
    for (int k : o.interior_idx) {
        dG(o, Gxp, k, {&o.xpos_conn, o.xpos_nbhs[k]}, GXP, AX_X, false);
        dG(o, Gxn, k, {&o.xneg_conn, o.xneg_nbhs[k]}, GXN, AX_X, false);
        dG(o, Gyp, k, {&o.ypos_conn, o.ypos_nbhs[k]}, GYP, AX_Y, false);
        dG(o, Gyn, k, {&o.yneg_conn, o.yneg_nbhs[k]}, GYN, AX_Y, false);
        dG(o, Gzp, k, {&o.zpos_conn, o.zpos_nbhs[k]}, GZP, AX_Z, false);
        dG(o, Gzn, k, {&o.zneg_conn, o.zneg_nbhs[k]}, GZN, AX_Z, false);
        for (int r = 0; r < 5; ++r)
            o.V5(o.flux_res, r + 1, k) = (Gxp[r] + Gxn[r] + Gyp[r] + Gyn[r] + Gzp[r] + Gzn[r]);
    }
}

// One direction of D_inv: implicit_D_inv_interior.f90:49-108 and the five
// blocks after it; sign +1 for the "pos" directions, -1 for "neg".
double dinv_dir(Oracle &o, int i, const ListRef &L, int axis, bool pos, double as) {
    Moments m = {0, 0, 0, 0, 0, 0};
    double sdx = 0, sdy = 0, sdz = 0;
    double x_i = o.x[i], y_i = o.y[i], z_i = o.z[i];
    for (int j = 1; j <= L.count; ++j) {
        int k = list_entry(o, L, j, i);
        double delx = o.x[k] - x_i, dely = o.y[k] - y_i, delz = o.z[k] - z_i;
        double dels = delx * o.TAN1(1, i) + dely * o.TAN1(2, i) + delz * o.TAN1(3, i);
        double delt = delx * o.TAN2(1, i) + dely * o.TAN2(2, i) + delz * o.TAN2(3, i);
        double deln = delx * o.NOR(1, i) + dely * o.NOR(2, i) + delz * o.NOR(3, i);
        double dist = std::sqrt(dels * dels + delt * delt + deln * deln);
        double weights = weight_of(o, dist);
        double dels_w = dels * weights, delt_w = delt * weights, deln_w = deln * weights;
        m.xx = m.xx + dels * dels_w;
        m.yy = m.yy + delt * delt_w;
        m.zz = m.zz + deln * deln_w;
        m.xy = m.xy + dels * delt_w;
        m.yz = m.yz + delt * deln_w;
        m.zx = m.zx + deln * dels_w;
        sdx = sdx + dels_w;
        sdy = sdy + delt_w;
        sdz = sdz + deln_w;
    }
    double det = det_of(m);
    double temp = axis == AX_X ? num_x(m, sdx, sdy, sdz)
                : axis == AX_Y ? num_y(m, sdx, sdy, sdz)
                               : num_z(m, sdx, sdy, sdz);
    double u = o.V5(o.prim, axis + 2, i);    // prim(2..4,i): global velocity
    if (pos) {
        double temp1 = u + as;
        return 0.50 * std::fabs(temp1 + std::fabs(temp1)) * temp / det;
    }
    double temp1 = u - as;
    return -(0.50 * std::fabs(temp1 - std::fabs(temp1)) * temp / det);
}

// implicit_D_inv_interior.f90:17-419, implicit_D_inv_wall.f90:16-361
double implicit_D_inv(Oracle &o, int i, bool wall) {
    double delta_t = o.delt[i];
    double as = std::sqrt(1.40 * o.V5(o.prim, 5, i) / o.V5(o.prim, 1, i));
    double dGxp = dinv_dir(o, i, {&o.xpos_conn, o.xpos_nbhs[i]}, AX_X, true, as);
    double dGxn = dinv_dir(o, i, {&o.xneg_conn, o.xneg_nbhs[i]}, AX_X, false, as);
    double dGyp = dinv_dir(o, i, {&o.ypos_conn, o.ypos_nbhs[i]}, AX_Y, true, as);
    double dGyn = dinv_dir(o, i, {&o.yneg_conn, o.yneg_nbhs[i]}, AX_Y, false, as);
    double temp;
    if (wall) {
        double dGzn = dinv_dir(o, i, {nullptr, o.nbhs[i]}, AX_Z, false, as);
        temp = (1.0 / delta_t) - 2.0 * (dGxp + dGxn + dGyp + dGyn + dGzn);
    } else {
        double dGzp = dinv_dir(o, i, {&o.zpos_conn, o.zpos_nbhs[i]}, AX_Z, true, as);
        double dGzn = dinv_dir(o, i, {&o.zneg_conn, o.zneg_nbhs[i]}, AX_Z, false, as);
        temp = (1.0 / delta_t) - (dGxp + dGxn + dGyp + dGyn + dGzp + dGzn);
    }
    return 1.0 / temp;
}

// One direction of LdelU / UdelU (implicit_LdelU_forward_sweep_interior.f90:
// 49-117 and its siblings): neighbours with alias below (forward) or above
// (backward) the point contribute G(prim of U_k + dU_k) - G(prim_k).
void sweep_dir(Oracle &o, double dG5[5], int i, const ListRef &L, int kind, int axis, bool forward) {
    Moments m = {0, 0, 0, 0, 0, 0};
    double sx[5] = {0}, sy[5] = {0}, sz[5] = {0};
    double x_i = o.x[i], y_i = o.y[i], z_i = o.z[i];
    double tan1[3] = {o.TAN1(1, i), o.TAN1(2, i), o.TAN1(3, i)};
    double tan2[3] = {o.TAN2(1, i), o.TAN2(2, i), o.TAN2(3, i)};
    double nor[3] = {o.NOR(1, i), o.NOR(2, i), o.NOR(3, i)};
    for (int j = 1; j <= L.count; ++j) {
        int k = list_entry(o, L, j, i);
        double delx = o.x[k] - x_i, dely = o.y[k] - y_i, delz = o.z[k] - z_i;
        double dels = delx * tan1[0] + dely * tan1[1] + delz * tan1[2];
        double delt = delx * tan2[0] + dely * tan2[1] + delz * tan2[2];
        double deln = delx * nor[0] + dely * nor[1] + delz * nor[2];
        double dist = std::sqrt(dels * dels + delt * delt + deln * deln);
        double weights = weight_of(o, dist);
        double dels_w = dels * weights, delt_w = delt * weights, deln_w = deln * weights;
        m.xx = m.xx + dels * dels_w;
        m.yy = m.yy + delt * delt_w;
        m.zz = m.zz + deln * deln_w;
        m.xy = m.xy + dels * delt_w;
        m.yz = m.yz + delt * deln_w;
        m.zx = m.zx + deln * dels_w;
        int alias_of_i = o.alias[i], alias_of_k = o.alias[k];
        bool take = forward ? (alias_of_k < alias_of_i) : (alias_of_k > alias_of_i);
        if (take) {
            double prim[5], Gold[5], Gnew[5], U[5];
            for (int r = 0; r < 5; ++r) prim[r] = o.V5(o.prim, r + 1, k);
            flux(kind, Gold, tan1, tan2, nor, prim);
            std::vector<double> &d = forward ? o.delUp : o.delUn;
            for (int r = 0; r < 5; ++r) U[r] = o.V5(d, r + 1, k) + o.V5(o.U, r + 1, k);
            get_primitive_vector(o, k, U, prim);
            flux(kind, Gnew, tan1, tan2, nor, prim);
            for (int r = 0; r < 5; ++r) {
                double t = Gnew[r] - Gold[r];
                sx[r] = sx[r] + t * dels_w;
                sy[r] = sy[r] + t * delt_w;
                sz[r] = sz[r] + t * deln_w;
            }
        }
    }
    double det = det_of(m);
    for (int r = 0; r < 5; ++r) {
        double temp = axis == AX_X ? num_x(m, sx[r], sy[r], sz[r])
                    : axis == AX_Y ? num_y(m, sx[r], sy[r], sz[r])
                                   : num_z(m, sx[r], sy[r], sz[r]);
        dG5[r] = temp / det;
    }
}

// implicit_{LdelU_forward,UdelU_backward}_sweep_{interior,wall}.f90
void sweep_LU(Oracle &o, int i, bool wall, bool forward, double out[5]) {
    double a[5], b[5], c[5], d[5], e[5], f[5];
    if (wall) {
        sweep_dir(o, a, i, {&o.xpos_conn, o.xpos_nbhs[i]}, GWXP, AX_X, forward);
        sweep_dir(o, b, i, {&o.xneg_conn, o.xneg_nbhs[i]}, GWXN, AX_X, forward);
        sweep_dir(o, c, i, {&o.ypos_conn, o.ypos_nbhs[i]}, GWYP, AX_Y, forward);
        sweep_dir(o, d, i, {&o.yneg_conn, o.yneg_nbhs[i]}, GWYN, AX_Y, forward);
        sweep_dir(o, e, i, {nullptr, o.nbhs[i]}, GZN, AX_Z, forward);
        for (int r = 0; r < 5; ++r) out[r] = 2.0 * (a[r] + b[r] + c[r] + d[r] + e[r]);
    } else {
        sweep_dir(o, a, i, {&o.xpos_conn, o.xpos_nbhs[i]}, GXP, AX_X, forward);
        sweep_dir(o, b, i, {&o.xneg_conn, o.xneg_nbhs[i]}, GXN, AX_X, forward);
        sweep_dir(o, c, i, {&o.ypos_conn, o.ypos_nbhs[i]}, GYP, AX_Y, forward);
        sweep_dir(o, d, i, {&o.yneg_conn, o.yneg_nbhs[i]}, GYN, AX_Y, forward);
        sweep_dir(o, e, i, {&o.zpos_conn, o.zpos_nbhs[i]}, GZP, AX_Z, forward);
        sweep_dir(o, f, i, {&o.zneg_conn, o.zneg_nbhs[i]}, GZN, AX_Z, forward);
        for (int r = 0; r < 5; ++r) out[r] = a[r] + b[r] + c[r] + d[r] + e[r] + f[r];
    }
}

int nearest_neighbour(Oracle &o, int p, bool skip_wall, double start) {
    double min_dist = start;
    int q = 0;
    for (int r = 1; r <= o.nbhs[p]; ++r) {
        int nbh = o.CONN(r, p);
        double dx = o.x[nbh] - o.x[p], dy = o.y[nbh] - o.y[p], dz = o.z[nbh] - o.z[p];
        double ds = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (ds < min_dist && (!skip_wall || o.status[nbh] != 1)) { min_dist = ds; q = nbh; }
    }
    return q;
}

// implicit_D_inv_outer.f90:17-363.  Every direction's loop assigns the
// neighbour's tangential offset to the variable that held the time step, so
// the 1/delt term uses the last conn neighbour's offset (or the time step
// when the point has no neighbours); the x-/y- terms carry no minus sign and
// the sum keeps the source's order.
double implicit_D_inv_outer(Oracle &o, int i) {
    double delt = o.delt[i];
    double as = std::sqrt(1.40 * o.V5(o.prim, 5, i) / o.V5(o.prim, 1, i));
    double dGxp = dinv_dir(o, i, {&o.xpos_conn, o.xpos_nbhs[i]}, AX_X, true, as);
    double dGxn = -dinv_dir(o, i, {&o.xneg_conn, o.xneg_nbhs[i]}, AX_X, false, as);
    double dGyp = dinv_dir(o, i, {&o.ypos_conn, o.ypos_nbhs[i]}, AX_Y, true, as);
    double dGyn = -dinv_dir(o, i, {&o.yneg_conn, o.yneg_nbhs[i]}, AX_Y, false, as);
    double dGzp = dinv_dir(o, i, {nullptr, o.nbhs[i]}, AX_Z, true, as);
    const ListRef lists[5] = {{&o.xpos_conn, o.xpos_nbhs[i]}, {&o.xneg_conn, o.xneg_nbhs[i]},
                              {&o.ypos_conn, o.ypos_nbhs[i]}, {&o.yneg_conn, o.yneg_nbhs[i]},
                              {nullptr, o.nbhs[i]}};
    for (const ListRef &L : lists) {
        if (L.count < 1) continue;
        int k = list_entry(o, L, L.count, i);
        double delx = o.x[k] - o.x[i], dely = o.y[k] - o.y[i], delz = o.z[k] - o.z[i];
        delt = delx * o.TAN2(1, i) + dely * o.TAN2(2, i) + delz * o.TAN2(3, i);
    }
    double temp = (1.0 / delt) - dGxp + dGxn - dGyp + dGyn - dGzp;
    return 1.0 / temp;
}

// implicit_{LdelU_forward,UdelU_backward}_sweep_outer.f90: octant fluxes on
// the x/y lists, the z+ split flux over the full conn.
void sweep_LU_outer(Oracle &o, int i, bool forward, double out[5]) {
    double a[5], b[5], c[5], d[5], e[5];
    sweep_dir(o, a, i, {&o.xpos_conn, o.xpos_nbhs[i]}, GOXP, AX_X, forward);
    sweep_dir(o, b, i, {&o.xneg_conn, o.xneg_nbhs[i]}, GOXN, AX_X, forward);
    sweep_dir(o, c, i, {&o.ypos_conn, o.ypos_nbhs[i]}, GOYP, AX_Y, forward);
    sweep_dir(o, d, i, {&o.yneg_conn, o.yneg_nbhs[i]}, GOYN, AX_Y, forward);
    sweep_dir(o, e, i, {nullptr, o.nbhs[i]}, GZP, AX_Z, forward);
    for (int r = 0; r < 5; ++r) out[r] = a[r] + b[r] + c[r] + d[r] + e[r];
}

// implicit_forward_and_reverse_sweeps_backup.f90:16-141: the point classes
// in turn, each in index order (reversed backward), outer points included;
// supersonic points copy their nearest non-wall neighbour.
void sweeps_backup(Oracle &o) {
    double LU[5];
    for (int k : o.wall_idx) {
        double D = implicit_D_inv(o, k, true);
        o.dinv[k] = D;
        sweep_LU(o, k, true, true, LU);
        for (int r = 0; r < 5; ++r) o.V5(o.delUp, r + 1, k) = -(D * (o.V5(o.flux_res, r + 1, k) + LU[r]));
    }
    for (int k : o.interior_idx) {
        double D = implicit_D_inv(o, k, false);
        o.dinv[k] = D;
        sweep_LU(o, k, false, true, LU);
        for (int r = 0; r < 5; ++r) o.V5(o.delUp, r + 1, k) = -(D * (o.V5(o.flux_res, r + 1, k) + LU[r]));
    }
    for (int k : o.outer_idx) {
        double D = implicit_D_inv_outer(o, k);
        o.dinv[k] = D;
        sweep_LU_outer(o, k, true, LU);
        for (int r = 0; r < 5; ++r) o.V5(o.delUp, r + 1, k) = -(D * (o.V5(o.flux_res, r + 1, k) + LU[r]));
    }
    for (int k : o.ss_inlet_idx) {
        int p = nearest_neighbour(o, k, true, 100000.0);
        for (int r = 1; r <= 5; ++r) o.V5(o.delUp, r, k) = o.V5(o.delUp, r, p);
    }
    for (int k : o.ss_outlet_idx) {
        int p = nearest_neighbour(o, k, true, 100000.0);
        for (int r = 1; r <= 5; ++r) o.V5(o.delUp, r, k) = o.V5(o.delUp, r, p);
    }
    for (auto it = o.wall_idx.rbegin(); it != o.wall_idx.rend(); ++it) {
        int k = *it;
        double D = implicit_D_inv(o, k, true);
        sweep_LU(o, k, true, false, LU);
        for (int r = 0; r < 5; ++r) o.V5(o.delUn, r + 1, k) = o.V5(o.delUp, r + 1, k) - D * LU[r];
    }
    for (auto it = o.interior_idx.rbegin(); it != o.interior_idx.rend(); ++it) {
        int k = *it;
        double D = implicit_D_inv(o, k, false);
        sweep_LU(o, k, false, false, LU);
        for (int r = 0; r < 5; ++r) o.V5(o.delUn, r + 1, k) = o.V5(o.delUp, r + 1, k) - D * LU[r];
    }
    for (auto it = o.outer_idx.rbegin(); it != o.outer_idx.rend(); ++it) {
        int k = *it;
        double D = implicit_D_inv_outer(o, k);
        sweep_LU_outer(o, k, false, LU);
        for (int r = 0; r < 5; ++r) o.V5(o.delUn, r + 1, k) = o.V5(o.delUp, r + 1, k) - D * LU[r];
    }
    for (auto it = o.ss_inlet_idx.rbegin(); it != o.ss_inlet_idx.rend(); ++it) {
        int k = *it, p = nearest_neighbour(o, k, true, 100000.0);
        for (int r = 1; r <= 5; ++r) o.V5(o.delUn, r, k) = o.V5(o.delUn, r, p);
    }
    for (auto it = o.ss_outlet_idx.rbegin(); it != o.ss_outlet_idx.rend(); ++it) {
        int k = *it, p = nearest_neighbour(o, k, true, 100000.0);
        for (int r = 1; r <= 5; ++r) o.V5(o.delUn, r, k) = o.V5(o.delUn, r, p);
    }
}

// implicit_forward_and_reverse_sweeps.f90:16-89
void implicit_forward_backward_sweeps(Oracle &o) {
    double LdelU[5];
    for (int i = 1; i <= o.N; ++i) {
        int p = o.point_with_alias[i];
        if (p == 0) continue;   // out of the reference's range; touches no point
        int st = o.status[p];
        if (st == 1 || st == 0) {
            ORACLE_PHASE(3);
            double D_inv = implicit_D_inv(o, p, st == 1);
            o.dinv[p] = D_inv;
            ORACLE_PHASE(4);
            sweep_LU(o, p, st == 1, true, LdelU);
            for (int r = 0; r < 5; ++r)
                o.V5(o.delUp, r + 1, p) = -(D_inv * (o.V5(o.flux_res, r + 1, p) + LdelU[r]));
        } else if (st == 5 || st == 6) {
            int q = nearest_neighbour(o, p, false, 1000000.0);
            for (int r = 1; r <= 5; ++r) o.V5(o.delUp, r, p) = o.V5(o.delUp, r, q);
        }
    }
    o.delUp_fwd = o.delUp;
    for (int i = o.N; i >= 1; --i) {
        int p = o.point_with_alias[i];
        if (p == 0) continue;
        int st = o.status[p];
        if (st == 1 || st == 0) {
            ORACLE_PHASE(7);    // the same D_inv again (implicit_forward_and_reverse_sweeps.f90:63)
            double D_inv = implicit_D_inv(o, p, st == 1);
            ORACLE_PHASE(5);
            sweep_LU(o, p, st == 1, false, LdelU);
            for (int r = 0; r < 5; ++r)
                o.V5(o.delUn, r + 1, p) = o.V5(o.delUp, r + 1, p) - D_inv * LdelU[r];
        } else if (st == 5 || st == 6) {
            int q = nearest_neighbour(o, p, false, 1000000.0);
            for (int r = 1; r <= 5; ++r) o.V5(o.delUn, r, p) = o.V5(o.delUn, r, q);
        }
    }
    for (int i = 1; i <= o.N; ++i)
        for (int r = 1; r <= 5; ++r) o.V5(o.delUp, r, i) = o.V5(o.delUn, r, i);
}

// state_update_implicit.f90:14-102
void state_update(Oracle &o) {
    double sum_res_sqr = 0.0;
    o.max_res = 0.0;
    double U[5];
    for (int k : o.wall_idx) {
        double temp = o.V5(o.U, 1, k);
        for (int r = 0; r < 5; ++r) U[r] = o.V5(o.U, r + 1, k) + o.V5(o.delUn, r + 1, k);
        double res_sqr = (U[0] - temp) * (U[0] - temp);
        if (res_sqr > o.max_res) { o.max_res = res_sqr; o.max_res_point = k; }
        sum_res_sqr = sum_res_sqr + res_sqr;
        conserved_to_primitive(o, k, U);
    }
    for (int k : o.outer_idx) {
        conserved_vector_Ubar(o, k, U);
        for (int r = 0; r < 5; ++r) U[r] = U[r] + o.V5(o.delUn, r + 1, k);
        conserved_to_primitive(o, k, U);
    }
    for (int k : o.interior_idx) {
        double temp = o.V5(o.U, 1, k);
        for (int r = 0; r < 5; ++r) U[r] = o.V5(o.U, r + 1, k) + o.V5(o.delUn, r + 1, k);
        double res_sqr = (U[0] - temp) * (U[0] - temp);
        if (res_sqr > o.max_res) { o.max_res = res_sqr; o.max_res_point = k; }
        sum_res_sqr = sum_res_sqr + res_sqr;
        conserved_to_primitive(o, k, U);
    }
    for (int k : o.ss_outlet_idx) {
        int p = nearest_neighbour(o, k, true, 100000.0);
        for (int r = 1; r <= 5; ++r) o.V5(o.prim, r, k) = o.V5(o.prim, r, p);
    }
    for (int k : o.ss_inlet_idx) {
        int p = nearest_neighbour(o, k, true, 100000.0);
        for (int r = 1; r <= 5; ++r) o.V5(o.prim, r, k) = o.V5(o.prim, r, p);
    }
    o.res_new = std::sqrt(sum_res_sqr) / (double)o.N;
    for (int i = 1; i <= o.N; ++i)
        for (int r = 1; r <= 5; ++r) o.V5(o.delUp, r, i) = o.V5(o.delUn, r, i);
}

// state_update.f90:14-124, the reference's other state_update_mod: zero
// normal momentum at the wall, an explicit update of outer points, and
// supersonic sources that may be wall points.
void state_update_explicit(Oracle &o) {
    double sum_res_sqr = 0.0;
    o.max_res = 0.0;
    double U[5];
    for (int k : o.wall_idx) {
        double temp = o.V5(o.U, 1, k);
        for (int r = 0; r < 5; ++r) U[r] = o.V5(o.U, r + 1, k) + o.V5(o.delUn, r + 1, k);
        U[3] = 0.0;
        double res_sqr = (U[0] - temp) * (U[0] - temp);
        if (res_sqr > o.max_res) { o.max_res = res_sqr; o.max_res_point = k; }
        sum_res_sqr = sum_res_sqr + res_sqr;
        conserved_to_primitive(o, k, U);
        for (int r = 1; r <= 5; ++r) o.V5(o.delUp, r, k) = o.V5(o.delUn, r, k);
    }
    for (int k : o.outer_idx) {
        conserved_vector_Ubar(o, k, U);
        for (int r = 0; r < 5; ++r) U[r] = U[r] - o.delt[k] * o.V5(o.flux_res, r + 1, k);
        conserved_to_primitive(o, k, U);
    }
    for (int k : o.interior_idx) {
        double temp = o.V5(o.U, 1, k);
        for (int r = 0; r < 5; ++r) U[r] = o.V5(o.U, r + 1, k) + o.V5(o.delUn, r + 1, k);
        double res_sqr = (U[0] - temp) * (U[0] - temp);
        if (res_sqr > o.max_res) { o.max_res = res_sqr; o.max_res_point = k; }
        sum_res_sqr = sum_res_sqr + res_sqr;
        conserved_to_primitive(o, k, U);
        for (int r = 1; r <= 5; ++r) o.V5(o.delUp, r, k) = o.V5(o.delUn, r, k);
    }
    for (int k : o.ss_outlet_idx) {
        int p = nearest_neighbour(o, k, false, 100000.0);
        for (int r = 1; r <= 5; ++r) o.V5(o.prim, r, k) = o.V5(o.prim, r, p);
    }
    for (int k : o.ss_inlet_idx) {
        int p = nearest_neighbour(o, k, false, 100000.0);
        for (int r = 1; r <= 5; ++r) o.V5(o.prim, r, k) = o.V5(o.prim, r, p);
    }
    o.res_new = std::sqrt(sum_res_sqr) / (double)o.N;
}

// fpi_solver.f90:20-45
void fpi_solver(Oracle &o, int t) {
    ORACLE_PHASE(0);
    compute_conserved_vector(o);
    eval_q_variables(o);
    ORACLE_PHASE(1);
    eval_q_derivatives(o);
    timestep_delt(o);
    ORACLE_PHASE(2);
    eval_flux_residual(o);
    ORACLE_PHASE(4);
    if (o.P.sweep_variant) sweeps_backup(o);
    else implicit_forward_backward_sweeps(o);
    ORACLE_PHASE(6);
    if (o.P.update_variant) state_update_explicit(o);
    else state_update(o);
    ORACLE_PHASE(7);
    if (t <= 2) {
        o.res_old = o.res_new;
        o.residue = 0.0;
    } else {
        o.residue = std::log10(o.res_new / o.res_old);
    }
}

}  // namespace

// ---------------------------------------------------------------- C API

extern "C" {

struct oracle_params_c {
    double power, vl_const, cfl;
    double rho_inf, u1_inf, u2_inf, u3_inf, pr_inf;
    int inner_iterations;
    int split_capacity;
    int update_variant;
    int sweep_variant;
};

void *oracle_create(const oracle_params_c *pp, int N, const int *status, const double *x,
                    const double *y, const double *z, const double *tan1, const double *tan2,
                    const double *nor, const int *nbhs, const int *conn, const double *min_dist) {
    Oracle *o = new Oracle();
    o->P.power = pp->power; o->P.vl_const = pp->vl_const; o->P.cfl = pp->cfl;
    o->P.rho_inf = pp->rho_inf; o->P.u1_inf = pp->u1_inf; o->P.u2_inf = pp->u2_inf;
    o->P.u3_inf = pp->u3_inf; o->P.pr_inf = pp->pr_inf;
    o->P.inner_iterations = pp->inner_iterations;
    o->P.split_capacity = pp->split_capacity;
    o->P.update_variant = pp->update_variant;
    o->P.sweep_variant = pp->sweep_variant;
    o->N = N;
    o->cap = pp->split_capacity;
    size_t n1 = (size_t)N + 1;
    o->x.assign(n1, 0.0); o->y.assign(n1, 0.0); o->z.assign(n1, 0.0);
    o->tan1.assign(n1 * 3, 0.0); o->tan2.assign(n1 * 3, 0.0); o->nor.assign(n1 * 3, 0.0);
    o->min_dist.assign(n1, 0.0);
    o->status.assign(n1, 0); o->nbhs.assign(n1, 0); o->conn.assign(n1 * 27, 0);
    for (int k = 1; k <= N; ++k) {
        o->x[k] = x[k - 1]; o->y[k] = y[k - 1]; o->z[k] = z[k - 1];
        for (int r = 0; r < 3; ++r) {
            o->tan1[(size_t)k * 3 + r] = tan1[(size_t)(k - 1) * 3 + r];
            o->tan2[(size_t)k * 3 + r] = tan2[(size_t)(k - 1) * 3 + r];
            o->nor[(size_t)k * 3 + r] = nor[(size_t)(k - 1) * 3 + r];
        }
        o->min_dist[k] = min_dist[k - 1];
        o->status[k] = status[k - 1];
        o->nbhs[k] = nbhs[k - 1];
        for (int r = 0; r < 27; ++r) o->conn[(size_t)k * 27 + r] = conn[(size_t)(k - 1) * 27 + r];
    }
    o->xpos_nbhs.assign(n1, 0); o->xneg_nbhs.assign(n1, 0); o->ypos_nbhs.assign(n1, 0);
    o->yneg_nbhs.assign(n1, 0); o->zpos_nbhs.assign(n1, 0); o->zneg_nbhs.assign(n1, 0);
    size_t lsz = (size_t)N * o->cap + 64;   // tail pad past the last column
    o->xpos_conn.assign(lsz, 0); o->xneg_conn.assign(lsz, 0); o->ypos_conn.assign(lsz, 0);
    o->yneg_conn.assign(lsz, 0); o->zpos_conn.assign(lsz, 0); o->zneg_conn.assign(lsz, 0);
    o->U.assign(n1 * 5, 0.0); o->delUp.assign(n1 * 5, 0.0); o->delUn.assign(n1 * 5, 0.0);
    o->prim.assign(n1 * 5, 0.0); o->flux_res.assign(n1 * 5, 0.0); o->q.assign(n1 * 5, 0.0);
    o->qm.assign(n1 * 10, 0.0); o->dq.assign(n1 * 15, 0.0); o->temp_dq.assign(n1 * 15, 0.0);
    o->delt.assign(n1, 0.0); o->dinv.assign(n1, 0.0);
    o->alias.assign(n1, 0); o->point_with_alias.assign(n1, 0);
    build_index_lists(*o);
    generate_split_stencils(*o);   // q_lskum.f90:25
    aliasing(*o);                  // q_lskum.f90:26
    return o;
}

void oracle_set_libm(int mode) { g_libm = mode; }

// initial_conditions.f90:18-29: prim given, delUp = delUn = 0
void oracle_set_prim(void *h, const double *prim) {
    Oracle *o = (Oracle *)h;
    for (int k = 1; k <= o->N; ++k)
        for (int r = 0; r < 5; ++r) {
            o->prim[(size_t)k * 5 + r] = prim[(size_t)(k - 1) * 5 + r];
            o->delUp[(size_t)k * 5 + r] = 0.0;
            o->delUn[(size_t)k * 5 + r] = 0.0;
        }
    o->res_old = o->res_new = o->residue = 0.0;
}

void oracle_fpi_step(void *h, int t, double *res_new, double *residue) {
    Oracle *o = (Oracle *)h;
    fpi_solver(*o, t);
    if (res_new) *res_new = o->res_new;
    if (residue) *residue = o->residue;
}

// Field ids match mfcfd.h: 0 PRIM(5,N) 1 U(5,N) 2 Q(5,N) 3 QM(2,5,N) 4 DQ(3,5,N)
// 5 DELT(N) 6 FLUX_RES(5,N) 7 DELUP(5,N) 8 DELUN(5,N) 9 D_INV(N)
int oracle_get(void *h, int field, double *out) {
    Oracle *o = (Oracle *)h;
    int N = o->N;
    auto copyv = [&](std::vector<double> &a, int w) {
        std::memcpy(out, a.data() + w, sizeof(double) * (size_t)N * w);
    };
    switch (field) {
    case 0: copyv(o->prim, 5); return 0;
    case 1: copyv(o->U, 5); return 0;
    case 2: copyv(o->q, 5); return 0;
    case 3: copyv(o->qm, 10); return 0;
    case 4: copyv(o->dq, 15); return 0;
    case 5: copyv(o->delt, 1); return 0;
    case 6: copyv(o->flux_res, 5); return 0;
    case 7: copyv(o->delUp, 5); return 0;
    case 8: copyv(o->delUn, 5); return 0;
    case 9: copyv(o->dinv, 1); return 0;
    case 10: if (o->delUp_fwd.empty()) return -1; copyv(o->delUp_fwd, 5); return 0;
    default: return -1;
    }
}

// The six split lists as the flux routines read them: counts (6,N) and the
// first `width` entries of each list (width, 6, N), 1-based; list order
// xpos, xneg, ypos, yneg, zpos, zneg.  Reads past the capacity follow the
// flat column-major storage like the Fortran does.
void oracle_get_stencils(void *h, int *counts, int *lists, int width) {
    Oracle *o = (Oracle *)h;
    std::vector<int> *arr[6] = {&o->xpos_conn, &o->xneg_conn, &o->ypos_conn,
                                &o->yneg_conn, &o->zpos_conn, &o->zneg_conn};
    std::vector<int> *cnt[6] = {&o->xpos_nbhs, &o->xneg_nbhs, &o->ypos_nbhs,
                                &o->yneg_nbhs, &o->zpos_nbhs, &o->zneg_nbhs};
    for (int k = 1; k <= o->N; ++k)
        for (int d = 0; d < 6; ++d) {
            int c = (*cnt[d])[k];
            counts[(size_t)(k - 1) * 6 + d] = c;
            for (int j = 1; j <= width; ++j)
                lists[((size_t)(k - 1) * 6 + d) * width + (j - 1)] =
                    (j <= c) ? o->SL(*arr[d], j, k) : 0;
        }
}

void oracle_get_alias(void *h, int *alias, int *point_with_alias) {
    Oracle *o = (Oracle *)h;
    for (int k = 1; k <= o->N; ++k) {
        alias[k - 1] = o->alias[k];
        point_with_alias[k - 1] = o->point_with_alias[k];
    }
}

void oracle_destroy(void *h) { delete (Oracle *)h; }

// Evaluate one libm function over an array: fn 0 exp, 1 log, 2 erf;
// mode 0 glibc, 1 mfmath.  For the accuracy tests of mfmath.h.
void oracle_libm_eval(int fn, int mode, const double *x, double *y, int n) {
    for (int i = 0; i < n; ++i) {
        double v = x[i];
        if (fn == 0) y[i] = mode ? mf_exp(v) : std::exp(v);
        else if (fn == 1) y[i] = mode ? mf_log(v) : std::log(v);
        else y[i] = mode ? mf_erf(v) : std::erf(v);
    }
}

}  // extern "C"
