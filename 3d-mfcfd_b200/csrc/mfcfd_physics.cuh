/*
 * mfcfd_physics.cuh - pointwise q-LSKUM physics as device functions.
 *
 * Every expression keeps the reference's operand order (Fortran evaluates
 * a*b*c as (a*b)*c and a+b+c as (a+b)+c) and the translation unit is built
 * with -fmad=false, so each multiply and add rounds separately as it does in
 * the reference's x86-64 build.  exp/log/erf come from mfmath.h.
 *
 * The flux-side functions are templates over the compute type R.  R = double
 * is the bit-matched path; R = float is the mixed-precision path's flux,
 * limiter and sweep arithmetic (CUDA's single-precision expf/logf/erff).
 * Every constant is written R(c), so the double instantiation performs the
 * same operations in the same order as a plain double expression.
 */
#pragma once

#include "mfmath.h"

namespace mfcfd {

#define MF_PI 3.141592653589793            /* 4*datan(1d0), parameter.f90:19 */
#define MF_LIM_EPS 9.99999974737875163555e-06  /* REAL*4 literal 10e-6, limiters.f90:242 */

// Elementary functions per compute type.
__device__ __forceinline__ double r_exp(double x) { return mf_exp(x); }
__device__ __forceinline__ float r_exp(float x) { return expf(x); }
__device__ __forceinline__ double r_log(double x) { return mf_log(x); }
__device__ __forceinline__ float r_log(float x) { return logf(x); }
__device__ __forceinline__ double r_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float r_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double r_abs(double x) { return fabs(x); }
__device__ __forceinline__ float r_abs(float x) { return fabsf(x); }

template <typename R>
struct FrameT { R t1[3], t2[3], n[3]; };
using Frame = FrameT<double>;

template <typename R>
__device__ __forceinline__ void load_frame(const double *f, FrameT<R> &F) {
#pragma unroll
    for (int r = 0; r < 3; ++r) { F.t1[r] = (R)f[r]; F.t2[r] = (R)f[3 + r]; F.n[r] = (R)f[6 + r]; }
}

// Flux kinds: split fluxes (split_fluxes.f90) and octant fluxes (octant_fluxes.f90).
enum FluxKind { GXP = 0, GXN, GYP, GYN, GZP, GZN, GWXP, GWXN, GWYP, GWYN, GOXP, GOXN, GOYP, GOYN, GNONE };

// Flux routine of list d (0 xpos .. 5 zneg) for a point class
// (flux_residual.f90:44-77, implicit_LdelU_forward_sweep_{interior,wall}.f90).
__host__ __device__ __forceinline__ int flux_kind(int cls, int d) {
    if (cls == 0) return d;                                   // interior: Gxp..Gzn
    if (cls == 1) return d < 4 ? GWXP + d : (d == 5 ? GZN : GNONE);  // wall
    if (cls == 2) return d < 4 ? GOXP + d : (d == 4 ? GZP : GNONE);  // outer
    return GNONE;
}

// Runtime choice among three register values.  Used instead of indexing a
// small array with a runtime index, which would place it in local memory.
template <typename R>
__device__ __forceinline__ R sel3(int a, R v0, R v1, R v2) {
    return a == 0 ? v0 : (a == 1 ? v1 : v2);
}

// Quantities every flux formula shares (split_fluxes.f90:24-40).
template <typename R>
struct FluxPreT {
    R rho, pr, ut1, ut2, un, beta, sb, spb, usq;
    __device__ __forceinline__ R ut(int a) const { return sel3(a, ut1, ut2, un); }
};
using FluxPre = FluxPreT<double>;

template <typename R>
__device__ __forceinline__ void flux_pre(const R prim[5], const FrameT<R> &F, FluxPreT<R> &P) {
    const R rho = prim[0], u1 = prim[1], u2 = prim[2], u3 = prim[3], pr = prim[4];
    P.rho = rho;
    P.pr = pr;
    P.ut1 = F.t1[0] * u1 + F.t1[1] * u2 + F.t1[2] * u3;
    P.ut2 = F.t2[0] * u1 + F.t2[1] * u2 + F.t2[2] * u3;
    P.un = F.n[0] * u1 + F.n[1] * u2 + F.n[2] * u3;
    P.beta = R(0.5) * rho / pr;
    P.sb = r_sqrt(P.beta);
    P.spb = r_sqrt(R(MF_PI) * P.beta);
    P.usq = P.ut1 * P.ut1 + P.ut2 * P.ut2 + P.un * P.un;
}

// Half-range terms along one axis: B = 0.5 exp(-S^2)/sqrt(pi beta),
// A+- = 0.5 (1 +- erf S) with S = u_axis sqrt(beta).
template <typename R>
struct AxisTermsT { R B, Ap, An; };
using AxisTerms = AxisTermsT<double>;

// The |S| < 1 erf polynomial does not need exp(-S^2), so it is evaluated
// unconditionally and overlaps the exp; the result equals mf_erf(S).
__device__ __forceinline__ void axis_terms(const FluxPreT<double> &P, int a, AxisTermsT<double> &T) {
    const double S = P.ut(a) * P.sb;
    const double e = mf_exp(-(S * S));
    const double small = mf_erf_small(S);
    T.B = 0.5 * e / P.spb;
    const double er = fabs(S) < 1.0 ? small : mf_erf_large(S, e);
    T.Ap = 0.5 * (1.0 + er);
    T.An = 0.5 * (1.0 - er);
}

__device__ __forceinline__ void axis_terms(const FluxPreT<float> &P, int a, AxisTermsT<float> &T) {
    const float S = P.ut(a) * P.sb;
    const float e = expf(-(S * S));
    const float er = erff(S);
    T.B = 0.5f * e / P.spb;
    T.Ap = 0.5f * (1.0f + er);
    T.An = 0.5f * (1.0f - er);
}

// Which axes a flux kind needs (bit a).
__host__ __device__ __forceinline__ int kind_axes(int kind) {
    switch (kind) {
    case GXP: case GXN: return 1;
    case GYP: case GYN: return 2;
    case GZP: case GZN: return 4;
    case GWXP: case GWXN: case GOXP: case GOXN: return 1 | 4;
    case GWYP: case GWYN: case GOYP: case GOYN: return 2 | 4;
    default: return 0;
    }
}

// One component c of flux `kind` given the shared terms and the axis terms
// of the three axes (only the axes the kind needs are read).
template <typename R>
__device__ __forceinline__ R flux_component(int kind, int c, const FluxPreT<R> &P, const AxisTermsT<R> &X,
                                            const AxisTermsT<R> &Y, const AxisTermsT<R> &Z) {
    const R rho = P.rho, pr = P.pr;
    const R ut1 = P.ut1, ut2 = P.ut2, un = P.un;
    const R half = R(0.5), two5 = R(2.5);
    if (kind <= GZN) {
        const int a = kind >> 1;
        const bool pos = (kind & 1) == 0;
        const R A = pos ? sel3(a, X.Ap, Y.Ap, Z.Ap) : sel3(a, X.An, Y.An, Z.An);
        const R B = sel3(a, X.B, Y.B, Z.B);
        const R ua = P.ut(a);
        const R temp1 = pos ? (ua * A + B) : (ua * A - B);
        if (c == 0) return rho * temp1;
        if (c == 4) {
            const R t = two5 * pr + half * rho * P.usq;
            return pos ? (t + pr) * ua * A + (t + half * pr) * B
                       : (t + pr) * ua * A - (t + half * pr) * B;
        }
        // c = 1..3: the axis component carries the pressure term
        const R uc = P.ut(c - 1);
        if (c - 1 == a) return pr * A + rho * uc * temp1;
        return rho * uc * temp1;
    }
    // octant fluxes: x variants pair S1 with S3, y variants S2 with S3
    const bool wall = kind <= GWYN;
    const int k4 = wall ? kind - GWXP : kind - GOXP;        // 0 xp, 1 xn, 2 yp, 3 yn
    const int a = k4 >> 1;
    const bool pos = (k4 & 1) == 0;
    const R A = pos ? (a == 0 ? X.Ap : Y.Ap) : (a == 0 ? X.An : Y.An);
    const R B = a == 0 ? X.B : Y.B;
    const R A3 = wall ? Z.An : Z.Ap;
    const R B3 = Z.B;
    const R ua = a == 0 ? ut1 : ut2;
    const R temp1 = pos ? (ua * A + B) : (ua * A - B);
    switch (c) {
    case 0: return rho * temp1 * A3;
    case 1: return a == 0 ? (pr * A + rho * ut1 * temp1) * A3 : rho * ut1 * temp1 * A3;
    case 2: return a == 1 ? (pr * A + rho * ut2 * temp1) * A3 : rho * ut2 * temp1 * A3;
    case 3: return wall ? rho * temp1 * (un * A3 - B3) : rho * temp1 * (un * A3 + B3);
    default: {
        const R temp2 = two5 * pr + half * rho * P.usq;
        const R temp3 = pos ? (temp2 + pr) * ua * A + (temp2 + half * pr) * B
                            : (temp2 + pr) * ua * A - (temp2 + half * pr) * B;
        return wall ? temp3 * A3 - half * rho * un * B3 * temp1
                    : temp3 * A3 + half * rho * un * B3 * temp1;
    }
    }
}

template <typename R>
__device__ __forceinline__ R flux_component(int kind, int c, const FluxPreT<R> &P, const AxisTermsT<R> *AT) {
    return flux_component(kind, c, P, AT[0], AT[1], AT[2]);
}

// qvariables_to_primitive_variables.f90:9-31
template <typename R>
__device__ __forceinline__ void qtilde_to_primitive(const R q[5], R prim[5]) {
    const R beta = -q[4] * R(0.5);
    const R temp = R(0.5) / beta;
    prim[1] = q[1] * temp;
    prim[2] = q[2] * temp;
    prim[3] = q[3] * temp;
    const R temp1 = q[0] + beta * (prim[1] * prim[1] + prim[2] * prim[2] + prim[3] * prim[3]);
    const R temp2 = temp1 - (r_log(beta) * R(2.5));
    prim[0] = r_exp(temp2);
    prim[4] = prim[0] * temp;
}

// get_primitive_vector.f90:10-41 and conserved_to_primitive_vector.f90:10-42
// (same arithmetic; U is rotated back from point k's frame).
template <typename R>
__device__ __forceinline__ void conserved_to_primitive(const R U[5], const FrameT<R> &F, R prim[5]) {
    prim[0] = U[0];
    R temp = R(1.0) / U[0];
    const R U2r = U[1], U3r = U[2], U4r = U[3];
    const R g1 = F.t1[0] * U2r + F.t2[0] * U3r + F.n[0] * U4r;
    const R g2 = F.t1[1] * U2r + F.t2[1] * U3r + F.n[1] * U4r;
    const R g3 = F.t1[2] * U2r + F.t2[2] * U3r + F.n[2] * U4r;
    prim[1] = temp * g1;
    prim[2] = temp * g2;
    prim[3] = temp * g3;
    temp = prim[1] * prim[1] + prim[2] * prim[2] + prim[3] * prim[3];
    prim[4] = R(0.4) * (U[4] - R(0.5) * prim[0] * temp);
}

// compute_conserved_vector.f90:20-32
__device__ __forceinline__ void primitive_to_rotated_conserved(const double p[5], const Frame &F, double U[5]) {
    U[0] = p[0];
    double temp1 = p[0] * p[1], temp2 = p[0] * p[2], temp3 = p[0] * p[3];
    U[1] = temp1 * F.t1[0] + temp2 * F.t1[1] + temp3 * F.t1[2];
    U[2] = temp1 * F.t2[0] + temp2 * F.t2[1] + temp3 * F.t2[2];
    U[3] = temp1 * F.n[0] + temp2 * F.n[1] + temp3 * F.n[2];
    temp1 = p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
    U[4] = 2.5 * p[4] + 0.5 * U[0] * temp1;
}

// q_variables.f90:19-38
__device__ __forceinline__ void primitive_to_q(const double p[5], double q[5]) {
    const double rho = p[0], u1 = p[1], u2 = p[2], u3 = p[3], pr = p[4];
    const double beta = 0.5 * rho / pr;
    q[0] = mf_log(rho) + (mf_log(beta) * 2.5) - beta * (u1 * u1 + u2 * u2 + u3 * u3);
    const double tb = 2.0 * beta;
    q[1] = tb * u1;
    q[2] = tb * u2;
    q[3] = tb * u3;
    q[4] = -tb;
}

// conserved_vector_Ubar.f90:8-64
__device__ __forceinline__ void conserved_vector_Ubar(const double p[5], const Frame &F, double rho_inf,
                                                      double u1_inf, double u2_inf, double u3_inf,
                                                      double pr_inf, double Ubar[5]) {
    const double u1ir = u1_inf * F.t1[0] + u2_inf * F.t1[1] + u3_inf * F.t1[2];
    const double u2ir = u1_inf * F.t2[0] + u2_inf * F.t2[1] + u3_inf * F.t2[2];
    const double u3ir = u1_inf * F.n[0] + u2_inf * F.n[1] + u3_inf * F.n[2];
    const double rho_e_inf = pr_inf * 2.5 + 0.5 * rho_inf * (u1ir * u1ir + u2ir * u2ir + u3ir * u3ir);
    double beta = (0.5 * rho_inf) / pr_inf;
    double S3 = u3ir * sqrt(beta);
    double e = mf_exp(-(S3 * S3));
    const double B3_inf = e / (2.0 * sqrt(MF_PI * beta));
    const double A3n_inf = 0.5 * (1.0 - mf_erf_given_exp(S3, e));
    const double rho = p[0], u1 = p[1], u2 = p[2], u3 = p[3], pr = p[4];
    const double u1r = u1 * F.t1[0] + u2 * F.t1[1] + u3 * F.t1[2];
    const double u2r = u1 * F.t2[0] + u2 * F.t2[1] + u3 * F.t2[2];
    const double u3r = u1 * F.n[0] + u2 * F.n[1] + u3 * F.n[2];
    const double rho_e = pr * 2.5 + 0.5 * rho * (u1r * u1r + u2r * u2r + u3r * u3r);
    beta = (0.5 * rho) / pr;
    S3 = u3r * sqrt(beta);
    e = mf_exp(-(S3 * S3));
    const double B3 = e / (2.0 * sqrt(MF_PI * beta));
    const double A3p = 0.5 * (1.0 + mf_erf_given_exp(S3, e));
    Ubar[0] = (rho_inf * A3n_inf) + (rho * A3p);
    Ubar[1] = (rho_inf * u1ir * A3n_inf) + (rho * u1r * A3p);
    Ubar[2] = (rho_inf * u2ir * A3n_inf) + (rho * u2r * A3p);
    double temp1 = rho_inf * (u3ir * A3n_inf - B3_inf);
    double temp2 = rho * (u3r * A3p + B3);
    Ubar[3] = temp1 + temp2;
    temp1 = (rho_e_inf * A3n_inf - 0.5 * rho_inf * u3ir * B3_inf);
    temp2 = (rho_e * A3p + 0.5 * rho * u3r * B3);
    Ubar[4] = temp1 + temp2;
}

// Cramer numerators in the reference's operand order
// (q_derivatives.f90:91-105; *_flux_dG*.f90:118-121).
__device__ __forceinline__ double cramer_num(int axis, const double *g, double fx, double fy, double fz) {
    const double xx = g[0], yy = g[1], zz = g[2], xy = g[3], yz = g[4], zx = g[5];
    if (axis == 0)
        return fx * (yy * zz - yz * yz) - fy * (xy * zz - zx * yz) + fz * (xy * yz - zx * yy);
    if (axis == 1)
        return xx * (fy * zz - yz * fz) - xy * (fx * zz - zx * fz) + zx * (fx * yz - zx * fy);
    return xx * (yy * fz - fy * yz) - xy * (xy * fz - fx * yz) + zx * (xy * fy - fx * yy);
}

}  // namespace mfcfd
