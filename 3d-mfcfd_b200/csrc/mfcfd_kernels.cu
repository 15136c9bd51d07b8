/*
 * mfcfd_kernels.cu - the FP64 q-LSKUM iteration on sm_100a.
 *
 * One iteration (fpi_solver.f90:27-36) is this launch sequence:
 *   k_qderiv      q_derivatives + timestep_delt     thread per point
 *   k_flux        eval_flux_residual                warp per point
 *   k_pending     sweep hand-off words set to "not yet published"
 *   k_dinv_gold   D_inv, fluxes of prim in the shared interior frame,
 *                 flux increments of points the sweeps do not update
 *   k_sweep_chain x2  forward / backward LU-SGS sweep: static warp chains
 *                 on all SMs (k_sweep_df: dynamic topological order;
 *                 k_sweep_levels: one CTA, level by level)
 *   k_update      state_update_implicit + next iteration's U and q
 *                 (k_update_ss: supersonic points' copies, in order)
 *   k_reduce_*    res_new (deterministic two-pass sum)
 * State stays resident in HBM in the reference's point-major layout.
 *
 * Built with -fmad=false: every multiply and add rounds separately, as in
 * the reference's build; see mfcfd_physics.cuh for the expression order.
 */
#include <cuda_runtime.h>

#include <mutex>
#include <type_traits>
#include <utility>
#include <string>

#include "mfcfd_internal.h"
#include "mfcfd_physics.cuh"

namespace mfcfd {

constexpr int FLUX_WARPS = 4;            // warps per CTA in k_flux
constexpr int FLUX_SMEM_PER_WARP = NDIR * MAX_SLOTS * 5 + MAX_SLOTS * 3;   // doubles
constexpr int SWEEP_THREADS = 512;
constexpr int SWEEP_WARPS = SWEEP_THREADS / 32;
constexpr int RED_THREADS = 256;
constexpr unsigned FULL = 0xffffffffu;

// ---------------------------------------------------------------- U and q

// compute_conserved_vector + eval_q_variables for every point.
__global__ void k_conserved_q(DevCloud d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    Frame F;
    load_frame(d.frame + 9 * (size_t)i, F);
    double p[5], U[5], q[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) p[r] = d.prim[5 * (size_t)i + r];
    primitive_to_rotated_conserved(p, F, U);
    primitive_to_q(p, q);
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        d.U[5 * (size_t)i + r] = U[r];
        d.q[5 * (size_t)i + r] = q[r];
    }
}

// ---------------------------------------------------------------- q-derivatives

// eval_q_derivatives (q_derivatives.f90:25-110) and timestep_delt
// (timestep_delt.f90:227-259), thread per point.  Weights come from d.wq
// (power != 0); with power = 0 they are exactly 1, and delx*delx*1 and
// 1*delx*temp round like the unweighted products.
__global__ void __launch_bounds__(128) k_qderiv(DevCloud d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const double xi = d.x[i], yi = d.y[i], zi = d.z[i];
    double qi[5], qmax[5], qmin[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) { qi[r] = d.q[5 * (size_t)i + r]; qmax[r] = qi[r]; qmin[r] = qi[r]; }
    double xx = 0, yy = 0, zz = 0, xy = 0, yz = 0, zx = 0;
    double sx[5] = {0, 0, 0, 0, 0}, sy[5] = {0, 0, 0, 0, 0}, sz[5] = {0, 0, 0, 0, 0};
    double min_delt = 1.0;
    const int nb = d.nbhs[i];
    const int32_t *cn = d.conn + (size_t)MAX_CONN * i;
    for (int j = 0; j < nb; ++j) {
        const int k = cn[j];
        const double w = d.wq ? d.wq[(size_t)MAX_CONN * i + j] : 1.0;
        double qk[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            qk[r] = d.q[5 * (size_t)k + r];
            if (qk[r] > qmax[r]) qmax[r] = qk[r];
            if (qk[r] < qmin[r]) qmin[r] = qk[r];
        }
        const double delx = d.x[k] - xi, dely = d.y[k] - yi, delz = d.z[k] - zi;
        const double dist = sqrt(delx * delx + dely * dely + delz * delz);
        xx = xx + delx * delx * w;
        yy = yy + dely * dely * w;
        zz = zz + delz * delz * w;
        xy = xy + delx * dely * w;
        yz = yz + dely * delz * w;
        zx = zx + delz * delx * w;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            const double t = qk[r] - qi[r];
            sx[r] = sx[r] + w * delx * t;
            sy[r] = sy[r] + w * dely * t;
            sz[r] = sz[r] + w * delz * t;
        }
        // timestep_delt.f90:235-253
        const double *pk = d.prim + 5 * (size_t)k;
        const double rho = pk[0], u1 = pk[1], u2 = pk[2], u3 = pk[3], pr = pk[4];
        const double mod_u = sqrt(u1 * u1 + u2 * u2 + u3 * u3);
        const double delt = d.cfl * dist / (mod_u + 3.0 * sqrt(pr / rho));
        if (delt < min_delt) min_delt = delt;
    }
    const double g[6] = {xx, yy, zz, xy, yz, zx};
    const double det = xx * (yy * zz - yz * yz) - xy * (xy * zz - yz * zx) + zx * (xy * yz - yy * zx);
    const double one_by_det = 1.0 / det;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        d.dq[15 * (size_t)i + 3 * r + 0] = cramer_num(0, g, sx[r], sy[r], sz[r]) * one_by_det;
        d.dq[15 * (size_t)i + 3 * r + 1] = cramer_num(1, g, sx[r], sy[r], sz[r]) * one_by_det;
        d.dq[15 * (size_t)i + 3 * r + 2] = cramer_num(2, g, sx[r], sy[r], sz[r]) * one_by_det;
        d.qm[10 * (size_t)i + 2 * r + 0] = qmax[r];
        d.qm[10 * (size_t)i + 2 * r + 1] = qmin[r];
    }
    d.delt[i] = min_delt;
}

// One inner iteration of the second-order q-derivatives
// (q_derivatives.f90:116-201): least squares over conn of the differences of
// the half-step reconstructions q - dq.del/2 at both ends, from dq_in into
// dq_out (the reference's point%temp, copied back after the pass).
__global__ void __launch_bounds__(128) k_qinner(DevCloud d, const double *dq_in, double *dq_out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const double xi = d.x[i], yi = d.y[i], zi = d.z[i];
    double qi[5], dqi[15];
#pragma unroll
    for (int r = 0; r < 5; ++r) qi[r] = d.q[5 * (size_t)i + r];
#pragma unroll
    for (int c = 0; c < 15; ++c) dqi[c] = dq_in[15 * (size_t)i + c];
    double xx = 0, yy = 0, zz = 0, xy = 0, yz = 0, zx = 0;
    double sx[5] = {0, 0, 0, 0, 0}, sy[5] = {0, 0, 0, 0, 0}, sz[5] = {0, 0, 0, 0, 0};
    const int nb = d.nbhs[i];
    const int32_t *cn = d.conn + (size_t)MAX_CONN * i;
    for (int j = 0; j < nb; ++j) {
        const int k = cn[j];
        const double delx = d.x[k] - xi, dely = d.y[k] - yi, delz = d.z[k] - zi;
        const double w = d.wq ? d.wq[(size_t)MAX_CONN * i + j] : 1.0;
        xx = xx + delx * delx * w;
        yy = yy + dely * dely * w;
        zz = zz + delz * delz * w;
        xy = xy + delx * dely * w;
        yz = yz + dely * delz * w;
        zx = zx + delz * delx * w;
        const double *dqk = dq_in + 15 * (size_t)k;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            const double qti = qi[r] - 0.5 * (delx * dqi[3 * r] + dely * dqi[3 * r + 1] + delz * dqi[3 * r + 2]);
            const double qtn = d.q[5 * (size_t)k + r] - 0.5 * (delx * dqk[3 * r] + dely * dqk[3 * r + 1] + delz * dqk[3 * r + 2]);
            const double t = qtn - qti;
            sx[r] = sx[r] + w * delx * t;
            sy[r] = sy[r] + w * dely * t;
            sz[r] = sz[r] + w * delz * t;
        }
    }
    const double g[6] = {xx, yy, zz, xy, yz, zx};
    const double det = xx * (yy * zz - yz * yz) - xy * (xy * zz - yz * zx) + zx * (xy * yz - yy * zx);
    const double one_by_det = 1.0 / det;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        dq_out[15 * (size_t)i + 3 * r + 0] = cramer_num(0, g, sx[r], sy[r], sz[r]) * one_by_det;
        dq_out[15 * (size_t)i + 3 * r + 1] = cramer_num(1, g, sx[r], sy[r], sz[r]) * one_by_det;
        dq_out[15 * (size_t)i + 3 * r + 2] = cramer_num(2, g, sx[r], sy[r], sz[r]) * one_by_det;
    }
}

// ---------------------------------------------------------------- hand-off words

// Hand-off of increments between warps.  Before the sweeps, k_dinv_gold sets
// dUp, dUn, dgf and dgb of every swept point to DU_PENDING, a signalling-NaN
// bit pattern that no arithmetic result has (arithmetic NaNs are quiet).  A
// producer stores its values with strong (relaxed, gpu-scope) 8-byte stores;
// a consumer polls the 8-byte words it needs with strong loads until none is
// DU_PENDING.  Each word is single-copy atomic, so a value read that is not
// DU_PENDING is the final one: no flags and no fences are needed.  The same
// hand-off carries the sweep inputs (flux_res, D_inv, Gold) from k_flux<true>
// to the forward sweep running beside it.
constexpr unsigned long long DU_PENDING = 0xFFF4DEADBEEF0001ull;

__device__ __forceinline__ unsigned long long ld_relaxed_b64(const double *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void ld_relaxed_v2(const double *p, unsigned long long &a, unsigned long long &b) {
    asm volatile("ld.relaxed.gpu.global.v2.b64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}
__device__ __forceinline__ void st_relaxed_f64(double *p, double v) {
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

// Polls give up after SPIN_LIMIT rounds (about a second; d.spin_limit when
// set), or soon after another lane gave up: the failure goes to *d.err (the
// host reports MFCFD_ERR_TIMEOUT and the iteration's results are invalid).
constexpr int SPIN_LIMIT = 1 << 21;

__device__ __forceinline__ bool spin_continue(int &it, const DevCloud &d) {
    ++it;
    if ((it & 1023) == 0) {
        if (*(volatile int *)d.err) return false;
        __nanosleep(64);
    }
    if (it > (d.spin_limit > 0 ? d.spin_limit : SPIN_LIMIT)) {
        atomicExch(d.err, 1);
        return false;
    }
    return true;
}

__device__ __forceinline__ bool is_pending(double v) {
    return (unsigned long long)__double_as_longlong(v) == DU_PENDING;
}

// Poll one word until it is published.
__device__ __forceinline__ double poll_word(const double *p, const DevCloud &d) {
    unsigned long long v;
    int spins = 0;
    do {
        v = ld_relaxed_b64(p);
    } while (v == DU_PENDING && spin_continue(spins, d));
    return __longlong_as_double((long long)v);
}

__device__ __forceinline__ bool ready5(const unsigned long long v[5]) {
    return v[0] != DU_PENDING && v[1] != DU_PENDING && v[2] != DU_PENDING && v[3] != DU_PENDING &&
           v[4] != DU_PENDING;
}

// ---------------------------------------------------------------- flux residual

// Limited midpoint reconstruction of point j's q toward the offset
// (delx, dely, delz), then q -> primitive (interior_flux_dGxpos.f90:92-96,
// limiters.f90:12-52, qvariables_to_primitive_variables.f90:9-31).
template <typename R>
__device__ __forceinline__ void reconstruct(const DevCloud &d, int j, R delx, R dely, R delz, R prim[5]) {
    const double *qj = d.q + 5 * (size_t)j;
    const double *dqj = d.dq + 15 * (size_t)j;
    const double *qmj = d.qm + 10 * (size_t)j;
    const R eps2 = (R)d.eps2[j];
    R qt[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        const R q = (R)qj[r];
        const R temp = delx * (R)dqj[3 * r] + dely * (R)dqj[3 * r + 1] + delz * (R)dqj[3 * r + 2];
        const R del_neg = (q - R(0.5) * temp) - q;
        R phi = R(1.0);
        if (!(r_abs(del_neg) <= R(MF_LIM_EPS))) {
            const R del_pos = del_neg > R(0.0) ? (R)qmj[2 * r] - q : (R)qmj[2 * r + 1] - q;
            R num = (del_pos * del_pos) + eps2;
            num = num * del_neg + R(2.0) * del_neg * del_neg * del_pos;
            R den = del_pos * del_pos + R(2.0) * del_neg * del_neg;
            den = den + del_neg * del_pos + eps2;
            den = den * del_neg;
            const R t = num / den;
            phi = (t < R(1.0)) ? t : R(1.0);
        }
        qt[r] = q - R(0.5) * phi * temp;
    }
    qtilde_to_primitive(qt, prim);
}

// Per-list diagonal terms of D_inv (implicit_D_inv_interior.f90:46-417 /
// implicit_D_inv_wall.f90:45-356 with the geometry-only sums precomputed).
// u: the velocity component of list dd's axis; as: the speed of sound;
// row: the geometry row (dd, or 5 for an outer point's z+ over conn).
__device__ __forceinline__ double dinv_term(const DevCloud &d, int i, int dd, double u, double as, int row) {
    const double *g = d.geo + (size_t)i * GEO_STRIDE + (row - dd) * 8;
    const double temp = g[dd * 8 + G_DNUM], det = g[dd * 8 + G_DET];
    if ((dd & 1) == 0) {
        const double t1 = u + as;
        return 0.50 * fabs(t1 + fabs(t1)) * temp / det;
    }
    const double t1 = u - as;
    return -(0.50 * fabs(t1 - fabs(t1)) * temp / det);
}

__device__ __forceinline__ double dinv_term(const DevCloud &d, int i, int dd, double u, double as) {
    return dinv_term(d, i, dd, u, as, dd);
}

// implicit_D_inv_outer.f90:17-363 (backup driver) from the terms of rows
// 0-3 and of row 5 (z+ over conn): no minus on the x-/y- terms, the source's
// order of operations, and 1/delt of the tangential offset the direction
// loops leave behind (outer_delt; NaN: the time step).
__device__ __forceinline__ double dinv_outer(const DevCloud &d, int i, const double g5[5]) {
    double dt = d.outer_delt[i];
    if (dt != dt) dt = d.delt[i];
    const double temp = (1.0 / dt) - g5[0] + (-g5[1]) - g5[2] + (-g5[3]) - g5[4];
    return 1.0 / temp;
}

__device__ __forceinline__ double dinv_combine(int cls, double delt, const double gd[NDIR]) {
    double temp;
    if (cls == CLS_WALL) temp = (1.0 / delt) - 2.0 * (gd[0] + gd[1] + gd[2] + gd[3] + gd[5]);
    else temp = (1.0 / delt) - (gd[0] + gd[1] + gd[2] + gd[3] + gd[4] + gd[5]);
    return 1.0 / temp;
}

// The sweep inputs of point i computed by one warp (same arithmetic as
// k_dinv_gold): lanes 0-5 the D_inv terms, lane (list, component) the flux
// of prim and, for an unswept point, of prim(U + dU) in the shared frame.
// Strong stores: the forward sweep polls for these words.  The fluxes are
// evaluated in R; D_inv stays double.
template <typename R>
__device__ __forceinline__ void sweep_inputs_warp(const DevCloud &d, int i, int lane) {
    double p[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) p[r] = d.prim[5 * (size_t)i + r];
    const bool swept = d.swept[i] != 0;
    if (swept && d.cls[i] <= CLS_WALL) {   // D_inv of wall and interior points
        const double as = sqrt(1.40 * p[4] / p[0]);
        const double u = (lane >> 1) == 0 ? p[1] : ((lane >> 1) == 1 ? p[2] : p[3]);
        const double t = lane < NDIR ? dinv_term(d, i, lane, u, as) : 0.0;
        double gd[NDIR];
#pragma unroll
        for (int dd = 0; dd < NDIR; ++dd) gd[dd] = __shfl_sync(FULL, t, dd);
        if (lane == 0) st_relaxed_f64(d.dinv + i, dinv_combine(d.cls[i], d.delt[i], gd));
    } else if (swept && d.cls[i] == CLS_OUTER) {      // backup driver
        const double as = sqrt(1.40 * p[4] / p[0]);
        const double u = lane < 2 ? p[1] : (lane < 4 ? p[2] : p[3]);
        const double t = lane < 5 ? dinv_term(d, i, lane, u, as, lane == 4 ? 5 : lane) : 0.0;
        double g5[5];
#pragma unroll
        for (int dd = 0; dd < 5; ++dd) g5[dd] = __shfl_sync(FULL, t, dd);
        if (lane == 0) st_relaxed_f64(d.dinv + i, dinv_outer(d, i, g5));
    }
    if (d.shared_frame && lane < 30) {
        const int dd = lane / 5, c = lane - 5 * dd;
        FrameT<R> F0;
        load_frame(d.frame0, F0);
        R pr[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) pr[r] = (R)p[r];
        FluxPreT<R> P;
        flux_pre(pr, F0, P);
        AxisTermsT<R> At;
        axis_terms(P, dd >> 1, At);
        const R gold = flux_component(dd, c, P, At, At, At);
        st_relaxed_f64(d.gold + 30 * (size_t)i + lane, (double)gold);
        if (!swept) {
            R U[5], pn[5];
            FrameT<R> F;
            load_frame(d.frame + 9 * (size_t)i, F);
#pragma unroll
            for (int r = 0; r < 5; ++r) U[r] = (R)(d.dUp[5 * (size_t)i + r] + d.U[5 * (size_t)i + r]);
            conserved_to_primitive(U, F, pn);
            flux_pre(pn, F0, P);
            axis_terms(P, dd >> 1, At);
            const double v = (double)(flux_component(dd, c, P, At, At, At) - gold);
            const size_t o = DG_STRIDE * (size_t)i + DG_LIST * dd + c;
            st_relaxed_f64(d.dgf + o, v);
            st_relaxed_f64(d.dgb + o, v);
        }
        if (d.dg_old) {   // backup driver: the increment from before the sweeps
            R U[5], pn[5];
            FrameT<R> F;
            load_frame(d.frame + 9 * (size_t)i, F);
#pragma unroll
            for (int r = 0; r < 5; ++r) U[r] = (R)(d.dU_old[5 * (size_t)i + r] + d.U[5 * (size_t)i + r]);
            conserved_to_primitive(U, F, pn);
            flux_pre(pn, F0, P);
            axis_terms(P, dd >> 1, At);
            st_relaxed_f64(d.dg_old + DG_STRIDE * (size_t)i + DG_LIST * dd + c,
                           (double)(flux_component(dd, c, P, At, At, At) - gold));
        }
    }
}

// eval_flux_residual (flux_residual.f90:40-81): one warp per point.  Lanes
// own the point's distinct neighbours: each reconstructs both ends of its
// pair once and evaluates the flux of every list the neighbour belongs to;
// then 30 lanes (list, component) sum the list terms in list order and solve
// the 3x3 least-squares system with the precomputed moments.
//
// FUSED (chain schedule): the warps take the points in the forward sweep's
// order (d.pre_order) and also produce the point's sweep inputs (D_inv,
// fluxes of prim in the shared frame, the fixed increment of an unswept
// point) with strong stores, while the forward sweep runs concurrently and
// polls for them (they start as DU_PENDING).
//
// R: the type of the reconstruction, limiter and flux arithmetic (float in
// mixed precision); the offsets, weights, list sums and 3x3 solves are double.
// RS: the type of the sweep inputs' fluxes (float whenever the sweeps run in
// FP32, so that a sweep differences fluxes evaluated the same way).
// Blocks of the flux kernel per SM the compiler must fit: four for the FP64
// evaluation (128 registers, 16 warps per SM).  Beside the forward sweep it
// then keeps ahead of the sweep, which otherwise polled for inputs not yet
// written (1.1M points: flux 22.1 against 26.5 ms, iteration 53.0 against
// 55.1 ms with the earlier remedy, a lead launch of the order's first 16%).
// FP32 keeps the default: it is well ahead anyway.
template <typename R>
constexpr int flux_min_blocks() { return sizeof(R) == 8 ? 4 : 1; }

template <bool FUSED, typename R, typename RS = R>
__global__ void __launch_bounds__(FLUX_WARPS * 32, flux_min_blocks<R>()) k_flux(DevCloud d, int i0, int i1) {
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *T = smem + warp * FLUX_SMEM_PER_WARP;     // T[(dir*32 + slot)*5 + c]
    double *W = T + NDIR * MAX_SLOTS * 5;             // W[slot*3 + axis]
    // positions [i0, i1) of the visiting order (pre_order when FUSED)
    for (int i = i0 + blockIdx.x * FLUX_WARPS + warp; i < i1; i += gridDim.x * FLUX_WARPS) {
        const int p = FUSED ? d.pre_order[i] : i;
        const int cls = d.cls[p];
        if (cls <= 2) {
            const int ns = d.nslot[p];
            if (lane < ns) {
                const int k = d.slot_nbr[(size_t)p * MAX_SLOTS + lane];
                const int mask = d.slot_mask[(size_t)p * MAX_SLOTS + lane];
                Frame F;
                load_frame(d.frame + 9 * (size_t)p, F);
                FrameT<R> FR;
#pragma unroll
                for (int r = 0; r < 3; ++r) { FR.t1[r] = (R)F.t1[r]; FR.t2[r] = (R)F.t2[r]; FR.n[r] = (R)F.n[r]; }
                const double delx = d.x[k] - d.x[p], dely = d.y[k] - d.y[p], delz = d.z[k] - d.z[p];
                // dels*weights, delt*weights, deln*weights (weights 1 for power 0)
                const double w = d.wf ? d.wf[(size_t)MAX_SLOTS * p + lane] : 1.0;
                W[lane * 3 + 0] = (delx * F.t1[0] + dely * F.t1[1] + delz * F.t1[2]) * w;
                W[lane * 3 + 1] = (delx * F.t2[0] + dely * F.t2[1] + delz * F.t2[2]) * w;
                W[lane * 3 + 2] = (delx * F.n[0] + dely * F.n[1] + delz * F.n[2]) * w;
                int axes = 0;
#pragma unroll
                for (int dd = 0; dd < NDIR; ++dd)
                    if (mask & (1 << dd)) axes |= kind_axes(flux_kind(cls, dd));
                R prim[5];
                FluxPreT<R> Pi, Pk;
                AxisTermsT<R> Ai[3], Ak[3];
                reconstruct<R>(d, p, (R)delx, (R)dely, (R)delz, prim);
                flux_pre(prim, FR, Pi);
                reconstruct<R>(d, k, (R)delx, (R)dely, (R)delz, prim);
                flux_pre(prim, FR, Pk);
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    if (axes & (1 << a)) {
                        axis_terms(Pi, a, Ai[a]);
                        axis_terms(Pk, a, Ak[a]);
                    }
                }
                for (int dd = 0; dd < NDIR; ++dd) {
                    if (!(mask & (1 << dd))) continue;
                    const int kind = flux_kind(cls, dd);
#pragma unroll
                    for (int c = 0; c < 5; ++c) {
                        const R gi = flux_component(kind, c, Pi, Ai);
                        const R gk = flux_component(kind, c, Pk, Ak);
                        T[(dd * MAX_SLOTS + lane) * 5 + c] = (double)(gk - gi);
                    }
                }
            }
            __syncwarp();
            double G = 0.0;
            if (lane < 30) {
                const int dd = lane / 5, c = lane - 5 * dd;
                const int cnt = d.list_cnt[(size_t)p * NDIR + dd];
                const uint8_t *ent = d.list_ent + ((size_t)p * NDIR + dd) * LIST_STRIDE;
                double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll 4
                for (int j = 0; j < cnt; ++j) {
                    const int s = ent[j];
                    const double t = T[(dd * MAX_SLOTS + s) * 5 + c];
                    sx = sx + t * W[s * 3 + 0];
                    sy = sy + t * W[s * 3 + 1];
                    sz = sz + t * W[s * 3 + 2];
                }
                const double *g = d.geo + (size_t)p * GEO_STRIDE + dd * 8;
                const double num = cramer_num(dd >> 1, g, sx, sy, sz);
                // outer_flux_dG*.f90:118-124 multiply by 1/det; the others divide
                G = (cls == CLS_OUTER) ? num * (1.0 / g[G_DET]) : num / g[G_DET];
            }
            double gd[NDIR];
#pragma unroll
            for (int dd = 0; dd < NDIR; ++dd) gd[dd] = __shfl_sync(FULL, G, dd * 5 + (lane % 5));
            if (lane < 5) {
                double r;
                if (cls == CLS_INTERIOR) r = gd[0] + gd[1] + gd[2] + gd[3] + gd[4] + gd[5];
                else if (cls == CLS_WALL) r = 2.0 * (gd[0] + gd[1] + gd[2] + gd[3] + gd[5]);
                else r = gd[0] + gd[1] + gd[2] + gd[3] + gd[4];
                if (FUSED) st_relaxed_f64(d.flux_res + 5 * (size_t)p + lane, r);
                else d.flux_res[5 * (size_t)p + lane] = r;
            }
        }
        if (FUSED) sweep_inputs_warp<RS>(d, p, lane);
        __syncwarp();
    }
}

// ---------------------------------------------------------------- D_inv and sweep inputs

// Fluxes of prim in the shared interior frame, all six directions.
__device__ __forceinline__ void flux6_frame0(const DevCloud &d, const double prim[5], double out[30]) {
    Frame F;
#pragma unroll
    for (int r = 0; r < 3; ++r) { F.t1[r] = d.frame0[r]; F.t2[r] = d.frame0[3 + r]; F.n[r] = d.frame0[6 + r]; }
    FluxPre P;
    flux_pre(prim, F, P);
    AxisTerms A[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) axis_terms(P, a, A[a]);
#pragma unroll
    for (int dd = 0; dd < NDIR; ++dd)
#pragma unroll
        for (int c = 0; c < 5; ++c) out[dd * 5 + c] = flux_component(dd, c, P, A);
}

// Before the sweeps: every published-increment word, and dU of every swept
// point, is set to DU_PENDING (coalesced grid-stride fill).  With inputs set,
// also the swept points' flux_res, D_inv and Gold, which k_flux<true>
// produces while the forward sweep runs.
__global__ void k_pending(DevCloud d, int inputs) {
    const double pend = __longlong_as_double((long long)DU_PENDING);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t ng = (size_t)d.n * DG_STRIDE, nu = (size_t)d.n * 5, n30 = (size_t)d.n * 30;
    for (size_t w = t0; w < ng; w += stride) {
        d.dgf[w] = pend;
        d.dgb[w] = pend;
        if (inputs && d.dg_old) d.dg_old[w] = pend;   // produced beside the forward sweep
    }
    for (size_t w = t0; w < nu; w += stride) {
        if (d.swept[w / 5]) {
            d.dUp[w] = pend;
            d.dUn[w] = pend;
            if (inputs && (d.cls[w / 5] <= CLS_WALL || d.cls[w / 5] == CLS_OUTER)) d.flux_res[w] = pend;
        }
    }
    if (inputs) {
        for (size_t w = t0; w < (size_t)d.n; w += stride)
            if (d.swept[w] && (d.cls[w] <= CLS_WALL || d.cls[w] == CLS_OUTER)) d.dinv[w] = pend;
        if (d.shared_frame)
            for (size_t w = t0; w < n30; w += stride)
                if (d.swept[w / 30]) d.gold[w] = pend;
    }
}

// implicit_D_inv_interior.f90:46-417 / implicit_D_inv_wall.f90:45-356 (see
// dinv_term); plus the sweep inputs that do not depend on the sweep: G(prim_k) in the shared frame for every point and the
// published increment G(prim(U_k + dU_k)) - G(prim_k) of points the sweeps
// never update (outer points, point 1), over the DU_PENDING that k_pending
// wrote there.
__global__ void __launch_bounds__(128) k_dinv_gold(DevCloud d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const int cls = d.cls[i];
    const double *p = d.prim + 5 * (size_t)i;
    if (d.swept[i] && cls <= CLS_WALL) {
        const double as = sqrt(1.40 * p[4] / p[0]);
        double gd[NDIR];
#pragma unroll
        for (int dd = 0; dd < NDIR; ++dd) gd[dd] = dinv_term(d, i, dd, p[1 + (dd >> 1)], as);
        d.dinv[i] = dinv_combine(cls, d.delt[i], gd);
    } else if (d.swept[i] && cls == CLS_OUTER) {   // backup driver
        const double as = sqrt(1.40 * p[4] / p[0]);
        double g5[5];
#pragma unroll
        for (int dd = 0; dd < 5; ++dd) g5[dd] = dinv_term(d, i, dd, p[1 + (dd >> 1)], as, dd == 4 ? 5 : dd);
        d.dinv[i] = dinv_outer(d, i, g5);
    }
    if (d.shared_frame) {
        double prim[5], gold[30];
#pragma unroll
        for (int r = 0; r < 5; ++r) prim[r] = p[r];
        flux6_frame0(d, prim, gold);
#pragma unroll
        for (int c = 0; c < 30; ++c) d.gold[30 * (size_t)i + c] = gold[c];
        if (!d.swept[i]) {
            double U[5], pn[5], gnew[30];
            Frame F;
            load_frame(d.frame + 9 * (size_t)i, F);
#pragma unroll
            for (int r = 0; r < 5; ++r) U[r] = d.dUp[5 * (size_t)i + r] + d.U[5 * (size_t)i + r];
            conserved_to_primitive(U, F, pn);
            flux6_frame0(d, pn, gnew);
#pragma unroll
            for (int c = 0; c < 30; ++c) {
                const double v = gnew[c] - gold[c];
                const size_t o = DG_STRIDE * (size_t)i + DG_LIST * (c / 5) + c % 5;
                d.dgf[o] = v;
                d.dgb[o] = v;
            }
        }
        if (d.dg_old) {   // backup driver: the increment from before the sweeps
            double U[5], pn[5], gnew[30];
            Frame F;
            load_frame(d.frame + 9 * (size_t)i, F);
#pragma unroll
            for (int r = 0; r < 5; ++r) U[r] = d.dU_old[5 * (size_t)i + r] + d.U[5 * (size_t)i + r];
            conserved_to_primitive(U, F, pn);
            flux6_frame0(d, pn, gnew);
#pragma unroll
            for (int c = 0; c < 30; ++c)
                d.dg_old[DG_STRIDE * (size_t)i + DG_LIST * (c / 5) + c % 5] = gnew[c] - gold[c];
        }
    }
}

// ---------------------------------------------------------------- LU-SGS sweeps

// Per-warp shared memory of the sweep kernels.  SweepStage holds everything a
// point reads that the sweep itself does not change (its terms, geometry,
// fluxes of prim in the shared frame, D_inv, U, frame, slot table); it is
// filled with cp.async, so the chain kernel loads the next point's stage
// while it works on the current one.
struct __align__(16) SweepStage {
    SweepEntry ent[SWEEP_MAX_ENTRIES];
    double geo[GEO_STRIDE];
    double gold[32];
    double U[6];
    double base[6];
    double frame[10];
    double dinv[2];
    int32_t slot_nbr[MAX_SLOTS];
    uint8_t slot_mask[MAX_SLOTS];
    uint32_t need;
    uint32_t old;                 // slots read from before the sweep (backup driver)
    int32_t pad[2];
};
constexpr int SW_T_DOUBLES = NDIR * MAX_SLOTS * 5;                  // term fluxes, >= SWEEP_MAX_ENTRIES * 5
constexpr int SW_RING_DOUBLES = CHAIN_RING * 30;                    // chain: last published increments
constexpr int SWEEP_SMEM_BYTES = SW_T_DOUBLES * 8 + (int)sizeof(SweepStage);   // one stage
constexpr int CHAIN_SMEM_BYTES = (SW_T_DOUBLES + SW_RING_DOUBLES) * 8 + 2 * (int)sizeof(SweepStage);
static_assert(SW_T_DOUBLES >= SWEEP_MAX_ENTRIES * 5, "T buffer too small");
static_assert(SW_T_DOUBLES * 8 >= SWEEP_MAX_ENTRIES * 5 * 8 + SWEEP_MAX_ENTRIES, "no room for the terms' flags");
static_assert(SW_T_DOUBLES == G0_DOUBLES && G0_DOUBLES % 2 == 0, "a g0 block is one T buffer of 16-byte pairs");
static_assert(SWEEP_MAX_ENTRIES <= 96, "entries are polled in three passes of 32");
static_assert(sizeof(SweepStage) % 16 == 0 && SWEEP_SMEM_BYTES % 16 == 0 && CHAIN_SMEM_BYTES % 16 == 0,
              "stage alignment");

enum SweepMode { MODE_LEVELS = 0, MODE_DATAFLOW = 1, MODE_CHAINS = 2 };

__device__ __forceinline__ void cp_async16(void *s, const void *g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(s)),
                 "l"(g)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void *s, const void *g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(s)),
                 "l"(g)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void *s, const void *g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(s)),
                 "l"(g)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ int item_count(uint32_t cnt, int e) { return (int)((cnt >> (5 * e)) & 31u); }

// The record of point p for the level and dataflow schedules (the chain
// schedule reads precomputed ones).
__device__ __forceinline__ ChainItem make_item(const DevCloud &d, int p, bool forward) {
    ChainItem it;
    it.p = p;
    it.off = forward ? d.fwd_off[p] : d.bwd_off[p];
    const uint8_t *cnt = (forward ? d.fwd_cnt : d.bwd_cnt) + (size_t)p * NDIR;
    it.cnt = 0;
#pragma unroll
    for (int e = 0; e < NDIR; ++e) it.cnt |= (uint32_t)cnt[e] << (5 * e);
    it.info = (d.cls[p] == CLS_WALL ? CI_WALL : 0u) | (d.consumer_shared[p] ? CI_SHARED : 0u) | CI_PUBLISH |
              (d.cls[p] == CLS_SUPERSONIC ? CI_COPY : 0u) | (d.cls[p] == CLS_OUTER ? CI_OUTER : 0u);
    return it;
}

// Issue the cp.async copies of one point's stage (all lanes; caller commits).
// Every source is 16-byte aligned for the 16-byte copies: entries are 32-byte
// records, geo rows 384 bytes, gold rows 240 bytes, slot rows 128 / 32 bytes.
__device__ __forceinline__ void stage_issue(const DevCloud &d, const ChainItem &it, bool forward, int lane,
                                            SweepStage *st) {
    const size_t p = (size_t)it.p;
    int total = 0;
#pragma unroll
    for (int e = 0; e < NDIR; ++e) total += item_count(it.cnt, e);
    const char *es = reinterpret_cast<const char *>((forward ? d.fwd_ent : d.bwd_ent) + it.off);
    char *ed = reinterpret_cast<char *>(st->ent);
    for (int j = lane; j < 2 * total; j += 32) cp_async16(ed + 16 * j, es + 16 * j);
    if (lane < GEO_STRIDE / 2) cp_async16(st->geo + 2 * lane, d.geo + p * GEO_STRIDE + 2 * lane);
    if (lane < 15) cp_async16(st->gold + 2 * lane, d.gold + 30 * p + 2 * lane);
    if (lane < 5) {
        cp_async8(st->U + lane, d.U + 5 * p + lane);
        cp_async8(st->base + lane, (forward ? d.flux_res : d.dUp) + 5 * p + lane);
    } else if (lane < 14) {
        cp_async8(st->frame + (lane - 5), d.frame + 9 * p + (lane - 5));
    } else if (lane == 14) {
        cp_async8(st->dinv, d.dinv + p);
    } else if (!(it.info & CI_SHARED)) {
        if (lane < 23) cp_async16(st->slot_nbr + 4 * (lane - 15), d.slot_nbr + p * MAX_SLOTS + 4 * (lane - 15));
        else if (lane < 25) cp_async16(st->slot_mask + 16 * (lane - 23), d.sweep_slot_mask + p * MAX_SLOTS + 16 * (lane - 23));
        else if (lane == 25) cp_async4(&st->need, (forward ? d.fwd_need : d.bwd_need) + p);
        else if (lane == 26) cp_async4(&st->old, (forward ? d.fwd_old : d.bwd_old) + p);
    }
}

// Phase A of a point outside the shared frame, one lane per neighbour slot:
// the fluxes of the neighbour's state at the start of the sweep in the
// point's frame, for every list the slot is in, into
// T[(list * MAX_SLOTS + slot) * 5 + component].  The sweep runs it in place,
// or k_g0 runs it for all such points before the sweeps (the same code, so
// the same bits).
template <typename R>
__device__ __forceinline__ void neighbour_fluxes(const DevCloud &d, int cls, const FrameT<R> &Fp, int k_slot,
                                                 int mask_slot, int lane, double *T) {
    R po[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) po[r] = (R)d.prim[5 * (size_t)k_slot + r];
    FluxPreT<R> Po;
    flux_pre(po, Fp, Po);
    int axes = 0;
#pragma unroll
    for (int e = 0; e < NDIR; ++e)
        if (mask_slot & (1 << e)) axes |= kind_axes(flux_kind(cls, e));
    AxisTermsT<R> Ao[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
        if (axes & (1 << a)) axis_terms(Po, a, Ao[a]);
    for (int e = 0; e < NDIR; ++e) {
        if (!(mask_slot & (1 << e))) continue;
        const int kind = flux_kind(cls, e);
#pragma unroll
        for (int cc = 0; cc < 5; ++cc)
            T[(e * MAX_SLOTS + lane) * 5 + cc] = (double)flux_component(kind, cc, Po, Ao);
    }
}

// Phase A of every g0 point (Topology::g0_pts) from the state at the start
// of the iteration, which both sweeps read: one warp per point.
template <typename R>
__global__ void __launch_bounds__(128) k_g0(DevCloud d) {
    const int w = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (w >= d.n_g0) return;
    const int p = d.g0_pts[w];
    if (lane >= d.nslot[p]) return;
    const int mask = d.sweep_slot_mask[(size_t)p * MAX_SLOTS + lane];
    if (!mask) return;
    FrameT<R> Fp;
    load_frame(d.frame + 9 * (size_t)p, Fp);
    neighbour_fluxes<R>(d, d.cls[p], Fp, d.slot_nbr[(size_t)p * MAX_SLOTS + lane], mask, lane,
                        d.g0 + (size_t)w * G0_DOUBLES);
}

// One point of the forward (LdelU) or backward (UdelU) sweep, processed by
// one warp (implicit_forward_and_reverse_sweeps.f90:30-37 / :61-68), from its
// stage in shared memory.
//
// Phase A (no dependency on the sweep): points outside the shared frame
// evaluate G(prim_k) of their neighbours.  Phase B: collect the neighbours'
// increments as they are published (points in the shared frame: the
// published flux increments; others: dU_k, then G(prim(U_k + dU_k)) -
// G(prim_k)).  Phase C: sum each list in list order (30 lanes: list x
// component), solve the 3x3 systems, update dU and publish this point's own
// flux increment.
//
// The chain schedule reads increments that this warp published within its
// last CHAIN_RING points from `ring` (slot in the term's ENT_RING bits) and
// writes its own to ring slot `ring_slot`; a point publishes to global memory
// only if some consumer reads it there (CI_PUBLISH).
//
// R: the type of the flux evaluations (float in mixed precision); the list
// sums, 3x3 solves, D_inv and the increments themselves are double.
//
// A CI_G0 point's phase A is a copy of its k_g0 block into T, which the
// chain kernel issued as a cp.async group before this call (followed by one
// more group, the next point's stage, when g0_newer); phase B waits for it.
// FOLD (mixed precision): each term's weight carries its list's 3x3 solve
// (folded when the handle is attached), so phase C sums weight x term;
// otherwise phase C sums
// the three weighted moments in FP64 and solves, as the reference does.
template <int MODE, typename R, bool FOLD = false>
__device__ void sweep_point(const DevCloud &d, const ChainItem &it, const SweepStage *st, bool forward, int lane,
                            double *T, double *ring, int ring_slot, bool g0_newer = false) {
    constexpr bool CHAINS = MODE == MODE_CHAINS;
    const int p = it.p;
    const bool wall = (it.info & CI_WALL) != 0;
    const bool shared = (it.info & CI_SHARED) != 0;
    const bool copy = (it.info & CI_COPY) != 0;       // supersonic point
    const bool outer = (it.info & CI_OUTER) != 0;     // backup driver
    const bool hold = p + 1 == d.withhold1;           // failure-detection hook: publish nothing
    const int cls = wall ? CLS_WALL : (outer ? CLS_OUTER : CLS_INTERIOR);
    const SweepEntry *E = st->ent;
    const int dd = lane / 5, c = lane - 5 * (lane / 5);
    int total = 0, lo = 0, hi = 0;
#pragma unroll
    for (int e = 0; e < NDIR; ++e) {
        const int ce = item_count(it.cnt, e);
        if (e < dd) lo += ce;
        if (e <= dd) hi += ce;
        total += ce;
    }

    // ---- phase A
    double g[7] = {0, 0, 0, 0, 0, 0, 1.0};
    double gold = 0.0;
    if (lane < 30) {
        const int grow = (outer && dd == 4) ? 5 : dd;   // outer z+ over conn: row 5
#pragma unroll
        for (int r = 0; r < 7; ++r) g[r] = st->geo[grow * 8 + r];
        gold = st->gold[lane];
    }
    double dinv = 0.0, base5 = 0.0;
    if (lane < 5) {
        dinv = st->dinv[0];
        base5 = st->base[lane];
    }
    // inputs the concurrent flux kernel had not produced when the stage was copied
    if (lane < 30 && is_pending(gold)) gold = poll_word(d.gold + 30 * (size_t)p + lane, d);
    if (lane < 5 && !copy) {
        if (is_pending(dinv)) dinv = poll_word(d.dinv + p, d);
        if (is_pending(base5)) base5 = poll_word((forward ? d.flux_res : d.dUp) + 5 * (size_t)p + lane, d);
    }
    double Up[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) Up[r] = st->U[r];
    FrameT<R> Fp;
    load_frame(st->frame, Fp);
    double dnew = 0.0;
    if (copy) {
        // implicit_forward_and_reverse_sweeps.f90:38-51 / :69-82: the
        // nearest neighbour's increment, updated earlier in this sweep or
        // from before it
        if (lane < 5) {
            const int q = E[0].k;
            double *dst = (forward ? d.dUp : d.dUn) + 5 * (size_t)p + lane;
            if (q >= 0)
                dnew = (E[0].pad & ENT_COPY_NEW) ? poll_word((forward ? d.dUp : d.dUn) + 5 * (size_t)q + lane, d)
                                                 : d.dU_old[5 * (size_t)q + lane];
            if (!hold) st_relaxed_f64(dst, dnew);
        }
    } else {
        double sx = 0.0, sy = 0.0, sz = 0.0, G0acc = 0.0;   // phase C's list sums
        const uint32_t need = shared ? 0u : st->need;
        const bool mine = !shared && (need >> lane) & 1u;
        const bool g0 = CHAINS && (it.info & CI_G0) != 0;   // warp-uniform
        int k_slot = 0, mask_slot = 0;
        if (mine) {
            k_slot = st->slot_nbr[lane];
            mask_slot = st->slot_mask[lane];
            if (!g0) neighbour_fluxes<R>(d, cls, Fp, k_slot, mask_slot, lane, T);
        }

        // ---- phase B
        // The list sums of phase C run in list order from `pos`; in the shared
        // frame they advance over the terms that have landed while later
        // ones are still awaited, so only the terms after the last arrival
        // remain once it lands (the additions keep their order).
        int pos = lo;
        if (shared) {
            // lane owns entries lane, lane+32, lane+64; all their loads are in
            // flight together, re-polling only the ones still pending; a
            // landed term's flag (past the 96 terms' values in T) tells the
            // summing lanes it is there
            const double *src = forward ? d.dgf : d.dgb;
            uint8_t *rdy = reinterpret_cast<uint8_t *>(T + 5 * SWEEP_MAX_ENTRIES);
            uint32_t pend = 0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int j = lane + 32 * q;
                if (j >= total) continue;
                const int pad = E[j].pad;
                if (CHAINS && (pad & ENT_RING)) {
                    const double *rs = ring + 30 * ((pad >> ENT_RING_SHIFT) & 15) + 5 * (pad & 255);
#pragma unroll
                    for (int cc = 0; cc < 5; ++cc) T[j * 5 + cc] = rs[cc];
                    rdy[j] = 1;
                } else {
                    pend |= 1u << q;
                    rdy[j] = 0;
                }
            }
            int spins = 0;
            for (;;) {
                if (pend) {
                    unsigned long long v[3][5];
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        if (!((pend >> q) & 1u)) continue;
                        const int j = lane + 32 * q;
                        // backup driver: a term from before the sweep reads dg_old
                        const double *base = (E[j].pad & ENT_OLD) ? d.dg_old : src;
                        const double *gs = base + DG_STRIDE * (size_t)E[j].k + DG_LIST * (E[j].pad & 255);
                        ld_relaxed_v2(gs, v[q][0], v[q][1]);
                        ld_relaxed_v2(gs + 2, v[q][2], v[q][3]);
                        v[q][4] = ld_relaxed_b64(gs + 4);
                    }
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        if (!((pend >> q) & 1u) || !ready5(v[q])) continue;
                        const int j = lane + 32 * q;
#pragma unroll
                        for (int cc = 0; cc < 5; ++cc) T[j * 5 + cc] = __longlong_as_double(v[q][cc]);
                        rdy[j] = 1;
                        pend &= ~(1u << q);
                    }
                    if (pend && !spin_continue(spins, d)) {
                        // the wait ran out (d.err is set): the terms stay unset
#pragma unroll
                        for (int q = 0; q < 3; ++q)
                            if ((pend >> q) & 1u) rdy[lane + 32 * q] = 1;
                        pend = 0;
                    }
                }
                __syncwarp();
                if (__all_sync(FULL, pend == 0)) break;
                if (lane < 30) {
                    while (pos < hi && rdy[pos]) {
                        const double t = T[pos * 5 + c];
                        if constexpr (FOLD) {
                            G0acc = G0acc + t * E[pos].w[0];
                        } else {
                            sx = sx + t * E[pos].w[0];
                            sy = sy + t * E[pos].w[1];
                            sz = sz + t * E[pos].w[2];
                        }
                        ++pos;
                    }
                }
                __syncwarp();
            }
        } else {
            FluxPreT<R> Pn;
            AxisTermsT<R> An[3];
            if (mine) {
                const bool old = (st->old >> lane) & 1u;   // backup driver: from before the sweep
                const double *dsrc = (old ? d.dU_old : (forward ? d.dUp : d.dUn)) + 5 * (size_t)k_slot;
                unsigned long long v[5];
                int spins = 0;
                do {
#pragma unroll
                    for (int r = 0; r < 5; ++r) v[r] = ld_relaxed_b64(dsrc + r);
                } while (!ready5(v) && spin_continue(spins, d));
                R U[5], pn[5];
#pragma unroll
                for (int r = 0; r < 5; ++r) U[r] = (R)(__longlong_as_double(v[r]) + d.U[5 * (size_t)k_slot + r]);
                FrameT<R> Fk;
                load_frame(d.frame + 9 * (size_t)k_slot, Fk);
                conserved_to_primitive(U, Fk, pn);
                flux_pre(pn, Fp, Pn);
                int axes = 0;
#pragma unroll
                for (int e = 0; e < NDIR; ++e)
                    if (mask_slot & (1 << e)) axes |= kind_axes(flux_kind(cls, e));
#pragma unroll
                for (int a = 0; a < 3; ++a)
                    if (axes & (1 << a)) axis_terms(Pn, a, An[a]);
            }
            if (g0) {
                // the copied phase-A fluxes: every lane's copies have landed
                if (g0_newer) cp_async_wait_one();
                else cp_async_wait_all();
                __syncwarp();
            }
            if (mine) {
                for (int e = 0; e < NDIR; ++e) {
                    if (!(mask_slot & (1 << e))) continue;
                    const int kind = flux_kind(cls, e);
#pragma unroll
                    for (int cc = 0; cc < 5; ++cc) {
                        double *t = &T[(e * MAX_SLOTS + lane) * 5 + cc];
                        *t = (double)(flux_component(kind, cc, Pn, An) - (R)*t);
                    }
                }
            }
        }
        __syncwarp();

        // ---- phase C (from pos: the terms not yet summed)
        double G = 0.0;
        if constexpr (FOLD) {
            // mixed precision: each term's weight already carries the list's
            // 3x3 solve (cofactors / det, FP64, computed at set-up)
            G = G0acc;
            if (lane < 30) {
#pragma unroll 4
                for (int jj = pos; jj < hi; ++jj) {
                    const double t = shared ? T[jj * 5 + c] : T[(dd * MAX_SLOTS + ((E[jj].pad >> 8) & 255)) * 5 + c];
                    G = G + t * E[jj].w[0];
                }
            }
        } else {
            if (lane < 30) {
                // unrolled so the next terms' shared-memory loads overlap; the
                // additions keep their order
#pragma unroll 4
                for (int jj = pos; jj < hi; ++jj) {
                    const double t = shared ? T[jj * 5 + c] : T[(dd * MAX_SLOTS + ((E[jj].pad >> 8) & 255)) * 5 + c];
                    sx = sx + t * E[jj].w[0];
                    sy = sy + t * E[jj].w[1];
                    sz = sz + t * E[jj].w[2];
                }
            }
            if (lane < 30) G = cramer_num(dd >> 1, g, sx, sy, sz) / g[6];
        }
        double gd[NDIR];
#pragma unroll
        for (int e = 0; e < NDIR; ++e) gd[e] = __shfl_sync(FULL, G, e * 5 + (lane % 5));
        if (lane < 5) {
            double lu;
            if (wall) lu = 2.0 * (gd[0] + gd[1] + gd[2] + gd[3] + gd[5]);
            else if (outer) lu = gd[0] + gd[1] + gd[2] + gd[3] + gd[4];   // *_sweep_outer.f90:406
            else lu = gd[0] + gd[1] + gd[2] + gd[3] + gd[4] + gd[5];
            if (forward) {
                dnew = -(dinv * (base5 + lu));
                if (!hold) st_relaxed_f64(d.dUp + 5 * (size_t)p + lane, dnew);
            } else {
                dnew = base5 - dinv * lu;
                if (!hold) st_relaxed_f64(d.dUn + 5 * (size_t)p + lane, dnew);
            }
        }
    }
    if (d.shared_frame) {
        // publish this point's increment for the consumers in the shared frame
        R U[5], pn[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) U[r] = (R)(__shfl_sync(FULL, dnew, r) + Up[r]);
        if (lane < 30) {
            conserved_to_primitive(U, Fp, pn);
            FrameT<R> F0;
            load_frame(d.frame0, F0);
            FluxPreT<R> P;
            flux_pre(pn, F0, P);
            AxisTermsT<R> At;
            axis_terms(P, dd >> 1, At);
            const double v = (double)(flux_component(dd, c, P, At, At, At) - (R)gold);
            if ((it.info & CI_PUBLISH) && !hold)
                st_relaxed_f64((forward ? d.dgf : d.dgb) + DG_STRIDE * (size_t)p + DG_LIST * dd + c, v);
            if (CHAINS) ring[30 * ring_slot + lane] = v;
        }
    }
    __syncwarp();
}

// Stage one point synchronously and sweep it (level and dataflow schedules).
template <int MODE>
__device__ __forceinline__ void sweep_point_sync(const DevCloud &d, int p, bool forward, int lane, char *smb) {
    double *T = reinterpret_cast<double *>(smb);
    SweepStage *st = reinterpret_cast<SweepStage *>(smb + SW_T_DOUBLES * 8);
    const ChainItem it = make_item(d, p, forward);
    stage_issue(d, it, forward, lane, st);
    cp_async_commit();
    cp_async_wait_all();
    __syncwarp();
    sweep_point<MODE, double>(d, it, st, forward, lane, T, nullptr, 0);
}

// Level-synchronous sweep in one CTA: the points of a level are independent
// (none reads another's increment), so warps take them in parallel and a
// block barrier separates levels; every poll succeeds at once.
__global__ void __launch_bounds__(SWEEP_THREADS, 1) k_sweep_levels(DevCloud d, int forward) {
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    char *smb = reinterpret_cast<char *>(smem) + warp * SWEEP_SMEM_BYTES;
    const int nl = forward ? d.n_fwd_levels : d.n_bwd_levels;
    const int32_t *lptr = forward ? d.fwd_lvl_ptr : d.bwd_lvl_ptr;
    const int32_t *lpts = forward ? d.fwd_lvl_pts : d.bwd_lvl_pts;
    for (int l = 0; l < nl; ++l) {
        const int a = lptr[l], b = lptr[l + 1];
        for (int idx = a + warp; idx < b; idx += SWEEP_WARPS)
            sweep_point_sync<MODE_LEVELS>(d, lpts[idx], forward != 0, lane, smb);
        __syncthreads();
    }
}

// Dataflow sweep over many SMs: each warp takes the next point of the
// level-major (topological) order from a global counter and polls for the
// increments it reads.  A point's dependencies are always taken before it by
// warps that are already running, so the polls end; each is bounded anyway.
constexpr int DF_WARPS = 4;

__global__ void __launch_bounds__(DF_WARPS * 32) k_sweep_df(DevCloud d, int forward) {
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    char *smb = reinterpret_cast<char *>(smem) + warp * SWEEP_SMEM_BYTES;
    int *counter = d.sweep_counter + (forward ? 0 : 1);
    const int32_t *order = forward ? d.fwd_lvl_pts : d.bwd_lvl_pts;
    const int total = d.n_swept;
    for (;;) {
        int idx = 0;
        if (lane == 0) idx = atomicAdd(counter, 1);
        idx = __shfl_sync(FULL, idx, 0);
        if (idx >= total) break;
        sweep_point_sync<MODE_DATAFLOW>(d, order[idx], forward != 0, lane, smb);
    }
}

// Chain sweep: each warp walks its own list of point records (fixed at
// set-up, topological order).  The stage of the next point is copied in
// while the current one is processed (two stage buffers).
//
// Residency: an SM holds three 4-warp blocks of the mixed-precision sweep
// (71 KB of shared memory each; at most 168 registers, which the launch
// bounds below ask for), two 4-warp blocks of the FP64 sweep (226
// registers) or one 8-warp block; in slots of a sixth of an SM, 2, 3 or 6
// (chain_block_slots).  The chain blocks running at once (one cloud, or the
// handles of a batch) take at most 6 * (SMs - CH_FREE_SMS) slots.  So all of
// them fit together, and at least CH_FREE_SMS SMs' worth of room stays
// free for blocks of the concurrent flux kernels, whose outputs the forward
// sweeps poll for (a flux kernel never waits, so the blocks it holds are
// released): every poll ends.
constexpr int CH_FREE_SMS = 16;

template <int WPB, bool FOLD>
constexpr int chain_min_blocks() {
    return (WPB == 4 && FOLD) ? 3 : 1;
}

// One block of a cloud's chain sweep: block `block` of the cloud's
// (ch_warps + WPB - 1) / WPB.  R: the type of the sweep's flux evaluations;
// FOLD: folded term weights (MFCFD_PRECISION_MIXED and MIXED_DC).  FP64
// <double, false>; mixed and defect correction <float, true>.
template <int WPB, typename R, bool FOLD>
__device__ __forceinline__ void chain_sweep(const DevCloud &d, int forward, int block) {
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    char *smb = reinterpret_cast<char *>(smem) + warp * CHAIN_SMEM_BYTES;
    double *T = reinterpret_cast<double *>(smb);
    double *ring = T + SW_T_DOUBLES;
    SweepStage *stg = reinterpret_cast<SweepStage *>(ring + SW_RING_DOUBLES);
    const int me = block * WPB + warp;
    if (me >= d.ch_warps) return;
    const int dir = forward ? 0 : 1;
    const int a = d.ch_ptr[dir][me], b = d.ch_ptr[dir][me + 1];
    if (a >= b) return;
    const ChainItem *items = d.ch_items[dir];
    ChainItem cur = items[a];
    stage_issue(d, cur, forward != 0, lane, &stg[0]);
    cp_async_commit();
    ChainItem nxt = a + 1 < b ? items[a + 1] : cur;
    for (int idx = a; idx < b; ++idx) {
        const int s = (idx - a) & 1;
        cp_async_wait_all();
        __syncwarp();
        if (cur.info & CI_G0) {
            // phase A of this point, computed before the sweep (k_g0): into T,
            // which the previous point no longer uses
            const char *src = reinterpret_cast<const char *>(d.g0 + (size_t)(cur.info >> CI_G0_SHIFT) * G0_DOUBLES);
            char *dst = reinterpret_cast<char *>(T);
            for (int j = lane; j < G0_DOUBLES / 2; j += 32) cp_async16(dst + 16 * j, src + 16 * j);
            cp_async_commit();
        }
        if (idx + 1 < b) {
            stage_issue(d, nxt, forward != 0, lane, &stg[s ^ 1]);
            cp_async_commit();
        }
        const ChainItem after = idx + 2 < b ? items[idx + 2] : nxt;
        sweep_point<MODE_CHAINS, R, FOLD>(d, cur, &stg[s], forward != 0, lane, T, ring, (idx - a) % CHAIN_RING,
                                          idx + 1 < b);
        cur = nxt;
        nxt = after;
    }
}

template <int WPB, typename R, bool FOLD>
__global__ void __launch_bounds__(WPB * 32, chain_min_blocks<WPB, FOLD>()) k_sweep_chain(DevCloud d, int forward) {
    chain_sweep<WPB, R, FOLD>(d, forward, blockIdx.x);
}

// The chain sweeps of a group of clouds in one launch: blocks
// [block_start[c], block_start[c + 1]) are cloud c's.  The clouds share
// nothing; a block finds its cloud and runs that cloud's schedule as the
// single-cloud kernel would.  The group lives in the launch's parameters, so
// every block reads its cloud's pointers from the constant bank.
template <int WPB, typename R, bool FOLD>
__global__ void __launch_bounds__(WPB * 32, chain_min_blocks<WPB, FOLD>())
    k_sweep_chain_group(const __grid_constant__ ChainGroup g, int forward) {
    int c = 0;
    while (c + 1 < g.count && (int)blockIdx.x >= g.block_start[c + 1]) ++c;
    chain_sweep<WPB, R, FOLD>(g.cloud[c], forward, (int)blockIdx.x - g.block_start[c]);
}

template <int WPB>
static int chain_smem() {
    return WPB * CHAIN_SMEM_BYTES;
}
// three 4-warp blocks per SM: 228 KB of shared memory, 1 KB of it reserved per block
static_assert(3 * (4 * CHAIN_SMEM_BYTES + 1024) <= 228 * 1024, "three 4-warp chain blocks per SM");
// A spread chain block asks for this much shared memory, so that no second
// block fits beside it (2 x (116 + 1) KB > 228 KB) and each of its four
// warps has one of the SM's four sub-partitions to itself.
constexpr int CHAIN_SPREAD_SMEM = 116 * 1024;
static_assert(2 * (CHAIN_SPREAD_SMEM + 1024) > 228 * 1024 && CHAIN_SPREAD_SMEM >= 4 * CHAIN_SMEM_BYTES,
              "a spread block holds its SM alone");

static int chain_smem_bytes(int wpb, int spread) {
    if (wpb == 4) return spread ? CHAIN_SPREAD_SMEM : chain_smem<4>();
    return chain_smem<8>();
}

// ---------------------------------------------------------------- state update

// state_update_implicit.f90:119-152 + 189-191 (or state_update.f90:29-78
// under MFCFD_UPDATE_EXPLICIT), then the next iteration's
// compute_conserved_vector / eval_q_variables into the other U/q buffer.
__global__ void k_update(DevCloud d, double *U_next, double *q_next) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const int cls = d.cls[i];
    Frame F;
    load_frame(d.frame + 9 * (size_t)i, F);
    double U[5], dn[5], p[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) dn[r] = d.dUn[5 * (size_t)i + r];
    double res = 0.0;
    const bool expl = d.update_variant == MFCFD_UPDATE_EXPLICIT;
    if (cls == CLS_WALL || cls == CLS_INTERIOR) {
        const double temp = d.U[5 * (size_t)i];
#pragma unroll
        for (int r = 0; r < 5; ++r) U[r] = d.U[5 * (size_t)i + r] + dn[r];
        if (expl && cls == CLS_WALL) U[3] = 0.0;   // state_update.f90:37
        res = (U[0] - temp) * (U[0] - temp);
        conserved_to_primitive(U, F, p);
    } else if (cls == CLS_OUTER) {
        double pc[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) pc[r] = d.prim[5 * (size_t)i + r];
        conserved_vector_Ubar(pc, F, d.rho_inf, d.u1_inf, d.u2_inf, d.u3_inf, d.pr_inf, U);
        if (expl) {   // state_update.f90:55-58
            const double dt = d.delt[i];
#pragma unroll
            for (int r = 0; r < 5; ++r) U[r] = U[r] - dt * d.flux_res[5 * (size_t)i + r];
        } else {
#pragma unroll
            for (int r = 0; r < 5; ++r) U[r] = U[r] + dn[r];
        }
        conserved_to_primitive(U, F, p);
    } else {
#pragma unroll
        for (int r = 0; r < 5; ++r) p[r] = d.prim[5 * (size_t)i + r];
    }
    d.res_sqr[i] = res;
    double Un[5], qn[5];
    primitive_to_rotated_conserved(p, F, Un);
    primitive_to_q(p, qn);
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        d.prim[5 * (size_t)i + r] = p[r];
        d.dUp[5 * (size_t)i + r] = dn[r];
        U_next[5 * (size_t)i + r] = Un[r];
        q_next[5 * (size_t)i + r] = qn[r];
    }
}

// Supersonic points after the state update (state_update_implicit.f90:
// 63-94): outlets, then inlets, each in index order, take the new state of
// their nearest non-wall neighbour.  One thread, in that order, since a
// source may be a supersonic point copied just before; then their next U
// and q.
__global__ void k_update_ss(DevCloud d, double *U_next, double *q_next) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int j = 0; j < d.n_ss; ++j) {
        const int k = d.ss_pts[j], src = d.ss_src[j];
        double p[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            p[r] = src >= 0 ? d.prim[5 * (size_t)src + r] : 0.0;
            d.prim[5 * (size_t)k + r] = p[r];
        }
        Frame F;
        load_frame(d.frame + 9 * (size_t)k, F);
        double Un[5], qn[5];
        primitive_to_rotated_conserved(p, F, Un);
        primitive_to_q(p, qn);
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            U_next[5 * (size_t)k + r] = Un[r];
            q_next[5 * (size_t)k + r] = qn[r];
        }
    }
}

// res_new = sqrt(sum over wall, interior of (dU1)^2) / N
// (state_update_implicit.f90:124-129, 187).  Fixed two-pass tree order, so
// the value is deterministic; it differs from the reference's left-to-right
// sum only by summation rounding.
__global__ void k_reduce_partial(DevCloud d) {
    __shared__ double s[RED_THREADS];
    const int per = (d.n_res + gridDim.x - 1) / gridDim.x;
    const int a = blockIdx.x * per, b = min(d.n_res, a + per);
    double acc = 0.0;
    for (int j = a + threadIdx.x; j < b; j += RED_THREADS) acc += d.res_sqr[d.res_order[j]];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) d.partial[blockIdx.x] = s[0];
}

__global__ void k_reduce_final(DevCloud d, int nblocks, int slot) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double acc = 0.0;
    for (int b = 0; b < nblocks; ++b) acc += d.partial[b];
    d.res_dev[slot] = sqrt(acc) / (double)d.n;
}

// ---------------------------------------------------------------- forces

// F = -sum over wall points of (p_i - p_inf) A_i nor_i, one block: thread t
// sums the wall points t, t + 256, ... in index order, then a fixed tree;
// A_i from area (per point) or area_each.  out[0..2] = F.
__global__ void __launch_bounds__(RED_THREADS) k_forces(DevCloud d, double area_each, const double *area,
                                                          double *out) {
    __shared__ double s[3][RED_THREADS];
    double f[3] = {0.0, 0.0, 0.0};
    for (int j = threadIdx.x; j < d.n_wall; j += RED_THREADS) {
        const int i = d.res_order[j];          // wall points first, index order
        const double a = area ? area[i] : area_each;
        const double dp = d.prim[5 * (size_t)i + 4] - d.pr_inf;
#pragma unroll
        for (int r = 0; r < 3; ++r) f[r] = f[r] - dp * a * d.frame[9 * (size_t)i + 6 + r];
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) s[r][threadIdx.x] = f[r];
    __syncthreads();
    for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
#pragma unroll
            for (int r = 0; r < 3; ++r) s[r][threadIdx.x] += s[r][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 3) out[threadIdx.x] = s[threadIdx.x][0];
}

cudaError_t launch_forces(const DevCloud &d, cudaStream_t s, double area_each, const double *area, double *out) {
    k_forces<<<1, RED_THREADS, 0, s>>>(d, area_each, area, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- launchers

int device_sms(int device) {
    static std::mutex mu;
    static int cache[256] = {0};
    if (device < 0 || device >= 256) return 1;
    std::lock_guard<std::mutex> lock(mu);
    if (!cache[device]) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms < 1) {
            (void)cudaGetLastError();
            sms = 1;
        }
        cache[device] = sms;
    }
    return cache[device];
}

// Mixed precision (MIXED, MIXED_DC): each sweep term's weight with its list's
// 3x3 least-squares solve folded in.  The list's derivative is num(axis,
// moments, sum w_j t_j) / det, linear in the sums, so every term gets one
// weight (cofactors . w_j) / det, in FP64, and the sweep sums w_j t_j
// directly.  fold: the three weights are saved first when `saved` is given
// (3 per term), then replaced; !fold: put back from `saved`.
__global__ void k_fold_terms(DevCloud d, int dir, double *saved, int fold) {
    const int *off = dir == 0 ? d.fwd_off : d.bwd_off;
    SweepEntry *ent = const_cast<SweepEntry *>(dir == 0 ? d.fwd_ent : d.bwd_ent);
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < d.n; p += gridDim.x * blockDim.x) {
        for (int e = off[p]; e < off[p + 1]; ++e) {
            SweepEntry &E = ent[e];
            if (E.pad & ENT_COPY) continue;
            if (!fold) {
                E.w[0] = saved[3 * (size_t)e];
                E.w[1] = saved[3 * (size_t)e + 1];
                E.w[2] = saved[3 * (size_t)e + 2];
                continue;
            }
            if (saved) {
                saved[3 * (size_t)e] = E.w[0];
                saved[3 * (size_t)e + 1] = E.w[1];
                saved[3 * (size_t)e + 2] = E.w[2];
            }
            const int dd = E.pad & 255;
            const bool outer_zp = d.sweep_variant == MFCFD_SWEEPS_BACKUP && d.cls[p] == CLS_OUTER && dd == 4;
            const double *g = d.geo + (size_t)p * GEO_STRIDE + (outer_zp ? 5 : dd) * 8;
            const double xx = g[G_XX], yy = g[G_YY], zz = g[G_ZZ], xy = g[G_XY], yz = g[G_YZ], zx = g[G_ZX];
            double a, b, c;
            if (dd / 2 == 0) { a = yy * zz - yz * yz; b = -(xy * zz - zx * yz); c = xy * yz - zx * yy; }
            else if (dd / 2 == 1) { a = -(xy * zz - zx * yz); b = xx * zz - zx * zx; c = -(xx * yz - xy * zx); }
            else { a = xy * yz - zx * yy; b = -(xx * yz - zx * xy); c = xx * yy - xy * xy; }
            const double w = (a * E.w[0] + b * E.w[1] + c * E.w[2]) / g[G_DET];
            E.w[0] = w;
            E.w[1] = 0.0;
            E.w[2] = 0.0;
        }
    }
}

cudaError_t launch_fold_terms(const DevCloud &d, double *const saved[2], bool fold, cudaStream_t s) {
    const int grid = (d.n + 255) / 256;
    for (int dir = 0; dir < 2; ++dir) k_fold_terms<<<grid, 256, 0, s>>>(d, dir, saved[dir], fold ? 1 : 0);
    return cudaGetLastError();
}

int reduction_blocks(int n) {
    int b = (n + 4095) / 4096;
    return b < 1 ? 1 : (b > 1024 ? 1024 : b);
}

// ---------------------------------------------------------------- allocation-free residual

// Scratch of mfcfd_residual_noalloc: one partial sum per reduction block plus
// the result slot.  A file-scope device array, so that entry point never
// allocates; 8 KB that every GPU loading the library holds until exit.
constexpr int NOALLOC_BLOCKS = MFCFD_NOALLOC_MAX_TERMS / 4096;
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_BLOCKS + 1];

// Device address of g_noalloc_scratch, looked up once per device.  In host
// code the symbol names a host-side stand-in, not device memory, so kernels
// must be given this address instead.
static std::mutex g_noalloc_mu;
static double *g_noalloc_ptr[256] = {nullptr};

int residual_noalloc(const DevCloud &d, cudaStream_t s, double *res_new, std::string &err) {
    if (d.n_res > MFCFD_NOALLOC_MAX_TERMS) {
        err = "mfcfd_residual_noalloc handles at most " + std::to_string(MFCFD_NOALLOC_MAX_TERMS) +
              " residual terms; this cloud has " + std::to_string(d.n_res);
        return MFCFD_ERR_UNSUPPORTED;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 256) {
        err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return MFCFD_ERR_CUDA;
    }
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) {
                err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
                return MFCFD_ERR_CUDA;
            }
            g_noalloc_ptr[dev] = static_cast<double *>(p);
        }
        scratch = g_noalloc_ptr[dev];
    }
    // Same partition as the iteration's own reduction (4096 terms a block),
    // so the value is the one mfcfd_fpi_step returned.  Every partial that
    // k_reduce_final reads is written first, so nothing needs clearing.
    int blocks = (d.n_res + 4095) / 4096;
    if (blocks < 1) blocks = 1;
    DevCloud dc = d;
    dc.partial = scratch;
    dc.res_dev = scratch + NOALLOC_BLOCKS;
    k_reduce_partial<<<blocks, RED_THREADS, 0, s>>>(dc);
    k_reduce_final<<<1, 32, 0, s>>>(dc, blocks, 0);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(res_new, scratch + NOALLOC_BLOCKS, sizeof(double),
                                              cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        err = std::string("residual_noalloc: ") + cudaGetErrorString(e);
        return MFCFD_ERR_CUDA;
    }
    return MFCFD_OK;
}

// Sets the kernels' shared-memory limits once per device.
static void set_attributes(int device) {
    static std::mutex mu;
    static bool done[256] = {false};
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0 || device >= 256 || done[device]) return;
    cudaFuncSetAttribute(k_flux<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         FLUX_WARPS * FLUX_SMEM_PER_WARP * 8);
    cudaFuncSetAttribute(k_flux<true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         FLUX_WARPS * FLUX_SMEM_PER_WARP * 8);
    cudaFuncSetAttribute(k_flux<true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         FLUX_WARPS * FLUX_SMEM_PER_WARP * 8);
    cudaFuncSetAttribute(k_flux<true, double, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         FLUX_WARPS * FLUX_SMEM_PER_WARP * 8);
    cudaFuncSetAttribute(k_sweep_levels, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         SWEEP_WARPS * SWEEP_SMEM_BYTES);
    cudaFuncSetAttribute(k_sweep_df, cudaFuncAttributeMaxDynamicSharedMemorySize, DF_WARPS * SWEEP_SMEM_BYTES);
    // three 4-warp blocks of the mixed-precision sweep per SM need the largest
    // shared-memory carveout; the other variants leave the choice to the
    // driver, which keeps more L1 for their loads and the flux kernel's
    cudaFuncSetAttribute(k_sweep_chain<4, float, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    cudaFuncSetAttribute(k_sweep_chain<4, double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, CHAIN_SPREAD_SMEM);
    cudaFuncSetAttribute(k_sweep_chain<8, double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, chain_smem<8>());
    cudaFuncSetAttribute(k_sweep_chain<4, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, CHAIN_SPREAD_SMEM);
    cudaFuncSetAttribute(k_sweep_chain<8, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, chain_smem<8>());
    cudaFuncSetAttribute(k_sweep_chain_group<4, float, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    cudaFuncSetAttribute(k_sweep_chain_group<4, double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         CHAIN_SPREAD_SMEM);
    cudaFuncSetAttribute(k_sweep_chain_group<8, double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         chain_smem<8>());
    cudaFuncSetAttribute(k_sweep_chain_group<4, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         CHAIN_SPREAD_SMEM);
    cudaFuncSetAttribute(k_sweep_chain_group<8, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         chain_smem<8>());
    done[device] = true;
}

void prepare_launches(int device) { set_attributes(device); }

int chain_slot_capacity(int device) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return 6 * (sms - CH_FREE_SMS);
}

int chain_block_slots(int device, int wpb, int precision, int spread) {
    static std::mutex mu;
    static int cache[256][2][3] = {};
    if (device < 0 || device >= 256 || spread) return 6;
    const int w8 = wpb == 8 ? 1 : 0, m = precision < 0 || precision > 2 ? 0 : precision;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (cache[device][w8][m]) return cache[device][w8][m];
    }
    set_attributes(device);
    int per_sm = 0;
    cudaError_t e;
    if (w8)
        e = m != 0 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_chain<8, float, true>, 256, chain_smem<8>())
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_chain<8, double, false>, 256, chain_smem<8>());
    else
        e = m != 0 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_chain<4, float, true>, 128, chain_smem<4>())
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_chain<4, double, false>, 128, chain_smem<4>());
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        per_sm = 1;
    }
    per_sm = per_sm < 1 ? 1 : (per_sm > 3 ? 3 : per_sm);
    std::lock_guard<std::mutex> lock(mu);
    return cache[device][w8][m] = 6 / per_sm;
}

bool chain_group_fits(int device, int wpb, int precision, int spread) {
    set_attributes(device);
    const bool mixed = precision != MFCFD_PRECISION_FP64;
    const int smem = chain_smem_bytes(wpb, spread);
    int one = 0, group = 0;
    cudaError_t e1, e2;
    if (wpb == 8) {
        e1 = mixed ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&one, k_sweep_chain<8, float, true>, 256, smem)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&one, k_sweep_chain<8, double, false>, 256, smem);
        e2 = mixed ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&group, k_sweep_chain_group<8, float, true>, 256, smem)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&group, k_sweep_chain_group<8, double, false>, 256,
                                                                   smem);
    } else {
        e1 = mixed ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&one, k_sweep_chain<4, float, true>, 128, smem)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&one, k_sweep_chain<4, double, false>, 128, smem);
        e2 = mixed ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&group, k_sweep_chain_group<4, float, true>, 128, smem)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&group, k_sweep_chain_group<4, double, false>, 128,
                                                                   smem);
    }
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return group >= 1 && group >= one;
}

int chain_shape(int device, int want, int spread, int *wpb, int *blocks) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    set_attributes(device);
    const int max_blocks = sms - CH_FREE_SMS;
    if (max_blocks < 1) return 0;
    if (spread) {
        // 4-warp blocks, one per SM
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_chain<4, double, false>, 4 * 32, CHAIN_SPREAD_SMEM);
        if (per_sm < 1) return 0;
        *wpb = 4;
        int b = (want + 3) / 4;
        b = b > max_blocks ? max_blocks : (b < 1 ? 1 : b);
        *blocks = b;
        return 4 * b;
    }
    *wpb = want <= 4 * max_blocks ? 4 : 8;
    // with 8-warp blocks, three quarters of the warps: more SMs stay with the
    // concurrent flux kernel, which then keeps ahead of the forward sweep
    if (*wpb == 8) want = want * 3 / 4;
    int per_sm = 0;
    if (*wpb == 4)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_chain<4, double, false>, 4 * 32, chain_smem<4>());
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_chain<8, double, false>, 8 * 32, chain_smem<8>());
    if (per_sm < 1) return 0;
    int b = (want + *wpb - 1) / *wpb;
    if (b > max_blocks) b = max_blocks;
    if (b < 1) b = 1;
    *blocks = b;
    // fewer warps than one block asked for (a single-warp chain measures the
    // per-point latency floor): the block's other warps exit at once
    return want < *wpb ? (want < 1 ? 1 : want) : b * *wpb;
}

// Rows [a, a + rows) of width w between the reference's index order and
// the storage order: scatter puts row i of src (a transfer buffer in index
// order) at storage row perm[a + i] of dst; gather does the reverse.
__global__ void k_rows(const double *src, double *dst, const int32_t *perm, int a, int rows, int w, int scatter) {
    const size_t total = (size_t)rows * w;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t i = t / w, c = t - i * w;
        const size_t s = (size_t)perm[a + i];
        if (scatter) dst[s * w + c] = src[t];
        else dst[t] = src[s * w + c];
    }
}

cudaError_t launch_rows(const double *src, double *dst, const int32_t *perm, int a, int rows, int w, bool scatter,
                        cudaStream_t s) {
    const size_t total = (size_t)rows * w;
    int dev = 0;
    cudaGetDevice(&dev);
    size_t blocks = (total + 255) / 256;
    const size_t cap = (size_t)device_sms(dev) * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    k_rows<<<(int)blocks, 256, 0, s>>>(src, dst, perm, a, rows, w, scatter ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_conserved_q(const DevCloud &d, cudaStream_t s) {
    k_conserved_q<<<(d.n + 127) / 128, 128, 0, s>>>(d);
    return cudaGetLastError();
}

// A launch with an explicit scheduling priority.  The chain sweep must have
// its blocks placed before those of the flux kernel beside it (which never
// waits, so it cannot hold the sweep up for good); the priority travels with
// the launch, so it holds in a captured graph as on a stream.
template <typename... Args, typename... Act>
static cudaError_t launch_prio(void (*kern)(Args...), int grid, int block, size_t smem, cudaStream_t s, bool high,
                               Act &&...args) {
    // least and greatest priority, looked up once (thread-safe initialisation:
    // group runs may launch from several host threads)
    static const std::pair<int, int> prio = [] {
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        return std::make_pair(lo, hi);
    }();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = high ? prio.second : prio.first;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Act>(args)...);
}

cudaError_t launch_chain_group(const ChainGroup &g, int wpb, int precision, int spread, int forward,
                               cudaStream_t s) {
    const int blocks = g.block_start[g.count];
    const int csm = chain_smem_bytes(wpb, spread);
    if (precision != MFCFD_PRECISION_FP64) {
        if (wpb == 4) return launch_prio(k_sweep_chain_group<4, float, true>, blocks, 4 * 32, csm, s, true, g, forward);
        return launch_prio(k_sweep_chain_group<8, float, true>, blocks, 8 * 32, csm, s, true, g, forward);
    }
    if (wpb == 4) return launch_prio(k_sweep_chain_group<4, double, false>, blocks, 4 * 32, csm, s, true, g, forward);
    return launch_prio(k_sweep_chain_group<8, double, false>, blocks, 8 * 32, csm, s, true, g, forward);
}

cudaError_t launch_iteration(const DevCloud &d, int iter_slot, const IterStreams &st, double *U_next,
                             double *q_next, cudaEvent_t *ev, IterPart part) {
    const int n = d.n;
    cudaStream_t s = st.main;
    int dev = 0;
    cudaGetDevice(&dev);
    set_attributes(dev);
    // dataflow grid: about the widest level in warps (more warps only add
    // pollers), within 8 per SM
    const int sms = device_sms(dev);
    int df_warps = d.max_width;
    df_warps = df_warps < 64 ? 64 : (df_warps > sms * 8 ? sms * 8 : df_warps);
    const int df_blocks = (df_warps + DF_WARPS - 1) / DF_WARPS;
    const bool chains = d.sweep_mode == MFCFD_SWEEP_CHAINS;
    const bool mixed = d.precision != MFCFD_PRECISION_FP64;    // FP32 sweeps; chain schedule only
    const bool dc = d.precision == MFCFD_PRECISION_MIXED_DC;   // ... with the FP64 flux residual
    auto sweep = [&](int forward) {
        if (chains) {
            const int blocks = (d.ch_warps + d.ch_wpb - 1) / d.ch_wpb;
            const int csm = chain_smem_bytes(d.ch_wpb, d.ch_spread);
            if (mixed) {   // MIXED and MIXED_DC: folded weights
                if (d.ch_wpb == 4) launch_prio(k_sweep_chain<4, float, true>, blocks, 4 * 32, csm, s, true, d, forward);
                else launch_prio(k_sweep_chain<8, float, true>, blocks, 8 * 32, csm, s, true, d, forward);
            } else {
                if (d.ch_wpb == 4) launch_prio(k_sweep_chain<4, double, false>, blocks, 4 * 32, csm, s, true, d, forward);
                else launch_prio(k_sweep_chain<8, double, false>, blocks, 8 * 32, csm, s, true, d, forward);
            }
        } else if (d.sweep_mode == MFCFD_SWEEP_LEVELS) {
            k_sweep_levels<<<1, SWEEP_THREADS, SWEEP_WARPS * SWEEP_SMEM_BYTES, s>>>(d, forward);
        } else {
            cudaMemsetAsync(d.sweep_counter + (forward ? 0 : 1), 0, sizeof(int), s);
            k_sweep_df<<<df_blocks, DF_WARPS * 32, DF_WARPS * SWEEP_SMEM_BYTES, s>>>(d, forward);
        }
    };
    auto mark = [&](int i, cudaStream_t on) { if (ev) cudaEventRecord(ev[i], on); };
    const int fblocks = (n + FLUX_WARPS - 1) / FLUX_WARPS;
    if (part != ITER_ALL && !chains) return cudaErrorInvalidValue;
    if (part == ITER_POST) goto post;
    mark(0, s);
    // supersonic copies may read a neighbour's increment from before the
    // sweeps, which k_pending is about to mark
    if (d.dU_old) cudaMemcpyAsync(d.dU_old, d.dUn, sizeof(double) * 5 * (size_t)n, cudaMemcpyDeviceToDevice, s);
    k_qderiv<<<(n + 127) / 128, 128, 0, s>>>(d);
    for (int j = 0; j < d.inner_iterations; ++j) {
        k_qinner<<<(n + 127) / 128, 128, 0, s>>>(d, d.dq, d.dq_tmp);
        cudaMemcpyAsync(d.dq, d.dq_tmp, sizeof(double) * 15 * (size_t)n, cudaMemcpyDeviceToDevice, s);
    }
    mark(1, s);
    if (chains && d.n_g0 > 0) {
        // phase A of the points outside the shared frame, for both sweeps
        const int gb = (int)(((size_t)d.n_g0 * 32 + 127) / 128);
        if (mixed) k_g0<float><<<gb, 128, 0, s>>>(d);
        else k_g0<double><<<gb, 128, 0, s>>>(d);
    }
    if (chains) {
        // the flux residual and the sweep inputs run on the side stream beside
        // the forward sweep, in its order; the sweep polls for them.  The flux
        // kernel is issued first: where kernels run one at a time (a profiler,
        // blocking launches) it completes before the sweep starts, and it
        // never waits on the sweep, so no order of execution can stall.  The
        // main stream's higher priority places the sweep's blocks first when
        // both run.
        k_pending<<<sms * 8, 256, 0, s>>>(d, 1);
        mark(3, s);
        const size_t fsm = FLUX_WARPS * FLUX_SMEM_PER_WARP * 8;
        auto flux = [&](int i0, int i1, int grid, cudaStream_t on, bool high) {
            if (dc) launch_prio(k_flux<true, double, float>, grid, FLUX_WARPS * 32, fsm, on, high, d, i0, i1);
            else if (mixed) launch_prio(k_flux<true, float>, grid, FLUX_WARPS * 32, fsm, on, high, d, i0, i1);
            else launch_prio(k_flux<true, double>, grid, FLUX_WARPS * 32, fsm, on, high, d, i0, i1);
        };
        cudaEventRecord(st.fork, s);
        cudaStreamWaitEvent(st.side, st.fork, 0);
        // a smaller grid walks the same order with its warps striding through it
        const int fgrid = d.flux_grid > 0 && d.flux_grid < fblocks ? d.flux_grid : fblocks;
        flux(0, n, fgrid, st.side, false);
        mark(2, st.side);
        cudaEventRecord(st.join, st.side);
        if (part == ITER_PRE) return cudaGetLastError();
        sweep(1);
        mark(4, s);
        cudaStreamWaitEvent(s, st.join, 0);
    } else {
        k_flux<false, double><<<fblocks, FLUX_WARPS * 32, FLUX_WARPS * FLUX_SMEM_PER_WARP * 8, s>>>(d, 0, n);
        mark(2, s);
        k_pending<<<sms * 8, 256, 0, s>>>(d, 0);
        k_dinv_gold<<<(n + 127) / 128, 128, 0, s>>>(d);
        mark(3, s);
        sweep(1);
        mark(4, s);
    }
    sweep(0);
    mark(5, s);
post:
    k_update<<<(n + 127) / 128, 128, 0, s>>>(d, U_next, q_next);
    if (d.n_ss > 0) k_update_ss<<<1, 32, 0, s>>>(d, U_next, q_next);
    mark(6, s);
    const int rb = reduction_blocks(d.n_res);
    k_reduce_partial<<<rb, RED_THREADS, 0, s>>>(d);
    k_reduce_final<<<1, 32, 0, s>>>(d, rb, iter_slot);
    mark(7, s);
    return cudaGetLastError();
}

}  // namespace mfcfd
