// Device-side Euler physics of the explicit path: primitive conversion,
// physical flux, slope limiters, MUSCL-Hancock cell stage, and the HLLC /
// FORCE / Lax-Friedrichs face stages.  Each function follows the reference
// routine cited beside it in operation order, except that a reciprocal of
// the density (or of epsilon) is reused where the reference divides several
// times by the same value, and that the gamma powers of the Toro wave-speed
// estimate use a Newton-refined integer root when 1/z is an integer.  Both
// change results by a few units in the last place (parity bound: 1e-12
// relative L-infinity per step).
#pragma once

#include <cmath>

#include "common.cuh"

namespace bamrex {

enum { LIM_MINBEE = 0, LIM_VAN_LEER = 1, LIM_VAN_ALBADA = 2, LIM_SUPERBEE = 3 };
enum { M_MUSCL = 0, M_HLLC = 1, M_SLIC = 4, M_FORCE = 5, M_LF = 6 };

// Minimum density / pressure of the wave-speed estimate (HLLC.H:255-260).
constexpr double kMinRho = 1e-14;
constexpr double kMinP = 1e-14;

// a[idx] for a runtime idx without local-memory indexing.
template <int N>
__device__ __forceinline__ double sel(const double (&a)[N], int idx)
{
    double r = a[0];
#pragma unroll
    for (int m = 1; m < N; ++m) r = (idx == m) ? a[m] : r;
    return r;
}

// primv_from_consv (Source/System/Euler/Euler.H:167-198); inv_rho = 1/rho.
template <int D>
__device__ __forceinline__ void to_prim(const double (&U)[D + 2], const Consts& k, double (&q)[D + 2],
                                        double& inv_rho)
{
    inv_rho = 1.0 / U[0];
    q[0] = U[0];
#pragma unroll
    for (int d = 0; d < D; ++d) q[1 + d] = U[1 + d] * inv_rho;
    double usq = q[1] * q[1];
#pragma unroll
    for (int d = 1; d < D; ++d) usq = usq + q[1 + d] * q[1 + d];
    q[1 + D] = k.gm1 * (U[1 + D] - 0.5 * k.eps * U[0] * usq);
}

// euler_flux<dir> / compute_flux_function<dir> (Euler.H:211-244, Euler.cpp:10-44).
template <int D, int DIR>
__device__ __forceinline__ void phys_flux(const double (&U)[D + 2], const double (&q)[D + 2], const Consts& k,
                                          double (&F)[D + 2])
{
    const double mn = U[1 + DIR];
    F[0] = mn;
#pragma unroll
    for (int d = 0; d < D; ++d) F[1 + d] = mn * q[1 + d];
    F[1 + DIR] += q[1 + D] * k.inv_eps;
    F[1 + D] = (U[1 + D] + q[1 + D]) * q[1 + DIR];
}

template <int D, int DIR>
__device__ __forceinline__ void phys_flux(const double (&U)[D + 2], const Consts& k, double (&F)[D + 2])
{
    double q[D + 2], ir;
    to_prim<D>(U, k, q, ir);
    phys_flux<D, DIR>(U, q, k, F);
}

// slope_limit<L> (Source/Fluxes/Limiters.H:29-73).
__device__ __forceinline__ double slope_limit(int lim, double r)
{
    if (r <= 0) return 0.0;
    switch (lim) {
    case LIM_MINBEE: return r > 1 ? fmin(2. / (1 + r), 1.) : r;
    case LIM_VAN_LEER: {
        const double ip = 1. / (1 + r);
        return fmin(2. * r * ip, 2. * ip);
    }
    case LIM_VAN_ALBADA: return fmin(r * (1 + r) / (1 + r * r), 2. / (1 + r));
    default: return (r <= 0.5) ? 2 * r : ((r <= 1) ? 1. : fmin(r, fmin(2. / (1 + r), 2.)));
    }
}

// The limiter value from the limiting-variable differences
// (Source/Fluxes/Flux_Helpers.cpp:103-111).
__device__ __forceinline__ double limiter_value(int lim, double numerator, double denom)
{
    if (numerator == 0. && denom == 0.) return slope_limit(lim, 1.0);
    if (denom == 0) return 0.0;
    return slope_limit(lim, numerator / denom);
}

// ---- fast gamma powers --------------------------------------------------
__device__ __forceinline__ double ipow_k(double y, int k)
{
    if (k == 7) {
        const double y2 = y * y, y3 = y2 * y, y6 = y3 * y3;
        return y6 * y;
    }
    if (k == 5) {
        const double y2 = y * y, y4 = y2 * y2;
        return y4 * y;
    }
    double r = y;
    for (int i = 1; i < k; ++i) r *= y;
    return r;
}

// x^(-z) for the clamped pressure x >= 1e-14 (HLLC.H:272).  With 1/z ~ k,
// x^(-1/k) comes from a float seed and two Newton steps of
// y <- y + y (1 - x y^k) / k, then x^(1/k - z) ~ 1 + (1/k - z) ln x.
__device__ __forceinline__ double pow_neg_z(double x, const Consts& c)
{
    if (c.root_k == 0 || !(x > 1e-30 && x < 1e30)) return pow(x, c.neg_z);
    const int k = c.root_k;
    const float lf = __log2f((float)x);
    double y = (double)exp2f(-lf / (float)k);
    const double ik = 1.0 / (double)k;
#pragma unroll
    for (int it = 0; it < 2; ++it) {
        const double e = fma(-x, ipow_k(y, k), 1.0);
        y = fma(y * e, ik, y);
    }
    return fma(y, c.root_dneg * (double)(lf * 0.69314718f), y);
}

// b^(1/z) (HLLC.H:270-273): b^k (1 + (1/z - k) ln b); non-positive or
// extreme b goes to pow() (a negative base gives NaN there, as in the
// reference, which then selects q_K = 1).
__device__ __forceinline__ double pow_inv_z(double b, const Consts& c)
{
    if (c.root_k == 0 || !(b > 1e-30 && b < 1e30)) return pow(b, c.inv_z);
    const double bk = ipow_k(b, c.root_k);
    return fma(bk, c.root_dpos * (double)(__log2f((float)b) * 0.69314718f), bk);
}

// ---- cell stage: reconstruct_and_half_time_step<limiter,dir> --------------
// (Source/Fluxes/Flux_Helpers.cpp:92-148) for one cell from its two
// neighbours along the sweep: returns the half-stepped L/R states.
template <int D, int DIR>
__device__ __forceinline__ void muscl_cell(const double (&Um)[D + 2], const double (&U0)[D + 2],
                                           const double (&Up)[D + 2], const Consts& k, double hdtdx,
                                           double (&UL)[D + 2], double (&UR)[D + 2])
{
    constexpr int NC = D + 2;
    double hphi[NC];
    if (k.uniform_var >= 0) {
        const int v = k.uniform_var;
        const double vL = sel(Um, v), vC = sel(U0, v), vR = sel(Up, v);
        const double lim = limiter_value(k.limiter, vC - vL, vR - vC);
#pragma unroll
        for (int n = 0; n < NC; ++n) hphi[n] = 0.5 * lim;
    } else {
        double Qm[NC], Q0[NC], Qp[NC], ir;
        if (k.need_prim) {
            to_prim<D>(Um, k, Qm, ir);
            to_prim<D>(U0, k, Q0, ir);
            to_prim<D>(Up, k, Qp, ir);
        } else {
#pragma unroll
            for (int n = 0; n < NC; ++n) Qm[n] = Q0[n] = Qp[n] = 0.0;
        }
#pragma unroll
        for (int n = 0; n < NC; ++n) {
            const int v = k.lim_var[n];
            const bool pr = k.lim_prim[n] != 0;
            const double vL = pr ? sel(Qm, v) : sel(Um, v);
            const double vC = pr ? sel(Q0, v) : sel(U0, v);
            const double vR = pr ? sel(Qp, v) : sel(Up, v);
            hphi[n] = 0.5 * limiter_value(k.limiter, vC - vL, vR - vC);
        }
    }
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        const double delta = 0.5 * (U0[n] - Um[n]) + 0.5 * (Up[n] - U0[n]);
        UL[n] = U0[n] - hphi[n] * delta;
        UR[n] = U0[n] + hphi[n] * delta;
    }
    double FL[NC], FR[NC];
    phys_flux<D, DIR>(UL, k, FL);
    phys_flux<D, DIR>(UR, k, FR);
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        const double dF = hdtdx * (FR[n] - FL[n]);
        UL[n] -= dF;
        UR[n] -= dF;
    }
}

// ---- face stage: HLLC (Source/Fluxes/HLLC.cpp:90-172 with
// estimate_wave_speed_HLLC_Toro, HLLC.H:214-309, and
// HLLC_interm_state_replace, HLLC.H:311-337).  L is the state left of the
// face, R the state right of it.
template <int D, int DIR>
__device__ __forceinline__ void hllc_face(const double (&L)[D + 2], const double (&R)[D + 2], const Consts& k,
                                          double (&F)[D + 2])
{
    constexpr int NC = D + 2;
    double qL[NC], qR[NC], irL, irR;
    to_prim<D>(L, k, qL, irL);
    to_prim<D>(R, k, qR, irR);
    const double rhoL = fmax(qL[0], kMinRho), rhoR = fmax(qR[0], kMinRho);
    const double pL = fmax(qL[1 + D], kMinP), pR = fmax(qR[1 + D], kMinP);
    const double uL = qL[1 + DIR], uR = qR[1 + DIR];
    const double icL = (qL[0] >= kMinRho) ? irL : 1.0 / kMinRho;
    const double icR = (qR[0] >= kMinRho) ? irR : 1.0 / kMinRho;
    const double cL = sqrt(k.gamma_inv_eps * pL * icL);
    const double cR = sqrt(k.gamma_inv_eps * pR * icR);
    const double base = (cL + cR - k.half_gm1 * (uR - uL)) / (cL * pow_neg_z(pL, k) + cR * pow_neg_z(pR, k));
    const double p_rr = pow_inv_z(base, k);
    const double qwL = (p_rr > pL) ? sqrt(1 + k.gp1_2g * (p_rr / pL - 1)) : 1.0;
    const double qwR = (p_rr > pR) ? sqrt(1 + k.gp1_2g * (p_rr / pR - 1)) : 1.0;
    const double SL = uL - cL * qwL;
    const double SR = uR + cR * qwR;
    const double dL = SL - uL, dR = SR - uR;
    const double denom = rhoL * dL - rhoR * dR;
    const double Ss = (denom != 0) ? ((pR - pL) * k.inv_eps + rhoL * uL * dL - rhoR * uR * dR) / denom : 0.0;

    // Branches of HLLC.cpp:101-167: the left states serve when S_L >= 0 or
    // S* >= 0; the star correction applies unless the face is supersonic.
    const bool useL = (SL >= 0.0) || (Ss >= 0.0);
    const bool star = useL ? (SL < 0.0) : (SR >= 0.0);
    double UK[NC], qK[NC];
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        UK[n] = useL ? L[n] : R[n];
        qK[n] = useL ? qL[n] : qR[n];
    }
    const double irK = useL ? irL : irR;
    const double SK = useL ? SL : SR;
    phys_flux<D, DIR>(UK, qK, k, F);
    if (star) {
        const double rhoK = qK[0], uK = qK[1 + DIR], pK = qK[1 + D];
        const double dK = SK - uK;
        const double scale = rhoK * dK / (SK - Ss);
        const double eterm = UK[1 + D] * irK + (Ss - uK) * (Ss * k.eps + pK / (rhoK * dK));
        F[0] = F[0] + SK * (scale - UK[0]);
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const double s = (d == DIR) ? Ss : qK[1 + d];
            F[1 + d] = F[1 + d] + SK * (s * scale - UK[1 + d]);
        }
        F[1 + D] = F[1 + D] + SK * (eterm * scale - UK[1 + D]);
    }
}

// ---- face stage: FORCE (compute_force_flux_LR, Source/Fluxes/Force.cpp:22-108)
template <int D, int DIR>
__device__ __forceinline__ void force_face(const double (&L)[D + 2], const double (&R)[D + 2], const Consts& k,
                                           double half_dx_dt, double dt_2dx, double (&F)[D + 2])
{
    constexpr int NC = D + 2;
    double fL[NC], fR[NC], H[NC], fH[NC];
    phys_flux<D, DIR>(L, k, fL);
    phys_flux<D, DIR>(R, k, fR);
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        F[n] = 0.5 * (half_dx_dt * (L[n] - R[n]) + 0.5 * (fL[n] + fR[n]));
        H[n] = 0.5 * (L[n] + R[n]) + dt_2dx * (fL[n] - fR[n]);
    }
    phys_flux<D, DIR>(H, k, fH);
#pragma unroll
    for (int n = 0; n < NC; ++n) F[n] += 0.5 * fH[n];
}

// ---- face stage: Lax-Friedrichs (compute_LF_flux, Source/Fluxes/Force.cpp:110-151)
template <int D, int DIR>
__device__ __forceinline__ void lf_face(const double (&L)[D + 2], const double (&R)[D + 2], const Consts& k,
                                        double half_dx_dt, double (&F)[D + 2])
{
    constexpr int NC = D + 2;
    double fL[NC], fR[NC];
    phys_flux<D, DIR>(L, k, fL);
    phys_flux<D, DIR>(R, k, fR);
#pragma unroll
    for (int n = 0; n < NC; ++n) F[n] = half_dx_dt * (L[n] - R[n]) + 0.5 * (fL[n] + fR[n]);
}

// |u| + c of a conserved state (max_wave_speed body, Euler.cpp:53-68).
template <int D>
__device__ __forceinline__ double wave_speed(const double (&U)[D + 2], const Consts& k)
{
    double q[D + 2], ir;
    to_prim<D>(U, k, q, ir);
    double vsq = q[1] * q[1];
#pragma unroll
    for (int d = 1; d < D; ++d) vsq = vsq + q[1 + d] * q[1 + d];
    return sqrt(k.gamma_inv_eps * q[1 + D] * ir) + sqrt(vsq);
}

// ======================================================================
// Fast path: MUSCL-Hancock + HLLC with a compile-time limiter, every
// component limited on the energy (the reference default,
// FluidSystem.cpp:65-69), and gamma with 1/z = 7 (gamma = 1.4).  Same
// arithmetic as above but branch-free (selects instead of branches) and with
// Newton-refined reciprocals, so each cell and face is one basic block the
// scheduler can interleave.
// ======================================================================

// 1/x by Newton-Raphson refinement, r <- r + r (1 - x r), applied twice to the
// hardware approximation (PTX rcp.approx.ftz.f64).  Within 1 ulp of the
// correctly rounded quotient for normal, finite x (checked against CUDA's
// division by the GPU parity tests).
__device__ __forceinline__ double rcp_nr(double x)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

// log2|x| in single precision from the exponent bits and the mantissa; valid
// over the whole normal double range (no float overflow).
__device__ __forceinline__ float log2_abs(double x)
{
    const long long bits = __double_as_longlong(x);
    const int ex = (int)((bits >> 52) & 0x7ff) - 1023;
    const double m = __longlong_as_double((bits & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
    return (float)ex + __log2f((float)m);
}

// x^(-z) with 1/z ~ 7 for x >= 1e-14 (HLLC.H:272), and 1/x as a by-product.
// Seed y0 = 2^(-log2(x)/7) in single precision, then one step of the series
// of (1 - e)^(-1/7), e = 1 - x y0^7 (third-order convergence: |e| ~ 1e-7
// leaves ~1e-22), then the factor x^(1/7 - z) ~ 1 + (1/7 - z) ln x.
// 1/x = y0^7 / (1 - e) ~ y0^7 (1 + e + e^2).
__device__ __forceinline__ void root7_neg_z(double x, const Consts& c, double& y, double& inv_x)
{
    const float lf = log2_abs(x);
    const float q = -lf * (1.0f / 7.0f);
    const float qi = floorf(q);
    const double p2 = __longlong_as_double((long long)((int)qi + 1023) << 52);
    const double y0 = p2 * (double)exp2f(q - qi);
    const double y2 = y0 * y0, y3 = y2 * y0, y6 = y3 * y3, y7 = y6 * y0;
    const double e = fma(-x, y7, 1.0);
    const double t = e * fma(e, 8.0 / 98.0, 1.0 / 7.0);
    y = fma(y0, t + c.root_dneg_l2 * (double)lf, y0);
    inv_x = fma(y7, fma(e, e, e), y7);
}

// b^(1/z) with 1/z = 7 + dpos: b^7 (1 + dpos ln b).  A negative base gives a
// negative result (the reference's pow gives NaN there); both make every
// "p_rr > p_K" test false, so the wave speeds agree.
__device__ __forceinline__ double pow7_inv_z(double b, const Consts& c)
{
    const double b2 = b * b, b3 = b2 * b, b6 = b3 * b3, b7 = b6 * b;
    return fma(b7, c.root_dpos_l2 * (double)log2_abs(b), b7);
}

template <int D>
__device__ __forceinline__ void to_prim_fast(const double (&U)[D + 2], const Consts& k, double (&q)[D + 2],
                                             double& inv_rho)
{
    inv_rho = rcp_nr(U[0]);
    q[0] = U[0];
#pragma unroll
    for (int d = 0; d < D; ++d) q[1 + d] = U[1 + d] * inv_rho;
    double usq = q[1] * q[1];
#pragma unroll
    for (int d = 1; d < D; ++d) usq = usq + q[1 + d] * q[1 + d];
    q[1 + D] = k.gm1 * (U[1 + D] - k.half_eps * U[0] * usq);
}

template <int D, int DIR>
__device__ __forceinline__ void phys_flux_fast(const double (&U)[D + 2], const Consts& k, double (&F)[D + 2])
{
    double q[D + 2], ir;
    to_prim_fast<D>(U, k, q, ir);
    phys_flux<D, DIR>(U, q, k, F);
}

// The limiter value of Flux_Helpers.cpp:103-111 and Limiters.H:29-73 without
// branches.
template <int LIM>
__device__ __forceinline__ double limiter_value_fast(double num, double den)
{
    const double r = num * rcp_nr(den);
    double phi;
    if constexpr (LIM == LIM_MINBEE) {
        const double t = fmin(2. * rcp_nr(1 + r), 1.);
        phi = (r > 1) ? t : r;
    } else if constexpr (LIM == LIM_VAN_LEER) {
        const double ip = rcp_nr(1 + r);
        phi = fmin(2. * r * ip, 2. * ip);
    } else if constexpr (LIM == LIM_VAN_ALBADA) {
        phi = fmin(r * (1 + r) * rcp_nr(1 + r * r), 2. * rcp_nr(1 + r));
    } else {
        const double t = fmin(r, fmin(2. * rcp_nr(1 + r), 2.));
        phi = (r <= 0.5) ? 2 * r : ((r <= 1) ? 1. : t);
    }
    phi = (r <= 0) ? 0.0 : phi;
    phi = (den == 0) ? 0.0 : phi;
    return (num == 0. && den == 0.) ? 1.0 : phi;
}

template <int D, int DIR, int LIM>
__device__ __forceinline__ void muscl_cell_fast(const double (&Um)[D + 2], const double (&U0)[D + 2],
                                                const double (&Up)[D + 2], const Consts& k, double hdtdx,
                                                double (&UL)[D + 2], double (&UR)[D + 2])
{
    constexpr int NC = D + 2;
    constexpr int E = D + 1;
    // 0.5 phi delta with delta = 0.5 (U0 - Um) + 0.5 (Up - U0) written as
    // 0.25 phi (Up - Um) (within an ulp of the reference's rounding)
    const double qphi = 0.25 * limiter_value_fast<LIM>(U0[E] - Um[E], Up[E] - U0[E]);
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        const double d2 = Up[n] - Um[n];
        UL[n] = fma(-qphi, d2, U0[n]);
        UR[n] = fma(qphi, d2, U0[n]);
    }
    double FL[NC], FR[NC];
    phys_flux_fast<D, DIR>(UL, k, FL);
    phys_flux_fast<D, DIR>(UR, k, FR);
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        const double dF = hdtdx * (FR[n] - FL[n]);
        UL[n] -= dF;
        UR[n] -= dF;
    }
}

template <int D, int DIR>
__device__ __forceinline__ void hllc_face_fast(const double (&L)[D + 2], const double (&R)[D + 2], const Consts& k,
                                               double (&F)[D + 2])
{
    constexpr int NC = D + 2;
    double qL[NC], qR[NC], irL, irR;
    to_prim_fast<D>(L, k, qL, irL);
    to_prim_fast<D>(R, k, qR, irR);
    const double rhoL = fmax(qL[0], kMinRho), rhoR = fmax(qR[0], kMinRho);
    const double pL = fmax(qL[1 + D], kMinP), pR = fmax(qR[1 + D], kMinP);
    const double uL = qL[1 + DIR], uR = qR[1 + DIR];
    const double icL = (qL[0] >= kMinRho) ? irL : 1.0 / kMinRho;
    const double icR = (qR[0] >= kMinRho) ? irR : 1.0 / kMinRho;
    const double cL = sqrt(k.gamma_inv_eps * pL * icL);
    const double cR = sqrt(k.gamma_inv_eps * pR * icR);
    double yL, yR, ipL, ipR;
    root7_neg_z(pL, k, yL, ipL);
    root7_neg_z(pR, k, yR, ipR);
    const double base = (cL + cR - k.half_gm1 * (uR - uL)) * rcp_nr(cL * yL + cR * yR);
    const double p_rr = pow7_inv_z(base, k);
    const double qwL = (p_rr > pL) ? sqrt(1 + k.gp1_2g * (p_rr * ipL - 1)) : 1.0;
    const double qwR = (p_rr > pR) ? sqrt(1 + k.gp1_2g * (p_rr * ipR - 1)) : 1.0;
    const double SL = uL - cL * qwL;
    const double SR = uR + cR * qwR;
    const double dL = SL - uL, dR = SR - uR;
    const double denom = rhoL * dL - rhoR * dR;
    const double Ss_raw = ((pR - pL) * k.inv_eps + rhoL * uL * dL - rhoR * uR * dR) * rcp_nr(denom);
    const double Ss = (denom != 0) ? Ss_raw : 0.0;

    const bool useL = (SL >= 0.0) || (Ss >= 0.0);
    const bool star = useL ? (SL < 0.0) : (SR >= 0.0);
    double UK[NC], qK[NC];
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        UK[n] = useL ? L[n] : R[n];
        qK[n] = useL ? qL[n] : qR[n];
    }
    const double irK = useL ? irL : irR;
    const double SK = useL ? SL : SR;
    phys_flux<D, DIR>(UK, qK, k, F);
    // star state (HLLC.H:311-337): with m = rho_K (S_K - u_K), b = S_K - S*,
    // scale = m / b = m^2 / (m b) and p_K / m = p_K b / (m b)
    const double rhoK = qK[0], uK = qK[1 + DIR], pK = qK[1 + D];
    const double m = rhoK * (SK - uK);
    const double bq = SK - Ss;
    const double rmb = rcp_nr(m * bq);
    const double scale = m * m * rmb;
    const double eterm = UK[1 + D] * irK + (Ss - uK) * (Ss * k.eps + pK * bq * rmb);
    F[0] = star ? F[0] + SK * (scale - UK[0]) : F[0];
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const double s = (d == DIR) ? Ss : qK[1 + d];
        F[1 + d] = star ? F[1 + d] + SK * (s * scale - UK[1 + d]) : F[1 + d];
    }
    F[1 + D] = star ? F[1 + D] + SK * (eterm * scale - UK[1 + D]) : F[1 + D];
}

template <int D>
__device__ __forceinline__ double wave_speed_fast(const double (&U)[D + 2], const Consts& k)
{
    double q[D + 2], ir;
    to_prim_fast<D>(U, k, q, ir);
    double vsq = q[1] * q[1];
#pragma unroll
    for (int d = 1; d < D; ++d) vsq = vsq + q[1 + d] * q[1 + d];
    return sqrt(k.gamma_inv_eps * q[1 + D] * ir) + sqrt(vsq);
}

// Method dispatch: cell stage (reconstruction + half step for MUSCL-Hancock
// and SLIC; identity for first-order methods) and face stage.  LIM >= 0
// selects the fast path (MUSCL-Hancock only) with that compile-time limiter;
// LIM = -1 is the general path (runtime limiter and limiting variables, any
// gamma).
template <int D, int DIR, int METHOD, int LIM = -1>
struct Scheme {
    static constexpr int NC = D + 2;
    static constexpr bool kReconstruct = (METHOD == M_MUSCL || METHOD == M_SLIC);
    static constexpr bool kFast = (LIM >= 0);
    static constexpr int kHalo = kReconstruct ? 2 : 1;
    static_assert(!kFast || METHOD == M_MUSCL, "the fast path is MUSCL-Hancock only");

    __device__ __forceinline__ static void cell(const double (&Um)[NC], const double (&U0)[NC],
                                                const double (&Up)[NC], const Consts& k, double hdtdx,
                                                double (&UL)[NC], double (&UR)[NC])
    {
        if constexpr (kFast) {
            muscl_cell_fast<D, DIR, (LIM < 0 ? 0 : LIM)>(Um, U0, Up, k, hdtdx, UL, UR);
        } else if constexpr (kReconstruct) {
            muscl_cell<D, DIR>(Um, U0, Up, k, hdtdx, UL, UR);
        } else {
#pragma unroll
            for (int n = 0; n < NC; ++n) UL[n] = UR[n] = U0[n];
        }
    }

    // L: state left of the face (UR of the left cell), R: state right of it.
    __device__ __forceinline__ static void face(const double (&L)[NC], const double (&R)[NC], const Consts& k,
                                                double half_dx_dt, double dt_2dx, double (&F)[NC])
    {
        if constexpr (kFast) {
            hllc_face_fast<D, DIR>(L, R, k, F);
        } else if constexpr (METHOD == M_MUSCL || METHOD == M_HLLC) {
            hllc_face<D, DIR>(L, R, k, F);
        } else if constexpr (METHOD == M_SLIC || METHOD == M_FORCE) {
            force_face<D, DIR>(L, R, k, half_dx_dt, dt_2dx, F);
        } else {
            lf_face<D, DIR>(L, R, k, half_dx_dt, F);
        }
    }

    __device__ __forceinline__ static double speed(const double (&U)[NC], const Consts& k)
    {
        if constexpr (kFast) return wave_speed_fast<D>(U, k);
        else return wave_speed<D>(U, k);
    }
};

}  // namespace bamrex
