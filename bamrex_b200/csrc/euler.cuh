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

// Method dispatch: cell stage (reconstruction + half step for MUSCL-Hancock
// and SLIC; identity for first-order methods) and face stage.
template <int D, int DIR, int METHOD>
struct Scheme {
    static constexpr int NC = D + 2;
    static constexpr bool kReconstruct = (METHOD == M_MUSCL || METHOD == M_SLIC);
    static constexpr int kHalo = kReconstruct ? 2 : 1;

    __device__ __forceinline__ static void cell(const double (&Um)[NC], const double (&U0)[NC],
                                                const double (&Up)[NC], const Consts& k, double hdtdx,
                                                double (&UL)[NC], double (&UR)[NC])
    {
        if constexpr (kReconstruct) {
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
        if constexpr (METHOD == M_MUSCL || METHOD == M_HLLC) {
            hllc_face<D, DIR>(L, R, k, F);
        } else if constexpr (METHOD == M_SLIC || METHOD == M_FORCE) {
            force_face<D, DIR>(L, R, k, half_dx_dt, dt_2dx, F);
        } else {
            lf_face<D, DIR>(L, R, k, half_dx_dt, F);
        }
    }
};

}  // namespace bamrex
