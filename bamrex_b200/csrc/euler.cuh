// Device-side Euler physics of the explicit path: primitive conversion,
// physical flux, slope limiters, MUSCL-Hancock cell stage, and the HLLC /
// FORCE / Lax-Friedrichs face stages, templated on the arithmetic type T
// (double: the drop-in path; float: the FP32-storage variant).  Each
// function follows the reference routine cited beside it in operation
// order, except that a reciprocal of the density (or of epsilon) is reused
// where the reference divides several times by the same value, and that the
// fast path evaluates the gamma powers of the Toro wave-speed estimate as a
// refined integer root.  In FP64 both change results by a few units in the
// last place (parity bound: 1e-12 relative L-infinity per step).
#pragma once

#include <cmath>

#include "common.cuh"

namespace bamrex {

enum { LIM_MINBEE = 0, LIM_VAN_LEER = 1, LIM_VAN_ALBADA = 2, LIM_SUPERBEE = 3 };
enum { M_MUSCL = 0, M_HLLC = 1, M_SLIC = 4, M_FORCE = 5, M_LF = 6 };

// Minimum density / pressure of the wave-speed estimate (HLLC.H:255-260).
constexpr double kMinRho = 1e-14;
constexpr double kMinP = 1e-14;

// The run constants in the arithmetic type of a kernel.
template <typename T>
struct K {
    T gamma, eps, inv_eps, gm1, half_gm1, z, neg_z, inv_z, gp1_2g, gamma_inv_eps, half_eps;
    double root_dneg_l2, root_dpos_l2;
    int root_k, limiter, uniform_var, need_prim;
    int lim_var[kMaxComp], lim_prim[kMaxComp];

    __device__ __forceinline__ explicit K(const Consts& c)
        : gamma((T)c.gamma), eps((T)c.eps), inv_eps((T)c.inv_eps), gm1((T)c.gm1), half_gm1((T)c.half_gm1),
          z((T)c.z), neg_z((T)c.neg_z), inv_z((T)c.inv_z), gp1_2g((T)c.gp1_2g), gamma_inv_eps((T)c.gamma_inv_eps),
          half_eps((T)c.half_eps), root_dneg_l2(c.root_dneg_l2), root_dpos_l2(c.root_dpos_l2), root_k(c.root_k),
          limiter(c.limiter), uniform_var(c.uniform_var), need_prim(c.need_prim)
    {
#pragma unroll
        for (int n = 0; n < kMaxComp; ++n) {
            lim_var[n] = c.lim_var[n];
            lim_prim[n] = c.lim_prim[n];
        }
    }
};

// a[idx] for a runtime idx without local-memory indexing.
template <typename T, int N>
__device__ __forceinline__ T sel(const T (&a)[N], int idx)
{
    T r = a[0];
#pragma unroll
    for (int m = 1; m < N; ++m) r = (idx == m) ? a[m] : r;
    return r;
}

// primv_from_consv (Source/System/Euler/Euler.H:167-198); inv_rho = 1/rho.
template <typename T, int D>
__device__ __forceinline__ void to_prim(const T (&U)[D + 2], const K<T>& k, T (&q)[D + 2], T& inv_rho)
{
    inv_rho = T(1) / U[0];
    q[0] = U[0];
#pragma unroll
    for (int d = 0; d < D; ++d) q[1 + d] = U[1 + d] * inv_rho;
    T usq = q[1] * q[1];
#pragma unroll
    for (int d = 1; d < D; ++d) usq = usq + q[1 + d] * q[1 + d];
    q[1 + D] = k.gm1 * (U[1 + D] - k.half_eps * U[0] * usq);
}

// euler_flux<dir> / compute_flux_function<dir> (Euler.H:211-244, Euler.cpp:10-44).
template <typename T, int D, int DIR>
__device__ __forceinline__ void phys_flux(const T (&U)[D + 2], const T (&q)[D + 2], const K<T>& k, T (&F)[D + 2])
{
    const T mn = U[1 + DIR];
    F[0] = mn;
#pragma unroll
    for (int d = 0; d < D; ++d) F[1 + d] = mn * q[1 + d];
    F[1 + DIR] += q[1 + D] * k.inv_eps;
    F[1 + D] = (U[1 + D] + q[1 + D]) * q[1 + DIR];
}

template <typename T, int D, int DIR>
__device__ __forceinline__ void phys_flux(const T (&U)[D + 2], const K<T>& k, T (&F)[D + 2])
{
    T q[D + 2], ir;
    to_prim<T, D>(U, k, q, ir);
    phys_flux<T, D, DIR>(U, q, k, F);
}

// slope_limit<L> (Source/Fluxes/Limiters.H:29-73).
template <typename T>
__device__ __forceinline__ T slope_limit(int lim, T r)
{
    if (r <= T(0)) return T(0);
    switch (lim) {
    case LIM_MINBEE: return r > T(1) ? fmin(T(2) / (T(1) + r), T(1)) : r;
    case LIM_VAN_LEER: {
        const T ip = T(1) / (T(1) + r);
        return fmin(T(2) * r * ip, T(2) * ip);
    }
    case LIM_VAN_ALBADA: return fmin(r * (T(1) + r) / (T(1) + r * r), T(2) / (T(1) + r));
    default: return (r <= T(0.5)) ? T(2) * r : ((r <= T(1)) ? T(1) : fmin(r, fmin(T(2) / (T(1) + r), T(2))));
    }
}

// The limiter value from the limiting-variable differences
// (Source/Fluxes/Flux_Helpers.cpp:103-111).
template <typename T>
__device__ __forceinline__ T limiter_value(int lim, T numerator, T denom)
{
    if (numerator == T(0) && denom == T(0)) return slope_limit<T>(lim, T(1));
    if (denom == T(0)) return T(0);
    return slope_limit<T>(lim, numerator / denom);
}

// ---- gamma powers of the general path ------------------------------------
template <typename T>
__device__ __forceinline__ T ipow_k(T y, int k)
{
    if (k == 7) {
        const T y2 = y * y, y3 = y2 * y, y6 = y3 * y3;
        return y6 * y;
    }
    if (k == 5) {
        const T y2 = y * y, y4 = y2 * y2;
        return y4 * y;
    }
    T r = y;
    for (int i = 1; i < k; ++i) r *= y;
    return r;
}

// x^(-z) for the clamped pressure x >= 1e-14 (HLLC.H:272).  With 1/z ~ k
// (and T = double), x^(-1/k) comes from a float seed and two Newton steps of
// y <- y + y (1 - x y^k) / k, then x^(1/k - z) ~ 1 + (1/k - z) ln x.
template <typename T>
__device__ __forceinline__ T pow_neg_z(T x, const K<T>& c)
{
    if constexpr (sizeof(T) == 4) {
        return pow(x, c.neg_z);
    } else {
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
        return fma(y, c.root_dneg_l2 * (double)lf, y);
    }
}

// b^(1/z) (HLLC.H:270-273): b^k (1 + (1/z - k) ln b) for T = double with an
// integer k; non-positive or extreme b goes to pow() (a negative base gives
// NaN there, as in the reference, which then selects q_K = 1).
template <typename T>
__device__ __forceinline__ T pow_inv_z(T b, const K<T>& c)
{
    if constexpr (sizeof(T) == 4) {
        return pow(b, c.inv_z);
    } else {
        if (c.root_k == 0 || !(b > 1e-30 && b < 1e30)) return pow(b, c.inv_z);
        const double bk = ipow_k(b, c.root_k);
        return fma(bk, c.root_dpos_l2 * (double)__log2f((float)b), bk);
    }
}

// ---- cell stage: reconstruct_and_half_time_step<limiter,dir> --------------
// (Source/Fluxes/Flux_Helpers.cpp:92-148) for one cell from its two
// neighbours along the sweep: returns the half-stepped L/R states.
template <typename T, int D, int DIR>
__device__ __forceinline__ void muscl_cell(const T (&Um)[D + 2], const T (&U0)[D + 2], const T (&Up)[D + 2],
                                           const K<T>& k, T hdtdx, T (&UL)[D + 2], T (&UR)[D + 2])
{
    constexpr int NC = D + 2;
    T hphi[NC];
    if (k.uniform_var >= 0) {
        const int v = k.uniform_var;
        const T vL = sel(Um, v), vC = sel(U0, v), vR = sel(Up, v);
        const T lim = limiter_value<T>(k.limiter, vC - vL, vR - vC);
#pragma unroll
        for (int n = 0; n < NC; ++n) hphi[n] = T(0.5) * lim;
    } else {
        T Qm[NC], Q0[NC], Qp[NC], ir;
        if (k.need_prim) {
            to_prim<T, D>(Um, k, Qm, ir);
            to_prim<T, D>(U0, k, Q0, ir);
            to_prim<T, D>(Up, k, Qp, ir);
        } else {
#pragma unroll
            for (int n = 0; n < NC; ++n) Qm[n] = Q0[n] = Qp[n] = T(0);
        }
#pragma unroll
        for (int n = 0; n < NC; ++n) {
            const int v = k.lim_var[n];
            const bool pr = k.lim_prim[n] != 0;
            const T vL = pr ? sel(Qm, v) : sel(Um, v);
            const T vC = pr ? sel(Q0, v) : sel(U0, v);
            const T vR = pr ? sel(Qp, v) : sel(Up, v);
            hphi[n] = T(0.5) * limiter_value<T>(k.limiter, vC - vL, vR - vC);
        }
    }
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        const T delta = T(0.5) * (U0[n] - Um[n]) + T(0.5) * (Up[n] - U0[n]);
        UL[n] = U0[n] - hphi[n] * delta;
        UR[n] = U0[n] + hphi[n] * delta;
    }
    T FL[NC], FR[NC];
    phys_flux<T, D, DIR>(UL, k, FL);
    phys_flux<T, D, DIR>(UR, k, FR);
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        const T dF = hdtdx * (FR[n] - FL[n]);
        UL[n] -= dF;
        UR[n] -= dF;
    }
}

// ---- face stage: HLLC (Source/Fluxes/HLLC.cpp:90-172 with
// estimate_wave_speed_HLLC_Toro, HLLC.H:214-309, and
// HLLC_interm_state_replace, HLLC.H:311-337).  L is the state left of the
// face, R the state right of it.
template <typename T, int D, int DIR>
__device__ __forceinline__ void hllc_face(const T (&L)[D + 2], const T (&R)[D + 2], const K<T>& k, T (&F)[D + 2])
{
    constexpr int NC = D + 2;
    T qL[NC], qR[NC], irL, irR;
    to_prim<T, D>(L, k, qL, irL);
    to_prim<T, D>(R, k, qR, irR);
    const T rhoL = fmax(qL[0], T(kMinRho)), rhoR = fmax(qR[0], T(kMinRho));
    const T pL = fmax(qL[1 + D], T(kMinP)), pR = fmax(qR[1 + D], T(kMinP));
    const T uL = qL[1 + DIR], uR = qR[1 + DIR];
    const T icL = (qL[0] >= T(kMinRho)) ? irL : T(1.0 / kMinRho);
    const T icR = (qR[0] >= T(kMinRho)) ? irR : T(1.0 / kMinRho);
    const T cL = sqrt(k.gamma_inv_eps * pL * icL);
    const T cR = sqrt(k.gamma_inv_eps * pR * icR);
    const T base = (cL + cR - k.half_gm1 * (uR - uL)) / (cL * pow_neg_z<T>(pL, k) + cR * pow_neg_z<T>(pR, k));
    const T p_rr = pow_inv_z<T>(base, k);
    const T qwL = (p_rr > pL) ? sqrt(T(1) + k.gp1_2g * (p_rr / pL - T(1))) : T(1);
    const T qwR = (p_rr > pR) ? sqrt(T(1) + k.gp1_2g * (p_rr / pR - T(1))) : T(1);
    const T SL = uL - cL * qwL;
    const T SR = uR + cR * qwR;
    const T dL = SL - uL, dR = SR - uR;
    const T denom = rhoL * dL - rhoR * dR;
    const T Ss = (denom != T(0)) ? ((pR - pL) * k.inv_eps + rhoL * uL * dL - rhoR * uR * dR) / denom : T(0);

    // Branches of HLLC.cpp:101-167: the left states serve when S_L >= 0 or
    // S* >= 0; the star correction applies unless the face is supersonic.
    const bool useL = (SL >= T(0)) || (Ss >= T(0));
    const bool star = useL ? (SL < T(0)) : (SR >= T(0));
    T UK[NC], qK[NC];
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        UK[n] = useL ? L[n] : R[n];
        qK[n] = useL ? qL[n] : qR[n];
    }
    const T irK = useL ? irL : irR;
    const T SK = useL ? SL : SR;
    phys_flux<T, D, DIR>(UK, qK, k, F);
    if (star) {
        const T rhoK = qK[0], uK = qK[1 + DIR], pK = qK[1 + D];
        const T dK = SK - uK;
        const T scale = rhoK * dK / (SK - Ss);
        const T eterm = UK[1 + D] * irK + (Ss - uK) * (Ss * k.eps + pK / (rhoK * dK));
        F[0] = F[0] + SK * (scale - UK[0]);
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const T s = (d == DIR) ? Ss : qK[1 + d];
            F[1 + d] = F[1 + d] + SK * (s * scale - UK[1 + d]);
        }
        F[1 + D] = F[1 + D] + SK * (eterm * scale - UK[1 + D]);
    }
}

// ---- face stage: FORCE (compute_force_flux_LR, Source/Fluxes/Force.cpp:22-108)
template <typename T, int D, int DIR>
__device__ __forceinline__ void force_face(const T (&L)[D + 2], const T (&R)[D + 2], const K<T>& k, T half_dx_dt,
                                           T dt_2dx, T (&F)[D + 2])
{
    constexpr int NC = D + 2;
    T fL[NC], fR[NC], H[NC], fH[NC];
    phys_flux<T, D, DIR>(L, k, fL);
    phys_flux<T, D, DIR>(R, k, fR);
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        F[n] = T(0.5) * (half_dx_dt * (L[n] - R[n]) + T(0.5) * (fL[n] + fR[n]));
        H[n] = T(0.5) * (L[n] + R[n]) + dt_2dx * (fL[n] - fR[n]);
    }
    phys_flux<T, D, DIR>(H, k, fH);
#pragma unroll
    for (int n = 0; n < NC; ++n) F[n] += T(0.5) * fH[n];
}

// ---- face stage: Lax-Friedrichs (compute_LF_flux, Source/Fluxes/Force.cpp:110-151)
template <typename T, int D, int DIR>
__device__ __forceinline__ void lf_face(const T (&L)[D + 2], const T (&R)[D + 2], const K<T>& k, T half_dx_dt,
                                        T (&F)[D + 2])
{
    constexpr int NC = D + 2;
    T fL[NC], fR[NC];
    phys_flux<T, D, DIR>(L, k, fL);
    phys_flux<T, D, DIR>(R, k, fR);
#pragma unroll
    for (int n = 0; n < NC; ++n) F[n] = half_dx_dt * (L[n] - R[n]) + T(0.5) * (fL[n] + fR[n]);
}

// |u| + c of a conserved state (max_wave_speed body, Euler.cpp:53-68).
template <typename T, int D>
__device__ __forceinline__ T wave_speed(const T (&U)[D + 2], const K<T>& k)
{
    T q[D + 2], ir;
    to_prim<T, D>(U, k, q, ir);
    T vsq = q[1] * q[1];
#pragma unroll
    for (int d = 1; d < D; ++d) vsq = vsq + q[1 + d] * q[1 + d];
    return sqrt(k.gamma_inv_eps * q[1 + D] * ir) + sqrt(vsq);
}

// ======================================================================
// Fast path: MUSCL-Hancock + HLLC with a compile-time limiter, every
// component limited on the energy (the reference default,
// FluidSystem.cpp:65-69), and gamma with 1/z = 7 (gamma = 1.4).  Same
// arithmetic as above but branch-free (selects instead of branches), with
// refined reciprocals in FP64 and the hardware approximations in FP32, so
// each cell and face is one basic block the scheduler can interleave.
// ======================================================================

// 1/x.  FP64: the hardware approximation r (PTX rcp.approx.ftz.f64; its
// relative error measured below 2^-19.9 on the B200 over 2^30 arguments)
// refined by one third-order step of the series 1/x = r / (1 - e) with
// e = 1 - x r: r (1 + e + e^2), three fused multiply-adds; within 1 ulp of
// the correctly rounded quotient for normal, finite x (the same probe), as
// two Newton steps are, for one multiply-add less.  FP32: the hardware
// approximation.
__device__ __forceinline__ double rcp_fast(double x)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    const double e = fma(-x, r, 1.0);
    return fma(r, fma(e, e, e), r);
}
__device__ __forceinline__ float rcp_fast(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// FP32 special-function approximations (PTX .approx.ftz.f32, a few ulp):
// the FP32-storage variant reports its error against the FP64 oracle
// instead of holding a bit-level bar.
__device__ __forceinline__ float sqrt_fast(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ double sqrt_fast(double x) { return sqrt(x); }

// sqrt(x) for a positive, normal, finite x without the special-case branch of
// sqrt(): the coupled iteration for g ~ sqrt(x), h ~ 1 / (2 sqrt(x)) seeded
// by the hardware reciprocal square root (PTX rsqrt.approx.ftz.f64, relative
// error below 2^-19.9): one step g += g r with r = 1/2 - g h (relative error
// ~1.5 e^2, e the seed's), then the correction g += h (x - g^2) with the
// seed's h, whose own error only scales the already tiny correction
// (P. Markstein, IA-64 and Elementary Functions, 2000).  Zero, infinity and
// subnormal x give NaN.  FP32: the hardware approximation.
__device__ __forceinline__ double sqrt_pos(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double g = x * y, h = 0.5 * y;
    const double r = fma(-g, h, 0.5);
    const double g1 = fma(g, r, g);
    const double d = fma(-g1, g1, x);
    return fma(d, h, g1);
}
__device__ __forceinline__ float sqrt_pos(float x) { return sqrt_fast(x); }

// sqrt(x) for every x with the IEEE special results (0 for 0, +inf for
// +inf, NaN for negative or NaN x), branch-free: subnormal x are scaled by
// 2^108 into the normal range before sqrt_pos and the root by 2^-54 after.
// Within one ulp of the correctly rounded root (sqrt_pos itself matched it
// on every one of 5e7 probed normal arguments).
__device__ __forceinline__ double sqrt_any(double x)
{
    const bool tiny = x < 0x1p-1022;
    const double r = sqrt_pos(tiny ? x * 0x1p108 : x);
    const double rs = tiny ? r * 0x1p-54 : r;
    return (x == 0.0 || x == __longlong_as_double(0x7ff0000000000000LL)) ? x : rs;
}
__device__ __forceinline__ float sqrt_any(float x) { return sqrt_fast(x); }
__device__ __forceinline__ float ex2_fast(float x)
{
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float lg2_fast(float x)
{
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
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
// FP64: seed y0 = 2^(-log2(x)/7) in single precision (the hardware
// approximations of log2 and exp2, a few ulp), then one step of the series
// of (1 - e)^(-1/7), e = 1 - x y0^7 (third-order convergence: |e| ~ 2e-6
// leaves ~5e-19), then the factor x^(1/7 - z) ~ 1 + (1/7 - z) ln x;
// 1/x = y0^7 / (1 - e) ~ y0^7 (1 + e + e^2).  FP32: exp2(-z log2 x) on the
// special-function unit.
__device__ __forceinline__ void root7_neg_z(double x, const K<double>& c, double& y, double& inv_x)
{
    const float lf = log2_abs(x);
    const float q = -lf * (1.0f / 7.0f);
    const float qi = floorf(q);
    const double p2 = __longlong_as_double((long long)((int)qi + 1023) << 52);
    const double y0 = p2 * (double)ex2_fast(q - qi);
    const double y2 = y0 * y0, y3 = y2 * y0, y6 = y3 * y3, y7 = y6 * y0;
    const double e = fma(-x, y7, 1.0);
    const double t = e * fma(e, 8.0 / 98.0, 1.0 / 7.0);
    y = fma(y0, t + c.root_dneg_l2 * (double)lf, y0);
    inv_x = fma(y7, fma(e, e, e), y7);
}
__device__ __forceinline__ void root7_neg_z(float x, const K<float>& c, float& y, float& inv_x)
{
    y = ex2_fast(c.neg_z * lg2_fast(x));
    inv_x = rcp_fast(x);
}

// b^(1/z) with 1/z = 7 + dpos: b^7 (1 + dpos ln b).  A negative base gives a
// negative result (the reference's pow gives NaN there); both make every
// "p_rr > p_K" test false, so the wave speeds agree.  FP32: exp2(log2(b)/z)
// (NaN for a negative base, as the reference).
__device__ __forceinline__ double pow7_inv_z(double b, const K<double>& c)
{
    const double b2 = b * b, b3 = b2 * b, b6 = b3 * b3, b7 = b6 * b;
    return fma(b7, c.root_dpos_l2 * (double)log2_abs(b), b7);
}
__device__ __forceinline__ float pow7_inv_z(float b, const K<float>& c)
{
    // lg2 of a negative base is NaN, as the reference's pow
    return ex2_fast(c.inv_z * lg2_fast(b));
}

template <typename T, int D>
__device__ __forceinline__ void to_prim_fast(const T (&U)[D + 2], const K<T>& k, T (&q)[D + 2], T& inv_rho)
{
    inv_rho = rcp_fast(U[0]);
    q[0] = U[0];
#pragma unroll
    for (int d = 0; d < D; ++d) q[1 + d] = U[1 + d] * inv_rho;
    T usq = q[1] * q[1];
#pragma unroll
    for (int d = 1; d < D; ++d) usq = usq + q[1 + d] * q[1 + d];
    q[1 + D] = k.gm1 * (U[1 + D] - k.half_eps * U[0] * usq);
}

template <typename T, int D, int DIR>
__device__ __forceinline__ void phys_flux_fast(const T (&U)[D + 2], const K<T>& k, T (&F)[D + 2])
{
    T q[D + 2], ir;
    to_prim_fast<T, D>(U, k, q, ir);
    phys_flux<T, D, DIR>(U, q, k, F);
}

// The limiter value of Flux_Helpers.cpp:103-111 and Limiters.H:29-73 without
// branches.  With r = num / den, minbee, van Leer and superbee are, for
// r > 0, a single quotient of num and den whose operands the case of r
// selects (minbee: num / den for r <= 1, 2 den / (den + num) above; van
// Leer: 2 min-side / (den + num); superbee: 2 num / den, 1, 2 den / (den +
// num)), so they take one reciprocal; the cases are decided from num and den
// exactly (r > 1 is |num| > |den| with equal signs), which agrees with the
// rounded quotient except where that rounds to exactly 1 or 1/2, and there
// both formulas give the same value to an ulp.
template <typename T, int LIM>
__device__ __forceinline__ T limiter_value_fast(T num, T den)
{
    const bool pos = (num > T(0) && den > T(0)) || (num < T(0) && den < T(0));  // r > 0
    const T an = fabs(num), ad = fabs(den);
    T phi;
    if constexpr (LIM == LIM_MINBEE) {
        const bool big = an > ad;  // r > 1
        phi = (big ? T(2) * den : num) * rcp_fast(big ? den + num : den);
    } else if constexpr (LIM == LIM_VAN_LEER) {
        // 2 r / (1 + r) for r <= 1, 2 / (1 + r) above
        phi = T(2) * (an > ad ? den : num) * rcp_fast(den + num);
    } else if constexpr (LIM == LIM_VAN_ALBADA) {
        const T r = num * rcp_fast(den);
        phi = fmin(r * (T(1) + r) * rcp_fast(T(1) + r * r), T(2) * rcp_fast(T(1) + r));
    } else {
        // 2 r for r <= 1/2, 1 for r <= 1, min(r, 2 / (1 + r), 2) = 2 / (1 + r) above
        const bool big = an > ad, half = T(2) * an <= ad;
        const T q = (big ? T(2) * den : T(2) * num) * rcp_fast(big ? den + num : den);
        phi = (half || big) ? q : T(1);
    }
    phi = pos ? phi : T(0);
    return (num == T(0) && den == T(0)) ? T(1) : phi;
}

template <typename T, int D, int DIR, int LIM>
__device__ __forceinline__ void muscl_cell_fast(const T (&Um)[D + 2], const T (&U0)[D + 2], const T (&Up)[D + 2],
                                                const K<T>& k, T hdtdx, T (&UL)[D + 2], T (&UR)[D + 2])
{
    constexpr int NC = D + 2;
    constexpr int E = D + 1;
    // 0.5 phi delta with delta = 0.5 (U0 - Um) + 0.5 (Up - U0) written as
    // 0.25 phi (Up - Um) (within an ulp of the reference's rounding)
    const T qphi = T(0.25) * limiter_value_fast<T, LIM>(U0[E] - Um[E], Up[E] - U0[E]);
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        const T d2 = Up[n] - Um[n];
        UL[n] = fma(-qphi, d2, U0[n]);
        UR[n] = fma(qphi, d2, U0[n]);
    }
    T FL[NC], FR[NC];
    phys_flux_fast<T, D, DIR>(UL, k, FL);
    phys_flux_fast<T, D, DIR>(UR, k, FR);
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        const T dF = hdtdx * (FR[n] - FL[n]);
        UL[n] -= dF;
        UR[n] -= dF;
    }
}

template <typename T, int D, int DIR>
__device__ __forceinline__ void hllc_face_fast(const T (&L)[D + 2], const T (&R)[D + 2], const K<T>& k,
                                               T (&F)[D + 2])
{
    constexpr int NC = D + 2;
    T qL[NC], qR[NC], irL, irR;
    to_prim_fast<T, D>(L, k, qL, irL);
    to_prim_fast<T, D>(R, k, qR, irR);
    const T rhoL = fmax(qL[0], T(kMinRho)), rhoR = fmax(qR[0], T(kMinRho));
    const T pL = fmax(qL[1 + D], T(kMinP)), pR = fmax(qR[1 + D], T(kMinP));
    const T uL = qL[1 + DIR], uR = qR[1 + DIR];
    const T icL = (qL[0] >= T(kMinRho)) ? irL : T(1.0 / kMinRho);
    const T icR = (qR[0] >= T(kMinRho)) ? irR : T(1.0 / kMinRho);
    // positive arguments: p >= 1e-14 and 1 / rho <= 1e14 (clamped above),
    // and 1 + (gamma+1)/(2 gamma) (p_rr / p - 1) > 1 under p_rr > p
    const T cL = sqrt_pos(k.gamma_inv_eps * pL * icL);
    const T cR = sqrt_pos(k.gamma_inv_eps * pR * icR);
    T yL, yR, ipL, ipR;
    root7_neg_z(pL, k, yL, ipL);
    root7_neg_z(pR, k, yR, ipR);
    const T base = (cL + cR - k.half_gm1 * (uR - uL)) * rcp_fast(cL * yL + cR * yR);
    const T p_rr = pow7_inv_z(base, k);
    const T qwL = (p_rr > pL) ? sqrt_pos(T(1) + k.gp1_2g * (p_rr * ipL - T(1))) : T(1);
    const T qwR = (p_rr > pR) ? sqrt_pos(T(1) + k.gp1_2g * (p_rr * ipR - T(1))) : T(1);
    const T SL = uL - cL * qwL;
    const T SR = uR + cR * qwR;
    const T dL = SL - uL, dR = SR - uR;
    const T denom = rhoL * dL - rhoR * dR;
    const T Ss_raw = ((pR - pL) * k.inv_eps + rhoL * uL * dL - rhoR * uR * dR) * rcp_fast(denom);
    const T Ss = (denom != T(0)) ? Ss_raw : T(0);

    const bool useL = (SL >= T(0)) || (Ss >= T(0));
    const bool star = useL ? (SL < T(0)) : (SR >= T(0));
    T UK[NC], qK[NC];
#pragma unroll
    for (int n = 0; n < NC; ++n) {
        UK[n] = useL ? L[n] : R[n];
        qK[n] = useL ? qL[n] : qR[n];
    }
    const T irK = useL ? irL : irR;
    const T SK = useL ? SL : SR;
    phys_flux<T, D, DIR>(UK, qK, k, F);
    // star state (HLLC.H:311-337): with m = rho_K (S_K - u_K), b = S_K - S*,
    // scale = m / b = m^2 / (m b) and p_K / m = p_K b / (m b)
    const T rhoK = qK[0], uK = qK[1 + DIR], pK = qK[1 + D];
    const T m = rhoK * (SK - uK);
    const T bq = SK - Ss;
    const T rmb = rcp_fast(m * bq);
    const T scale = m * m * rmb;
    const T eterm = UK[1 + D] * irK + (Ss - uK) * (Ss * k.eps + pK * bq * rmb);
    F[0] = star ? F[0] + SK * (scale - UK[0]) : F[0];
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const T s = (d == DIR) ? Ss : qK[1 + d];
        F[1 + d] = star ? F[1 + d] + SK * (s * scale - UK[1 + d]) : F[1 + d];
    }
    F[1 + D] = star ? F[1 + D] + SK * (eterm * scale - UK[1 + D]) : F[1 + D];
}

template <typename T, int D>
__device__ __forceinline__ T wave_speed_fast(const T (&U)[D + 2], const K<T>& k)
{
    T q[D + 2], ir;
    to_prim_fast<T, D>(U, k, q, ir);
    T vsq = q[1] * q[1];
#pragma unroll
    for (int d = 1; d < D; ++d) vsq = vsq + q[1 + d] * q[1 + d];
    return sqrt_any(k.gamma_inv_eps * q[1 + D] * ir) + sqrt_any(vsq);
}

// Method dispatch: cell stage (reconstruction + half step for MUSCL-Hancock
// and SLIC; identity for first-order methods) and face stage.  LIM >= 0
// selects the fast path (MUSCL-Hancock only) with that compile-time limiter;
// LIM = -1 is the general path (runtime limiter and limiting variables, any
// gamma).
template <typename T, int D, int DIR, int METHOD, int LIM = -1>
struct Scheme {
    static constexpr int NC = D + 2;
    static constexpr bool kReconstruct = (METHOD == M_MUSCL || METHOD == M_SLIC);
    static constexpr bool kFast = (LIM >= 0);
    static constexpr int kHalo = kReconstruct ? 2 : 1;
    static_assert(!kFast || METHOD == M_MUSCL, "the fast path is MUSCL-Hancock only");

    __device__ __forceinline__ static void cell(const T (&Um)[NC], const T (&U0)[NC], const T (&Up)[NC],
                                                const K<T>& k, T hdtdx, T (&UL)[NC], T (&UR)[NC])
    {
        if constexpr (kFast) {
            muscl_cell_fast<T, D, DIR, (LIM < 0 ? 0 : LIM)>(Um, U0, Up, k, hdtdx, UL, UR);
        } else if constexpr (kReconstruct) {
            muscl_cell<T, D, DIR>(Um, U0, Up, k, hdtdx, UL, UR);
        } else {
#pragma unroll
            for (int n = 0; n < NC; ++n) UL[n] = UR[n] = U0[n];
        }
    }

    // L: state left of the face (UR of the left cell), R: state right of it.
    __device__ __forceinline__ static void face(const T (&L)[NC], const T (&R)[NC], const K<T>& k, T half_dx_dt,
                                                T dt_2dx, T (&F)[NC])
    {
        if constexpr (kFast) {
            hllc_face_fast<T, D, DIR>(L, R, k, F);
        } else if constexpr (METHOD == M_MUSCL || METHOD == M_HLLC) {
            hllc_face<T, D, DIR>(L, R, k, F);
        } else if constexpr (METHOD == M_SLIC || METHOD == M_FORCE) {
            force_face<T, D, DIR>(L, R, k, half_dx_dt, dt_2dx, F);
        } else {
            lf_face<T, D, DIR>(L, R, k, half_dx_dt, F);
        }
    }

    __device__ __forceinline__ static T speed(const T (&U)[NC], const K<T>& k)
    {
        if constexpr (kFast) return wave_speed_fast<T, D>(U, k);
        else return wave_speed<T, D>(U, k);
    }
};

}  // namespace bamrex
