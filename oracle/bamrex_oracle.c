/*
 * bamrex_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C CPU restatement of BAMReX's explicit finite-volume path, used as
 * the parity checker for the CUDA kernels and as the timed CPU baseline
 * ("port").  It is never linked into, loaded by, or called from the product
 * library (bamrex_b200/libbamrex_cuda.so); only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may use it.
 *
 * The reference itself cannot be compiled here (it needs the AMReX library,
 * which is neither vendored nor installed), so this file restates, function by
 * function and in the same floating-point operation order, the reference
 * sources cited beside each routine (paths are relative to the BAMReX tree).
 * It keeps the reference's multi-pass structure (per-box temporaries for the
 * reconstructed states and flux-function values) so that its timing reflects
 * the reference CPU algorithm.  Build with -ffp-contract=off for parity.
 *
 * Pinning: the routines here are checked against the reference's own
 * known-answer tests (Tests/HLLC01.cpp + Tests/hllc_test.H wave speeds,
 * Tests/Euler01.cpp + Tests/BoxTest.H conversions and max wave speed,
 * Tests/Limiters01.cpp minmod) by tests/test_oracle_pins.py.  The reference
 * tests do not pin the composite MUSCL-Hancock flux; that composite is the
 * line-by-line restatement below.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define O_MAXC 8 /* MAX_NCOMP = PUInd::size, Source/System/Parm.H:9 */

/* NumericalMethods::Method order, Source/NumericalMethods.H:10-19 */
enum { M_MUSCL = 0, M_HLLC = 1, M_IMEX = 2, M_RCM = 3, M_SLIC = 4, M_FORCE = 5, M_LF = 6 };
/* AMREX_ENUM(Limiter, minbee, van_leer, van_albada, superbee), Source/Fluxes/Limiters.H:13 */
enum { L_MINBEE = 0, L_VANLEER = 1, L_VANALBADA = 2, L_SUPERBEE = 3 };
/* BC kinds (BAMReXBCType transmissive/periodic/reflective), Source/BoundaryConditions/BCs.cpp:226-266 */
enum { BC_TRANSMISSIVE = 0, BC_PERIODIC = 1, BC_REFLECTIVE = 2 };

/* Subset of Parm (Source/System/Parm.H:14-61) that the explicit path reads. */
typedef struct {
    double adiabatic;
    double epsilon;
    int limiter;
    unsigned int limiter_indices[O_MAXC];
    unsigned char limit_on_primv[O_MAXC];
    unsigned char need_primitive_for_limiting;
} oracle_parm;

/* An amrex::Array4<Real>: element (i,j,k,n) at
 * p[(i-begin0) + (j-begin1)*jstride + (k-begin2)*kstride + n*nstride]. */
typedef struct {
    double *p;
    long long jstride, kstride, nstride;
    int begin[3];
    int end[3]; /* exclusive */
    int ncomp;
} o_a4;

static inline double *A4(const o_a4 *a, int i, int j, int k, int n)
{
    return a->p + (long long)(i - a->begin[0]) + (long long)(j - a->begin[1]) * a->jstride
           + (long long)(k - a->begin[2]) * a->kstride + (long long)n * a->nstride;
}

typedef struct { int lo[3], hi[3]; } o_box;

static o_box grow_all(o_box b, int D, int g)
{
    for (int d = 0; d < D; ++d) { b.lo[d] -= g; b.hi[d] += g; }
    return b;
}
static o_box grow_dir(o_box b, int dir, int g) { b.lo[dir] -= g; b.hi[dir] += g; return b; }
static o_box surrounding_nodes(o_box b, int dir) { b.hi[dir] += 1; return b; }

static o_a4 alloc_fab(o_box b, int ncomp)
{
    o_a4 a;
    long long nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1, nz = b.hi[2] - b.lo[2] + 1;
    a.jstride = nx; a.kstride = nx * ny; a.nstride = nx * ny * nz;
    for (int d = 0; d < 3; ++d) { a.begin[d] = b.lo[d]; a.end[d] = b.hi[d] + 1; }
    a.ncomp = ncomp;
    a.p = (double *)malloc(sizeof(double) * (size_t)(a.nstride * ncomp));
    return a;
}
static o_a4 sub_fab(o_a4 a, int comp0, int ncomp)
{
    o_a4 s = a; s.p = a.p + (long long)comp0 * a.nstride; s.ncomp = ncomp; return s;
}

/* ------------------------------------------------------------------ */
/* Euler kernels: Source/System/Euler/Euler.H:138-254                   */
/* ------------------------------------------------------------------ */

/* consv_from_primv, Euler.H:138-165 */
void oracle_consv_from_primv(int D, const double *q, double adia, double eps, double *u)
{
    u[0] = q[0];
    for (int d = 0; d < D; ++d) u[1 + d] = q[0] * q[1 + d];
    const double pressure = q[1 + D];
    const double vol_internal_energy = pressure / (adia - 1);
    double u_sq = q[1] * q[1];
    for (int d = 1; d < D; ++d) u_sq = u_sq + q[1 + d] * q[1 + d];
    u[1 + D] = vol_internal_energy + 0.5 * eps * q[0] * u_sq;
}

/* primv_from_consv, Euler.H:167-198 */
void oracle_primv_from_consv(int D, const double *u, double adia, double eps, double *q)
{
    q[0] = u[0];
    for (int d = 0; d < D; ++d) q[1 + d] = u[1 + d] / u[0];
    double u_sq = q[1] * q[1];
    for (int d = 1; d < D; ++d) u_sq = u_sq + q[1 + d] * q[1 + d];
    q[1 + D] = (adia - 1) * (u[1 + D] - 0.5 * eps * u[0] * u_sq);
}

/* euler_flux<dir>, Euler.H:211-244 (also compute_flux_function, Euler.cpp:10-44) */
void oracle_euler_flux(int D, int dir, const double *u, double adia, double eps, double *f)
{
    double q[O_MAXC];
    oracle_primv_from_consv(D, u, adia, eps, q);
    const double pressure = q[1 + D];
    const double energy = u[1 + D];
    f[0] = u[1 + dir];
    for (int d = 0; d < D; ++d) f[1 + d] = u[1 + dir] * q[1 + d];
    f[1 + dir] += pressure / eps;
    f[1 + D] = (energy + pressure) * q[1 + dir];
}

/* ------------------------------------------------------------------ */
/* Limiters: Source/Fluxes/Limiters.H:29-80                             */
/* ------------------------------------------------------------------ */
static double o_minbee(double r) { return r <= 0 ? 0 : (r > 1 ? fmin(2. / (1 + r), 1.) : r); }
static double o_van_leer(double r) { return r <= 0 ? 0 : fmin(2. * r / (1 + r), 2. / (1 + r)); }
static double o_van_albada(double r) { return r <= 0 ? 0 : fmin(r * (1 + r) / (1 + r * r), 2. / (1 + r)); }
static double o_superbee(double r)
{
    return (r <= 0) ? 0
                    : ((0 < r && r <= 0.5) ? 2 * r
                                            : ((0.5 < r && r <= 1) ? 1 : fmin(r, fmin(2. / (1 + r), 2.))));
}
double oracle_slope_limit(int limiter, double r)
{
    switch (limiter) {
    case L_MINBEE: return o_minbee(r);
    case L_VANLEER: return o_van_leer(r);
    case L_VANALBADA: return o_van_albada(r);
    case L_SUPERBEE: return o_superbee(r);
    }
    return NAN;
}
/* minmod, Limiters.H:75-80 */
double oracle_minmod(double dL, double dR)
{
    return (dL > 0 && dR > 0) ? fmin(dL, dR) : ((dL < 0 && dR < 0) ? fmax(dL, dR) : 0);
}

/* ------------------------------------------------------------------ */
/* HLLC pieces: Source/Fluxes/HLLC.H:214-337                            */
/* ------------------------------------------------------------------ */

/* estimate_wave_speed_HLLC_Toro<dir>, HLLC.H:214-309, on two conserved states */
void oracle_wave_speed_toro(int D, int dir, const double *uL, const double *uR, double adiabatic_L,
                            double adiabatic_R, double epsilon, double *out /* S_L, S_R, S_* */)
{
    double qL[O_MAXC], qR[O_MAXC];
    oracle_primv_from_consv(D, uL, adiabatic_L, epsilon, qL);
    oracle_primv_from_consv(D, uR, adiabatic_R, epsilon, qR);
    double density_L = qL[0], density_R = qR[0];
    double p_L = qL[1 + D], p_R = qR[1 + D];
    const double u_L = qL[1 + dir], u_R = qR[1 + dir];
    const double min_rho = 1e-14, min_p = 1e-14;
    density_L = fmax(density_L, min_rho);
    density_R = fmax(density_R, min_rho);
    p_L = fmax(p_L, min_p);
    p_R = fmax(p_R, min_p);
    const double c_L = sqrt(adiabatic_L * p_L / (density_L * epsilon));
    const double c_R = sqrt(adiabatic_R * p_R / (density_R * epsilon));
    const double adiabatic = adiabatic_L;
    const double z = (adiabatic - 1) / (2 * adiabatic);
    const double p_rr = pow((c_L + c_R - (adiabatic - 1) / 2 * (u_R - u_L))
                                / (c_L * pow(p_L, -z) + c_R * pow(p_R, -z)),
                            1 / z);
    const double q_L = (p_rr > p_L) ? sqrt(1 + (adiabatic + 1) / (2 * adiabatic) * (p_rr / p_L - 1)) : 1;
    const double q_R = (p_rr > p_R) ? sqrt(1 + (adiabatic + 1) / (2 * adiabatic) * (p_rr / p_R - 1)) : 1;
    const double speed_L = u_L - c_L * q_L;
    const double speed_R = u_R + c_R * q_R;
    const double denom = (density_L * (speed_L - u_L) - density_R * (speed_R - u_R));
    const double speed_interm
        = (denom != 0) ? ((p_R - p_L) / epsilon + density_L * u_L * (speed_L - u_L)
                          - density_R * u_R * (speed_R - u_R))
                             / denom
                       : 0;
    out[0] = speed_L;
    out[1] = speed_R;
    out[2] = speed_interm;
}

/* HLLC_interm_state_replace<dir>, HLLC.H:311-337 (q: primitive, overwritten) */
static void o_interm_state_replace(int D, int dir, double *q, double energy, double speed_K,
                                   double speed_interm, double epsilon)
{
    const double density = q[0];
    const double u_K = q[1 + dir];
    const double pressure = q[1 + D];
    q[0] = 1;
    q[1 + dir] = speed_interm;
    const double scale_factor = density * (speed_K - u_K) / (speed_K - speed_interm);
    q[1 + D] = energy / density
               + (speed_interm - u_K) * (speed_interm * epsilon + pressure / (density * (speed_K - u_K)));
    for (int i = 0; i < D + 2; ++i) q[i] *= scale_factor;
}

/* One HLLC face: the body of compute_HLLC_flux_LR_euler's ParallelFor,
 * Source/Fluxes/HLLC.cpp:90-172.  uL is the state at i-1 of the L array, uR
 * the state at i of the R array. */
void oracle_hllc_face(int D, int dir, const double *uL, const double *uR, double adiabatic,
                      double epsilon, double *f)
{
    const int NC = D + 2;
    double s[3];
    oracle_wave_speed_toro(D, dir, uL, uR, adiabatic, adiabatic, epsilon, s);
    const double speed_L = s[0], speed_R = s[1], speed_interm = s[2];
    double fl[O_MAXC], q[O_MAXC];
    if (0 <= speed_L) {
        oracle_euler_flux(D, dir, uL, adiabatic, epsilon, fl);
        for (int n = 0; n < NC; ++n) f[n] = fl[n];
    } else if (speed_L <= 0 && 0 <= speed_interm) {
        oracle_euler_flux(D, dir, uL, adiabatic, epsilon, fl);
        oracle_primv_from_consv(D, uL, adiabatic, epsilon, q);
        o_interm_state_replace(D, dir, q, uL[1 + D], speed_L, speed_interm, epsilon);
        for (int n = 0; n < NC; ++n) f[n] = fl[n] + speed_L * (q[n] - uL[n]);
    } else if (speed_interm <= 0 && 0 <= speed_R) {
        oracle_euler_flux(D, dir, uR, adiabatic, epsilon, fl);
        oracle_primv_from_consv(D, uR, adiabatic, epsilon, q);
        o_interm_state_replace(D, dir, q, uR[1 + D], speed_R, speed_interm, epsilon);
        for (int n = 0; n < NC; ++n) f[n] = fl[n] + speed_R * (q[n] - uR[n]);
    } else if (0 >= speed_R) {
        oracle_euler_flux(D, dir, uR, adiabatic, epsilon, fl);
        for (int n = 0; n < NC; ++n) f[n] = fl[n];
    } else {
        /* NaN wave speeds: the reference leaves the flux unwritten (HLLC.cpp:168-171). */
        for (int n = 0; n < NC; ++n) f[n] = NAN;
    }
}

/* ------------------------------------------------------------------ */
/* Box-level passes (multi-pass, as the reference)                      */
/* ------------------------------------------------------------------ */

static void load_state(const o_a4 *a, int i, int j, int k, int NC, double *u)
{
    for (int n = 0; n < NC; ++n) u[n] = *A4(a, i, j, k, n);
}

/* FluidSystem::FillFluxes -> compute_flux_function<dir>,
 * Source/System/FluidSystem.cpp:142-160, Source/System/Euler/Euler.cpp:10-44 */
static void o_fill_fluxes(int D, int dir, o_box bx, o_a4 *flux, const o_a4 *U, double adia, double eps)
{
    const int NC = D + 2;
    double u[O_MAXC], f[O_MAXC];
    for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
        for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
            for (int i = bx.lo[0]; i <= bx.hi[0]; ++i) {
                load_state(U, i, j, k, NC, u);
                oracle_euler_flux(D, dir, u, adia, eps, f);
                for (int n = 0; n < NC; ++n) *A4(flux, i, j, k, n) = f[n];
            }
}

/* FluidSystem::UtoQ, Source/System/FluidSystem.cpp:162-180 */
static void o_u_to_q(int D, o_box bx, o_a4 *Q, const o_a4 *U, double adia, double eps)
{
    const int NC = D + 2;
    double u[O_MAXC], q[O_MAXC];
    for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
        for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
            for (int i = bx.lo[0]; i <= bx.hi[0]; ++i) {
                load_state(U, i, j, k, NC, u);
                oracle_primv_from_consv(D, u, adia, eps, q);
                for (int n = 0; n < NC; ++n) *A4(Q, i, j, k, n) = q[n];
            }
}

/* calc_limiting_var, Source/Fluxes/CalcLimitingVal.H:9-22 */
static double o_limiting_var(const o_a4 *U, const o_a4 *Q, const oracle_parm *parm, int i, int j, int k, int n)
{
    if (parm->limit_on_primv[n]) return *A4(Q, i, j, k, (int)parm->limiter_indices[n]);
    return *A4(U, i, j, k, (int)parm->limiter_indices[n]);
}

/* reconstruct_and_half_time_step<limiter,dir>, Source/Fluxes/Flux_Helpers.cpp:52-149 */
static void o_reconstruct_and_half_time_step(int D, int dir, o_box gbx, o_a4 *hsL, o_a4 *hsR,
                                             const o_a4 *consv, const double *dx_arr, double dt,
                                             const oracle_parm *parm)
{
    const int NC = D + 2;
    const double dx = dx_arr[dir];
    const o_box gbx2 = grow_dir(gbx, dir, 1);
    o_a4 tmp = alloc_fab(parm->need_primitive_for_limiting ? gbx2 : gbx, NC * (parm->need_primitive_for_limiting ? 3 : 2));
    o_a4 ffL = sub_fab(tmp, 0, NC), ffR = sub_fab(tmp, NC, NC), Q = tmp;
    if (parm->need_primitive_for_limiting) {
        Q = sub_fab(tmp, 2 * NC, NC);
        o_u_to_q(D, gbx2, &Q, consv, parm->adiabatic, parm->epsilon);
    }
    const int io = dir == 0, jo = dir == 1, ko = dir == 2;
    for (int n = 0; n < NC; ++n)
        for (int k = gbx.lo[2]; k <= gbx.hi[2]; ++k)
            for (int j = gbx.lo[1]; j <= gbx.hi[1]; ++j)
                for (int i = gbx.lo[0]; i <= gbx.hi[0]; ++i) {
                    const double val_C = o_limiting_var(consv, &Q, parm, i, j, k, n);
                    const double val_L = o_limiting_var(consv, &Q, parm, i - io, j - jo, k - ko, n);
                    const double val_R = o_limiting_var(consv, &Q, parm, i + io, j + jo, k + ko, n);
                    const double numerator = val_C - val_L;
                    const double denom = val_R - val_C;
                    double limiter_val;
                    if (numerator == 0. && denom == 0.)
                        limiter_val = oracle_slope_limit(parm->limiter, 1);
                    else if (denom == 0)
                        limiter_val = 0;
                    else
                        limiter_val = oracle_slope_limit(parm->limiter, numerator / denom);
                    const double omega = 0;
                    const double uc = *A4(consv, i, j, k, n);
                    const double delta_left = uc - *A4(consv, i - io, j - jo, k - ko, n);
                    const double delta_right = *A4(consv, i + io, j + jo, k + ko, n) - uc;
                    const double delta = 0.5 * (1 + omega) * delta_left + 0.5 * (1 - omega) * delta_right;
                    *A4(hsL, i, j, k, n) = uc - 0.5 * limiter_val * delta;
                    *A4(hsR, i, j, k, n) = uc + 0.5 * limiter_val * delta;
                }
    o_fill_fluxes(D, dir, gbx, &ffL, hsL, parm->adiabatic, parm->epsilon);
    o_fill_fluxes(D, dir, gbx, &ffR, hsR, parm->adiabatic, parm->epsilon);
    const double hdtdx = 0.5 * dt / dx;
    for (int n = 0; n < NC; ++n)
        for (int k = gbx.lo[2]; k <= gbx.hi[2]; ++k)
            for (int j = gbx.lo[1]; j <= gbx.hi[1]; ++j)
                for (int i = gbx.lo[0]; i <= gbx.hi[0]; ++i) {
                    *A4(hsL, i, j, k, n) -= hdtdx * (*A4(&ffR, i, j, k, n) - *A4(&ffL, i, j, k, n));
                    *A4(hsR, i, j, k, n) -= hdtdx * (*A4(&ffR, i, j, k, n) - *A4(&ffL, i, j, k, n));
                }
    free(tmp.p);
}

/* compute_HLLC_flux_LR_euler<dir>, Source/Fluxes/HLLC.cpp:64-173 */
static void o_hllc_flux_LR(int D, int dir, o_box bx, o_a4 *flux, const o_a4 *cL, const o_a4 *cR,
                           const oracle_parm *parm)
{
    const int NC = D + 2;
    const o_box fb = surrounding_nodes(bx, dir);
    const int io = dir == 0, jo = dir == 1, ko = dir == 2;
    double uL[O_MAXC], uR[O_MAXC], f[O_MAXC];
    for (int k = fb.lo[2]; k <= fb.hi[2]; ++k)
        for (int j = fb.lo[1]; j <= fb.hi[1]; ++j)
            for (int i = fb.lo[0]; i <= fb.hi[0]; ++i) {
                load_state(cL, i - io, j - jo, k - ko, NC, uL);
                load_state(cR, i, j, k, NC, uR);
                oracle_hllc_face(D, dir, uL, uR, parm->adiabatic, parm->epsilon, f);
                for (int n = 0; n < NC; ++n) *A4(flux, i, j, k, n) = f[n];
            }
}

/* compute_force_flux_LR<dir>, Source/Fluxes/Force.cpp:22-108 */
static void o_force_flux_LR(int D, int dir, o_box bx, o_a4 *flux, const o_a4 *cL, const o_a4 *cR,
                            const double *dx_arr, double dt, const oracle_parm *parm)
{
    const int NC = D + 2;
    const double dx = dx_arr[dir];
    const o_box ghost_bx = grow_dir(bx, dir, 1);
    const o_box flux_bx = (o_box){ { bx.lo[0], bx.lo[1], bx.lo[2] }, { bx.hi[0], bx.hi[1], bx.hi[2] } };
    o_box fbx = flux_bx;
    fbx.hi[dir] += 1; /* growHi(bx, dir, 1) */
    o_a4 tmp = alloc_fab(ghost_bx, NC * 3);
    o_a4 ffL = sub_fab(tmp, 0, NC), ffR = sub_fab(tmp, NC, NC), half = sub_fab(tmp, 2 * NC, NC);
    o_fill_fluxes(D, dir, ghost_bx, &ffL, cL, parm->adiabatic, parm->epsilon);
    o_fill_fluxes(D, dir, ghost_bx, &ffR, cR, parm->adiabatic, parm->epsilon);
    const int io = dir == 0, jo = dir == 1, ko = dir == 2;
    for (int n = 0; n < NC; ++n)
        for (int k = fbx.lo[2]; k <= fbx.hi[2]; ++k)
            for (int j = fbx.lo[1]; j <= fbx.hi[1]; ++j)
                for (int i = fbx.lo[0]; i <= fbx.hi[0]; ++i) {
                    const double l = *A4(cL, i - io, j - jo, k - ko, n), r = *A4(cR, i, j, k, n);
                    const double fl = *A4(&ffL, i - io, j - jo, k - ko, n), fr = *A4(&ffR, i, j, k, n);
                    *A4(flux, i, j, k, n) = 0.5 * ((0.5 * dx / dt) * (l - r) + 0.5 * (fl + fr));
                    *A4(&half, i, j, k, n) = 0.5 * (l + r) + (dt / (2 * dx)) * (fl - fr);
                }
    o_fill_fluxes(D, dir, fbx, &ffL, &half, parm->adiabatic, parm->epsilon);
    for (int n = 0; n < NC; ++n)
        for (int k = fbx.lo[2]; k <= fbx.hi[2]; ++k)
            for (int j = fbx.lo[1]; j <= fbx.hi[1]; ++j)
                for (int i = fbx.lo[0]; i <= fbx.hi[0]; ++i)
                    *A4(flux, i, j, k, n) += 0.5 * *A4(&ffL, i, j, k, n);
    free(tmp.p);
}

/* compute_LF_flux<dir>, Source/Fluxes/Force.cpp:110-151 */
static void o_lf_flux(int D, int dir, o_box bx, o_a4 *flux, const o_a4 *consv, const double *dx_arr,
                      double dt, const oracle_parm *parm)
{
    const int NC = D + 2;
    const double dx = dx_arr[dir];
    const o_box ghost_bx = grow_all(bx, D, 1);
    const o_box fb = surrounding_nodes(bx, dir);
    o_a4 ff = alloc_fab(ghost_bx, NC);
    o_fill_fluxes(D, dir, ghost_bx, &ff, consv, parm->adiabatic, parm->epsilon);
    const int io = dir == 0, jo = dir == 1, ko = dir == 2;
    for (int n = 0; n < NC; ++n)
        for (int k = fb.lo[2]; k <= fb.hi[2]; ++k)
            for (int j = fb.lo[1]; j <= fb.hi[1]; ++j)
                for (int i = fb.lo[0]; i <= fb.hi[0]; ++i)
                    *A4(flux, i, j, k, n) = 0.5 * dx / dt * (*A4(consv, i - io, j - jo, k - ko, n) - *A4(consv, i, j, k, n))
                                            + 0.5 * (*A4(&ff, i - io, j - jo, k - ko, n) + *A4(&ff, i, j, k, n));
    free(ff.p);
}

/* The Fluxes.H dispatch (Source/Fluxes/Fluxes.H:26-257) over the method enum:
 * compute_MUSCL_hancock_flux (MUSCL_Hancock.cpp:16-52), compute_HLLC_flux
 * (Fluxes.H:192-204), compute_SLIC_flux (SLIC.cpp:12-49), compute_force_flux
 * (Force.cpp:9-20), compute_LF_flux.  bx: valid box; flux covers
 * surroundingNodes(bx, dir).  Returns 0, or -1 for an unsupported method. */
int oracle_compute_flux(int D, int method, int dir, const int *lo, const int *hi, o_a4 flux, o_a4 consv,
                        const double *dx, double dt, const oracle_parm *parm)
{
    o_box bx;
    for (int d = 0; d < 3; ++d) { bx.lo[d] = lo[d]; bx.hi[d] = hi[d]; }
    const int NC = D + 2;
    if (method == M_MUSCL || method == M_SLIC) {
        /* MUSCL: grow(bx,1) in every direction (MUSCL_Hancock.cpp:29);
         * SLIC: grow(bx,dir,1) (SLIC.cpp:24) */
        const o_box gb = method == M_MUSCL ? grow_all(bx, D, 1) : grow_dir(bx, dir, 1);
        o_a4 tmp = alloc_fab(gb, 2 * NC);
        o_a4 hsL = sub_fab(tmp, 0, NC), hsR = sub_fab(tmp, NC, NC);
        o_reconstruct_and_half_time_step(D, dir, gb, &hsL, &hsR, &consv, dx, dt, parm);
        /* reconstructed L/R passed swapped (MUSCL_Hancock.cpp:50-51, SLIC.cpp:45-46) */
        if (method == M_MUSCL)
            o_hllc_flux_LR(D, dir, bx, &flux, &hsR, &hsL, parm);
        else
            o_force_flux_LR(D, dir, bx, &flux, &hsR, &hsL, dx, dt, parm);
        free(tmp.p);
        return 0;
    }
    if (method == M_HLLC) { o_hllc_flux_LR(D, dir, bx, &flux, &consv, &consv, parm); return 0; }
    if (method == M_FORCE) { o_force_flux_LR(D, dir, bx, &flux, &consv, &consv, dx, dt, parm); return 0; }
    if (method == M_LF) { o_lf_flux(D, dir, bx, &flux, &consv, dx, dt, parm); return 0; }
    return -1;
}

/* compute_{HLLC,force}_flux_LR with separate L/R arrays (Fluxes.H:79-87, 179-187).
 * kind: M_HLLC or M_FORCE. */
int oracle_compute_flux_LR(int D, int kind, int dir, const int *lo, const int *hi, o_a4 flux, o_a4 cL,
                           o_a4 cR, const double *dx, double dt, const oracle_parm *parm)
{
    o_box bx;
    for (int d = 0; d < 3; ++d) { bx.lo[d] = lo[d]; bx.hi[d] = hi[d]; }
    if (kind == M_HLLC) { o_hllc_flux_LR(D, dir, bx, &flux, &cL, &cR, parm); return 0; }
    if (kind == M_FORCE) { o_force_flux_LR(D, dir, bx, &flux, &cL, &cR, dx, dt, parm); return 0; }
    return -1;
}

/* The per-sweep conservative update, Source/AmrLevelAdv_advance.cpp:330-341
 * (division form dt / dx[d]). */
void oracle_sweep_update(int D, int dir, const int *lo, const int *hi, o_a4 Uout, o_a4 Uin, o_a4 flux,
                         const double *dx, double dt)
{
    const int NC = D + 2;
    const int io = dir == 0, jo = dir == 1, ko = dir == 2;
    for (int n = 0; n < NC; ++n)
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i)
                    *A4(&Uout, i, j, k, n) = *A4(&Uin, i, j, k, n)
                                             - (dt / dx[dir]) * (*A4(&flux, i + io, j + jo, k + ko, n) - *A4(&flux, i, j, k, n));
}

/* Unsplit box update, Source/Fluxes/Update.H:99-130 (multiplication form dt*idx). */
void oracle_conservative_update(int D, const int *lo, const int *hi, o_a4 out, o_a4 in, const o_a4 *fluxes,
                                double dt, const double *idx)
{
    const int NC = D + 2;
    double dtdx[3];
    for (int d = 0; d < D; ++d) dtdx[d] = dt * idx[d];
    for (int n = 0; n < NC; ++n)
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i) {
                    double v = *A4(&in, i, j, k, n);
                    v = v - dtdx[0] * (*A4(&fluxes[0], i + 1, j, k, n) - *A4(&fluxes[0], i, j, k, n));
                    if (D > 1) v = v - dtdx[1] * (*A4(&fluxes[1], i, j + 1, k, n) - *A4(&fluxes[1], i, j, k, n));
                    if (D > 2) v = v - dtdx[2] * (*A4(&fluxes[2], i, j, k + 1, n) - *A4(&fluxes[2], i, j, k, n));
                    *A4(&out, i, j, k, n) = v;
                }
}

/* ------------------------------------------------------------------ */
/* Level: boxes of one AMR level in one flat buffer                     */
/* ------------------------------------------------------------------ */

typedef struct {
    int D, nboxes, ngrow;
    int dom_lo[3], dom_hi[3];
    int bc_lo[3], bc_hi[3];
    double dx[3];
    const int *boxes;          /* nboxes x 6: lo[3], hi[3] */
    const long long *offsets;  /* nboxes: element offset of each fab */
    const long long *strides;  /* nboxes x 3: jstride, kstride, nstride */
} o_level;

static o_a4 level_fab(const o_level *L, double *buf, int b)
{
    o_a4 a;
    a.p = buf + L->offsets[b];
    a.jstride = L->strides[3 * b];
    a.kstride = L->strides[3 * b + 1];
    a.nstride = L->strides[3 * b + 2];
    for (int d = 0; d < 3; ++d) {
        const int g = d < L->D ? L->ngrow : 0;
        a.begin[d] = L->boxes[6 * b + d] - g;
        a.end[d] = L->boxes[6 * b + 3 + d] + g + 1;
    }
    a.ncomp = L->D + 2;
    return a;
}
static o_box level_box(const o_level *L, int b)
{
    o_box bx;
    for (int d = 0; d < 3; ++d) { bx.lo[d] = L->boxes[6 * b + d]; bx.hi[d] = L->boxes[6 * b + 3 + d]; }
    return bx;
}

/* Cell -> owning box lookup over the domain (built per call). */
static int *build_owner(const o_level *L)
{
    long long nx = L->dom_hi[0] - L->dom_lo[0] + 1, ny = L->dom_hi[1] - L->dom_lo[1] + 1,
              nz = L->dom_hi[2] - L->dom_lo[2] + 1;
    int *own = (int *)malloc(sizeof(int) * (size_t)(nx * ny * nz));
    for (long long c = 0; c < nx * ny * nz; ++c) own[c] = -1;
    for (int b = 0; b < L->nboxes; ++b) {
        o_box bx = level_box(L, b);
        for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
            for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
                for (int i = bx.lo[0]; i <= bx.hi[0]; ++i)
                    own[(i - L->dom_lo[0]) + nx * ((j - L->dom_lo[1]) + ny * (long long)(k - L->dom_lo[2]))] = b;
    }
    return own;
}

/* bamrexBCData::fill_consv_boundary (Source/BoundaryConditions/BCs.cpp:429-442):
 * FillBoundary (intra-level copies, periodic images) followed by PhysBCFunct
 * with the BCRecs of BCs.cpp:215-266: transmissive -> foextrap (ghost takes
 * the nearest interior value), periodic -> int_dir, reflective ->
 * reflect_even for every component and reflect_odd for the normal momentum.
 * Every ghost cell of every fab is filled; a cell outside the domain in
 * several directions has each direction's rule applied. Returns the number of
 * ghost cells that found no owning box (0 on a level that covers the domain). */
int oracle_fill_boundary(const o_level *L, double *buf)
{
    const int D = L->D, NC = D + 2;
    int *own = build_owner(L);
    long long nx = L->dom_hi[0] - L->dom_lo[0] + 1, ny = L->dom_hi[1] - L->dom_lo[1] + 1;
    int missing = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : missing)
    for (int b = 0; b < L->nboxes; ++b) {
        o_a4 dst = level_fab(L, buf, b);
        o_box vb = level_box(L, b);
        for (int k = dst.begin[2]; k < dst.end[2]; ++k)
            for (int j = dst.begin[1]; j < dst.end[1]; ++j)
                for (int i = dst.begin[0]; i < dst.end[0]; ++i) {
                    int c[3] = { i, j, k };
                    if (c[0] >= vb.lo[0] && c[0] <= vb.hi[0] && c[1] >= vb.lo[1] && c[1] <= vb.hi[1]
                        && c[2] >= vb.lo[2] && c[2] <= vb.hi[2])
                        continue;
                    int m[3] = { i, j, k };
                    double sign[O_MAXC];
                    for (int n = 0; n < NC; ++n) sign[n] = 1.0;
                    for (int d = 0; d < D; ++d) {
                        const int lo = L->dom_lo[d], hi = L->dom_hi[d], len = hi - lo + 1;
                        if (m[d] < lo || m[d] > hi) {
                            const int bc = m[d] < lo ? L->bc_lo[d] : L->bc_hi[d];
                            if (bc == BC_PERIODIC) {
                                m[d] = lo + (((m[d] - lo) % len) + len) % len;
                            } else if (bc == BC_TRANSMISSIVE) {
                                m[d] = m[d] < lo ? lo : hi;
                            } else { /* reflective: mirror about the face */
                                m[d] = m[d] < lo ? (2 * lo - 1 - m[d]) : (2 * hi + 1 - m[d]);
                                sign[1 + d] = -sign[1 + d];
                            }
                        }
                    }
                    const int ob = own[(m[0] - L->dom_lo[0]) + nx * ((m[1] - L->dom_lo[1]) + ny * (long long)(m[2] - L->dom_lo[2]))];
                    if (ob < 0) { ++missing; continue; }
                    o_a4 src = level_fab(L, buf, ob);
                    for (int n = 0; n < NC; ++n) *A4(&dst, i, j, k, n) = sign[n] * *A4(&src, m[0], m[1], m[2], n);
                }
    }
    free(own);
    return missing;
}

/* max_wave_speed, Source/System/Euler/Euler.cpp:46-74, over valid cells */
double oracle_max_wave_speed(const o_level *L, double *buf, double adiabatic, double epsilon)
{
    const int D = L->D, NC = D + 2;
    double best = -INFINITY;
#pragma omp parallel for schedule(dynamic) reduction(max : best)
    for (int b = 0; b < L->nboxes; ++b) {
        o_a4 a = level_fab(L, buf, b);
        o_box bx = level_box(L, b);
        double u[O_MAXC], q[O_MAXC];
        for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
            for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
                for (int i = bx.lo[0]; i <= bx.hi[0]; ++i) {
                    load_state(&a, i, j, k, NC, u);
                    oracle_primv_from_consv(D, u, adiabatic, epsilon, q);
                    double vsq = q[1] * q[1];
                    for (int d = 1; d < D; ++d) vsq = vsq + q[1 + d] * q[1 + d];
                    const double velocity = sqrt(vsq);
                    const double w = sqrt(adiabatic * q[1 + D] / (q[0] * epsilon)) + velocity;
                    if (w > best) best = w;
                }
    }
    return best;
}

/* AmrLevelAdv::estTimeStep for the explicit methods (Source/AmrLevelAdv.cpp:395-477)
 * -> FluidSystem::ExplicitTimeStepDimSplit (Source/System/FluidSystem.cpp:194-206). */
double oracle_est_time_step(const o_level *L, double *buf, double adiabatic, double epsilon, double cfl)
{
    const double max_speed = oracle_max_wave_speed(L, buf, adiabatic, epsilon);
    double dt_est = 1.0e20;
    for (int d = 0; d < L->D; ++d) {
        const double v = L->dx[d] / max_speed;
        dt_est = v < dt_est ? v : dt_est;
    }
    return dt_est * cfl;
}

/* AmrLevelAdv::advance_explicit, Source/AmrLevelAdv_advance.cpp:261-360, with
 * S1 the ghost-filled input (Sborder) and S2 a second buffer with the same
 * layout (Sborder2, a copy of S1 on entry).  Box loops run in parallel as the
 * reference's OpenMP MFIter loop (:284-290).  The result is left in S1
 * (valid cells; the reference copies it to S_new at :438).  If flux_out is
 * non-null, flux_out[d] receives the fluxes of sweep d (level flux layout:
 * per box surroundingNodes(bx,d) with offsets flux_off[d][b] and strides
 * flux_str[d][3b..3b+2]).  Returns 0 on success. */
int oracle_advance_explicit(const o_level *L, double *S1, double *S2, double time, double dt, int method,
                            const oracle_parm *parm, double *const *flux_out, const long long *const *flux_off,
                            const long long *const *flux_str, int nthreads)
{
    (void)time;
    const int D = L->D, NC = D + 2;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    double *MFin = S1, *MFout = S2;
    int err = 0;
    for (int d = 0; d < D; ++d) {
#pragma omp parallel for schedule(dynamic) reduction(| : err)
        for (int b = 0; b < L->nboxes; ++b) {
            o_box bx = level_box(L, b);
            o_a4 Uin = level_fab(L, MFin, b), Uout = level_fab(L, MFout, b);
            o_box fb = surrounding_nodes(bx, d);
            o_a4 flux;
            int own_flux = 0;
            if (flux_out && flux_out[d]) {
                flux.p = flux_out[d] + flux_off[d][b];
                flux.jstride = flux_str[d][3 * b];
                flux.kstride = flux_str[d][3 * b + 1];
                flux.nstride = flux_str[d][3 * b + 2];
                for (int q = 0; q < 3; ++q) { flux.begin[q] = fb.lo[q]; flux.end[q] = fb.hi[q] + 1; }
                flux.ncomp = NC;
            } else {
                flux = alloc_fab(fb, NC);
                own_flux = 1;
            }
            if (oracle_compute_flux(D, method, d, bx.lo, bx.hi, flux, Uin, L->dx, dt, parm) != 0) err |= 1;
            oracle_sweep_update(D, d, bx.lo, bx.hi, Uout, Uin, flux, L->dx, dt);
            if (own_flux) free(flux.p);
        }
        oracle_fill_boundary(L, MFout);
        double *t = MFin; MFin = MFout; MFout = t;
    }
    if (MFin != S1) {
        /* MultiFab::Copy(S_new, *MFin, ...) with S_new := S1 (valid + ghosts). */
#pragma omp parallel for schedule(dynamic)
        for (int b = 0; b < L->nboxes; ++b) {
            o_a4 src = level_fab(L, MFin, b), dst = level_fab(L, S1, b);
            const long long n = (long long)src.nstride * NC;
            memcpy(dst.p, src.p, sizeof(double) * (size_t)n);
        }
    }
    return err;
}

/* One sweep of advance_explicit (Source/AmrLevelAdv_advance.cpp:290-341) in
 * direction d over every box: Sout's valid cells from Sin (ghost-filled).
 * Ghost cells of Sout are not touched. */
int oracle_sweep_dir(const o_level *L, const double *Sin, double *Sout, int d, double dt, int method,
                     const oracle_parm *parm)
{
    const int D = L->D, NC = D + 2;
    int err = 0;
#pragma omp parallel for schedule(dynamic) reduction(| : err)
    for (int b = 0; b < L->nboxes; ++b) {
        o_box bx = level_box(L, b);
        o_a4 Uin = level_fab(L, (double *)Sin, b), Uout = level_fab(L, Sout, b);
        o_box fb = surrounding_nodes(bx, d);
        o_a4 flux = alloc_fab(fb, NC);
        if (oracle_compute_flux(D, method, d, bx.lo, bx.hi, flux, Uin, L->dx, dt, parm) != 0) err |= 1;
        oracle_sweep_update(D, d, bx.lo, bx.hi, Uout, Uin, flux, L->dx, dt);
        free(flux.p);
    }
    return err;
}

int oracle_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
