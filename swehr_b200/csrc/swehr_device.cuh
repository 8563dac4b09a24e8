/*
 * swehr_device.cuh -- FP64 per-face and per-cell arithmetic of the SWEHR time
 * step (csdms-contrib/swehr SWEHR.c:808-1591), shared by every FP64 kernel.
 *
 * Each function keeps the reference's operation order (a*b/c is (a*b)/c,
 * sums left to right) and takes its elementary functions from swehr_math.h,
 * so with FP contraction off (--fmad=false) the results are bit-identical to
 * the CPU restatement built with the same math.
 *
 * Device layout: every field is a plane of nx rows (index i) by `pitch`
 * doubles (index j, contiguous, pitch a multiple of 32), cell (i,j) (1-based)
 * at [(i-1)*pitch + (j-1)].  A state set holds NP = 10 + 2S planes:
 *   h hu hv vinf maxvel maxdepth totm dep totsed gz | U_1..U_S | M_1..M_S
 * Two sets alternate between steps; the topography has three planes
 * (z of the previous, current and next step) so the lagged slopes the
 * reference's serial sweep reads (SWEHR.c:1135,1203,1243,1293,1304) can be
 * recomputed from the previous step's z.  gz of a set is the GZ the wave
 * pass of the step reading that set uses (SWEHR.c:1279 one step late): the
 * update writes it with the rest of the new state.
 */
#pragma once
#include <stdint.h>

#include "swehr_math.h"

namespace swehr {

enum { P_H = 0, P_HU, P_HV, P_VINF, P_MAXVEL, P_MAXDEP, P_TOTM, P_DEP, P_TOTSED, P_GZ, P_FIXED };

/* Real-valued constants of the step in the arithmetic type R of a form
 * (double for the plain form, float for the mixed form's bulk). */
template <class R>
struct RealC {
    R g, hfilm, hfx10, rhos, rhow, rho0, porod, oneoverdx, half_odx;
    R fa, cohesion, neg1ml, cthreshold, one_m_bb, hc, dde, b, af, afr;
    R h0, h0x3, h0x6, h0x9, mtstar0, a, ad, F, J, roughness, uc, uc2, c109s, rhos08;
    R ds[16], pf[16], a13[16], a13sq[16];
};

struct DevParams {
    int32_t nx, ny, S, pitch;
    int32_t rnum, inflow, storm, budget;
    int32_t bndry[4];
    int32_t outlet_row, npoints, xpoint[6], ypoint[6];
    int32_t has_ks, has_solid;   /* per-cell Ks plane; interior solid mask (SOLID, SWEHR.c:597) */
    /* rows this context updates (1-based, local): 1..nx for a whole domain;
     * a slab of a larger domain holds up to two neighbour rows on each inner
     * side that it reads but does not update.  row0: global row of local row
     * 0 (positions of the moving storm).  slab: the CFL time step waits for
     * the largest wave speed over every slab (k_slab_finalize). */
    int32_t own_lo, own_hi, row0, slab;
    int64_t plane;        /* doubles per plane (>= nx*pitch, multiple of 32) */
    double dx, oneoverdx, half_odx, tend, rint, stageint;
    double g, hfilm, hfx10, rhos, rhow, rho0, porod, invporo;
    double nu, fa, cohesion, neg1ml, cthreshold, one_m_bb, hc, dde, b, af, afr;
    double h0, h0x3, h0x6, h0x9, mtstar0, a, ad, F, J;
    double roughness, ks, theta0, thetas, hf, uc, uc2, cstable, maxstep;
    double c109s;         /* 1.09*(rhos/rhow-1), settlingvelocity (SWEHR.c:433-435) */
    double rhos08;        /* 0.8*rhos */
    double inv_rhos;      /* 1/rhos (the mixed form's deposited thickness) */
    /* correctly rounded reciprocals of the constant divisors J, 6 h0, 0.2 and
     * thetas - theta0, for exact division by remainder correction (divk);
     * divk_ok: every constant divisor lies in [2^-100, 2^100] */
    double inv_J, inv_h0x6, inv_p2, inv_dtheta;
    int32_t divk_ok, pad_divk;
    double storm_peak, storm_r2, storm_x0, storm_y0, storm_vx, storm_vy;
    double ds[16], pf[16], a13[16], a13sq[16];
    RealC<double> kd;     /* the constants above, for templated kernels */
    RealC<float> kf;      /* the same, rounded to float, for the mixed form */
};

template <class R>
__device__ __forceinline__ const RealC<R> &kc(const DevParams &P);
template <>
__device__ __forceinline__ const RealC<double> &kc<double>(const DevParams &P) { return P.kd; }
template <>
__device__ __forceinline__ const RealC<float> &kc<float>(const DevParams &P) { return P.kf; }

/* Device control block of one simulation (one per scenario). */
/* host-visible progress of one scenario of a batch, written when it ends a step */
struct ScenSummary {
    double t, dt, courant;
    int64_t step;
    int32_t status, active;
};

struct Ctl {
    double t;             /* time at the start of the pending step */
    double dt, courant;   /* time step of the pending step */
    double t_stop;
    int64_t step;         /* completed steps */
    int64_t max_step;     /* stop once step reaches this */
    unsigned long long smax_bits;
    uint32_t wave_ticket, update_ticket;
    int32_t active;       /* 1 while steps remain */
    int32_t pending;      /* 1 between the wave pass and the update pass of a step */
    int32_t cfl;          /* Courant > 1 seen on the pending step */
    int32_t status;
    double stageinterval;
    int64_t stagecnt, stagecap;
    int64_t launches;
    double budget_hi[64], budget_lo[64];   /* running compensated budget sums */
    double budget_step[64];                 /* this step's partials in batched mode */
    double rain_now;                        /* uniform rain rate of the current / last step */
    double t_prev;                          /* start time of the last completed step */
    double sed0[16];
    int32_t dev_error;                      /* a bounded device-side wait gave up (SWEHR_TIMEOUT) */
    int32_t pad_err;
};

/* budget term slots */
enum {
    B_RAIN = 0, B_OUT, B_CLAMP, B_BULK, B_INF,
    B_ROUND,                  /* storage/arithmetic rounding of h (the mixed form's FP32 representation) */
    B_DET = 6,                /* + class */
    B_SOUT = 6 + 16,          /* + class */
    B_SROUND = 6 + 32,        /* + class: rounding of U_k + M_k */
    B_NTERMS = 6 + 48
};

__device__ __forceinline__ int64_t cidx(const DevParams &P, int i, int j)
{
    return (int64_t)(i - 1) * P.pitch + (j - 1);
}

/* hllc, SWEHR.c:327-409.  Writes T[0..2] and returns max |wave speed|. */
__device__ __forceinline__ double hllc(double hl, double hr, double uhl, double uhr, double vhl, double vhr,
                                       double g, double hfilm, double &T0, double &T1, double &T2)
{
    double ul = 0, vl = 0, ur = 0, vr = 0;
    if (hl > hfilm) { ul = uhl / hl; vl = vhl / hl; }
    if (hr > hfilm) { ur = uhr / hr; vr = vhr / hr; }
    double cl = sw_sqrt_pow(g * hl), cr = sw_sqrt_pow(g * hr);
    double d = ul + 2 * cl - ur - 2 * cr;
    double hs = (d * d) / (16 * g);
    double us = .5 * (ul + ur) + cl - cr;
    double cs = sw_sqrt_pow(g * hs);
    double sl = ul - cl;
    if (us - cs < sl) sl = us - cs;
    double sm = us;
    double sr = ur + cr;
    if (us + cs > sr) sr = us + cs;
    if (hl <= hfilm) { sl = ur - 2 * cr; sm = sl; sr = ur + cr; }
    if (hr <= hfilm) { sl = ul - cl; sr = ul + 2 * cl; sm = sr; }
    double f0 = __longlong_as_double(0x7ff8000000000000LL), f1 = f0;
    if (sl >= 0) {
        f0 = hl * ul;
        f1 = hl * ul * ul + .5 * g * hl * hl;
    }
    if (sl <= 0 && sr >= 0) {
        f0 = (sr * (hl * ul) - sl * (hr * ur) + sl * sr * (hr - hl)) / (sr - sl);
        f1 = (sr * (hl * ul * ul + .5 * g * hl * hl) - sl * (hr * ur * ur + .5 * g * hr * hr)
              + sl * sr * (hr * ur - hl * ul)) / (sr - sl);
    }
    if (sr <= 0) {
        f0 = hr * ur;
        f1 = hr * ur * ur + .5 * g * hr * hr;
    }
    T0 = f0;
    T1 = f1;
    T2 = (sm >= 0) ? f0 * vl : f0 * vr;
    double s = 0;
    if (fabs(sl) > s) s = fabs(sl);
    if (fabs(sr) > s) s = fabs(sr);
    if (fabs(sm) > s) s = fabs(sm);
    return s;
}

/* SOLID[i][j] as the reference's sweeps read it (m: the nx x pitch byte
 * mask): inside the grid the mask; at j = ny+1 -- the y-face test at
 * SWEHR.c:1206,1211 reads one column past the row -- the next row's first
 * cell SOLID[i+1][1], and 0 past the last row; 0 elsewhere. */
__device__ __forceinline__ bool solid_at(const DevParams &P, const uint8_t *__restrict__ m, int i, int j)
{
    if (i < 1 || i > P.nx || j < 1) return false;
    if (j <= P.ny) return m[cidx(P, i, j)] != 0;
    if (j == P.ny + 1 && i < P.nx) return m[cidx(P, i + 1, 1)] != 0;
    return false;
}

/* SWEHR.c:1240-1257 */
__device__ __forceinline__ double slope_x(const DevParams &P, const double *__restrict__ z, int i, int j)
{
    if (i != 1 && i != P.nx) return P.half_odx * (z[cidx(P, i + 1, j)] - z[cidx(P, i - 1, j)]);
    if (i == P.nx) return P.oneoverdx * (z[cidx(P, i, j)] - z[cidx(P, i - 1, j)]);
    return P.oneoverdx * (z[cidx(P, i + 1, j)] - z[cidx(P, i, j)]);
}

/* SWEHR.c:1260-1277 */
__device__ __forceinline__ double slope_y(const DevParams &P, const double *__restrict__ z, int i, int j)
{
    if (j != 1 && j != P.ny) return P.half_odx * (z[cidx(P, i, j + 1)] - z[cidx(P, i, j - 1)]);
    if (j == P.ny) return P.oneoverdx * (z[cidx(P, i, j)] - z[cidx(P, i, j - 1)]);
    return P.oneoverdx * (z[cidx(P, i, j + 1)] - z[cidx(P, i, j)]);
}

/* GZ of a cell computed from a topography plane (SWEHR.c:1279, 764) */
__device__ __forceinline__ double gz_of(const DevParams &P, const double *__restrict__ z, int i, int j)
{
    double sx = slope_x(P, z, i, j), sy = slope_y(P, z, i, j);
    return P.g / sw_sqrt_pow(sx * sx + sy * sy + 1);
}

/* uniform rain, SWEHR.c:813-814 */
__device__ __forceinline__ double rain_at(const DevParams &P, const double *__restrict__ rain, double t)
{
    int rind = (int)fmin(ceil(t / P.rint + 0.01), (double)P.rnum);
    return rain[rind - 1];
}

/* hard-wired inflow ghost at j = ny+1, SWEHR.c:1019-1034 */
__device__ __forceinline__ void inflow_ghost(double t, double &h, double &hv, double &sed)
{
    double vin = fmax(-0.035, t / 100 * -0.035);
    double hin = sw_pow(fabs(vin) * 0.045 / sw_sqrt_pow(0.7), 0.6);
    double ukin = fmin(500.0, t / 100 * 500) * hin;
    h = hin;
    hv = vin;
    sed = ukin / hin;
}

/* Budget accumulation in double-double (two-sum). */
__device__ __forceinline__ void dd_add(double &hi, double &lo, double x)
{
    double s = hi + x;
    double bb = s - hi;
    double e = (hi - (s - bb)) + (x - bb);
    hi = s;
    lo += e;
}

}  // namespace swehr
