/*
 * swehr_step_f64.cu -- the plain FP64 form of one SWEHR time step on sm_100a.
 * Compiled with --fmad=false: no contraction, so every cell is bit-identical
 * to the CPU restatement built with the project's math.
 *
 * A step is two stream-ordered launches and needs no grid barrier:
 *   wave   : largest wave speed over every face (SWEHR.c:1092-1230's Smax),
 *            block max -> atomicMax; the last block to finish computes dt,
 *            the Courant check (SWEHR.c:1409-1413) and arms the update.
 *   update : per cell, the four face fluxes, the sources (SWEHR.c:1233-1401)
 *            and the update (SWEHR.c:1417-1588), reading set n%2 and writing
 *            set (n+1)%2; the last block sums the budget partials, advances
 *            t and the step counter, records a stage row when one is due
 *            (SWEHR.c:1593-1676) and disarms stepping at t >= tend, t_stop,
 *            the step limit or a CFL error.
 * Both kernels read the step counter from the control block to pick their
 * buffers, so every step is the same pair of launches and a chunk of steps
 * is captured once as a CUDA graph.  Nothing spins or waits on the device.
 */
#include <cuda_runtime.h>

#include "swehr_device.cuh"
#include "swehr_faces.cuh"
#include "swehr_kernels.h"

namespace swehr {

/* ------------------------------------------------------------- wave --- */
__global__ void __launch_bounds__(NB_THREADS) k_wave(const DevParams P, const Bufs B, Ctl *ctl)
{
    if (!ctl->active) return;
    const int64_t n = ctl->step;
    const double t = ctl->t;
    const double *src = B.set[n & 1];
    const double *zp = B.z[(n + 2) % 3];
    double inh = 0, inhv = 0, insed = 0;
    if (P.inflow) inflow_ghost(t, inh, inhv, insed);
    const int64_t total = (int64_t)P.nx * P.ny;
    double smax = 0;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < total; c += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(c / P.ny) + 1, j = (int)(c % P.ny) + 1;
        Face f;
        double s = face_x(P, src, zp, i, j, f);
        if (s > smax) smax = s;
        s = face_y(P, src, zp, i, j, inh, inhv, f);
        if (s > smax) smax = s;
        if (i == 1) {
            s = face_x(P, src, zp, 0, j, f);
            if (s > smax) smax = s;
        }
        if (j == 1) {
            s = face_y(P, src, zp, i, 0, inh, inhv, f);
            if (s > smax) smax = s;
        }
    }
    __shared__ double red[NB_THREADS / 32];
    __shared__ bool last;
    smax = warp_max(smax);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = smax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0;
        for (int w = 0; w < NB_THREADS / 32; w++) m = (red[w] > m) ? red[w] : m;
        atomicMax(&ctl->smax_bits, (unsigned long long)__double_as_longlong(m));
        __threadfence();
        unsigned tk = atomicAdd(&ctl->wave_ticket, 1u);
        last = (tk == gridDim.x - 1);
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    /* CFL time step, SWEHR.c:1409-1413 */
    double Smax = __longlong_as_double((long long)atomicAdd(&ctl->smax_bits, 0ull));
    double dt = P.cstable * P.dx / Smax;
    if (dt > P.maxstep) dt = P.maxstep;
    if (t + dt > P.tend) dt = P.tend - t;
    double courant = Smax * dt * P.oneoverdx;
    ctl->dt = dt;
    ctl->courant = courant;
    ctl->cfl = courant > 1;
    ctl->smax_bits = 0ull;
    ctl->wave_ticket = 0u;
    ctl->pending = 1;
}

/* ----------------------------------------------------------- update --- */
template <int MAXS>
struct Acc {
    double rain, out, clamp, bulk, inf;
    double det[MAXS], sout[MAXS];
};

template <int MAXS>
__device__ __forceinline__ void update_cell(const DevParams &P, const double *__restrict__ src,
                                            double *__restrict__ dst, const double *__restrict__ zp,
                                            const double *__restrict__ zc, double *__restrict__ zn,
                                            const double *__restrict__ ksf, int i, int j, double t, double dt,
                                            double Rr, double inh, double inhv, double insed, Acc<MAXS> &acc)
{
    const int64_t pl = P.plane;
    const int64_t q = cidx(P, i, j);
    const int S = P.S;
    const double hfilm = P.hfilm, rhos = P.rhos, rhow = P.rhow;
    const double h0v = src[P_H * pl + q], hu0 = src[P_HU * pl + q], hv0 = src[P_HV * pl + q];
    const double totsed0 = src[P_TOTSED * pl + q], totm0 = src[P_TOTM * pl + q], dep0 = src[P_DEP * pl + q];
    double rho0c = rhow * (1 - totsed0) + rhos * totsed0;
    if (rho0c > P.rhos08) rho0c = P.rhos08;
    const double Rc = P.storm ? storm_at(P, t, i, j) : Rr;

    /* four faces */
    Face fxl, fxr, fyl, fyr;
    face_x(P, src, zp, i - 1, j, fxl);
    face_x(P, src, zp, i, j, fxr);
    face_y(P, src, zp, i, j - 1, inh, inhv, fyl);
    face_y(P, src, zp, i, j, inh, inhv, fyr);

    /* sources, SWEHR.c:1239-1320 */
    const double g = P.g;
    const double sx = slope_x(P, zc, i, j), sy = slope_y(P, zc, i, j);
    const double syl = slope_y(P, zp, i, j);
    const double gx = g * sx / sw_sqrt_pow(sx * sx + syl * syl + 1);
    const double SXf = -gx * h0v;
    const double gy = g * sy / sw_sqrt_pow(sx * sx + sy * sy + 1);
    const double SYf = -gy * h0v;
    const double gz = g / sw_sqrt_pow(sx * sx + sy * sy + 1);
    const double slope = sw_sqrt_pow(sx * sx + sy * sy);
    double gammax = 0, gammay = 0;
    if (i > 1 && i < P.nx)
        gammax -= (rhos - rho0c) * gz * h0v * h0v / (2 * rho0c) * .5 * P.oneoverdx
                  * (src[P_TOTSED * pl + cidx(P, i + 1, j)] - src[P_TOTSED * pl + cidx(P, i - 1, j)]);
    if (j > 1 && j < P.ny)
        gammay -= (rhos - rho0c) * gz * h0v * h0v / (2 * rho0c) * .5 * P.oneoverdx
                  * (src[P_TOTSED * pl + cidx(P, i, j + 1)] - src[P_TOTSED * pl + cidx(P, i, j - 1)]);
    /* slope stability, SWEHR.c:1292-1312 */
    double fail = 0;
    {
        const int iu = (i < P.nx) ? i + 1 : P.nx, id = (i > 1) ? i - 1 : 1;
        const int ju = (j < P.ny) ? j + 1 : P.ny, jd = (j > 1) ? j - 1 : 1;
        const double sxu = (iu == i) ? sx : slope_x(P, zp, iu, j);
        const double sxd = (id == i) ? sx : slope_x(P, zc, id, j);
        const double syu = (ju == j) ? sy : slope_y(P, zp, i, ju);
        const double syd = (jd == j) ? sy : slope_y(P, zc, i, jd);
        const double rho0 = P.rho0;
        double pgfx = dep0 * rho0 * gz * 0.5 * P.oneoverdx
                      * (src[P_DEP * pl + cidx(P, iu, j)] * sw_cos_atan(fabs(sxu))
                         - src[P_DEP * pl + cidx(P, id, j)] * sw_cos_atan(fabs(sxd)));
        if (pgfx * sx > 0) pgfx = -1 * fabs(pgfx);
        if (pgfx * sx < 0) pgfx = fabs(pgfx);
        const double lhs = (rho0 * gz * dep0 + rho0c * gz * h0v) * sw_sin_atan(fabs(sy));
        const double nrm = (rho0 * gz * dep0 + rho0c * gz * h0v) * sw_cos_atan(fabs(sy)) - rhow * gz * (dep0 + h0v);
        if (fail == 0 && (lhs > (P.cohesion + nrm * P.fa + pgfx))) fail = 1;
        double pgfy = dep0 * rho0 * gz * 0.5 * P.oneoverdx
                      * (src[P_DEP * pl + cidx(P, i, ju)] * sw_cos_atan(fabs(syu))
                         - src[P_DEP * pl + cidx(P, i, jd)] * sw_cos_atan(fabs(syd)));
        if (pgfy * sy > 0) pgfy = -1 * fabs(pgfy);
        if (pgfy * sy < 0) pgfy = fabs(pgfy);
        if (fail == 0 && (lhs > (P.cohesion + nrm * P.fa + pgfy))) fail = 1;
    }
    double dfmask = fmin(1.0, (totsed0 - 0.2) / 0.2);
    if (h0v < P.h0x9 || totsed0 < 0.2) dfmask = 0;
    double betax = P.neg1ml * gz * h0v * P.fa;
    double betay = P.neg1ml * gz * h0v * P.fa;
    if (hu0 < 0) betax = -1 * betax;
    if (hv0 < 0) betay = -1 * betay;

    /* Hairsine-Rose, class-independent parts (SWEHR.c:1330-1360, 1382) */
    const double hvert = h0v / sw_cos_atan(fabs(slope));
    double mtstar = P.mtstar0;
    const bool deepv = hvert > P.h0;
    double depthfac = 1.0;
    if (deepv) {
        depthfac = sw_pow(P.h0 / hvert, P.b);
        mtstar = P.mtstar0 * depthfac;
    }
    const double Hs = fmin(1.0, totm0 / mtstar);
    const bool swash = (h0v > P.hfx10 && totsed0 < 0.6);
    double SF = 0;
    if (swash) {
        double manning = (h0v <= P.hc) ? P.roughness * sw_pow(h0v / P.hc, P.dde) : P.roughness;
        double qq = sw_sqrt_pow(hu0 * hu0 + hv0 * hv0);
        SF = manning * manning * qq * qq / sw_pow(h0v, 3.333);
    }
    const double vfconc = sw_pow(1 - fmin(totsed0, 0.99), 4.0);
    const bool debris = (h0v > P.h0x9 && totsed0 > P.cthreshold);

    /* conservative update + Green-Ampt, SWEHR.c:1424-1452 */
    const double dtdx = dt * P.oneoverdx;
    double h = h0v - dtdx * (fxr.F0 - fxl.F0) - dtdx * (fyr.F0 - fyl.F0) + dt * Rc;
    double hu = hu0 - dtdx * (fxr.Fu - fxl.Fu) - dtdx * (fyr.Fu - fyl.Fu) + dt * SXf + dt * gammax + dt * dfmask * betax;
    double hv = hv0 - dtdx * (fxr.Fv - fxl.Fv) - dtdx * (fyr.Fv - fyl.Fv) + dt * SYf + dt * gammay + dt * dfmask * betay;
    const double ks = P.has_ks ? ksf[q] : P.ks;
    const double vinf0 = src[P_VINF * pl + q];
    const double zf = vinf0 / (P.thetas - P.theta0);
    const double infl = fmin(h - hfilm, dt * ks * (zf + P.hf + h) / zf);
    const double vinf = vinf0 + infl;
    h -= infl;

    /* classes: advection, exchange with the deposited layer (SWEHR.c:1454-1511) */
    double Uk[MAXS];
    double z = zc[q];
    double totm = 0, dep = 0, chtemp = 0, bulk = 0;
#pragma unroll
    for (int k = 0; k < MAXS; k++) {
        if (k >= S) break;
        const int64_t qk = (P_FIXED + k) * pl + q;
        double u = src[qk] - dtdx * (fxr.F0 * face_sed(P, src, fxr, k, insed) - fxl.F0 * face_sed(P, src, fxl, k, insed))
                   - dtdx * (fyr.F0 * face_sed(P, src, fyr, k, insed) - fyl.F0 * face_sed(P, src, fyl, k, insed));
        Uk[k] = u;
    }
#pragma unroll
    for (int k = 0; k < MAXS; k++) {
        if (k >= S) break;
        const int64_t qm = (P_FIXED + S + k) * pl + q;
        const double Mk0 = src[qm];
        /* sources of class k from the state at the start of the step (SWEHR.c:1324-1399) */
        double E1 = 0, E2 = 0, E3 = 0, E4 = 0;
        if (swash) {
            E1 = (1 - Hs) * P.pf[k] * P.a * Rc;
            if (totm0 > 1e-8 && Mk0 > 1e-8) E2 = Hs * Mk0 / totm0 * P.ad * Rc;
            if (deepv) { E1 = E1 * depthfac; E2 = E2 * depthfac; }
            E3 = spe(hu0, hv0, h0v, P.af, rho0c, gz, totsed0, SF, P.ds[k], P.uc);
            E3 = (1 - Hs) * P.pf[k] * P.F / P.J * E3;
            if (totm0 > 1e-6 && Mk0 > 0) {
                E4 = spe(hu0, hv0, h0v, P.afr, rho0c, gz, totsed0, SF, P.ds[k], P.uc2);
                E4 = P.one_m_bb * Hs * Mk0 / totm0 * P.F / ((rhos - rho0c) / rhos * gz * h0v) * E4;
            }
        }
        double VF = sw_sqrt_pow(P.a13sq[k] + P.c109s * gz * P.ds[k]) - P.a13[k];
        VF = VF * vfconc;
        if (P.ds[k] > 0.0001 && h0v < P.h0x9) VF = 2e-3 + fmax(h0v - P.h0x3, 0.0) * (VF - 2e-3) / P.h0x6;
        if (P.ds[k] > 0.002 && h0v < P.h0x9) VF = 2e-3 + fmax(h0v - P.h0x3, 0.0) * (VF - 2e-3) / P.h0x6;
        if (debris) { E1 = E2 = E3 = E4 = 0; VF = 0; }

        double Mk = Mk0;
        double u = Uk[k];
        if (h < P.hfx10) {
            Mk += dt * E1 + u;
            u = 0;
            acc.det[k] += dt * E1;
        } else {
            chtemp = u;
            const double redetach = fmin(Mk, dt * (E2 + E4));
            const double dec = sw_exp(-VF / h * (0.5 * dt));
            u = dec * u;
            u = u + dt * (E1 + E3) + redetach;
            u = dec * u;
            z = z - P.invporo * (u - chtemp);
            Mk = Mk + dt * (E1 + E3) - (u - chtemp);
            acc.det[k] += dt * (E1 + E3);
            if (fail == 1) {
                z = z - 0.99 * Mk / P.porod;
                u = u + 0.99 * Mk;
                totm = 0;
                Mk = 0.01 * Mk;
                dep = 0;
            }
        }
        const double dh = (u - chtemp) / P.porod;
        h = h + dh;
        bulk += dh;
        totm += Mk;
        dep += Mk / rhos;
        Uk[k] = u;
        dst[qm] = Mk;
    }

    /* derived fields and the dry clamp, SWEHR.c:1513-1551 */
    double totsed = 0, clamp = 0;
    if (h > hfilm) {
#pragma unroll
        for (int k = 0; k < MAXS; k++) {
            if (k >= S) break;
            totsed += (Uk[k] / h) / rhos;
            dst[(P_FIXED + k) * pl + q] = Uk[k];
        }
    } else {
        clamp = hfilm - h;
        h = hfilm;
        hu = 0;
        hv = 0;
#pragma unroll
        for (int k = 0; k < MAXS; k++) {
            if (k >= S) break;
            const int64_t qm = (P_FIXED + S + k) * pl + q;
            z = z + P.invporo * Uk[k];
            dst[qm] = dst[qm] + Uk[k];
            dst[(P_FIXED + k) * pl + q] = 0.0;
        }
    }
    /* implicit friction, SWEHR.c:1553-1565 */
    double vel1 = 0, vel2 = 0;
    if (h > hfilm) {
        double manning = (h <= P.hc) ? P.roughness * sw_pow(h / P.hc, P.dde) : P.roughness;
        double SFf = manning * manning * gz * sw_sqrt_pow(hu * hu + hv * hv) * 1 / sw_pow(h, 2.333);
        hu = hu / (1 + dt * SFf);
        hv = hv / (1 + dt * SFf);
        vel1 = hu / h;
        vel2 = hv / h;
    }
    /* maxima, SWEHR.c:1578-1588 (RHO is recomputed from TOTSED when read) */
    double maxvel = src[P_MAXVEL * pl + q], maxdep = src[P_MAXDEP * pl + q];
    const double vmag = sw_sqrt_pow(vel1 * vel1 + vel2 * vel2);
    if (vmag > maxvel) maxvel = vmag;
    if (h > maxdep) maxdep = h;
    dst[P_H * pl + q] = h;
    dst[P_HU * pl + q] = hu;
    dst[P_HV * pl + q] = hv;
    dst[P_VINF * pl + q] = vinf;
    dst[P_MAXVEL * pl + q] = maxvel;
    dst[P_MAXDEP * pl + q] = maxdep;
    dst[P_TOTM * pl + q] = totm;
    dst[P_DEP * pl + q] = dep;
    dst[P_TOTSED * pl + q] = totsed;
    zn[q] = z;

    acc.rain += dt * Rc;
    acc.inf += infl;
    acc.clamp += clamp;
    acc.bulk += bulk;
    /* boundary faces carry water and sediment out of the domain */
    if (i == 1) {
        acc.out -= dtdx * fxl.F0;
        for (int k = 0; k < S && k < MAXS; k++) acc.sout[k] -= dtdx * (fxl.F0 * face_sed(P, src, fxl, k, insed));
    }
    if (i == P.nx) {
        acc.out += dtdx * fxr.F0;
        for (int k = 0; k < S && k < MAXS; k++) acc.sout[k] += dtdx * (fxr.F0 * face_sed(P, src, fxr, k, insed));
    }
    if (j == 1) {
        acc.out -= dtdx * fyl.F0;
        for (int k = 0; k < S && k < MAXS; k++) acc.sout[k] -= dtdx * (fyl.F0 * face_sed(P, src, fyl, k, insed));
    }
    if (j == P.ny) {
        acc.out += dtdx * fyr.F0;
        for (int k = 0; k < S && k < MAXS; k++) acc.sout[k] += dtdx * (fyr.F0 * face_sed(P, src, fyr, k, insed));
    }
}

/* stage row of SWEHR.c:1593-1676 from the new state (one block) */
__device__ void stage_sample(const DevParams &P, const double *__restrict__ st, Ctl *ctl, double tnew,
                             double *stage, double *saveflow)
{
    __shared__ double bv[NB_THREADS];
    __shared__ int bi[NB_THREADS];
    const int64_t pl = P.plane;
    const int row = P.outlet_row;
    double best = 0;
    int besti = 1;
    for (int i = 1 + threadIdx.x; i <= P.nx; i += blockDim.x) {
        double h = st[P_H * pl + cidx(P, i, row)];
        if (h > best) { best = h; besti = i; }
    }
    bv[threadIdx.x] = best;
    bi[threadIdx.x] = besti;
    __syncthreads();
    if (threadIdx.x != 0) return;
    int outlet = 1;
    double ob = 0;
    for (int w = 0; w < (int)blockDim.x; w++) {
        if (bv[w] > ob || (bv[w] == ob && bv[w] > 0 && bi[w] < outlet)) { ob = bv[w]; outlet = bi[w]; }
    }
    int64_t r = ctl->stagecnt;
    double *row_out = stage + r * 24;
    int64_t qo = cidx(P, outlet, row);
    double ho = st[P_H * pl + qo];
    double v1 = ho > P.hfilm ? st[P_HU * pl + qo] / ho : 0, v2 = ho > P.hfilm ? st[P_HV * pl + qo] / ho : 0;
    row_out[0] = tnew;
    row_out[1] = ho;
    row_out[2] = sw_sqrt_pow(v1 * v1 + v2 * v2);
    row_out[3] = st[P_TOTSED * pl + qo];
    for (int k = 0; k < 10; k++) {
        row_out[4 + k] = (k < P.S) ? st[(P_FIXED + P.S + k) * pl + qo] : 0;
        row_out[14 + k] = (k < P.S) ? st[(P_FIXED + k) * pl + qo] : 0;
    }
    double *pr = saveflow + r * 18;
    for (int m = 0; m < 6; m++) {
        int xi = P.xpoint[m], yj = P.ypoint[m];
        if (m >= P.npoints || xi < 1 || xi > P.nx || yj < 1 || yj > P.ny) {
            pr[3 * m] = pr[3 * m + 1] = pr[3 * m + 2] = __longlong_as_double(0x7ff8000000000000LL);
            continue;
        }
        int64_t qp = cidx(P, xi, yj);
        double hp = st[P_H * pl + qp];
        double w1 = hp > P.hfilm ? st[P_HU * pl + qp] / hp : 0, w2 = hp > P.hfilm ? st[P_HV * pl + qp] / hp : 0;
        pr[3 * m] = hp;
        pr[3 * m + 1] = sw_sqrt_pow(w1 * w1 + w2 * w2);
        pr[3 * m + 2] = st[P_TOTSED * pl + qp];
    }
    ctl->stagecnt = r + 1;
    ctl->stageinterval += P.stageint;
}

template <int MAXS>
__global__ void __launch_bounds__(NB_THREADS) k_update(const DevParams P, const Bufs B, Ctl *ctl,
                                                        const double *__restrict__ rain, double *partials,
                                                        double *stage, double *saveflow)
{
    if (!ctl->pending) return;
    const int64_t n = ctl->step;
    const double t = ctl->t, dt = ctl->dt;
    const double *src = B.set[n & 1];
    double *dst = B.set[(n + 1) & 1];
    const double *zp = B.z[(n + 2) % 3], *zc = B.z[n % 3];
    double *zn = B.z[(n + 1) % 3];
    double inh = 0, inhv = 0, insed = 0;
    if (P.inflow) inflow_ghost(t, inh, inhv, insed);
    const double Rr = P.storm ? 0.0 : rain_at(P, rain, t);
    Acc<MAXS> acc;
    acc.rain = acc.out = acc.clamp = acc.bulk = acc.inf = 0;
#pragma unroll
    for (int k = 0; k < MAXS; k++) acc.det[k] = acc.sout[k] = 0;
    const int64_t total = (int64_t)P.nx * P.ny;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < total; c += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(c / P.ny) + 1, j = (int)(c % P.ny) + 1;
        update_cell<MAXS>(P, src, dst, zp, zc, zn, B.ks, i, j, t, dt, Rr, inh, inhv, insed, acc);
    }
    /* budget partials of this block: warp shuffles then warps in order */
    __shared__ double red[NB_THREADS / 32][B_NTERMS];
    __shared__ bool last;
    if (P.budget) {
        double v[B_NTERMS];
        v[B_RAIN] = acc.rain; v[B_OUT] = acc.out; v[B_CLAMP] = acc.clamp; v[B_BULK] = acc.bulk; v[B_INF] = acc.inf;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            v[B_DET + k] = (k < MAXS) ? acc.det[k < MAXS ? k : 0] : 0.0;
            v[B_SOUT + k] = (k < MAXS) ? acc.sout[k < MAXS ? k : 0] : 0.0;
        }
#pragma unroll
        for (int m = 0; m < B_NTERMS; m++) {
            double s = warp_sum(v[m]);
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][m] = s;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        if (P.budget) {
            for (int m = 0; m < B_NTERMS; m++) {
                double s = 0;
                for (int w = 0; w < NB_THREADS / 32; w++) s += red[w][m];
                partials[(int64_t)blockIdx.x * B_NTERMS + m] = s;
            }
        }
        __threadfence();
        unsigned tk = atomicAdd(&ctl->update_ticket, 1u);
        last = (tk == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (P.budget && threadIdx.x < B_NTERMS) {
        double hi = 0, lo = 0;
        for (unsigned b = 0; b < gridDim.x; b++) dd_add(hi, lo, ((volatile double *)partials)[(int64_t)b * B_NTERMS + threadIdx.x]);
        double H = ctl->budget_hi[threadIdx.x], L = ctl->budget_lo[threadIdx.x];
        dd_add(H, L, hi);
        L += lo;
        ctl->budget_hi[threadIdx.x] = H;
        ctl->budget_lo[threadIdx.x] = L;
    }
    const double tnew = (ctl->cfl ? 2 * P.tend : t) + dt;
    const bool stage_due = tnew > ctl->stageinterval && ctl->stagecnt < ctl->stagecap;
    if (stage_due) stage_sample(P, dst, ctl, tnew, stage, saveflow);
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->t = tnew;
        ctl->step = n + 1;
        ctl->pending = 0;
        ctl->update_ticket = 0u;
        if (ctl->cfl) ctl->status = 1;
        if (!(dt > 0) && !ctl->cfl) ctl->status = 2;   /* time would not advance: stop instead of spinning */
        if (ctl->cfl || !(dt > 0) || !(tnew < P.tend) || !(tnew < ctl->t_stop) || n + 1 >= ctl->max_step)
            ctl->active = 0;
        ctl->launches += 2;
    }
}

/* ------------------------------------------------------------ launch --- */
int launch_step_f64(const DevParams &P, const Bufs &B, Ctl *ctl, const double *rain, double *partials,
                    double *stage, double *saveflow, int grid, cudaStream_t s, cudaEvent_t ev0, cudaEvent_t ev1)
{
    k_wave<<<grid, NB_THREADS, 0, s>>>(P, B, ctl);
    if (ev0) cudaEventRecord(ev0, s);
    if (P.S <= 4)
        k_update<4><<<grid, NB_THREADS, 0, s>>>(P, B, ctl, rain, partials, stage, saveflow);
    else if (P.S <= 8)
        k_update<8><<<grid, NB_THREADS, 0, s>>>(P, B, ctl, rain, partials, stage, saveflow);
    else
        k_update<16><<<grid, NB_THREADS, 0, s>>>(P, B, ctl, rain, partials, stage, saveflow);
    if (ev1) cudaEventRecord(ev1, s);
    return (int)cudaGetLastError();
}

int step_grid_f64(const DevParams &P, int num_sms)
{
    int64_t total = (int64_t)P.nx * P.ny;
    int64_t blocks = (total + NB_THREADS - 1) / NB_THREADS;
    int64_t cap = (int64_t)num_sms * 4;
    return (int)(blocks < cap ? blocks : cap);
}

}  // namespace swehr
