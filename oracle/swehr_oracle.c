/*
 * swehr_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement of the SWEHR explicit time step (csdms-contrib/swehr,
 * SWEHR.c:808-1591), used by tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg as the checker.  The product path never links, loads or
 * calls it.
 *
 * It is compiled twice from this one source:
 *   -DORC_GLIBC  : elementary functions from glibc libm exactly as the
 *                  reference calls them.  Pinned bit-for-bit against the
 *                  reference itself (oracle/_ref, built from SWEHR.c by
 *                  oracle/build_ref.py) on the shipped example, small grids
 *                  and the 200x50 hillslope (tests/test_oracle_pin.py).
 *   (default)    : elementary functions from swehr_b200/csrc/swehr_math.h,
 *                  the same bodies the CUDA kernels use, so the FP64 GPU
 *                  path must agree with this build bit-for-bit.
 *
 * The reference sweeps cells serially and reads some neighbours after they
 * were updated in the same sweep.  This restatement makes every such read
 * explicit so each phase is order-independent:
 *   - face fluxes use the gravity GZ of the left/lower cell from the
 *     previous step (SWEHR.c:1135,1203 run before 1279) -> GZ(z_prev);
 *   - GX uses the cell's own SLOPEY from the previous step (1243);
 *   - slope failure reads SLOPEX at IUP and SLOPEY at JUP from the previous
 *     step and at IDOWN/JDOWN from this step (1293, 1304);
 * where z_prev is the topography at the start of the previous step (the
 * slopes only depend on TOPO, which only sweep 2 modifies).  At the first
 * step z_prev = z, matching the setup pass (721-803).
 *
 * Zero-initialised state: the reference reads U[1], M, TOTM, DEP, TOTSED,
 * SOLID and TRACER before writing them (SWEHR.c:248, 1285, 1293, 1332);
 * fresh heap pages are zero there, and they are zero here.
 *
 * Interior solid cells (an optional SOLID mask; the stock program leaves
 * it zero): the topography fill of initialcondition (SWEHR.c:288-322), the
 * reflecting fluxes at solid/flow faces (SWEHR.c:1137-1146, 1205-1214), no
 * sources in solid cells (SWEHR.c:1233) -- so their slopes and GZ keep the
 * setup values their neighbours then read -- and zero water and suspended
 * sediment there (SWEHR.c:1566-1574).  NEARSOLIDX/Y only select the
 * reconstruction order near solid cells, and the order is first everywhere
 * (order=1, SWEHR.c:635), so they change nothing and are not kept.
 *
 * Left out because nothing observable depends on them: TRACER (only feeds
 * its own flux, never an output), UOLD/VELOLD/TOPOOLD/D/FAILCNT/BEDFLUX*
 * (write-only).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/swehr.h"

#ifdef ORC_GLIBC
#define M_POWH(x) pow((x), .5)
#define M_POW2(x) pow((x), 2)
#define M_POW(x, y) pow((x), (y))
#define M_EXP(x) exp(x)
#define M_COSATAN(x) cos(atan(x))
#define M_SINATAN(x) sin(atan(x))
#else
#include "../swehr_b200/csrc/swehr_math.h"
#define M_POWH(x) sw_sqrt_pow(x)
#define M_POW2(x) ((x) * (x))
#define M_POW(x, y) sw_pow((x), (y))
#define M_EXP(x) sw_exp(x)
#define M_COSATAN(x) sw_cos_atan(x)
#define M_SINATAN(x) sw_sin_atan(x)
#endif

#define ORC_STAGE_COLS 24
#define ORC_POINT_COLS 18

typedef struct orc_ctx {
    swehr_params p;
    int nx, ny, S, N;
    double *h, *hu, *hv, *z, *zp, *vinf, *maxvel, *maxdep, *totm, *dep, *totsed, *rho, *ks;
    double *U, *M, *sed;          /* class-major: [k*N + c] */
    int32_t *solid;               /* interior solid mask (SOLID, SWEHR.c:597), NULL when none */
    double *sx0, *sy0, *gz0;      /* setup slopes and gravity: a solid cell keeps them (SWEHR.c:721-803, 1233) */
    double *rain;
    double ds[SWEHR_MAX_CLASSES], pf[SWEHR_MAX_CLASSES];
    /* per-step scratch */
    double *sxn, *syn, *sxp, *syp, *gzp;
    double *fx, *fy;              /* face fluxes, (3+S) per face */
    double *srcf;                 /* per-cell sources: SXf SYf GAMMAX GAMMAY DFMASK BETAX BETAY FAIL GZ */
    double *E, *VF;               /* [(4*k + e)*N + c], [k*N + c] */
    double t, dt, courant, R;
    double t_prev;                /* start time of the last completed step */
    int64_t steps;
    int status;
    /* stage series */
    double stageinterval;
    int64_t stagecnt, stagecap;
    double *stage, *saveflow;
    /* budget */
    double b_rain, b_out, b_clamp, b_bulk, b_inf, b_water0;
    double b_det[SWEHR_MAX_CLASSES], b_sout[SWEHR_MAX_CLASSES], b_sed0[SWEHR_MAX_CLASSES];
    /* branch counters over the run (cell-steps), read by the tests to show a
     * case exercises them: slope failure (SWEHR.c:1295-1311), the debris-flow
     * forcing (DFMASK > 0, SWEHR.c:1315-1316) and the debris-flow override of
     * every source (SWEHR.c:1392-1400) */
    int64_t n_fail, n_dfmask, n_debris;
    /* slab runs (test of the multi-GPU decomposition): rows own_lo..own_hi
     * are this instance's; its largest wave speed counts only their faces */
    int own_lo, own_hi;
    double smax_own, R_step;
} orc_ctx;

#define IDX(c, i, j) (((size_t)(i) - 1) * (size_t)(c)->ny + ((size_t)(j) - 1))

/* SWEHR.c:327-409 (hllc).  Returns the largest |wave speed|. */
static double orc_hllc(double hl, double hr, double uhl, double uhr, double vhl, double vhr,
                       double g, double hfilm, double T[3])
{
    double ul = 0, vl = 0, ur = 0, vr = 0;
    if (hl > hfilm) { ul = uhl / hl; vl = vhl / hl; }
    if (hr > hfilm) { ur = uhr / hr; vr = vhr / hr; }
    double cl = M_POWH(g * hl), cr = M_POWH(g * hr);
    double hs = M_POW2(ul + 2 * cl - ur - 2 * cr) / (16 * g);
    double us = .5 * (ul + ur) + cl - cr;
    double cs = M_POWH(g * hs);
    double sl = ul - cl;
    if (us - cs < sl) sl = us - cs;
    double sm = us;
    double sr = ur + cr;
    if (us + cs > sr) sr = us + cs;
    if (hl <= hfilm) { sl = ur - 2 * cr; sm = sl; sr = ur + cr; }
    if (hr <= hfilm) { sl = ul - cl; sr = ul + 2 * cl; sm = sr; }
    double f0 = NAN, f1 = NAN;
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
    T[0] = f0;
    T[1] = f1;
    T[2] = (sm >= 0) ? f0 * vl : f0 * vr;
    double s = 0;
    if (fabs(sl) > s) s = fabs(sl);
    if (fabs(sr) > s) s = fabs(sr);
    if (fabs(sm) > s) s = fabs(sm);
    return s;
}

/* SWEHR.c:1240-1257 (and 725-742): x slope of a topography array */
static double orc_slopex(const orc_ctx *c, const double *z, int i, int j, double oneoverdx)
{
    if (i != 1 && i != c->nx) return 0.5 * oneoverdx * (z[IDX(c, i + 1, j)] - z[IDX(c, i - 1, j)]);
    if (i == c->nx) return oneoverdx * (z[IDX(c, i, j)] - z[IDX(c, i - 1, j)]);
    return oneoverdx * (z[IDX(c, i + 1, j)] - z[IDX(c, i, j)]);
}

/* SWEHR.c:1260-1277 */
static double orc_slopey(const orc_ctx *c, const double *z, int i, int j, double oneoverdx)
{
    if (j != 1 && j != c->ny) return 0.5 * oneoverdx * (z[IDX(c, i, j + 1)] - z[IDX(c, i, j - 1)]);
    if (j == c->ny) return oneoverdx * (z[IDX(c, i, j)] - z[IDX(c, i, j - 1)]);
    return oneoverdx * (z[IDX(c, i, j + 1)] - z[IDX(c, i, j)]);
}

/* Rain rate at time t, SWEHR.c:813-814 (uniform hyetograph), or the moving
 * storm extension when storm_peak > 0. */
static double orc_rain(const orc_ctx *c, double t)
{
    int rind = (int)fmin(ceil(t / c->p.rint + 0.01), c->p.rnum);
    return c->rain[rind - 1];
}

static double orc_storm(const orc_ctx *c, double t, int i, int j)
{
    const swehr_params *p = &c->p;
    double x = ((double)i - 0.5) * p->dx - (p->storm_x0 + p->storm_vx * t);
    double y = ((double)j - 0.5) * p->dx - (p->storm_y0 + p->storm_vy * t);
    double r2 = (x * x + y * y) / (p->storm_radius * p->storm_radius);
    return p->storm_peak * M_EXP(-0.5 * r2);
}

/* State of a face neighbour, interior or ghost (SWEHR.c:816-1035).  Ghosts
 * copy the adjacent interior cell; a solid side negates the normal momentum;
 * the inflow row j=ny+1 is the hard-wired time ramp. */
typedef struct { double h, hu, hv; const double *sed; size_t sstride; double sedin; int inflow; } orc_nb;

static void orc_neighbour(const orc_ctx *c, int i, int j, const double inflow[3], double sedin, orc_nb *o)
{
    const swehr_params *p = &c->p;
    int si = i, sj = j;
    double su = 1, sv = 1;
    o->inflow = 0;
    if (i == 0) { si = 1; if (p->bndry[0] == 1) su = -1; }
    else if (i == c->nx + 1) { si = c->nx; if (p->bndry[2] == 1) su = -1; }
    else if (j == 0) { sj = 1; if (p->bndry[1] == 1) sv = -1; }
    else if (j == c->ny + 1) {
        if (p->inflow) {
            o->h = inflow[0]; o->hu = inflow[1]; o->hv = inflow[2];
            o->inflow = 1; o->sedin = sedin; o->sed = NULL; o->sstride = 0;
            return;
        }
        sj = c->ny; if (p->bndry[3] == 1) sv = -1;
    }
    size_t q = IDX(c, si, sj);
    o->h = c->h[q];
    o->hu = (su < 0) ? -c->hu[q] : c->hu[q];
    o->hv = (sv < 0) ? -c->hv[q] : c->hv[q];
    o->sed = c->sed + q;
    o->sstride = (size_t)c->N;
}

/* SOLID[i][j] as the reference reads it: inside the grid the mask; at
 * j = ny+1 (the y-face test at SWEHR.c:1206,1211 reads one column past the
 * row) the next row's first cell, SOLID[i+1][1], and past the last row 0 (the
 * patched reference pads the matrix with zeros there); 0 elsewhere. */
static int orc_solid(const orc_ctx *c, int i, int j)
{
    if (!c->solid || i < 1 || i > c->nx || j < 1) return 0;
    if (j <= c->ny) return c->solid[IDX(c, i, j)] != 0;
    if (j == c->ny + 1 && i < c->nx) return c->solid[IDX(c, i + 1, 1)] != 0;
    return 0;
}

/* initialcondition's topography fill around solid cells (SWEHR.c:288-322),
 * serial and in place, in the reference's order */
static void orc_solid_fill(orc_ctx *c, double *T)
{
    const int nx = c->nx, ny = c->ny;
#define S_(a, b) (c->solid[IDX(c, (a), (b))] != 0)
#define T_(a, b) T[IDX(c, (a), (b))]
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++) {
            int iup = i + 1 < nx ? i + 1 : nx, idown = i - 1 > 1 ? i - 1 : 1;
            int jup = j + 1 < ny ? j + 1 : ny, jdown = j - 1 > 1 ? j - 1 : 1;
            if (S_(i, j)) {
                if (!S_(iup, j)) T_(i, j) = T_(iup, j);
                if (!S_(idown, j)) T_(i, j) = T_(idown, j);
                if (!S_(iup, jup)) T_(i, j) = T_(iup, jup);
                if (!S_(iup, jdown)) T_(i, j) = T_(iup, jdown);
                if (!S_(idown, jup)) T_(i, j) = T_(idown, jup);
                if (!S_(idown, jdown)) T_(i, j) = T_(idown, jdown);
                if (!S_(i, jup)) T_(i, j) = T_(i, jup);
                if (!S_(i, jdown)) T_(i, j) = T_(i, jdown);
            }
            if (S_(iup, j) && !S_(i, j)) T_(iup, j) = T_(i, j);
            if (S_(idown, j) && !S_(i, j)) T_(idown, j) = T_(i, j);
            if (S_(i, jup) && !S_(i, j)) T_(i, jup) = T_(i, j);
            if (S_(i, jdown) && !S_(i, j)) T_(i, jdown) = T_(i, j);
        }
#undef S_
#undef T_
}

static double orc_nbsed(const orc_nb *o, int k)
{
    return o->inflow ? o->sedin : o->sed[(size_t)k * o->sstride];
}

/* streampowererosion, SWEHR.c:412-426 */
static double orc_spe(double uh, double vh, double h, double beta, double rho, double g,
                      double sedconc, double sf, double minmorph, double uc)
{
    double q = M_POWH(uh * uh + vh * vh);
    double omega = rho * g * sf * q;
    double E = 0;
    if (omega > uc && sedconc < 0.6 && h > minmorph) E = beta * (omega - uc);
    return E;
}

/* Phases 1-3 of a step (slopes, faces, sources); the largest wave speed of
 * the owned faces goes to c->smax_own.  orc_commit finishes the step. */
static void orc_prepare(orc_ctx *c)
{
    const swehr_params *p = &c->p;
    const int nx = c->nx, ny = c->ny, S = c->S, N = c->N, NF = 3 + S;
    const double oneoverdx = 1 / p->dx;
    const double g = p->g, hfilm = p->hfilm, rhos = p->rhos, rhow = p->rhow, phi = p->phi;
    const double rho0 = rhow * phi + rhos * (1 - phi);
    const double t = c->t;
    const int storm = p->storm_peak > 0;
    double R = storm ? 0.0 : orc_rain(c, t);

    /* hard-wired inflow ghost (SWEHR.c:1019-1034) */
    double inflow[3] = {0, 0, 0}, sedin = 0;
    if (p->inflow) {
        double vin = fmax(-0.035, t / 100 * -0.035);
        double hin = M_POW(fabs(vin) * 0.045 / M_POWH(0.7), 0.6);
        double ukin = fmin(500, t / 100 * 500) * hin;
        inflow[0] = hin; inflow[1] = 0; inflow[2] = vin;
        sedin = ukin / hin;
    }

    /* phase 1: slopes from this step's z and the previous step's z */
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++) {
            size_t q = IDX(c, i, j);
            c->sxn[q] = orc_slopex(c, c->z, i, j, oneoverdx);
            c->syn[q] = orc_slopey(c, c->z, i, j, oneoverdx);
            double sxp = orc_slopex(c, c->zp, i, j, oneoverdx);
            double syp = orc_slopey(c, c->zp, i, j, oneoverdx);
            c->sxp[q] = sxp;
            c->syp[q] = syp;
            c->gzp[q] = g / M_POWH(sxp * sxp + syp * syp + 1);
            if (c->solid && c->solid[q]) {         /* never recomputed (SWEHR.c:1233) */
                c->sxn[q] = c->sxp[q] = c->sx0[q];
                c->syn[q] = c->syp[q] = c->sy0[q];
                c->gzp[q] = c->gz0[q];
            }
        }

    /* phase 2: face fluxes and the largest wave speed (SWEHR.c:1092-1230) */
    double smax = 0;
#pragma omp parallel for schedule(static) reduction(max : smax)
    for (int i = 0; i <= nx; i++) {
        for (int j = 0; j <= ny; j++) {
            double T[3];
            orc_nb L, Rn;
            if (j != 0) { /* x face i+1/2 */
                orc_neighbour(c, i, j, inflow, sedin, &L);
                orc_neighbour(c, i + 1, j, inflow, sedin, &Rn);
                double gl = c->gzp[IDX(c, i == 0 ? 1 : i, j)];
                double s = orc_hllc(L.h, Rn.h, L.hu, Rn.hu, L.hv, Rn.hv, gl, hfilm, T);
                if (c->solid && i >= 1 && i < nx) {    /* reflecting faces, SWEHR.c:1137-1146 */
                    int sl = orc_solid(c, i, j), sr = orc_solid(c, i + 1, j);
                    if (sl && !sr) s = orc_hllc(Rn.h, Rn.h, -Rn.hu, Rn.hu, Rn.hv, Rn.hv, gl, hfilm, T);
                    else if (!sl && sr) s = orc_hllc(L.h, L.h, L.hu, -L.hu, L.hv, L.hv, gl, hfilm, T);
                }
                double *f = c->fx + ((size_t)i * ny + (j - 1)) * NF;
                f[0] = T[0]; f[1] = T[1]; f[2] = T[2];
                for (int k = 0; k < S; k++)
                    f[3 + k] = (T[0] > 0) ? T[0] * orc_nbsed(&L, k) : T[0] * orc_nbsed(&Rn, k);
                if (s > smax && ((i >= c->own_lo && i <= c->own_hi) || (i == 0 && c->own_lo == 1))) smax = s;
            }
            if (i != 0) { /* y face j+1/2 */
                orc_neighbour(c, i, j, inflow, sedin, &L);
                orc_neighbour(c, i, j + 1, inflow, sedin, &Rn);
                double gl = c->gzp[IDX(c, i, j == 0 ? 1 : j)];
                double s = orc_hllc(L.h, Rn.h, L.hv, Rn.hv, L.hu, Rn.hu, gl, hfilm, T);
                if (c->solid && j >= 1) {              /* reflecting faces, SWEHR.c:1205-1214 */
                    int sl = orc_solid(c, i, j), sr = orc_solid(c, i, j + 1);
                    if (sl && !sr) s = orc_hllc(Rn.h, Rn.h, -Rn.hv, Rn.hv, Rn.hu, Rn.hu, gl, hfilm, T);
                    else if (!sl && sr) s = orc_hllc(L.h, L.h, L.hv, -L.hv, L.hu, L.hu, gl, hfilm, T);
                }
                double *f = c->fy + ((size_t)(i - 1) * (ny + 1) + j) * NF;
                f[0] = T[0]; f[1] = T[2]; f[2] = T[1];
                for (int k = 0; k < S; k++)
                    f[3 + k] = (T[0] > 0) ? T[0] * orc_nbsed(&L, k) : T[0] * orc_nbsed(&Rn, k);
                if (s > smax && i >= c->own_lo && i <= c->own_hi) smax = s;
            }
        }
    }

    /* phase 3: sources from the state at the start of the step (SWEHR.c:1233-1401) */
    int64_t n_fail = 0, n_dfmask = 0, n_debris = 0;
#pragma omp parallel for schedule(static) reduction(+ : n_fail, n_dfmask, n_debris)
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++) {
            size_t q = IDX(c, i, j);
            if (c->solid && c->solid[q]) continue;     /* no sources in a solid cell (SWEHR.c:1233) */
            double h = c->h[q], hu = c->hu[q], hv = c->hv[q];
            double rho = c->rho[q], totsed = c->totsed[q], totm = c->totm[q], dep = c->dep[q];
            double Rc = storm ? orc_storm(c, t, i, j) : R;
            double sx = c->sxn[q], syl = c->syp[q], sy = c->syn[q];
            double gx = g * sx / M_POWH(sx * sx + syl * syl + 1);
            double SXf = -gx * h;
            double gy = g * sy / M_POWH(sx * sx + sy * sy + 1);
            double SYf = -gy * h;
            double gz = g / M_POWH(sx * sx + sy * sy + 1);
            double slope = M_POWH(sx * sx + sy * sy);
            double gammax = 0, gammay = 0;
            if (i > 1 && i < nx)
                gammax -= (rhos - rho) * gz * h * h / (2 * rho) * .5 * oneoverdx
                          * (c->totsed[IDX(c, i + 1, j)] - c->totsed[IDX(c, i - 1, j)]);
            if (j > 1 && j < ny)
                gammay -= (rhos - rho) * gz * h * h / (2 * rho) * .5 * oneoverdx
                          * (c->totsed[IDX(c, i, j + 1)] - c->totsed[IDX(c, i, j - 1)]);
            /* slope stability of the deposited layer (SWEHR.c:1292-1312) */
            double fail = 0;
            int iu = (i < nx) ? i + 1 : nx, id = (i > 1) ? i - 1 : 1;
            int ju = (j < ny) ? j + 1 : ny, jd = (j > 1) ? j - 1 : 1;
            double sxu = (iu == i) ? sx : c->sxp[IDX(c, iu, j)];
            double sxd = c->sxn[IDX(c, id, j)];
            double syu = (ju == j) ? sy : c->syp[IDX(c, i, ju)];
            double syd = c->syn[IDX(c, i, jd)];
            double pgfx = dep * rho0 * gz * 0.5 * oneoverdx
                          * (c->dep[IDX(c, iu, j)] * M_COSATAN(fabs(sxu)) - c->dep[IDX(c, id, j)] * M_COSATAN(fabs(sxd)));
            if (pgfx * sx > 0) pgfx = -1 * fabs(pgfx);
            if (pgfx * sx < 0) pgfx = fabs(pgfx);
            double lhs = (rho0 * gz * dep + rho * gz * h) * M_SINATAN(fabs(sy));
            double nrm = (rho0 * gz * dep + rho * gz * h) * M_COSATAN(fabs(sy)) - rhow * gz * (dep + h);
            if (fail == 0 && (lhs > (p->cohesion + nrm * p->frictionangle + pgfx))) fail = 1;
            double pgfy = dep * rho0 * gz * 0.5 * oneoverdx
                          * (c->dep[IDX(c, i, ju)] * M_COSATAN(fabs(syu)) - c->dep[IDX(c, i, jd)] * M_COSATAN(fabs(syd)));
            if (pgfy * sy > 0) pgfy = -1 * fabs(pgfy);
            if (pgfy * sy < 0) pgfy = fabs(pgfy);
            if (fail == 0 && (lhs > (p->cohesion + nrm * p->frictionangle + pgfy))) fail = 1;
            /* debris-flow terms (SWEHR.c:1315-1320) */
            double dfmask = fmin(1, (totsed - 0.2) / 0.2);
            if (h < 9 * p->h0 || totsed < 0.2) dfmask = 0;
            double betax = -(1 - p->lambda) * gz * h * p->frictionangle;
            double betay = -(1 - p->lambda) * gz * h * p->frictionangle;
            if (hu < 0) betax = -1 * betax;
            if (hv < 0) betay = -1 * betay;
            n_fail += fail == 1;
            n_dfmask += dfmask > 0;
            n_debris += (h > 9 * p->h0 && totsed > p->cthreshold);
            double *sf = c->srcf + q * 9;
            sf[0] = SXf; sf[1] = SYf; sf[2] = gammax; sf[3] = gammay; sf[4] = dfmask;
            sf[5] = betax; sf[6] = betay; sf[7] = fail; sf[8] = gz;
            /* Hairsine-Rose sources per class (SWEHR.c:1322-1401) */
            double hvert = h / M_COSATAN(fabs(slope));
            double mtstar = p->mtstar0;
            if (hvert > p->h0) mtstar = p->mtstar0 * M_POW(p->h0 / hvert, p->b);
            double Hs = fmin(1, totm / mtstar);
            double manning = (h <= p->hcfriction)
                                 ? p->roughness * M_POW(h / p->hcfriction, p->depthdependentexponent)
                                 : p->roughness;
            double qq = M_POWH(hu * hu + hv * hv);
            double SF = manning * manning * qq * qq / M_POW(h, 3.333);
            int swash = (h > 10 * hfilm && totsed < 0.6);
            double depthfac = (swash && hvert > p->h0) ? M_POW(p->h0 / hvert, p->b) : 1.0;
            double vfconc = M_POW(1 - fmin(totsed, 0.99), 4);
            for (int k = 0; k < S; k++) {
                double Mk = c->M[(size_t)k * N + q];
                double E1 = 0, E2 = 0, E3 = 0, E4 = 0;
                if (swash) {
                    E1 = (1 - Hs) * c->pf[k] * p->a * Rc;
                    if (totm > 1e-8 && Mk > 1e-8) E2 = Hs * Mk / totm * p->ad * Rc;
                    if (hvert > p->h0) { E1 = E1 * depthfac; E2 = E2 * depthfac; }
                    E3 = orc_spe(hu, hv, h, p->af, rho, gz, totsed, SF, c->ds[k], p->uc);
                    E3 = (1 - Hs) * c->pf[k] * p->F / p->J * E3;
                    if (totm > 1e-6 && Mk > 0) {
                        E4 = orc_spe(hu, hv, h, p->afr, rho, gz, totsed, SF, c->ds[k], p->uc2);
                        E4 = (1 - p->betabedload) * Hs * Mk / totm * p->F / ((rhos - rho) / rhos * gz * h) * E4;
                    } else E4 = 0;
                }
                double d = c->ds[k];
                double s = rhos / rhow - 1;
                double VF = M_POWH(M_POW2(13.95 * p->nu / d) + 1.09 * s * gz * d) - 13.95 * p->nu / d;
                VF = VF * vfconc;
                if (d > 0.0001 && h < 9 * p->h0) VF = 2e-3 + fmax(h - 3 * p->h0, 0) * (VF - 2e-3) / (6 * p->h0);
                if (d > 0.002 && h < 9 * p->h0) VF = 2e-3 + fmax(h - 3 * p->h0, 0) * (VF - 2e-3) / (6 * p->h0);
                if (h > 9 * p->h0 && totsed > p->cthreshold) { E1 = E2 = E3 = E4 = 0; VF = 0; }
                c->E[(size_t)(4 * k + 0) * N + q] = E1;
                c->E[(size_t)(4 * k + 1) * N + q] = E2;
                c->E[(size_t)(4 * k + 2) * N + q] = E3;
                c->E[(size_t)(4 * k + 3) * N + q] = E4;
                c->VF[(size_t)k * N + q] = VF;
            }
        }

    c->n_fail += n_fail;
    c->n_dfmask += n_dfmask;
    c->n_debris += n_debris;
    c->smax_own = smax;
    c->R_step = R;
}

/* The rest of a step given the largest wave speed over every face of the
 * domain: the CFL time step, the cell update, time and series. */
static int orc_commit(orc_ctx *c, double smax)
{
    const swehr_params *p = &c->p;
    const int nx = c->nx, ny = c->ny, S = c->S, N = c->N, NF = 3 + S;
    const double oneoverdx = 1 / p->dx;
    const double hfilm = p->hfilm, rhos = p->rhos, rhow = p->rhow, phi = p->phi;
    const double t = c->t;
    const int storm = p->storm_peak > 0;
    const double R = c->R_step;

    /* CFL time step (SWEHR.c:1409-1413) */
    double dt = p->cstable * p->dx / smax;
    if (dt > p->maxstep) dt = p->maxstep;
    if (t + dt > p->tend) dt = p->tend - t;
    double courant = smax * dt * oneoverdx;
    int cfl = courant > 1;

    /* previous-step topography for the next step's lagged slopes */
    memcpy(c->zp, c->z, (size_t)N * sizeof(double));

    /* phase 4: cell update (SWEHR.c:1417-1588) */
    double b_out = 0, b_clamp = 0, b_bulk = 0, b_inf = 0, b_rain = 0;
    double b_det[SWEHR_MAX_CLASSES] = {0}, b_sout[SWEHR_MAX_CLASSES] = {0};
    double b_solw = 0, b_sols[SWEHR_MAX_CLASSES] = {0};
#pragma omp parallel for schedule(static) reduction(+ : b_clamp, b_bulk, b_inf, b_rain, b_solw, b_det[:SWEHR_MAX_CLASSES], b_sols[:SWEHR_MAX_CLASSES])
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++) {
            size_t q = IDX(c, i, j);
            if (c->solid && c->solid[q]) {
                /* outside the domain: no water, momentum or suspended sediment
                 * (SWEHR.c:1566-1574); what a written state held there leaves
                 * the budget as outflow */
                b_solw += c->h[q];
                c->h[q] = 0; c->hu[q] = 0; c->hv[q] = 0;
                for (int k = 0; k < S; k++) {
                    size_t qk = (size_t)k * N + q;
                    b_sols[k] += c->U[qk];
                    c->U[qk] = 0;
                    c->sed[qk] = 0;
                }
                double rho = rhow * (1 - c->totsed[q]) + rhos * c->totsed[q];
                if (rho > 0.8 * rhos) rho = 0.8 * rhos;
                c->rho[q] = rho;
                if (0.0 > c->maxvel[q]) c->maxvel[q] = 0.0;
                if (0.0 > c->maxdep[q]) c->maxdep[q] = 0.0;
                continue;
            }
            const double *fxl = c->fx + ((size_t)(i - 1) * ny + (j - 1)) * NF;
            const double *fxr = c->fx + ((size_t)i * ny + (j - 1)) * NF;
            const double *fyl = c->fy + ((size_t)(i - 1) * (ny + 1) + (j - 1)) * NF;
            const double *fyr = c->fy + ((size_t)(i - 1) * (ny + 1) + j) * NF;
            const double *sf = c->srcf + q * 9;
            double Rc = storm ? orc_storm(c, t, i, j) : R;
            double chtemp = 0, redetach = 0;
            double h = c->h[q] - dt * oneoverdx * (fxr[0] - fxl[0]) - dt * oneoverdx * (fyr[0] - fyl[0]) + dt * Rc;
            double hu = c->hu[q] - dt * oneoverdx * (fxr[1] - fxl[1]) - dt * oneoverdx * (fyr[1] - fyl[1])
                        + dt * sf[0] + dt * sf[2] + dt * sf[4] * sf[5];
            double hv = c->hv[q] - dt * oneoverdx * (fxr[2] - fxl[2]) - dt * oneoverdx * (fyr[2] - fyl[2])
                        + dt * sf[1] + dt * sf[3] + dt * sf[4] * sf[6];
            double ksq = c->ks ? c->ks[q] : p->ks;
            double zf = c->vinf[q] / (p->thetas - p->theta0);
            double infl = fmin(h - hfilm, dt * ksq * (zf + p->hf + h) / zf);
            c->vinf[q] += infl;
            h -= infl;
            double Uk[SWEHR_MAX_CLASSES];
            for (int k = 0; k < S; k++) {
                size_t qk = (size_t)k * N + q;
                Uk[k] = c->U[qk] - dt * oneoverdx * (fxr[3 + k] - fxl[3 + k]) - dt * oneoverdx * (fyr[3 + k] - fyl[3 + k]);
            }
            double z = c->z[q];
            double totm = 0, dep = 0;
            double fail = sf[7];
            double bulk = 0;
            for (int k = 0; k < S; k++) {
                size_t qk = (size_t)k * N + q;
                double E1 = c->E[(size_t)(4 * k + 0) * N + q], E2 = c->E[(size_t)(4 * k + 1) * N + q];
                double E3 = c->E[(size_t)(4 * k + 2) * N + q], E4 = c->E[(size_t)(4 * k + 3) * N + q];
                double VF = c->VF[qk];
                double Mk = c->M[qk];
                if (h < 10 * hfilm) {
                    Mk += dt * E1 + Uk[k];
                    Uk[k] = 0;
                    b_det[k] += dt * E1;
                } else {
                    chtemp = Uk[k];
                    redetach = fmin(Mk, dt * (E2 + E4));
                    Uk[k] = M_EXP(-VF / h * (0.5 * dt)) * Uk[k];
                    Uk[k] = Uk[k] + dt * (E1 + E3) + redetach;
                    Uk[k] = M_EXP(-VF / h * (0.5 * dt)) * Uk[k];
                    z = z - 1 / (rhos * (1 - phi)) * (Uk[k] - chtemp);
                    Mk = Mk + dt * (E1 + E3) - (Uk[k] - chtemp);
                    b_det[k] += dt * (E1 + E3);
                    if (fail == 1) {
                        z = z - 0.99 * Mk / (rhos * (1 - phi));
                        Uk[k] = Uk[k] + 0.99 * Mk;
                        totm = 0;
                        Mk = 0.01 * Mk;
                        dep = 0;
                    }
                }
                double dh = (Uk[k] - chtemp) / (rhos * (1 - phi));
                h = h + dh;
                bulk += dh;
                totm += Mk;
                dep += Mk / rhos;
                c->M[qk] = Mk;
            }
            double totsed = 0, clamp = 0;
            if (h > hfilm) {
                for (int k = 0; k < S; k++) {
                    size_t qk = (size_t)k * N + q;
                    double s = Uk[k] / h;
                    totsed += s / rhos;
                    if (s < -1e-5) s = 0;
                    c->sed[qk] = s;
                    c->U[qk] = Uk[k];
                }
            } else {
                clamp = hfilm - h;
                h = hfilm;
                hu = 0;
                hv = 0;
                for (int k = 0; k < S; k++) {
                    size_t qk = (size_t)k * N + q;
                    z = z + 1 / (rhos * (1 - phi)) * Uk[k];
                    c->M[qk] = c->M[qk] + Uk[k];
                    c->U[qk] = 0;
                    c->sed[qk] = 0;
                }
            }
            double vel1 = 0, vel2 = 0;
            if (h > hfilm) {
                double manning = (h <= p->hcfriction)
                                     ? p->roughness * M_POW(h / p->hcfriction, p->depthdependentexponent)
                                     : p->roughness;
                double SFf = manning * manning * sf[8] * M_POWH(hu * hu + hv * hv) * 1 / M_POW(h, 2.333);
                hu = hu / (1 + dt * SFf);
                hv = hv / (1 + dt * SFf);
                vel1 = hu / h;
                vel2 = hv / h;
            }
            double rho = rhow * (1 - totsed) + rhos * totsed;
            if (rho > 0.8 * rhos) rho = 0.8 * rhos;
            double vmag = M_POWH(vel1 * vel1 + vel2 * vel2);
            if (vmag > c->maxvel[q]) c->maxvel[q] = vmag;
            if (h > c->maxdep[q]) c->maxdep[q] = h;
            c->h[q] = h; c->hu[q] = hu; c->hv[q] = hv; c->z[q] = z;
            c->totm[q] = totm; c->dep[q] = dep; c->totsed[q] = totsed; c->rho[q] = rho;
            b_rain += dt * Rc;
            b_inf += infl;
            b_clamp += clamp;
            b_bulk += bulk;
        }
    /* boundary outflow of water and sediment over this step */
    for (int j = 1; j <= ny; j++) {
        const double *fl = c->fx + ((size_t)0 * ny + (j - 1)) * NF;
        const double *fr = c->fx + ((size_t)nx * ny + (j - 1)) * NF;
        b_out += dt * oneoverdx * (fr[0] - fl[0]);
        for (int k = 0; k < S; k++) b_sout[k] += dt * oneoverdx * (fr[3 + k] - fl[3 + k]);
    }
    for (int i = 1; i <= nx; i++) {
        const double *fl = c->fy + ((size_t)(i - 1) * (ny + 1) + 0) * NF;
        const double *fr = c->fy + ((size_t)(i - 1) * (ny + 1) + ny) * NF;
        b_out += dt * oneoverdx * (fr[0] - fl[0]);
        for (int k = 0; k < S; k++) b_sout[k] += dt * oneoverdx * (fr[3 + k] - fl[3 + k]);
    }
    b_out += b_solw;
    for (int k = 0; k < S; k++) b_sout[k] += b_sols[k];
    c->b_rain += b_rain; c->b_out += b_out; c->b_clamp += b_clamp; c->b_bulk += b_bulk; c->b_inf += b_inf;
    for (int k = 0; k < S; k++) { c->b_det[k] += b_det[k]; c->b_sout[k] += b_sout[k]; }

    c->dt = dt;
    c->courant = courant;
    c->R = R;
    c->t_prev = t;
    c->t = cfl ? 2 * p->tend : t;
    c->t += dt;
    c->steps++;

    /* stage and point series (SWEHR.c:1593-1676) */
    if (c->t > c->stageinterval && c->stagecnt < c->stagecap) {
        int orow = p->outlet_row;
        int outlet = 1;
        double best = 0;
        for (int i = 1; i <= nx; i++)
            if (c->h[IDX(c, i, orow)] > best) { best = c->h[IDX(c, i, orow)]; outlet = i; }
        c->stageinterval += p->stageint;
        double *row = c->stage + c->stagecnt * ORC_STAGE_COLS;
        size_t qo = IDX(c, outlet, orow);
        double ho = c->h[qo];
        double v1 = ho > hfilm ? c->hu[qo] / ho : 0, v2 = ho > hfilm ? c->hv[qo] / ho : 0;
        row[0] = c->t;
        row[1] = ho;
        row[2] = M_POWH(v1 * v1 + v2 * v2);
        row[3] = c->totsed[qo];
        for (int k = 0; k < 10; k++) {
            row[4 + k] = (k < S) ? c->M[(size_t)k * N + qo] : 0;
            row[14 + k] = (k < S) ? c->U[(size_t)k * N + qo] : 0;
        }
        double *pr = c->saveflow + c->stagecnt * ORC_POINT_COLS;
        for (int m = 0; m < 6; m++) {
            int xi = p->xpoint[m], yj = p->ypoint[m];
            if (m >= p->npoints || xi < 1 || xi > nx || yj < 1 || yj > ny) {
                pr[3 * m] = pr[3 * m + 1] = pr[3 * m + 2] = NAN;
                continue;
            }
            size_t qp = IDX(c, xi, yj);
            double hp = c->h[qp];
            double w1 = hp > hfilm ? c->hu[qp] / hp : 0, w2 = hp > hfilm ? c->hv[qp] / hp : 0;
            pr[3 * m] = hp;
            pr[3 * m + 1] = M_POWH(w1 * w1 + w2 * w2);
            pr[3 * m + 2] = c->totsed[qp];
        }
        c->stagecnt++;
    }
    return cfl ? SWEHR_CFL_ERROR : SWEHR_OK;
}

static int orc_step(orc_ctx *c)
{
    orc_prepare(c);
    return orc_commit(c, c->smax_own);
}

/* ---------------------------------------------------------------- ABI --- */

static void *orc_alloc(size_t n)
{
    void *p = calloc(n ? n : 1, sizeof(double));
    return p;
}

orc_ctx *orc_create(const swehr_params *p, const swehr_inputs *in)
{
    if (!p || !in || !in->topo || !in->rain || !in->ds || !in->pfrac) return NULL;
    if (p->nx < 2 || p->ny < 2 || p->sclass < 1 || p->sclass > SWEHR_MAX_CLASSES || p->rnum < 1) return NULL;
    orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
    c->p = *p;
    c->nx = p->nx; c->ny = p->ny; c->S = p->sclass; c->N = p->nx * p->ny;
    size_t N = (size_t)c->N, S = (size_t)c->S;
    double **fields[] = {&c->h, &c->hu, &c->hv, &c->z, &c->zp, &c->vinf, &c->maxvel, &c->maxdep,
                         &c->totm, &c->dep, &c->totsed, &c->rho, &c->sxn, &c->syn, &c->sxp, &c->syp, &c->gzp};
    for (size_t f = 0; f < sizeof fields / sizeof fields[0]; f++) *fields[f] = (double *)orc_alloc(N);
    c->U = (double *)orc_alloc(N * S);
    c->M = (double *)orc_alloc(N * S);
    c->sed = (double *)orc_alloc(N * S);
    c->E = (double *)orc_alloc(N * S * 4);
    c->VF = (double *)orc_alloc(N * S);
    c->srcf = (double *)orc_alloc(N * 9);
    c->fx = (double *)orc_alloc((size_t)(p->nx + 1) * p->ny * (3 + S));
    c->fy = (double *)orc_alloc((size_t)p->nx * (p->ny + 1) * (3 + S));
    c->rain = (double *)orc_alloc((size_t)p->rnum);
    memcpy(c->rain, in->rain, (size_t)p->rnum * sizeof(double));
    for (size_t k = 0; k < S; k++) { c->ds[k] = in->ds[k]; c->pf[k] = in->pfrac[k]; }
    if (in->ks) {
        c->ks = (double *)orc_alloc(N);
        memcpy(c->ks, in->ks, N * sizeof(double));
    }
    for (size_t q = 0; q < N; q++) c->z[q] = in->topo[q];
    if (in->solid) {
        c->solid = (int32_t *)calloc(N, sizeof(int32_t));
        for (size_t q = 0; q < N; q++) c->solid[q] = in->solid[q] != 0;
        orc_solid_fill(c, c->z);
        c->sx0 = (double *)orc_alloc(N);
        c->sy0 = (double *)orc_alloc(N);
        c->gz0 = (double *)orc_alloc(N);
        const double odx = 1 / p->dx;
        for (int i = 1; i <= c->nx; i++)
            for (int j = 1; j <= c->ny; j++) {
                size_t q = IDX(c, i, j);
                double sx = orc_slopex(c, c->z, i, j, odx), sy = orc_slopey(c, c->z, i, j, odx);
                c->sx0[q] = sx;
                c->sy0[q] = sy;
                c->gz0[q] = p->g / M_POWH(sx * sx + sy * sy + 1);
            }
    }
    for (size_t q = 0; q < N; q++) {
        c->zp[q] = c->z[q];
        c->vinf[q] = p->vinf0;
        c->rho[q] = p->rhow * (1 - 0.0) + p->rhos * 0.0;   /* initialcondition, SWEHR.c:270 */
    }
    c->own_lo = 1;
    c->own_hi = c->nx;
    c->stagecap = 200000;
    c->stage = (double *)orc_alloc((size_t)c->stagecap * ORC_STAGE_COLS);
    c->saveflow = (double *)orc_alloc((size_t)c->stagecap * ORC_POINT_COLS);
    double w0 = 0;
    for (size_t q = 0; q < N; q++) w0 += c->h[q] + c->vinf[q];
    c->b_water0 = w0;
    return c;
}

void orc_destroy(orc_ctx *c)
{
    if (!c) return;
    double *bufs[] = {c->h, c->hu, c->hv, c->z, c->zp, c->vinf, c->maxvel, c->maxdep, c->totm, c->dep,
                      c->totsed, c->rho, c->sxn, c->syn, c->sxp, c->syp, c->gzp, c->U, c->M, c->sed,
                      c->E, c->VF, c->srcf, c->fx, c->fy, c->rain, c->ks, c->stage, c->saveflow,
                      c->sx0, c->sy0, c->gz0};
    for (size_t f = 0; f < sizeof bufs / sizeof bufs[0]; f++) free(bufs[f]);
    free(c->solid);
    free(c);
}

int orc_advance(orc_ctx *c, double t_stop, int64_t max_steps, swehr_progress *pr)
{
    int st = SWEHR_OK;
    int64_t n = 0;
    if (c->status == SWEHR_CFL_ERROR) return SWEHR_CFL_ERROR;
    while (c->t < c->p.tend && c->t < t_stop && (max_steps < 0 || n < max_steps)) {
        st = orc_step(c);
        n++;
        if (st != SWEHR_OK) { c->status = st; break; }
    }
    if (pr) {
        memset(pr, 0, sizeof *pr);
        pr->t = c->t; pr->dt = c->dt; pr->courant = c->courant; pr->rain = c->R;
        pr->steps = c->steps; pr->steps_this_call = n; pr->status = st;
        pr->done = c->t >= c->p.tend;
        pr->t_step = c->t_prev;
    }
    return st;
}

int orc_read_field(orc_ctx *c, int field, int k, double *dst)
{
    size_t N = (size_t)c->N;
    const double *src = NULL;
    if ((field == SWEHR_FIELD_U || field == SWEHR_FIELD_M || field == SWEHR_FIELD_SED) && (k < 1 || k > c->S))
        return SWEHR_INVALID;
    switch (field) {
    case SWEHR_FIELD_H: src = c->h; break;
    case SWEHR_FIELD_HU: src = c->hu; break;
    case SWEHR_FIELD_HV: src = c->hv; break;
    case SWEHR_FIELD_Z: src = c->z; break;
    case SWEHR_FIELD_VINF: src = c->vinf; break;
    case SWEHR_FIELD_U: src = c->U + (size_t)(k - 1) * N; break;
    case SWEHR_FIELD_M: src = c->M + (size_t)(k - 1) * N; break;
    case SWEHR_FIELD_SED: src = c->sed + (size_t)(k - 1) * N; break;
    case SWEHR_FIELD_TOTM: src = c->totm; break;
    case SWEHR_FIELD_TOTSED: src = c->totsed; break;
    case SWEHR_FIELD_MAXVEL: src = c->maxvel; break;
    case SWEHR_FIELD_MAXDEPTH: src = c->maxdep; break;
    case SWEHR_FIELD_DEP: src = c->dep; break;
    case SWEHR_FIELD_VEL:
        for (size_t q = 0; q < N; q++) {
            double h = c->h[q];
            double v1 = h > c->p.hfilm ? c->hu[q] / h : 0, v2 = h > c->p.hfilm ? c->hv[q] / h : 0;
            dst[q] = M_POWH(v1 * v1 + v2 * v2);
        }
        return SWEHR_OK;
    default: return SWEHR_INVALID;
    }
    memcpy(dst, src, N * sizeof(double));
    return SWEHR_OK;
}

int orc_read_series(orc_ctx *c, double *stage, double *saveflow, int64_t max_rows, int64_t *rows)
{
    int64_t n = c->stagecnt < max_rows ? c->stagecnt : max_rows;
    if (stage) memcpy(stage, c->stage, (size_t)n * ORC_STAGE_COLS * sizeof(double));
    if (saveflow) memcpy(saveflow, c->saveflow, (size_t)n * ORC_POINT_COLS * sizeof(double));
    if (rows) *rows = n;
    return SWEHR_OK;
}

int orc_get_budget(orc_ctx *c, swehr_budget *b)
{
    memset(b, 0, sizeof *b);
    size_t N = (size_t)c->N;
    double w = 0;
    for (size_t q = 0; q < N; q++) w += c->h[q] + c->vinf[q];
    b->water_now = w;
    b->water_init = c->b_water0;
    b->rain_in = c->b_rain; b->outflow = c->b_out; b->clamp_gain = c->b_clamp;
    b->bulking = c->b_bulk; b->infiltration = c->b_inf;
    b->water_residual = (w - c->b_water0) - (c->b_rain - c->b_out + c->b_clamp + c->b_bulk);
    b->sclass = c->S;
    for (int k = 0; k < c->S; k++) {
        double s = 0;
        for (size_t q = 0; q < N; q++) s += c->U[(size_t)k * N + q] + c->M[(size_t)k * N + q];
        b->sed_now[k] = s;
        b->sed_init[k] = c->b_sed0[k];
        b->detach[k] = c->b_det[k];
        b->sed_outflow[k] = c->b_sout[k];
        b->sed_residual[k] = (s - c->b_sed0[k]) - (c->b_det[k] - c->b_sout[k]);
    }
    b->valid = 1;
    return SWEHR_OK;
}

double orc_time(orc_ctx *c) { return c->t; }

/* Slab runs: own rows lo..hi (1-based) -- only their faces enter the wave
 * speed; orc_step_prepare returns that speed, orc_step_commit finishes the
 * step with the largest one over all slabs; orc_rows copies every state
 * array of rows lo..hi out of (set = 0) or into (set = 1) buf, in the order
 * h hu hv z zp vinf maxvel maxdep totm dep totsed rho, then U_k, M_k, SED_k
 * per class: (12 + 3S) * ny values per row. */
void orc_set_own(orc_ctx *c, int lo, int hi)
{
    c->own_lo = lo;
    c->own_hi = hi;
}

double orc_step_prepare(orc_ctx *c)
{
    orc_prepare(c);
    return c->smax_own;
}

int orc_step_commit(orc_ctx *c, double smax)
{
    int st = orc_commit(c, smax);
    if (st != SWEHR_OK) c->status = st;
    return st;
}

int orc_rows(orc_ctx *c, int lo, int hi, double *buf, int set)
{
    if (lo < 1 || hi > c->nx || lo > hi) return SWEHR_INVALID;
    const size_t ny = (size_t)c->ny, N = (size_t)c->N, n = (size_t)(hi - lo + 1) * ny, off = (size_t)(lo - 1) * ny;
    double *planes[12] = {c->h, c->hu, c->hv, c->z, c->zp, c->vinf, c->maxvel, c->maxdep,
                          c->totm, c->dep, c->totsed, c->rho};
    size_t pos = 0;
    for (int f = 0; f < 12; f++, pos += n) {
        if (set) memcpy(planes[f] + off, buf + pos, n * sizeof(double));
        else memcpy(buf + pos, planes[f] + off, n * sizeof(double));
    }
    double *groups[3] = {c->U, c->M, c->sed};
    for (int g = 0; g < 3; g++)
        for (int k = 0; k < c->S; k++, pos += n) {
            double *pl = groups[g] + (size_t)k * N + off;
            if (set) memcpy(pl, buf + pos, n * sizeof(double));
            else memcpy(buf + pos, pl, n * sizeof(double));
        }
    return SWEHR_OK;
}

/* branch counters: 0 slope failures, 1 cells with debris forcing (DFMASK > 0),
 * 2 cells under the debris-flow override; cell-steps since creation */
int64_t orc_counter(orc_ctx *c, int which)
{
    return which == 0 ? c->n_fail : which == 1 ? c->n_dfmask : which == 2 ? c->n_debris : -1;
}
int64_t orc_steps(orc_ctx *c) { return c->steps; }

int orc_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* The update kernel's division by a constant c through its correctly rounded
 * reciprocal yc (two remainder corrections), restated for the test that
 * checks it against IEEE division on the CPU; same guards as the kernel. */
double orc_divk(double a, double c, double yc)
{
    double aa = fabs(a);
    if (aa >= 0x1p-900 && aa <= 0x1p900) {
        double q = a * yc;
        double r = fma(-c, q, a);
        q = fma(r, yc, q);
        r = fma(-c, q, a);
        return fma(r, yc, q);
    }
    if (a == 0 && c > 0) return a;
    return a / c;
}

/* count of n pseudo-random dividends (a xorshift stream from seed, spread
 * over [2^-960, 2^960] with both signs and random significands) whose
 * orc_divk quotient differs in any bit from a / c */
int64_t orc_divk_check(double c, int64_t n, uint64_t seed)
{
    double yc = 1.0 / c;
    int64_t bad = 0;
    uint64_t x = seed ? seed : 88172645463325252ull;
    for (int64_t k = 0; k < n; k++) {
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;
        uint64_t e = 1023 - 960 + (x % 1921);                 /* exponent 2^-960 .. 2^960 */
        uint64_t bits = ((x >> 11) & 0x000fffffffffffffull) | (e << 52) | ((x & 1) << 63);
        double a;
        memcpy(&a, &bits, sizeof a);
        double q1 = orc_divk(a, c, yc), q2 = a / c;
        if (memcmp(&q1, &q2, sizeof q1) != 0) bad++;
    }
    return bad;
}

/* Elementary-function entry points for the accuracy tests. */
double orc_m_pow(double x, double y) { return M_POW(x, y); }
double orc_m_powh(double x) { return M_POWH(x); }
double orc_m_exp(double x) { return M_EXP(x); }
double orc_m_cosatan(double x) { return M_COSATAN(x); }
double orc_m_sinatan(double x) { return M_SINATAN(x); }
