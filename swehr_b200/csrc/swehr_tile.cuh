/*
 * swehr_tile.cuh -- tiled kernels of one SWEHR time step (FP64 form).
 *
 * A CTA of 256 threads owns 8 x 32 cells (i x j, j contiguous in HBM) and
 * loops over tiles (persistent grid).  Per tile:
 *   A. the tile plus a one-cell halo (10 x 34 cells, ghosts resolved per
 *      SWEHR.c:816-1035) is staged in shared memory: h, the velocities
 *      u = hu/h and v = hv/h (0 when dry, SWEHR.c:333-352), the previous
 *      step's gravity GZ and sqrt(GZ h) of every cell that is the left/lower
 *      cell of a face, SED_k, TOTSED and DEP;
 *   B. every face of the tile is solved once (SWEHR.c:327-409) into shared
 *      memory: 9x32 x-faces and 8x33 y-faces for 256 cells;
 *   C. one thread per cell: sources (SWEHR.c:1239-1401), the conservative,
 *      Green-Ampt and class updates (SWEHR.c:1424-1511), the dry clamp,
 *      friction and maxima (SWEHR.c:1513-1588).
 * Every value is produced by the same operations in the same order as the
 * CPU restatement, so the FP64 results are bit-identical to it.
 *
 * The slope-failure test (SWEHR.c:1292-1312) costs six cos/sin(atan) and
 * neighbour slopes per cell but can only fire on steep, thick deposits: a
 * bound that needs none of them (sin(atan s) <= s, cos(atan s) >= 1 - s^2/2,
 * cos <= 1 in the pressure-gradient term) proves "no failure" with a 1e-6
 * relative margin for nearly every cell; the exact test runs otherwise.
 */
#pragma once
#include "swehr_device.cuh"
#include "swehr_faces.cuh"

namespace swehr {

#define T_I 8
#define T_J 32
#define H_I (T_I + 2)
#define H_J (T_J + 2)
#define N_H (H_I * H_J)
#define N_FX ((T_I + 1) * T_J)
#define N_FY (T_I * (T_J + 1))
#define TILE_THREADS 256

/* shared-memory layout of one tile (doubles), S classes */
struct TileLayout {
    int h, u, v, g, c, ts, dep, sed, fx, fy, up, red, total;
    __host__ __device__ static TileLayout make(int S)
    {
        TileLayout L;
        int o = 0;
        L.h = o; o += N_H;
        L.u = o; o += N_H;
        L.v = o; o += N_H;
        L.g = o; o += N_H;
        L.c = o; o += N_H;
        L.ts = o; o += N_H;
        L.dep = o; o += N_H;
        L.sed = o; o += S * N_H;
        L.fx = o; o += 3 * N_FX;
        L.fy = o; o += 3 * N_FY;
        L.up = o; o += (N_FX + N_FY + 7) / 8;          /* one byte per face */
        L.red = o; o += (TILE_THREADS / 32) * B_NTERMS;
        L.total = o;
        return L;
    }
};

/* hllc of SWEHR.c:327-409 with the velocities already formed
 * (nl = normal/ul, tl = tangential/vl; both 0 for a dry side) and the left
 * side's sqrt(g hl) given.  Same operations as hllc(). */
__device__ __forceinline__ double hllc_v(double hl, double hr, double nl, double nr, double tl, double tr,
                                         double g, double cl, double hfilm, double &T0, double &T1, double &T2)
{
    const double cr = sw_sqrt_pow(g * hr);
    const double d = nl + 2 * cl - nr - 2 * cr;
    const double hs = (d * d) / (16 * g);
    const double us = .5 * (nl + nr) + cl - cr;
    const double cs = sw_sqrt_pow(g * hs);
    double sl = nl - cl;
    if (us - cs < sl) sl = us - cs;
    double sm = us;
    double sr = nr + cr;
    if (us + cs > sr) sr = us + cs;
    if (hl <= hfilm) { sl = nr - 2 * cr; sm = sl; sr = nr + cr; }
    if (hr <= hfilm) { sl = nl - cl; sr = nl + 2 * cl; sm = sr; }
    double f0 = __longlong_as_double(0x7ff8000000000000LL), f1 = f0;
    if (sl >= 0) {
        f0 = hl * nl;
        f1 = hl * nl * nl + .5 * g * hl * hl;
    }
    if (sl <= 0 && sr >= 0) {
        f0 = (sr * (hl * nl) - sl * (hr * nr) + sl * sr * (hr - hl)) / (sr - sl);
        f1 = (sr * (hl * nl * nl + .5 * g * hl * hl) - sl * (hr * nr * nr + .5 * g * hr * hr)
              + sl * sr * (hr * nr - hl * nl)) / (sr - sl);
    }
    if (sr <= 0) {
        f0 = hr * nr;
        f1 = hr * nr * nr + .5 * g * hr * hr;
    }
    T0 = f0;
    T1 = f1;
    T2 = (sm >= 0) ? f0 * tl : f0 * tr;
    double s = 0;
    if (fabs(sl) > s) s = fabs(sl);
    if (fabs(sr) > s) s = fabs(sr);
    if (fabs(sm) > s) s = fabs(sm);
    return s;
}

/* wave speed only (the same sl, sr, sm as hllc_v) */
__device__ __forceinline__ double hll_speed(double hl, double hr, double nl, double nr, double g, double cl,
                                            double hfilm)
{
    const double cr = sw_sqrt_pow(g * hr);
    const double d = nl + 2 * cl - nr - 2 * cr;
    const double hs = (d * d) / (16 * g);
    const double us = .5 * (nl + nr) + cl - cr;
    const double cs = sw_sqrt_pow(g * hs);
    double sl = nl - cl;
    if (us - cs < sl) sl = us - cs;
    double sm = us;
    double sr = nr + cr;
    if (us + cs > sr) sr = us + cs;
    if (hl <= hfilm) { sl = nr - 2 * cr; sm = sl; sr = nr + cr; }
    if (hr <= hfilm) { sl = nl - cl; sr = nl + 2 * cl; sm = sr; }
    double s = 0;
    if (fabs(sl) > s) s = fabs(sl);
    if (fabs(sr) > s) s = fabs(sr);
    if (fabs(sm) > s) s = fabs(sm);
    return s;
}

struct TileCoord {
    int i0, j0;
};

__device__ __forceinline__ TileCoord tile_coord(const DevParams &P, int64_t tile)
{
    const int ntj = (P.ny + T_J - 1) / T_J;
    TileCoord t;
    t.i0 = (int)(tile / ntj) * T_I + 1;
    t.j0 = (int)(tile % ntj) * T_J + 1;
    return t;
}

/* Stage A: halo cells of the tile.  what: 0 = wave pass (h u v g c),
 * 1 = update pass (+ SED_k, TOTSED, DEP). */
template <int WHAT>
__device__ __forceinline__ void stage_halo(const DevParams &P, const double *__restrict__ src,
                                           const double *__restrict__ zp, TileCoord tc, double *sm,
                                           const TileLayout &TL, double inh, double inhv, double insed)
{
    const int64_t pl = P.plane;
    for (int idx = threadIdx.x; idx < N_H; idx += TILE_THREADS) {
        const int hi = idx / H_J, hj = idx % H_J;
        const int gi = tc.i0 - 1 + hi, gj = tc.j0 - 1 + hj;
        const bool hcorner = (hi == 0 || hi == H_I - 1) && (hj == 0 || hj == H_J - 1);
        const bool gx = gi == 0 || gi == P.nx + 1, gy = gj == 0 || gj == P.ny + 1;
        if (hcorner || gi > P.nx + 1 || gj > P.ny + 1 || (gx && gy)) continue;
        const int si = gi < 1 ? 1 : (gi > P.nx ? P.nx : gi);
        const int sj = gj < 1 ? 1 : (gj > P.ny ? P.ny : gj);
        const bool inflow = gj == P.ny + 1 && P.inflow;
        double h, hu, hv;
        const int64_t q = cidx(P, si, sj);
        if (inflow) {
            h = inh; hu = 0; hv = inhv;
        } else {
            h = src[P_H * pl + q];
            hu = src[P_HU * pl + q];
            hv = src[P_HV * pl + q];
            if ((gi == 0 && P.bndry[0] == 1) || (gi == P.nx + 1 && P.bndry[2] == 1)) hu = -hu;
            if ((gj == 0 && P.bndry[1] == 1) || (gj == P.ny + 1 && P.bndry[3] == 1)) hv = -hv;
        }
        double u = 0, v = 0;
        if (h > P.hfilm) { u = hu / h; v = hv / h; }
        sm[TL.h + idx] = h;
        sm[TL.u + idx] = u;
        sm[TL.v + idx] = v;
        if (hi <= T_I && hj <= T_J) {
            const double g = gz_of(P, zp, si, sj);
            sm[TL.g + idx] = g;
            sm[TL.c + idx] = sw_sqrt_pow(g * h);
        }
        if (WHAT == 1) {
            for (int k = 0; k < P.S; k++)
                sm[TL.sed + k * N_H + idx] = inflow ? insed : sed_of(src[(P_FIXED + k) * pl + q], h, P.hfilm);
            if (!gx && !gy) {
                sm[TL.ts + idx] = src[P_TOTSED * pl + q];
                sm[TL.dep + idx] = src[P_DEP * pl + q];
            }
        }
    }
}

/* ------------------------------------------------------------------ wave */
__global__ void __launch_bounds__(TILE_THREADS) k_wave_tile(const DevParams P, const Bufs B, Ctl *ctl)
{
    if (!ctl->active) return;
    extern __shared__ double sm[];
    const TileLayout TL = TileLayout::make(0);
    const int64_t n = ctl->step;
    const double t = ctl->t;
    const double *src = B.set[n & 1];
    const double *zp = B.z[(n + 2) % 3];
    double inh = 0, inhv = 0, insed = 0;
    if (P.inflow) inflow_ghost(t, inh, inhv, insed);
    const int64_t ntiles = (int64_t)((P.nx + T_I - 1) / T_I) * ((P.ny + T_J - 1) / T_J);
    double smax = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const TileCoord tc = tile_coord(P, tile);
        stage_halo<0>(P, src, zp, tc, sm, TL, inh, inhv, insed);
        __syncthreads();
        /* faces owned by the tile: i+1/2 and j+1/2 of its cells, plus the
         * domain's low boundary faces 1/2 */
        for (int f = threadIdx.x; f < N_FX + N_FY; f += TILE_THREADS) {
            if (f < N_FX) {
                const int fi = f / T_J, fj = f % T_J;
                const int gi = tc.i0 - 1 + fi, gj = tc.j0 + fj;
                if (gj > P.ny || gi > P.nx || (fi == 0 && gi != 0)) continue;
                const int L = fi * H_J + fj + 1, R = L + H_J;
                const double s = hll_speed(sm[TL.h + L], sm[TL.h + R], sm[TL.u + L], sm[TL.u + R], sm[TL.g + L],
                                           sm[TL.c + L], P.hfilm);
                smax = (s > smax) ? s : smax;
            } else {
                const int f2 = f - N_FX;
                const int fi = f2 / (T_J + 1), fj = f2 % (T_J + 1);
                const int gi = tc.i0 + fi, gj = tc.j0 - 1 + fj;
                if (gi > P.nx || gj > P.ny || (fj == 0 && gj != 0)) continue;
                const int L = (fi + 1) * H_J + fj, R = L + 1;
                const double s = hll_speed(sm[TL.h + L], sm[TL.h + R], sm[TL.v + L], sm[TL.v + R], sm[TL.g + L],
                                           sm[TL.c + L], P.hfilm);
                smax = (s > smax) ? s : smax;
            }
        }
        __syncthreads();
    }
    __shared__ double red[TILE_THREADS / 32];
    __shared__ bool last;
    smax = warp_max(smax);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = smax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0;
        for (int w = 0; w < TILE_THREADS / 32; w++) m = (red[w] > m) ? red[w] : m;
        atomicMax(&ctl->smax_bits, (unsigned long long)__double_as_longlong(m));
        __threadfence();
        unsigned tk = atomicAdd(&ctl->wave_ticket, 1u);
        last = (tk == gridDim.x - 1);
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    /* CFL time step, SWEHR.c:1409-1413 */
    const double Smax = __longlong_as_double((long long)atomicAdd(&ctl->smax_bits, 0ull));
    double dt = P.cstable * P.dx / Smax;
    if (dt > P.maxstep) dt = P.maxstep;
    if (t + dt > P.tend) dt = P.tend - t;
    const double courant = Smax * dt * P.oneoverdx;
    ctl->dt = dt;
    ctl->courant = courant;
    ctl->cfl = courant > 1;
    ctl->smax_bits = 0ull;
    ctl->wave_ticket = 0u;
    ctl->pending = 1;
}

/* ---------------------------------------------------------------- update */
template <int MAXS, bool BUDGET>
struct Acc2 {
    double rain, out, clamp, bulk, inf;
    double det[BUDGET ? MAXS : 1], sout[BUDGET ? MAXS : 1];
};

/* Parameters of the exact slope-failure test (passed by value: a pointer to
 * the kernel's parameter block would force a local copy of all of it). */
struct FailArgs {
    int32_t nx, ny, pitch, pad_;
    int64_t plane;
    double oneoverdx, half_odx, rho0, rhow, cohesion, fa;
};

__device__ __forceinline__ double fa_slope_x(const FailArgs &A, const double *__restrict__ z, int i, int j)
{
    const int64_t p = A.pitch;
    const int64_t q = (int64_t)(i - 1) * p + (j - 1);
    if (i != 1 && i != A.nx) return A.half_odx * (z[q + p] - z[q - p]);
    if (i == A.nx) return A.oneoverdx * (z[q] - z[q - p]);
    return A.oneoverdx * (z[q + p] - z[q]);
}

__device__ __forceinline__ double fa_slope_y(const FailArgs &A, const double *__restrict__ z, int i, int j)
{
    const int64_t q = (int64_t)(i - 1) * A.pitch + (j - 1);
    if (j != 1 && j != A.ny) return A.half_odx * (z[q + 1] - z[q - 1]);
    if (j == A.ny) return A.oneoverdx * (z[q] - z[q - 1]);
    return A.oneoverdx * (z[q + 1] - z[q]);
}

/* Exact slope-failure test, SWEHR.c:1292-1312 (rarely needed). */
__device__ __noinline__ double fail_exact(const FailArgs A, const double *__restrict__ dep_plane,
                                          const double *__restrict__ zp, const double *__restrict__ zc, int i, int j,
                                          double sx, double sy, double gz, double dep0, double rho0c, double h0v)
{
    const int iu = (i < A.nx) ? i + 1 : A.nx, id = (i > 1) ? i - 1 : 1;
    const int ju = (j < A.ny) ? j + 1 : A.ny, jd = (j > 1) ? j - 1 : 1;
    const double sxu = (iu == i) ? sx : fa_slope_x(A, zp, iu, j);
    const double sxd = (id == i) ? sx : fa_slope_x(A, zc, id, j);
    const double syu = (ju == j) ? sy : fa_slope_y(A, zp, i, ju);
    const double syd = (jd == j) ? sy : fa_slope_y(A, zc, i, jd);
    const double rho0 = A.rho0;
    auto D = [&](int ii, int jj) { return dep_plane[(int64_t)(ii - 1) * A.pitch + (jj - 1)]; };
    double fail = 0;
    double pgfx = dep0 * rho0 * gz * 0.5 * A.oneoverdx
                  * (D(iu, j) * sw_cos_atan(fabs(sxu)) - D(id, j) * sw_cos_atan(fabs(sxd)));
    if (pgfx * sx > 0) pgfx = -1 * fabs(pgfx);
    if (pgfx * sx < 0) pgfx = fabs(pgfx);
    const double lhs = (rho0 * gz * dep0 + rho0c * gz * h0v) * sw_sin_atan(fabs(sy));
    const double nrm = (rho0 * gz * dep0 + rho0c * gz * h0v) * sw_cos_atan(fabs(sy)) - A.rhow * gz * (dep0 + h0v);
    if (fail == 0 && (lhs > (A.cohesion + nrm * A.fa + pgfx))) fail = 1;
    double pgfy = dep0 * rho0 * gz * 0.5 * A.oneoverdx
                  * (D(i, ju) * sw_cos_atan(fabs(syu)) - D(i, jd) * sw_cos_atan(fabs(syd)));
    if (pgfy * sy > 0) pgfy = -1 * fabs(pgfy);
    if (pgfy * sy < 0) pgfy = fabs(pgfy);
    if (fail == 0 && (lhs > (A.cohesion + nrm * A.fa + pgfy))) fail = 1;
    return fail;
}

template <int MAXS, bool BUDGET>
__device__ __forceinline__ void tile_cell(const DevParams &P, const double *__restrict__ src, double *__restrict__ dst,
                                          const double *__restrict__ zp, const double *__restrict__ zc,
                                          double *__restrict__ zn, const double *__restrict__ ksf, const double *sm,
                                          const TileLayout &TL, TileCoord tc, double t, double dt, double Rr,
                                          Acc2<MAXS, BUDGET> &acc)
{
    const int ti = threadIdx.x / T_J, tj = threadIdx.x % T_J;
    const int i = tc.i0 + ti, j = tc.j0 + tj;
    if (i > P.nx || j > P.ny) return;
    const int64_t pl = P.plane;
    const int64_t q = cidx(P, i, j);
    const int S = P.S;
    const double hfilm = P.hfilm, rhos = P.rhos, rhow = P.rhow;
    const int hs = (ti + 1) * H_J + (tj + 1);                      /* this cell in halo coords */
    const double h0v = sm[TL.h + hs];
    const double hu0 = src[P_HU * pl + q], hv0 = src[P_HV * pl + q];
    const double totsed0 = sm[TL.ts + hs], dep0 = sm[TL.dep + hs];
    const double totm0 = src[P_TOTM * pl + q];
    double rho0c = rhow * (1 - totsed0) + rhos * totsed0;
    if (rho0c > P.rhos08) rho0c = P.rhos08;
    const double Rc = P.storm ? storm_at(P, t, i, j) : Rr;

    /* faces of this cell (computed in stage B) */
    const int fxl = ti * T_J + tj, fxr = (ti + 1) * T_J + tj;
    const int fyl = ti * (T_J + 1) + tj, fyr = fyl + 1;
    const unsigned char *up = reinterpret_cast<const unsigned char *>(sm + TL.up);
    const double *FX = sm + TL.fx, *FY = sm + TL.fy;
    const double fxl0 = FX[3 * fxl], fxl1 = FX[3 * fxl + 1], fxl2 = FX[3 * fxl + 2];
    const double fxr0 = FX[3 * fxr], fxr1 = FX[3 * fxr + 1], fxr2 = FX[3 * fxr + 2];
    const double fyl0 = FY[3 * fyl], fyl1 = FY[3 * fyl + 1], fyl2 = FY[3 * fyl + 2];
    const double fyr0 = FY[3 * fyr], fyr1 = FY[3 * fyr + 1], fyr2 = FY[3 * fyr + 2];
    /* upwind cells of the sediment fluxes, halo index */
    const int uxl = up[fxl] ? hs : hs - H_J;
    const int uxr = up[fxr] ? hs + H_J : hs;
    const int uyl = up[N_FX + fyl] ? hs : hs - 1;
    const int uyr = up[N_FX + fyr] ? hs + 1 : hs;

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
                  * (sm[TL.ts + hs + H_J] - sm[TL.ts + hs - H_J]);
    if (j > 1 && j < P.ny)
        gammay -= (rhos - rho0c) * gz * h0v * h0v / (2 * rho0c) * .5 * P.oneoverdx
                  * (sm[TL.ts + hs + 1] - sm[TL.ts + hs - 1]);
    /* slope stability: provable "no failure" first, exact test otherwise */
    double fail = 0;
    {
        const double rho0 = P.rho0;
        const double A = rho0 * gz * dep0 + rho0c * gz * h0v;
        const double s = fabs(sy);
        const double depx = fabs(sm[TL.dep + (i < P.nx ? hs + H_J : hs)]) + fabs(sm[TL.dep + (i > 1 ? hs - H_J : hs)]);
        const double depy = fabs(sm[TL.dep + (j < P.ny ? hs + 1 : hs)]) + fabs(sm[TL.dep + (j > 1 ? hs - 1 : hs)]);
        const double pb = fabs(dep0) * rho0 * fabs(gz) * 0.5 * P.oneoverdx * fmax(depx, depy);
        const double w = P.rhow * gz * (dep0 + h0v);
        const double lhs_ub = A * s;
        const double rhs_lb = P.cohesion + (A * (1 - 0.5 * s * s) - w) * P.fa - pb;
        const double margin = 1e-6 * (fabs(A) * (1 + s) + P.cohesion + fabs(w) * P.fa + pb) + 1e-300;
        const bool safe = A >= 0 && gz > 0 && P.fa >= 0 && lhs_ub + margin < rhs_lb;
        if (!safe) {
            FailArgs fa;
            fa.nx = P.nx; fa.ny = P.ny; fa.pitch = P.pitch; fa.pad_ = 0; fa.plane = P.plane;
            fa.oneoverdx = P.oneoverdx; fa.half_odx = P.half_odx; fa.rho0 = P.rho0; fa.rhow = P.rhow;
            fa.cohesion = P.cohesion; fa.fa = P.fa;
            fail = fail_exact(fa, src + P_DEP * pl, zp, zc, i, j, sx, sy, gz, dep0, rho0c, h0v);
        }
    }
    double dfmask = fmin(1.0, (totsed0 - 0.2) / 0.2);
    if (h0v < P.h0x9 || totsed0 < 0.2) dfmask = 0;
    double betax = P.neg1ml * gz * h0v * P.fa;
    double betay = P.neg1ml * gz * h0v * P.fa;
    if (hu0 < 0) betax = -1 * betax;
    if (hv0 < 0) betay = -1 * betay;

    /* Hairsine-Rose, class-independent parts (SWEHR.c:1330-1382) */
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
    double E3b = 0, E4b = 0, e4den = 1;
    if (swash) {
        const double manning = (h0v <= P.hc) ? P.roughness * sw_pow(h0v / P.hc, P.dde) : P.roughness;
        const double qq = sw_sqrt_pow(hu0 * hu0 + hv0 * hv0);
        const double SF = manning * manning * qq * qq / sw_pow(h0v, 3.333);
        /* streampowererosion (SWEHR.c:412-426): omega is the same for every
         * class; only the h > d_k condition differs */
        const double omega = rho0c * gz * SF * qq;
        if (omega > P.uc && totsed0 < 0.6) E3b = P.af * (omega - P.uc);
        if (omega > P.uc2 && totsed0 < 0.6) E4b = P.afr * (omega - P.uc2);
        e4den = (rhos - rho0c) / rhos * gz * h0v;
    }
    const double vfconc = sw_pow(1 - fmin(totsed0, 0.99), 4.0);
    const bool debris = (h0v > P.h0x9 && totsed0 > P.cthreshold);

    /* conservative update + Green-Ampt, SWEHR.c:1424-1452 */
    const double dtdx = dt * P.oneoverdx;
    double h = h0v - dtdx * (fxr0 - fxl0) - dtdx * (fyr0 - fyl0) + dt * Rc;
    double hu = hu0 - dtdx * (fxr1 - fxl1) - dtdx * (fyr1 - fyl1) + dt * SXf + dt * gammax + dt * dfmask * betax;
    double hv = hv0 - dtdx * (fxr2 - fxl2) - dtdx * (fyr2 - fyl2) + dt * SYf + dt * gammay + dt * dfmask * betay;
    const double ks = P.has_ks ? ksf[q] : P.ks;
    const double vinf0 = src[P_VINF * pl + q];
    const double zf = vinf0 / (P.thetas - P.theta0);
    const double infl = fmin(h - hfilm, dt * ks * (zf + P.hf + h) / zf);
    const double vinf = vinf0 + infl;
    h -= infl;

    /* classes (SWEHR.c:1454-1511) */
    const double *SED = sm + TL.sed;
    double Uk[MAXS];
#pragma unroll
    for (int k = 0; k < MAXS; k++) {
        if (k >= S) break;
        const double *sk = SED + k * N_H;
        Uk[k] = src[(P_FIXED + k) * pl + q] - dtdx * (fxr0 * sk[uxr] - fxl0 * sk[uxl])
                - dtdx * (fyr0 * sk[uyr] - fyl0 * sk[uyl]);
    }
    double z = zc[q];
    double totm = 0, dep = 0, chtemp = 0, bulk = 0;
#pragma unroll
    for (int k = 0; k < MAXS; k++) {
        if (k >= S) break;
        const int64_t qm = (P_FIXED + S + k) * pl + q;
        const double Mk0 = src[qm];
        double E1 = 0, E2 = 0, E3 = 0, E4 = 0;
        if (swash) {
            E1 = (1 - Hs) * P.pf[k] * P.a * Rc;
            if (totm0 > 1e-8 && Mk0 > 1e-8) E2 = Hs * Mk0 / totm0 * P.ad * Rc;
            if (deepv) { E1 = E1 * depthfac; E2 = E2 * depthfac; }
            E3 = (1 - Hs) * P.pf[k] * P.F / P.J * (h0v > P.ds[k] ? E3b : 0.0);
            if (totm0 > 1e-6 && Mk0 > 0)
                E4 = P.one_m_bb * Hs * Mk0 / totm0 * P.F / e4den * (h0v > P.ds[k] ? E4b : 0.0);
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
            if (BUDGET) acc.det[k] += dt * E1;
        } else {
            chtemp = u;
            const double redetach = fmin(Mk, dt * (E2 + E4));
            const double dec = sw_exp(-VF / h * (0.5 * dt));
            u = dec * u;
            u = u + dt * (E1 + E3) + redetach;
            u = dec * u;
            z = z - P.invporo * (u - chtemp);
            Mk = Mk + dt * (E1 + E3) - (u - chtemp);
            if (BUDGET) acc.det[k] += dt * (E1 + E3);
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
        const double manning = (h <= P.hc) ? P.roughness * sw_pow(h / P.hc, P.dde) : P.roughness;
        const double SFf = manning * manning * gz * sw_sqrt_pow(hu * hu + hv * hv) * 1 / sw_pow(h, 2.333);
        hu = hu / (1 + dt * SFf);
        hv = hv / (1 + dt * SFf);
        vel1 = hu / h;
        vel2 = hv / h;
    }
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

    if (BUDGET) {
        acc.rain += dt * Rc;
        acc.inf += infl;
        acc.clamp += clamp;
        acc.bulk += bulk;
        if (i == 1 || i == P.nx || j == 1 || j == P.ny) {
#pragma unroll
            for (int k = 0; k < MAXS; k++) {
                if (k >= S) break;
                const double *sk = SED + k * N_H;
                if (i == 1) acc.sout[k] -= dtdx * (fxl0 * sk[uxl]);
                if (i == P.nx) acc.sout[k] += dtdx * (fxr0 * sk[uxr]);
                if (j == 1) acc.sout[k] -= dtdx * (fyl0 * sk[uyl]);
                if (j == P.ny) acc.sout[k] += dtdx * (fyr0 * sk[uyr]);
            }
            if (i == 1) acc.out -= dtdx * fxl0;
            if (i == P.nx) acc.out += dtdx * fxr0;
            if (j == 1) acc.out -= dtdx * fyl0;
            if (j == P.ny) acc.out += dtdx * fyr0;
        }
    }
}

/* stage row of SWEHR.c:1593-1676 from the new state (one block) */
__device__ __forceinline__ void stage_sample_tile(const DevParams &P, const double *__restrict__ st, Ctl *ctl, double tnew,
                                  double *stage, double *saveflow, double *scratch)
{
    double *bv = scratch;
    int *bi = reinterpret_cast<int *>(scratch + TILE_THREADS);
    const int64_t pl = P.plane;
    const int row = P.outlet_row;
    double best = 0;
    int besti = 1;
    for (int i = 1 + threadIdx.x; i <= P.nx; i += blockDim.x) {
        const double h = st[P_H * pl + cidx(P, i, row)];
        if (h > best) { best = h; besti = i; }
    }
    bv[threadIdx.x] = best;
    bi[threadIdx.x] = besti;
    __syncthreads();
    if (threadIdx.x != 0) return;
    int outlet = 1;
    double ob = 0;
    for (int w = 0; w < (int)blockDim.x; w++)
        if (bv[w] > ob || (bv[w] == ob && bv[w] > 0 && bi[w] < outlet)) { ob = bv[w]; outlet = bi[w]; }
    const int64_t r = ctl->stagecnt;
    double *row_out = stage + r * 24;
    const int64_t qo = cidx(P, outlet, row);
    const double ho = st[P_H * pl + qo];
    const double v1 = ho > P.hfilm ? st[P_HU * pl + qo] / ho : 0, v2 = ho > P.hfilm ? st[P_HV * pl + qo] / ho : 0;
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
        const int xi = P.xpoint[m], yj = P.ypoint[m];
        if (m >= P.npoints || xi < 1 || xi > P.nx || yj < 1 || yj > P.ny) {
            pr[3 * m] = pr[3 * m + 1] = pr[3 * m + 2] = __longlong_as_double(0x7ff8000000000000LL);
            continue;
        }
        const int64_t qp = cidx(P, xi, yj);
        const double hp = st[P_H * pl + qp];
        const double w1 = hp > P.hfilm ? st[P_HU * pl + qp] / hp : 0, w2 = hp > P.hfilm ? st[P_HV * pl + qp] / hp : 0;
        pr[3 * m] = hp;
        pr[3 * m + 1] = sw_sqrt_pow(w1 * w1 + w2 * w2);
        pr[3 * m + 2] = st[P_TOTSED * pl + qp];
    }
    ctl->stagecnt = r + 1;
    ctl->stageinterval += P.stageint;
}

template <int MAXS, bool BUDGET>
__global__ void __launch_bounds__(TILE_THREADS, 2) k_update_tile(const DevParams P, const Bufs B, Ctl *ctl,
                                                                  const double *__restrict__ rain, double *partials,
                                                                  double *stage, double *saveflow)
{
    if (!ctl->pending) return;
    extern __shared__ double sm[];
    const TileLayout TL = TileLayout::make(P.S);
    const int64_t n = ctl->step;
    const double t = ctl->t, dt = ctl->dt;
    const double *src = B.set[n & 1];
    double *dst = B.set[(n + 1) & 1];
    const double *zp = B.z[(n + 2) % 3], *zc = B.z[n % 3];
    double *zn = B.z[(n + 1) % 3];
    double inh = 0, inhv = 0, insed = 0;
    if (P.inflow) inflow_ghost(t, inh, inhv, insed);
    const double Rr = P.storm ? 0.0 : rain_at(P, rain, t);
    Acc2<MAXS, BUDGET> acc;
    acc.rain = acc.out = acc.clamp = acc.bulk = acc.inf = 0;
#pragma unroll
    for (int k = 0; k < (BUDGET ? MAXS : 1); k++) acc.det[k] = acc.sout[k] = 0;
    const int64_t ntiles = (int64_t)((P.nx + T_I - 1) / T_I) * ((P.ny + T_J - 1) / T_J);
    unsigned char *upb = reinterpret_cast<unsigned char *>(sm + TL.up);
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const TileCoord tc = tile_coord(P, tile);
        stage_halo<1>(P, src, zp, tc, sm, TL, inh, inhv, insed);
        __syncthreads();
        /* stage B: faces */
        for (int f = threadIdx.x; f < N_FX + N_FY; f += TILE_THREADS) {
            double T0, T1, T2;
            if (f < N_FX) {
                const int fi = f / T_J, fj = f % T_J;
                const int gi = tc.i0 - 1 + fi, gj = tc.j0 + fj;
                if (gj > P.ny || gi > P.nx) continue;
                const int L = fi * H_J + fj + 1, R = L + H_J;
                hllc_v(sm[TL.h + L], sm[TL.h + R], sm[TL.u + L], sm[TL.u + R], sm[TL.v + L], sm[TL.v + R],
                       sm[TL.g + L], sm[TL.c + L], P.hfilm, T0, T1, T2);
                double *F = sm + TL.fx + 3 * f;
                F[0] = T0; F[1] = T1; F[2] = T2;
                upb[f] = (T0 > 0) ? 0 : 1;
            } else {
                const int f2 = f - N_FX;
                const int fi = f2 / (T_J + 1), fj = f2 % (T_J + 1);
                const int gi = tc.i0 + fi, gj = tc.j0 - 1 + fj;
                if (gi > P.nx || gj > P.ny) continue;
                const int L = (fi + 1) * H_J + fj, R = L + 1;
                hllc_v(sm[TL.h + L], sm[TL.h + R], sm[TL.v + L], sm[TL.v + R], sm[TL.u + L], sm[TL.u + R],
                       sm[TL.g + L], sm[TL.c + L], P.hfilm, T0, T1, T2);
                double *F = sm + TL.fy + 3 * f2;
                F[0] = T0; F[1] = T2; F[2] = T1;
                upb[f] = (T0 > 0) ? 0 : 1;
            }
        }
        __syncthreads();
        tile_cell<MAXS, BUDGET>(P, src, dst, zp, zc, zn, B.ks, sm, TL, tc, t, dt, Rr, acc);
        __syncthreads();
    }
    __shared__ bool last;
    double *red = sm + TL.red;
    if (BUDGET) {
        double v[B_NTERMS];
        v[B_RAIN] = acc.rain; v[B_OUT] = acc.out; v[B_CLAMP] = acc.clamp; v[B_BULK] = acc.bulk; v[B_INF] = acc.inf;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            v[B_DET + k] = (k < MAXS) ? acc.det[k < MAXS ? k : 0] : 0.0;
            v[B_SOUT + k] = (k < MAXS) ? acc.sout[k < MAXS ? k : 0] : 0.0;
        }
#pragma unroll
        for (int m = 0; m < B_NTERMS; m++) {
            const double s = warp_sum(v[m]);
            if ((threadIdx.x & 31) == 0) red[(threadIdx.x >> 5) * B_NTERMS + m] = s;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        if (BUDGET) {
            for (int m = 0; m < B_NTERMS; m++) {
                double s = 0;
                for (int w = 0; w < TILE_THREADS / 32; w++) s += red[w * B_NTERMS + m];
                partials[(int64_t)blockIdx.x * B_NTERMS + m] = s;
            }
        }
        __threadfence();
        const unsigned tk = atomicAdd(&ctl->update_ticket, 1u);
        last = (tk == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (BUDGET && threadIdx.x < B_NTERMS) {
        double hi = 0, lo = 0;
        for (unsigned b = 0; b < gridDim.x; b++)
            dd_add(hi, lo, ((volatile double *)partials)[(int64_t)b * B_NTERMS + threadIdx.x]);
        double Hh = ctl->budget_hi[threadIdx.x], Ll = ctl->budget_lo[threadIdx.x];
        dd_add(Hh, Ll, hi);
        Ll += lo;
        ctl->budget_hi[threadIdx.x] = Hh;
        ctl->budget_lo[threadIdx.x] = Ll;
    }
    const double tnew = (ctl->cfl ? 2 * P.tend : t) + dt;
    const bool stage_due = tnew > ctl->stageinterval && ctl->stagecnt < ctl->stagecap;
    __syncthreads();
    if (stage_due) stage_sample_tile(P, dst, ctl, tnew, stage, saveflow, sm);
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->t = tnew;
        ctl->step = n + 1;
        ctl->pending = 0;
        ctl->update_ticket = 0u;
        if (ctl->cfl) ctl->status = 1;
        if (!(dt > 0) && !ctl->cfl) ctl->status = 2;
        if (ctl->cfl || !(dt > 0) || !(tnew < P.tend) || !(tnew < ctl->t_stop) || n + 1 >= ctl->max_step)
            ctl->active = 0;
        ctl->launches += 2;
    }
}

}  // namespace swehr
