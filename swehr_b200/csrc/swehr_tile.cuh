/*
 * swehr_tile.cuh -- tiled kernels of one SWEHR time step, templated on the
 * arithmetic of the form:
 *   PolicyF64  plain form: every value FP64, elementary functions from
 *              swehr_math.h; with --fmad=false bit-identical to the CPU
 *              restatement built with the same math;
 *   PolicyF32  mixed form: h, hu, hv, U_k, the maxima, TOTM, DEP, TOTSED and
 *              Ks stored and computed in FP32 with the SFU intrinsics; z, the
 *              cumulative infiltration and its Green-Ampt update, the
 *              deposited mass M_k, dt/t and the budgets stay FP64.
 *
 * A CTA of 256 threads owns 8 x 32 cells (i x j, j contiguous in HBM) and
 * loops over tiles (persistent grid) of the rows the context updates (all
 * rows, or a slab's own rows: DevParams own_lo..own_hi).  Per tile:
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
#include "swehr_kernels.h"
#include "swehr_tma.cuh"

#include <cuda_pipeline_primitives.h>

/* Tile shape: T_I x T_J cells, one per thread of a 256-thread block.  A
 * translation unit may build the kernels for another shape by defining
 * SWEHR_TILE_I, SWEHR_TILE_J and SWEHR_TILE_NS before including this
 * header: everything below then lives in the inline namespace
 * swehr::SWEHR_TILE_NS, so two shapes in one library never share a symbol.
 * The per-cell arithmetic does not depend on the shape. */
#ifndef SWEHR_TILE_I
#define SWEHR_TILE_I 8
#define SWEHR_TILE_J 32
#define SWEHR_TILE_NS t8x32
#endif
static_assert(SWEHR_TILE_I * SWEHR_TILE_J == 256, "a tile is one cell per thread of a 256-thread block");
static_assert(SWEHR_TILE_J % 4 == 0, "staged rows start 16-byte aligned");

namespace swehr {
inline namespace SWEHR_TILE_NS {

#define T_I SWEHR_TILE_I
#define T_J SWEHR_TILE_J
#define H_I (T_I + 2)
#define H_J (T_J + 2)
#define N_H (H_I * H_J)
#define N_FX ((T_I + 1) * T_J)
#define N_FY (T_I * (T_J + 1))
#define TILE_THREADS 256

/* ------------------------------------------------------------ policies --- */
struct PolicyF64 {
    typedef double R;
    static constexpr int kMinBlocks = 2;      /* CTAs per SM the update kernel is register-budgeted for */
    static constexpr int kBatchMinBlocks = 2; /* ... and the batched update kernel */
    /* the class loop of the cell update kept rolled: its unrolled body (eight
     * inline exp and division sequences) costs more in instruction fetch
     * than unrolling gains (measured: update -4 % rolled) */
    static constexpr bool kRollClasses = true;
    /* wave pass: two cells per thread (16-byte loads) at 3 CTAs per SM (80
     * registers); measured against one cell per thread at 5 CTAs: wet steps
     * -0.06 ms, early steps +0.03 ms per 4096^2 step */
    static constexpr int kWaveMinBlocks = 3;
    /* skip the division of the density-gradient term where the TOTSED
     * gradient is an exact zero (see tile_cell; measured: early steps -1 %) */
    static constexpr bool kKnownResults = true;
    static __device__ __forceinline__ R sqrtp(R x) { return sw_sqrt_pow(x); }
    static __device__ __forceinline__ R pow(R x, R y) { return sw_pow(x, y); }
    static __device__ __forceinline__ R exp(R x) { return sw_exp(x); }
    static __device__ __forceinline__ R cos_atan(R x) { return sw_cos_atan(x); }
    static __device__ __forceinline__ R sin_atan(R x) { return sw_sin_atan(x); }
    static __device__ __forceinline__ R div(R a, R b) { return a / b; }
    /* a / b where a is often an exact zero: a zero over a positive divisor
     * is that zero (sign included), so the division sequence is skipped; any
     * other operands divide as usual (bit-identical to a / b) */
    static __device__ __forceinline__ R divz(R a, R b)
    {
        if (a == 0 && b > 0) return a;
        return a / b;
    }
    /* sqrtp of an argument that is often an exact zero (sqrtp(+-0) = +0) */
    static __device__ __forceinline__ R sqrtz(R x)
    {
        if (x == 0) return R(0);
        return sqrtp(x);
    }
    static __device__ __forceinline__ R qnan() { return __longlong_as_double(0x7ff8000000000000LL); }
    /* a / c for a constant divisor c in [2^-100, 2^100] whose correctly
     * rounded reciprocal yc the host computed, without the division
     * sequence: q0 = a yc, then two remainder corrections (Markstein).  The
     * first leaves q within one ulp of a/c (a faithful quotient), so the
     * second remainder a - c q is exact and q + r yc rounds to the correctly
     * rounded a/c (Markstein's theorem for a reciprocal within half an ulp).
     * Taken only for |a| in [2^-900, 2^900], where no step under- or
     * overflows; a zero over the positive c is that zero; anything else, or
     * a launch whose constants are out of range (ok = 0), divides as usual.
     * The result is the IEEE quotient a / c in every case. */
    static __device__ __forceinline__ R divk(R a, R c, R yc, int ok)
    {
        const R aa = fabs(a);
        if (ok && aa >= 0x1p-900 && aa <= 0x1p900) {
            R q = a * yc;
            R r = fma(-c, q, a);
            q = fma(r, yc, q);
            r = fma(-c, q, a);
            return fma(r, yc, q);
        }
        if (a == 0 && c > 0) return a;
        return a / c;
    }
    /* The flow-detachment terms E3 = (num / J) m and E4 = ((A / T) F / e) m
     * of SWEHR.c:1365-1375, where the factor m (the excess stream power) is
     * an exact zero wherever flow is below its critical power: the IEEE
     * product of a finite quotient with a zero is a zero whose sign is the
     * xor of the operands' signs, so the division sequences are skipped when
     * m == 0 and the ranges below keep every intermediate finite; anything
     * else is computed as written (bit-identical either way). */
    static __device__ __forceinline__ R zero_xor(long long s) { return __longlong_as_double(s & (1LL << 63)); }
    static __device__ __forceinline__ R e3_term(R num, R J, R yJ, int ok, R m)
    {
        if (m == 0 && ok && fabs(num) <= 0x1p900)
            return zero_xor(__double_as_longlong(num) ^ __double_as_longlong(J) ^ __double_as_longlong(m));
        return divk(num, J, yJ, ok) * m;
    }
    /* T > 1e-6 here (SWEHR.c:1368) */
    static __device__ __forceinline__ R e4_term(R A, R T, R F, R e, R m)
    {
        const R ae = fabs(e);
        if (m == 0 && fabs(A) <= 0x1p500 && fabs(F) <= 0x1p100 && ae >= 0x1p-300 && ae <= 0x1p300)
            return zero_xor(__double_as_longlong(A) ^ __double_as_longlong(T) ^ __double_as_longlong(F) ^
                            __double_as_longlong(e) ^ __double_as_longlong(m));
        return div(div(A, T) * F, e) * m;
    }
    /* settling velocity of Cao 2006 (SWEHR.c:435): sqrt(A^2 + c) - A, in the
     * reference's operation order */
    static __device__ __forceinline__ R settle(R A, R A2, R c) { return sqrtp(A2 + c) - A; }
    /* deposited thickness of a deposited mass, DEP += M_k / rhos (SWEHR.c:1510) */
    static __device__ __forceinline__ double dep_of(double M, const DevParams &P)
    {
        return divk(M, P.rhos, P.inv_rhos, P.divk_ok);
    }
};

struct PolicyF32 {
    typedef float R;
    static constexpr int kMinBlocks = 3;
    /* the batched update reads its scenario's parameters from shared memory,
     * not the constant bank, and needs more registers: at 3 CTAs per SM it
     * spilled ~260 B per thread; at 2 (128 registers) the 256-scenario
     * ensemble steps 1.2 % faster */
    static constexpr int kBatchMinBlocks = 2;
    /* unrolled: 17 % faster than rolled with the class count exact */
    static constexpr bool kRollClasses = false;
    static constexpr int kWaveMinBlocks = 5;      /* 48 registers: four cells per thread without spills */
    static constexpr bool kKnownResults = false;
    /* sqrt on the SFU, x * rsqrt(x) (~3 ulp): the mixed form's ~25 square
     * roots per cell (wave speeds, gravity, settling, friction) cost a third
     * of the IEEE sequence; +0 for x <= 0 (the reference's pow(x, 0.5) of a
     * zero).  The product is rounded on its own (never fused into a later
     * add), so the single-domain and batched kernels compute the same value. */
    static __device__ __forceinline__ R sqrtp(R x) { return x > 0.f ? __fmul_rn(x, rsqrtf(x)) : 0.f; }
    /* x^y for x > 0 as x^n * 2^(f log2 x), n = floor(y), f = y - n in [0,1):
     * the integer power by multiplication (|n| <= 4), the fractional one on
     * the SFU.  The SFU's log2 error is then scaled by f < 1 instead of y, so
     * x^3.333 of a 10 um film errs ~1e-6 instead of ~1e-5 (about 12
     * instructions against ~50 for powf).  Other exponents use powf. */
    static __device__ __forceinline__ R pow(R x, R y)
    {
        if (y == 0.5f) return sqrtp(x);
        if (y == 1.f) return x;
        if (y == 2.f) return x * x;
        if (y == 4.f) { const float x2 = x * x; return x2 * x2; }
        const float n = floorf(y);
        if (x > 0.f && x < 3.0e38f && n >= -4.f && n <= 4.f) {
            const float f = y - n;
            float p = 1.f;
            const float b = n < 0.f ? __frcp_rn(x) : x;
            for (int k = 0; k < (int)fabsf(n); k++) p *= b;
            return f == 0.f ? p : p * exp2f(f * __log2f(x));
        }
        return powf(x, y);
    }
    static __device__ __forceinline__ R exp(R x) { return __expf(x); }
    static __device__ __forceinline__ R cos_atan(R x) { return rsqrtf(1.f + x * x); }
    static __device__ __forceinline__ R sin_atan(R x) { return x * rsqrtf(1.f + x * x); }
    static __device__ __forceinline__ R div(R a, R b) { return __fdividef(a, b); }
    static __device__ __forceinline__ R divz(R a, R b) { return div(a, b); }
    static __device__ __forceinline__ R sqrtz(R x) { return sqrtp(x); }
    static __device__ __forceinline__ R divk(R a, R c, R, int) { return div(a, c); }
    static __device__ __forceinline__ R e3_term(R num, R J, R yJ, int ok, R m) { return divk(num, J, yJ, ok) * m; }
    static __device__ __forceinline__ R e4_term(R A, R T, R F, R e, R m) { return div(div(A, T) * F, e) * m; }
    static __device__ __forceinline__ R qnan() { return __int_as_float(0x7fc00000); }
    /* settling velocity sqrt(A^2 + c) - A rewritten as c / (sqrt(A^2 + c) + A):
     * equal in exact arithmetic, but for fine classes (d = 2 um: A = 8.37,
     * c = 3e-5) the reference's difference cancels ~7 digits, all of FP32's */
    static __device__ __forceinline__ R settle(R A, R A2, R c) { return __fdividef(c, sqrtp(A2 + c) + A); }
    /* DEP is stored in FP32 here: a reciprocal multiply is exact enough */
    static __device__ __forceinline__ double dep_of(double M, const DevParams &P) { return M * P.inv_rhos; }
};

/* hllc of SWEHR.c:327-409 with the velocities already formed
 * (nl = normal/ul, tl = tangential/vl; both 0 for a dry side) and the left
 * side's sqrt(g hl) given.  Same operations as hllc(). */
template <class PP>
__device__ __forceinline__ typename PP::R hllc_v(typename PP::R hl, typename PP::R hr, typename PP::R nl,
                                                 typename PP::R nr, typename PP::R tl, typename PP::R tr,
                                                 typename PP::R g, typename PP::R cl, typename PP::R hfilm,
                                                 typename PP::R &T0, typename PP::R &T1, typename PP::R &T2)
{
    typedef typename PP::R R;
    const R half = R(0.5);
    const R cr = PP::sqrtp(g * hr);
    const R d = nl + 2 * cl - nr - 2 * cr;
    const R hs = PP::divz(d * d, 16 * g);
    const R us = half * (nl + nr) + cl - cr;
    const R cs = PP::sqrtz(g * hs);
    R sl = nl - cl;
    if (us - cs < sl) sl = us - cs;
    R sm = us;
    R sr = nr + cr;
    if (us + cs > sr) sr = us + cs;
    if (hl <= hfilm) { sl = nr - 2 * cr; sm = sl; sr = nr + cr; }
    if (hr <= hfilm) { sl = nl - cl; sr = nl + 2 * cl; sm = sr; }
    R f0 = PP::qnan(), f1 = f0;
    if (sl >= 0) {
        f0 = hl * nl;
        f1 = hl * nl * nl + half * g * hl * hl;
    }
    if (sl <= 0 && sr >= 0) {
        f0 = PP::divz(sr * (hl * nl) - sl * (hr * nr) + sl * sr * (hr - hl), sr - sl);
        f1 = PP::div(sr * (hl * nl * nl + half * g * hl * hl) - sl * (hr * nr * nr + half * g * hr * hr)
                         + sl * sr * (hr * nr - hl * nl),
                     sr - sl);
    }
    if (sr <= 0) {
        f0 = hr * nr;
        f1 = hr * nr * nr + half * g * hr * hr;
    }
    T0 = f0;
    T1 = f1;
    T2 = (sm >= 0) ? f0 * tl : f0 * tr;
    R s = 0;
    if (fabs(sl) > s) s = fabs(sl);
    if (fabs(sr) > s) s = fabs(sr);
    if (fabs(sm) > s) s = fabs(sm);
    return s;
}

/* The normal velocity of a state mirrored across a solid face: the
 * reference negates the momentum and divides, (-hu)/h, when the side is wet
 * (exactly -(hu/h), a zero included) and takes +0 when it is dry
 * (SWEHR.c:333-352 on the arguments of SWEHR.c:1140,1145,1208,1213). */
template <class PP>
__device__ __forceinline__ typename PP::R mirror_v(typename PP::R vel, typename PP::R h, typename PP::R hfilm)
{
    return h > hfilm ? -vel : typename PP::R(0);
}

/* wave speed only (the same sl, sr, sm as hllc_v) */
template <class PP>
__device__ __forceinline__ typename PP::R hll_speed(typename PP::R hl, typename PP::R hr, typename PP::R nl,
                                                    typename PP::R nr, typename PP::R g, typename PP::R cl,
                                                    typename PP::R hfilm)
{
    typedef typename PP::R R;
    const R cr = PP::sqrtp(g * hr);
    const R d = nl + 2 * cl - nr - 2 * cr;
    const R hs = PP::divz(d * d, 16 * g);
    const R us = R(0.5) * (nl + nr) + cl - cr;
    const R cs = PP::sqrtz(g * hs);
    R sl = nl - cl;
    if (us - cs < sl) sl = us - cs;
    R sm = us;
    R sr = nr + cr;
    if (us + cs > sr) sr = us + cs;
    if (hl <= hfilm) { sl = nr - 2 * cr; sm = sl; sr = nr + cr; }
    if (hr <= hfilm) { sl = nl - cl; sr = nl + 2 * cl; sm = sr; }
    R s = 0;
    if (fabs(sl) > s) s = fabs(sl);
    if (fabs(sr) > s) s = fabs(sr);
    if (fabs(sm) > s) s = fabs(sm);
    return s;
}

struct TileCoord {
    int i0, j0;
};

/* tiles cover the rows the context updates (own_lo..own_hi) */
__device__ __forceinline__ TileCoord tile_coord(const DevParams &P, int64_t tile)
{
    const int ntj = (P.ny + T_J - 1) / T_J;
    TileCoord t;
    t.i0 = (int)(tile / ntj) * T_I + P.own_lo;
    t.j0 = (int)(tile % ntj) * T_J + 1;
    return t;
}

/* -------------------------------------------------------------- staging ---
 * Every global load of a tile is issued up front as an asynchronous copy
 * (cp.async of 16 bytes, or one tensor-map box per plane) into shared memory,
 * so the arithmetic never waits on HBM and other CTAs on the SM compute while
 * this one's copies fly.
 *   halo planes  h hu hv totsed dep U_1..U_S   10 rows x (32 + 2 pad) columns
 *   cell planes  totm maxvel maxdep [ks] (RS), vinf M_1..M_S (double)   8 x 32
 *   topography   z_prev 12 x 36, z 10 x 36 (double)
 * A staged row of a plane of T starts pad = 16 / sizeof(T) columns left of
 * the tile: row r is grid row i0-1+r, column c is grid column (0-based)
 * j0-1-pad+c, so every staged row starts 16-byte aligned in HBM and halo
 * cell (hi, hj) sits at (hi, hj+pad-1).  (Counts above are for the 8 x 32
 * tile.)  Rows or columns outside the grid are not loaded: ghosts are
 * resolved from their source cells afterwards (SWEHR.c:816-1035). */
template <class T>
struct Cols {
    static constexpr int pad = 16 / (int)sizeof(T);   /* staged columns left of the tile */
    static constexpr int rj = T_J + 2 * pad;          /* staged columns per row */
};
#define R_J (T_J + 4)       /* staged columns of the (double) topography windows */
#define HALO_ROWS H_I
#define ZP_ROWS (T_I + 4)
#define ZC_ROWS (T_I + 2)

static_assert((size_t)(TILE_THREADS / 32) * B_NTERMS * sizeof(double) <= 4 * N_H * sizeof(float),
              "budget reduction fits in the face-state arrays it reuses");

struct StagedLayout {
    /* byte offsets from the start of dynamic shared memory */
    size_t halo, cell_r, cell_d, zp, zc, u, v, g, c, sed, fx, fy, up, red, total;
    int nhalo, ncellr, ncelld;
    int hps;              /* elements from one halo plane to the next (rows x staged columns, rounded to 128 bytes) */
    int stage_m;          /* M_k staged here (else read from global memory by the cell stage) */
    /* stage_m: staging M_k costs 2 KB of shared memory per class; the
     * launcher picks the kernel that stages it only where that costs no
     * resident blocks (a compile-time choice of each kernel) */
    __host__ __device__ static StagedLayout make(int S, size_t rs, int stage_m = 1)
    {
        StagedLayout L;
        size_t o = 0;
        /* every region starts 128-byte aligned (a tile copy's destination) */
        auto take = [&](size_t bytes) { size_t at = o; o += (bytes + 127) / 128 * 128; return at; };
        const size_t rj = (size_t)T_J + 2 * (16 / rs);
        L.hps = (int)(((size_t)HALO_ROWS * rj * rs + 127) / 128 * 128 / rs);
        L.stage_m = stage_m;
        L.nhalo = 5 + S;
        L.ncellr = 4;
        L.ncelld = L.stage_m ? 1 + S : 1;
        L.halo = take((size_t)L.nhalo * L.hps * rs);
        L.cell_r = take((size_t)L.ncellr * T_I * T_J * rs);
        L.cell_d = take((size_t)L.ncelld * T_I * T_J * sizeof(double));
        L.zp = take((size_t)ZP_ROWS * R_J * sizeof(double));
        L.zc = take((size_t)ZC_ROWS * R_J * sizeof(double));
        L.u = take((size_t)N_H * rs);
        L.v = take((size_t)N_H * rs);
        L.g = take((size_t)N_H * rs);
        L.c = take((size_t)N_H * rs);
        L.sed = take((size_t)S * N_H * rs);
        L.fx = take((size_t)3 * N_FX * rs);
        L.fy = take((size_t)3 * N_FY * rs);
        L.up = take((size_t)(N_FX + N_FY));
        /* the budget reduction runs after a tile's cells are done, when the
         * face states u, v, g, c are dead: it reuses their space */
        L.red = L.u;
        L.total = o;
        return L;
    }
};

/* halo planes, in staging order */
enum { HP_H = 0, HP_HU, HP_HV, HP_TS, HP_DEP, HP_U };
/* cell planes: RS then double */
enum { CR_TOTM = 0, CR_MAXVEL, CR_MAXDEP, CR_KS };
enum { CD_VINF = 0, CD_M };

template <class RS>
__device__ __forceinline__ const RS *halo_plane_src(const SetV<RS> &s, int p, int64_t pl)
{
    switch (p) {
    case HP_H: return s.h;
    case HP_HU: return s.hu;
    case HP_HV: return s.hv;
    case HP_TS: return s.totsed;
    case HP_DEP: return s.dep;
    default: return s.U + (int64_t)(p - HP_U) * pl;
    }
}

/* pair copy global -> shared: 2 elements of T (8 or 16 bytes) */
template <class T>
__device__ __forceinline__ void cp_pair(void *dst, const T *src)
{
    __pipeline_memcpy_async(dst, src, 2 * sizeof(T));
}

/* 16-byte copy global -> shared (both addresses 16-byte aligned) */
__device__ __forceinline__ void cp16(void *dst, const void *src) { __pipeline_memcpy_async(dst, src, 16); }

/* Issue the tile's asynchronous copies (halo planes, z_prev and z windows,
 * cell planes).  Each thread owns fixed (row, vector) slots and walks the
 * planes with a pointer step, so the per-copy cost is one add.  Halo rows
 * and topography windows move 16 bytes per copy (2 doubles or 4 floats). */
template <class RS, int NS = 0>
__device__ __forceinline__ void stage_load(const DevParams &P, const SetV<RS> &src, const double *__restrict__ zp,
                                           const double *__restrict__ zc, const RS *__restrict__ ks, TileCoord tc,
                                           unsigned char *smb, const StagedLayout &L)
{
    const int64_t pl = P.plane;
    const int S = NS ? NS : P.S;
    constexpr int VEC = Cols<RS>::pad;                         /* elements per 16-byte copy */
    constexpr int RJ = Cols<RS>::rj, NV = RJ / VEC;            /* copies per halo row: 18 (double), 10 (float) */
    const int c0 = tc.j0 - 1 - Cols<RS>::pad;                  /* 0-based grid column of staged column 0 */
    const int tid = threadIdx.x;
    static_assert(HALO_ROWS * NV <= TILE_THREADS, "one halo slot per thread");
    /* halo planes: 10 rows x NV vectors */
    if (tid < HALO_ROWS * NV) {
        const int r = tid / NV, kv = tid - r * NV;
        const int gi = tc.i0 - 1 + r, col = c0 + VEC * kv;
        /* columns past ny are row padding no cell reads (a ghost column
         * takes its source cell's values): not loaded; a vector starting
         * before ny ends inside the row (pitch is a multiple of 32) */
        if (gi >= 1 && gi <= P.nx && col >= 0 && col < P.ny) {
            const int64_t go = (int64_t)(gi - 1) * P.pitch + col;
            RS *d = reinterpret_cast<RS *>(smb + L.halo) + r * RJ + VEC * kv;
            const int ps = L.hps;
            cp16(d + HP_H * ps, src.h + go);
            cp16(d + HP_HU * ps, src.hu + go);
            cp16(d + HP_HV * ps, src.hv + go);
            cp16(d + HP_TS * ps, src.totsed + go);
            cp16(d + HP_DEP * ps, src.dep + go);
            const RS *u = src.U + go;
            for (int k = 0; k < S; k++) cp16(d + (HP_U + k) * ps, u + (int64_t)k * pl);
        }
    }
    /* topography: z_prev 12 rows, z 10 rows, 18 pairs each */
    {
        constexpr int NHS = HALO_ROWS * NV;
        const int slot = tid < NHS ? tid + (TILE_THREADS - NHS) : tid - NHS;
        const int nzs = (ZP_ROWS + ZC_ROWS) * (R_J / 2);                   /* 396 */
        for (int s = slot; s < nzs; s += TILE_THREADS) {
            const bool isp = s < ZP_ROWS * (R_J / 2);
            const int s2 = isp ? s : s - ZP_ROWS * (R_J / 2);
            const int r = s2 / (R_J / 2), k2 = s2 - r * (R_J / 2);
            const int gi = (isp ? tc.i0 - 2 : tc.i0 - 1) + r, col = tc.j0 - 3 + 2 * k2;   /* double windows: pad 2 */
            if (gi < 1 || gi > P.nx || col < 0 || col >= P.ny) continue;
            double *d = reinterpret_cast<double *>(smb + (isp ? L.zp : L.zc)) + r * R_J + 2 * k2;
            cp16(d, (isp ? zp : zc) + (int64_t)(gi - 1) * P.pitch + col);
        }
    }
    /* cell planes: 8 rows x 16 pairs = 128 slots; threads 128..255 */
    if (tid >= TILE_THREADS - T_I * (T_J / 2)) {
        const int s = tid - (TILE_THREADS - T_I * (T_J / 2));
        const int r = s / (T_J / 2), k2 = s - r * (T_J / 2);
        const int gi = tc.i0 + r, col = tc.j0 - 1 + 2 * k2;
        if (gi <= P.nx && col < P.ny) {
            const int64_t go = (int64_t)(gi - 1) * P.pitch + col;
            RS *cr = reinterpret_cast<RS *>(smb + L.cell_r) + r * T_J + 2 * k2;
            double *cd = reinterpret_cast<double *>(smb + L.cell_d) + r * T_J + 2 * k2;
            const int ps = T_I * T_J;
            cp_pair(cr + CR_TOTM * ps, src.totm + go);
            cp_pair(cr + CR_MAXVEL * ps, src.maxvel + go);
            cp_pair(cr + CR_MAXDEP * ps, src.maxdep + go);
            if (P.has_ks) cp_pair(cr + CR_KS * ps, ks + go);
            cp_pair(cd + CD_VINF * ps, src.vinf + go);
            if (L.stage_m) {
                const double *m = src.M + go;
                for (int k = 0; k < S; k++) cp_pair(cd + (CD_M + k) * ps, m + (int64_t)k * pl);
            }
        }
    }
    __pipeline_commit();
}

/* Plane numbers of a state set in its tensor maps: the plain form's set
 * is one FP64 block (swehr_device.cuh), the mixed form's an FP32 block
 * (h hu hv maxvel maxdep totm dep totsed gz U_1..U_S) followed by an FP64
 * block (vinf M_1..M_S).  `d_*` index the set's FP64 planes. */
template <class RS>
struct SetPlanes;
template <>
struct SetPlanes<double> {
    enum { h = P_H, hu = P_HU, hv = P_HV, maxvel = P_MAXVEL, maxdep = P_MAXDEP, totm = P_TOTM, dep = P_DEP,
           totsed = P_TOTSED, U = P_FIXED, d_vinf = P_VINF };
    static __device__ __forceinline__ int d_M(int S) { return P_FIXED + S; }
};
template <>
struct SetPlanes<float> {
    enum { h = 0, hu = 1, hv = 2, maxvel = 3, maxdep = 4, totm = 5, dep = 6, totsed = 7, U = 9, d_vinf = 0 };
    static __device__ __forceinline__ int d_M(int) { return 1; }
};

/* The same staging as stage_load as tensor-map box copies (planes of one
 * domain), issued by one thread onto the tile's mbarrier: halo boxes of
 * Cols<RS>::rj columns x halo rows at column j0-1-pad, row i0-2 (0-based),
 * the z_prev window one row higher and taller (doubles, column j0-3), cell
 * boxes T_J x T_I at (j0-1, i0-1).  j0-1 is a multiple of T_J and pad is 16
 * bytes of the plane's type, so every box starts on a 16-byte column
 * boundary; rows or columns outside the grid arrive as zeros. */
template <class RS>
__device__ __forceinline__ void stage_load_tma(const DevParams &P, const TmaMaps &tm, int set, int64_t n,
                                               TileCoord tc, unsigned char *smb, const StagedLayout &L,
                                               uint64_t *bar)
{
    typedef SetPlanes<RS> SP;
    const uint32_t hb = (uint32_t)(HALO_ROWS * Cols<RS>::rj * sizeof(RS));
    const uint32_t cbr = (uint32_t)(T_I * T_J * sizeof(RS)), cbd = (uint32_t)(T_I * T_J * sizeof(double));
    const uint32_t bytes = (uint32_t)(5 + P.S) * hb + (uint32_t)((ZP_ROWS + ZC_ROWS) * R_J * sizeof(double)) +
                           (3u + (P.has_ks ? 1u : 0u)) * cbr + (1u + (L.stage_m ? (uint32_t)P.S : 0u)) * cbd;
    mbar_expect_tx(bar, bytes);
    const CUtensorMap *mh = &tm.m[TM_HALO0 + set], *mc = &tm.m[TM_CELL0 + set], *md = &tm.m[TM_CELLD0 + set];
    const int hx = tc.j0 - 1 - Cols<RS>::pad, hy = tc.i0 - 2, zx = tc.j0 - 3, cx = tc.j0 - 1, cy = tc.i0 - 1;
    RS *halo = reinterpret_cast<RS *>(smb + L.halo);
    tma_load_3d(halo + HP_H * L.hps, mh, bar, hx, hy, SP::h);
    tma_load_3d(halo + HP_HU * L.hps, mh, bar, hx, hy, SP::hu);
    tma_load_3d(halo + HP_HV * L.hps, mh, bar, hx, hy, SP::hv);
    tma_load_3d(halo + HP_TS * L.hps, mh, bar, hx, hy, SP::totsed);
    tma_load_3d(halo + HP_DEP * L.hps, mh, bar, hx, hy, SP::dep);
    for (int k = 0; k < P.S; k++) tma_load_3d(halo + (HP_U + k) * L.hps, mh, bar, hx, hy, SP::U + k);
    tma_load_3d(smb + L.zp, &tm.m[TM_ZP], bar, zx, tc.i0 - 3, (int)((n + 2) % 3));
    tma_load_3d(smb + L.zc, &tm.m[TM_ZC], bar, zx, hy, (int)(n % 3));
    RS *cr = reinterpret_cast<RS *>(smb + L.cell_r);
    double *cd = reinterpret_cast<double *>(smb + L.cell_d);
    const int ps = T_I * T_J;
    tma_load_3d(cr + CR_TOTM * ps, mc, bar, cx, cy, SP::totm);
    tma_load_3d(cr + CR_MAXVEL * ps, mc, bar, cx, cy, SP::maxvel);
    tma_load_3d(cr + CR_MAXDEP * ps, mc, bar, cx, cy, SP::maxdep);
    if (P.has_ks) tma_load_3d(cr + CR_KS * ps, &tm.m[TM_KS], bar, cx, cy, 0);
    tma_load_3d(cd + CD_VINF * ps, md, bar, cx, cy, SP::d_vinf);
    if (L.stage_m)
        for (int k = 0; k < P.S; k++) tma_load_3d(cd + (CD_M + k) * ps, md, bar, cx, cy, SP::d_M(P.S) + k);
}

/* slopes from a staged topography tile, same operations as slope_x/slope_y
 * (SWEHR.c:1240-1277); (r, c) is the staged position of grid cell (i, j) */
__device__ __forceinline__ double sslope_x(const DevParams &P, const double *zs, int r, int c, int i)
{
    if (i != 1 && i != P.nx) return P.half_odx * (zs[(r + 1) * R_J + c] - zs[(r - 1) * R_J + c]);
    if (i == P.nx) return P.oneoverdx * (zs[r * R_J + c] - zs[(r - 1) * R_J + c]);
    return P.oneoverdx * (zs[(r + 1) * R_J + c] - zs[r * R_J + c]);
}

__device__ __forceinline__ double sslope_y(const DevParams &P, const double *zs, int r, int c, int j)
{
    if (j != 1 && j != P.ny) return P.half_odx * (zs[r * R_J + c + 1] - zs[r * R_J + c - 1]);
    if (j == P.ny) return P.oneoverdx * (zs[r * R_J + c] - zs[r * R_J + c - 1]);
    return P.oneoverdx * (zs[r * R_J + c + 1] - zs[r * R_J + c]);
}

/* Derived halo values from the staged planes: h, u = hu/h, v = hv/h (0 when
 * dry), GZ of the previous step and sqrt(GZ h) for left/lower face cells,
 * SED_k.  Ghost cells read their source cell (SWEHR.c:816-1035). */
template <class PP, class RS, int NS = 0>
__device__ __forceinline__ void stage_derive(const DevParams &P, const SetV<RS> &src, TileCoord tc, unsigned char *smb,
                                             const StagedLayout &L, typename PP::R inh, typename PP::R inhv,
                                             typename PP::R insed)
{
    typedef typename PP::R R;
    const int S = NS ? NS : P.S;
    const RealC<R> &K = kc<R>(P);
    const RS *halo = reinterpret_cast<const RS *>(smb + L.halo);
    const double *zps = reinterpret_cast<const double *>(smb + L.zp);
    R *su = reinterpret_cast<R *>(smb + L.u), *sv = reinterpret_cast<R *>(smb + L.v);
    R *sg = reinterpret_cast<R *>(smb + L.g), *sc = reinterpret_cast<R *>(smb + L.c);
    R *ssed = reinterpret_cast<R *>(smb + L.sed);
    for (int idx = threadIdx.x; idx < N_H; idx += TILE_THREADS) {
        const int hi = idx / H_J, hj = idx - hi * H_J;
        const int gi = tc.i0 - 1 + hi, gj = tc.j0 - 1 + hj;
        const bool hcorner = (hi == 0 || hi == H_I - 1) && (hj == 0 || hj == H_J - 1);
        const bool gx = gi == 0 || gi == P.nx + 1, gy = gj == 0 || gj == P.ny + 1;
        if (hcorner || gi > P.nx + 1 || gj > P.ny + 1 || (gx && gy)) continue;
        const int si = gi < 1 ? 1 : (gi > P.nx ? P.nx : gi);
        const int sj = gj < 1 ? 1 : (gj > P.ny ? P.ny : gj);
        /* staged position of the source in the RS planes, and its column in the topography windows */
        const int sr = si - (tc.i0 - 1), scol = sj - tc.j0 + Cols<RS>::pad, zcol = sj - tc.j0 + 2;
        const int so = sr * Cols<RS>::rj + scol;
        const bool inflow = gj == P.ny + 1 && P.inflow;
        R h, hu, hv;
        if (inflow) {
            h = inh; hu = 0; hv = inhv;
        } else {
            h = (R)halo[HP_H * L.hps + so];
            hu = (R)halo[HP_HU * L.hps + so];
            hv = (R)halo[HP_HV * L.hps + so];
            if ((gi == 0 && P.bndry[0] == 1) || (gi == P.nx + 1 && P.bndry[2] == 1)) hu = -hu;
            if ((gj == 0 && P.bndry[1] == 1) || (gj == P.ny + 1 && P.bndry[3] == 1)) hv = -hv;
        }
        R u = 0, v = 0;
        if (h > K.hfilm) { u = PP::div(hu, h); v = PP::div(hv, h); }
        if (gx || gy) {
            /* ghost cells are never read through the staged planes: keep h there */
            reinterpret_cast<RS *>(smb + L.halo)[HP_H * L.hps + hi * Cols<RS>::rj + hj + Cols<RS>::pad - 1] = (RS)h;
        }
        su[idx] = u;
        sv[idx] = v;
        if (hi <= T_I && hj <= T_J) {
            R g;
            if (P.has_solid) {
                /* the state's GZ plane: the previous step's GZ of a flow cell,
                 * the set-up GZ a solid cell keeps (SWEHR.c:1233) */
                g = (R)src.gz[cidx(P, si, sj)];
            } else {
                /* GZ of the previous step at the source cell, SWEHR.c:1279 via z_prev */
                const int zr = si - (tc.i0 - 2);
                const R sx = (R)sslope_x(P, zps, zr, zcol, si), sy = (R)sslope_y(P, zps, zr, zcol, sj);
                g = PP::div(K.g, PP::sqrtp(sx * sx + sy * sy + 1));
            }
            sg[idx] = g;
            sc[idx] = PP::sqrtp(g * h);
        }
        auto sed_k = [&](int k) {
            R s = 0;
            if (inflow) s = insed;
            else if (h > K.hfilm) {
                s = PP::div((R)halo[(HP_U + k) * L.hps + so], h);
                if (s < R(-1e-5)) s = 0;
            }
            ssed[k * N_H + idx] = s;
        };
        if (PP::kRollClasses) {          /* one division sequence in the code, not four */
#pragma unroll 1
            for (int k = 0; k < S; k++) sed_k(k);
        } else {
#pragma unroll
            for (int k = 0; k < S; k++) sed_k(k);
        }
    }
}

/* halo-cell depth as staged (ghosts filled by stage_derive) */
template <class RS>
__device__ __forceinline__ const RS *staged_h(const unsigned char *smb, const StagedLayout &L)
{
    return reinterpret_cast<const RS *>(smb + L.halo) + HP_H * L.hps;
}

/* ------------------------------------------------------------------ wave */
/* Largest wave speed over the faces cell (i, j) owns: i+1/2 and j+1/2, plus
 * the domain's faces 1/2 when i == 1 or j == 1, so every face of
 * SWEHR.c:1092-1230's Smax is taken once.  The cell's velocities, its GZ of
 * the previous step and sqrt(GZ h) are formed once and serve as the left
 * state of its faces; of the right cells only depth and normal velocity are
 * needed.  Ghost cells follow the reference's boundary copies
 * (SWEHR.c:816-1035): the source cell's state with the normal momentum
 * negated at a wall, the hard-wired inflow at j = ny+1.  Reads global memory
 * directly (no staging, no barrier): the pass is light, and a max does not
 * depend on the order the faces are visited in. */
/* GZ of cell (i, j) from a topography plane, SWEHR.c:1279 (the wave pass's
 * lagged GZ, computed one step ahead by the update and at initialisation) */
template <class PP>
__device__ __forceinline__ typename PP::R lagged_gz(const DevParams &P, const double *__restrict__ z, int i, int j)
{
    typedef typename PP::R R;
    const RealC<R> &K = kc<R>(P);
    const R sx = (R)slope_x(P, z, i, j), sy = (R)slope_y(P, z, i, j);
    return PP::div(K.g, PP::sqrtp(sx * sx + sy * sy + 1));
}

/* wave_cell with the cell's lagged GZ given (g).  solid: the interior
 * solid mask, or nullptr; a face between a solid and a flow cell takes the
 * flow cell's state mirrored across it (SWEHR.c:1137-1146 for i+1/2 with
 * 1 <= i < nx, 1205-1214 for j+1/2, the latter reading the mask one column
 * past the row at j = ny, see solid_at), with the GZ of the face's left
 * (lower) cell as every face does. */
template <class PP, class RS>
__device__ __forceinline__ typename PP::R wave_cell_g(const DevParams &P, const SetV<RS> &src, int i, int j,
                                                      typename PP::R inh, typename PP::R inhv, typename PP::R g,
                                                      const uint8_t *__restrict__ solid = nullptr)
{
    typedef typename PP::R R;
    const RealC<R> &K = kc<R>(P);
    const int64_t q = cidx(P, i, j);
    const R h = (R)src.h[q], hu = (R)src.hu[q], hv = (R)src.hv[q];
    R u = 0, v = 0;
    if (h > K.hfilm) {
        u = PP::div(hu, h);
        v = PP::div(hv, h);
    }
    const R c = PP::sqrtp(g * h);
    const bool here_solid = solid && solid_at(P, solid, i, j);
    R smax = 0, s;
    /* x face i+1/2 */
    if (i < P.nx) {
        const int64_t qr = q + P.pitch;
        const R hr = (R)src.h[qr];
        const R ur = hr > K.hfilm ? PP::div((R)src.hu[qr], hr) : R(0);
        const bool right_solid = solid && solid_at(P, solid, i + 1, j);
        if (here_solid && !right_solid)
            s = hll_speed<PP>(hr, hr, mirror_v<PP>(ur, hr, K.hfilm), ur, g, PP::sqrtp(g * hr), K.hfilm);
        else if (!here_solid && right_solid) s = hll_speed<PP>(h, h, u, mirror_v<PP>(u, h, K.hfilm), g, c, K.hfilm);
        else s = hll_speed<PP>(h, hr, u, ur, g, c, K.hfilm);
    } else {
        s = hll_speed<PP>(h, h, u, P.bndry[2] == 1 ? -u : u, g, c, K.hfilm);
    }
    smax = (s > smax) ? s : smax;
    /* y face j+1/2: the right state is cell (i, j+1), or at j = ny the ghost
     * (the inflow ramp, or this cell with its normal velocity negated at a wall) */
    {
        R hr, vr;
        if (j < P.ny) {
            const int64_t qr = q + 1;
            hr = (R)src.h[qr];
            vr = hr > K.hfilm ? PP::div((R)src.hv[qr], hr) : R(0);
        } else if (P.inflow) {
            hr = (R)(RS)inh;                     /* the ghost's depth as the tile pass staged it */
            vr = inh > K.hfilm ? PP::div(inhv, inh) : R(0);
        } else {
            hr = h;
            vr = P.bndry[3] == 1 ? -v : v;
        }
        const bool right_solid = solid && solid_at(P, solid, i, j + 1);
        if (here_solid && !right_solid)
            s = hll_speed<PP>(hr, hr, mirror_v<PP>(vr, hr, K.hfilm), vr, g, PP::sqrtp(g * hr), K.hfilm);
        else if (!here_solid && right_solid) s = hll_speed<PP>(h, h, v, mirror_v<PP>(v, h, K.hfilm), g, c, K.hfilm);
        else s = hll_speed<PP>(h, hr, v, vr, g, c, K.hfilm);
    }
    smax = (s > smax) ? s : smax;
    /* the domain's faces 1/2: ghost on the left, this cell on the right */
    if (i == 1) {
        s = hll_speed<PP>(h, h, P.bndry[0] == 1 ? -u : u, u, g, c, K.hfilm);
        smax = (s > smax) ? s : smax;
    }
    if (j == 1) {
        s = hll_speed<PP>(h, h, P.bndry[1] == 1 ? -v : v, v, g, c, K.hfilm);
        smax = (s > smax) ? s : smax;
    }
    return smax;
}

template <class PP, class RS>
__device__ __forceinline__ typename PP::R wave_cell(const DevParams &P, const SetV<RS> &src, int i, int j,
                                                    typename PP::R inh, typename PP::R inhv,
                                                    const uint8_t *__restrict__ solid)
{
    /* GZ of the previous step, written by its update */
    return wave_cell_g<PP, RS>(P, src, i, j, inh, inhv, (typename PP::R)src.gz[cidx(P, i, j)], solid);
}

/* V = 16 / sizeof(RS) consecutive elements of a plane with one 16-byte
 * load (p is 16-byte aligned: the vector starts on a column multiple of V
 * of a row whose pitch is a multiple of 32), converted to R */
template <class RS, class R>
__device__ __forceinline__ void load_vec(const RS *__restrict__ p, R *out)
{
    if constexpr (sizeof(RS) == 4) {
        const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
        out[0] = (R)a.x; out[1] = (R)a.y; out[2] = (R)a.z; out[3] = (R)a.w;
    } else {
        const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
        out[0] = (R)a.x; out[1] = (R)a.y;
    }
}

/* Largest wave speed over the faces of V consecutive cells (i, j0..j0+V-1)
 * of a row, j0-1 a multiple of V: the same faces and the same operations as
 * wave_cell_g for each cell (no interior solid cells), with every plane read
 * V cells per load.  A cell's normal velocity towards its right neighbour in
 * the vector is that neighbour's own velocity, formed once. */
template <class PP, class RS>
__device__ __forceinline__ typename PP::R wave_vec(const DevParams &P, const SetV<RS> &src, int i, int j0,
                                                   typename PP::R inh, typename PP::R inhv)
{
    typedef typename PP::R R;
    constexpr int V = Cols<RS>::pad;
    const RealC<R> &K = kc<R>(P);
    const int64_t q = cidx(P, i, j0);
    R h[V], hu[V], hv[V], g[V], u[V], v[V], hd[V], hud[V];
    load_vec<RS, R>(src.h + q, h);
    load_vec<RS, R>(src.hu + q, hu);
    load_vec<RS, R>(src.hv + q, hv);
    load_vec<RS, R>(src.gz + q, g);
    const bool below = i < P.nx;
    if (below) {
        load_vec<RS, R>(src.h + q + P.pitch, hd);
        load_vec<RS, R>(src.hu + q + P.pitch, hud);
    }
    /* the cell after the vector, for the last cell's y face */
    const int jl = j0 + V;
    R hn = 0, hvn = 0;
    if (jl <= P.ny) {
        hn = (R)src.h[q + V];
        hvn = (R)src.hv[q + V];
    }
#pragma unroll
    for (int k = 0; k < V; k++) {
        u[k] = 0;
        v[k] = 0;
        if (h[k] > K.hfilm) {
            u[k] = PP::div(hu[k], h[k]);
            v[k] = PP::div(hv[k], h[k]);
        }
    }
    R smax = 0, s;
#pragma unroll
    for (int k = 0; k < V; k++) {
        const int j = j0 + k;
        if (j > P.ny) break;
        const R c = PP::sqrtp(g[k] * h[k]);
        /* x face i+1/2 */
        if (below) {
            const R ur = hd[k] > K.hfilm ? PP::div(hud[k], hd[k]) : R(0);
            s = hll_speed<PP>(h[k], hd[k], u[k], ur, g[k], c, K.hfilm);
        } else {
            s = hll_speed<PP>(h[k], h[k], u[k], P.bndry[2] == 1 ? -u[k] : u[k], g[k], c, K.hfilm);
        }
        smax = (s > smax) ? s : smax;
        /* y face j+1/2 */
        R hr, vr;
        if (j < P.ny) {
            if (k + 1 < V) {
                hr = h[k + 1];
                vr = v[k + 1];
            } else {
                hr = hn;
                vr = hn > K.hfilm ? PP::div(hvn, hn) : R(0);
            }
        } else if (P.inflow) {
            hr = (R)(RS)inh;
            vr = inh > K.hfilm ? PP::div(inhv, inh) : R(0);
        } else {
            hr = h[k];
            vr = P.bndry[3] == 1 ? -v[k] : v[k];
        }
        s = hll_speed<PP>(h[k], hr, v[k], vr, g[k], c, K.hfilm);
        smax = (s > smax) ? s : smax;
        /* the domain's faces 1/2 */
        if (i == 1) {
            s = hll_speed<PP>(h[k], h[k], P.bndry[0] == 1 ? -u[k] : u[k], u[k], g[k], c, K.hfilm);
            smax = (s > smax) ? s : smax;
        }
        if (j == 1) {
            s = hll_speed<PP>(h[k], h[k], P.bndry[1] == 1 ? -v[k] : v[k], v[k], g[k], c, K.hfilm);
            smax = (s > smax) ? s : smax;
        }
    }
    return smax;
}

/* block maximum of the threads' partial maxima (result valid in thread 0) */
__device__ __forceinline__ double block_max(double v, double *red8)
{
    v = warp_max(v);
    if ((threadIdx.x & 31) == 0) red8[threadIdx.x >> 5] = v;
    __syncthreads();
    double m = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < TILE_THREADS / 32; w++) m = (red8[w] > m) ? red8[w] : m;
    __syncthreads();
    return m;
}

/* CFL time step once every face of the step is in (SWEHR.c:1409-1413); one thread */
__device__ __forceinline__ void wave_finalize(const DevParams &P, Ctl *ctl)
{
    __threadfence();
    const double t = ctl->t;
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

template <class PP, class RS>
__global__ void __launch_bounds__(TILE_THREADS, PP::kWaveMinBlocks) k_wave_cells(const DevParams P, const BufsT<RS> B, Ctl *ctl)
{
    typedef typename PP::R R;
    if (!ctl->active) return;
    __shared__ double red8[TILE_THREADS / 32];
    __shared__ bool last;
    const int64_t n = ctl->step;
    const double t = ctl->t;
    const SetV<RS> src = B.set[n & 1];
    double inh = 0, inhv = 0, insed = 0;
    if (P.inflow) inflow_ghost(t, inh, inhv, insed);
    /* cells in i-major order, j contiguous; (i, j) advanced by the stride */
    /* the cells of the rows this context updates; a face belongs to the
     * row of its lower (left) cell, face 1/2 to row 1 */
    R smax = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t c0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (!P.has_solid) {
        /* V cells per thread and 16-byte loads (the pass is bound by load latency) */
        constexpr int V = Cols<RS>::pad;
        const int nv = (P.ny + V - 1) / V;
        const int64_t total = (int64_t)(P.own_hi - P.own_lo + 1) * nv;
        for (int64_t c = c0; c < total; c += stride) {
            const int r = (int)(c / nv);
            const int i = r + P.own_lo, j0 = (int)(c - (int64_t)r * nv) * V + 1;
            const R s = wave_vec<PP, RS>(P, src, i, j0, (R)inh, (R)inhv);
            smax = (s > smax) ? s : smax;
        }
    } else {
        const int64_t total = (int64_t)(P.own_hi - P.own_lo + 1) * P.ny;
        const int si = (int)(stride / P.ny), sj = (int)(stride - (int64_t)si * P.ny);
        int i = (int)(c0 / P.ny) + P.own_lo, j = (int)(c0 - (int64_t)(i - P.own_lo) * P.ny) + 1;
        for (int64_t c = c0; c < total; c += stride) {
            const R s = wave_cell<PP, RS>(P, src, i, j, (R)inh, (R)inhv, B.solid);
            smax = (s > smax) ? s : smax;
            i += si;
            j += sj;
            if (j > P.ny) { j -= P.ny; i++; }
        }
    }
    const double m = block_max((double)smax, red8);
    if (threadIdx.x == 0) {
        atomicMax(&ctl->smax_bits, (unsigned long long)__double_as_longlong(m));
        __threadfence();
        last = (atomicAdd(&ctl->wave_ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        if (P.slab)
            ctl->wave_ticket = 0u;       /* dt waits for the largest speed over every slab */
        else
            wave_finalize(P, ctl);
    }
}

/* the gz plane of the set step n reads, from its previous-step topography
 * (at creation, and after the topography is written) */
template <class PP, class RS>
__global__ void k_init_gz(const DevParams P, const BufsT<RS> B, int64_t n)
{
    const SetV<RS> st = B.set[n & 1];
    const double *zp = B.z[(n + 2) % 3];
    const int64_t total = (int64_t)P.nx * P.ny;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < total; c += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(c / P.ny) + 1, j = (int)(c - (int64_t)(i - 1) * P.ny) + 1;
        st.gz[cidx(P, i, j)] = (RS)lagged_gz<PP>(P, zp, i, j);
    }
}

/* ---------------------------------------------------------------- update */
template <int MAXS, bool BUDGET>
struct Acc2 {
    double rain, out, clamp, bulk, inf, round;
    double det[BUDGET ? MAXS : 1], sout[BUDGET ? MAXS : 1], sround[BUDGET ? MAXS : 1];
};

/* Parameters of the exact slope-failure test (passed by value: a pointer to
 * the kernel's parameter block would force a local copy of all of it). */
struct FailArgs {
    int32_t nx, ny, pitch, pad_;
    int64_t plane;
    double oneoverdx, half_odx, rho0, rhow, cohesion, fa;
    const uint8_t *solid;      /* interior solid mask or nullptr */
    const double *z0;          /* set-up topography: a solid neighbour's slopes */
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

/* Exact slope-failure test, SWEHR.c:1292-1312, in the form's arithmetic
 * (rarely needed: see the bound in tile_cell). */
template <class PP, class RS>
__device__ __noinline__ typename PP::R fail_exact(const FailArgs A, const RS *__restrict__ dep_plane,
                                                  const double *__restrict__ zp, const double *__restrict__ zc,
                                                  int i, int j, typename PP::R sx, typename PP::R sy,
                                                  typename PP::R gz, typename PP::R dep0, typename PP::R rho0c,
                                                  typename PP::R h0v)
{
    typedef typename PP::R R;
    const int iu = (i < A.nx) ? i + 1 : A.nx, id = (i > 1) ? i - 1 : 1;
    const int ju = (j < A.ny) ? j + 1 : A.ny, jd = (j > 1) ? j - 1 : 1;
    /* a solid neighbour never recomputed its slopes (SWEHR.c:1233): they are the set-up ones */
    auto zfor = [&](int ii, int jj, const double *z) {
        return (A.solid && A.solid[(int64_t)(ii - 1) * A.pitch + (jj - 1)]) ? A.z0 : z;
    };
    const R sxu = (iu == i) ? sx : (R)fa_slope_x(A, zfor(iu, j, zp), iu, j);
    const R sxd = (id == i) ? sx : (R)fa_slope_x(A, zfor(id, j, zc), id, j);
    const R syu = (ju == j) ? sy : (R)fa_slope_y(A, zfor(i, ju, zp), i, ju);
    const R syd = (jd == j) ? sy : (R)fa_slope_y(A, zfor(i, jd, zc), i, jd);
    const R rho0 = (R)A.rho0, half = R(0.5), odx = (R)A.oneoverdx;
    auto D = [&](int ii, int jj) { return (R)dep_plane[(int64_t)(ii - 1) * A.pitch + (jj - 1)]; };
    R fail = 0;
    R pgfx = dep0 * rho0 * gz * half * odx
             * (D(iu, j) * PP::cos_atan(fabs(sxu)) - D(id, j) * PP::cos_atan(fabs(sxd)));
    if (pgfx * sx > 0) pgfx = -1 * fabs(pgfx);
    if (pgfx * sx < 0) pgfx = fabs(pgfx);
    const R lhs = (rho0 * gz * dep0 + rho0c * gz * h0v) * PP::sin_atan(fabs(sy));
    const R nrm = (rho0 * gz * dep0 + rho0c * gz * h0v) * PP::cos_atan(fabs(sy)) - (R)A.rhow * gz * (dep0 + h0v);
    if (fail == 0 && (lhs > ((R)A.cohesion + nrm * (R)A.fa + pgfx))) fail = 1;
    R pgfy = dep0 * rho0 * gz * half * odx
             * (D(i, ju) * PP::cos_atan(fabs(syu)) - D(i, jd) * PP::cos_atan(fabs(syd)));
    if (pgfy * sy > 0) pgfy = -1 * fabs(pgfy);
    if (pgfy * sy < 0) pgfy = fabs(pgfy);
    if (fail == 0 && (lhs > ((R)A.cohesion + nrm * (R)A.fa + pgfy))) fail = 1;
    return fail;
}

/* moving storm in the form's arithmetic (positions in FP64) */
template <class PP>
__device__ __forceinline__ typename PP::R storm_r(const DevParams &P, double t, int i, int j)
{
    typedef typename PP::R R;
    const double x = ((double)(i + P.row0) - 0.5) * P.dx - (P.storm_x0 + P.storm_vx * t);
    const double y = ((double)j - 0.5) * P.dx - (P.storm_y0 + P.storm_vy * t);
    const double r2 = (x * x + y * y) / P.storm_r2;
    return (R)P.storm_peak * PP::exp(R(-0.5 * r2));
}

/* A solid cell in the update (SWEHR.c:1421 false branch, 1566-1574): no
 * water, momentum or suspended sediment; everything else -- deposit,
 * infiltration, topography, maxima, its GZ -- as it was.  What a written
 * state held there leaves the budget as outflow.  (Inlined: a call taking
 * the kernel's parameter block by reference would copy all of it to local
 * memory in every thread.) */
template <class PP, class RS, int MAXS, bool BUDGET>
__device__ __forceinline__ void solid_cell(const DevParams &P, const SetV<RS> &src, const SetV<RS> &dst,
                                        const double *__restrict__ zc, double *__restrict__ zn, int64_t q,
                                        Acc2<MAXS, BUDGET> &acc)
{
    const int64_t pl = P.plane;
    if (BUDGET) acc.out += (double)src.h[q];
    dst.h[q] = (RS)0;
    dst.hu[q] = (RS)0;
    dst.hv[q] = (RS)0;
    for (int k = 0; k < P.S; k++) {
        if (BUDGET && k < MAXS) acc.sout[k] += (double)src.U[k * pl + q];
        dst.U[k * pl + q] = (RS)0;
        dst.M[k * pl + q] = src.M[k * pl + q];
    }
    dst.vinf[q] = src.vinf[q];
    RS mv = src.maxvel[q], md = src.maxdep[q];
    if ((RS)0 > mv) mv = (RS)0;
    if ((RS)0 > md) md = (RS)0;
    dst.maxvel[q] = mv;
    dst.maxdep[q] = md;
    dst.totm[q] = src.totm[q];
    dst.dep[q] = src.dep[q];
    dst.totsed[q] = src.totsed[q];
    dst.gz[q] = src.gz[q];
    zn[q] = zc[q];
}

template <class PP, class RS, int MAXS, bool BUDGET, int NS = 0>
__device__ __forceinline__ void tile_cell(const DevParams &P, const SetV<RS> &src, const SetV<RS> &dst,
                                          const double *__restrict__ zp, const double *__restrict__ zc,
                                          double *__restrict__ zn, const unsigned char *smb, const StagedLayout &L,
                                          TileCoord tc, double t, double dt, double Rr, Acc2<MAXS, BUDGET> &acc,
                                          const uint8_t *__restrict__ solid, const double *__restrict__ z0)
{
    typedef typename PP::R R;
    const RealC<R> &K = kc<R>(P);
    const int ti = threadIdx.x / T_J, tj = threadIdx.x % T_J;
    const int i = tc.i0 + ti, j = tc.j0 + tj;
    if (i > P.own_hi || j > P.ny) return;
    const int64_t pl = P.plane;
    const int64_t q = cidx(P, i, j);
    if (P.has_solid && solid[q]) {
        solid_cell<PP, RS, MAXS, BUDGET>(P, src, dst, zc, zn, q, acc);
        return;
    }
    const int S = NS ? NS : P.S;
    const R hfilm = K.hfilm, rhos = K.rhos, rhow = K.rhow, one = 1, half = R(0.5);
    const int hs = (ti + 1) * H_J + (tj + 1);                      /* this cell in halo coords */
    constexpr int RJ = Cols<RS>::rj;
    const int so = (ti + 1) * RJ + (tj + Cols<RS>::pad);          /* ... and in the staged planes */
    const int cs = ti * T_J + tj;                                  /* ... and in the cell planes */
    const RS *halo = reinterpret_cast<const RS *>(smb + L.halo);
    const RS *cellr = reinterpret_cast<const RS *>(smb + L.cell_r);
    const double *celld = reinterpret_cast<const double *>(smb + L.cell_d);
    const RS *sTS = halo + HP_TS * L.hps, *sDEP = halo + HP_DEP * L.hps;
    const R h0v = (R)halo[HP_H * L.hps + so];
    const R hu0 = (R)halo[HP_HU * L.hps + so], hv0 = (R)halo[HP_HV * L.hps + so];
    const R totsed0 = (R)sTS[so], dep0 = (R)sDEP[so];
    const R totm0 = (R)cellr[CR_TOTM * T_I * T_J + cs];
    R rho0c = rhow * (1 - totsed0) + rhos * totsed0;
    if (rho0c > K.rhos08) rho0c = K.rhos08;
    const R Rc = P.storm ? storm_r<PP>(P, t, i, j) : (R)Rr;
    const R dtr = (R)dt;

    /* faces of this cell (computed in stage B) */
    const int fxl = ti * T_J + tj, fxr = (ti + 1) * T_J + tj;
    const int fyl = ti * (T_J + 1) + tj, fyr = fyl + 1;
    const R *FX = reinterpret_cast<const R *>(smb + L.fx), *FY = reinterpret_cast<const R *>(smb + L.fy);
    const unsigned char *up = smb + L.up;
    const R fxl0 = FX[3 * fxl], fxl1 = FX[3 * fxl + 1], fxl2 = FX[3 * fxl + 2];
    const R fxr0 = FX[3 * fxr], fxr1 = FX[3 * fxr + 1], fxr2 = FX[3 * fxr + 2];
    const R fyl0 = FY[3 * fyl], fyl1 = FY[3 * fyl + 1], fyl2 = FY[3 * fyl + 2];
    const R fyr0 = FY[3 * fyr], fyr1 = FY[3 * fyr + 1], fyr2 = FY[3 * fyr + 2];
    /* upwind cells of the sediment fluxes, halo index */
    const int uxl = up[fxl] ? hs : hs - H_J;
    const int uxr = up[fxr] ? hs + H_J : hs;
    const int uyl = up[N_FX + fyl] ? hs : hs - 1;
    const int uyr = up[N_FX + fyr] ? hs + 1 : hs;

    /* sources, SWEHR.c:1239-1320 */
    const R g = K.g;
    const double *zps = reinterpret_cast<const double *>(smb + L.zp), *zcs = reinterpret_cast<const double *>(smb + L.zc);
    const R sx = (R)sslope_x(P, zcs, ti + 1, tj + 2, i), sy = (R)sslope_y(P, zcs, ti + 1, tj + 2, j);
    const R syl = (R)sslope_y(P, zps, ti + 2, tj + 2, j);
    const R gx = PP::div(g * sx, PP::sqrtp(sx * sx + syl * syl + 1));
    const R SXf = -gx * h0v;
    const R gy = PP::div(g * sy, PP::sqrtp(sx * sx + sy * sy + 1));
    const R SYf = -gy * h0v;
    const R gz = PP::div(g, PP::sqrtp(sx * sx + sy * sy + 1));
    const R slope = PP::sqrtp(sx * sx + sy * sy);
    /* variable-density forcing (SWEHR.c:1283-1290).  Where the TOTSED
     * difference is an exact zero the term is a zero times a finite
     * quotient, and 0 - (+-0) = +0: the FP64 form keeps gamma = +0 without
     * the division sequence when the ranges keep the quotient finite. */
    R gammax = 0, gammay = 0;
    auto zero_gradient = [&](int a, int b) {
        return PP::kKnownResults && (R)sTS[a] - (R)sTS[b] == 0 && fabs((rhos - rho0c) * gz * h0v * h0v) <= R(0x1p800) &&
               2 * rho0c >= R(0x1p-100);
    };
    if (i > 1 && i < P.nx && !zero_gradient(so + RJ, so - RJ))
        gammax -= PP::div((rhos - rho0c) * gz * h0v * h0v, 2 * rho0c) * half * K.oneoverdx
                  * ((R)sTS[so + RJ] - (R)sTS[so - RJ]);
    if (j > 1 && j < P.ny && !zero_gradient(so + 1, so - 1))
        gammay -= PP::div((rhos - rho0c) * gz * h0v * h0v, 2 * rho0c) * half * K.oneoverdx
                  * ((R)sTS[so + 1] - (R)sTS[so - 1]);
    /* slope stability: provable "no failure" first, exact test otherwise */
    R fail = 0;
    {
        const R rho0 = K.rho0;
        const R A = rho0 * gz * dep0 + rho0c * gz * h0v;
        const R s = fabs(sy);
        const R depx = fabs((R)sDEP[i < P.nx ? so + RJ : so]) + fabs((R)sDEP[i > 1 ? so - RJ : so]);
        const R depy = fabs((R)sDEP[j < P.ny ? so + 1 : so]) + fabs((R)sDEP[j > 1 ? so - 1 : so]);
        const R pb = fabs(dep0) * rho0 * fabs(gz) * half * K.oneoverdx * fmax(depx, depy);
        const R w = rhow * gz * (dep0 + h0v);
        const R lhs_ub = A * s;
        const R rhs_lb = K.cohesion + (A * (1 - half * s * s) - w) * K.fa - pb;
        const R margin = R(1e-5) * (fabs(A) * (1 + s) + K.cohesion + fabs(w) * K.fa + pb) + R(1e-30);
        const bool safe = A >= 0 && gz > 0 && K.fa >= 0 && lhs_ub + margin < rhs_lb;
        if (!safe) {
            FailArgs fa;
            fa.nx = P.nx; fa.ny = P.ny; fa.pitch = P.pitch; fa.pad_ = 0; fa.plane = P.plane;
            fa.oneoverdx = P.oneoverdx; fa.half_odx = P.half_odx; fa.rho0 = P.rho0; fa.rhow = P.rhow;
            fa.cohesion = P.cohesion; fa.fa = P.fa;
            fa.solid = P.has_solid ? solid : nullptr; fa.z0 = z0;
            fail = fail_exact<PP, RS>(fa, src.dep, zp, zc, i, j, sx, sy, gz, dep0, rho0c, h0v);
        }
    }
    R dfmask = fmin(one, PP::divk(totsed0 - R(0.2), R(0.2), (R)P.inv_p2, P.divk_ok));
    if (h0v < K.h0x9 || totsed0 < R(0.2)) dfmask = 0;
    R betax = K.neg1ml * gz * h0v * K.fa;
    R betay = K.neg1ml * gz * h0v * K.fa;
    if (hu0 < 0) betax = -1 * betax;
    if (hv0 < 0) betay = -1 * betay;

    /* Hairsine-Rose, class-independent parts (SWEHR.c:1330-1382) */
    const R hvert = PP::div(h0v, PP::cos_atan(fabs(slope)));
    R mtstar = K.mtstar0;
    const bool deepv = hvert > K.h0;
    R depthfac = 1;
    if (deepv) {
        depthfac = PP::pow(PP::div(K.h0, hvert), K.b);
        mtstar = K.mtstar0 * depthfac;
    }
    const R Hs = fmin(one, PP::divz(totm0, mtstar));
    const bool swash = (h0v > K.hfx10 && totsed0 < R(0.6));
    R E3b = 0, E4b = 0, e4den = 1;
    if (swash) {
        const R manning = (h0v <= K.hc) ? K.roughness * PP::pow(PP::div(h0v, K.hc), K.dde) : K.roughness;
        const R qq = PP::sqrtp(hu0 * hu0 + hv0 * hv0);
        const R SF = PP::div(manning * manning * qq * qq, PP::pow(h0v, R(3.333)));
        /* streampowererosion (SWEHR.c:412-426): omega is the same for every
         * class; only the h > d_k condition differs */
        const R omega = rho0c * gz * SF * qq;
        if (omega > K.uc && totsed0 < R(0.6)) E3b = K.af * (omega - K.uc);
        if (omega > K.uc2 && totsed0 < R(0.6)) E4b = K.afr * (omega - K.uc2);
        e4den = PP::divk(rhos - rho0c, rhos, (R)P.inv_rhos, P.divk_ok) * gz * h0v;
    }
    const R vfconc = PP::pow(1 - fmin(totsed0, R(0.99)), R(4.0));
    const bool debris = (h0v > K.h0x9 && totsed0 > K.cthreshold);

    /* conservative update, SWEHR.c:1424-1446 */
    const R dtdx = dtr * K.oneoverdx;
    R h = h0v - dtdx * (fxr0 - fxl0) - dtdx * (fyr0 - fyl0) + dtr * Rc;
    R hu = hu0 - dtdx * (fxr1 - fxl1) - dtdx * (fyr1 - fyl1) + dtr * SXf + dtr * gammax + dtr * dfmask * betax;
    R hv = hv0 - dtdx * (fxr2 - fxl2) - dtdx * (fyr2 - fyl2) + dtr * SYf + dtr * gammay + dtr * dfmask * betay;
    /* Green-Ampt in FP64 (SWEHR.c:1449-1452) */
    const double ks = P.has_ks ? (double)cellr[CR_KS * T_I * T_J + cs] : P.ks;
    const double vinf0 = celld[CD_VINF * T_I * T_J + cs];
    const double zf = PolicyF64::divk(vinf0, P.thetas - P.theta0, P.inv_dtheta, P.divk_ok);
    const double hd = (double)h;
    const double infl = fmin(hd - P.hfilm, dt * ks * (zf + P.hf + hd) / zf);
    const double vinf = vinf0 + infl;
    h = (R)(hd - infl);

    /* classes (SWEHR.c:1454-1511).  U_k after the face fluxes, then its
     * final value: the FP64 form (rolled class loop) forms it at the top of
     * class k's iteration and keeps the final value in this cell's own slot
     * of the staged U_k plane (no other thread reads that slot once the faces
     * are solved), so no per-class array stays live in registers; the mixed
     * form's unrolled loops keep them in registers (faster there). */
    constexpr bool kSlot = PP::kRollClasses;
    static_assert(sizeof(R) == sizeof(RS), "the staged U_k slot holds a U_k value");
    const R *SED = reinterpret_cast<const R *>(smb + L.sed);
    RS *Uslot = reinterpret_cast<RS *>(const_cast<unsigned char *>(smb) + L.halo) + HP_U * L.hps + so;
    const int hps = L.hps;
    R Ureg[kSlot ? 1 : MAXS];
    if constexpr (!kSlot) {
#pragma unroll
        for (int k = 0; k < MAXS; k++) {
            if (k >= S) break;
            const R *sk = SED + k * N_H;
            Ureg[k] = (R)Uslot[k * hps] - dtdx * (fxr0 * sk[uxr] - fxl0 * sk[uxl])
                      - dtdx * (fyr0 * sk[uyr] - fyl0 * sk[uyl]);
        }
    }
    double z = zcs[(ti + 1) * R_J + (tj + 2)];
    double totm = 0, dep = 0;
    R chtemp = 0, bulk = 0;
#pragma unroll ((BUDGET || !kSlot) ? MAXS : 1)
    for (int k = 0; k < MAXS; k++) {
        if (k >= S) break;
        const int64_t qm = k * pl + q;
        const R *sk = SED + k * N_H;
        const RS u_in = Uslot[k * hps];
        R uflux;
        if constexpr (kSlot)
            uflux = (R)u_in - dtdx * (fxr0 * sk[uxr] - fxl0 * sk[uxl]) - dtdx * (fyr0 * sk[uyr] - fyl0 * sk[uyl]);
        else
            uflux = Ureg[kSlot ? 0 : k];
        const double Mk0 = L.stage_m ? celld[(CD_M + k) * T_I * T_J + cs] : __ldg(src.M + qm);
        const R Mk0r = (R)Mk0;
        /* Rain-splash detachment of the original soil is the only source the
         * shallow branch uses; the other sources and the settling velocity
         * are formed only in the deep branch, where they are read (the same
         * values, computed only when needed). */
        R E1 = 0;
        if (swash && !debris) {
            E1 = (1 - Hs) * K.pf[k] * K.a * Rc;
            if (deepv) E1 = E1 * depthfac;
        }

        double Mk = Mk0;
        R u = uflux;
        double det_k = 0;         /* original soil detached into U_k + M_k this step (budget) */
        if (h < K.hfx10) {
            Mk += (double)(dtr * E1 + u);
            u = 0;
            if (BUDGET) det_k = (double)(dtr * E1);
        } else {
            R E2 = 0, E3 = 0, E4 = 0, VF = 0;
            if (swash && !debris) {
                if (totm0 > R(1e-8) && Mk0r > R(1e-8)) E2 = PP::div(Hs * Mk0r, totm0) * K.ad * Rc;
                if (deepv) E2 = E2 * depthfac;
                E3 = PP::e3_term((1 - Hs) * K.pf[k] * K.F, K.J, (R)P.inv_J, P.divk_ok, h0v > K.ds[k] ? E3b : R(0));
                if (totm0 > R(1e-6) && Mk0r > 0)
                    E4 = PP::e4_term(K.one_m_bb * Hs * Mk0r, totm0, K.F, e4den, h0v > K.ds[k] ? E4b : R(0));
            }
            if (!debris) {
                VF = PP::settle(K.a13[k], K.a13sq[k], K.c109s * gz * K.ds[k]);
                VF = VF * vfconc;
                if (K.ds[k] > R(0.0001) && h0v < K.h0x9)
                    VF = R(2e-3) + PP::divk(fmax(h0v - K.h0x3, R(0)) * (VF - R(2e-3)), K.h0x6, (R)P.inv_h0x6, P.divk_ok);
                if (K.ds[k] > R(0.002) && h0v < K.h0x9)
                    VF = R(2e-3) + PP::divk(fmax(h0v - K.h0x3, R(0)) * (VF - R(2e-3)), K.h0x6, (R)P.inv_h0x6, P.divk_ok);
            }
            chtemp = u;
            const R redetach = fmin(Mk0r, dtr * (E2 + E4));
            const R dec = PP::exp(PP::div(-VF, h) * (half * dtr));
            u = dec * u;
            u = u + dtr * (E1 + E3) + redetach;
            u = dec * u;
            z = z - P.invporo * (double)(u - chtemp);
            Mk = Mk + (double)(dtr * (E1 + E3)) - (double)(u - chtemp);
            if (BUDGET) det_k = (double)(dtr * (E1 + E3));
            if (fail == 1) {
                z = z - 0.99 * Mk / P.porod;
                u = u + (R)(0.99 * Mk);
                totm = 0;
                Mk = 0.01 * Mk;
                dep = 0;
            }
        }
        const R dh = PP::divk(u - chtemp, K.porod, (R)P.invporo, P.divk_ok);
        h = h + dh;
        bulk += dh;
        totm += Mk;
        dep += PP::dep_of(Mk, P);
        if constexpr (kSlot)
            Uslot[k * hps] = (RS)u;
        else
            Ureg[kSlot ? 0 : k] = u;
        if (L.stage_m)         /* the cell's own staged slot: read back below, no global round trip */
            const_cast<double *>(celld)[(CD_M + k) * T_I * T_J + cs] = Mk;
        else
            dst.M[qm] = Mk;
        if (BUDGET) {
            /* U_k + M_k changes only by the face fluxes and detachment; what
             * the arithmetic and storage add on top is accounted as rounding */
            const double div = ((double)(fxr0 * sk[uxr]) - (double)(fxl0 * sk[uxl]))
                               + ((double)(fyr0 * sk[uyr]) - (double)(fyl0 * sk[uyl]));
            const double change = ((double)(RS)u - (double)u_in) + (Mk - Mk0);
            acc.det[k] += det_k;
            acc.sround[k] += change - (-(dt * P.oneoverdx) * div + det_k);
        }
    }

    /* derived fields and the dry clamp, SWEHR.c:1513-1551 */
    R totsed = 0, clamp = 0;
    if (h > hfilm) {
#pragma unroll
        for (int k = 0; k < MAXS; k++) {
            if (k >= S) break;
            const R uk = kSlot ? (R)Uslot[k * hps] : Ureg[kSlot ? 0 : k];
            totsed += PP::divk(PP::divz(uk, h), rhos, (R)P.inv_rhos, P.divk_ok);
            dst.U[k * pl + q] = (RS)uk;
            if (L.stage_m) dst.M[k * pl + q] = celld[(CD_M + k) * T_I * T_J + cs];
        }
    } else {
        clamp = hfilm - h;
        h = hfilm;
        hu = 0;
        hv = 0;
#pragma unroll
        for (int k = 0; k < MAXS; k++) {
            if (k >= S) break;
            const int64_t qm = k * pl + q;
            const R uk = kSlot ? (R)Uslot[k * hps] : Ureg[kSlot ? 0 : k];
            z = z + P.invporo * (double)uk;
            const double mk = L.stage_m ? celld[(CD_M + k) * T_I * T_J + cs] : dst.M[qm];
            dst.M[qm] = mk + (double)uk;
            dst.U[qm] = (RS)0;
        }
    }
    /* implicit friction, SWEHR.c:1553-1565 */
    R vel1 = 0, vel2 = 0;
    if (h > hfilm) {
        const R manning = (h <= K.hc) ? K.roughness * PP::pow(PP::div(h, K.hc), K.dde) : K.roughness;
        const R SFf = PP::div(manning * manning * gz * PP::sqrtp(hu * hu + hv * hv) * 1, PP::pow(h, R(2.333)));
        hu = PP::div(hu, 1 + dtr * SFf);
        hv = PP::div(hv, 1 + dtr * SFf);
        vel1 = PP::div(hu, h);
        vel2 = PP::div(hv, h);
    }
    R maxvel = (R)cellr[CR_MAXVEL * T_I * T_J + cs], maxdep = (R)cellr[CR_MAXDEP * T_I * T_J + cs];
    const R vmag = PP::sqrtz(vel1 * vel1 + vel2 * vel2);
    if (vmag > maxvel) maxvel = vmag;
    if (h > maxdep) maxdep = h;
    dst.h[q] = (RS)h;
    dst.hu[q] = (RS)hu;
    dst.hv[q] = (RS)hv;
    dst.vinf[q] = vinf;
    dst.maxvel[q] = (RS)maxvel;
    dst.maxdep[q] = (RS)maxdep;
    dst.totm[q] = (RS)totm;
    dst.dep[q] = (RS)dep;
    dst.totsed[q] = (RS)totsed;
    dst.gz[q] = (RS)gz;                /* the next step's lagged GZ: this step's topography */
    zn[q] = z;

    if (BUDGET) {
        /* water: the state changes by the face fluxes, rain, infiltration,
         * bulking and the dry clamp; the arithmetic and storage rounding of h
         * is accounted separately so the budget closes exactly */
        const double dtdx_d = dt * P.oneoverdx;
        const double div = ((double)fxr0 - (double)fxl0) + ((double)fyr0 - (double)fyl0);
        const double accounted = -dtdx_d * div + dt * (double)Rc - infl + (double)bulk + (double)clamp;
        acc.round += ((double)(RS)h - (double)h0v) - accounted;
        acc.rain += dt * (double)Rc;
        acc.inf += infl;
        acc.clamp += (double)clamp;
        acc.bulk += (double)bulk;
        if (i == 1 || i == P.nx || j == 1 || j == P.ny) {
#pragma unroll
            for (int k = 0; k < MAXS; k++) {
                if (k >= S) break;
                const R *sk = SED + k * N_H;
                if (i == 1) acc.sout[k] -= dtdx_d * (double)(fxl0 * sk[uxl]);
                if (i == P.nx) acc.sout[k] += dtdx_d * (double)(fxr0 * sk[uxr]);
                if (j == 1) acc.sout[k] -= dtdx_d * (double)(fyl0 * sk[uyl]);
                if (j == P.ny) acc.sout[k] += dtdx_d * (double)(fyr0 * sk[uyr]);
            }
            if (i == 1) acc.out -= dtdx_d * (double)fxl0;
            if (i == P.nx) acc.out += dtdx_d * (double)fxr0;
            if (j == 1) acc.out -= dtdx_d * (double)fyl0;
            if (j == P.ny) acc.out += dtdx_d * (double)fyr0;
        }
    }
}

/* stage row of SWEHR.c:1593-1676 from the new state (one block) */
template <class PP, class RS>
__device__ __forceinline__ void stage_sample_tile(const DevParams &P, const SetV<RS> &st, Ctl *ctl, double tnew,
                                                  double *stage, double *saveflow, double *scratch)
{
    double *bv = scratch;
    int *bi = reinterpret_cast<int *>(scratch + TILE_THREADS);
    const int64_t pl = P.plane;
    const int row = P.outlet_row;
    double best = 0;
    int besti = 1;
    for (int i = 1 + threadIdx.x; i <= P.nx; i += blockDim.x) {
        const double h = (double)st.h[cidx(P, i, row)];
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
    const double ho = (double)st.h[qo];
    const double v1 = ho > P.hfilm ? (double)st.hu[qo] / ho : 0, v2 = ho > P.hfilm ? (double)st.hv[qo] / ho : 0;
    row_out[0] = tnew;
    row_out[1] = ho;
    row_out[2] = sw_sqrt_pow(v1 * v1 + v2 * v2);
    row_out[3] = (double)st.totsed[qo];
    for (int k = 0; k < 10; k++) {
        row_out[4 + k] = (k < P.S) ? st.M[k * pl + qo] : 0;
        row_out[14 + k] = (k < P.S) ? (double)st.U[k * pl + qo] : 0;
    }
    double *pr = saveflow + r * 18;
    for (int m = 0; m < 6; m++) {
        const int xi = P.xpoint[m], yj = P.ypoint[m];
        if (m >= P.npoints || xi < 1 || xi > P.nx || yj < 1 || yj > P.ny) {
            pr[3 * m] = pr[3 * m + 1] = pr[3 * m + 2] = __longlong_as_double(0x7ff8000000000000LL);
            continue;
        }
        const int64_t qp = cidx(P, xi, yj);
        const double hp = (double)st.h[qp];
        const double w1 = hp > P.hfilm ? (double)st.hu[qp] / hp : 0, w2 = hp > P.hfilm ? (double)st.hv[qp] / hp : 0;
        pr[3 * m] = hp;
        pr[3 * m + 1] = sw_sqrt_pow(w1 * w1 + w2 * w2);
        pr[3 * m + 2] = (double)st.totsed[qp];
    }
    ctl->stagecnt = r + 1;
    ctl->stageinterval += P.stageint;
}

/* Update of one tile: stages A (staging), B (faces), C (cells).  The whole
 * block calls it. */
template <class PP, class RS, int MAXS, bool BUDGET, bool TMA = false, int NS = 0>
__device__ __forceinline__ void update_tile(const DevParams &P, const BufsT<RS> &B, int64_t n, double t, double dt,
                                            double Rr, TileCoord tc, unsigned char *smb, const StagedLayout &L,
                                            Acc2<MAXS, BUDGET> &acc, const TmaMaps *tm = nullptr,
                                            uint64_t *bar = nullptr, uint32_t *phase = nullptr, Ctl *ctl = nullptr)
{
    typedef typename PP::R R;
    const RealC<R> &K = kc<R>(P);
    const SetV<RS> src = B.set[n & 1];
    const SetV<RS> dst = B.set[(n + 1) & 1];
    const double *zp = B.z[(n + 2) % 3], *zc = B.z[n % 3];
    double *zn = B.z[(n + 1) % 3];
    double inh = 0, inhv = 0, insed = 0;
    if (P.inflow) inflow_ghost(t, inh, inhv, insed);
    unsigned char *upb = smb + L.up;
    const R *su = reinterpret_cast<const R *>(smb + L.u), *sv = reinterpret_cast<const R *>(smb + L.v);
    const R *sg = reinterpret_cast<const R *>(smb + L.g), *sc = reinterpret_cast<const R *>(smb + L.c);
    R *sfx = reinterpret_cast<R *>(smb + L.fx), *sfy = reinterpret_cast<R *>(smb + L.fy);
    if constexpr (TMA) {
        /* the previous tile's reads and writes of these buffers are done
         * (the barrier ending it); order them before the copies that land */
        if (threadIdx.x == 0) {
            fence_proxy_async_smem();
            stage_load_tma<RS>(P, *tm, (int)(n & 1), n, tc, smb, L, bar);
        }
        if (!mbar_wait_bounded(bar, *phase & 1u) && threadIdx.x == 0) ctl->dev_error = 1;
        *phase += 1;
        __syncthreads();
    } else {
        stage_load<RS, NS>(P, src, zp, zc, B.ks, tc, smb, L);
        __pipeline_wait_prior(0);
        __syncthreads();
    }
    stage_derive<PP, RS, NS>(P, src, tc, smb, L, (R)inh, (R)inhv, (R)insed);
    __syncthreads();
    const RS *sh = staged_h<RS>(smb, L);
    /* stage B: every face of the tile (SWEHR.c:1099-1230) */
    for (int f = threadIdx.x; f < N_FX + N_FY; f += TILE_THREADS) {
        R T0, T1, T2;
        if (f < N_FX) {
            const int fi = f / T_J, fj = f - fi * T_J;
            const int gi = tc.i0 - 1 + fi, gj = tc.j0 + fj;
            if (gj > P.ny || gi > P.nx) continue;
            const int Lh = fi * H_J + fj + 1, Rh = Lh + H_J;
            const R hl = (R)sh[fi * Cols<RS>::rj + fj + Cols<RS>::pad], hr = (R)sh[(fi + 1) * Cols<RS>::rj + fj + Cols<RS>::pad];
            int var = 0;                 /* 1: solid left, 2: solid right (SWEHR.c:1137-1146) */
            if (P.has_solid && gi >= 1 && gi < P.nx) {
                const bool sl = solid_at(P, B.solid, gi, gj), sr = solid_at(P, B.solid, gi + 1, gj);
                var = (sl && !sr) ? 1 : ((!sl && sr) ? 2 : 0);
            }
            /* the mirrored normal velocity is (-hu)/h when wet (a zero keeps its
             * negated sign, as in the reference) and +0 when dry */
            if (var == 1)
                hllc_v<PP>(hr, hr, mirror_v<PP>(su[Rh], hr, K.hfilm), su[Rh], sv[Rh], sv[Rh], sg[Lh],
                           PP::sqrtp(sg[Lh] * hr), K.hfilm, T0, T1, T2);
            else if (var == 2)
                hllc_v<PP>(hl, hl, su[Lh], mirror_v<PP>(su[Lh], hl, K.hfilm), sv[Lh], sv[Lh], sg[Lh], sc[Lh], K.hfilm,
                           T0, T1, T2);
            else
                hllc_v<PP>(hl, hr, su[Lh], su[Rh], sv[Lh], sv[Rh], sg[Lh], sc[Lh], K.hfilm, T0, T1, T2);
            R *F = sfx + 3 * f;
            F[0] = T0; F[1] = T1; F[2] = T2;
            upb[f] = (T0 > 0) ? 0 : 1;
        } else {
            const int f2 = f - N_FX;
            const int fi = f2 / (T_J + 1), fj = f2 - fi * (T_J + 1);
            const int gi = tc.i0 + fi, gj = tc.j0 - 1 + fj;
            if (gi > P.nx || gj > P.ny) continue;
            const int Lh = (fi + 1) * H_J + fj, Rh = Lh + 1;
            const R hl = (R)sh[(fi + 1) * Cols<RS>::rj + fj + Cols<RS>::pad - 1],
                    hr = (R)sh[(fi + 1) * Cols<RS>::rj + fj + Cols<RS>::pad];
            int var = 0;                 /* 1: solid below, 2: solid above (SWEHR.c:1205-1214) */
            if (P.has_solid && gj >= 1) {
                const bool sl = solid_at(P, B.solid, gi, gj), sr = solid_at(P, B.solid, gi, gj + 1);
                var = (sl && !sr) ? 1 : ((!sl && sr) ? 2 : 0);
            }
            if (var == 1)
                hllc_v<PP>(hr, hr, mirror_v<PP>(sv[Rh], hr, K.hfilm), sv[Rh], su[Rh], su[Rh], sg[Lh],
                           PP::sqrtp(sg[Lh] * hr), K.hfilm, T0, T1, T2);
            else if (var == 2)
                hllc_v<PP>(hl, hl, sv[Lh], mirror_v<PP>(sv[Lh], hl, K.hfilm), su[Lh], su[Lh], sg[Lh], sc[Lh], K.hfilm,
                           T0, T1, T2);
            else
                hllc_v<PP>(hl, hr, sv[Lh], sv[Rh], su[Lh], su[Rh], sg[Lh], sc[Lh], K.hfilm, T0, T1, T2);
            R *F = sfy + 3 * f2;
            F[0] = T0; F[1] = T2; F[2] = T1;
            upb[f] = (T0 > 0) ? 0 : 1;
        }
    }
    __syncthreads();
    tile_cell<PP, RS, MAXS, BUDGET, NS>(P, src, dst, zp, zc, zn, smb, L, tc, t, dt, Rr, acc, B.solid, B.z0);
    __syncthreads();
}

/* Block sum of the budget accumulators into red[B_NTERMS] (thread 0 holds
 * the block's totals afterwards); fixed order, so deterministic. */
template <int MAXS, bool BUDGET>
__device__ __forceinline__ void budget_block_sum(const Acc2<MAXS, BUDGET> &acc, double *red)
{
    double v[B_NTERMS];
    v[B_RAIN] = acc.rain; v[B_OUT] = acc.out; v[B_CLAMP] = acc.clamp; v[B_BULK] = acc.bulk; v[B_INF] = acc.inf;
    v[B_ROUND] = acc.round;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        v[B_DET + k] = (k < MAXS) ? acc.det[k < MAXS ? k : 0] : 0.0;
        v[B_SOUT + k] = (k < MAXS) ? acc.sout[k < MAXS ? k : 0] : 0.0;
        v[B_SROUND + k] = (k < MAXS) ? acc.sround[k < MAXS ? k : 0] : 0.0;
    }
#pragma unroll
    for (int m = 0; m < B_NTERMS; m++) {
        const double s = warp_sum(v[m]);
        if ((threadIdx.x & 31) == 0) red[(threadIdx.x >> 5) * B_NTERMS + m] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int m = 0; m < B_NTERMS; m++) {
            double s = 0;
            for (int w = 0; w < TILE_THREADS / 32; w++) s += red[w * B_NTERMS + m];
            red[m] = s;
        }
    __syncthreads();
}

template <int MAXS, bool BUDGET>
__device__ __forceinline__ void acc_zero(Acc2<MAXS, BUDGET> &acc)
{
    acc.rain = acc.out = acc.clamp = acc.bulk = acc.inf = acc.round = 0;
#pragma unroll
    for (int k = 0; k < (BUDGET ? MAXS : 1); k++) acc.det[k] = acc.sout[k] = acc.sround[k] = 0;
}

/* End of a step once every cell is written (whole block): time, step
 * counter, stage row (SWEHR.c:1591-1676), stop conditions. */
template <class PP, class RS>
__device__ __forceinline__ void update_finalize(const DevParams &P, const SetV<RS> &dst, Ctl *ctl, double *stage,
                                                double *saveflow, unsigned char *smb)
{
    __threadfence();
    const int64_t n = ctl->step;
    const double t = ctl->t, dt = ctl->dt;
    const double tnew = (ctl->cfl ? 2 * P.tend : t) + dt;
    const bool stage_due = tnew > ctl->stageinterval && ctl->stagecnt < ctl->stagecap;
    __syncthreads();
    if (stage_due) stage_sample_tile<PP, RS>(P, dst, ctl, tnew, stage, saveflow, reinterpret_cast<double *>(smb));
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->t_prev = t;
        ctl->t = tnew;
        ctl->step = n + 1;
        ctl->pending = 0;
        ctl->update_ticket = 0u;
        if (ctl->cfl) ctl->status = 1;
        if (!(dt > 0) && !ctl->cfl) ctl->status = 2;
        if (ctl->dev_error) {
            ctl->status = 3;
            ctl->active = 0;
        }
        if (ctl->cfl || !(dt > 0) || !(tnew < P.tend) || !(tnew < ctl->t_stop) || n + 1 >= ctl->max_step)
            ctl->active = 0;
        ctl->launches += 2;
    }
}

__device__ __forceinline__ void budget_fold(Ctl *ctl, int m, double hi, double lo)
{
    double Hh = ctl->budget_hi[m], Ll = ctl->budget_lo[m];
    dd_add(Hh, Ll, hi);
    Ll += lo;
    ctl->budget_hi[m] = Hh;
    ctl->budget_lo[m] = Ll;
}

template <class PP, class RS, int MAXS, bool BUDGET, bool STAGE_M, bool TMA, int NS>
__global__ void __launch_bounds__(TILE_THREADS, PP::kMinBlocks) k_update_tile(const DevParams P, const BufsT<RS> B, Ctl *ctl,
                                                                  const double *__restrict__ rain, double *partials,
                                                                  double *stage, double *saveflow,
                                                                  const __grid_constant__ TmaMaps tm)
{
    typedef typename PP::R R;
    if (!ctl->pending) return;
    extern __shared__ __align__(128) unsigned char smb_raw[];
    /* tile-copy destinations must start on 128 bytes: with tensor-map loads
     * the launch adds 128 bytes and the staging starts at the next boundary */
    unsigned char *smb = TMA ? reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smb_raw) + 127) &
                                                                ~static_cast<uintptr_t>(127))
                             : smb_raw;
    __shared__ bool last;
    __shared__ __align__(8) uint64_t tma_bar;
    uint32_t tma_phase = 0;
    if constexpr (TMA) {
        if (threadIdx.x == 0) {
            mbar_init(&tma_bar, 1);
            mbar_init_fence();
        }
        __syncthreads();
    }
    const StagedLayout L = StagedLayout::make(P.S, sizeof(R), STAGE_M);
    const int64_t n = ctl->step;
    const double t = ctl->t, dt = ctl->dt;
    const double Rr = P.storm ? 0.0 : rain_at(P, rain, t);
    Acc2<MAXS, BUDGET> acc;
    acc_zero(acc);
    const int64_t ntiles = (int64_t)((P.own_hi - P.own_lo + T_I) / T_I) * ((P.ny + T_J - 1) / T_J);
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
        update_tile<PP, RS, MAXS, BUDGET, TMA, NS>(P, B, n, t, dt, Rr, tile_coord(P, tile), smb, L, acc, &tm, &tma_bar,
                                               &tma_phase, ctl);
    double *red = reinterpret_cast<double *>(smb + L.red);
    if (BUDGET) budget_block_sum(acc, red);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        if (BUDGET)
            for (int m = 0; m < B_NTERMS; m++) partials[(int64_t)blockIdx.x * B_NTERMS + m] = red[m];
        __threadfence();
        last = (atomicAdd(&ctl->update_ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (BUDGET && threadIdx.x < B_NTERMS) {
        double hi = 0, lo = 0;
        for (unsigned b = 0; b < gridDim.x; b++)
            dd_add(hi, lo, ((volatile double *)partials)[(int64_t)b * B_NTERMS + threadIdx.x]);
        budget_fold(ctl, threadIdx.x, hi, lo);
    }
    if (threadIdx.x == 0) ctl->rain_now = Rr;
    update_finalize<PP, RS>(P, B.set[(n + 1) & 1], ctl, stage, saveflow, smb);
}

/* ------------------------------------------------------------- batched ---
 * Many independent scenarios of uneven sizes stepped by one launch of each
 * kernel.  The tiles of all scenarios form one list (scenario s owns tiles
 * [tile0, tile0 + ntiles)); a persistent grid walks it.  Each scenario keeps
 * its own control block, dt, t and stage rows: the block that completes a
 * scenario's last tile finalizes that scenario.  Finished scenarios' tiles
 * are skipped with one load.  Per-cell arithmetic is the single-domain
 * arithmetic, so every scenario's result is identical alone or in a batch.
 * Budget sums of a batched step are block partials added with atomics
 * (order-dependent rounding of the budget terms only). */
/* Copy scenario sid's descriptor into the block's shared copy (the whole
 * block calls it).  Parameters then come from a shared object no other store
 * can alias, instead of global memory the compiler would have to re-read
 * after every store.  Thread 0 also snapshots the scenario's step state: it
 * cannot change while this block still holds uncounted tiles of it (the
 * scenario's pass ends only once every tile is counted). */
/* Work distribution of the batched passes: a block takes a chunk of
 * consecutive tiles of the list at a time from a global counter, so blocks
 * that start late or draw slow tiles take fewer (a fixed stride leaves the
 * whole launch waiting on the slowest block), and consecutive tiles mostly
 * share one scenario's descriptor.  Chunks are the largest power of two up
 * to TILE_CHUNK tiles that still gives every block at least eight of them
 * (on 256 scenarios each doubling from 1 to 8 tiles measured faster), down
 * to single tiles, so a small pool (a serving mix of a few
 * requests) still spreads over all blocks.  The whole block calls
 * grab_chunk; it returns false once the list is exhausted. */
#define TILE_CHUNK 8
struct TileChunk {
    int64_t g0;
    int n;
    int sid[TILE_CHUNK];
};

__device__ __forceinline__ bool grab_chunk(unsigned long long *counter, const int32_t *__restrict__ map, int64_t total,
                                           TileChunk &ch)
{
    __syncthreads();                                             /* the previous chunk is done with */
    if (threadIdx.x == 0) {
        int size = TILE_CHUNK;
        while (size > 1 && total < (int64_t)8 * size * gridDim.x) size >>= 1;
        const int64_t g0 = (int64_t)atomicAdd(counter, (unsigned long long)size);
        const int64_t rest = total - g0;
        ch.g0 = g0;
        ch.n = rest <= 0 ? 0 : (rest < size ? (int)rest : size);
        for (int c = 0; c < ch.n; c++) ch.sid[c] = map[g0 + c];
    }
    __syncthreads();
    return ch.n > 0;
}

struct StepSnap {
    double t, dt, rain;
    int64_t n;
    int32_t go;                          /* active (wave pass) / pending (update pass) */
};

template <class RS>
__device__ __forceinline__ void load_desc(const ScenDesc<RS> *tab, int sid, ScenDesc<RS> &sd, StepSnap &snap,
                                          bool update_pass)
{
    static_assert(sizeof(ScenDesc<RS>) % 8 == 0, "descriptor copied in 8-byte words");
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(tab + sid);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(&sd);
    __syncthreads();                                             /* the previous run is done with sd */
    for (int w = threadIdx.x; w < (int)(sizeof(ScenDesc<RS>) / 8); w += blockDim.x) dst[w] = src[w];
    if (threadIdx.x == 0) {
        const Ctl *ctl = tab[sid].ctl;
        snap.go = update_pass ? ctl->pending : ctl->active;
        snap.n = ctl->step;
        snap.t = ctl->t;
        snap.dt = ctl->dt;
        snap.rain = ctl->rain_now;
    }
    __syncthreads();
}

/* Batched wave pass.  A block takes chunks of the tile list (grab_chunk) and
 * keeps a run per scenario: consecutive tiles of one scenario share the
 * descriptor copy and a running max, and the scenario's ticket is advanced
 * by the run's tile count once, when the block moves on (or finishes). */
template <class PP, class RS>
__global__ void __launch_bounds__(TILE_THREADS) k_wave_batch(const BatchHdr<RS> *__restrict__ hdr)
{
    typedef typename PP::R R;
    __shared__ double red8[TILE_THREADS / 32];
    __shared__ __align__(16) ScenDesc<RS> sd;
    __shared__ StepSnap snap;
    const ScenDesc<RS> *tab = hdr->tab;
    const int32_t *map = hdr->tile_scen;
    const int64_t total = hdr->total_tiles;
    int cur = -1;
    unsigned run = 0;                    /* tiles of `cur` done and not yet counted */
    R smax = 0;
    double snap_inh = 0, snap_inhv = 0;  /* the scenario's inflow ghost at this step */
    auto flush = [&]() {
        const double m = block_max((double)smax, red8);
        if (threadIdx.x == 0) {
            Ctl *ctl = sd.ctl;
            atomicMax(&ctl->smax_bits, (unsigned long long)__double_as_longlong(m));
            __threadfence();
            if (atomicAdd(&ctl->wave_ticket, run) == (unsigned)sd.ntiles - run) {
                wave_finalize(sd.P, ctl);
                /* the step's uniform rain rate, read by every update tile */
                ctl->rain_now = sd.P.storm ? 0.0 : rain_at(sd.P, sd.rain, snap.t);
            }
        }
        run = 0;
        smax = 0;
    };
    __shared__ TileChunk chunk;
    if (blockIdx.x == 0 && threadIdx.x == 0) hdr->grab[1] = 0ull;  /* the update pass's counter, for after us */
    for (;;) {
        if (!grab_chunk(hdr->grab, map, total, chunk)) break;
        for (int c = 0; c < chunk.n; c++) {
            const int64_t g = chunk.g0 + c;
            const int sid = chunk.sid[c];                        /* uniform across the block */
            if (sid != cur) {
                if (run) flush();
                load_desc(tab, sid, sd, snap, false);
                cur = sid;
                double insed = 0;
                snap_inh = snap_inhv = 0;
                if (sd.P.inflow) inflow_ghost(snap.t, snap_inh, snap_inhv, insed);
            }
            if (!snap.go) continue;
            const int64_t n = snap.n;
            const TileCoord tc = tile_coord(sd.P, g - sd.tile0);
            const int i = tc.i0 + (int)threadIdx.x / T_J, j = tc.j0 + (int)threadIdx.x % T_J;
            if (i <= sd.P.nx && j <= sd.P.ny) {
                const R s = wave_cell<PP, RS>(sd.P, sd.B.set[n & 1], i, j, (R)snap_inh, (R)snap_inhv,
                                              sd.P.has_solid ? sd.B.solid : nullptr);
                smax = (s > smax) ? s : smax;
            }
            run++;
        }
    }
    if (run) flush();
}

/* Batched update pass, with the same per-scenario runs: budget accumulators
 * carry across a run and are summed, counted and folded once per run. */
template <class PP, class RS, int MAXS, bool BUDGET, bool STAGE_M, int NS>
__global__ void __launch_bounds__(TILE_THREADS, PP::kBatchMinBlocks) k_update_batch(const BatchHdr<RS> *__restrict__ hdr)
{
    typedef typename PP::R R;
    extern __shared__ __align__(128) unsigned char smb[];
    __shared__ bool last;
    __shared__ __align__(16) ScenDesc<RS> sd;
    __shared__ StepSnap snap;
    const ScenDesc<RS> *tab = hdr->tab;
    const int32_t *map = hdr->tile_scen;
    const int64_t total = hdr->total_tiles;
    int cur = -1;
    unsigned run = 0;
    Acc2<MAXS, BUDGET> acc;
    acc_zero(acc);
    /* the staging layout of the current scenario, uniform across the block:
     * kept in shared memory rather than in every thread's registers */
    __shared__ StagedLayout L;
    if (threadIdx.x == 0) L = StagedLayout::make(1, sizeof(R), STAGE_M);
    auto flush = [&]() {
        Ctl *ctl = sd.ctl;
        double *red = reinterpret_cast<double *>(smb + L.red);
        const bool bud = BUDGET && sd.P.budget;
        if (bud) budget_block_sum(acc, red);
        __syncthreads();
        /* release the run's writes, count its tiles; the scenario's last run
         * acquires everyone's writes before finalizing (one thread fences on
         * either side of the barrier) */
        if (threadIdx.x == 0) {
            if (bud)
                for (int m = 0; m < B_NTERMS; m++) atomicAdd(&ctl->budget_step[m], red[m]);
            __threadfence();
            const bool l = atomicAdd(&ctl->update_ticket, run) == (unsigned)sd.ntiles - run;
            if (l) __threadfence();
            last = l;
        }
        __syncthreads();
        if (last) {
            if (bud && threadIdx.x < B_NTERMS) {
                const double v = atomicAdd(&ctl->budget_step[threadIdx.x], 0.0);
                ctl->budget_step[threadIdx.x] = 0.0;
                budget_fold(ctl, threadIdx.x, v, 0.0);
            }
            update_finalize<PP, RS>(sd.P, sd.B.set[(snap.n + 1) & 1], ctl, sd.stage, sd.saveflow, smb);
            if (threadIdx.x == 0) {
                ScenSummary *q = sd.sum;
                q->t = ctl->t; q->dt = ctl->dt; q->courant = ctl->courant; q->step = ctl->step;
                q->status = ctl->status; q->active = ctl->active;
            }
        }
        run = 0;
        acc_zero(acc);
    };
    __shared__ TileChunk chunk;
    if (blockIdx.x == 0 && threadIdx.x == 0) hdr->grab[0] = 0ull;  /* the wave pass's counter, for the next step */
    for (;;) {
        if (!grab_chunk(hdr->grab + 1, map, total, chunk)) break;
        for (int c = 0; c < chunk.n; c++) {
            const int64_t g = chunk.g0 + c;
            const int sid = chunk.sid[c];                        /* uniform across the block */
            if (sid != cur) {
                if (run) flush();
                load_desc(tab, sid, sd, snap, true);
                cur = sid;
                if (threadIdx.x == 0) L = StagedLayout::make(sd.P.S, sizeof(R), STAGE_M);
                __syncthreads();
            }
            if (!snap.go) continue;
            update_tile<PP, RS, MAXS, BUDGET, false, NS>(sd.P, sd.B, snap.n, snap.t, snap.dt, snap.rain,
                                              tile_coord(sd.P, g - sd.tile0), smb, L, acc);
            run++;
        }
    }
    if (run) flush();
}

}  // inline namespace SWEHR_TILE_NS
}  // namespace swehr
