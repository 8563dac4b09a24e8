/*
 * swehr_faces.cuh -- face-neighbour states and HLL face fluxes of the FP64
 * form, read straight from a state set (SWEHR.c:816-1035 ghosts,
 * 1099-1230 face fluxes), plus warp reductions.  Shared by every FP64 kernel.
 */
#pragma once
#include "swehr_device.cuh"

namespace swehr {

#define NB_THREADS 256

/* x-face neighbour (i in 0..nx+1, j in 1..ny), ghosts per SWEHR.c:817-864, 913-960 */
__device__ __forceinline__ Nb nb_x(const DevParams &P, const double *__restrict__ src, int i, int j)
{
    Nb o;
    o.inflow = 0;
    int si = i;
    bool neg = false;
    if (i == 0) { si = 1; neg = P.bndry[0] == 1; }
    else if (i == P.nx + 1) { si = P.nx; neg = P.bndry[2] == 1; }
    o.q = cidx(P, si, j);
    o.h = src[P_H * P.plane + o.q];
    double hu = src[P_HU * P.plane + o.q];
    o.hu = neg ? -hu : hu;
    o.hv = src[P_HV * P.plane + o.q];
    return o;
}

/* y-face neighbour (i in 1..nx, j in 0..ny+1), SWEHR.c:865-912, 961-1035 */
__device__ __forceinline__ Nb nb_y(const DevParams &P, const double *__restrict__ src, int i, int j,
                                   double inh, double inhv)
{
    Nb o;
    o.inflow = 0;
    int sj = j;
    bool neg = false;
    if (j == 0) { sj = 1; neg = P.bndry[1] == 1; }
    else if (j == P.ny + 1) {
        if (P.inflow) {
            o.h = inh; o.hu = 0; o.hv = inhv; o.q = 0; o.inflow = 1;
            return o;
        }
        sj = P.ny; neg = P.bndry[3] == 1;
    }
    o.q = cidx(P, i, sj);
    o.h = src[P_H * P.plane + o.q];
    o.hu = src[P_HU * P.plane + o.q];
    double hv = src[P_HV * P.plane + o.q];
    o.hv = neg ? -hv : hv;
    return o;
}

struct Face {
    double F0, Fu, Fv;   /* fluxes of h, hu, hv */
    int64_t qup;         /* upwind cell for the sediment fluxes */
    int up_inflow;
};

/* x face between (iL, j) and (iL+1, j), iL in 0..nx (SWEHR.c:1099-1163) */
__device__ __forceinline__ double face_x(const DevParams &P, const double *__restrict__ src,
                                         const double *__restrict__ zp, int iL, int j, Face &f)
{
    Nb L = nb_x(P, src, iL, j), R = nb_x(P, src, iL + 1, j);
    double g = gz_of(P, zp, iL == 0 ? 1 : iL, j);
    double T0, T1, T2;
    double s = hllc(L.h, R.h, L.hu, R.hu, L.hv, R.hv, g, P.hfilm, T0, T1, T2);
    f.F0 = T0; f.Fu = T1; f.Fv = T2;
    f.qup = (T0 > 0) ? L.q : R.q;
    f.up_inflow = 0;
    return s;
}

/* y face between (i, jL) and (i, jL+1), jL in 0..ny (SWEHR.c:1167-1230) */
__device__ __forceinline__ double face_y(const DevParams &P, const double *__restrict__ src,
                                         const double *__restrict__ zp, int i, int jL, double inh, double inhv,
                                         Face &f)
{
    Nb L = nb_y(P, src, i, jL, inh, inhv), R = nb_y(P, src, i, jL + 1, inh, inhv);
    double g = gz_of(P, zp, i, jL == 0 ? 1 : jL);
    double T0, T1, T2;
    double s = hllc(L.h, R.h, L.hv, R.hv, L.hu, R.hu, g, P.hfilm, T0, T1, T2);
    f.F0 = T0; f.Fu = T2; f.Fv = T1;
    if (T0 > 0) { f.qup = L.q; f.up_inflow = L.inflow; }
    else { f.qup = R.q; f.up_inflow = R.inflow; }
    return s;
}

__device__ __forceinline__ double face_sed(const DevParams &P, const double *__restrict__ src, const Face &f,
                                           int k, double sedin)
{
    if (f.up_inflow) return sedin;
    return sed_of(src[(P_FIXED + k) * P.plane + f.qup], src[P_H * P.plane + f.qup], P.hfilm);
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_down_sync(0xffffffffu, v, o);
        v = (w > v) ? w : v;
    }
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace swehr
