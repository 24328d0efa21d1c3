// xm_math.cuh -- FP64 arithmetic shared by the zone builder and the pair
// kernels.  Every operation is an explicitly rounded IEEE operation
// (__dmul_rn / __dadd_rn / __fma_rn on the device, which the compiler never
// contracts), so the unit vectors and chord lengths are the same bits on
// every run and equal to a host evaluation of the same formulas with
// -ffp-contract=off.
//
// sincos: Cody & Waite (1980) reduction by pi/2 split into three doubles,
// then truncated Taylor series on |r| <= pi/4 (sin to r^17, cos to r^18).
// The constants are the doubles nearest to pi/2 (three-way split), 2/pi and
// (-1)^k/n!; gen_sincos_consts.py derives them from Machin's formula and
// exact rationals.  Error <= 1 ulp against a correctly rounded sin/cos on
// |x| <= 8.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define XM_RAD2DEG 57.295779513082323   // Common.h:9 (degrees per radian)
#define XM_TWO_PI 6.2831853071795864769252867665590057683943387987502116419498  // Worker.cu:23

#define XM_PIO2_1 0x1.921fb54442d18p+0
#define XM_PIO2_2 0x1.1a62633145c07p-54
#define XM_PIO2_3 -0x1.f1976b7ed8fbcp-110
#define XM_2_OVER_PI 0x1.45f306dc9c883p-1
#define XM_S1 -0x1.5555555555555p-3
#define XM_S2 0x1.1111111111111p-7
#define XM_S3 -0x1.a01a01a01a01ap-13
#define XM_S4 0x1.71de3a556c734p-19
#define XM_S5 -0x1.ae64567f544e4p-26
#define XM_S6 0x1.6124613a86d09p-33
#define XM_S7 -0x1.ae7f3e733b81fp-41
#define XM_S8 0x1.952c77030ad4ap-49
#define XM_C1 -0x1.0000000000000p-1
#define XM_C2 0x1.5555555555555p-5
#define XM_C3 -0x1.6c16c16c16c17p-10
#define XM_C4 0x1.a01a01a01a01ap-16
#define XM_C5 -0x1.27e4fb7789f5cp-22
#define XM_C6 0x1.1eed8eff8d898p-29
#define XM_C7 -0x1.93974a8c07c9dp-37
#define XM_C8 0x1.ae7f3e733b81fp-45
#define XM_C9 -0x1.6827863b97d97p-53

namespace xm {

__device__ __forceinline__ void sincos_p(double x, double *s, double *c)
{
    double kd = rint(__dmul_rn(x, XM_2_OVER_PI));
    double r = __fma_rn(-kd, XM_PIO2_1, x);
    r = __fma_rn(-kd, XM_PIO2_2, r);
    r = __fma_rn(-kd, XM_PIO2_3, r);
    double r2 = __dmul_rn(r, r);
    double ps = XM_S8;
    ps = __fma_rn(ps, r2, XM_S7);
    ps = __fma_rn(ps, r2, XM_S6);
    ps = __fma_rn(ps, r2, XM_S5);
    ps = __fma_rn(ps, r2, XM_S4);
    ps = __fma_rn(ps, r2, XM_S3);
    ps = __fma_rn(ps, r2, XM_S2);
    ps = __fma_rn(ps, r2, XM_S1);
    double r3 = __dmul_rn(r2, r);
    double sn = __fma_rn(r3, ps, r);
    double pc = XM_C9;
    pc = __fma_rn(pc, r2, XM_C8);
    pc = __fma_rn(pc, r2, XM_C7);
    pc = __fma_rn(pc, r2, XM_C6);
    pc = __fma_rn(pc, r2, XM_C5);
    pc = __fma_rn(pc, r2, XM_C4);
    pc = __fma_rn(pc, r2, XM_C3);
    pc = __fma_rn(pc, r2, XM_C2);
    pc = __fma_rn(pc, r2, XM_C1);
    double cs = __fma_rn(r2, pc, 1.0);
    int q = (int)((long long)kd & 3);
    double ss = (q & 1) ? cs : sn;
    double cc = (q & 1) ? sn : cs;
    *s = (q == 2 || q == 3) ? -ss : ss;
    *c = (q == 1 || q == 2) ? -cc : cc;
}

// Unit vector of (ra, dec) in radians: (cd cr, cd sr, sd) -- Worker.cu:31-40.
__device__ __forceinline__ void radec2xyz(double ra, double dec, double &x, double &y, double &z)
{
    double sr, cr, sd, cd;
    sincos_p(ra, &sr, &cr);
    sincos_p(dec, &sd, &cd);
    x = __dmul_rn(cd, cr);
    y = __dmul_rn(cd, sr);
    z = sd;
}

// Squared chord, evaluated as (dx*dx + dy*dy) + dz*dz (Worker.cu:93-96).
__device__ __forceinline__ double chord2(double x1, double y1, double z1, double x2, double y2,
                                         double z2)
{
    double dx = __dsub_rn(x1, x2), dy = __dsub_rn(y1, y2), dz = __dsub_rn(z1, z2);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Zone id floor((dec + 90) / zh) (Sorter.cu:20-24); -1 if dropped.  dec = +90
// landing on n_zones is kept in the last zone.
__device__ __forceinline__ int zone_of(double dec_deg, double zh_deg, int n_zones)
{
    double zd = floor(__ddiv_rn(__dadd_rn(dec_deg, 90.0), zh_deg));
    if (!(zd >= 0.0)) return -1;
    if (zd >= (double)n_zones) {
        if (zd == (double)n_zones && dec_deg <= 90.0) return n_zones - 1;
        return -1;
    }
    return (int)zd;
}

// Quantised ra: floor(ra_rad * 2^31 / pi), i.e. 2^32 steps per turn, clamped
// to [0, 2^32 - 1] (NaN and negative values map to 0).  Monotone in ra.
#define XM_RAQ_SCALE 0x1.45f306dc9c883p+29
__device__ __forceinline__ uint32_t raq32(double ra_rad)
{
    const double x = floor(__dmul_rn(ra_rad, XM_RAQ_SCALE));
    if (!(x > 0.0)) return 0u;
    if (x >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)x;
}

// Order-preserving map of a double to uint64 (negative values flipped).
__device__ __forceinline__ unsigned long long order_key(double v)
{
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

}  // namespace xm
