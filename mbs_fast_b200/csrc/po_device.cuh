// po_device.cuh — device-side data layout and math of the PO diffraction
// kernels (sm_100a).
//
// The physics follows MBS-fast's HandlerPO path:
//   aperture integral   reference src/cuda/GpuDiffraction.cu:876-1062,
//                       CPU twin src/handler/HandlerPO.cpp:2655-2739
//   Jones rotation      GpuDiffraction.cu:816-856 (no 0.5: the Mueller weight
//                       carries 0.25, GpuDiffraction.cu:2319-2329)
//   Jones -> Mueller    GpuDiffraction.cu:1645-1739, src/math/Mueller.hpp:37-87
//
// Phases are carried in turns (radians / 2 pi) in FP64.  Range reduction is
// exact in FP64: adding 1.5*2^52 to 4u rounds it to the nearest integer n
// (quadrant n mod 4) and u - n/4 is exact (Sterbenz), so the reduced
// argument's only error is the FP64 rounding of the phase itself.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mbs {

constexpr int kMaxNv = 31;              // BeamEdgeData::MAX_EDGES - 1 (Handler.h:374)
constexpr double kSmallPhase = 1e-3;    // HandlerPO_fast.h:170
constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kPi = 3.14159265358979323846264338327950;
constexpr double kInvTwoPi = 0.15915494309189533576888376337251;
constexpr double kMagic52 = 6755399441055744.0;   // 1.5 * 2^52
constexpr double kMagic29 = 805306368.0;          // 1.5 * 2^29 (ulp 2^-23)

// Device copy of one prepared beam (PreparedBeam, HandlerPO.h:14-47), in a
// fixed 288-byte record.  Built by the pack kernel from mbs_po_beams.
struct __align__(16) DevBeam {
    double a0, b0;       // bd.hor, bd.ver (GpuDiffraction.cu:301-302)
    double h[3];         // aperture horizontal axis
    double v[3];         // aperture vertical axis
    double c[3];         // beam centre
    double area;
    double rot[12];      // NT, NP, nxDT, nxDP
    double jp[8];        // J_phased
    double opath;        // origBeam.opticalPath (extinction phase reference)
    double sp_thr2;      // small-phase prefilter on A^2+B^2 (pack kernel)
    int32_t vbeg;        // first vertex
    int32_t nv;
    int32_t flags;       // MBS_PO_BEAM_EXTERNAL
    float   near2;       // FP32 near-forward zone on A^2+B^2 (pack kernel)
};
static_assert(sizeof(DevBeam) == 288, "DevBeam layout");

// One polygon vertex; a NaN slope marks an edge that is invalid for that
// branch (BeamEdgeData::edge_valid_x / edge_valid_y).
struct __align__(16) DevVert {
    double x, y, syx, sxy;
};
static_assert(sizeof(DevVert) == 32, "DevVert layout");

struct WaveConst {
    double k;             // wave index
    double cw_re, cw_im;  // complWave
    double icw_re, icw_im;// invComplWave
    double eps1;
    double eps1_f32;      // max(eps1, 3e-5): FP32 singular-edge threshold
    double wavelength;
    double ot_far_ref, ot_ping;
    int legacy_sign;
    int ot_phase_avg;
};

// ---------------------------------------------------------------- FP64 math

// sin and cos of 2*pi*u.  Exact quadrant reduction (see file header), then
// Taylor polynomials of sin (to x^17) and cos (to x^16) on |x| <= pi/4,
// whose truncation error is below 1e-17.  Coefficients are 1/n! rounded to
// double.
__device__ __forceinline__ void sincos_turns(double u, double &s, double &c)
{
    const double t = fma(u, 4.0, kMagic52);
    const double n = t - kMagic52;
    const int q = __double2loint(t) & 3;
    const double x = fma(n, -0.25, u) * kTwoPi;
    const double x2 = x * x;
    double ps = 2.8114572543455206e-15;          // 1/17!
    ps = fma(ps, x2, -7.6471637318198164e-13);   // -1/15!
    ps = fma(ps, x2, 1.6059043836821613e-10);    // 1/13!
    ps = fma(ps, x2, -2.5052108385441720e-08);   // -1/11!
    ps = fma(ps, x2, 2.7557319223985893e-06);    // 1/9!
    ps = fma(ps, x2, -1.9841269841269841e-04);   // -1/7!
    ps = fma(ps, x2, 8.3333333333333333e-03);    // 1/5!
    ps = fma(ps, x2, -1.6666666666666666e-01);   // -1/3!
    const double sx = fma(x * x2, ps, x);
    double pc = 4.7794773323873853e-14;          // 1/16!
    pc = fma(pc, x2, -1.1470745597729725e-11);   // -1/14!
    pc = fma(pc, x2, 2.0876756987868099e-09);    // 1/12!
    pc = fma(pc, x2, -2.7557319223985888e-07);   // -1/10!
    pc = fma(pc, x2, 2.4801587301587302e-05);    // 1/8!
    pc = fma(pc, x2, -1.3888888888888889e-03);   // -1/6!
    pc = fma(pc, x2, 4.1666666666666664e-02);    // 1/4!
    pc = fma(pc, x2, -0.5);                      // -1/2!
    const double cx = fma(x2, pc, 1.0);
    const double ss = (q & 1) ? cx : sx;
    const double cc = (q & 1) ? sx : cx;
    s = (q & 2) ? -ss : ss;
    c = ((q + 1) & 2) ? -cc : cc;
}

// sin and cos of 2*pi*u from a table of the 128 angles 2*pi*k/128 (tab[k] =
// (sin, cos), filled by sincos_turns): u = k/128 + r exactly (|r| <= 1/256
// turn, the reduction is exact as in sincos_turns), then the angle-addition
// formulas with the Taylor polynomials of sin(2 pi r) (to r^7) and cos(2 pi r)
// (to r^6) in r itself (coefficients (2 pi)^n / n!, rounded to double), whose
// truncation errors are below 1e-20 and 4e-18.  15 FP64 operations and one
// shared-memory load against about 22 operations and 8 selects of the
// quadrant form.
__device__ __forceinline__ void sincos_turns_tab(double u, const double2 *tab, double &s, double &c)
{
    const double t = fma(u, 128.0, kMagic52);
    const double n = t - kMagic52;
    const int k = __double2loint(t) & 127;
    const double r = fma(n, -0.0078125, u);          // exact, |r| <= 1/256 turn
    const double r2 = r * r;
    double ps = -76.70585975306139;                  // -(2 pi)^7 / 7!
    ps = fma(ps, r2, 81.60524927607506);             //  (2 pi)^5 / 5!
    ps = fma(ps, r2, -41.34170224039976);            // -(2 pi)^3 / 3!
    ps = fma(ps, r2, 6.283185307179586);             //   2 pi
    const double sx = r * ps;                        // sin(2 pi r)
    double pc = -85.45681720669373;                  // -(2 pi)^6 / 6!
    pc = fma(pc, r2, 64.9393940226683);              //  (2 pi)^4 / 4!
    pc = fma(pc, r2, -19.739208802178716);           // -(2 pi)^2 / 2!
    const double cx = fma(r2, pc, 1.0);              // cos(2 pi r)
    const double2 sc = tab[k];
    s = fma(sc.x, cx, sc.y * sx);
    c = fma(sc.y, cx, -(sc.x * sx));
}

__device__ __forceinline__ void sincos_rad(double x, double &s, double &c)
{
    sincos_turns(x * kInvTwoPi, s, c);
}

// Reciprocal: hardware approximation refined by one Newton step.
__device__ __forceinline__ double rcp64(double x)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    const double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    const double e2 = fma(-x, r, 1.0);
    return fma(r, e2, r);
}

__device__ __forceinline__ float rcp32(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// sin(x)/x (HandlerPO_fast.h:228-237 / GpuDiffraction.cu:940-949, which use
// the series through x^4 below |x| = 1e-4).  Below |x| = 0.1 the Taylor
// series through x^8 is exact to double rounding (the first omitted term,
// x^10/11!, is below 3e-18), which covers the nearly singular edges of the
// rare pass (|x| <= k eps |delta|, a few 1e-2 at most for FP32C thresholds)
// without a sine, a cosine and a division in FP64.
__device__ __forceinline__ double stable_sinc(double x)
{
    const double x2 = x * x;
    if (x2 < 1e-2) {
        double p = 1.0 / 362880.0;     //  1/9!
        p = fma(p, x2, -1.0 / 5040.0);  // -1/7!
        p = fma(p, x2, 1.0 / 120.0);    //  1/5!
        p = fma(p, x2, -1.0 / 6.0);     // -1/3!
        return fma(p, x2, 1.0);
    }
    double s, c;
    sincos_rad(x, s, c);
    return s / x;
}

// exp(i*phaseStart)*(exp(i*k*c*delta)-1)/c in half-angle form for a nearly
// zero edge coefficient (HandlerPO_fast.h:242-257, GpuDiffraction.cu:951-970).
__device__ __forceinline__ void stable_edge(double pr, double pi, double delta,
                                            double c, double k,
                                            double &sr, double &si)
{
    const double z = k * c * delta;
    const double sh = stable_sinc(0.5 * z);
    const double lr = -0.5 * k * k * c * delta * delta * sh * sh;
    const double li = k * delta * stable_sinc(z);
    sr += pr * lr - pi * li;
    si += pr * li + pi * lr;
}

// Second-order polygon-moment factor for a small phase span
// (HandlerPO_fast.h:161-226, GpuDiffraction.cu:876-938).  Returns false when
// some vertex phase exceeds 1e-3.
__device__ __forceinline__ bool small_phase_factor(const DevVert *v, int nv, double A, double B,
                                                   double k, double &fr, double &fi)
{
    if (nv < 3)
        return false;
    const double qx = k * A, qy = k * B;
    for (int i = 0; i < nv; ++i)
        if (fabs(qx * v[i].x + qy * v[i].y) > kSmallPhase)
            return false;
    double twiceArea = 0, fx6 = 0, fy6 = 0, sx12 = 0, sy12 = 0, sxy24 = 0;
    double minX = 1.7976931348623157e308, maxX = -1.7976931348623157e308;
    double minY = minX, maxY = maxX;
    for (int i = 0; i < nv; ++i) {
        const int j = (i + 1 < nv) ? i + 1 : 0;
        const double xi = v[i].x, yi = v[i].y;
        const double xj = v[j].x, yj = v[j].y;
        const double cross = xi * yj - xj * yi;
        twiceArea += cross;
        fx6 += (xi + xj) * cross;
        fy6 += (yi + yj) * cross;
        sx12 += (xi * xi + xi * xj + xj * xj) * cross;
        sy12 += (yi * yi + yi * yj + yj * yj) * cross;
        sxy24 += (2.0 * xi * yi + xi * yj + xj * yi + 2.0 * xj * yj) * cross;
        minX = fmin(minX, xi); maxX = fmax(maxX, xi);
        minY = fmin(minY, yi); maxY = fmax(maxY, yi);
    }
    const double areaScale = fmax((maxX - minX) * (maxY - minY), 2.2250738585072014e-308);
    if (fabs(twiceArea) <= 0x1p-40 * areaScale) {
        fr = 1.0;
        fi = 0.0;
        return true;
    }
    const double invArea = 2.0 / twiceArea;
    const double mX = (fx6 / 6.0) * invArea, mY = (fy6 / 6.0) * invArea;
    const double mXX = (sx12 / 12.0) * invArea, mYY = (sy12 / 12.0) * invArea;
    const double mXY = (sxy24 / 24.0) * invArea;
    const double mp = qx * mX + qy * mY;
    const double mp2 = qx * qx * mXX + 2.0 * qx * qy * mXY + qy * qy * mYY;
    fr = 1.0 - 0.5 * mp2;
    fi = mp;
    return true;
}

// ---------------------------------------------------------- Jones -> Mueller

// Jones -> Mueller times weight, added into out[16] (Mueller.hpp:37-87).
template <typename T>
__device__ __forceinline__ void mueller_add(const T *j, T weight, T *out, int stride = 1)
{
    const T j00r = j[0], j00i = j[1], j01r = j[2], j01i = j[3];
    const T j10r = j[4], j10i = j[5], j11r = j[6], j11i = j[7];
    const T a11 = j00r * j00r + j00i * j00i, a12 = j01r * j01r + j01i * j01i;
    const T a21 = j10r * j10r + j10i * j10i, a22 = j11r * j11r + j11i * j11i;
    const T half = T(0.5);
    T A1 = a11 + a21, A2 = a12 + a22;
    out[0 * stride] += ((A1 + A2) * half) * weight;
    out[1 * stride] += ((A1 - A2) * half) * weight;
    A1 = a11 - a21; A2 = a12 - a22;
    out[4 * stride] += ((A1 + A2) * half) * weight;
    out[5 * stride] += ((A1 - A2) * half) * weight;
    T c1r = j00r * j01r + j00i * j01i, c1i = j00i * j01r - j00r * j01i;
    T c2r = j11r * j10r + j11i * j10i, c2i = j11i * j10r - j11r * j10i;
    out[2 * stride] += (-c1r - c2r) * weight;
    out[3 * stride] += (c2i - c1i) * weight;
    out[6 * stride] += (c2r - c1r) * weight;
    out[7 * stride] += (-c1i - c2i) * weight;
    c1r = j00r * j10r + j00i * j10i; c1i = j00i * j10r - j00r * j10i;
    c2r = j11r * j01r + j11i * j01i; c2i = j11i * j01r - j11r * j01i;
    out[8 * stride] += (-c1r - c2r) * weight;
    out[9 * stride] += (c2r - c1r) * weight;
    out[12 * stride] += (c1i - c2i) * weight;
    out[13 * stride] += (c2i + c1i) * weight;
    c1r = j00r * j11r + j00i * j11i; c1i = j00i * j11r - j00r * j11i;
    c2r = j01r * j10r + j01i * j10i; c2i = j01i * j10r - j01r * j10i;
    out[10 * stride] += (c1r + c2r) * weight;
    out[11 * stride] += (c1i - c2i) * weight;
    out[14 * stride] += (-c1i - c2i) * weight;
    out[15 * stride] += (c1r - c2r) * weight;
}

}  // namespace mbs
