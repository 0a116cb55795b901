// po_device.cuh — device-side data layout and math of the PO diffraction
// kernels (sm_100a).
//
// The physics follows MBS-fast's HandlerPO path:
//   aperture integral   reference src/cuda/GpuDiffraction.cu:876-1062,
//                       CPU twin src/handler/HandlerPO.cpp:2655-2739
//   Jones rotation      GpuDiffraction.cu:816-856 (no 0.5: the Mueller weight
//                       carries 0.25, GpuDiffraction.cu:2319-2329)
//   Jones -> Mueller    GpuDiffraction.cu:1645-1739, src/math/Mueller.hpp:37-87
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mbs {

constexpr int kMaxNv = 31;              // BeamEdgeData::MAX_EDGES - 1 (Handler.h:374)
constexpr double kSmallPhase = 1e-3;    // HandlerPO_fast.h:170
constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kInvTwoPi = 0.15915494309189533576888376337251;

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
    double sp_thr2;      // small-phase prefilter on A^2+B^2 (see pack kernel)
    int32_t vbeg;        // first vertex
    int32_t nv;
    int32_t flags;       // MBS_PO_BEAM_EXTERNAL
    int32_t pad;
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

__device__ __forceinline__ void sincos_fp64(double x, double *s, double *c)
{
    sincos(x, s, c);
}

// HandlerPO_fast.h:228-237 / GpuDiffraction.cu:940-949.
__device__ __forceinline__ double stable_sinc(double x)
{
    if (fabs(x) < 1e-4) {
        const double x2 = x * x;
        return 1.0 - x2 / 6.0 + x2 * x2 / 120.0;
    }
    return sin(x) / x;
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
__device__ __forceinline__ bool small_phase_factor(const double *vx, const double *vy,
                                                   int stride, int nv, double A, double B,
                                                   double k, double &fr, double &fi)
{
    if (nv < 3)
        return false;
    const double qx = k * A, qy = k * B;
    for (int i = 0; i < nv; ++i)
        if (fabs(qx * vx[i * stride] + qy * vy[i * stride]) > kSmallPhase)
            return false;
    double twiceArea = 0, fx6 = 0, fy6 = 0, sx12 = 0, sy12 = 0, sxy24 = 0;
    double minX = 1.7976931348623157e308, maxX = -1.7976931348623157e308;
    double minY = minX, maxY = maxX;
    for (int i = 0; i < nv; ++i) {
        const int j = (i + 1 < nv) ? i + 1 : 0;
        const double xi = vx[i * stride], yi = vy[i * stride];
        const double xj = vx[j * stride], yj = vy[j * stride];
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

// Jones -> Mueller times weight, added into out[16] (Mueller.hpp:37-87).
template <typename T>
__device__ __forceinline__ void mueller_add(const T *j, T weight, T *out)
{
    const T j00r = j[0], j00i = j[1], j01r = j[2], j01i = j[3];
    const T j10r = j[4], j10i = j[5], j11r = j[6], j11i = j[7];
    const T a11 = j00r * j00r + j00i * j00i, a12 = j01r * j01r + j01i * j01i;
    const T a21 = j10r * j10r + j10i * j10i, a22 = j11r * j11r + j11i * j11i;
    const T half = T(0.5);
    T A1 = a11 + a21, A2 = a12 + a22;
    out[0] += ((A1 + A2) * half) * weight;
    out[1] += ((A1 - A2) * half) * weight;
    A1 = a11 - a21; A2 = a12 - a22;
    out[4] += ((A1 + A2) * half) * weight;
    out[5] += ((A1 - A2) * half) * weight;
    T c1r = j00r * j01r + j00i * j01i, c1i = j00i * j01r - j00r * j01i;
    T c2r = j11r * j10r + j11i * j10i, c2i = j11i * j10r - j11r * j10i;
    out[2] += (-c1r - c2r) * weight;
    out[3] += (c2i - c1i) * weight;
    out[6] += (c2r - c1r) * weight;
    out[7] += (-c1i - c2i) * weight;
    c1r = j00r * j10r + j00i * j10i; c1i = j00i * j10r - j00r * j10i;
    c2r = j11r * j01r + j11i * j01i; c2i = j11i * j01r - j11r * j01i;
    out[8] += (-c1r - c2r) * weight;
    out[9] += (c2r - c1r) * weight;
    out[12] += (c1i - c2i) * weight;
    out[13] += (c2i + c1i) * weight;
    c1r = j00r * j11r + j00i * j11i; c1i = j00i * j11r - j00r * j11i;
    c2r = j01r * j10r + j01i * j10i; c2i = j01i * j10r - j01r * j10i;
    out[10] += (c1r + c2r) * weight;
    out[11] += (c1i - c2i) * weight;
    out[14] += (-c1i - c2i) * weight;
    out[15] += (c1r - c2r) * weight;
}

}  // namespace mbs
