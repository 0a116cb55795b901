// po_b200.cu — B200 (sm_100a) kernels and C ABI of the PO diffraction library.
//
// Data path of one call (replaces HandlerPO::HandleOrientationsToLocalGpu,
// reference src/cuda/GpuDiffraction.cu:4159-4778):
//   1. stage:    flat mbs_po_beams arrays -> HBM (one cudaMemcpyAsync each),
//                then po_pack_kernel builds fixed DevBeam/DevVert records.
//   2. diffract: po_diffract_kernel<Prec,NS>, one CTA per (azimuth bin,
//                zenith tile, orientation chunk).  Each thread owns one
//                direction and accumulates the coherent Jones sum over the
//                orientation's beams (staged per azimuth in shared memory),
//                converts it to Mueller and accumulates the orientation
//                average in registers.  No atomics: each chunk writes its own
//                partial Mueller plane.
//   3. reduce:   po_reduce_kernel adds the chunk partials in a fixed order
//                into the caller's accumulator (deterministic).
#include "mbs_po_b200.h"
#include "po_device.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace mbs;

namespace {

// ------------------------------------------------------------ parameters ---

constexpr int kStageBeams = 64;     // beams per shared-memory stage
constexpr int kStageVerts = 512;    // vertices per shared-memory stage

struct GridDev {
    int n_az = 0, n_zen = 0;
    double *st = nullptr, *ct = nullptr;      // [n_zen+1]
    double *sphi = nullptr, *cphi = nullptr;  // [n_az]
    double *vf = nullptr;                     // [n_az*(n_zen+1)*3]
};

struct KParams {
    const DevBeam *beams;
    const DevVert *verts;
    const int32_t *vbeg;       // [n_beams+1]
    const int32_t *beam_off;   // [n_orient+1]
    const double *weight;      // [n_orient]
    const double *st, *ct, *sphi, *cphi, *vf;
    int n_az, n_t;             // n_t = n_zen+1
    int n_orient;
    int orient_per_chunk;
    int tile;                  // directions per CTA (== blockDim.x)
    int tiles_per_row;
    WaveConst wc;
    double *partial;           // [n_chunks][16][G]
    double *partial_ns;        // [n_chunks][16][G] or null
};

// ------------------------------------------------------------ pack kernel --

struct PackParams {
    int64_t n_beams;
    const int64_t *vert_off;
    const double *vx, *vy, *syx, *sxy;
    const uint8_t *eflags;
    const double *geom;
    const uint8_t *bflags;
    double k;
    DevBeam *beams;
    DevVert *verts;
    int32_t *vbeg;
    int *status;   // set to 1 on a malformed beam
};

__global__ void po_pack_kernel(PackParams P)
{
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b > P.n_beams)
        return;
    const int64_t v0 = P.vert_off[b];
    P.vbeg[b] = (int32_t)v0;
    if (b == P.n_beams)
        return;
    const int nv = (int)(P.vert_off[b + 1] - v0);
    if (nv < 3 || nv > kMaxNv) {
        atomicExch(P.status, 1);
        return;
    }
    const double *g = P.geom + b * MBS_PO_GEOM_STRIDE;
    DevBeam d;
    // a0 = bd.hor, b0 = bd.ver as the reference packs them (GpuDiffraction.cu:301-302)
    d.a0 = g[MBS_PO_G_BD] * g[MBS_PO_G_HOR] + g[MBS_PO_G_BD + 1] * g[MBS_PO_G_HOR + 1]
         + g[MBS_PO_G_BD + 2] * g[MBS_PO_G_HOR + 2];
    d.b0 = g[MBS_PO_G_BD] * g[MBS_PO_G_VER] + g[MBS_PO_G_BD + 1] * g[MBS_PO_G_VER + 1]
         + g[MBS_PO_G_BD + 2] * g[MBS_PO_G_VER + 2];
    for (int i = 0; i < 3; ++i) {
        d.h[i] = g[MBS_PO_G_HOR + i];
        d.v[i] = g[MBS_PO_G_VER + i];
        d.c[i] = g[MBS_PO_G_CEN + i];
    }
    d.area = g[MBS_PO_G_AREA];
    for (int i = 0; i < 12; ++i)
        d.rot[i] = g[MBS_PO_G_NT + i];
    for (int i = 0; i < 8; ++i)
        d.jp[i] = g[MBS_PO_G_JP + i];
    d.opath = g[MBS_PO_G_OPATH];
    d.vbeg = (int32_t)v0;
    d.nv = nv;
    d.flags = P.bflags[b];
    d.pad = 0;
    // Small-phase prefilter.  max_v |q.v| >= |q| * sqrt(lambda_min(S)) with
    // S the second-moment matrix of the vertices, so the moment branch
    // (max_v |k(A x_v + B y_v)| <= 1e-3) is impossible once
    // k^2 (A^2+B^2) lambda_min > 1e-6.
    double sxx = 0, sxy_ = 0, syy = 0;
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int e = 0; e < nv; ++e) {
        const double x = P.vx[v0 + e], y = P.vy[v0 + e];
        sxx += x * x; sxy_ += x * y; syy += y * y;
        DevVert dv;
        dv.x = x;
        dv.y = y;
        const uint8_t f = P.eflags[v0 + e];
        dv.syx = (f & MBS_PO_EDGE_VALID_X) ? P.syx[v0 + e] : nan;
        dv.sxy = (f & MBS_PO_EDGE_VALID_Y) ? P.sxy[v0 + e] : nan;
        P.verts[v0 + e] = dv;
    }
    sxx /= nv; sxy_ /= nv; syy /= nv;
    const double hm = 0.5 * (sxx + syy), hd = 0.5 * (sxx - syy);
    const double lmin = hm - sqrt(hd * hd + sxy_ * sxy_);
    const double kl2 = P.k * P.k * lmin;
    // 0.98 keeps the prefilter conservative against rounding of lmin.
    d.sp_thr2 = (kl2 > 1e-300) ? (kSmallPhase * kSmallPhase) / (0.98 * kl2) : 1.0e300;
    P.beams[b] = d;
}

// ------------------------------------------------------- diffraction kernel

// Shared-memory record of one beam for the CTA's azimuth (the per-azimuth
// coefficients of precompute_theta_coeffs, HandlerPO_fast.h:504-560).
struct __align__(16) SBeam {
    double a_sin, a_cos, a0;   // A(theta) = sin*a_sin + cos*a_cos + a0
    double b_sin, b_cos, b0;
    double cm_sin, cm_cos;     // internal-beam common phase (folded into vertices)
    double area, thr2;
    double rot[12];
    double jp[8];
    float  fa[6];              // FP32 copies of the A/B coefficients
    float  frot[12];
    float  fjp[8];
    float  farea, fthr2;
    int32_t vs;                // first vertex in the stage
    int32_t nv;
    int32_t flags;
    int32_t gbeam;             // global beam index
};

// Per vertex: phase(theta) = sin*ps + cos*pc + p0 (radians for FP64,
// turns for FP32C), slopes (NaN = invalid edge for that branch).
struct __align__(16) SVert {
    double ps, pc, p0;
    double x, y;
    double syx, sxy;
    float fsyx, fsxy;
};

template <int Prec>
struct Acc;

template <>
struct Acc<MBS_PO_FP64> {
    double j[8];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < 8; ++i) j[i] = 0.0;
    }
    __device__ __forceinline__ void add(const double *d) {
#pragma unroll
        for (int i = 0; i < 8; ++i) j[i] += d[i];
    }
    __device__ __forceinline__ void get(double *o) const {
#pragma unroll
        for (int i = 0; i < 8; ++i) o[i] = j[i];
    }
};

// FP32 Jones sums with Kahan compensation.
template <>
struct Acc<MBS_PO_FP32C> {
    float s[8], c[8];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < 8; ++i) { s[i] = 0.f; c[i] = 0.f; }
    }
    __device__ __forceinline__ void add(const float *d) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float y = __fsub_rn(d[i], c[i]);
            const float t = __fadd_rn(s[i], y);
            c[i] = __fsub_rn(__fsub_rn(t, s[i]), y);
            s[i] = t;
        }
    }
    __device__ __forceinline__ void get(double *o) const {
#pragma unroll
        for (int i = 0; i < 8; ++i) o[i] = (double)s[i] - (double)c[i];
    }
};

// Per-thread direction constants.
struct DirCtx {
    double st, ct, cp, sp;
    double dir[3], vf[3], vt[3], w[3], u[3];
};

__device__ __forceinline__ void cross3(const double *a, const double *b, double *o)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// Rotation of the beam's Jones matrix into the scattering basis
// (GpuDiffraction.cu:831-856), rewritten with the per-direction vectors
// w = vt x dir and u = vf x dir:  (dir x NT).vt = NT.w, (dir x NT).vf = NT.u;
// the dir(dir.nxDT) terms vanish because vt and vf are orthogonal to dir.
template <typename T>
__device__ __forceinline__ void rotation(const T *rot, const T *w, const T *u,
                                         const T *vt, const T *vf, T *r)
{
    const T *NT = rot, *NP = rot + 3, *DT = rot + 6, *DP = rot + 9;
    r[0] = NT[0] * w[0] + NT[1] * w[1] + NT[2] * w[2] + DT[0] * vt[0] + DT[1] * vt[1] + DT[2] * vt[2];
    r[1] = NP[0] * w[0] + NP[1] * w[1] + NP[2] * w[2] + DP[0] * vt[0] + DP[1] * vt[1] + DP[2] * vt[2];
    r[2] = NT[0] * u[0] + NT[1] * u[1] + NT[2] * u[2] + DT[0] * vf[0] + DT[1] * vf[1] + DT[2] * vf[2];
    r[3] = NP[0] * u[0] + NP[1] * u[1] + NP[2] * u[2] + DP[0] * vf[0] + DP[1] * vf[1] + DP[2] * vf[2];
}

// d = (F R) x J_phased (GpuDiffraction.cu:1149-1164).
template <typename T>
__device__ __forceinline__ void jones_product(T fr, T fi, const T *r, const T *jp, T *d)
{
    const T s00r = fr * r[0], s00i = fi * r[0];
    const T s01r = fr * r[1], s01i = fi * r[1];
    const T s10r = fr * r[2], s10i = fi * r[2];
    const T s11r = fr * r[3], s11i = fi * r[3];
    d[0] = s00r * jp[0] - s00i * jp[1] + s01r * jp[4] - s01i * jp[5];
    d[1] = s00r * jp[1] + s00i * jp[0] + s01r * jp[5] + s01i * jp[4];
    d[2] = s00r * jp[2] - s00i * jp[3] + s01r * jp[6] - s01i * jp[7];
    d[3] = s00r * jp[3] + s00i * jp[2] + s01r * jp[7] + s01i * jp[6];
    d[4] = s10r * jp[0] - s10i * jp[1] + s11r * jp[4] - s11i * jp[5];
    d[5] = s10r * jp[1] + s10i * jp[0] + s11r * jp[5] + s11i * jp[4];
    d[6] = s10r * jp[2] - s10i * jp[3] + s11r * jp[6] - s11i * jp[7];
    d[7] = s10r * jp[3] + s10i * jp[2] + s11r * jp[7] + s11i * jp[6];
}

// Moment branch in FP64 from the global records (rare).  Returns false when
// the exact test rejects the small-phase branch.
__device__ bool small_phase_fp64(const DevBeam &gb, const DevVert *gv, const DirCtx &dc,
                                 const WaveConst &wc, double &fr, double &fi)
{
    const double a_sin = -dc.cp * gb.h[0] - dc.sp * gb.h[1];
    const double b_sin = -dc.cp * gb.v[0] - dc.sp * gb.v[1];
    const double A = dc.st * a_sin + dc.ct * gb.h[2] + gb.a0;
    const double B = dc.st * b_sin + dc.ct * gb.v[2] + gb.b0;
    double pr, pi;
    if (!small_phase_factor(&gv[gb.vbeg].x, &gv[gb.vbeg].y, 4, gb.nv, A, B, wc.k, pr, pi))
        return false;
    const double sgn = wc.legacy_sign ? 1.0 : -1.0;
    const double ar = sgn * wc.icw_re * gb.area, ai = sgn * wc.icw_im * gb.area;
    fr = ar * pr - ai * pi;
    fi = ar * pi + ai * pr;
    if (!(gb.flags & MBS_PO_BEAM_EXTERNAL)) {
        // common internal-beam phase (GpuDiffraction.cu:1106-1143)
        const double cm = -wc.k * (dc.st * (dc.cp * gb.c[0] + dc.sp * gb.c[1]) + dc.ct * (-gb.c[2]));
        double s, c;
        sincos_fp64(cm, &s, &c);
        const double tr = fr * c - fi * s;
        fi = fr * s + fi * c;
        fr = tr;
    }
    return true;
}

// FP64 contribution of one beam to one direction.
__device__ __forceinline__ bool beam_fp64(const SBeam &b, const SVert *sv, const DevBeam *gbeams,
                                          const DevVert *gverts, const DirCtx &dc,
                                          const WaveConst &wc, double *d)
{
    const double A = fma(dc.st, b.a_sin, fma(dc.ct, b.a_cos, b.a0));
    const double B = fma(dc.st, b.b_sin, fma(dc.ct, b.b_cos, b.b0));
    double fr, fi;
    bool done = false;
    if (A * A + B * B <= b.thr2)
        done = small_phase_fp64(gbeams[b.gbeam], gverts, dc, wc, fr, fi);
    if (!done) {
        const bool useX = fabs(B) > fabs(A);
        const double al = useX ? A : B, be = useX ? B : A;
        const SVert *v = sv + b.vs;
        const int nv = b.nv;
        double s0, c0;
        sincos_fp64(fma(dc.st, v[0].ps, fma(dc.ct, v[0].pc, v[0].p0)), &s0, &c0);
        double cprev = c0, sprev = s0, sr = 0.0, si = 0.0;
        for (int e = 0; e < nv; ++e) {
            const int en = (e + 1 < nv) ? e + 1 : 0;
            double cn = c0, sn = s0;
            if (en != 0)
                sincos_fp64(fma(dc.st, v[en].ps, fma(dc.ct, v[en].pc, v[en].p0)), &sn, &cn);
            const double s = useX ? v[e].syx : v[e].sxy;
            if (s == s) {
                const double coef = fma(s, be, al);   // A + s*B  or  A*s + B
                const double ac = fabs(coef);
                const double inv = (ac > wc.eps1) ? 1.0 / coef : 0.0;
                sr = fma(cn - cprev, inv, sr);
                si = fma(sn - sprev, inv, si);
                if (ac <= wc.eps1) {
                    const double delta = useX ? (v[en].x - v[e].x) : (v[en].y - v[e].y);
                    stable_edge(cprev, sprev, delta, coef, wc.k, sr, si);
                }
            }
            cprev = cn;
            sprev = sn;
        }
        const double m = useX ? 1.0 / B : -1.0 / A;
        sr *= m;
        si *= m;
        fr = wc.cw_re * sr - wc.cw_im * si;
        fi = wc.cw_re * si + wc.cw_im * sr;
    }
    if (isnan(fr))
        return false;
    double r[4];
    rotation(b.rot, dc.w, dc.u, dc.vt, dc.vf, r);
    jones_product(fr, fi, r, b.jp, d);
    return true;
}

// Fraction of the phase u (in turns) as a float in [-0.5, 0.5): adding
// 1.5*2^29 leaves frac(u) rounded to 2^-23 in the low 23 mantissa bits.
__device__ __forceinline__ float turn_fraction(double u)
{
    const double t = u + 805306368.0;
    const unsigned lo = (unsigned)__double2loint(t);
    float f = __int_as_float(0x3F800000u | (lo & 0x007FFFFFu)) - 1.0f;
    return f >= 0.5f ? f - 1.0f : f;
}

__device__ __forceinline__ void phasor_f32(double u, float &s, float &c)
{
    __sincosf(turn_fraction(u) * 6.28318530717958647f, &s, &c);
}

// FP32C contribution of one beam to one direction.
__device__ __forceinline__ bool beam_fp32c(const SBeam &b, const SVert *sv, const DevBeam *gbeams,
                                           const DevVert *gverts, const DirCtx &dc,
                                           const float *fdir, const WaveConst &wc, float *d)
{
    const float st = fdir[0], ct = fdir[1];
    const float A = fmaf(st, b.fa[0], fmaf(ct, b.fa[1], b.fa[2]));
    const float B = fmaf(st, b.fa[3], fmaf(ct, b.fa[4], b.fa[5]));
    float fr, fi;
    bool done = false;
    if (A * A + B * B <= b.fthr2) {
        double dr, di;
        done = small_phase_fp64(gbeams[b.gbeam], gverts, dc, wc, dr, di);
        fr = (float)dr;
        fi = (float)di;
    }
    if (!done) {
        const bool useX = fabsf(B) > fabsf(A);
        const float al = useX ? A : B, be = useX ? B : A;
        const float eps = (float)wc.eps1_f32;
        const SVert *v = sv + b.vs;
        const int nv = b.nv;
        float s0, c0;
        phasor_f32(fma(dc.st, v[0].ps, fma(dc.ct, v[0].pc, v[0].p0)), s0, c0);
        float cprev = c0, sprev = s0, sr = 0.f, si = 0.f;
        for (int e = 0; e < nv; ++e) {
            const int en = (e + 1 < nv) ? e + 1 : 0;
            float cn = c0, sn = s0;
            if (en != 0)
                phasor_f32(fma(dc.st, v[en].ps, fma(dc.ct, v[en].pc, v[en].p0)), sn, cn);
            const float s = useX ? v[e].fsyx : v[e].fsxy;
            if (s == s) {
                const float coef = fmaf(s, be, al);
                const float ac = fabsf(coef);
                if (ac > eps) {
                    const float inv = __frcp_rn(coef);
                    sr = fmaf(cn - cprev, inv, sr);
                    si = fmaf(sn - sprev, inv, si);
                } else {
                    // near-singular edge: FP64 half-angle form (rare)
                    const DevBeam &gb = gbeams[b.gbeam];
                    const DevVert *gv = gverts + gb.vbeg;
                    const double a_sin = -dc.cp * gb.h[0] - dc.sp * gb.h[1];
                    const double b_sin = -dc.cp * gb.v[0] - dc.sp * gb.v[1];
                    const double Ad = dc.st * a_sin + dc.ct * gb.h[2] + gb.a0;
                    const double Bd = dc.st * b_sin + dc.ct * gb.v[2] + gb.b0;
                    const double sd = useX ? gv[e].syx : gv[e].sxy;
                    const double cd = useX ? fma(sd, Bd, Ad) : fma(sd, Ad, Bd);
                    const double delta = useX ? (gv[en].x - gv[e].x) : (gv[en].y - gv[e].y);
                    double dsr = 0.0, dsi = 0.0;
                    if (fabs(cd) > wc.eps1) {
                        // exact difference quotient from the FP64 phases
                        const double ud0 = fma(dc.st, v[e].ps, fma(dc.ct, v[e].pc, v[e].p0)) * kTwoPi;
                        const double ud1 = fma(dc.st, v[en].ps, fma(dc.ct, v[en].pc, v[en].p0)) * kTwoPi;
                        double s1, c1, s2, c2;
                        sincos_fp64(ud0, &s1, &c1);
                        sincos_fp64(ud1, &s2, &c2);
                        dsr = (c2 - c1) / cd;
                        dsi = (s2 - s1) / cd;
                    } else {
                        stable_edge((double)cprev, (double)sprev, delta, cd, wc.k, dsr, dsi);
                    }
                    sr += (float)dsr;
                    si += (float)dsi;
                }
            }
            cprev = cn;
            sprev = sn;
        }
        const float m = useX ? __frcp_rn(B) : -__frcp_rn(A);
        sr *= m;
        si *= m;
        const float cwr = (float)wc.cw_re, cwi = (float)wc.cw_im;
        fr = cwr * sr - cwi * si;
        fi = cwr * si + cwi * sr;
    }
    if (isnan(fr))
        return false;
    float r[4];
    rotation(b.frot, fdir + 2, fdir + 5, fdir + 8, fdir + 11, r);
    jones_product(fr, fi, r, b.fjp, d);
    return true;
}

template <int Prec, bool NS>
__global__ void __launch_bounds__(128) po_diffract_kernel(KParams P)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SBeam *sb = reinterpret_cast<SBeam *>(smem_raw);
    SVert *sv = reinterpret_cast<SVert *>(smem_raw + kStageBeams * sizeof(SBeam));

    const int p = blockIdx.x / P.tiles_per_row;
    const int tile = blockIdx.x - p * P.tiles_per_row;
    const int t = tile * P.tile + threadIdx.x;
    const bool active = t < P.n_t;
    const int chunk = blockIdx.y;
    const int o0 = chunk * P.orient_per_chunk;
    const int o1 = min(P.n_orient, o0 + P.orient_per_chunk);
    const WaveConst &wc = P.wc;
    const double k = wc.k;
    const double cp = P.cphi[p], sp = P.sphi[p];

    DirCtx dc;
    {
        const int tt = active ? t : P.n_t - 1;
        dc.st = P.st[tt];
        dc.ct = P.ct[tt];
        dc.cp = cp;
        dc.sp = sp;
        dc.dir[0] = dc.st * cp;
        dc.dir[1] = dc.st * sp;
        dc.dir[2] = -dc.ct;
        const double *vfp = P.vf + ((size_t)p * P.n_t + tt) * 3;
        dc.vf[0] = vfp[0]; dc.vf[1] = vfp[1]; dc.vf[2] = vfp[2];
        cross3(dc.vf, dc.dir, dc.u);          // u = vf x dir
        const double l2 = dc.u[0] * dc.u[0] + dc.u[1] * dc.u[1] + dc.u[2] * dc.u[2];
        const double il = (l2 > 1e-30) ? rsqrt(l2) : 1.0;   // transverse_basis_gpu
        dc.vt[0] = dc.u[0] * il; dc.vt[1] = dc.u[1] * il; dc.vt[2] = dc.u[2] * il;
        cross3(dc.vt, dc.dir, dc.w);          // w = vt x dir
    }
    float fdir[14];
    fdir[0] = (float)dc.st;
    fdir[1] = (float)dc.ct;
    for (int i = 0; i < 3; ++i) {
        fdir[2 + i] = (float)dc.w[i];
        fdir[5 + i] = (float)dc.u[i];
        fdir[8 + i] = (float)dc.vt[i];
        fdir[11 + i] = (float)dc.vf[i];
    }

    double M[16], Mns[NS ? 16 : 1];
#pragma unroll
    for (int i = 0; i < 16; ++i) M[i] = 0.0;
    if (NS) {
#pragma unroll
        for (int i = 0; i < (NS ? 16 : 1); ++i) Mns[i] = 0.0;
    }
    const double turn = (Prec == MBS_PO_FP32C) ? kInvTwoPi : 1.0;

    for (int o = o0; o < o1; ++o) {
        Acc<Prec> J, Jn;
        J.zero();
        Jn.zero();
        const int b0 = P.beam_off[o], b1 = P.beam_off[o + 1];
        for (int bs = b0; bs < b1;) {
            // stage [bs, be): at most kStageBeams beams and kStageVerts vertices
            int lo = bs + 1, hi = min(b1, bs + kStageBeams);
            const int vb0 = P.vbeg[bs];
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (P.vbeg[mid] - vb0 <= kStageVerts) lo = mid; else hi = mid - 1;
            }
            const int be = lo;
            const int nb = be - bs;
            for (int i = threadIdx.x; i < nb; i += blockDim.x) {
                const DevBeam &g = P.beams[bs + i];
                SBeam s;
                s.a_sin = -cp * g.h[0] - sp * g.h[1];
                s.a_cos = g.h[2];
                s.a0 = g.a0;
                s.b_sin = -cp * g.v[0] - sp * g.v[1];
                s.b_cos = g.v[2];
                s.b0 = g.b0;
                const bool internal = !(g.flags & MBS_PO_BEAM_EXTERNAL);
                s.cm_sin = internal ? -k * (cp * g.c[0] + sp * g.c[1]) : 0.0;
                s.cm_cos = internal ? -k * (-g.c[2]) : 0.0;
                s.area = g.area;
                s.thr2 = g.sp_thr2;
                for (int q = 0; q < 12; ++q) { s.rot[q] = g.rot[q]; s.frot[q] = (float)g.rot[q]; }
                for (int q = 0; q < 8; ++q) { s.jp[q] = g.jp[q]; s.fjp[q] = (float)g.jp[q]; }
                s.fa[0] = (float)s.a_sin; s.fa[1] = (float)s.a_cos; s.fa[2] = (float)s.a0;
                s.fa[3] = (float)s.b_sin; s.fa[4] = (float)s.b_cos; s.fa[5] = (float)s.b0;
                s.farea = (float)s.area;
                // FP32 prefilter: widen for the rounding of A, B in float.
                s.fthr2 = (float)fmin(4.0 * g.sp_thr2 + 1e-12, 3.0e38);
                s.vs = g.vbeg - vb0;
                s.nv = g.nv;
                s.flags = g.flags;
                s.gbeam = bs + i;
                for (int e = 0; e < g.nv; ++e) {
                    const DevVert gv = P.verts[g.vbeg + e];
                    SVert w;
                    w.ps = (k * (s.a_sin * gv.x + s.b_sin * gv.y) + s.cm_sin) * turn;
                    w.pc = (k * (s.a_cos * gv.x + s.b_cos * gv.y) + s.cm_cos) * turn;
                    w.p0 = (k * (s.a0 * gv.x + s.b0 * gv.y)) * turn;
                    w.x = gv.x;
                    w.y = gv.y;
                    w.syx = gv.syx;
                    w.sxy = gv.sxy;
                    w.fsyx = (float)gv.syx;
                    w.fsxy = (float)gv.sxy;
                    sv[s.vs + e] = w;
                }
                sb[i] = s;
            }
            __syncthreads();
            if (active) {
                for (int j = 0; j < nb; ++j) {
                    const SBeam &b = sb[j];
                    if constexpr (Prec == MBS_PO_FP64) {
                        double d[8];
                        if (beam_fp64(b, sv, P.beams, P.verts, dc, wc, d)) {
                            J.add(d);
                            if (NS && !(b.flags & MBS_PO_BEAM_EXTERNAL))
                                Jn.add(d);
                        }
                    } else {
                        float d[8];
                        if (beam_fp32c(b, sv, P.beams, P.verts, dc, fdir, wc, d)) {
                            J.add(d);
                            if (NS && !(b.flags & MBS_PO_BEAM_EXTERNAL))
                                Jn.add(d);
                        }
                    }
                }
            }
            __syncthreads();
            bs = be;
        }
        if (active) {
            const double wgt = P.weight[o] * 0.25;
            double j[8];
            J.get(j);
            mueller_add(j, wgt, M);
            if (NS) {
                Jn.get(j);
                mueller_add(j, wgt, Mns);
            }
        }
    }
    if (active) {
        const size_t G = (size_t)P.n_az * P.n_t;
        const size_t g = (size_t)p * P.n_t + t;
        double *out = P.partial + (size_t)chunk * 16 * G + g;
#pragma unroll
        for (int i = 0; i < 16; ++i)
            out[i * G] = M[i];
        if (NS) {
            double *outn = P.partial_ns + (size_t)chunk * 16 * G + g;
#pragma unroll
            for (int i = 0; i < (NS ? 16 : 1); ++i)
                outn[i * G] = Mns[i];
        }
    }
}

// out[g*16+k] += sum_c partial[c][k][g], in chunk order.
__global__ void po_reduce_kernel(const double *__restrict__ partial, int n_chunks,
                                 int64_t G, double *__restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G * 16)
        return;
    const int64_t k = i / G, g = i - k * G;
    double s = 0.0;
    for (int c = 0; c < n_chunks; ++c)
        s += partial[(int64_t)c * 16 * G + i];
    out[g * 16 + k] += s;
}

// --------------------------------------------------------- extinction kernel
// One thread per orientation: HandlerPO::ComputeForwardExtinctionOt
// (reference HandlerPO.cpp:1812-2009) at theta = 0, phi = 0.
__global__ void po_extinction_kernel(const DevBeam *beams, const DevVert *verts,
                                     const int32_t *beam_off, const double *weight,
                                     int n_orient, WaveConst wc, double *cext)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n_orient)
        return;
    const double k = wc.k;
    double f00r = 0, f00i = 0, f11r = 0, f11i = 0;
    const double vf[3] = {0.0, 1.0, 0.0}, dir[3] = {0.0, 0.0, -1.0};
    double u[3], vt[3], w[3];
    cross3(vf, dir, u);
    const double l2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const double il = rsqrt(l2);
    vt[0] = u[0] * il; vt[1] = u[1] * il; vt[2] = u[2] * il;
    cross3(vt, dir, w);
    for (int b = beam_off[o]; b < beam_off[o + 1]; ++b) {
        const DevBeam &g = beams[b];
        const bool external = (g.flags & MBS_PO_BEAM_EXTERNAL) != 0;
        if (wc.ot_phase_avg && !external)
            continue;
        const DevVert *v = verts + g.vbeg;
        const int nv = g.nv;
        const double A = 1.0 * g.h[2] + g.a0;
        const double B = 1.0 * g.v[2] + g.b0;
        double fr, fi, pr, pi;
        if (small_phase_factor(&v[0].x, &v[0].y, 4, nv, A, B, k, pr, pi)) {
            const double sgn = wc.legacy_sign ? 1.0 : -1.0;
            const double ar = sgn * wc.icw_re * g.area, ai = sgn * wc.icw_im * g.area;
            fr = ar * pr - ai * pi;
            fi = ar * pi + ai * pr;
        } else {
            const bool useX = fabs(B) > fabs(A);
            double sr = 0, si = 0;
            double c0, s0;
            sincos_fp64(k * (g.h[2] * v[0].x + g.v[2] * v[0].y) + k * (g.a0 * v[0].x + g.b0 * v[0].y), &s0, &c0);
            double cprev = c0, sprev = s0;
            for (int e = 0; e < nv; ++e) {
                const int en = (e + 1 < nv) ? e + 1 : 0;
                double cn = c0, sn = s0;
                if (en != 0)
                    sincos_fp64(k * (g.h[2] * v[en].x + g.v[2] * v[en].y) + k * (g.a0 * v[en].x + g.b0 * v[en].y), &sn, &cn);
                const double s = useX ? v[e].syx : v[e].sxy;
                if (s == s) {
                    const double coef = useX ? A + s * B : A * s + B;
                    const double inv = fabs(coef) > wc.eps1 ? 1.0 / coef : 0.0;
                    sr += (cn - cprev) * inv;
                    si += (sn - sprev) * inv;
                    if (fabs(coef) <= wc.eps1)
                        stable_edge(cprev, sprev, useX ? v[en].x - v[e].x : v[en].y - v[e].y, coef, k, sr, si);
                }
                cprev = cn;
                sprev = sn;
            }
            if (useX) {
                if (fabs(B) <= wc.eps1) continue;
                sr /= B; si /= B;
            } else {
                if (fabs(A) <= wc.eps1) continue;
                sr *= -1.0 / A; si *= -1.0 / A;
            }
            fr = wc.cw_re * sr - wc.cw_im * si;
            fi = wc.cw_re * si + wc.cw_im * sr;
        }
        if (isnan(fr))
            continue;
        const double ref = external ? g.opath : wc.ot_far_ref;
        double dpr = 1.0, dpi = 0.0;
        if (!external)
            sincos_fp64(-k * (1.0 * (-g.c[2]) + ref), &dpi, &dpr);
        else if (ref != 0.0)
            sincos_fp64(-k * ref, &dpi, &dpr);
        const double cr = fr * dpr - fi * dpi, ci = fr * dpi + fi * dpr;
        double r[4], d[8];
        rotation(g.rot, w, u, vt, vf, r);
        // reference rotation carries 0.5 on the CPU (HandlerPO_fast.h:643-646)
        for (int q = 0; q < 4; ++q) r[q] *= 0.5;
        jones_product(cr, ci, r, g.jp, d);
        f00r += d[0]; f00i += d[1];
        f11r += d[6]; f11i += d[7];
    }
    const double fwr = f00r + f11r, fwi = f00i + f11i;
    double amp = fwi;
    if (wc.ot_ping != 0.0) {
        double sn, cs;
        sincos_fp64(2.0 * k * wc.ot_ping, &sn, &cs);
        amp = fwi * cs - fwr * sn;
    }
    const double c = wc.wavelength * amp * weight[o];
    cext[o] = isfinite(c) ? c : 0.0;
}

}  // namespace

// =============================================================== host side ==

struct mbs_po_staged {
    DevBeam *beams = nullptr;
    DevVert *verts = nullptr;
    int32_t *vbeg = nullptr;
    int32_t *beam_off = nullptr;
    double *weight = nullptr;
    int n_orient = 0;
    int64_t n_beams = 0, n_verts = 0;
    int64_t cap_beams = 0, cap_verts = 0, cap_orient = 0, cap_vbeg = 0;
    int max_nv = 0;
    std::vector<int64_t> beams_per_orient_prefix;   // host copy for statistics
    int64_t sum_beams = 0;
    int64_t sum_verts = 0;
};

struct mbs_po_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    bool has_grid = false, has_wave = false;
    GridDev grid;
    mbs_po_wave wave{};
    WaveConst wc{};
    // scratch
    double *partial = nullptr;
    size_t partial_cap = 0;      // doubles
    double *macc = nullptr;      // [2][G*16] device accumulators for host calls
    size_t macc_cap = 0;
    double *hres = nullptr;      // pinned [2][G*16]
    size_t hres_cap = 0;
    // raw upload buffers for staging
    void *raw = nullptr;
    size_t raw_cap = 0;
    int *d_status = nullptr;
    mbs_po_staged host_staged;   // reused by mbs_po_diffract
    cudaEvent_t ev[6] = {};
};

namespace {

int fail(mbs_po_ctx *ctx, int code, const std::string &msg)
{
    if (ctx)
        ctx->err = msg;
    return code;
}

int cuda_fail(mbs_po_ctx *ctx, cudaError_t e, const char *where)
{
    return fail(ctx, MBS_PO_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(expr, where)                                   \
    do {                                                  \
        cudaError_t e_ = (expr);                          \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
    } while (0)

template <typename T>
int ensure(mbs_po_ctx *ctx, T *&ptr, size_t &cap, size_t n, const char *what)
{
    if (n <= cap && ptr)
        return MBS_PO_OK;
    if (ptr)
        cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    const size_t alloc = std::max<size_t>(n, 1);
    cudaError_t e = cudaMalloc((void **)&ptr, alloc * sizeof(T));
    if (e != cudaSuccess)
        return fail(ctx, MBS_PO_ENOMEM, std::string("cudaMalloc ") + what + ": " + cudaGetErrorString(e));
    cap = alloc;
    return MBS_PO_OK;
}

int ensure64(mbs_po_ctx *ctx, DevBeam *&p, int64_t &cap, int64_t n)
{
    size_t c = (size_t)cap;
    int rc = ensure(ctx, p, c, (size_t)n, "beams");
    cap = (int64_t)c;
    return rc;
}

void staged_release(mbs_po_staged *s)
{
    cudaFree(s->beams);
    cudaFree(s->verts);
    cudaFree(s->vbeg);
    cudaFree(s->beam_off);
    cudaFree(s->weight);
    s->beams = nullptr;
    s->verts = nullptr;
    s->vbeg = nullptr;
    s->beam_off = nullptr;
    s->weight = nullptr;
    s->cap_beams = s->cap_verts = s->cap_orient = s->cap_vbeg = 0;
}

int validate(mbs_po_ctx *ctx, const mbs_po_beams *b)
{
    if (!b || b->n_orient < 0 || b->n_beams < 0 || b->n_verts < 0)
        return fail(ctx, MBS_PO_EINVAL, "null or negative-sized batch");
    if (b->n_beams >= (int64_t)1 << 31 || b->n_verts >= (int64_t)1 << 31)
        return fail(ctx, MBS_PO_ERANGE, "batch exceeds 2^31 beams or vertices");
    if (b->n_orient > 0 && (!b->beam_offsets || !b->orient_weight))
        return fail(ctx, MBS_PO_EINVAL, "missing orientation arrays");
    if (b->n_beams > 0 && (!b->vert_offsets || !b->vx || !b->vy || !b->slope_yx || !b->slope_xy
                           || !b->edge_flags || !b->beam_geom || !b->beam_flags))
        return fail(ctx, MBS_PO_EINVAL, "missing beam arrays");
    if (b->n_orient > 0 && (b->beam_offsets[0] != 0 || b->beam_offsets[b->n_orient] != b->n_beams))
        return fail(ctx, MBS_PO_EINVAL, "beam_offsets must run from 0 to n_beams");
    for (int o = 0; o < b->n_orient; ++o)
        if (b->beam_offsets[o + 1] < b->beam_offsets[o])
            return fail(ctx, MBS_PO_EINVAL, "beam_offsets not monotonic");
    if (b->n_beams > 0 && (b->vert_offsets[0] != 0 || b->vert_offsets[b->n_beams] != b->n_verts))
        return fail(ctx, MBS_PO_EINVAL, "vert_offsets must run from 0 to n_verts");
    for (int64_t i = 0; i < b->n_beams; ++i) {
        const int64_t nv = b->vert_offsets[i + 1] - b->vert_offsets[i];
        if (nv < 3 || nv > kMaxNv)
            return fail(ctx, MBS_PO_EBEAM, "beam " + std::to_string(i) + " has " + std::to_string(nv)
                                               + " vertices (valid edge data needs 3..31)");
    }
    return MBS_PO_OK;
}

}  // namespace

// ------------------------------------------------------------------ C ABI --

extern "C" const char *mbs_po_version(void)
{
    return "mbs-b200 0.1 sm_100a (FP64 plain + FP32 compensated PO diffraction)";
}

extern "C" int mbs_po_create(mbs_po_ctx **out, int device)
{
    if (!out)
        return MBS_PO_EINVAL;
    *out = nullptr;
    mbs_po_ctx *ctx = new mbs_po_ctx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    for (int i = 0; i < 6 && e == cudaSuccess; ++i)
        e = cudaEventCreate(&ctx->ev[i]);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&ctx->d_status, sizeof(int));
    if (e != cudaSuccess) {
        delete ctx;
        return MBS_PO_ECUDA;
    }
    *out = ctx;
    return MBS_PO_OK;
}

extern "C" int mbs_po_destroy(mbs_po_ctx *ctx)
{
    if (!ctx)
        return MBS_PO_EINVAL;
    cudaSetDevice(ctx->device);
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->grid.st);
    cudaFree(ctx->grid.ct);
    cudaFree(ctx->grid.sphi);
    cudaFree(ctx->grid.cphi);
    cudaFree(ctx->grid.vf);
    cudaFree(ctx->partial);
    cudaFree(ctx->macc);
    cudaFreeHost(ctx->hres);
    cudaFree(ctx->raw);
    cudaFree(ctx->d_status);
    staged_release(&ctx->host_staged);
    for (int i = 0; i < 6; ++i)
        if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
    if (ctx->stream)
        cudaStreamDestroy(ctx->stream);
    delete ctx;
    return MBS_PO_OK;
}

extern "C" const char *mbs_po_last_error(const mbs_po_ctx *ctx)
{
    return ctx ? ctx->err.c_str() : "null context";
}

extern "C" int mbs_po_set_grid(mbs_po_ctx *ctx, const mbs_po_grid *g)
{
    if (!ctx || !g || g->n_az <= 0 || g->n_zen < 0 || !g->theta || !g->vf)
        return fail(ctx, MBS_PO_EINVAL, "bad grid");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int nT = g->n_zen + 1, nAz = g->n_az;
    std::vector<double> st(nT), ct(nT), sphi(nAz), cphi(nAz);
    for (int t = 0; t < nT; ++t) {   // GpuDiffraction.cu:4536-4541
        st[t] = std::sin(g->theta[t]);
        ct[t] = std::cos(g->theta[t]);
    }
    for (int p = 0; p < nAz; ++p) {  // GpuDiffraction.cu:4543-4548
        const double phi = p * g->az_step;
        sphi[p] = std::sin(phi);
        cphi[p] = std::cos(phi);
    }
    GridDev &d = ctx->grid;
    cudaFree(d.st); cudaFree(d.ct); cudaFree(d.sphi); cudaFree(d.cphi); cudaFree(d.vf);
    d = GridDev();
    const size_t nvf = (size_t)nAz * nT * 3;
    CK(cudaMalloc((void **)&d.st, nT * sizeof(double)), "cudaMalloc grid");
    CK(cudaMalloc((void **)&d.ct, nT * sizeof(double)), "cudaMalloc grid");
    CK(cudaMalloc((void **)&d.sphi, nAz * sizeof(double)), "cudaMalloc grid");
    CK(cudaMalloc((void **)&d.cphi, nAz * sizeof(double)), "cudaMalloc grid");
    CK(cudaMalloc((void **)&d.vf, nvf * sizeof(double)), "cudaMalloc grid");
    CK(cudaMemcpy(d.st, st.data(), nT * sizeof(double), cudaMemcpyHostToDevice), "grid copy");
    CK(cudaMemcpy(d.ct, ct.data(), nT * sizeof(double), cudaMemcpyHostToDevice), "grid copy");
    CK(cudaMemcpy(d.sphi, sphi.data(), nAz * sizeof(double), cudaMemcpyHostToDevice), "grid copy");
    CK(cudaMemcpy(d.cphi, cphi.data(), nAz * sizeof(double), cudaMemcpyHostToDevice), "grid copy");
    CK(cudaMemcpy(d.vf, g->vf, nvf * sizeof(double), cudaMemcpyHostToDevice), "grid copy");
    d.n_az = nAz;
    d.n_zen = g->n_zen;
    ctx->has_grid = true;
    return MBS_PO_OK;
}

extern "C" int mbs_po_set_wave(mbs_po_ctx *ctx, const mbs_po_wave *w)
{
    if (!ctx || !w || !(w->wave_index > 0.0))
        return fail(ctx, MBS_PO_EINVAL, "bad wave constants");
    ctx->wave = *w;
    WaveConst &c = ctx->wc;
    c.k = w->wave_index;
    c.cw_re = w->compl_wave_re;
    c.cw_im = w->compl_wave_im;
    c.icw_re = w->inv_compl_wave_re;
    c.icw_im = w->inv_compl_wave_im;
    c.eps1 = w->eps1;
    c.eps1_f32 = std::max(w->eps1, 3e-5);   // GpuDiffraction.cu:498-512
    c.wavelength = w->wavelength;
    c.ot_far_ref = w->ot_far_reference_path;
    c.ot_ping = w->ot_ping_distance;
    c.legacy_sign = w->legacy_sign;
    c.ot_phase_avg = w->ot_phase_average;
    ctx->has_wave = true;
    return MBS_PO_OK;
}

namespace {

// Upload a batch and build device records into `s` (capacity reused).
int stage_into(mbs_po_ctx *ctx, const mbs_po_beams *b, mbs_po_staged *s, cudaStream_t st)
{
    int rc = validate(ctx, b);
    if (rc)
        return rc;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int64_t nB = b->n_beams, nV = b->n_verts, nO = b->n_orient;
    // raw upload area: vert_off, vx, vy, syx, sxy, geom (doubles/int64), flags (bytes)
    const size_t bytes_vo = (nB + 1) * 8, bytes_v = nV * 8, bytes_g = nB * MBS_PO_GEOM_STRIDE * 8;
    const size_t off_vo = 0, off_vx = off_vo + bytes_vo, off_vy = off_vx + bytes_v;
    const size_t off_syx = off_vy + bytes_v, off_sxy = off_syx + bytes_v, off_g = off_sxy + bytes_v;
    const size_t off_ef = off_g + bytes_g, off_bf = off_ef + ((nV + 15) & ~(size_t)15);
    const size_t raw_bytes = off_bf + ((nB + 15) & ~(size_t)15) + 16;
    size_t rawcap = ctx->raw_cap;
    unsigned char *raw = (unsigned char *)ctx->raw;
    if (raw_bytes > rawcap || !raw) {
        cudaFree(raw);
        ctx->raw = nullptr;
        ctx->raw_cap = 0;
        cudaError_t e = cudaMalloc(&ctx->raw, raw_bytes);
        if (e != cudaSuccess)
            return fail(ctx, MBS_PO_ENOMEM, std::string("cudaMalloc staging: ") + cudaGetErrorString(e));
        ctx->raw_cap = raw_bytes;
        raw = (unsigned char *)ctx->raw;
    }
    size_t cap;
    cap = (size_t)s->cap_verts;
    if ((rc = ensure(ctx, s->verts, cap, (size_t)std::max<int64_t>(nV, 1), "verts"))) return rc;
    s->cap_verts = (int64_t)cap;
    if ((rc = ensure64(ctx, s->beams, s->cap_beams, std::max<int64_t>(nB, 1)))) return rc;
    if (s->cap_vbeg < nB + 1 || !s->vbeg) {
        cudaFree(s->vbeg);
        s->vbeg = nullptr;
        s->cap_vbeg = 0;
        CK(cudaMalloc((void **)&s->vbeg, (size_t)(nB + 1) * sizeof(int32_t)), "cudaMalloc vbeg");
        s->cap_vbeg = nB + 1;
    }
    if ((size_t)s->cap_orient < (size_t)nO + 1 || !s->beam_off) {
        cudaFree(s->beam_off);
        cudaFree(s->weight);
        s->beam_off = nullptr;
        s->weight = nullptr;
        CK(cudaMalloc((void **)&s->beam_off, (nO + 1) * sizeof(int32_t)), "cudaMalloc offsets");
        CK(cudaMalloc((void **)&s->weight, std::max<int64_t>(nO, 1) * sizeof(double)), "cudaMalloc weights");
        s->cap_orient = nO + 1;
    }
    // orientation offsets to int32 on the host (small)
    std::vector<int32_t> boff(nO + 1);
    for (int64_t o = 0; o <= nO; ++o)
        boff[o] = (int32_t)b->beam_offsets[o];
    CK(cudaMemcpyAsync(s->beam_off, boff.data(), (nO + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, st), "H2D offsets");
    if (nO > 0)
        CK(cudaMemcpyAsync(s->weight, b->orient_weight, nO * sizeof(double), cudaMemcpyHostToDevice, st), "H2D weights");
    if (nB > 0) {
        CK(cudaMemcpyAsync(raw + off_vo, b->vert_offsets, bytes_vo, cudaMemcpyHostToDevice, st), "H2D vert_offsets");
        CK(cudaMemcpyAsync(raw + off_vx, b->vx, bytes_v, cudaMemcpyHostToDevice, st), "H2D vx");
        CK(cudaMemcpyAsync(raw + off_vy, b->vy, bytes_v, cudaMemcpyHostToDevice, st), "H2D vy");
        CK(cudaMemcpyAsync(raw + off_syx, b->slope_yx, bytes_v, cudaMemcpyHostToDevice, st), "H2D slope_yx");
        CK(cudaMemcpyAsync(raw + off_sxy, b->slope_xy, bytes_v, cudaMemcpyHostToDevice, st), "H2D slope_xy");
        CK(cudaMemcpyAsync(raw + off_g, b->beam_geom, bytes_g, cudaMemcpyHostToDevice, st), "H2D geom");
        CK(cudaMemcpyAsync(raw + off_ef, b->edge_flags, nV, cudaMemcpyHostToDevice, st), "H2D edge_flags");
        CK(cudaMemcpyAsync(raw + off_bf, b->beam_flags, nB, cudaMemcpyHostToDevice, st), "H2D beam_flags");
        CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st), "memset status");
        PackParams P;
        P.n_beams = nB;
        P.vert_off = (const int64_t *)(raw + off_vo);
        P.vx = (const double *)(raw + off_vx);
        P.vy = (const double *)(raw + off_vy);
        P.syx = (const double *)(raw + off_syx);
        P.sxy = (const double *)(raw + off_sxy);
        P.eflags = raw + off_ef;
        P.geom = (const double *)(raw + off_g);
        P.bflags = raw + off_bf;
        P.k = ctx->has_wave ? ctx->wc.k : 1.0;
        P.beams = s->beams;
        P.verts = s->verts;
        P.vbeg = s->vbeg;
        P.status = ctx->d_status;
        const int threads = 128;
        const int blocks = (int)((nB + 1 + threads - 1) / threads);
        po_pack_kernel<<<blocks, threads, 0, st>>>(P);
        CK(cudaGetLastError(), "pack kernel launch");
        int status = 0;
        CK(cudaMemcpyAsync(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H status");
        CK(cudaStreamSynchronize(st), "pack sync");
        if (status)
            return fail(ctx, MBS_PO_EBEAM, "malformed beam in batch");
    }
    s->n_orient = (int)nO;
    s->n_beams = nB;
    s->n_verts = nV;
    s->sum_beams = nB;
    s->sum_verts = nV;
    int mx = 0;
    for (int64_t i = 0; i < nB; ++i)
        mx = std::max<int>(mx, (int)(b->vert_offsets[i + 1] - b->vert_offsets[i]));
    s->max_nv = mx;
    return MBS_PO_OK;
}

struct LaunchPlan {
    int tile, tiles_per_row, n_chunks, orient_per_chunk;
};

LaunchPlan plan_launch(int n_az, int n_t, int n_orient)
{
    LaunchPlan L;
    L.tile = 128;
    L.tiles_per_row = (n_t + L.tile - 1) / L.tile;
    const long long ctas_per_chunk = (long long)n_az * L.tiles_per_row;
    int sms = 148;
    {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) == cudaSuccess
            && cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
            sms = v;
    }
    const long long target = (long long)sms * 4 * 4;   // ~4 waves of 4 CTAs per SM
    long long chunks = (target + ctas_per_chunk - 1) / ctas_per_chunk;
    chunks = std::max<long long>(1, std::min<long long>(chunks, std::max(1, n_orient)));
    chunks = std::min<long long>(chunks, 64);
    L.orient_per_chunk = (int)((n_orient + chunks - 1) / chunks);
    L.n_chunks = (int)((n_orient + L.orient_per_chunk - 1) / std::max(1, L.orient_per_chunk));
    if (L.n_chunks < 1) L.n_chunks = 1;
    return L;
}

int run_diffract(mbs_po_ctx *ctx, const mbs_po_staged *s, int precision, double *M_dev,
                 double *Mns_dev, cudaStream_t st, mbs_po_stats *stats)
{
    if (!ctx->has_grid || !ctx->has_wave)
        return fail(ctx, MBS_PO_ESTATE, "grid and wave constants must be set first");
    if (precision != MBS_PO_FP64 && precision != MBS_PO_FP32C)
        return fail(ctx, MBS_PO_EINVAL, "unknown precision");
    const int nAz = ctx->grid.n_az, nT = ctx->grid.n_zen + 1;
    const int64_t G = (int64_t)nAz * nT;
    if (stats) {
        stats->launches = 0;
        stats->n_chunks = 0;
        stats->kernel_ms = stats->reduce_ms = 0.0;
        stats->beam_dir_evals = s->n_beams * G;
        stats->vert_dir_evals = s->n_verts * G;
    }
    if (s->n_orient == 0 || s->n_beams == 0 || G == 0)
        return MBS_PO_OK;
    const LaunchPlan L = plan_launch(nAz, nT, s->n_orient);
    const bool ns = Mns_dev != nullptr;
    const size_t plane = (size_t)16 * G;
    int rc;
    if ((rc = ensure(ctx, ctx->partial, ctx->partial_cap, plane * L.n_chunks * (ns ? 2 : 1), "partials")))
        return rc;
    KParams P;
    P.beams = s->beams;
    P.verts = s->verts;
    P.vbeg = s->vbeg;
    P.beam_off = s->beam_off;
    P.weight = s->weight;
    P.st = ctx->grid.st;
    P.ct = ctx->grid.ct;
    P.sphi = ctx->grid.sphi;
    P.cphi = ctx->grid.cphi;
    P.vf = ctx->grid.vf;
    P.n_az = nAz;
    P.n_t = nT;
    P.n_orient = s->n_orient;
    P.orient_per_chunk = L.orient_per_chunk;
    P.tile = L.tile;
    P.tiles_per_row = L.tiles_per_row;
    P.wc = ctx->wc;
    P.partial = ctx->partial;
    P.partial_ns = ns ? ctx->partial + plane * L.n_chunks : nullptr;
    const size_t smem = kStageBeams * sizeof(SBeam) + kStageVerts * sizeof(SVert);
    dim3 grid((unsigned)(nAz * L.tiles_per_row), (unsigned)L.n_chunks);
    auto launch = [&](auto kern) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, L.tile, smem, st>>>(P);
        return cudaGetLastError();
    };
    CK(cudaEventRecord(ctx->ev[0], st), "event");
    cudaError_t e;
    if (precision == MBS_PO_FP64)
        e = ns ? launch(po_diffract_kernel<MBS_PO_FP64, true>) : launch(po_diffract_kernel<MBS_PO_FP64, false>);
    else
        e = ns ? launch(po_diffract_kernel<MBS_PO_FP32C, true>) : launch(po_diffract_kernel<MBS_PO_FP32C, false>);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "diffraction kernel launch");
    CK(cudaEventRecord(ctx->ev[1], st), "event");
    const int rb = 256;
    const int rg = (int)((G * 16 + rb - 1) / rb);
    po_reduce_kernel<<<rg, rb, 0, st>>>(ctx->partial, L.n_chunks, G, M_dev);
    CK(cudaGetLastError(), "reduce launch");
    if (ns) {
        po_reduce_kernel<<<rg, rb, 0, st>>>(P.partial_ns, L.n_chunks, G, Mns_dev);
        CK(cudaGetLastError(), "reduce launch");
    }
    CK(cudaEventRecord(ctx->ev[2], st), "event");
    if (stats) {
        CK(cudaEventSynchronize(ctx->ev[2]), "event sync");
        float a = 0, b2 = 0;
        cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&b2, ctx->ev[1], ctx->ev[2]);
        stats->kernel_ms = a;
        stats->reduce_ms = b2;
        stats->launches = 1 + (ns ? 2 : 1);
        stats->n_chunks = L.n_chunks;
    }
    return MBS_PO_OK;
}

}  // namespace

extern "C" int mbs_po_stage(mbs_po_ctx *ctx, const mbs_po_beams *beams, mbs_po_staged **out)
{
    if (!ctx || !out)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    *out = nullptr;
    mbs_po_staged *s = new mbs_po_staged();
    int rc = stage_into(ctx, beams, s, ctx->stream);
    if (rc) {
        staged_release(s);
        delete s;
        return rc;
    }
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        staged_release(s);
        delete s;
        return cuda_fail(ctx, e, "stage sync");
    }
    *out = s;
    return MBS_PO_OK;
}

extern "C" int mbs_po_staged_free(mbs_po_ctx *ctx, mbs_po_staged *s)
{
    if (!s)
        return MBS_PO_EINVAL;
    if (ctx)
        cudaSetDevice(ctx->device);
    staged_release(s);
    delete s;
    return MBS_PO_OK;
}

extern "C" int mbs_po_diffract_staged(mbs_po_ctx *ctx, const mbs_po_staged *s, int precision,
                                      double *M_dev, double *Mns_dev, void *stream,
                                      mbs_po_stats *stats)
{
    if (!ctx || !s || !M_dev)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    return run_diffract(ctx, s, precision, M_dev, Mns_dev, (cudaStream_t)stream, stats);
}

extern "C" int mbs_po_diffract(mbs_po_ctx *ctx, const mbs_po_beams *beams, int precision,
                               double *M_accum, double *Mns_accum, mbs_po_stats *stats)
{
    if (!ctx || !beams || !M_accum)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    if (!ctx->has_grid || !ctx->has_wave)
        return fail(ctx, MBS_PO_ESTATE, "grid and wave constants must be set first");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int64_t G = (int64_t)ctx->grid.n_az * (ctx->grid.n_zen + 1);
    if (beams->n_orient == 0 || beams->n_beams == 0 || G == 0)
        return validate(ctx, beams);
    cudaStream_t st = ctx->stream;
    const bool ns = Mns_accum != nullptr;
    const size_t n = (size_t)G * 16;
    int rc;
    if ((rc = ensure(ctx, ctx->macc, ctx->macc_cap, n * 2, "accumulators")))
        return rc;
    if (ctx->hres_cap < n * 2 || !ctx->hres) {
        cudaFreeHost(ctx->hres);
        ctx->hres = nullptr;
        ctx->hres_cap = 0;
        CK(cudaMallocHost((void **)&ctx->hres, n * 2 * sizeof(double)), "cudaMallocHost");
        ctx->hres_cap = n * 2;
    }
    CK(cudaEventRecord(ctx->ev[3], st), "event");
    if ((rc = stage_into(ctx, beams, &ctx->host_staged, st)))
        return rc;
    CK(cudaEventRecord(ctx->ev[4], st), "event");
    CK(cudaMemsetAsync(ctx->macc, 0, n * (ns ? 2 : 1) * sizeof(double), st), "memset acc");
    rc = run_diffract(ctx, &ctx->host_staged, precision, ctx->macc, ns ? ctx->macc + n : nullptr, st, stats);
    if (rc)
        return rc;
    CK(cudaEventRecord(ctx->ev[5], st), "event");
    CK(cudaMemcpyAsync(ctx->hres, ctx->macc, n * (ns ? 2 : 1) * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    CK(cudaStreamSynchronize(st), "sync");
    float h2d = 0.f;
    cudaEventElapsedTime(&h2d, ctx->ev[3], ctx->ev[4]);
    for (size_t i = 0; i < n; ++i)
        M_accum[i] += ctx->hres[i];
    if (ns)
        for (size_t i = 0; i < n; ++i)
            Mns_accum[i] += ctx->hres[n + i];
    if (stats) {
        stats->h2d_ms = h2d;
        stats->d2h_ms = 0.0;
    }
    return MBS_PO_OK;
}

extern "C" int mbs_po_extinction(mbs_po_ctx *ctx, const mbs_po_beams *beams, double *cext_out)
{
    if (!ctx || !beams || !cext_out)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    if (!ctx->has_wave)
        return fail(ctx, MBS_PO_ESTATE, "wave constants must be set first");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (beams->n_orient == 0)
        return MBS_PO_OK;
    cudaStream_t st = ctx->stream;
    int rc = stage_into(ctx, beams, &ctx->host_staged, st);
    if (rc)
        return rc;
    double *d = nullptr;
    size_t cap = 0;
    if ((rc = ensure(ctx, d, cap, (size_t)beams->n_orient, "cext")))
        return rc;
    const int th = 128;
    po_extinction_kernel<<<(beams->n_orient + th - 1) / th, th, 0, st>>>(
        ctx->host_staged.beams, ctx->host_staged.verts, ctx->host_staged.beam_off,
        ctx->host_staged.weight, beams->n_orient, ctx->wc, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(cext_out, d, beams->n_orient * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    cudaFree(d);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "extinction");
    return MBS_PO_OK;
}

extern "C" int mbs_po_select_batch(mbs_po_ctx *ctx, const mbs_po_beams *beams, int start,
                                   int max_count, double mem_fraction, int *count_out)
{
    if (!ctx || !beams || !count_out || start < 0 || start > beams->n_orient)
        return fail(ctx, MBS_PO_EINVAL, "bad arguments");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    size_t freeB = 0, totalB = 0;
    CK(cudaMemGetInfo(&freeB, &totalB), "cudaMemGetInfo");
    if (!(mem_fraction > 0.1 && mem_fraction <= 0.98))
        mem_fraction = 0.88;   // MBS_GPU_MEM_FRACTION default (GpuDiffraction.cu:391-401)
    const int64_t G = ctx->has_grid ? (int64_t)ctx->grid.n_az * (ctx->grid.n_zen + 1) : 0;
    // fixed: partials (up to 64 chunks x 2 planes) + accumulators + 128 MiB slack
    const double fixed = (double)G * 16 * 8 * (64 * 2 + 2) + (128.0 * (1 << 20));
    double budget = freeB * mem_fraction - fixed;
    int count = 0;
    const int end = std::min(beams->n_orient, start + std::max(0, max_count));
    for (int o = start; o < end; ++o) {
        const int64_t b0 = beams->beam_offsets[o], b1 = beams->beam_offsets[o + 1];
        const int64_t nv = b1 > b0 ? beams->vert_offsets[b1] - beams->vert_offsets[b0] : 0;
        // device records + raw upload copies
        const double need = (double)(b1 - b0) * (sizeof(DevBeam) + MBS_PO_GEOM_STRIDE * 8 + 8 + 1 + 4)
                          + (double)nv * (sizeof(DevVert) + 4 * 8 + 1) + 16;
        if (need > budget && count > 0)
            break;
        budget -= need;
        ++count;
    }
    *count_out = std::max(count, end > start ? 1 : 0);
    return MBS_PO_OK;
}

// ------------------------------------------------------------ peak probe --
// Independent FFMA chains: measures this device's FP32 FMA throughput, the
// denominator of the diffraction kernel's roofline fraction.
namespace {
__global__ void __launch_bounds__(256) po_fp32_probe_kernel(float *out, int iters, float a, float b)
{
    float x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
        x[i] = threadIdx.x * 1e-3f + i;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
#pragma unroll
            for (int i = 0; i < 8; ++i)
                x[i] = fmaf(x[i], a, b);
        }
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i)
        s += x[i];
    if (s == 1234.5f)
        out[blockIdx.x] = s;
}
}  // namespace

extern "C" int mbs_po_probe_fp32_peak(mbs_po_ctx *ctx, double *tflops)
{
    if (!ctx || !tflops)
        return MBS_PO_EINVAL;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    float *out = nullptr;
    CK(cudaMalloc((void **)&out, (size_t)sms * 64 * sizeof(float)), "cudaMalloc probe");
    const int blocks = sms * 8, threads = 256, iters = 4096;
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(ctx->ev[0], ctx->stream);
        po_fp32_probe_kernel<<<blocks, threads, 0, ctx->stream>>>(out, iters, 0.999999f, 1e-6f);
        cudaEventRecord(ctx->ev[1], ctx->stream);
        cudaError_t e = cudaEventSynchronize(ctx->ev[1]);
        if (e != cudaSuccess) {
            cudaFree(out);
            return cuda_fail(ctx, e, "probe");
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
        if (rep > 0)
            best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaFree(out);
    *tflops = best;
    return MBS_PO_OK;
}
