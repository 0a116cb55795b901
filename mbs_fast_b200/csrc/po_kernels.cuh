// po_kernels.cuh — the sm_100a kernels of the PO diffraction path.
//
//   po_pack_kernel       flat mbs_po_beams arrays -> device beam records
//   po_diffract_kernel   fused aperture integral -> coherent Jones sum ->
//                        Mueller -> orientation average (one CTA per azimuth
//                        bin x zenith tile x orientation chunk)
//   po_pole_kernel       the polar zenith rows, whose direction and basis are
//                        the same for every azimuth bin
//   po_reduce_kernel     deterministic sum of the chunk partials
//   po_extinction_kernel optical-theorem extinction per orientation
#pragma once

#include "mbs_po_b200.h"
#include "po_device.cuh"

namespace mbs {

// ------------------------------------------------------------------ records

// Azimuth-independent per-beam coefficients, precomputed at staging.
//   A(t, phi) = sin t (-(cos phi h0 + sin phi h1)) + cos t h2 + a0, B likewise.
//   With vf = (-sin phi, cos phi, 0) off the poles, u = vt = -(cos phi cos t,
//   sin phi cos t, sin t) and w = vt x dir = -vf, so the rotation of
//   GpuDiffraction.cu:831-856 is R = R0 + cos t Rc + sin t Rs with
//     R0 = sin phi X1 + cos phi X2,  Rc = -(cos phi Y1 + sin phi Y2),  Rs = Z
//   X1 = [[NTx, NPx], [-DTx, -DPx]], X2 = [[-NTy, -NPy], [DTy, DPy]],
//   Y1 = [[DTx, DPx], [NTx, NPx]],   Y2 = [[DTy, DPy], [NTy, NPy]],
//   Z  = [[-DTz, -DPz], [-NTz, -NPz]]  (NT, NP, DT = nxDT, DP = nxDP).
//   Q holds complWave * (X J_phased) for X1, X2, Y1, Y2, Z (4 complex
//   entries each), so d = s m (P0 + cos t Pc + sin t Ps) with
//   P0 = sin phi Q1 + cos phi Q2, Pc = -(cos phi Q3 + sin phi Q4), Ps = Q5.
struct __align__(16) BeamRec {
    double ab[8];     // h0 h1 h2 a0 v0 v1 v2 b0
    double Q[40];
    double slab[4];   // k (xa, ya) / 1.25e-3, k (xb, yb) / 1.25e-3 (see pack kernel)
    float nearr2;     // FP32C near-forward zone: A^2+B^2 <= nearr2
    int32_t vbeg;
    int32_t nv;
    int32_t pad;
};

// Per vertex, azimuth-independent parts of the phase in turns:
//   phase(t, phi) = sin t ps + cos t pc + p0,  ps = -(cos phi X + sin phi Y)
// (internal beams include the common beam-centre phase, GpuDiffraction.cu:1110-1122).
// Slopes of the x and y branches; an edge invalid for a branch (|dx| or |dy|
// below the geometry tolerance, Handler.cpp:674-692) gets the slope 1e30, so
// its coefficient is ~1e30 |B| (or |A|) and its term ~1e-30 of the others:
// the reference skips it.
struct __align__(16) VertRec {
    double X, Y, pc, p0;
    double syx, sxy;
};

// Both record arrays are stored as structures of arrays: word w of record i
// at base[w * stride + i], so the lanes of a warp that fill consecutive
// records read consecutive words (full 32-byte sectors) instead of one
// scattered sector per lane.
constexpr int kBrecWords = 54;   // ab[8] Q[40] slab[4] (nearr2 | vbeg) (nv | 0)
constexpr int kVrecWords = 6;    // X Y pc p0 syx sxy

struct BrecRef {
    const double *p;   // word 0 of the record
    int64_t s;         // stride between words
    __device__ __forceinline__ double ab(int i) const { return p[i * s]; }
    __device__ __forceinline__ double Q(int i) const { return p[(8 + i) * s]; }
    __device__ __forceinline__ double slab(int i) const { return p[(48 + i) * s]; }
    __device__ __forceinline__ float nearr2() const { return __int_as_float(__double2loint(p[52 * s])); }
    __device__ __forceinline__ int nv() const { return __double2loint(p[53 * s]); }
};

struct VrecRef {
    const double *p;
    int64_t s;
    __device__ __forceinline__ double X() const { return p[0]; }
    __device__ __forceinline__ double Y() const { return p[s]; }
    __device__ __forceinline__ double pc() const { return p[2 * s]; }
    __device__ __forceinline__ double p0() const { return p[3 * s]; }
    __device__ __forceinline__ double syx() const { return p[4 * s]; }
    __device__ __forceinline__ double sxy() const { return p[5 * s]; }
};

__device__ __forceinline__ void store_brec(double *base, int64_t s, int64_t i, const BeamRec &r)
{
    double *p = base + i;
    for (int w = 0; w < 8; ++w)
        p[w * s] = r.ab[w];
    for (int w = 0; w < 40; ++w)
        p[(8 + w) * s] = r.Q[w];
    for (int w = 0; w < 4; ++w)
        p[(48 + w) * s] = r.slab[w];
    p[52 * s] = __hiloint2double(r.vbeg, __float_as_int(r.nearr2));
    p[53 * s] = __hiloint2double(0, r.nv);
}

__device__ __forceinline__ void store_vrec(double *base, int64_t s, int64_t i, const VertRec &r)
{
    double *p = base + i;
    p[0] = r.X;
    p[s] = r.Y;
    p[2 * s] = r.pc;
    p[3 * s] = r.p0;
    p[4 * s] = r.syx;
    p[5 * s] = r.sxy;
}

constexpr double kInvalidSlope = 1.0e30;
constexpr int kMomentOrder = 6;      // near-forward expansion order
constexpr int kNumMoments = 28;      // (6+1)(6+2)/2
// Angular half-width of the FP32C near-forward zone in radians of vertex
// phase.  Inside it every |q.r| <= kNearPhase and the edge sum cancels
// badly in FP32; the sixth-order moment expansion there truncates at
// kNearPhase^7/7! < 1.3e-8.
constexpr double kNearPhase = 0.25;

struct KParams {
    const DevBeam *beams;
    const DevVert *verts;
    const double *brec;        // [kBrecWords][brec_stride]
    const double *vrec;        // [kVrecWords][vrec_stride]
    int64_t brec_stride, vrec_stride;
    const double *moments;     // [n_beams][kNumMoments] c_pq = <x^p y^q>/(p! q!)
    const int32_t *vbeg;       // [n_beams+1]
    const int32_t *beam_off;   // [n_orient+1]
    const double *weight;      // [n_orient]
    const double *st, *ct, *sphi, *cphi, *vf;
    const int8_t *row_kind;    // [n_t] 0 regular, 1 polar (po_pole_kernel), 2 general
    int n_az, n_t;             // n_t = n_zen+1
    int n_orient;
    int orient_per_chunk;
    int tiles_per_row;
    // Output sets (size instances of a multi-size batch): set s owns the
    // orientations [s*orient_per_set, (s+1)*orient_per_set) and the chunks
    // [s*chunks_per_set, (s+1)*chunks_per_set).  One set: the whole batch.
    int orient_per_set;
    int chunks_per_set;
    // Work items (chunk, azimuth bin, zenith tile), chunk-major: the
    // persistent CTAs of po_diffract_kernel take them in order from *work.
    int *work;
    int n_items;
    WaveConst wc;
    double *partial;           // [n_chunks][16][G]
    double *partial_ns;        // [n_chunks][16][G] or null
};

// Orientation range [o0, o1) of an orientation chunk; chunks never span
// two output sets.
__device__ __forceinline__ void chunk_range(const KParams &P, int chunk, int &o0, int &o1)
{
    const int set = chunk / P.chunks_per_set;
    const int base = set * P.orient_per_set;
    o0 = base + (chunk - set * P.chunks_per_set) * P.orient_per_chunk;
    o1 = min(min(base + P.orient_per_set, P.n_orient), o0 + P.orient_per_chunk);
}

// ------------------------------------------------------------ pack kernel

// Size scaling of a staged instance (multi-size scan): the reference's
// ScalePreparedOrientation (TracerPOTotal.cpp:2682-2747) and the scaled
// packing of pack_prepared_gpu_beam (GpuDiffraction.cu:281-357): vertex
// coordinates and the beam centre times s, area times s^2, and the Jones
// matrix re-phased from the unphased one,
//   J_phased = sign * absorption(s) * J * exp(i k s path),
//   absorption(s) = mean over absorption paths L of (L > DBL_EPSILON ?
//                   exp(cAbs L s) : 1)   (GpuDiffraction.cu:257-271).
struct ScaleParams {
    const double *scales;       // [n_inst] or null (one instance, s = 1, no re-phasing)
    const double *raw;          // [n_beams][MBS_PO_RAW_STRIDE]
    const int64_t *abs_off;     // [n_beams+1] or null
    const double *abs_paths;
    double k_rephase;           // wave number of the re-phasing
    double abs_coeff;
};

struct PackParams {
    int64_t n_beams;            // beams of one instance
    int64_t n_verts;            // vertices of one instance
    const int64_t *vert_off;
    const double *vx, *vy, *syx, *sxy;
    const uint8_t *eflags;
    const double *geom;
    const uint8_t *bflags;
    ScaleParams sc;
    WaveConst wc;
    DevBeam *beams;
    DevVert *verts;
    double *brec;               // [kBrecWords][brec_stride]
    double *vrec;               // [kVrecWords][vrec_stride]
    int64_t brec_stride, vrec_stride;
    double *moments;
    int32_t *vbeg;
    int *status;   // set to 1 on a malformed beam
};

// Binomial coefficients C(n, k), n, k <= 2 kMomentOrder (zero for k > n).
__constant__ double kBinom[13][13] = {
    {1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0},
    {1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0},
    {1.0, 2.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0},
    {1.0, 3.0, 3.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0},
    {1.0, 4.0, 6.0, 4.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0},
    {1.0, 5.0, 10.0, 10.0, 5.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0},
    {1.0, 6.0, 15.0, 20.0, 15.0, 6.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0},
    {1.0, 7.0, 21.0, 35.0, 35.0, 21.0, 7.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0},
    {1.0, 8.0, 28.0, 56.0, 70.0, 56.0, 28.0, 8.0, 1.0, 0.0, 0.0, 0.0, 0.0},
    {1.0, 9.0, 36.0, 84.0, 126.0, 126.0, 84.0, 36.0, 9.0, 1.0, 0.0, 0.0, 0.0},
    {1.0, 10.0, 45.0, 120.0, 210.0, 252.0, 210.0, 120.0, 45.0, 10.0, 1.0, 0.0, 0.0},
    {1.0, 11.0, 55.0, 165.0, 330.0, 462.0, 462.0, 330.0, 165.0, 55.0, 11.0, 1.0, 0.0},
    {1.0, 12.0, 66.0, 220.0, 495.0, 792.0, 924.0, 792.0, 495.0, 220.0, 66.0, 12.0, 1.0}};

// Grid: x over the beams of one instance (+1 for the terminal vertex
// offset), y = instance.  Instance i writes beams [i n_beams, (i+1) n_beams)
// and vertices [i n_verts, (i+1) n_verts) of the record arrays.
__global__ void po_pack_kernel(PackParams P)
{
    const int64_t bl = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (bl > P.n_beams)
        return;
    const int inst = blockIdx.y;
    const int64_t ob = (int64_t)inst * P.n_beams, ov = (int64_t)inst * P.n_verts;
    const int64_t v0l = P.vert_off[bl];
    P.vbeg[ob + bl] = (int32_t)(ov + v0l);
    if (bl == P.n_beams)
        return;
    const int64_t b = ob + bl;
    const int64_t v0 = ov + v0l;
    const int nv = (int)(P.vert_off[bl + 1] - v0l);
    if (nv < 3 || nv > kMaxNv) {
        atomicExch(P.status, 1);
        return;
    }
    const WaveConst &wc = P.wc;
    const double k = wc.k, kt = wc.k * kInvTwoPi;
    const double *g = P.geom + bl * MBS_PO_GEOM_STRIDE;
    const double scl = P.sc.scales ? P.sc.scales[inst] : 1.0;
    // scaled vertex coordinates (x s, y s)
    double vx[kMaxNv], vy[kMaxNv];
    for (int e = 0; e < nv; ++e) {
        vx[e] = P.vx[v0l + e] * scl;
        vy[e] = P.vy[v0l + e] * scl;
    }
    DevBeam d;
    // a0 = bd.hor, b0 = bd.ver (GpuDiffraction.cu:301-302)
    d.a0 = g[MBS_PO_G_BD] * g[MBS_PO_G_HOR] + g[MBS_PO_G_BD + 1] * g[MBS_PO_G_HOR + 1]
         + g[MBS_PO_G_BD + 2] * g[MBS_PO_G_HOR + 2];
    d.b0 = g[MBS_PO_G_BD] * g[MBS_PO_G_VER] + g[MBS_PO_G_BD + 1] * g[MBS_PO_G_VER + 1]
         + g[MBS_PO_G_BD + 2] * g[MBS_PO_G_VER + 2];
    for (int i = 0; i < 3; ++i) {
        d.h[i] = g[MBS_PO_G_HOR + i];
        d.v[i] = g[MBS_PO_G_VER + i];
        d.c[i] = g[MBS_PO_G_CEN + i] * scl;
    }
    d.area = g[MBS_PO_G_AREA] * (scl * scl);
    for (int i = 0; i < 12; ++i)
        d.rot[i] = g[MBS_PO_G_NT + i];
    if (P.sc.scales) {
        const double *raw = P.sc.raw + bl * MBS_PO_RAW_STRIDE;
        double sn, cs;
        sincos(P.sc.k_rephase * raw[MBS_PO_R_PATH] * scl, &sn, &cs);
        double absorption = 1.0;
        if (P.sc.abs_off) {
            const int64_t a0 = P.sc.abs_off[bl], a1 = P.sc.abs_off[bl + 1];
            if (a1 > a0) {
                double sum = 0.0;
                for (int64_t a = a0; a < a1; ++a) {
                    const double path = P.sc.abs_paths[a];
                    sum += (path > 2.220446049250313e-16) ? exp(P.sc.abs_coeff * path * scl) : 1.0;
                }
                absorption = sum / (double)(a1 - a0);
            }
        }
        const double f = raw[MBS_PO_R_SIGN] * absorption;
        for (int i = 0; i < 4; ++i) {
            const double jr = raw[MBS_PO_R_J + 2 * i], ji = raw[MBS_PO_R_J + 2 * i + 1];
            d.jp[2 * i] = f * (jr * cs - ji * sn);
            d.jp[2 * i + 1] = f * (jr * sn + ji * cs);
        }
    } else {
        for (int i = 0; i < 8; ++i)
            d.jp[i] = g[MBS_PO_G_JP + i];
    }
    d.opath = g[MBS_PO_G_OPATH] * scl;
    d.vbeg = (int32_t)v0;
    d.nv = nv;
    d.flags = P.bflags[bl];
    const bool internal = !(d.flags & MBS_PO_BEAM_EXTERNAL);

    // vertices: general records, phase coefficients, second moments
    double sxx = 0, sxy = 0, syy = 0, rmax2 = 0;
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int e = 0; e < nv; ++e) {
        const double x = vx[e], y = vy[e];
        sxx += x * x; sxy += x * y; syy += y * y;
        rmax2 = fmax(rmax2, x * x + y * y);
        const uint8_t f = P.eflags[v0l + e];
        DevVert dv;
        dv.x = x;
        dv.y = y;
        dv.syx = (f & MBS_PO_EDGE_VALID_X) ? P.syx[v0l + e] : nan;
        dv.sxy = (f & MBS_PO_EDGE_VALID_Y) ? P.sxy[v0l + e] : nan;
        P.verts[v0 + e] = dv;
        VertRec vr;
        vr.X = kt * (d.h[0] * x + d.v[0] * y) + (internal ? kt * d.c[0] : 0.0);
        vr.Y = kt * (d.h[1] * x + d.v[1] * y) + (internal ? kt * d.c[1] : 0.0);
        vr.pc = kt * (d.h[2] * x + d.v[2] * y) + (internal ? kt * d.c[2] : 0.0);
        vr.p0 = kt * (d.a0 * x + d.b0 * y);
        vr.syx = (f & MBS_PO_EDGE_VALID_X) ? P.syx[v0l + e] : kInvalidSlope;
        vr.sxy = (f & MBS_PO_EDGE_VALID_Y) ? P.sxy[v0l + e] : kInvalidSlope;
        store_vrec(P.vrec, P.vrec_stride, v0 + e, vr);
    }
    // Small-phase candidates.  The reference's moment branch needs every
    // vertex phase |k(A x_v + B y_v)| <= 1e-3 (HandlerPO_fast.h:161-173); in
    // particular for the vertex a farthest from the origin and the vertex b
    // farthest from the line through a.  Those two slabs in (A, B), widened
    // by 25% for rounding, bound the candidates tightly even for sliver
    // apertures; candidates take the exact FP64 test.
    int ia = 0;
    for (int e = 1; e < nv; ++e) {
        if (vx[e] * vx[e] + vy[e] * vy[e] > vx[ia] * vx[ia] + vy[ia] * vy[ia])
            ia = e;
    }
    const double xa = vx[ia], ya = vy[ia];
    int ib = ia == 0 ? 1 : 0;
    for (int e = 0; e < nv; ++e) {
        if (fabs(xa * vy[e] - ya * vx[e]) > fabs(xa * vy[ib] - ya * vx[ib]))
            ib = e;
    }
    const double slab_scale = k / (1.25 * kSmallPhase);
    double slab[4] = {xa * slab_scale, ya * slab_scale, vx[ib] * slab_scale, vy[ib] * slab_scale};
    (void)sxx; (void)sxy; (void)syy;
    d.sp_thr2 = 0.0;
    // FP32C near-forward zone: |q| rmax <= kNearPhase, so every vertex phase
    // is within kNearPhase and the moment expansion converges; 0.9 keeps the
    // zone inside that bound after the FP32 rounding of A and B.
    const double kr2 = k * k * rmax2;
    d.near2 = (float)((kr2 > 1e-300) ? 0.9 * kNearPhase * kNearPhase / kr2 : 0.0);
    P.beams[b] = d;

    BeamRec r;
    r.ab[0] = d.h[0]; r.ab[1] = d.h[1]; r.ab[2] = d.h[2]; r.ab[3] = d.a0;
    r.ab[4] = d.v[0]; r.ab[5] = d.v[1]; r.ab[6] = d.v[2]; r.ab[7] = d.b0;
    const double *NT = d.rot, *NP = d.rot + 3, *DT = d.rot + 6, *DP = d.rot + 9;
    const double X[5][4] = {
        {NT[0], NP[0], -DT[0], -DP[0]},     // X1
        {-NT[1], -NP[1], DT[1], DP[1]},     // X2
        {DT[0], DP[0], NT[0], NP[0]},       // Y1
        {DT[1], DP[1], NT[1], NP[1]},       // Y2
        {-DT[2], -DP[2], -NT[2], -NP[2]}};  // Z
    const double *j = d.jp;
    for (int q = 0; q < 5; ++q) {
        const double r00 = X[q][0], r01 = X[q][1], r10 = X[q][2], r11 = X[q][3];
        double m[8];   // X J
        m[0] = r00 * j[0] + r01 * j[4]; m[1] = r00 * j[1] + r01 * j[5];
        m[2] = r00 * j[2] + r01 * j[6]; m[3] = r00 * j[3] + r01 * j[7];
        m[4] = r10 * j[0] + r11 * j[4]; m[5] = r10 * j[1] + r11 * j[5];
        m[6] = r10 * j[2] + r11 * j[6]; m[7] = r10 * j[3] + r11 * j[7];
        for (int e = 0; e < 4; ++e) {
            r.Q[q * 8 + 2 * e] = wc.cw_re * m[2 * e] - wc.cw_im * m[2 * e + 1];
            r.Q[q * 8 + 2 * e + 1] = wc.cw_re * m[2 * e + 1] + wc.cw_im * m[2 * e];
        }
    }
    for (int i = 0; i < 4; ++i)
        r.slab[i] = slab[i];
    r.nearr2 = d.near2;
    r.vbeg = (int32_t)v0;
    r.nv = nv;
    r.pad = 0;
    store_brec(P.brec, P.brec_stride, b, r);

    // Polygon moments I(p,q) = integral of x^p y^q over the aperture, by
    // Green's theorem over the edges (exact for polygons), normalised by
    // the signed area: c_pq = <x^p y^q> / (p! q!).  Per edge (i -> j):
    //   I(p,q) += p! q!/(p+q+2)! (x_i y_j - x_j y_i)
    //             sum_{a<=p, c<=q} C(a+c, c) C(p+q-a-c, q-c) x_i^a x_j^(p-a) y_i^c y_j^(q-c)
    double *mom = P.moments + b * kNumMoments;
    double area2 = 0.0, minX = 1e300, maxX = -1e300, minY = 1e300, maxY = -1e300;
    for (int e = 0; e < nv; ++e) {
        const int en = (e + 1 < nv) ? e + 1 : 0;
        area2 += vx[e] * vy[en] - vx[en] * vy[e];
        minX = fmin(minX, vx[e]); maxX = fmax(maxX, vx[e]);
        minY = fmin(minY, vy[e]); maxY = fmax(maxY, vy[e]);
    }
    const bool degenerate = fabs(area2) <= 0x1p-40 * fmax((maxX - minX) * (maxY - minY), 2.2250738585072014e-308);
    double fact[kMomentOrder + 3];
    fact[0] = 1.0;
    for (int i = 1; i < kMomentOrder + 3; ++i)
        fact[i] = fact[i - 1] * i;
    double I[kNumMoments];
    for (int i = 0; i < kNumMoments; ++i)
        I[i] = 0.0;
    if (!degenerate) {
        for (int e = 0; e < nv; ++e) {
            const int en = (e + 1 < nv) ? e + 1 : 0;
            double pxi[kMomentOrder + 1], pxj[kMomentOrder + 1], pyi[kMomentOrder + 1], pyj[kMomentOrder + 1];
            pxi[0] = pxj[0] = pyi[0] = pyj[0] = 1.0;
            for (int a = 1; a <= kMomentOrder; ++a) {
                pxi[a] = pxi[a - 1] * vx[e];
                pxj[a] = pxj[a - 1] * vx[en];
                pyi[a] = pyi[a - 1] * vy[e];
                pyj[a] = pyj[a - 1] * vy[en];
            }
            const double cross = vx[e] * vy[en] - vx[en] * vy[e];
            int idx = 0;
            for (int n = 0; n <= kMomentOrder; ++n) {
                for (int p = n; p >= 0; --p, ++idx) {
                    const int q = n - p;
                    double t = 0.0;
                    for (int a = 0; a <= p; ++a)
                        for (int c = 0; c <= q; ++c)
                            t += kBinom[a + c][c] * kBinom[p + q - a - c][q - c]
                               * pxi[a] * pxj[p - a] * pyi[c] * pyj[q - c];
                    I[idx] += cross * t;
                }
            }
        }
    }
    int idx = 0;
    for (int n = 0; n <= kMomentOrder; ++n) {
        for (int p = n; p >= 0; --p, ++idx) {
            const int q = n - p;
            if (degenerate) {
                mom[idx] = (n == 0) ? 1.0 : 0.0;
                continue;
            }
            const double In = I[idx] * fact[p] * fact[q] / fact[p + q + 2];
            mom[idx] = (In / (0.5 * area2)) / (fact[p] * fact[q]);
        }
    }
}

// ----------------------------------------------------- general FP64 path
// Used for the rare (beam, direction) pairs that leave the vectorised path:
// irregular polar rows, near-singular FP32 edges and the small-phase
// candidates of the FP64 kernel.  Everything is recomputed in FP64 from the
// general records, as compute_beam_jones_context does
// (GpuDiffraction.cu:1064-1165).

struct DirFull {
    double st, ct, cp, sp;
    double dir[3], vf[3], vt[3], u[3], w[3];
};

__device__ __forceinline__ void cross3(const double *a, const double *b, double *o)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ __forceinline__ void dir_full(const KParams &P, int p, int t, DirFull &d)
{
    d.st = P.st[t];
    d.ct = P.ct[t];
    d.cp = P.cphi[p];
    d.sp = P.sphi[p];
    d.dir[0] = d.st * d.cp;
    d.dir[1] = d.st * d.sp;
    d.dir[2] = -d.ct;
    const double *vfp = P.vf + ((size_t)p * P.n_t + t) * 3;
    d.vf[0] = vfp[0]; d.vf[1] = vfp[1]; d.vf[2] = vfp[2];
    cross3(d.vf, d.dir, d.u);                 // u = vf x dir
    const double l2 = d.u[0] * d.u[0] + d.u[1] * d.u[1] + d.u[2] * d.u[2];
    const double il = (l2 > 1e-30) ? rsqrt(l2) : 1.0;   // transverse_basis_gpu
    d.vt[0] = d.u[0] * il; d.vt[1] = d.u[1] * il; d.vt[2] = d.u[2] * il;
    cross3(d.vt, d.dir, d.w);                 // w = vt x dir
}

// One beam's Jones contribution d[8] to one direction in FP64.  Returns
// false when the reference would skip the beam (NaN integral).
// `singular` = false drops nearly singular edges (|C_e| <= eps1) instead of
// taking their stable quotient, the reference's singularCorrection = 0.
__device__ __noinline__ bool beam_general(const DevBeam &g, const DevVert *gv, const DirFull &dc,
                                          const WaveConst &wc, double *d, bool singular = true)
{
    const double k = wc.k;
    const double a_sin = -dc.cp * g.h[0] - dc.sp * g.h[1];
    const double b_sin = -dc.cp * g.v[0] - dc.sp * g.v[1];
    const double A = fma(dc.st, a_sin, fma(dc.ct, g.h[2], g.a0));
    const double B = fma(dc.st, b_sin, fma(dc.ct, g.v[2], g.b0));
    const bool internal = !(g.flags & MBS_PO_BEAM_EXTERNAL);
    const double cm = internal ? -k * (dc.st * (dc.cp * g.c[0] + dc.sp * g.c[1]) + dc.ct * (-g.c[2])) : 0.0;
    const DevVert *v = gv + g.vbeg;
    const int nv = g.nv;
    double fr, fi, pr, pi;
    if (small_phase_factor(v, nv, A, B, k, pr, pi)) {
        const double sgn = wc.legacy_sign ? 1.0 : -1.0;
        const double ar = sgn * wc.icw_re * g.area, ai = sgn * wc.icw_im * g.area;
        fr = ar * pr - ai * pi;
        fi = ar * pi + ai * pr;
        if (internal) {
            double s, c;
            sincos_rad(cm, s, c);
            const double tr = fr * c - fi * s;
            fi = fr * s + fi * c;
            fr = tr;
        }
    } else {
        const bool useX = fabs(B) > fabs(A);
        const double qx = k * A * kInvTwoPi, qy = k * B * kInvTwoPi, cmt = cm * kInvTwoPi;
        double s0, c0;
        sincos_turns(fma(qx, v[0].x, fma(qy, v[0].y, cmt)), s0, c0);
        double cprev = c0, sprev = s0, sr = 0.0, si = 0.0;
        for (int e = 0; e < nv; ++e) {
            const int en = (e + 1 < nv) ? e + 1 : 0;
            double cn = c0, sn = s0;
            if (en != 0)
                sincos_turns(fma(qx, v[en].x, fma(qy, v[en].y, cmt)), sn, cn);
            const double coef = useX ? fma(v[e].syx, B, A) : fma(v[e].sxy, A, B);
            const double ac = fabs(coef);
            if (ac > wc.eps1) {
                const double inv = 1.0 / coef;
                sr = fma(cn - cprev, inv, sr);
                si = fma(sn - sprev, inv, si);
            } else if (singular && ac <= wc.eps1) {   // valid, nearly singular edge (NaN: invalid edge)
                const double delta = useX ? (v[en].x - v[e].x) : (v[en].y - v[e].y);
                stable_edge(cprev, sprev, delta, coef, k, sr, si);
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
    // rotation (GpuDiffraction.cu:831-856) with w = vt x dir, u = vf x dir:
    // (dir x NT).vt = NT.w and (dir x NT).vf = NT.u; the dir(dir.nxDT)
    // terms vanish since vt and vf are orthogonal to dir.
    const double *NT = g.rot, *NP = g.rot + 3, *DT = g.rot + 6, *DP = g.rot + 9;
    const double r00 = NT[0] * dc.w[0] + NT[1] * dc.w[1] + NT[2] * dc.w[2] + DT[0] * dc.vt[0] + DT[1] * dc.vt[1] + DT[2] * dc.vt[2];
    const double r01 = NP[0] * dc.w[0] + NP[1] * dc.w[1] + NP[2] * dc.w[2] + DP[0] * dc.vt[0] + DP[1] * dc.vt[1] + DP[2] * dc.vt[2];
    const double r10 = NT[0] * dc.u[0] + NT[1] * dc.u[1] + NT[2] * dc.u[2] + DT[0] * dc.vf[0] + DT[1] * dc.vf[1] + DT[2] * dc.vf[2];
    const double r11 = NP[0] * dc.u[0] + NP[1] * dc.u[1] + NP[2] * dc.u[2] + DP[0] * dc.vf[0] + DP[1] * dc.vf[1] + DP[2] * dc.vf[2];
    const double *jp = g.jp;
    const double s00r = fr * r00, s00i = fi * r00, s01r = fr * r01, s01i = fi * r01;
    const double s10r = fr * r10, s10i = fi * r10, s11r = fr * r11, s11i = fi * r11;
    d[0] = s00r * jp[0] - s00i * jp[1] + s01r * jp[4] - s01i * jp[5];
    d[1] = s00r * jp[1] + s00i * jp[0] + s01r * jp[5] + s01i * jp[4];
    d[2] = s00r * jp[2] - s00i * jp[3] + s01r * jp[6] - s01i * jp[7];
    d[3] = s00r * jp[3] + s00i * jp[2] + s01r * jp[7] + s01i * jp[6];
    d[4] = s10r * jp[0] - s10i * jp[1] + s11r * jp[4] - s11i * jp[5];
    d[5] = s10r * jp[1] + s10i * jp[0] + s11r * jp[5] + s11i * jp[4];
    d[6] = s10r * jp[2] - s10i * jp[3] + s11r * jp[6] - s11i * jp[7];
    d[7] = s10r * jp[3] + s10i * jp[2] + s11r * jp[7] + s11i * jp[6];
    return true;
}

// FP32C near-forward zone: the aperture integral from the sixth-order
// moment expansion in FP64,  F = areaLimit sum_pq i^(p+q) qx^p qy^q c_pq,
// times the internal-beam common phase, returned as the edge-sum
// equivalent s = F / complWave so the caller applies P0 + cos t Pc + sin t Ps.
__device__ __noinline__ void near_forward_s(const DevBeam &g, const double *mom, double st, double ct,
                                            double cp, double sp, const WaveConst &wc,
                                            float &sr, float &si)
{
    const double k = wc.k;
    const double a_sin = -cp * g.h[0] - sp * g.h[1];
    const double b_sin = -cp * g.v[0] - sp * g.v[1];
    const double qx = k * fma(st, a_sin, fma(ct, g.h[2], g.a0));
    const double qy = k * fma(st, b_sin, fma(ct, g.v[2], g.b0));
    double px[kMomentOrder + 1], py[kMomentOrder + 1];
    px[0] = 1.0; py[0] = 1.0;
    for (int i = 1; i <= kMomentOrder; ++i) {
        px[i] = px[i - 1] * qx;
        py[i] = py[i - 1] * qy;
    }
    double re = 0.0, im = 0.0;
    int idx = 0;
    for (int n = 0; n <= kMomentOrder; ++n) {
        double s = 0.0;
        for (int p = n; p >= 0; --p, ++idx)
            s = fma(mom[idx], px[p] * py[n - p], s);
        switch (n & 3) {
        case 0: re += s; break;
        case 1: im += s; break;
        case 2: re -= s; break;
        default: im -= s; break;
        }
    }
    const double sgn = wc.legacy_sign ? 1.0 : -1.0;
    const double ar = sgn * wc.icw_re * g.area, ai = sgn * wc.icw_im * g.area;
    double fr = ar * re - ai * im, fi = ar * im + ai * re;
    if (!(g.flags & MBS_PO_BEAM_EXTERNAL)) {
        const double cm = -k * (st * (cp * g.c[0] + sp * g.c[1]) + ct * (-g.c[2]));
        double s, c;
        sincos_rad(cm, s, c);
        const double tr = fr * c - fi * s;
        fi = fr * s + fi * c;
        fr = tr;
    }
    // s = F / complWave
    const double n2 = wc.cw_re * wc.cw_re + wc.cw_im * wc.cw_im;
    sr = (float)((fr * wc.cw_re + fi * wc.cw_im) / n2);
    si = (float)((fi * wc.cw_re - fr * wc.cw_im) / n2);
}

// ----------------------------------------------- shared-memory records
// Per (beam, azimuth of the CTA), laid out for 16-byte vector loads: every
// lane of a warp reads the same record (a broadcast), so a beam costs ten
// (FP32C) or eighteen (FP64) shared loads per thread for all DPT directions.
//   A(t) = sin t a[0] + cos t a[1] + a[2],  B(t) = sin t a[3] + cos t a[4] + a[5]
//   P0, Pc, Ps: complWave (R J) parts, 4 complex entries each (see BeamRec)
//   slab: small-phase candidate test, nearr2: FP32C near-forward zone

//   zone: nonzero when some direction of the CTA's zenith tile may fall in
//   the near-forward zone or pass the slab test (tile_zone_possible)

template <typename T>
struct BeamRegs {
    T a[6];
    T slab[4];
    float nearr2;
    int nv, vs, gbeam, zone;
};

template <typename T>
struct SBeamRaw;

template <>
struct __align__(16) SBeamRaw<float> {
    float4 q[10];   // a0 a3 a1 a4 | a2 a5 slab0 slab1 | slab2 slab3 nearr2 nv | P[24] | gbeam vs zone
                    // ((a0, a3), (a1, a4), (a2, a5): operand pairs of the packed A, B;
                    // P entries 2h, 2h+1 of P0, Pc, Ps as (re, re, im, im): the
                    // real and the imaginary operand pairs of the packed Jones update)
};

template <>
struct __align__(16) SBeamRaw<double> {
    double2 q[18];  // a0a1 a2a3 a4a5 | slab | slab | P[24] | (zone,nv) (gbeam,vs)
                    // (FP64 has no near-forward zone: the nearr2 word holds the zone flag)
};

// The zenith tile of a work item seen from the stage fill: every direction
// w = (sin t, cos t) the CTA evaluates lies within del of wc = (stc, ctc).
struct TileZone {
    double stc, ctc, del;
};

// Whether some direction of the tile can pass the per-pair zone tests of
// the hot loop for a beam with azimuth-folded coefficients a (A = sin t a0
// + cos t a1 + a2, B = sin t a3 + cos t a4 + a5): the FP32C near-forward
// test A^2 + B^2 <= nearr2 and the slab test |A s0 + B s1| <= 1 and
// |A s2 + B s3| <= 1.  A, B and the slab forms are affine in w, so over
// the tile they stay within |gradient| del of their values at wc.  The
// margins cover the hot loop's FP32 rounding of the coefficients, of
// sin t, cos t and of the sums (below 2.5e-7 of sum |a_i| for A and B), so
// a tile reported clear holds no pair that the per-pair tests would mark,
// and skipping those tests there leaves every result unchanged.
__device__ __forceinline__ bool tile_zone_possible(const double *a, const double *slab, float nearr2,
                                                   bool f32, const TileZone &z)
{
    const double Ac = fma(a[0], z.stc, fma(a[1], z.ctc, a[2]));
    const double Bc = fma(a[3], z.stc, fma(a[4], z.ctc, a[5]));
    const double amax = fabs(a[0]) + fabs(a[1]) + fabs(a[2]) + fabs(a[3]) + fabs(a[4]) + fabs(a[5]);
    const double marg = 1e-6 * amax + 1e-300;
    if (f32) {
        const double gq = sqrt(a[0] * a[0] + a[1] * a[1] + a[3] * a[3] + a[4] * a[4]);
        const double ql = sqrt(Ac * Ac + Bc * Bc) - gq * z.del - 2.0 * marg;
        if (!(ql > 0.0 && ql * ql > (double)nearr2 * (1.0 + 1e-5)))
            return true;
    }
    bool clear = false;
#pragma unroll
    for (int k = 0; k < 4; k += 2) {
        const double s0 = slab[k], s1 = slab[k + 1];
        const double uc = fma(Ac, s0, Bc * s1);
        const double g0 = fma(a[0], s0, a[3] * s1), g1 = fma(a[1], s0, a[4] * s1);
        const double mu = 2.0 * marg * (fabs(s0) + fabs(s1)) + 1e-6;
        clear = clear || fabs(uc) - sqrt(g0 * g0 + g1 * g1) * z.del > 1.0 + mu;
    }
    return !clear;
}

template <typename T>
struct SVertRaw;

template <>
struct __align__(16) SVertRaw<float> {
    double2 q[2];   // (ps, pc) (p0, slopes syx|sxy as two floats)
};

template <>
struct __align__(16) SVertRaw<double> {
    double2 q[3];   // (ps, pc) (p0, syx) (sxy, unused)
};

template <typename T, int TPB>
struct StageCfg {
    static constexpr int kBeams = TPB;
    static constexpr int kVerts = 4 * TPB;
    static constexpr size_t kBytes = kBeams * sizeof(SBeamRaw<T>) + kVerts * sizeof(SVertRaw<T>);
};

__device__ __forceinline__ void fill_beam(const BrecRef &r, double cp, double sp, int vs, int gbeam,
                                          const TileZone &z, SBeamRaw<float> &s)
{
    float a[6], P[24];
    const double ad[6] = {-(cp * r.ab(0) + sp * r.ab(1)), r.ab(2), r.ab(3),
                          -(cp * r.ab(4) + sp * r.ab(5)), r.ab(6), r.ab(7)};
    const double sl[4] = {r.slab(0), r.slab(1), r.slab(2), r.slab(3)};
    const int zone = tile_zone_possible(ad, sl, r.nearr2(), true, z) ? 1 : 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
        a[i] = (float)ad[i];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        P[e] = (float)(sp * r.Q(e) + cp * r.Q(8 + e));
        P[8 + e] = (float)(-(cp * r.Q(16 + e) + sp * r.Q(24 + e)));
        P[16 + e] = (float)r.Q(32 + e);
    }
    s.q[0] = make_float4(a[0], a[3], a[1], a[4]);
    s.q[1] = make_float4(a[2], a[5], (float)sl[0], (float)sl[1]);
    s.q[2] = make_float4((float)sl[2], (float)sl[3], r.nearr2(), __int_as_float(r.nv()));
#pragma unroll
    for (int i = 0; i < 6; ++i)
        s.q[3 + i] = make_float4(P[4 * i], P[4 * i + 2], P[4 * i + 1], P[4 * i + 3]);
    s.q[9] = make_float4(__int_as_float(gbeam), __int_as_float(vs), __int_as_float(zone), 0.f);
}

__device__ __forceinline__ void fill_beam(const BrecRef &r, double cp, double sp, int vs, int gbeam,
                                          const TileZone &z, SBeamRaw<double> &s)
{
    const double ad[6] = {-(cp * r.ab(0) + sp * r.ab(1)), r.ab(2), r.ab(3),
                          -(cp * r.ab(4) + sp * r.ab(5)), r.ab(6), r.ab(7)};
    const double sl[4] = {r.slab(0), r.slab(1), r.slab(2), r.slab(3)};
    const int zone = tile_zone_possible(ad, sl, 0.f, false, z) ? 1 : 0;
    s.q[0] = make_double2(ad[0], ad[1]);
    s.q[1] = make_double2(ad[2], ad[3]);
    s.q[2] = make_double2(ad[4], ad[5]);
    s.q[3] = make_double2(sl[0], sl[1]);
    s.q[4] = make_double2(sl[2], sl[3]);
#pragma unroll
    for (int e = 0; e < 8; e += 2) {
        s.q[5 + e / 2] = make_double2(sp * r.Q(e) + cp * r.Q(8 + e), sp * r.Q(e + 1) + cp * r.Q(9 + e));
        s.q[9 + e / 2] = make_double2(-(cp * r.Q(16 + e) + sp * r.Q(24 + e)),
                                      -(cp * r.Q(17 + e) + sp * r.Q(25 + e)));
        s.q[13 + e / 2] = make_double2(r.Q(32 + e), r.Q(33 + e));
    }
    s.q[17] = make_double2(__hiloint2double(r.nv(), zone), __hiloint2double(vs, gbeam));
}

// FP32C: p0 carries the range-reduction constant 1.5*2^29 + 1/2, so the
// phase sum st ps + ct pc + p0 lands directly in [2^29, 2^30), where the low
// 23 mantissa bits hold frac(u + 1/2) (three roundings of at most 2^-24 turn).
__device__ __forceinline__ void fill_vert(const VrecRef &r, double cp, double sp, SVertRaw<float> &w)
{
    w.q[0] = make_double2(-(cp * r.X() + sp * r.Y()), r.pc());
    w.q[1] = make_double2(r.p0() + (kMagic29 + 0.5),
                          __hiloint2double(__float_as_int((float)r.sxy()), __float_as_int((float)r.syx())));
}

__device__ __forceinline__ void fill_vert(const VrecRef &r, double cp, double sp, SVertRaw<double> &w)
{
    w.q[0] = make_double2(-(cp * r.X() + sp * r.Y()), r.pc());
    w.q[1] = make_double2(r.p0(), r.syx());
    w.q[2] = make_double2(r.sxy(), 0.0);
}

__device__ __forceinline__ void load_beam(const SBeamRaw<float> &s, BeamRegs<float> &b)
{
    const float4 q0 = s.q[0], q1 = s.q[1], q2 = s.q[2], q9 = s.q[9];
    b.a[0] = q0.x; b.a[3] = q0.y; b.a[1] = q0.z; b.a[4] = q0.w; b.a[2] = q1.x; b.a[5] = q1.y;
    b.slab[0] = q1.z; b.slab[1] = q1.w; b.slab[2] = q2.x; b.slab[3] = q2.y;
    b.nearr2 = q2.z;
    b.nv = __float_as_int(q2.w);
    b.gbeam = __float_as_int(q9.x);
    b.vs = __float_as_int(q9.y);
    b.zone = __float_as_int(q9.z);
}

__device__ __forceinline__ void load_beam(const SBeamRaw<double> &s, BeamRegs<double> &b)
{
    const double2 q0 = s.q[0], q1 = s.q[1], q2 = s.q[2], q3 = s.q[3], q4 = s.q[4], q17 = s.q[17];
    b.a[0] = q0.x; b.a[1] = q0.y; b.a[2] = q1.x; b.a[3] = q1.y; b.a[4] = q2.x; b.a[5] = q2.y;
    b.slab[0] = q3.x; b.slab[1] = q3.y; b.slab[2] = q4.x; b.slab[3] = q4.y;
    b.nearr2 = 0.f;
    b.zone = __double2loint(q17.x);
    b.nv = __double2hiint(q17.x);
    b.vs = __double2hiint(q17.y);
    b.gbeam = __double2loint(q17.y);
}

__device__ __forceinline__ void load_P(const SBeamRaw<float> &s, float *P)
{
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const float4 q = s.q[3 + i];
        P[4 * i] = q.x; P[4 * i + 1] = q.z; P[4 * i + 2] = q.y; P[4 * i + 3] = q.w;
    }
}

__device__ __forceinline__ void load_P(const SBeamRaw<double> &s, double *P)
{
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        const double2 q = s.q[5 + i];
        P[2 * i] = q.x; P[2 * i + 1] = q.y;
    }
}

// P0, Pc, Ps entries 2h and 2h+1 (re, im each) of a beam record.
__device__ __forceinline__ void load_P_pair(const SBeamRaw<float> &s, int h, float *p0, float *pc,
                                            float *ps)
{
    const float4 a = s.q[3 + h], b = s.q[5 + h], c = s.q[7 + h];
    p0[0] = a.x; p0[1] = a.z; p0[2] = a.y; p0[3] = a.w;
    pc[0] = b.x; pc[1] = b.z; pc[2] = b.y; pc[3] = b.w;
    ps[0] = c.x; ps[1] = c.z; ps[2] = c.y; ps[3] = c.w;
}

// FP32C packed form of load_P_pair: (re 2h, re 2h+1) and (im 2h, im 2h+1)
// operand pairs of P0, Pc and Ps, straight from the record's layout.
__device__ __forceinline__ void load_P_packed(const SBeamRaw<float> &s, int h, float2 &p0r, float2 &p0i,
                                              float2 &pcr, float2 &pci, float2 &psr, float2 &psi)
{
    const float4 a = s.q[3 + h], b = s.q[5 + h], c = s.q[7 + h];
    p0r = make_float2(a.x, a.y); p0i = make_float2(a.z, a.w);
    pcr = make_float2(b.x, b.y); pci = make_float2(b.z, b.w);
    psr = make_float2(c.x, c.y); psi = make_float2(c.z, c.w);
}

__device__ __forceinline__ void load_P_pair(const SBeamRaw<double> &s, int h, double *p0, double *pc,
                                            double *ps)
{
    const double2 a0 = s.q[5 + 2 * h], a1 = s.q[6 + 2 * h];
    const double2 b0 = s.q[9 + 2 * h], b1 = s.q[10 + 2 * h];
    const double2 c0 = s.q[13 + 2 * h], c1 = s.q[14 + 2 * h];
    p0[0] = a0.x; p0[1] = a0.y; p0[2] = a1.x; p0[3] = a1.y;
    pc[0] = b0.x; pc[1] = b0.y; pc[2] = b1.x; pc[3] = b1.y;
    ps[0] = c0.x; ps[1] = c0.y; ps[2] = c1.x; ps[3] = c1.y;
}

struct VertRegs {
    double ps, pc, p0;
};

__device__ __forceinline__ void load_vert(const SVertRaw<float> &w, VertRegs &v, float &syx, float &sxy)
{
    const double2 q0 = w.q[0], q1 = w.q[1];
    v.ps = q0.x; v.pc = q0.y; v.p0 = q1.x;
    syx = __int_as_float(__double2loint(q1.y));
    sxy = __int_as_float(__double2hiint(q1.y));
}

__device__ __forceinline__ void load_vert(const SVertRaw<double> &w, VertRegs &v, double &syx, double &sxy)
{
    const double2 q0 = w.q[0], q1 = w.q[1], q2 = w.q[2];
    v.ps = q0.x; v.pc = q0.y; v.p0 = q1.x;
    syx = q1.y;
    sxy = q2.x;
}

// Vertex phasor (cos, sin) of 2 pi u, u = st ps + ct pc + p0 in turns.
__device__ __forceinline__ void vertex_phasor(double st, double ct, const VertRegs &w, double &s,
                                              double &c)
{
    sincos_turns(fma(st, w.ps, fma(ct, w.pc, w.p0)), s, c);
}

// FP32C: the offset sum (p0 holds 1.5*2^29 + 1/2, see fill_vert) leaves
// frac(u + 1/2) in the low 23 mantissa bits; as a float y = 1.f in [1, 2),
// 2 pi (y - 3/2) = y 2 pi - 3 pi is the reduced angle in [-pi, pi) (one FFMA,
// no FP64->FP32 conversion); then the hardware sine and cosine.
__device__ __forceinline__ void vertex_phasor(double st, double ct, const VertRegs &w, float &s,
                                              float &c)
{
    const double t = fma(st, w.ps, fma(ct, w.pc, w.p0));
    const unsigned lo = (unsigned)__double2loint(t);
    const float x = fmaf(__int_as_float(0x3F800000u | (lo & 0x007FFFFFu)), 6.28318530717958647f,
                         -9.42477796076937972f);
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(s) : "f"(x));
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(c) : "f"(x));
}

// FP64 phasor through the kernel's sine table.
__device__ __forceinline__ void vertex_phasor_t(double st, double ct, const VertRegs &w,
                                                const double2 *tab, double &s, double &c)
{
    sincos_turns_tab(fma(st, w.ps, fma(ct, w.pc, w.p0)), tab, s, c);
}

// The same for two directions of one vertex: the two reductions to the
// angle in one FFMA2 (each lane rounds as the FFMA above, so the phasors are
// bitwise those of two single calls).
__device__ __forceinline__ void vertex_phasor2(double st0, double ct0, double st1, double ct1,
                                               const VertRegs &w, float2 &cs0, float2 &cs1)
{
    const double t0 = fma(st0, w.ps, fma(ct0, w.pc, w.p0));
    const double t1 = fma(st1, w.ps, fma(ct1, w.pc, w.p0));
    const unsigned lo0 = (unsigned)__double2loint(t0), lo1 = (unsigned)__double2loint(t1);
    const float2 y = make_float2(__int_as_float(0x3F800000u | (lo0 & 0x007FFFFFu)),
                                 __int_as_float(0x3F800000u | (lo1 & 0x007FFFFFu)));
    const float2 x = __ffma2_rn(y, make_float2(6.28318530717958647f, 6.28318530717958647f),
                                make_float2(-9.42477796076937972f, -9.42477796076937972f));
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(cs0.y) : "f"(x.x));
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(cs0.x) : "f"(x.x));
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(cs1.y) : "f"(x.y));
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(cs1.x) : "f"(x.y));
}

// Phasors (cos, sin) of one vertex for a thread's DPT directions, handed to
// out(d, phasor): directions in pairs, an odd last one alone.
template <int DPT, typename Out>
__device__ __forceinline__ void vertex_phasors(const double *st, const double *ct, const VertRegs &w,
                                               Out &&out)
{
#pragma unroll
    for (int d = 0; d + 1 < DPT; d += 2) {
        float2 a, b;
        vertex_phasor2(st[d], ct[d], st[d + 1], ct[d + 1], w, a, b);
        out(d, a);
        out(d + 1, b);
    }
    if (DPT & 1) {
        float2 c;
        vertex_phasor(st[DPT - 1], ct[DPT - 1], w, c.y, c.x);
        out(DPT - 1, c);
    }
}

__device__ __forceinline__ double rcp_t(double x) { return rcp64(x); }
__device__ __forceinline__ float rcp_t(float x) { return rcp32(x); }

// Edge sums S_d = sum_e (P(e+1) - P(e)) / C_e of one beam for the DPT
// directions of a thread.  The reference's two branches share one form,
// C_e = X2 + slope_e X1 with (X1, X2, slope) = (B, A, slope_yx) when |B| > |A|
// (x branch) and (A, B, slope_xy) otherwise (y branch).  All vertex phasors
// are independent, so the NV*DPT chains interleave.  mn[d] receives the
// smallest |C_e| (nearly singular edges go to the FP64 pass).
template <typename T, int DPT, int NV>
__device__ __forceinline__ void edge_sums_fixed(const SVertRaw<T> *v, const double *st, const double *ct,
                                                const T *X1, const T *X2, const bool *useX,
                                                T *sr, T *si, T *mn, const double2 *tab)
{
    T c[DPT][NV], s[DPT][NV], syx[NV], sxy[NV];
#pragma unroll
    for (int e = 0; e < NV; ++e) {
        VertRegs w;
        load_vert(v[e], w, syx[e], sxy[e]);
#pragma unroll
        for (int d = 0; d < DPT; ++d)
            vertex_phasor_t(st[d], ct[d], w, tab, s[d][e], c[d][e]);
    }
#pragma unroll
    for (int d = 0; d < DPT; ++d) {
        mn[d] = T(1e30);
        sr[d] = T(0);
        si[d] = T(0);
    }
    // consecutive edges share one reciprocal: 1/a = b/(ab), 1/b = a/(ab)
    // (FP64 here: coefficients between eps1 and about 1e30 |X1| keep the
    // product far from overflow and underflow; a pair with a smaller one is
    // marked and its sums discarded)
#pragma unroll
    for (int e = 0; e < NV; e += 2) {
#pragma unroll
        for (int d = 0; d < DPT; ++d) {
            const T ca = fma(useX[d] ? syx[e] : sxy[e], X1[d], X2[d]);
            const int e1 = (e + 1 < NV) ? e + 1 : 0;
            if (e + 1 < NV) {
                const T cb = fma(useX[d] ? syx[e1] : sxy[e1], X1[d], X2[d]);
                const T r = rcp_t(ca * cb);
                const T ia = cb * r, ib = ca * r;
                const int e2 = (e + 2 < NV) ? e + 2 : 0;
                mn[d] = fmin(mn[d], fmin(fabs(ca), fabs(cb)));
                sr[d] = fma(c[d][e1] - c[d][e], ia, sr[d]);
                si[d] = fma(s[d][e1] - s[d][e], ia, si[d]);
                sr[d] = fma(c[d][e2] - c[d][e1], ib, sr[d]);
                si[d] = fma(s[d][e2] - s[d][e1], ib, si[d]);
            } else {
                const T inv = rcp_t(ca);
                mn[d] = fmin(mn[d], fabs(ca));
                sr[d] = fma(c[d][0] - c[d][e], inv, sr[d]);
                si[d] = fma(s[d][0] - s[d][e], inv, si[d]);
            }
        }
    }
}

// FP32C edge sums in two parts.  The head (vertices 0-2, edges 0 and 1:
// every aperture has at least three vertices) sits in the beam loop's
// straight-line code with the beam's A, B and zone tests, so their chains
// interleave; the tail (the remaining vertices and edges, the closing edge
// back to vertex 0) follows the warp-uniform switch on the vertex count.
// The sums add the edges in order (edge e from vertex e to e + 1, the last
// back to vertex 0); consecutive edges share one reciprocal (rcp_pair).  The
// edge differences are one packed FP32x2 operation each (the same rounding
// as two subtractions: (-1) c_e + c_{e+1} is exact before its single
// rounding).
__device__ __forceinline__ void edge_step_f32(float2 a, float2 b, float slope, float X1, float X2,
                                              float &sr, float &si, float &mn)
{
    const float coef = fmaf(slope, X1, X2);
    const float inv = rcp32(coef);
    mn = fminf(mn, fabsf(coef));
    const float2 df = __ffma2_rn(a, make_float2(-1.f, -1.f), b);
    sr = fmaf(df.x, inv, sr);
    si = fmaf(df.y, inv, si);
}

// 1/a and 1/b from one reciprocal: r = 1/(a b), 1/a = b r, 1/b = a r (one
// MUFU instead of two, three more multiplications).  An edge reaches the hot
// loop's sums only with |a|, |b| > eps (else the pair goes to the FP64 pass),
// so the product does not underflow.  An invalid edge's coefficient (slope
// 1e30: about 1e30 |X1|) overflows the product only when the other one
// exceeds about 3e8; both quotients are then 0 instead of below 1e-30 and
// 3e-9, terms far below the FP32 rounding of the sum.
__device__ __forceinline__ void rcp_pair(float a, float b, float &ia, float &ib)
{
    const float r = rcp32(a * b);
    ia = b * r;
    ib = a * r;
}

// Two consecutive edges (vertex phasors a -> b -> c, slopes sa, sb) with
// one reciprocal for both coefficients; otherwise edge_step_f32 twice.
__device__ __forceinline__ void edge_pair_f32(float2 a, float2 b, float2 c, float sa, float sb, float X1,
                                              float X2, float &sr, float &si, float &mn)
{
    const float ca = fmaf(sa, X1, X2), cb = fmaf(sb, X1, X2);
    float ia, ib;
    rcp_pair(ca, cb, ia, ib);
    mn = fminf(mn, fminf(fabsf(ca), fabsf(cb)));
    const float2 da = __ffma2_rn(a, make_float2(-1.f, -1.f), b);
    const float2 db = __ffma2_rn(b, make_float2(-1.f, -1.f), c);
    sr = fmaf(da.x, ia, sr);
    si = fmaf(da.y, ia, si);
    sr = fmaf(db.x, ib, sr);
    si = fmaf(db.y, ib, si);
}

template <int DPT>
struct EdgeHead {
    float2 c0[DPT], c2[DPT];   // phasors of vertices 0 and 2
    float syx2, sxy2;          // slopes of vertex 2's edge
};

template <int DPT>
__device__ __forceinline__ void edge_head_f32(const SVertRaw<float> *v, const double *st, const double *ct,
                                              const float *X1, const float *X2, const bool *useX,
                                              EdgeHead<DPT> &h, float *sr, float *si, float *mn)
{
    float2 c1[DPT];
    float syx0, sxy0, syx1, sxy1;
    VertRegs w0, w1, w2;
    load_vert(v[0], w0, syx0, sxy0);
    load_vert(v[1], w1, syx1, sxy1);
    load_vert(v[2], w2, h.syx2, h.sxy2);
    // the head's phasors with the reductions of two directions paired (the
    // tail keeps single ones: pairing there too made the step 3 % longer)
    vertex_phasors<DPT>(st, ct, w0, [&](int d, float2 p) { h.c0[d] = p; });
    vertex_phasors<DPT>(st, ct, w1, [&](int d, float2 p) { c1[d] = p; });
    vertex_phasors<DPT>(st, ct, w2, [&](int d, float2 p) { h.c2[d] = p; });
#pragma unroll
    for (int d = 0; d < DPT; ++d) {
        mn[d] = 1e30f;
        sr[d] = 0.f;
        si[d] = 0.f;
        edge_pair_f32(h.c0[d], c1[d], h.c2[d], useX[d] ? syx0 : sxy0, useX[d] ? syx1 : sxy1, X1[d], X2[d],
                      sr[d], si[d], mn[d]);
    }
}

template <int DPT, int NV>
__device__ __forceinline__ void edge_tail_fixed_f32(const SVertRaw<float> *v, const double *st, const double *ct,
                                                    const float *X1, const float *X2, const bool *useX,
                                                    const EdgeHead<DPT> &h, float *sr, float *si, float *mn)
{
    constexpr int kM = NV > 3 ? NV - 3 : 1;
    float2 cs[DPT][kM];
    float syx[kM], sxy[kM];
#pragma unroll
    for (int e = 3; e < NV; ++e) {
        VertRegs w;
        load_vert(v[e], w, syx[e - 3], sxy[e - 3]);
#pragma unroll
        for (int d = 0; d < DPT; ++d)
            vertex_phasor(st[d], ct[d], w, cs[d][e - 3].y, cs[d][e - 3].x);
    }
    // edges in pairs (2, 3), (4, 5); an odd last edge alone
#pragma unroll
    for (int e = 2; e < NV; e += 2) {
#pragma unroll
        for (int d = 0; d < DPT; ++d) {
            const float2 a = e == 2 ? h.c2[d] : cs[d][e - 3];
            const float2 b = e + 1 < NV ? cs[d][e - 2] : h.c0[d];
            const float slope = e == 2 ? (useX[d] ? h.syx2 : h.sxy2)
                                       : (useX[d] ? syx[e - 3] : sxy[e - 3]);
            if (e + 1 < NV) {
                const float2 c = e + 2 < NV ? cs[d][e - 1] : h.c0[d];
                edge_pair_f32(a, b, c, slope, useX[d] ? syx[e - 2] : sxy[e - 2], X1[d], X2[d], sr[d],
                              si[d], mn[d]);
            } else {
                edge_step_f32(a, b, slope, X1[d], X2[d], sr[d], si[d], mn[d]);
            }
        }
    }
}

template <int DPT>
__device__ __forceinline__ void edge_tail_loop_f32(const SVertRaw<float> *v, int nv, const double *st,
                                                   const double *ct, const float *X1, const float *X2,
                                                   const bool *useX, const EdgeHead<DPT> &h, float *sr,
                                                   float *si, float *mn)
{
    float2 prev[DPT];
#pragma unroll
    for (int d = 0; d < DPT; ++d)
        prev[d] = h.c2[d];
    float syx = h.syx2, sxy = h.sxy2;
    for (int e = 2; e < nv; ++e) {
        const bool last = e + 1 == nv;
        const float syx_e = syx, sxy_e = sxy;
        VertRegs w;
        if (!last)
            load_vert(v[e + 1], w, syx, sxy);
#pragma unroll
        for (int d = 0; d < DPT; ++d) {
            float2 nx = h.c0[d];
            if (!last)
                vertex_phasor(st[d], ct[d], w, nx.y, nx.x);
            edge_step_f32(prev[d], nx, useX[d] ? syx_e : sxy_e, X1[d], X2[d], sr[d], si[d], mn[d]);
            prev[d] = nx;
        }
    }
}

template <typename T, int DPT>
__device__ __forceinline__ void edge_sums_loop(const SVertRaw<T> *v, int nv, const double *st,
                                               const double *ct, const T *X1, const T *X2,
                                               const bool *useX, T *sr, T *si, T *mn,
                                               const double2 *tab)
{
    T c0[DPT], s0[DPT], cp_[DPT], sp_[DPT];
    T syx, sxy;
    VertRegs w;
    load_vert(v[0], w, syx, sxy);
#pragma unroll
    for (int d = 0; d < DPT; ++d) {
        vertex_phasor_t(st[d], ct[d], w, tab, s0[d], c0[d]);
        cp_[d] = c0[d];
        sp_[d] = s0[d];
        mn[d] = T(1e30);
        sr[d] = T(0);
        si[d] = T(0);
    }
    for (int e = 0; e < nv; ++e) {
        const bool last = e + 1 == nv;
        const T syx_e = syx, sxy_e = sxy;
        if (!last)
            load_vert(v[e + 1], w, syx, sxy);
#pragma unroll
        for (int d = 0; d < DPT; ++d) {
            T cn = c0[d], sn = s0[d];
            if (!last)
                vertex_phasor_t(st[d], ct[d], w, tab, sn, cn);
            const T coef = fma(useX[d] ? syx_e : sxy_e, X1[d], X2[d]);
            const T inv = rcp_t(coef);
            mn[d] = fmin(mn[d], fabs(coef));
            sr[d] = fma(cn - cp_[d], inv, sr[d]);
            si[d] = fma(sn - sp_[d], inv, si[d]);
            cp_[d] = cn;
            sp_[d] = sn;
        }
    }
}

// FP64 edge sums of one beam (the FP32C path uses edge_head_f32 and the
// tails above): fixed vertex counts unrolled, longer apertures in a loop.
template <typename T, int DPT>
__device__ __forceinline__ void edge_sums(const SVertRaw<T> *v, int nv, const double *st,
                                          const double *ct, const T *X1, const T *X2,
                                          const bool *useX, T *sr, T *si, T *mn,
                                          const double2 *tab)
{
    static_assert(sizeof(T) == 8, "FP64 path");
    switch (nv) {   // warp-uniform: every lane evaluates the same beam
    case 3: edge_sums_fixed<T, DPT, 3>(v, st, ct, X1, X2, useX, sr, si, mn, tab); break;
    case 4: edge_sums_fixed<T, DPT, 4>(v, st, ct, X1, X2, useX, sr, si, mn, tab); break;
    case 5: edge_sums_fixed<T, DPT, 5>(v, st, ct, X1, X2, useX, sr, si, mn, tab); break;
    case 6: edge_sums_fixed<T, DPT, 6>(v, st, ct, X1, X2, useX, sr, si, mn, tab); break;
    default: edge_sums_loop<T, DPT>(v, nv, st, ct, X1, X2, useX, sr, si, mn, tab); break;
    }
}

// The rare pairs of one direction, in FP64: the near-forward moment
// expansion (FP32C), or the complete general evaluation (small-phase
// candidates, nearly singular edges, irregular polar rows).  Writes the
// Jones contribution to the thread's shared-memory slot out[0..7] (stride
// `stride`), so the caller's registers never leave the register file;
// returns false when the beam contributes nothing.
template <typename T>
__device__ __noinline__ bool beam_rare(const KParams &P, int gbeam, const SBeamRaw<T> *sbr, int p,
                                       int t, bool near, T *out, int stride)
{
    constexpr bool kF32 = sizeof(T) == 4;
    const double st = P.st[t], ct = P.ct[t], cp = P.cphi[p], sp = P.sphi[p];
    if (kF32 && near) {
        float sr, si;
        near_forward_s(P.beams[gbeam], P.moments + (size_t)gbeam * kNumMoments, st, ct, cp, sp,
                       P.wc, sr, si);
        T Pm[24];
        load_P(*sbr, Pm);
        const T stT = (T)st, ctT = (T)ct;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const T rr = fma(stT, Pm[16 + 2 * e], fma(ctT, Pm[8 + 2 * e], Pm[2 * e]));
            const T ri = fma(stT, Pm[17 + 2 * e], fma(ctT, Pm[9 + 2 * e], Pm[2 * e + 1]));
            out[(2 * e) * stride] = fma((T)sr, rr, -(T)si * ri);
            out[(2 * e + 1) * stride] = fma((T)sr, ri, (T)si * rr);
        }
        return true;
    }
    DirFull dc;
    dir_full(P, p, t, dc);
    double dd[8];
    const bool ok = beam_general(P.beams[gbeam], P.verts, dc, P.wc, dd);
#pragma unroll
    for (int q = 0; q < 8; ++q)
        out[q * stride] = (T)dd[q];
    return ok;
}

// A pair marked only for a nearly singular edge (|C_e| <= eps): the fast
// path's arithmetic from the shared-memory records, with every edge whose
// |C_e| <= eps taken in the stable form of the same quotient,
//   (e^{i phi_{e+1}} - e^{i phi_e}) / C_e = e^{i phi_e} (e^{iz} - 1) / C_e,
//   z = k C_e delta_e (delta_e: the edge's x or y extent on the branch),
// in FP64 (stable_edge, the reference's singular correction,
// GpuDiffraction.cu:951-970).  The result equals the general evaluation
// (beam_general) without its global-memory walk over the beam; the edge
// extents come from the two vertices' general records.  Writes the Jones
// contribution to out[0..7] (stride `stride`); returns false when the sum
// is not finite, where the general evaluation drops the beam.
template <typename T>
__device__ __noinline__ bool beam_sing(const KParams &P, const SBeamRaw<T> *sbr, const SVertRaw<T> *sv,
                                       int vglob, double st, double ct, T *out, int stride)
{
    constexpr bool kF32 = sizeof(T) == 4;
    BeamRegs<T> b;
    load_beam(*sbr, b);
    const T stT = (T)st, ctT = (T)ct;
    const T A = fma(stT, b.a[0], fma(ctT, b.a[1], b.a[2]));
    const T B = fma(stT, b.a[3], fma(ctT, b.a[4], b.a[5]));
    const bool useX = fabs(B) > fabs(A);
    const T X1 = useX ? B : A, X2 = useX ? A : B;
    const T eps = (T)(kF32 ? P.wc.eps1_f32 : P.wc.eps1);
    const SVertRaw<T> *v = sv + b.vs;
    const DevVert *gv = P.verts + vglob + b.vs;
    VertRegs w;
    T syx, sxy, c0, s0;
    load_vert(v[0], w, syx, sxy);
    vertex_phasor(st, ct, w, s0, c0);
    T cprev = c0, sprev = s0, sr = T(0), si = T(0);
    double dr = 0.0, di = 0.0;
    for (int e = 0; e < b.nv; ++e) {
        const int en = (e + 1 < b.nv) ? e + 1 : 0;
        const T syx_e = syx, sxy_e = sxy;
        T cn = c0, sn = s0;
        if (en != 0) {
            load_vert(v[en], w, syx, sxy);
            vertex_phasor(st, ct, w, sn, cn);
        }
        const T coef = fma(useX ? syx_e : sxy_e, X1, X2);
        if (fabs(coef) > eps) {
            const T inv = rcp_t(coef);
            sr = fma(cn - cprev, inv, sr);
            si = fma(sn - sprev, inv, si);
        } else if (fabs(coef) <= eps) {           // NaN: invalid edge, dropped
            const double delta = useX ? gv[en].x - gv[e].x : gv[en].y - gv[e].y;
            stable_edge((double)cprev, (double)sprev, delta, (double)coef, P.wc.k, dr, di);
        }
        cprev = cn;
        sprev = sn;
    }
    const T m = rcp_t(useX ? B : -A);
    const T s_r = (sr + (T)dr) * m, s_i = (si + (T)di) * m;
    if (!isfinite(s_r) || !isfinite(s_i))
        return false;
    T Pm[24];
    load_P(*sbr, Pm);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const T rr = fma(stT, Pm[16 + 2 * e], fma(ctT, Pm[8 + 2 * e], Pm[2 * e]));
        const T ri = fma(stT, Pm[17 + 2 * e], fma(ctT, Pm[9 + 2 * e], Pm[2 * e + 1]));
        out[(2 * e) * stride] = fma(s_r, rr, -s_i * ri);
        out[(2 * e + 1) * stride] = fma(s_r, ri, s_i * rr);
    }
    return true;
}

// Accumulator of the coherent Jones sum of one orientation for one
// direction.  FP32: plain sums over blocks of kFlushEvery beams in
// registers, folded into a Kahan-compensated running sum kept in shared
// memory (s, c with stride) at every block end.  FP64: plain sums.  Blocks
// of 32 beams: against 16 the step is 1.7 % shorter and the FP32C error
// against FP64 unchanged (it comes from the FP32 trigonometry, not from the
// block sums).
constexpr int kFlushEvery = 32;

template <typename T>
struct JonesAcc {
    T b[8];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < 8; ++i) b[i] = T(0);
    }
    __device__ __forceinline__ void add(const T *d) {
#pragma unroll
        for (int i = 0; i < 8; ++i) b[i] += d[i];
    }
    __device__ __forceinline__ void fold(float *s, float *c, int stride) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float si = s[i * stride], ci = c[i * stride];
            const float y = __fsub_rn((float)b[i], ci);
            const float t = __fadd_rn(si, y);
            c[i * stride] = __fsub_rn(__fsub_rn(t, si), y);
            s[i * stride] = t;
            b[i] = T(0);
        }
    }
};

// Fused diffraction kernel, persistent: each CTA takes work items
// (orientation chunk, azimuth bin, zenith tile) from a global counter.  Each
// thread owns DPT directions of an item (zenith rows t0 + d*TPB of the
// item's azimuth).  T = float selects FP32C.
template <typename T, int TPB, int DPT, bool NS, int MINB>
__global__ void __launch_bounds__(TPB, MINB) po_diffract_kernel(KParams P)
{
    using Cfg = StageCfg<T, TPB>;
    constexpr int kDirs = TPB * DPT;
    constexpr bool kF32 = sizeof(T) == 4;
    constexpr int kSets = NS ? 2 : 1;        // full and no-shadow sums
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SBeamRaw<T> *sb = reinterpret_cast<SBeamRaw<T> *>(smem_raw);
    SVertRaw<T> *sv = reinterpret_cast<SVertRaw<T> *>(smem_raw + Cfg::kBeams * sizeof(SBeamRaw<T>));
    // rare-path result slot per thread: [8][TPB]
    T *rsm = reinterpret_cast<T *>(smem_raw + Cfg::kBytes);
    // FP32C: Kahan running sums of the Jones matrices, [kSets][s, c][8][kDirs]
    float *Ksm = reinterpret_cast<float *>(rsm + 8 * TPB);
    // per thread: bit masks of the stage's pairs for the FP64 pass, [DPT][words][TPB]
    constexpr int kMaskWords = (Cfg::kBeams + 31) / 32;
    uint32_t *rmask = reinterpret_cast<uint32_t *>(Ksm + (kF32 ? kSets * 16 * kDirs : 0));

    const T eps = (T)(kF32 ? P.wc.eps1_f32 : P.wc.eps1);
    T *rslot = rsm + threadIdx.x;
    const int items_per_chunk = P.n_az * P.tiles_per_row;
    __shared__ int s_item;
    __shared__ double s_zdel[TPB / 32];
    __shared__ int s_rwarp[TPB / 32], s_rbase[TPB], s_rok[TPB];   // the spread FP64 pass
    // FP64: sin and cos of the 128 angles 2 pi k / 128 for the vertex phasors
    __shared__ double2 s_sincos[kF32 ? 1 : 128];
    if constexpr (!kF32) {
        for (int i = threadIdx.x; i < 128; i += TPB) {
            double sv_, cv_;
            sincos_turns(i * 0.0078125, sv_, cv_);
            s_sincos[i] = make_double2(sv_, cv_);
        }
    }

    // Persistent: take work items until none are left, so CTAs of uneven
    // cost (rare FP64 pairs, ragged beam counts) balance across the SMs.
    for (;;) {
    __syncthreads();   // the previous item is finished with s_item and the stage
    if (threadIdx.x == 0)
        s_item = atomicAdd(P.work, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= P.n_items)
        break;
    const int chunk = item / items_per_chunk;
    const int pt = item - chunk * items_per_chunk;
    const int p = pt / P.tiles_per_row;
    const int tile = pt - p * P.tiles_per_row;
    int o0, o1;
    chunk_range(P, chunk, o0, o1);
    const double cp = P.cphi[p], sp = P.sphi[p];

    int t[DPT];
    bool active[DPT], general[DPT];
    double st[DPT], ct[DPT];
    T stT[DPT], ctT[DPT];
#pragma unroll
    for (int d = 0; d < DPT; ++d) {
        const int tr = tile * kDirs + d * TPB + threadIdx.x;
        t[d] = tr < P.n_t ? tr : P.n_t - 1;
        const int kind = P.row_kind[t[d]];
        active[d] = tr < P.n_t && kind != 1;
        general[d] = kind == 2;
        st[d] = P.st[t[d]];
        ct[d] = P.ct[t[d]];
        stT[d] = (T)st[d];
        ctT[d] = (T)ct[d];
    }
    float2 st2[DPT], ct2[DPT];   // FP32C: (sin t, sin t), (cos t, cos t) operand pairs
#pragma unroll
    for (int d = 0; d < DPT; ++d) {
        st2[d] = make_float2((float)stT[d], (float)stT[d]);
        ct2[d] = make_float2((float)ctT[d], (float)ctT[d]);
    }
    const size_t G = (size_t)P.n_az * P.n_t;
    // spread of the tile's directions around its middle row, for the zone
    // flags of the stage fill (read there after the fill's first barrier)
    {
        const int tm = min(tile * kDirs + kDirs / 2, P.n_t - 1);
        const double stc = P.st[tm], ctc = P.ct[tm];
        double dd = 0.0;
#pragma unroll
        for (int d = 0; d < DPT; ++d)
            dd = fmax(dd, (st[d] - stc) * (st[d] - stc) + (ct[d] - ctc) * (ct[d] - ctc));
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            dd = fmax(dd, __shfl_xor_sync(0xffffffffu, dd, off));
        if ((threadIdx.x & 31) == 0)
            s_zdel[threadIdx.x >> 5] = dd;
    }

    for (int o = o0; o < o1; ++o) {
        JonesAcc<T> J[DPT], Jn[NS ? DPT : 1];
#pragma unroll
        for (int d = 0; d < DPT; ++d) {
            J[d].zero();
            if (NS) Jn[d].zero();
        }
        if (kF32) {
            for (int i = threadIdx.x; i < kSets * 16 * kDirs; i += TPB)
                Ksm[i] = 0.f;
        }
        const int b0 = P.beam_off[o], b1 = P.beam_off[o + 1];
        for (int bs = b0; bs < b1;) {
            // stage [bs, be): at most kBeams beams and kVerts vertices
            const int vb0 = P.vbeg[bs];
            int be = min(b1, bs + Cfg::kBeams);
            if (P.vbeg[be] - vb0 > Cfg::kVerts) {
                int lo = bs + 1, hi = be;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (P.vbeg[mid] - vb0 <= Cfg::kVerts) lo = mid; else hi = mid - 1;
                }
                be = lo;
            }
            const int nb = be - bs;
            const int nvs = P.vbeg[be] - vb0;
            __syncthreads();   // previous stage fully consumed
            TileZone tz;
            {
                const int tm = min(tile * kDirs + kDirs / 2, P.n_t - 1);
                double dd = 0.0;
#pragma unroll
                for (int w = 0; w < TPB / 32; ++w)
                    dd = fmax(dd, s_zdel[w]);
                tz.stc = P.st[tm];
                tz.ctc = P.ct[tm];
                tz.del = sqrt(dd) * (1.0 + 1e-12);
            }
            for (int i = threadIdx.x; i < nb; i += TPB)
                fill_beam(BrecRef{P.brec + bs + i, P.brec_stride}, cp, sp, P.vbeg[bs + i] - vb0, bs + i, tz,
                          sb[i]);
            for (int i = threadIdx.x; i < nvs; i += TPB)
                fill_vert(VrecRef{P.vrec + vb0 + i, P.vrec_stride}, cp, sp, sv[i]);
            __syncthreads();
            // Hot loop: every (beam, direction) pair on the vectorised path;
            // pairs that need FP64 (near-forward zone, small-phase candidates,
            // nearly singular edges, irregular rows) contribute nothing here
            // and are marked in the thread's bit mask for the pass below.
            uint32_t bits[DPT];
#pragma unroll
            for (int d = 0; d < DPT; ++d)
                bits[d] = 0u;
            // blocks of kFlushEvery beams: the mask store and the Kahan fold
            // run between blocks, not as tests inside the beam loop
            static_assert(32 % kFlushEvery == 0, "mask words hold whole blocks");
            for (int j0 = 0; j0 < nb; j0 += kFlushEvery) {
            const int j1 = min(nb, j0 + kFlushEvery);
            for (int j = j0; j < j1; ++j) {
                BeamRegs<T> b;
                load_beam(sb[j], b);
                T X1[DPT], X2[DPT], sr[DPT], si[DPT], mn[DPT], mden[DPT], Av[DPT], Bv[DPT];
                bool useX[DPT], rare[DPT];
#pragma unroll
                for (int d = 0; d < DPT; ++d) {
                    T A, B;
                    if constexpr (kF32) {
                        const float2 ab = __ffma2_rn(st2[d], make_float2(b.a[0], b.a[3]),
                                                     __ffma2_rn(ct2[d], make_float2(b.a[1], b.a[4]),
                                                                make_float2(b.a[2], b.a[5])));
                        A = ab.x;
                        B = ab.y;
                    } else {
                        A = fma(stT[d], b.a[0], fma(ctT[d], b.a[1], b.a[2]));
                        B = fma(stT[d], b.a[3], fma(ctT[d], b.a[4], b.a[5]));
                    }
                    useX[d] = fabs(B) > fabs(A);
                    X1[d] = useX[d] ? B : A;
                    X2[d] = useX[d] ? A : B;
                    mden[d] = useX[d] ? B : -A;          // x branch: 1/B, y branch: -1/A
                    Av[d] = A;
                    Bv[d] = B;
                    rare[d] = general[d];
                }
                // the zone tests only where the stage fill found the tile
                // may reach the zone (warp-uniform: one beam per iteration)
                if (b.zone) {
#pragma unroll
                    for (int d = 0; d < DPT; ++d) {
                        const T A = Av[d], B = Bv[d];
                        const bool near = kF32 && (float)(A * A + B * B) <= b.nearr2;
                        const bool cand = fabs(fma(A, b.slab[0], B * b.slab[1])) <= T(1)
                                       && fabs(fma(A, b.slab[2], B * b.slab[3])) <= T(1);
                        rare[d] = rare[d] || near || cand;
                    }
                }
                if constexpr (kF32) {
                    EdgeHead<DPT> eh;
                    const SVertRaw<float> *vb = sv + b.vs;
                    edge_head_f32<DPT>(vb, st, ct, X1, X2, useX, eh, sr, si, mn);
                    switch (b.nv) {   // warp-uniform: every lane evaluates the same beam
                    case 3: edge_tail_fixed_f32<DPT, 3>(vb, st, ct, X1, X2, useX, eh, sr, si, mn); break;
                    case 4: edge_tail_fixed_f32<DPT, 4>(vb, st, ct, X1, X2, useX, eh, sr, si, mn); break;
                    case 5: edge_tail_fixed_f32<DPT, 5>(vb, st, ct, X1, X2, useX, eh, sr, si, mn); break;
                    case 6: edge_tail_fixed_f32<DPT, 6>(vb, st, ct, X1, X2, useX, eh, sr, si, mn); break;
                    default: edge_tail_loop_f32<DPT>(vb, b.nv, st, ct, X1, X2, useX, eh, sr, si, mn); break;
                    }
                } else {
                    edge_sums<T, DPT>(sv + b.vs, b.nv, st, ct, X1, X2, useX, sr, si, mn, s_sincos);
                }
                T s_r[DPT], s_i[DPT];
#pragma unroll
                for (int d = 0; d < DPT; ++d) {
                    rare[d] = (rare[d] || mn[d] <= eps) && active[d];
                    bits[d] |= (rare[d] ? 1u : 0u) << (j & 31);
                    // select, not multiply: a marked pair may hold inf or NaN sums
                    const T m = rcp_t(mden[d]);
                    s_r[d] = rare[d] ? T(0) : sr[d] * m;
                    s_i[d] = rare[d] ? T(0) : si[d] * m;
                }
                const T fi = (NS && !(P.beams[b.gbeam].flags & MBS_PO_BEAM_EXTERNAL)) ? T(1) : T(0);
                // J += s x (P0 + cos t Pc + sin t Ps), two complex entries at a time
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if constexpr (kF32 && !NS) {
                        // entries 2h and 2h+1 side by side: R = P0 + cos t Pc + sin t Ps
                        // as (re, re) and (im, im) pairs, then J_re += -s_i R_i + s_r R_r
                        // and J_im += s_i R_r + s_r R_i, the scalar form's operations
                        // lane by lane (no operand pair needs its halves swapped)
                        float2 p0r, p0i, pcr, pci, psr, psi;
                        load_P_packed(sb[j], h, p0r, p0i, pcr, pci, psr, psi);
#pragma unroll
                        for (int d = 0; d < DPT; ++d) {
                            const float2 srr = make_float2(s_r[d], s_r[d]);
                            const float2 sii = make_float2(s_i[d], s_i[d]);
                            const float2 nsi = make_float2(-s_i[d], -s_i[d]);
                            const float2 Rr = __ffma2_rn(st2[d], psr, __ffma2_rn(ct2[d], pcr, p0r));
                            const float2 Ri = __ffma2_rn(st2[d], psi, __ffma2_rn(ct2[d], pci, p0i));
                            float2 jr = make_float2(J[d].b[4 * h], J[d].b[4 * h + 2]);
                            float2 ji = make_float2(J[d].b[4 * h + 1], J[d].b[4 * h + 3]);
                            jr = __ffma2_rn(nsi, Ri, jr);
                            jr = __ffma2_rn(srr, Rr, jr);
                            ji = __ffma2_rn(sii, Rr, ji);
                            ji = __ffma2_rn(srr, Ri, ji);
                            J[d].b[4 * h] = jr.x;
                            J[d].b[4 * h + 2] = jr.y;
                            J[d].b[4 * h + 1] = ji.x;
                            J[d].b[4 * h + 3] = ji.y;
                        }
                    } else {
                        T p0[4], pc[4], ps[4];
                        load_P_pair(sb[j], h, p0, pc, ps);
#pragma unroll
                        for (int d = 0; d < DPT; ++d) {
#pragma unroll
                            for (int e = 0; e < 2; ++e) {
                                const int q = 4 * h + 2 * e;
                                const T rr = fma(stT[d], ps[2 * e], fma(ctT[d], pc[2 * e], p0[2 * e]));
                                const T ri = fma(stT[d], ps[2 * e + 1], fma(ctT[d], pc[2 * e + 1], p0[2 * e + 1]));
                                J[d].b[q] = fma(s_r[d], rr, fma(-s_i[d], ri, J[d].b[q]));
                                J[d].b[q + 1] = fma(s_r[d], ri, fma(s_i[d], rr, J[d].b[q + 1]));
                                if (NS) {
                                    Jn[NS ? d : 0].b[q] = fma(fi * s_r[d], rr, fma(-fi * s_i[d], ri, Jn[NS ? d : 0].b[q]));
                                    Jn[NS ? d : 0].b[q + 1] = fma(fi * s_r[d], ri, fma(fi * s_i[d], rr, Jn[NS ? d : 0].b[q + 1]));
                                }
                            }
                        }
                    }
                }
            }
            if ((j1 & 31) == 0 || j1 == nb) {
#pragma unroll
                for (int d = 0; d < DPT; ++d) {
                    rmask[(d * kMaskWords + ((j1 - 1) >> 5)) * TPB + threadIdx.x] = bits[d];
                    bits[d] = 0u;
                }
            }
            if (kF32 && j1 - j0 == kFlushEvery) {
#pragma unroll
                for (int d = 0; d < DPT; ++d) {
                    const int slot = d * TPB + threadIdx.x;
                    J[d].fold(Ksm + slot, Ksm + 8 * kDirs + slot, kDirs);
                    if (NS)
                        Jn[NS ? d : 0].fold(Ksm + 16 * kDirs + slot, Ksm + 24 * kDirs + slot, kDirs);
                }
            }
            }
            // FP64 pass over the stage's marked pairs, spread over all the
            // CTA's threads: a pair's owner (the thread whose direction it
            // is) seldom has company in its warp, so per-owner loops left most
            // lanes idle and the CTA waiting at the next stage for its
            // busiest warp.  The marked pairs are numbered owner by owner in
            // the owners' (direction, beam) order; in rounds of TPB, thread i
            // evaluates pair r0 + i into its result slot, then every owner
            // adds its own results in that order, the order of a per-owner
            // loop, so the sums are the same bit for bit.
            {
                const int words = (nb + 31) >> 5;
                const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
                int cnt = 0;
#pragma unroll
                for (int d = 0; d < DPT; ++d)
                    for (int w = 0; w < words; ++w)
                        cnt += __popc(rmask[(d * kMaskWords + w) * TPB + threadIdx.x]);
                int incl = cnt;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, incl, off);
                    if (lane >= off)
                        incl += v;
                }
                if (lane == 31)
                    s_rwarp[warp] = incl;
                __syncthreads();   // the warp totals and every thread's masks are visible
                int base = incl - cnt, total = 0;
#pragma unroll
                for (int w2 = 0; w2 < TPB / 32; ++w2) {
                    const int v = s_rwarp[w2];
                    base += w2 < warp ? v : 0;
                    total += v;
                }
                s_rbase[threadIdx.x] = base;
                __syncthreads();
                // the owner's cursor over its own marked pairs
                int cd = 0, cw = 0;
                uint32_t cm = words > 0 ? rmask[threadIdx.x] : 0u;
                for (int r0 = 0; r0 < total; r0 += TPB) {
                    const int q = r0 + threadIdx.x;
                    int okv = 0;
                    if (q < total) {
                        int lo = 0, hi = TPB - 1;   // owner: the last o with s_rbase[o] <= q
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (s_rbase[mid] <= q) lo = mid; else hi = mid - 1;
                        }
                        const int o = lo;
                        int k = q - s_rbase[o], od = 0, j = 0;
                        bool found = false;
                        for (int d2 = 0; d2 < DPT && !found; ++d2)
                            for (int w = 0; w < words && !found; ++w) {
                                uint32_t m = rmask[(d2 * kMaskWords + w) * TPB + o];
                                const int c = __popc(m);
                                if (k < c) {
                                    for (int i = 0; i < k; ++i)
                                        m &= m - 1;
                                    j = w * 32 + __ffs(m) - 1;
                                    od = d2;
                                    found = true;
                                } else {
                                    k -= c;
                                }
                            }
                        const int to = tile * kDirs + od * TPB + o;   // < n_t: marked pairs are active
                        const double sto = P.st[to], cto = P.ct[to];
                        const bool gen = P.row_kind[to] == 2;
                        const T stTo = (T)sto, ctTo = (T)cto;
                        BeamRegs<T> b;
                        load_beam(sb[j], b);
                        const T A = fma(stTo, b.a[0], fma(ctTo, b.a[1], b.a[2]));
                        const T B = fma(stTo, b.a[3], fma(ctTo, b.a[4], b.a[5]));
                        const bool near = kF32 && !gen && (float)(A * A + B * B) <= b.nearr2;
                        const bool cand = fabs(fma(A, b.slab[0], B * b.slab[1])) <= T(1)
                                       && fabs(fma(A, b.slab[2], B * b.slab[3])) <= T(1);
                        okv = ((gen || near || cand)
                                   ? beam_rare<T>(P, b.gbeam, &sb[j], p, to, near, rslot, TPB)
                                   : beam_sing<T>(P, &sb[j], sv, vb0, sto, cto, rslot, TPB)) ? 1 : 0;
                    }
                    s_rok[threadIdx.x] = okv;
                    __syncthreads();   // this round's results are in the slots
                    const int q0 = max(base, r0), q1 = min(base + cnt, r0 + TPB);
                    for (int qq = q0; qq < q1; ++qq) {
                        while (cm == 0u) {
                            if (++cw == words) {
                                cw = 0;
                                ++cd;
                            }
                            cm = rmask[(cd * kMaskWords + cw) * TPB + threadIdx.x];
                        }
                        const int j = cw * 32 + __ffs(cm) - 1;
                        cm &= cm - 1;
                        const int slot = qq - r0;
                        if (s_rok[slot]) {
                            T dj[8];
#pragma unroll
                            for (int i = 0; i < 8; ++i)
                                dj[i] = rsm[slot + i * TPB];
#pragma unroll
                            for (int d2 = 0; d2 < DPT; ++d2)
                                if (d2 == cd) {
                                    J[d2].add(dj);
                                    if (NS) {
                                        BeamRegs<T> bj;
                                        load_beam(sb[j], bj);
                                        if (!(P.beams[bj.gbeam].flags & MBS_PO_BEAM_EXTERNAL))
                                            Jn[NS ? d2 : 0].add(dj);
                                    }
                                }
                        }
                    }
                    __syncthreads();   // the slots are read before the next round
                }
            }
            if (kF32) {
#pragma unroll
                for (int d = 0; d < DPT; ++d) {
                    const int slot = d * TPB + threadIdx.x;
                    J[d].fold(Ksm + slot, Ksm + 8 * kDirs + slot, kDirs);
                    if (NS)
                        Jn[NS ? d : 0].fold(Ksm + 16 * kDirs + slot, Ksm + 24 * kDirs + slot, kDirs);
                }
            }
            bs = be;
        }
        // Mueller of this orientation, weighted, added to the chunk's
        // partial plane in global memory (coalesced: consecutive threads
        // own consecutive directions; the first orientation initialises).
        // The adds are reductions performed in L2 (no load on the thread's
        // path); each partial element has a single owner thread, whose adds
        // reach it in program order, so the sums are deterministic.
        const double wgt = P.weight[o] * 0.25;
#pragma unroll
        for (int d = 0; d < DPT; ++d) {
            if (!active[d])
                continue;
            const int slot = d * TPB + threadIdx.x;
            const size_t g = (size_t)p * P.n_t + t[d];
            for (int set = 0; set < kSets; ++set) {
                double j[8];
                if (kF32) {
                    const float *s = Ksm + set * 16 * kDirs + slot;
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        j[i] = (double)s[i * kDirs] - (double)s[(8 + i) * kDirs];
                } else {
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        j[i] = (double)(set == 0 ? J[d].b[i] : Jn[NS ? d : 0].b[i]);
                }
                double m[16];
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    m[i] = 0.0;
                mueller_add(j, wgt, m);
                double *out = (set == 0 ? P.partial : P.partial_ns) + (size_t)chunk * 16 * G + g;
                if (o == o0) {
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                        out[i * G] = m[i];
                } else {
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                        atomicAdd(out + i * G, m[i]);
                }
            }
        }
    }
    }   // work items
}

template <typename T, int TPB, int DPT, bool NS>
constexpr size_t diffract_smem_bytes()
{
    return StageCfg<T, TPB>::kBytes + 8 * TPB * sizeof(T)
         + (sizeof(T) == 4 ? (NS ? 2 : 1) * 16 * TPB * DPT * sizeof(float) : 0)
         + (size_t)DPT * ((StageCfg<T, TPB>::kBeams + 31) / 32) * TPB * sizeof(uint32_t);
}

// Polar zenith rows (row_kind 1): every azimuth bin has the same direction
// and polarisation basis there (Handler.h:147-160), so the row is evaluated
// once per orientation in FP64 and written to all azimuth bins.  Grid:
// x = orientation chunk, y = polar row index; threads stride over the
// chunk's orientations, then a fixed-order tree sums them.
template <bool NS>
__global__ void __launch_bounds__(256) po_pole_kernel(KParams P, const int32_t *pole_rows)
{
    __shared__ double red[256];
    const int chunk = blockIdx.x;
    const int t = pole_rows[blockIdx.y];
    int o0, o1;
    chunk_range(P, chunk, o0, o1);
    DirFull dc;
    dir_full(P, 0, t, dc);
    double M[16], Mn[NS ? 16 : 1];
#pragma unroll
    for (int i = 0; i < 16; ++i) M[i] = 0.0;
    if (NS) {
#pragma unroll
        for (int i = 0; i < (NS ? 16 : 1); ++i) Mn[i] = 0.0;
    }
    for (int o = o0 + threadIdx.x; o < o1; o += blockDim.x) {
        double J[8] = {0, 0, 0, 0, 0, 0, 0, 0}, Jn[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int b = P.beam_off[o]; b < P.beam_off[o + 1]; ++b) {
            double d[8];
            if (beam_general(P.beams[b], P.verts, dc, P.wc, d)) {
                for (int q = 0; q < 8; ++q) J[q] += d[q];
                if (NS && !(P.beams[b].flags & MBS_PO_BEAM_EXTERNAL))
                    for (int q = 0; q < 8; ++q) Jn[q] += d[q];
            }
        }
        const double wgt = P.weight[o] * 0.25;
        mueller_add(J, wgt, M);
        if (NS)
            mueller_add(Jn, wgt, Mn);
    }
    const size_t G = (size_t)P.n_az * P.n_t;
    for (int set = 0; set < (NS ? 2 : 1); ++set) {
        double *out = (set == 0 ? P.partial : P.partial_ns) + (size_t)chunk * 16 * G;
        for (int i = 0; i < 16; ++i) {
            red[threadIdx.x] = set == 0 ? M[i] : Mn[NS ? i : 0];
            __syncthreads();
            for (int s = blockDim.x / 2; s > 0; s >>= 1) {
                if ((int)threadIdx.x < s)
                    red[threadIdx.x] += red[threadIdx.x + s];
                __syncthreads();
            }
            const double v = red[0];
            for (int pp = threadIdx.x; pp < P.n_az; pp += blockDim.x)
                out[(size_t)i * G + (size_t)pp * P.n_t + t] = v;
            __syncthreads();
        }
    }
}

// out[set][g*16+k] += sum_c partial[set chunks c][k][g], in chunk order
// (deterministic).  Grid: x over 16 G, y = output set.
__global__ void po_reduce_kernel(const double *__restrict__ partial, int chunks_per_set,
                                 int64_t G, double *__restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G * 16)
        return;
    const int set = blockIdx.y;
    partial += (int64_t)set * chunks_per_set * 16 * G;
    out += (int64_t)set * 16 * G;
    const int64_t k = i / G, g = i - k * G;
    double s = 0.0;
    for (int c = 0; c < chunks_per_set; ++c)
        s += partial[(int64_t)c * 16 * G + i];
    out[g * 16 + k] += s;
}

// Azimuth interpolation of a Mueller grid (the FFT-phi path): for every output
// azimuth p, out[p][r] += sum_m W[p][m] low[m][r], r running over the
// (zenith row, element) entries of one azimuth plane (plane = rows * 16
// doubles, coalesced across the block).  W [n_full][n_low] is the linear map
// of the zero-padded DFT upsampling (see phi_weights on the host); the
// block keeps its output azimuth's row of W in shared memory.
__global__ void __launch_bounds__(256) po_phi_interp_kernel(const double *__restrict__ low,
                                                            const double *__restrict__ W, int n_low,
                                                            int64_t plane, double *__restrict__ out)
{
    extern __shared__ double w_row[];
    const int p = blockIdx.y;
    for (int m = threadIdx.x; m < n_low; m += blockDim.x)
        w_row[m] = W[(size_t)p * n_low + m];
    __syncthreads();
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= plane)
        return;
    double acc = 0.0;
    for (int m = 0; m < n_low; ++m)
        acc = fma(w_row[m], low[(size_t)m * plane + r], acc);
    out[(size_t)p * plane + r] += acc;
}

// ------------------------------------------------------- azimuth average
// Per zenith row t the azimuth average of M(p, t) L(2 az_p), az_p = -p 2 pi / n_az
// (L the Stokes rotation [1 0 0 0; 0 c s 0; 0 -s c 0; 0 0 0 1]), the polar
// rows unrotated and projected (PoleMueller ApplyForward / ApplyBackward),
// as HandlerPOTotal::WriteMatricesToFile writes them (reference
// src/handler/HandlerPOTotal.cpp:49-96).  One CTA per row (grid y: one
// Mueller grid after another); threads stride over azimuth bins, fixed-order
// tree sum (deterministic).  rows[y][t][16].
__global__ void __launch_bounds__(128) po_phi_average_kernel(const double *__restrict__ M, int n_az,
                                                            int n_t, const double *__restrict__ theta,
                                                            double *__restrict__ rows)
{
    __shared__ double red[16][128];
    const int t = blockIdx.x;
    // y: independent grids (one per orientation for per-orientation rows)
    M += (size_t)blockIdx.y * n_az * n_t * 16;
    rows += (size_t)blockIdx.y * n_t * 16;
    const double th = theta[t];
    const double tol = 256.0 * 2.220446049250313e-16;   // PoleMueller angular tolerance
    const bool fwd = fabs(th) <= tol;
    const bool bwd = fabs(th - kPi) <= tol;
    double S[16];
#pragma unroll
    for (int q = 0; q < 16; ++q)
        S[q] = 0.0;
    for (int p = threadIdx.x; p < n_az; p += blockDim.x) {
        const double *m = M + ((size_t)p * n_t + t) * 16;
        if (fwd || bwd) {
#pragma unroll
            for (int q = 0; q < 16; ++q)
                S[q] += m[q];
            continue;
        }
        double sn, c;
        sincos(2.0 * (-p * (2.0 * kPi / n_az)), &sn, &c);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const double m0 = m[4 * r], m1 = m[4 * r + 1], m2 = m[4 * r + 2], m3 = m[4 * r + 3];
            S[4 * r + 0] += m0;
            S[4 * r + 1] += m1 * c - m2 * sn;
            S[4 * r + 2] += m1 * sn + m2 * c;
            S[4 * r + 3] += m3;
        }
    }
#pragma unroll
    for (int q = 0; q < 16; ++q)
        red[q][threadIdx.x] = S[q];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < 16; ++q)
                red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double R[16];
        for (int q = 0; q < 16; ++q)
            R[q] = red[q][0] / n_az;
        if (fwd || bwd) {
            const double M00 = R[0], M33 = R[15], M03 = R[3];
            const double M11 = bwd ? 0.5 * (R[5] - R[10]) : 0.5 * (R[5] + R[10]);
            for (int q = 0; q < 16; ++q)
                R[q] = 0.0;
            R[0] = M00; R[5] = M11; R[10] = bwd ? -M11 : M11; R[15] = M33;
            R[3] = M03; R[12] = M03;
        }
        for (int q = 0; q < 16; ++q)
            rows[(size_t)t * 16 + q] = R[q];
    }
}

// Scattering cross-section sum_t M11(t) dcos2pi(t) and the asymmetry
// parameter g = sum_t cos(theta_t) M11(t) dcos2pi(t) / that sum over the
// averaged rows.  One CTA, fixed-order tree sum; out[0] = C_sca, out[1] = g.
__global__ void __launch_bounds__(256) po_csca_kernel(const double *__restrict__ rows, int n_t,
                                                     const double *__restrict__ theta,
                                                     const double *__restrict__ dcos2pi,
                                                     double *__restrict__ out)
{
    __shared__ double a[256], b[256];
    double sa = 0.0, sb = 0.0;
    for (int t = threadIdx.x; t < n_t; t += blockDim.x) {
        const double v = rows[(size_t)t * 16] * dcos2pi[t];
        sa += v;
        sb += cos(theta[t]) * v;
    }
    a[threadIdx.x] = sa;
    b[threadIdx.x] = sb;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            a[threadIdx.x] += a[threadIdx.x + w];
            b[threadIdx.x] += b[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = a[0];
        out[1] = a[0] != 0.0 ? b[0] / a[0] : 0.0;
    }
}

// ------------------------------------------------------------ theta scan
// Incoherent, azimuth-summed M11 on a list of zenith angles (reference
// theta_m11_kernel, GpuDiffraction.cu:1909-1956, called by DiffractThetasGpu
// :4780-4970).  Grid: x = zenith point, y = beam chunk; the CTA strides over
// (beam, azimuth bin) pairs of its chunk and sums in a fixed-order tree, so
// out_partial[chunk][t] is deterministic.
__global__ void __launch_bounds__(256) po_thetas_kernel(
    const DevBeam *beams, const DevVert *verts, const int32_t *beam_off, const double *weight,
    int n_orient, int64_t n_beams, int beams_per_chunk, const double *st, const double *ct,
    const double *sphi, const double *cphi, int n_az, int n_points, WaveConst wc,
    double *out_partial)
{
    __shared__ double red[256];
    const int t = blockIdx.x;
    const int64_t b0 = (int64_t)blockIdx.y * beams_per_chunk;
    const int64_t b1 = min(n_beams, b0 + beams_per_chunk);
    const int64_t pairs = (b1 - b0) * n_az;
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < pairs; i += blockDim.x) {
        const int64_t b = b0 + i / n_az;
        const int p = (int)(i - (b - b0) * n_az);
        // orientation of beam b: last o with beam_off[o] <= b
        int lo = 0, hi = n_orient;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (beam_off[mid] <= b) lo = mid; else hi = mid;
        }
        DirFull dc;
        dc.st = st[t];
        dc.ct = ct[t];
        dc.cp = cphi[p];
        dc.sp = sphi[p];
        dc.dir[0] = dc.st * dc.cp;
        dc.dir[1] = dc.st * dc.sp;
        dc.dir[2] = -dc.ct;
        dc.vf[0] = -dc.sp; dc.vf[1] = dc.cp; dc.vf[2] = 0.0;
        cross3(dc.vf, dc.dir, dc.u);
        const double l2 = dc.u[0] * dc.u[0] + dc.u[1] * dc.u[1] + dc.u[2] * dc.u[2];
        const double il = (l2 > 1e-30) ? rsqrt(l2) : 1.0;
        dc.vt[0] = dc.u[0] * il; dc.vt[1] = dc.u[1] * il; dc.vt[2] = dc.u[2] * il;
        cross3(dc.vt, dc.dir, dc.w);
        double d[8];
        if (beam_general(beams[b], verts, dc, wc, d, false)) {
            double e = 0.0;
#pragma unroll
            for (int q = 0; q < 8; ++q)
                e = fma(d[q], d[q], e);
            acc += 0.5 * e * weight[lo] / (double)(n_az + 1);
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        out_partial[(size_t)blockIdx.y * n_points + t] = red[0];
}

// m11[t] = sum over chunks of partial[c][t], chunk order.
__global__ void po_thetas_sum_kernel(const double *partial, int n_chunks, int n_points, double *m11)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_points)
        return;
    double s = 0.0;
    for (int c = 0; c < n_chunks; ++c)
        s += partial[(size_t)c * n_points + t];
    m11[t] = s;
}

// --------------------------------------------------------- extinction
// One thread per orientation: HandlerPO::ComputeForwardExtinctionOt
// (reference HandlerPO.cpp:1812-2009) at zenith 0, azimuth 0.
__global__ void po_extinction_kernel(const DevBeam *beams, const DevVert *verts,
                                     const int32_t *beam_off, const double *weight,
                                     int n_orient, WaveConst wc, double *cext)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n_orient)
        return;
    const double k = wc.k;
    DirFull dc;
    dc.st = 0.0; dc.ct = 1.0; dc.cp = 1.0; dc.sp = 0.0;
    dc.dir[0] = 0.0; dc.dir[1] = 0.0; dc.dir[2] = -1.0;
    dc.vf[0] = 0.0; dc.vf[1] = 1.0; dc.vf[2] = 0.0;
    cross3(dc.vf, dc.dir, dc.u);
    dc.vt[0] = dc.u[0]; dc.vt[1] = dc.u[1]; dc.vt[2] = dc.u[2];
    cross3(dc.vt, dc.dir, dc.w);
    double f00r = 0, f00i = 0, f11r = 0, f11i = 0;
    for (int b = beam_off[o]; b < beam_off[o + 1]; ++b) {
        DevBeam g = beams[b];
        const bool external = (g.flags & MBS_PO_BEAM_EXTERNAL) != 0;
        if (wc.ot_phase_avg && !external)
            continue;
        // The extinction phase reference differs from the scattering one
        // (HandlerPO.cpp:1965-1977): external beams take exp(-ik opticalPath),
        // internal ones exp(-ik(cos t dp_cos + farReference)).  beam_general
        // is run on a copy flagged external (no common phase), and the
        // reference's factor is applied here.
        const double ref = external ? g.opath : wc.ot_far_ref;
        g.flags |= MBS_PO_BEAM_EXTERNAL;
        // The reference drops beams whose 1/A or 1/B divisor is nearly
        // singular at this direction (HandlerPO.cpp:1920-1921, 1945-1946).
        const double A = g.h[2] + g.a0, B = g.v[2] + g.b0;
        double dd[8], pr, pi;
        const bool small = small_phase_factor(verts + g.vbeg, g.nv, A, B, k, pr, pi);
        if (!small && ((fabs(B) > fabs(A)) ? fabs(B) <= wc.eps1 : fabs(A) <= wc.eps1))
            continue;
        if (!beam_general(g, verts, dc, wc, dd))
            continue;
        double ph = 0.0;
        if (!external)
            ph = -k * (1.0 * (-g.c[2]) + ref);
        else if (ref != 0.0)
            ph = -k * ref;
        double s = 0.0, c = 1.0;
        if (ph != 0.0)
            sincos_rad(ph, s, c);
        // the CPU rotation carries 0.5 (HandlerPO_fast.h:643-646)
        f00r += 0.5 * (dd[0] * c - dd[1] * s); f00i += 0.5 * (dd[0] * s + dd[1] * c);
        f11r += 0.5 * (dd[6] * c - dd[7] * s); f11i += 0.5 * (dd[6] * s + dd[7] * c);
    }
    const double fwr = f00r + f11r, fwi = f00i + f11i;
    double amp = fwi;
    if (wc.ot_ping != 0.0) {
        double sn, cs;
        sincos_rad(2.0 * k * wc.ot_ping, sn, cs);
        amp = fwi * cs - fwr * sn;
    }
    const double cv = wc.wavelength * amp * weight[o];
    cext[o] = isfinite(cv) ? cv : 0.0;
}

// ------------------------------------------------------------ peak probe
// Independent FFMA chains: this device's FP32 FMA throughput, the
// denominator of the diffraction kernels' roofline fraction.
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

// Independent DFMA chains: this device's FP64 FMA throughput, the
// denominator of the FP64 diffraction kernel's roofline fraction.
__global__ void __launch_bounds__(256) po_fp64_probe_kernel(double *out, int iters, double a, double b)
{
    double x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
        x[i] = threadIdx.x * 1e-3 + i;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
#pragma unroll
            for (int i = 0; i < 8; ++i)
                x[i] = fma(x[i], a, b);
        }
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
        s += x[i];
    if (s == 1234.5)
        out[blockIdx.x] = s;
}

}  // namespace mbs
