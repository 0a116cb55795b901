/*
 * po_oracle.c — TEST INFRASTRUCTURE (the checker), not product code.
 *
 * Plain-C double-precision restatement of MBS-fast's CPU PO diffraction path
 * on the flat mbs_po_beams batch.  Each function cites the reference code it
 * restates.  Trigonometry uses libm sincos() where the reference uses its own
 * AVX polynomial (HandlerPO_fast.h:116-146), so results agree with the
 * reference to rounding (checked in tests/test_oracle_pin.py), not bit for bit.
 */
#define _GNU_SOURCE
#include "po_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cplx;

static inline cplx cmul(cplx a, cplx b)
{
    cplx r = { a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re };
    return r;
}

/* small_phase_polygon_factor (HandlerPO_fast.h:161-226). */
static int small_phase_factor(const double *vx, const double *vy, int nv,
                              double A, double B, double k,
                              double *fr, double *fi)
{
    if (nv < 3)
        return 0;
    const double qx = k * A, qy = k * B;
    double maxPhase = 0.0;
    for (int i = 0; i < nv; ++i)
    {
        const double ph = fabs(qx * vx[i] + qy * vy[i]);
        if (ph > maxPhase)
            maxPhase = ph;
    }
    if (maxPhase > 1e-3)
        return 0;
    double twiceArea = 0, fx6 = 0, fy6 = 0, sx12 = 0, sy12 = 0, sxy24 = 0;
    double minX = DBL_MAX, maxX = -DBL_MAX, minY = DBL_MAX, maxY = -DBL_MAX;
    for (int i = 0; i < nv; ++i)
    {
        const int j = (i + 1 < nv) ? i + 1 : 0;
        const double xi = vx[i], yi = vy[i], xj = vx[j], yj = vy[j];
        const double cross = xi * yj - xj * yi;
        twiceArea += cross;
        fx6 += (xi + xj) * cross;
        fy6 += (yi + yj) * cross;
        sx12 += (xi * xi + xi * xj + xj * xj) * cross;
        sy12 += (yi * yi + yi * yj + yj * yj) * cross;
        sxy24 += (2.0 * xi * yi + xi * yj + xj * yi + 2.0 * xj * yj) * cross;
        if (xi < minX) minX = xi;
        if (xi > maxX) maxX = xi;
        if (yi < minY) minY = yi;
        if (yi > maxY) maxY = yi;
    }
    double areaScale = (maxX - minX) * (maxY - minY);
    if (areaScale < DBL_MIN)
        areaScale = DBL_MIN;
    if (fabs(twiceArea) <= 0x1p-40 * areaScale)
    {
        *fr = 1.0;
        *fi = 0.0;
        return 1;
    }
    const double invArea = 2.0 / twiceArea;
    const double mX = (fx6 / 6.0) * invArea, mY = (fy6 / 6.0) * invArea;
    const double mXX = (sx12 / 12.0) * invArea, mYY = (sy12 / 12.0) * invArea;
    const double mXY = (sxy24 / 24.0) * invArea;
    const double mp = qx * mX + qy * mY;
    const double mp2 = qx * qx * mXX + 2.0 * qx * qy * mXY + qy * qy * mYY;
    *fr = 1.0 - 0.5 * mp2;
    *fi = mp;
    return 1;
}

static inline double stable_sinc(double x)
{   /* HandlerPO_fast.h:228-237 */
    if (fabs(x) < 1e-4)
    {
        const double x2 = x * x;
        return 1.0 - x2 / 6.0 + x2 * x2 / 120.0;
    }
    return sin(x) / x;
}

/* add_stable_edge_quotient (HandlerPO_fast.h:242-257). */
static inline void stable_edge(double pr, double pi, double delta, double c,
                               double k, double *sr, double *si)
{
    const double z = k * c * delta;
    const double sh = stable_sinc(0.5 * z);
    const double lr = -0.5 * k * k * c * delta * delta * sh * sh;
    const double li = k * delta * stable_sinc(z);
    *sr += pr * lr - pi * li;
    *si += pr * li + pi * lr;
}

/* Aperture integral of one beam for one direction: the small-phase branch,
 * else the edge sum over precomputed vertex phasors (HandlerPO.cpp:2675-2739). */
static cplx aperture(const mbs_po_beams *b, int64_t v0, int nv, double A, double B,
                     const double *vc, const double *vs, double area,
                     const mbs_po_wave *w, int singular)
{
    const double k = w->wave_index;
    double fr, fi;
    cplx F;
    if (small_phase_factor(b->vx + v0, b->vy + v0, nv, A, B, k, &fr, &fi))
    {
        const double sgn = w->legacy_sign ? 1.0 : -1.0;
        const cplx areaLimit = { sgn * w->inv_compl_wave_re * area,
                                 sgn * w->inv_compl_wave_im * area };
        const cplx f = { fr, fi };
        return cmul(areaLimit, f);
    }
    double sr = 0, si = 0;
    if (fabs(B) > fabs(A))
    {
        for (int e = 0; e < nv; ++e)
        {
            if (!(b->edge_flags[v0 + e] & MBS_PO_EDGE_VALID_X))
                continue;
            const int en = (e + 1 < nv) ? e + 1 : 0;
            const double Ci = A + b->slope_yx[v0 + e] * B;
            const double inv = (fabs(Ci) > w->eps1) ? 1.0 / Ci : 0.0;
            sr += (vc[en] - vc[e]) * inv;
            si += (vs[en] - vs[e]) * inv;
            if (singular && fabs(Ci) <= w->eps1)
                stable_edge(vc[e], vs[e], b->vx[v0 + en] - b->vx[v0 + e], Ci, k, &sr, &si);
        }
        const double invB = 1.0 / B;
        sr *= invB;
        si *= invB;
    }
    else
    {
        for (int e = 0; e < nv; ++e)
        {
            if (!(b->edge_flags[v0 + e] & MBS_PO_EDGE_VALID_Y))
                continue;
            const int en = (e + 1 < nv) ? e + 1 : 0;
            const double Ei = A * b->slope_xy[v0 + e] + B;
            const double inv = (fabs(Ei) > w->eps1) ? 1.0 / Ei : 0.0;
            sr += (vc[en] - vc[e]) * inv;
            si += (vs[en] - vs[e]) * inv;
            if (singular && fabs(Ei) <= w->eps1)
                stable_edge(vc[e], vs[e], b->vy[v0 + en] - b->vy[v0 + e], Ei, k, &sr, &si);
        }
        const double invNA = -1.0 / A;
        sr *= invNA;
        si *= invNA;
    }
    const cplx cw = { w->compl_wave_re, w->compl_wave_im };
    const cplx s = { sr, si };
    F = cmul(cw, s);
    return F;
}

/* rotate_jones_inline (HandlerPO_fast.h:600-683), including the 0.5. */
static void rotate_jones(const double *g, const double *vf, const double *dir,
                         double *r)
{
    double vt[3] = { vf[1] * dir[2] - vf[2] * dir[1],
                     vf[2] * dir[0] - vf[0] * dir[2],
                     vf[0] * dir[1] - vf[1] * dir[0] };
    const double l2 = vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2];
    if (l2 > 1e-30)
    {
        const double il = 1.0 / sqrt(l2);
        vt[0] *= il; vt[1] *= il; vt[2] *= il;
    }
    const double *NT = g + MBS_PO_G_NT, *NP = g + MBS_PO_G_NP;
    const double *DT = g + MBS_PO_G_NXDT, *DP = g + MBS_PO_G_NXDP;
    const double dDT = dir[0] * DT[0] + dir[1] * DT[1] + dir[2] * DT[2];
    const double cT[3] = { (dir[1] * NT[2] - dir[2] * NT[1]) + DT[0] - dir[0] * dDT,
                           (dir[2] * NT[0] - dir[0] * NT[2]) + DT[1] - dir[1] * dDT,
                           (dir[0] * NT[1] - dir[1] * NT[0]) + DT[2] - dir[2] * dDT };
    const double dDP = dir[0] * DP[0] + dir[1] * DP[1] + dir[2] * DP[2];
    const double cP[3] = { (dir[1] * NP[2] - dir[2] * NP[1]) + DP[0] - dir[0] * dDP,
                           (dir[2] * NP[0] - dir[0] * NP[2]) + DP[1] - dir[1] * dDP,
                           (dir[0] * NP[1] - dir[1] * NP[0]) + DP[2] - dir[2] * dDP };
    r[0] = (cT[0] * vt[0] + cT[1] * vt[1] + cT[2] * vt[2]) * 0.5;
    r[1] = (cP[0] * vt[0] + cP[1] * vt[1] + cP[2] * vt[2]) * 0.5;
    r[2] = (cT[0] * vf[0] + cT[1] * vf[1] + cT[2] * vf[2]) * 0.5;
    r[3] = (cP[0] * vf[0] + cP[1] * vf[1] + cP[2] * vf[2]) * 0.5;
}

/* d = (F * e^{i dirPhase} * R) x J_phased (HandlerPO.cpp:2745-2767). */
static void beam_jones(cplx F, cplx dp, const double *r, const double *jp, double *d)
{
    const cplx c = cmul(F, dp);
    const double s00r = c.re * r[0], s00i = c.im * r[0];
    const double s01r = c.re * r[1], s01i = c.im * r[1];
    const double s10r = c.re * r[2], s10i = c.im * r[2];
    const double s11r = c.re * r[3], s11i = c.im * r[3];
    const double j00r = jp[0], j00i = jp[1], j01r = jp[2], j01i = jp[3];
    const double j10r = jp[4], j10i = jp[5], j11r = jp[6], j11i = jp[7];
    d[0] = s00r * j00r - s00i * j00i + s01r * j10r - s01i * j10i;
    d[1] = s00r * j00i + s00i * j00r + s01r * j10i + s01i * j10r;
    d[2] = s00r * j01r - s00i * j01i + s01r * j11r - s01i * j11i;
    d[3] = s00r * j01i + s00i * j01r + s01r * j11i + s01i * j11r;
    d[4] = s10r * j00r - s10i * j00i + s11r * j10r - s11i * j10i;
    d[5] = s10r * j00i + s10i * j00r + s11r * j10i + s11i * j10r;
    d[6] = s10r * j01r - s10i * j01i + s11r * j11r - s11i * j11i;
    d[7] = s10r * j01i + s10i * j01r + s11r * j11i + s11i * j11r;
}

/* Coherent Jones sum of one orientation (HandlerPO.cpp:2561-2793): J and Jns
 * are [n_az*(n_zen+1)*8], overwritten. */
static void orientation_jones(const mbs_po_beams *b, const mbs_po_grid *g,
                              const mbs_po_wave *w, int o, double *J, double *Jns,
                              double *scratch)
{
    const int nAz = g->n_az, nT = g->n_zen + 1;
    const double k = w->wave_index;
    memset(J, 0, sizeof(double) * (size_t)nAz * nT * 8);
    if (Jns)
        memset(Jns, 0, sizeof(double) * (size_t)nAz * nT * 8);
    double *st = scratch, *ct = scratch + nT;
    double *vc = ct + nT, *vs = vc + 32;
    for (int t = 0; t < nT; ++t)
        sincos(g->theta[t], &st[t], &ct[t]);
    for (int64_t i = b->beam_offsets[o]; i < b->beam_offsets[o + 1]; ++i)
    {
        const int64_t v0 = b->vert_offsets[i];
        const int nv = (int)(b->vert_offsets[i + 1] - v0);
        const double *gm = b->beam_geom + (size_t)i * MBS_PO_GEOM_STRIDE;
        const double *hor = gm + MBS_PO_G_HOR, *ver = gm + MBS_PO_G_VER;
        const double *bd = gm + MBS_PO_G_BD, *cen = gm + MBS_PO_G_CEN;
        const int external = (b->beam_flags[i] & MBS_PO_BEAM_EXTERNAL) != 0;
        const double a0 = bd[0] * hor[0] + bd[1] * hor[1] + bd[2] * hor[2];
        const double b0 = bd[0] * ver[0] + bd[1] * ver[1] + bd[2] * ver[2];
        for (int p = 0; p < nAz; ++p)
        {
            double sp, cp;
            sincos(p * g->az_step, &sp, &cp);
            /* precompute_theta_coeffs (HandlerPO_fast.h:504-560) */
            const double a_sin = -cp * hor[0] - sp * hor[1], a_cos = hor[2];
            const double b_sin = -cp * ver[0] - sp * ver[1], b_cos = ver[2];
            for (int t = 0; t < nT; ++t)
            {
                const double A = st[t] * a_sin + ct[t] * a_cos + a0;
                const double B = st[t] * b_sin + ct[t] * b_cos + b0;
                for (int v = 0; v < nv; ++v)
                {
                    const double x = b->vx[v0 + v], y = b->vy[v0 + v];
                    const double ph = st[t] * (k * (a_sin * x + b_sin * y))
                                    + ct[t] * (k * (a_cos * x + b_cos * y))
                                    + k * (a0 * x + b0 * y);
                    sincos(ph, &vs[v], &vc[v]);
                }
                cplx dp = { 1.0, 0.0 };
                if (!external)
                {
                    const double arg = -k * (st[t] * (cp * cen[0] + sp * cen[1]) + ct[t] * (-cen[2]));
                    sincos(arg, &dp.im, &dp.re);
                }
                const cplx F = aperture(b, v0, nv, A, B, vc, vs, gm[MBS_PO_G_AREA], w, 1);
                if (isnan(F.re))
                    continue;
                const double dir[3] = { st[t] * cp, st[t] * sp, -ct[t] };
                const double *vf = g->vf + ((size_t)p * nT + t) * 3;
                double r[4], d[8];
                rotate_jones(gm, vf, dir, r);
                beam_jones(F, dp, r, gm + MBS_PO_G_JP, d);
                double *Jc = J + ((size_t)p * nT + t) * 8;
                for (int q = 0; q < 8; ++q)
                    Jc[q] += d[q];
                if (Jns && !external)
                {
                    double *Jn = Jns + ((size_t)p * nT + t) * 8;
                    for (int q = 0; q < 8; ++q)
                        Jn[q] += d[q];
                }
            }
        }
    }
}

void po_oracle_jones_to_mueller(const double *j, double weight, double *out)
{   /* AddMuellerFromJones (Mueller.hpp:37-87) */
    const double j00r = j[0], j00i = j[1], j01r = j[2], j01i = j[3];
    const double j10r = j[4], j10i = j[5], j11r = j[6], j11i = j[7];
    const double a11 = j00r * j00r + j00i * j00i, a12 = j01r * j01r + j01i * j01i;
    const double a21 = j10r * j10r + j10i * j10i, a22 = j11r * j11r + j11i * j11i;
    double A1 = a11 + a21, A2 = a12 + a22;
    out[0] += ((A1 + A2) * 0.5) * weight;
    out[1] += ((A1 - A2) * 0.5) * weight;
    A1 = a11 - a21; A2 = a12 - a22;
    out[4] += ((A1 + A2) * 0.5) * weight;
    out[5] += ((A1 - A2) * 0.5) * weight;
    double c1r = j00r * j01r + j00i * j01i, c1i = j00i * j01r - j00r * j01i;
    double c2r = j11r * j10r + j11i * j10i, c2i = j11i * j10r - j11r * j10i;
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

int po_oracle_jones(const mbs_po_beams *b, const mbs_po_grid *g,
                    const mbs_po_wave *w, int orient, double *J, double *Jns)
{
    if (!b || !g || !w || !J || orient < 0 || orient >= b->n_orient)
        return MBS_PO_EINVAL;
    double *scratch = (double *)malloc(sizeof(double) * (2 * (g->n_zen + 1) + 64));
    if (!scratch)
        return MBS_PO_ENOMEM;
    orientation_jones(b, g, w, orient, J, Jns, scratch);
    free(scratch);
    return MBS_PO_OK;
}

int po_oracle_diffract(const mbs_po_beams *b, const mbs_po_grid *g,
                       const mbs_po_wave *w, int n_threads,
                       double *M, double *Mns)
{
    if (!b || !g || !w || !M)
        return MBS_PO_EINVAL;
    const int nAz = g->n_az, nT = g->n_zen + 1;
    const size_t nDir = (size_t)nAz * nT;
    int nth = 1;
#ifdef _OPENMP
    nth = n_threads > 0 ? n_threads : omp_get_max_threads();
#endif
    if (nth > b->n_orient)
        nth = b->n_orient > 0 ? b->n_orient : 1;
    double *acc = (double *)calloc((size_t)nth * nDir * 32, sizeof(double));
    if (!acc)
        return MBS_PO_ENOMEM;
    int rc = MBS_PO_OK;
#pragma omp parallel num_threads(nth)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *myM = acc + (size_t)tid * nDir * 32;
        double *myMns = myM + nDir * 16;
        double *J = (double *)malloc(sizeof(double) * nDir * 16);
        double *scratch = (double *)malloc(sizeof(double) * (2 * nT + 64));
        if (!J || !scratch)
        {
#pragma omp atomic write
            rc = MBS_PO_ENOMEM;
        }
        else
        {
            double *Jns = J + nDir * 8;
#pragma omp for schedule(static)
            for (int o = 0; o < b->n_orient; ++o)
            {
                orientation_jones(b, g, w, o, J, Jns, scratch);
                const double wt = b->orient_weight[o];
                for (size_t d = 0; d < nDir; ++d)
                {
                    po_oracle_jones_to_mueller(J + d * 8, wt, myM + d * 16);
                    po_oracle_jones_to_mueller(Jns + d * 8, wt, myMns + d * 16);
                }
            }
        }
        free(J);
        free(scratch);
    }
    /* merge per-thread accumulators in thread order (deterministic) */
    for (int t = 0; t < nth && rc == MBS_PO_OK; ++t)
    {
        const double *m = acc + (size_t)t * nDir * 32;
        for (size_t i = 0; i < nDir * 16; ++i)
            M[i] += m[i];
        if (Mns)
            for (size_t i = 0; i < nDir * 16; ++i)
                Mns[i] += m[nDir * 16 + i];
    }
    free(acc);
    return rc;
}

double po_oracle_extinction(const mbs_po_beams *b, const mbs_po_wave *w, int o)
{   /* HandlerPO::ComputeForwardExtinctionOt (HandlerPO.cpp:1812-2009) */
    const double k = w->wave_index;
    cplx f00 = { 0, 0 }, f11 = { 0, 0 };
    double vc[32], vs[32];
    const double vf[3] = { 0.0, 1.0, 0.0 }, dir[3] = { 0.0, 0.0, -1.0 };
    for (int64_t i = b->beam_offsets[o]; i < b->beam_offsets[o + 1]; ++i)
    {
        const int external = (b->beam_flags[i] & MBS_PO_BEAM_EXTERNAL) != 0;
        if (w->ot_phase_average && !external)
            continue;
        const int64_t v0 = b->vert_offsets[i];
        const int nv = (int)(b->vert_offsets[i + 1] - v0);
        if (nv <= 0 || nv >= 32)
            continue;
        const double *gm = b->beam_geom + (size_t)i * MBS_PO_GEOM_STRIDE;
        const double *hor = gm + MBS_PO_G_HOR, *ver = gm + MBS_PO_G_VER, *bd = gm + MBS_PO_G_BD;
        /* theta = 0, phi = 0: A = a_cos + a0, B = b_cos + b0 */
        const double a0 = bd[0] * hor[0] + bd[1] * hor[1] + bd[2] * hor[2];
        const double b0 = bd[0] * ver[0] + bd[1] * ver[1] + bd[2] * ver[2];
        const double A = 1.0 * hor[2] + a0, B = 1.0 * ver[2] + b0;
        double fr, fi;
        cplx F;
        if (small_phase_factor(b->vx + v0, b->vy + v0, nv, A, B, k, &fr, &fi))
        {
            const double sgn = w->legacy_sign ? 1.0 : -1.0;
            const cplx al = { sgn * w->inv_compl_wave_re * gm[MBS_PO_G_AREA],
                              sgn * w->inv_compl_wave_im * gm[MBS_PO_G_AREA] };
            const cplx f = { fr, fi };
            F = cmul(al, f);
        }
        else
        {
            for (int v = 0; v < nv; ++v)
            {
                const double x = b->vx[v0 + v], y = b->vy[v0 + v];
                const double ph = 1.0 * (k * (hor[2] * x + ver[2] * y)) + k * (a0 * x + b0 * y);
                sincos(ph, &vs[v], &vc[v]);
            }
            double sr = 0, si = 0;
            if (fabs(B) > fabs(A))
            {
                for (int e = 0; e < nv; ++e)
                {
                    if (!(b->edge_flags[v0 + e] & MBS_PO_EDGE_VALID_X))
                        continue;
                    const int en = (e + 1 < nv) ? e + 1 : 0;
                    const double Ci = A + b->slope_yx[v0 + e] * B;
                    const double inv = (fabs(Ci) > w->eps1) ? 1.0 / Ci : 0.0;
                    sr += (vc[en] - vc[e]) * inv;
                    si += (vs[en] - vs[e]) * inv;
                    if (fabs(Ci) <= w->eps1)
                        stable_edge(vc[e], vs[e], b->vx[v0 + en] - b->vx[v0 + e], Ci, k, &sr, &si);
                }
                if (fabs(B) <= w->eps1)
                    continue;
                sr /= B;
                si /= B;
            }
            else
            {
                for (int e = 0; e < nv; ++e)
                {
                    if (!(b->edge_flags[v0 + e] & MBS_PO_EDGE_VALID_Y))
                        continue;
                    const int en = (e + 1 < nv) ? e + 1 : 0;
                    const double Ei = A * b->slope_xy[v0 + e] + B;
                    const double inv = (fabs(Ei) > w->eps1) ? 1.0 / Ei : 0.0;
                    sr += (vc[en] - vc[e]) * inv;
                    si += (vs[en] - vs[e]) * inv;
                    if (fabs(Ei) <= w->eps1)
                        stable_edge(vc[e], vs[e], b->vy[v0 + en] - b->vy[v0 + e], Ei, k, &sr, &si);
                }
                if (fabs(A) <= w->eps1)
                    continue;
                const double inA = -1.0 / A;
                sr *= inA;
                si *= inA;
            }
            const cplx cw = { w->compl_wave_re, w->compl_wave_im };
            const cplx s = { sr, si };
            F = cmul(cw, s);
        }
        if (isnan(F.re))
            continue;
        const double ref = external ? gm[MBS_PO_G_OPATH] : w->ot_far_reference_path;
        cplx dp = { 1.0, 0.0 };
        if (!external)
        {
            const double cen_z = gm[MBS_PO_G_CEN + 2];
            sincos(-k * (1.0 * (-cen_z) + ref), &dp.im, &dp.re);
        }
        else if (ref != 0.0)
            sincos(-k * ref, &dp.im, &dp.re);
        double r[4], d[8];
        rotate_jones(gm, vf, dir, r);
        beam_jones(F, dp, r, gm + MBS_PO_G_JP, d);
        f00.re += d[0]; f00.im += d[1];
        f11.re += d[6]; f11.im += d[7];
    }
    const cplx fwd = { f00.re + f11.re, f00.im + f11.im };
    double amp = fwd.im;
    if (w->ot_ping_distance != 0.0)
    {
        double sn, cs;
        sincos(2.0 * k * w->ot_ping_distance, &sn, &cs);
        amp = fwd.im * cs - fwd.re * sn;
    }
    const double cext = w->wavelength * amp * b->orient_weight[o];
    return isfinite(cext) ? cext : 0.0;
}

int po_oracle_phi_average(const double *M, int n_az, int n_zen,
                          const double *theta, const double *dcos2pi,
                          double *rows, double *csca, double *asym)
{   /* HandlerPOTotal::WriteMatricesToFile (HandlerPOTotal.cpp:49-96) */
    const double tol = 256.0 * DBL_EPSILON;   /* PoleMueller::AngularTolerance */
    double cs = 0.0, cg = 0.0;
    for (int t = 0; t <= n_zen; ++t)
    {
        double S[16] = { 0 };
        const int fwd = fabs(theta[t]) <= tol;
        const int bwd = fabs(theta[t] - M_PI) <= tol;
        for (int p = 0; p < n_az; ++p)
        {
            const double *m = M + ((size_t)p * (n_zen + 1) + t) * 16;
            if (fwd || bwd)
            {
                for (int q = 0; q < 16; ++q)
                    S[q] += m[q];
                continue;
            }
            /* m * L, L = [1 0 0 0; 0 c s 0; 0 -s c 0; 0 0 0 1], angle 2*(-p*step) */
            const double az = -p * (2.0 * M_PI / n_az);
            const double c = cos(2 * az), s = sin(2 * az);
            for (int r = 0; r < 4; ++r)
            {
                const double m0 = m[4 * r], m1 = m[4 * r + 1], m2 = m[4 * r + 2], m3 = m[4 * r + 3];
                S[4 * r + 0] += m0;
                S[4 * r + 1] += m1 * c - m2 * s;
                S[4 * r + 2] += m1 * s + m2 * c;
                S[4 * r + 3] += m3;
            }
        }
        for (int q = 0; q < 16; ++q)
            S[q] /= n_az;
        if (bwd || fwd)
        {   /* PoleMueller::ApplyBackward / ApplyForward */
            const double M00 = S[0], M33 = S[15], M03 = S[3];
            const double M11 = bwd ? 0.5 * (S[5] - S[10]) : 0.5 * (S[5] + S[10]);
            memset(S, 0, sizeof(S));
            S[0] = M00; S[5] = M11; S[10] = bwd ? -M11 : M11; S[15] = M33;
            S[3] = M03; S[12] = M03;
        }
        if (rows)
            memcpy(rows + (size_t)t * 16, S, sizeof(S));
        cs += S[0] * dcos2pi[t];
        cg += cos(theta[t]) * S[0] * dcos2pi[t];
    }
    if (csca)
        *csca = cs;
    if (asym)
        *asym = cs != 0.0 ? cg / cs : 0.0;
    return MBS_PO_OK;
}

int po_oracle_thetas_m11(const mbs_po_beams *b, const mbs_po_wave *w, int n_az, double az_step,
                         const double *theta, int n, int singular, double *m11)
{   /* theta_m11_kernel (GpuDiffraction.cu:1909-1956) over DiffractThetasGpu's
       tables (:4780-4970): per beam and azimuth bin p < n_az the squared
       norm of the GPU-convention Jones contribution (rotation without the
       0.5, i.e. twice this file's); the reference drops nearly singular
       edges there (singular = 0). */
    const double k = w->wave_index;
#pragma omp parallel for schedule(dynamic, 1)
    for (int t = 0; t < n; ++t)
    {
        double st, ct, vc[32], vs[32], acc = 0.0;
        sincos(theta[t], &st, &ct);
        for (int o = 0; o < b->n_orient; ++o)
        {
            const double wo = b->orient_weight[o];
            for (int64_t i = b->beam_offsets[o]; i < b->beam_offsets[o + 1]; ++i)
            {
                const int64_t v0 = b->vert_offsets[i];
                const int nv = (int)(b->vert_offsets[i + 1] - v0);
                const double *gm = b->beam_geom + (size_t)i * MBS_PO_GEOM_STRIDE;
                const double *hor = gm + MBS_PO_G_HOR, *ver = gm + MBS_PO_G_VER;
                const double *bd = gm + MBS_PO_G_BD, *cen = gm + MBS_PO_G_CEN;
                const int external = (b->beam_flags[i] & MBS_PO_BEAM_EXTERNAL) != 0;
                const double a0 = bd[0] * hor[0] + bd[1] * hor[1] + bd[2] * hor[2];
                const double b0 = bd[0] * ver[0] + bd[1] * ver[1] + bd[2] * ver[2];
                for (int p = 0; p < n_az; ++p)
                {
                    double sp, cp;
                    sincos(p * az_step, &sp, &cp);
                    const double a_sin = -cp * hor[0] - sp * hor[1], a_cos = hor[2];
                    const double b_sin = -cp * ver[0] - sp * ver[1], b_cos = ver[2];
                    const double A = st * a_sin + ct * a_cos + a0;
                    const double B = st * b_sin + ct * b_cos + b0;
                    for (int v = 0; v < nv; ++v)
                    {
                        const double x = b->vx[v0 + v], y = b->vy[v0 + v];
                        sincos(k * (A * x + B * y), &vs[v], &vc[v]);
                    }
                    cplx dp = { 1.0, 0.0 };
                    if (!external)
                    {
                        const double arg = -k * (st * (cp * cen[0] + sp * cen[1]) + ct * (-cen[2]));
                        sincos(arg, &dp.im, &dp.re);
                    }
                    const cplx F = aperture(b, v0, nv, A, B, vc, vs, gm[MBS_PO_G_AREA], w, singular);
                    if (isnan(F.re))
                        continue;
                    const double dir[3] = { st * cp, st * sp, -ct };
                    const double vf[3] = { -sp, cp, 0.0 };
                    double r[4], d[8];
                    rotate_jones(gm, vf, dir, r);
                    beam_jones(F, dp, r, gm + MBS_PO_G_JP, d);
                    double e = 0.0;
                    for (int q = 0; q < 8; ++q)
                        e += d[q] * d[q];
                    acc += 0.5 * (4.0 * e) * wo / (double)(n_az + 1);
                }
            }
        }
        m11[t] = acc;
    }
    return 0;
}
