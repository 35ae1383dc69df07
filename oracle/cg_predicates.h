/*
 * TEST INFRASTRUCTURE ONLY -- part of the CPU oracle, never linked into the product.
 *
 * Exact geometric predicates for the oracle, written from the published method of
 * J. R. Shewchuk, "Adaptive Precision Floating-Point Arithmetic and Fast Robust Geometric
 * Predicates", Discrete Comput. Geom. 18 (1997): a fast floating-point filter, and when the
 * filter cannot decide, exact evaluation with non-overlapping floating-point expansions
 * (two_sum / two_product / expansion sums). two_product uses fma(), which is exact.
 *
 * Why exact predicates: the reference delegates Delaunay construction to CGAL's
 * Exact_predicates_inexact_constructions_kernel (inc/models/DelaunayCGAL.h:18), so "the"
 * reference topology is the Delaunay triangulation decided by exact orientation / in-circle
 * tests on double coordinates. Any exact implementation decides the same triangulation for
 * points in general position.
 *
 * All predicates here take coordinates RELATIVE to a centre point that sits at the origin,
 * which is how the reference feeds its local triangulations (src/models/DelaunayLoc.cpp:171-273:
 * DTring[0] = (0,0), the others are Box->minDist displacements).
 */
#ifndef CG_PREDICATES_H
#define CG_PREDICATES_H

#include <math.h>

#define CG_EXP_MAX 160

static inline void cgp_two_sum(double a, double b, double *x, double *y)
{
    double s = a + b;
    double bv = s - a;
    double av = s - bv;
    double br = b - bv;
    double ar = a - av;
    *x = s;
    *y = ar + br;
}

static inline void cgp_two_prod(double a, double b, double *x, double *y)
{
    double p = a * b;
    *x = p;
    *y = fma(a, b, -p);
}

/* h = e + f, both non-overlapping expansions in increasing magnitude; zero elimination.
 * Straightforward "grow by each component" summation (Shewchuk's GROW-EXPANSION applied
 * repeatedly); quadratic but the expansions here are short. */
static inline int cgp_grow(int elen, const double *e, double b, double *h)
{
    double q = b, hh;
    int hidx = 0;
    for (int i = 0; i < elen; ++i) {
        double qn;
        cgp_two_sum(q, e[i], &qn, &hh);
        q = qn;
        if (hh != 0.0) h[hidx++] = hh;
    }
    if (q != 0.0 || hidx == 0) h[hidx++] = q;
    return hidx;
}

static inline int cgp_sum(int elen, const double *e, int flen, const double *f, double *h)
{
    double a[CG_EXP_MAX], b[CG_EXP_MAX];
    int n = elen;
    for (int i = 0; i < elen; ++i) a[i] = e[i];
    double *cur = a, *nxt = b;
    for (int j = 0; j < flen; ++j) {
        n = cgp_grow(n, cur, f[j], nxt);
        double *t = cur; cur = nxt; nxt = t;
    }
    for (int i = 0; i < n; ++i) h[i] = cur[i];
    return n;
}

/* h = e * b (SCALE-EXPANSION with zero elimination) */
static inline int cgp_scale(int elen, const double *e, double b, double *h)
{
    double q, hh, p1, p0, sum;
    int hidx = 0;
    cgp_two_prod(e[0], b, &q, &hh);
    if (hh != 0.0) h[hidx++] = hh;
    for (int i = 1; i < elen; ++i) {
        cgp_two_prod(e[i], b, &p1, &p0);
        cgp_two_sum(q, p0, &sum, &hh);
        if (hh != 0.0) h[hidx++] = hh;
        cgp_two_sum(p1, sum, &q, &hh);
        if (hh != 0.0) h[hidx++] = hh;
    }
    if (q != 0.0 || hidx == 0) h[hidx++] = q;
    return hidx;
}

static inline int cgp_mul(int elen, const double *e, int flen, const double *f, double *h)
{
    double acc[CG_EXP_MAX], tmp[CG_EXP_MAX], nxt[CG_EXP_MAX];
    int n = 1;
    acc[0] = 0.0;
    for (int j = 0; j < flen; ++j) {
        int m = cgp_scale(elen, e, f[j], tmp);
        n = cgp_sum(n, acc, m, tmp, nxt);
        for (int i = 0; i < n; ++i) acc[i] = nxt[i];
    }
    for (int i = 0; i < n; ++i) h[i] = acc[i];
    return n;
}

static inline int cgp_sign_exp(int n, const double *e)
{
    for (int i = n - 1; i >= 0; --i) {
        if (e[i] > 0.0) return 1;
        if (e[i] < 0.0) return -1;
    }
    return 0;
}

/* a x b - c x d (cross-like), exact, as an expansion */
static inline int cgp_diff_prod(double a, double b, double c, double d, double *h)
{
    double p1, e1, p2, e2;
    double x[2], y[2];
    cgp_two_prod(a, b, &p1, &e1);
    cgp_two_prod(c, d, &p2, &e2);
    x[0] = e1; x[1] = p1;
    y[0] = -e2; y[1] = -p2;
    return cgp_sum(2, x, 2, y, h);
}

/* sign of orient(0, a, b) = ax*by - ay*bx : +1 when b is counter-clockwise of a */
static inline int cg_orient0(double ax, double ay, double bx, double by)
{
    double l = ax * by, r = ay * bx;
    double det = l - r;
    double bound = 4.0e-16 * (fabs(l) + fabs(r));
    if (det > bound) return 1;
    if (-det > bound) return -1;
    double h[8];
    int n = cgp_diff_prod(ax, by, ay, bx, h);
    return cgp_sign_exp(n, h);
}

/* D(a,b,c) = |a|^2 (b x c) - |b|^2 (a x c) + |c|^2 (a x b).
 * For (0,a,b) counter-clockwise: D < 0  <=>  c strictly inside the circle through 0, a, b;
 * D == 0 <=> cocircular. Returns sign(D). */
static inline int cg_incircle0(double ax, double ay, double bx, double by, double cx, double cy)
{
    double aa = ax * ax + ay * ay, bb = bx * bx + by * by, cc = cx * cx + cy * cy;
    double bxc = bx * cy - by * cx, axc = ax * cy - ay * cx, axb = ax * by - ay * bx;
    double det = aa * bxc - bb * axc + cc * axb;
    double perm = aa * (fabs(bx * cy) + fabs(by * cx)) + bb * (fabs(ax * cy) + fabs(ay * cx)) +
                  cc * (fabs(ax * by) + fabs(ay * bx));
    double bound = 4.0e-15 * perm;
    if (det > bound) return 1;
    if (-det > bound) return -1;

    double e_aa[8], e_bb[8], e_cc[8], e_bxc[8], e_axc[8], e_axb[8];
    double t[2], u[2];
    int naa, nbb, ncc;
    cgp_two_prod(ax, ax, &t[1], &t[0]); cgp_two_prod(ay, ay, &u[1], &u[0]);
    naa = cgp_sum(2, t, 2, u, e_aa);
    cgp_two_prod(bx, bx, &t[1], &t[0]); cgp_two_prod(by, by, &u[1], &u[0]);
    nbb = cgp_sum(2, t, 2, u, e_bb);
    cgp_two_prod(cx, cx, &t[1], &t[0]); cgp_two_prod(cy, cy, &u[1], &u[0]);
    ncc = cgp_sum(2, t, 2, u, e_cc);
    int nbxc = cgp_diff_prod(bx, cy, by, cx, e_bxc);
    int naxc = cgp_diff_prod(ax, cy, ay, cx, e_axc);
    int naxb = cgp_diff_prod(ax, by, ay, bx, e_axb);

    double t1[CG_EXP_MAX], t2[CG_EXP_MAX], t3[CG_EXP_MAX], s12[CG_EXP_MAX], s[CG_EXP_MAX];
    int n1 = cgp_mul(naa, e_aa, nbxc, e_bxc, t1);
    int n2 = cgp_mul(nbb, e_bb, naxc, e_axc, t2);
    for (int i = 0; i < n2; ++i) t2[i] = -t2[i];
    int n3 = cgp_mul(ncc, e_cc, naxb, e_axb, t3);
    int n12 = cgp_sum(n1, t1, n2, t2, s12);
    int ns = cgp_sum(n12, s12, n3, t3, s);
    return cgp_sign_exp(ns, s);
}

#endif
