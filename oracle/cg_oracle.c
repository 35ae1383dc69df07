/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle (see cg_oracle.h). Never linked into the product.
 *
 * Plain C, FP64, single-threaded: a restatement of the reference's CPU path. Citations are to
 * files of abaso/cellGPU. Where the reference calls CGAL (not vendored; CGAL 4.9 with the
 * Exact_predicates_inexact_constructions_kernel, inc/models/DelaunayCGAL.h:7-32) this file states
 * the Delaunay triangulation itself with exact predicates (cg_predicates.h).
 */
#include "cg_oracle.h"
#include "cg_predicates.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------ */
/* periodic square box: inc/utility/gpubox.h                                                   */
/* ------------------------------------------------------------------------------------------ */

/* gpubox::minDist for a rectangular box (inc/utility/gpubox.h:154-165): while-loop wrapping by the
 * box sides with half-box thresholds, result = p1 - p2 mapped to the nearest image. */
void cgo_min_dist(const double *box, const double *p1, const double *p2, double *out)
{
    double Lx = box[0], Ly = box[1];
    double hx = Lx * 0.5, hy = Ly * 0.5;
    double x = p1[0] - p2[0];
    double y = p1[1] - p2[1];
    if (!(fabs(x) <= 2.0 * Lx)) x -= Lx * rint(x / Lx); /* bound the loops (never taken in-box) */
    if (!(fabs(y) <= 2.0 * Ly)) y -= Ly * rint(y / Ly);
    while (x < -hx) x += Lx;
    while (y < -hy) y += Ly;
    while (x > hx) x -= Lx;
    while (y > hy) y -= Ly;
    out[0] = x;
    out[1] = y;
}

/* gpubox::putInBoxReal -> invTrans, putInBox, Trans (inc/utility/gpubox.h:131-152) for a
 * rectangular box: v = (1/L) * p, wrap v into [0,1) by +-1.0 loops, p = L * v. */
void cgo_put_in_box(const double *box, double *p)
{
    double ix = 1.0 / box[0], iy = 1.0 / box[1];
    double vx = ix * p[0];
    double vy = iy * p[1];
    if (!(vx >= -1.0 && vx < 2.0)) vx -= floor(vx); /* bound the loops (never taken for small moves) */
    if (!(vy >= -1.0 && vy < 2.0)) vy -= floor(vy);
    while (vx < 0) vx += 1.0;
    while (vy < 0) vy += 1.0;
    while (vx >= 1.0) vx -= 1.0;
    while (vy >= 1.0) vy -= 1.0;
    p[0] = box[0] * vx;
    p[1] = box[1] * vy;
}

/* ------------------------------------------------------------------------------------------ */
/* geometry primitives: inc/utility/functions.h                                                */
/* ------------------------------------------------------------------------------------------ */

/* Circumcenter(x1,x2,xc) through the origin (inc/utility/functions.h:34-43) */
static void circumcenter0(const double *x1, const double *x2, double *xc)
{
    double x1n = x1[0] * x1[0] + x1[1] * x1[1];
    double x2n = x2[0] * x2[0] + x2[1] * x2[1];
    double den = 0.5 / (x1[0] * x2[1] - x1[1] * x2[0]);
    xc[0] = den * (x1n * x2[1] - x1[1] * x2n);
    xc[1] = den * (x1[0] * x2n - x1n * x2[0]);
}

/* Circumcenter(x1,x2,x3) (inc/utility/functions.h:46-62) */
static void circumcenter3(const double *x1, const double *x2, const double *x3, double *xc)
{
    double amcx = x1[0] - x3[0], amcy = x1[1] - x3[1];
    double amc2 = amcx * amcx + amcy * amcy;
    double bmcx = x2[0] - x3[0], bmcy = x2[1] - x3[1];
    double bmc2 = bmcx * bmcx + bmcy * bmcy;
    double den = 0.5 / (amcx * bmcy - amcy * bmcx);
    xc[0] = x3[0] + den * (amc2 * bmcy - amcy * bmc2);
    xc[1] = x3[1] + den * (amcx * bmc2 - amc2 * bmcx);
}

/* TriangleArea (inc/utility/functions.h:224-227) */
static double triangle_area0(const double *p1, const double *p2)
{
    return fabs(0.5 * (p1[0] * p2[1] - p1[1] * p2[0]));
}

/* SignedPolygonAreaPart (inc/utility/functions.h:217-220) */
static double signed_area_part(const double *p1, const double *p2)
{
    return 0.5 * (p1[0] + p2[0]) * (p2[1] - p1[1]);
}

/* ------------------------------------------------------------------------------------------ */
/* Delaunay star of the origin: the role of DelaunayCGAL::LocalTriangulation                   */
/* (src/models/DelaunayCGAL.cpp:8-48) -- returns the CCW neighbour cycle of candidate 0 in    */
/* the reference, here of the origin among the candidates.                                      */
/* ------------------------------------------------------------------------------------------ */

/* Gift wrapping around the origin. The nearest candidate is always a Delaunay neighbour. From a
 * neighbour a, the next CCW neighbour b is the candidate strictly counter-clockwise of a whose
 * circle through (0,a,b) contains no other counter-clockwise candidate; the circles through 0 and
 * a form a pencil, so one pass keeping the "innermost" circle finds it. */
int cgo_local_star(int m, const double *rel, int cap, int *out)
{
    if (m < 3) return -1;
    int start = 0;
    double best = rel[0] * rel[0] + rel[1] * rel[1];
    for (int i = 1; i < m; ++i) {
        double d = rel[2 * i] * rel[2 * i] + rel[2 * i + 1] * rel[2 * i + 1];
        if (d < best) { best = d; start = i; }
    }
    int count = 0;
    int a = start;
    for (int guard = 0; guard < m + 1; ++guard) {
        if (count >= cap) return -2;
        out[count++] = a;
        const double *pa = rel + 2 * a;
        int b = -1;
        for (int c = 0; c < m; ++c) {
            if (c == a) continue;
            const double *pc = rel + 2 * c;
            if (cg_orient0(pa[0], pa[1], pc[0], pc[1]) <= 0) continue;
            if (b < 0) { b = c; continue; }
            const double *pb = rel + 2 * b;
            if (cg_incircle0(pa[0], pa[1], pb[0], pb[1], pc[0], pc[1]) < 0) b = c;
        }
        if (b < 0) return -1;
        if (b == start) return count;
        a = b;
    }
    return -1;
}

/* O(m^3) enumeration: (0,a,b) is a Delaunay triangle iff it is CCW and no other candidate lies
 * strictly inside its circumcircle. Then chain the triangles around the origin. */
int cgo_local_star_bruteforce(int m, const double *rel, int cap, int *out)
{
    int *next = (int *)malloc(sizeof(int) * m);
    for (int i = 0; i < m; ++i) next[i] = -1;
    int any = -1;
    for (int a = 0; a < m; ++a) {
        for (int b = 0; b < m; ++b) {
            if (a == b) continue;
            const double *pa = rel + 2 * a, *pb = rel + 2 * b;
            if (cg_orient0(pa[0], pa[1], pb[0], pb[1]) <= 0) continue;
            int empty = 1;
            for (int c = 0; c < m && empty; ++c) {
                if (c == a || c == b) continue;
                const double *pc = rel + 2 * c;
                if (cg_incircle0(pa[0], pa[1], pb[0], pb[1], pc[0], pc[1]) < 0) empty = 0;
            }
            if (empty) { next[a] = b; any = a; }
        }
    }
    if (any < 0) { free(next); return -1; }
    /* start at the nearest point like cgo_local_star */
    int start = 0;
    double best = rel[0] * rel[0] + rel[1] * rel[1];
    for (int i = 1; i < m; ++i) {
        double d = rel[2 * i] * rel[2 * i] + rel[2 * i + 1] * rel[2 * i + 1];
        if (d < best) { best = d; start = i; }
    }
    int count = 0, a = start;
    while (1) {
        if (count >= cap || count > m) { free(next); return -2; }
        out[count++] = a;
        a = next[a];
        if (a < 0) { free(next); return -1; }
        if (a == start) break;
    }
    free(next);
    return count;
}

/* ------------------------------------------------------------------------------------------ */
/* periodic Delaunay triangulation (role of DelaunayCGAL::PeriodicTriangulationSquareDomain,   */
/* src/models/DelaunayCGAL.cpp:164-229, called by voronoiModelBase::globalTriangulationCGAL,   */
/* src/models/voronoiModelBase.cpp:281-351)                                                    */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    int nbx, nby;      /* bins per side */
    double bsx, bsy;   /* bin sides */
    int *start, *cells;
} grid_t;

static void grid_build(grid_t *g, int N, const double *pos, const double *box)
{
    g->nbx = (int)floor(box[0]);
    if (g->nbx < 1) g->nbx = 1;
    g->nby = (int)floor(box[1]);
    if (g->nby < 1) g->nby = 1;
    g->bsx = box[0] / g->nbx;
    g->bsy = box[1] / g->nby;
    int nbins = g->nbx * g->nby;
    g->start = (int *)calloc(nbins + 1, sizeof(int));
    g->cells = (int *)malloc(sizeof(int) * (N > 0 ? N : 1));
    int *bin = (int *)malloc(sizeof(int) * (N > 0 ? N : 1));
    for (int i = 0; i < N; ++i) {
        int bx = (int)floor(pos[2 * i] / g->bsx), by = (int)floor(pos[2 * i + 1] / g->bsy);
        if (bx < 0) bx = 0;
        if (bx >= g->nbx) bx = g->nbx - 1;
        if (by < 0) by = 0;
        if (by >= g->nby) by = g->nby - 1;
        bin[i] = by * g->nbx + bx;
        g->start[bin[i] + 1]++;
    }
    for (int b = 0; b < nbins; ++b) g->start[b + 1] += g->start[b];
    int *fill = (int *)malloc(sizeof(int) * nbins);
    memcpy(fill, g->start, sizeof(int) * nbins);
    for (int i = 0; i < N; ++i) g->cells[fill[bin[i]]++] = i;
    free(fill);
    free(bin);
}

static void grid_free(grid_t *g)
{
    free(g->start);
    free(g->cells);
}

/* Delaunay star of point i: candidates are all points whose minimum image lies within radius R;
 * the star is accepted when every star triangle's circumcircle lies inside that radius, which
 * makes it the exact star. Writes global indices (CCW, rotated to the smallest index). */
static int star_of(int i, const double *pos, const double *box, const grid_t *g, int cap, int *row)
{
    double bs = g->bsx > g->bsy ? g->bsx : g->bsy;
    double half = 0.5 * (box[0] < box[1] ? box[0] : box[1]);
    double R = 2.5 * bs;
    int mcap = 256;
    double *rel = (double *)malloc(sizeof(double) * 2 * mcap);
    int *idx = (int *)malloc(sizeof(int) * mcap);
    int *loc = (int *)malloc(sizeof(int) * mcap);
    int result = -1;
    for (int attempt = 0; attempt < 12; ++attempt) {
        if (R > half) R = half;
        int wx = (int)ceil(R / g->bsx) + 1, wy = (int)ceil(R / g->bsy) + 1;
        if (2 * wx + 1 > g->nbx) wx = (g->nbx - 1) / 2;
        if (2 * wy + 1 > g->nby) wy = (g->nby - 1) / 2;
        int cbx = (int)floor(pos[2 * i] / g->bsx), cby = (int)floor(pos[2 * i + 1] / g->bsy);
        if (cbx >= g->nbx) cbx = g->nbx - 1;
        if (cby >= g->nby) cby = g->nby - 1;
        int m = 0;
        for (int dy = -wy; dy <= wy; ++dy)
            for (int dx = -wx; dx <= wx; ++dx) {
                int bx = ((cbx + dx) % g->nbx + g->nbx) % g->nbx;
                int by = ((cby + dy) % g->nby + g->nby) % g->nby;
                int b = by * g->nbx + bx;
                for (int s = g->start[b]; s < g->start[b + 1]; ++s) {
                    int j = g->cells[s];
                    if (j == i) continue;
                    double d[2];
                    cgo_min_dist(box, pos + 2 * j, pos + 2 * i, d);
                    if (d[0] * d[0] + d[1] * d[1] > R * R) continue;
                    if (m == mcap) {
                        mcap *= 2;
                        rel = (double *)realloc(rel, sizeof(double) * 2 * mcap);
                        idx = (int *)realloc(idx, sizeof(int) * mcap);
                        loc = (int *)realloc(loc, sizeof(int) * mcap);
                    }
                    rel[2 * m] = d[0];
                    rel[2 * m + 1] = d[1];
                    idx[m] = j;
                    ++m;
                }
            }
        int z = cgo_local_star(m, rel, mcap, loc);
        if (z > 0) {
            int ok = 1;
            for (int n = 0; n < z && ok; ++n) {
                const double *a = rel + 2 * loc[n];
                const double *b = rel + 2 * loc[(n + 1) % z];
                double q[2];
                circumcenter0(a, b, q);
                double r = sqrt(q[0] * q[0] + q[1] * q[1]);
                if (!(2.0 * r < R * (1.0 - 1e-9))) ok = 0;
            }
            if (ok) {
                if (z > cap) { result = -2; break; }
                int s0 = 0;
                for (int n = 1; n < z; ++n)
                    if (idx[loc[n]] < idx[loc[s0]]) s0 = n;
                for (int n = 0; n < z; ++n) row[n] = idx[loc[(s0 + n) % z]];
                result = z;
                break;
            }
        }
        if (R >= half) break;
        R *= 1.5;
    }
    free(rel);
    free(idx);
    free(loc);
    return result;
}

int cgo_periodic_delaunay(int N, const double *pos, const double *box, int K, int *nn, int *nbr)
{
    grid_t g;
    grid_build(&g, N, pos, box);
    int *row = (int *)malloc(sizeof(int) * 512);
    int status = 0;
    long total = 0;
    for (int i = 0; i < N; ++i) {
        int z = star_of(i, pos, box, &g, 512, row);
        if (z < 0) { status = -1; break; }
        if (z > K) { status = -2; break; }
        nn[i] = z;
        for (int n = 0; n < z; ++n) nbr[i * K + n] = row[n];
        total += z;
    }
    /* the Euler check of voronoiModelBase::globalTriangulationCGAL (src/models/voronoiModelBase.cpp:342-350) */
    if (status == 0 && total != 6L * N) status = -3;
    free(row);
    grid_free(&g);
    return status;
}

int cgo_topology_mismatch(int N, const double *pos, const double *box, int K, const int *nn, const int *nbr)
{
    grid_t g;
    grid_build(&g, N, pos, box);
    int *row = (int *)malloc(sizeof(int) * 512);
    int bad = 0;
    for (int i = 0; i < N; ++i) {
        int z = star_of(i, pos, box, &g, 512, row);
        if (z != nn[i]) { ++bad; continue; }
        /* compare as cycles rotated to the smallest index */
        int s0 = 0;
        for (int n = 1; n < z; ++n)
            if (nbr[i * K + n] < nbr[i * K + s0]) s0 = n;
        for (int n = 0; n < z; ++n)
            if (nbr[i * K + (s0 + n) % z] != row[n]) { ++bad; break; }
    }
    free(row);
    grid_free(&g);
    return bad;
}

/* ------------------------------------------------------------------------------------------ */
/* Voronoi model                                                                               */
/* ------------------------------------------------------------------------------------------ */

/* voronoiModelBase::computeGeometryCPU (src/models/voronoiModelBase.cpp:783-846): Voronoi vertex
 * nn = circumcentre of (0, r_{nn-1}, r_nn); A = sum |triangle|, P = sum |edge|, summed from nn=0
 * with vlast = voro[z-1]. */
void cgo_voronoi_geometry(int N, const double *pos, const double *box, int K, const int *nn, const int *nbr,
                          double *AP)
{
    double voro[2 * 64];
    for (int i = 0; i < N; ++i) {
        int z = nn[i];
        const double *pi = pos + 2 * i;
        double rij[2], rik[2];
        cgo_min_dist(box, pos + 2 * nbr[i * K + z - 1], pi, rij);
        for (int n = 0; n < z; ++n) {
            cgo_min_dist(box, pos + 2 * nbr[i * K + n], pi, rik);
            circumcenter0(rij, rik, voro + 2 * n);
            rij[0] = rik[0];
            rij[1] = rik[1];
        }
        double A = 0.0, P = 0.0;
        const double *vlast = voro + 2 * (z - 1);
        for (int n = 0; n < z; ++n) {
            const double *vnext = voro + 2 * n;
            A += triangle_area0(vlast, vnext);
            double dx = vlast[0] - vnext[0], dy = vlast[1] - vnext[1];
            P += sqrt(dx * dx + dy * dy);
            vlast = vnext;
        }
        AP[2 * i] = A;
        AP[2 * i + 1] = P;
    }
}

/* VoronoiQuadraticEnergy::computeVoronoiForceCPU (src/models/voronoiQuadraticEnergy.cpp:172-378),
 * the gather form: for each Voronoi vertex of cell i, the derivative of the energies of the three
 * cells sharing it, times dh/dr_i; the third Voronoi vertex (vother) is found through the
 * neighbour row of the base neighbour (lines 258-267). The 1e-18 norm clamp is THRESHOLD
 * (inc/std_include.h:16). Returns <0 on an inconsistent triangulation (the reference throws). */
/* line tension between unlike cells: one gamma (ntypes == 0) or a row-major ntypes x ntypes matrix */
typedef struct {
    const int *ctype;
    int ntypes;
    double gamma;
    const double *tmat;
} tension_t;

/* weight of the edge between a cell of type a and one of type b, as the reference reads it:
 * gamma, or tensionMatrix[cellTypeIndexer(b, a)] = row a, column b
 * (src/models/voronoiQuadraticEnergyWithTension.cpp:22-36, 612-620) */
static double tension_w(const tension_t *t, int a, int b)
{
    if (!t || t->ctype[a] == t->ctype[b]) return 0.0;
    return t->ntypes ? t->tmat[t->ctype[a] * t->ntypes + t->ctype[b]] : t->gamma;
}

static int voronoi_forces_impl(int N, const double *pos, const double *box, int K, const int *nn, const int *nbr,
                               const double *AP, const double *APpref, double KA, double KP, const tension_t *ten,
                               double *F);

int cgo_voronoi_forces(int N, const double *pos, const double *box, int K, const int *nn, const int *nbr,
                       const double *AP, const double *APpref, double KA, double KP, double *F)
{
    return voronoi_forces_impl(N, pos, box, K, nn, nbr, AP, APpref, KA, KP, NULL, F);
}

/* VoronoiQuadraticEnergyWithTension::computeVoronoiSimpleTensionForceCPU and
 * computeVoronoiTensionForceCPU (src/models/voronoiQuadraticEnergyWithTension.cpp:236-744): the
 * force above plus, at each Voronoi vertex, the unit-vector derivatives of the unlike edges met
 * there, each edge once from each of the two of the vertex's three cells that share it (the dT
 * terms of lines 351-361, 413-422 and 443-452). ntypes == 0: one gamma for every unlike pair. */
int cgo_voronoi_tension_forces(int N, const double *pos, const double *box, int K, const int *nn, const int *nbr,
                               const double *AP, const double *APpref, double KA, double KP, const int *ctype,
                               int ntypes, double gamma, const double *tmat, double *F)
{
    tension_t t = {ctype, ntypes, gamma, tmat};
    return voronoi_forces_impl(N, pos, box, K, nn, nbr, AP, APpref, KA, KP, &t, F);
}

/* VoronoiQuadraticEnergyWithTension::computeEnergy (:101-159): the quadratic energy plus gamma l
 * over every unlike Voronoi edge counted once (from its lower-indexed cell); the edge of
 * neighbour n runs from Voronoi vertex n to vertex n+1. */
double cgo_voronoi_tension_energy(int N, const double *pos, const double *box, int K, const int *nn,
                                  const int *nbr, const double *AP, const double *APpref, double KA, double KP,
                                  const int *ctype, int ntypes, double gamma, const double *tmat)
{
    tension_t t = {ctype, ntypes, gamma, tmat};
    double E = cgo_voronoi_energy(N, AP, APpref, KA, KP);
    double voro[2 * 64];
    for (int i = 0; i < N; ++i) {
        int z = nn[i];
        const int *ns = nbr + i * K;
        double rij[2], rik[2];
        cgo_min_dist(box, pos + 2 * ns[z - 1], pos + 2 * i, rij);
        for (int n = 0; n < z; ++n) {
            cgo_min_dist(box, pos + 2 * ns[n], pos + 2 * i, rik);
            circumcenter0(rij, rik, voro + 2 * n);
            rij[0] = rik[0];
            rij[1] = rik[1];
        }
        for (int n = 0; n < z; ++n) {
            if (i >= ns[n] || ctype[i] == ctype[ns[n]]) continue;
            const double *a = voro + 2 * n, *b = voro + 2 * ((n + 1) % z);
            double dx = a[0] - b[0], dy = a[1] - b[1];
            E += sqrt(dx * dx + dy * dy) * tension_w(&t, i, ns[n]);
        }
    }
    return E;
}

static int voronoi_forces_impl(int N, const double *pos, const double *box, int K, const int *nn, const int *nbr,
                               const double *AP, const double *APpref, double KA, double KP, const tension_t *ten,
                               double *F)
{
    const double thr = 1e-18;
    double voro[2 * 64];
    double dh[4 * 64];
    for (int i = 0; i < N; ++i) {
        int z = nn[i];
        const int *ns = nbr + i * K;
        const double *pi = pos + 2 * i;
        double rij[2], rik[2];
        cgo_min_dist(box, pos + 2 * ns[z - 1], pi, rij);
        for (int n = 0; n < z; ++n) {
            cgo_min_dist(box, pos + 2 * ns[n], pi, rik);
            circumcenter0(rij, rik, voro + 2 * n);
            double rjk[2] = {rik[0] - rij[0], rik[1] - rij[1]};
            double rik2 = rik[0] * rik[0] + rik[1] * rik[1];
            double rij2 = rij[0] * rij[0] + rij[1] * rij[1];
            double rijrjk = rij[0] * rjk[0] + rij[1] * rjk[1];
            double rikrjk = rik[0] * rjk[0] + rik[1] * rjk[1];
            double betaD = -rik2 * rijrjk;
            double gammaD = rij2 * rikrjk;
            double cp = rij[0] * rjk[1] - rij[1] * rjk[0];
            double D = 2 * cp * cp;
            double zx = betaD * rij[0] + gammaD * rik[0];
            double zy = betaD * rij[1] + gammaD * rik[1];
            double dbx = 2 * rijrjk * rik[0] + rik2 * rjk[0];
            double dby = 2 * rijrjk * rik[1] + rik2 * rjk[1];
            double dgx = -2 * rikrjk * rij[0] - rij2 * rjk[0];
            double dgy = -2 * rikrjk * rij[1] - rij2 * rjk[1];
            double ddx = (-2.0 * rjk[1]) / cp;
            double ddy = (2.0 * rjk[0]) / cp;
            /* dhdri = Id + 1/D*(dyad(rij,dbDdri)+dyad(rik,dgDdri)-(betaD+gammaD)*Id-dyad(z,dDdriOD)) */
            double invD = 1.0 / D;
            double m11 = rij[0] * dbx + rik[0] * dgx - (betaD + gammaD) - zx * ddx;
            double m12 = rij[0] * dby + rik[0] * dgy - zx * ddy;
            double m21 = rij[1] * dbx + rik[1] * dgx - zy * ddx;
            double m22 = rij[1] * dby + rik[1] * dgy - (betaD + gammaD) - zy * ddy;
            dh[4 * n + 0] = 1.0 + invD * m11;
            dh[4 * n + 1] = invD * m12;
            dh[4 * n + 2] = invD * m21;
            dh[4 * n + 3] = 1.0 + invD * m22;
            rij[0] = rik[0];
            rij[1] = rik[1];
        }
        double fx = 0.0, fy = 0.0;
        double Adiff = KA * (AP[2 * i] - APpref[2 * i]);
        double Pdiff = KP * (AP[2 * i + 1] - APpref[2 * i + 1]);
        const double *vlast = voro + 2 * (z - 1);
        for (int n = 0; n < z; ++n) {
            const double *vcur = voro + 2 * n;
            const double *vnext = voro + 2 * ((n + 1) % z);
            int base = ns[n];
            int oi = n - 1;
            if (oi < 0) oi += z;
            int other = ns[oi];
            double dAi[2] = {0.5 * (vlast[1] - vnext[1]), 0.5 * (vnext[0] - vlast[0])};
            double dl[2] = {vlast[0] - vcur[0], vlast[1] - vcur[1]};
            double dln = sqrt(dl[0] * dl[0] + dl[1] * dl[1]);
            double dn[2] = {vcur[0] - vnext[0], vcur[1] - vnext[1]};
            double dnn = sqrt(dn[0] * dn[0] + dn[1] * dn[1]);
            if (dnn < thr) dnn = thr;
            if (dln < thr) dln = thr;
            double dPi[2] = {dl[0] / dln - dn[0] / dnn, dl[1] / dln - dn[1] / dnn};
            /* own unlike edges at vcur: (vcur, vnext) shared with base, (vlast, vcur) with other */
            double wib = tension_w(ten, i, base), wio = tension_w(ten, i, other);
            double dT[2] = {-wib * dn[0] / dnn + wio * dl[0] / dln, -wib * dn[1] / dnn + wio * dl[1] / dln};

            int z2 = nn[base];
            int dto = -1;
            for (int n2 = 0; n2 < z2; ++n2)
                if (nbr[base * K + n2] == other) dto = nbr[base * K + (n2 + 1) % z2];
            if (dto == other || dto == base || dto == -1) return -1;
            double r1[2], r2[2], r3[2], vother[2];
            cgo_min_dist(box, pos + 2 * other, pi, r1);
            cgo_min_dist(box, pos + 2 * base, pi, r2);
            cgo_min_dist(box, pos + 2 * dto, pi, r3);
            circumcenter3(r1, r2, r3, vother);

            double Akd = KA * (AP[2 * base] - APpref[2 * base]);
            double Pkd = KP * (AP[2 * base + 1] - APpref[2 * base + 1]);
            double Ajd = KA * (AP[2 * other] - APpref[2 * other]);
            double Pjd = KP * (AP[2 * other + 1] - APpref[2 * other + 1]);

            double dAk[2] = {0.5 * (vnext[1] - vother[1]), 0.5 * (vother[0] - vnext[0])};
            dl[0] = vnext[0] - vcur[0]; dl[1] = vnext[1] - vcur[1];
            dln = sqrt(dl[0] * dl[0] + dl[1] * dl[1]);
            dn[0] = vcur[0] - vother[0]; dn[1] = vcur[1] - vother[1];
            dnn = sqrt(dn[0] * dn[0] + dn[1] * dn[1]);
            if (dnn < thr) dnn = thr;
            if (dln < thr) dln = thr;
            double dPk[2] = {dl[0] / dln - dn[0] / dnn, dl[1] / dln - dn[1] / dnn};
            /* base's unlike edges at vcur: (vcur, vnext) with i, (vcur, vother) with other */
            double wbo = tension_w(ten, base, other);
            dT[0] += wib * dl[0] / dln - wbo * dn[0] / dnn;
            dT[1] += wib * dl[1] / dln - wbo * dn[1] / dnn;

            double dAj[2] = {0.5 * (vother[1] - vlast[1]), 0.5 * (vlast[0] - vother[0])};
            dl[0] = vother[0] - vcur[0]; dl[1] = vother[1] - vcur[1];
            dln = sqrt(dl[0] * dl[0] + dl[1] * dl[1]);
            dn[0] = vcur[0] - vlast[0]; dn[1] = vcur[1] - vlast[1];
            dnn = sqrt(dn[0] * dn[0] + dn[1] * dn[1]);
            if (dnn < thr) dnn = thr;
            if (dln < thr) dln = thr;
            double dPj[2] = {dl[0] / dln - dn[0] / dnn, dl[1] / dln - dn[1] / dnn};
            /* other's unlike edges at vcur: (vlast, vcur) with i, (vother, vcur) with base */
            dT[0] += -wio * dn[0] / dnn + wbo * dl[0] / dln;
            dT[1] += -wio * dn[1] / dnn + wbo * dl[1] / dln;

            double ex = 2.0 * Adiff * dAi[0] + 2.0 * Pdiff * dPi[0];
            double ey = 2.0 * Adiff * dAi[1] + 2.0 * Pdiff * dPi[1];
            ex += 2.0 * Akd * dAk[0] + 2.0 * Pkd * dPk[0];
            ey += 2.0 * Akd * dAk[1] + 2.0 * Pkd * dPk[1];
            ex += 2.0 * Ajd * dAj[0] + 2.0 * Pjd * dPj[0];
            ey += 2.0 * Ajd * dAj[1] + 2.0 * Pjd * dPj[1];
            ex += dT[0];
            ey += dT[1];
            /* v*M (inc/utility/Matrix.h:128-135) */
            const double *M = dh + 4 * n;
            fx += ex * M[0] + ey * M[2];
            fy += ex * M[1] + ey * M[3];
            vlast = vcur;
        }
        F[2 * i] = fx;
        F[2 * i + 1] = fy;
    }
    return 0;
}

/* VoronoiQuadraticEnergy::computeEnergy (src/models/voronoiQuadraticEnergy.cpp:384-397) */
double cgo_voronoi_energy(int N, const double *AP, const double *APpref, double KA, double KP)
{
    double E = 0.0;
    for (int n = 0; n < N; ++n) {
        double da = AP[2 * n] - APpref[2 * n], dp = AP[2 * n + 1] - APpref[2 * n + 1];
        E += KA * da * da;
        E += KP * dp * dp;
    }
    return E;
}

/* selfPropelledParticleDynamics::integrateEquationsOfMotionCPU
 * (src/updaters/selfPropelledParticleDynamics.cpp:67-101) with the normal deviate supplied, then
 * voronoiModelBase::movePointsCPU (src/models/voronoiModelBase.cpp:141-163). */
void cgo_spp_step(int N, double *pos, const double *box, const double *F, double *theta, const double *motility,
                  const double *noise, double dt, double mu)
{
    for (int i = 0; i < N; ++i) {
        double v0 = motility[2 * i], Dr = motility[2 * i + 1];
        double vx = v0 * cos(theta[i]);
        double vy = v0 * sin(theta[i]);
        double dx = dt * (vx + mu * F[2 * i]);
        double dy = dt * (vy + mu * F[2 * i + 1]);
        double th = theta[i];
        if (!(vx == 0. && vy == 0.)) th = atan2(vy, vx);
        theta[i] = th + noise[i] * sqrt(2.0 * dt * Dr);
        pos[2 * i] += dx;
        pos[2 * i + 1] += dy;
        cgo_put_in_box(box, pos + 2 * i);
    }
}

int cgo_voronoi_spp_run(int N, double *pos, const double *box, int K, int *nn, int *nbr, double *theta,
                        const double *motility, const double *APpref, double KA, double KP, double dt,
                        double mu, int n_steps, const double *noise, double *F_out, double *AP_out)
{
    double *AP = (double *)malloc(sizeof(double) * 2 * N);
    double *F = (double *)malloc(sizeof(double) * 2 * N);
    int st = 0;
    for (int s = 0; s < n_steps; ++s) {
        cgo_voronoi_geometry(N, pos, box, K, nn, nbr, AP);
        st = cgo_voronoi_forces(N, pos, box, K, nn, nbr, AP, APpref, KA, KP, F);
        if (st) break;
        if (F_out && s == n_steps - 1) memcpy(F_out, F, sizeof(double) * 2 * N);
        if (AP_out && s == n_steps - 1) memcpy(AP_out, AP, sizeof(double) * 2 * N);
        cgo_spp_step(N, pos, box, F, theta, motility, noise + (size_t)s * N, dt, mu);
        st = cgo_periodic_delaunay(N, pos, box, K, nn, nbr);
        if (st) break;
    }
    free(AP);
    free(F);
    return st;
}

/* brownianParticleDynamics::integrateEquationsOfMotionCPU (src/updaters/brownianParticleDynamics.cpp:92-109):
 * two normals per degree of freedom, x then y, in index order. */
void cgo_brownian_disp(int N, const double *F, const double *noise2, double dt, double mu, double T,
                       double *disp)
{
    for (int i = 0; i < N; ++i) {
        double r1 = noise2[2 * i], r2 = noise2[2 * i + 1];
        disp[2 * i] = r1 * sqrt(2.0 * dt * T * mu) + dt * mu * F[2 * i];
        disp[2 * i + 1] = r2 * sqrt(2.0 * dt * T * mu) + dt * mu * F[2 * i + 1];
    }
}

/* ------------------------------------------------------------------------------------------ */
/* vertex model                                                                                */
/* ------------------------------------------------------------------------------------------ */

static int slot_of(const int *row, int z, int v)
{
    for (int s = 0; s < z; ++s)
        if (row[s] == v) return s;
    return -1;
}

int cgo_vertex_from_delaunay(int N, const double *pos, const double *box, int K, const int *nn, const int *nbr,
                             int vmax, double *vpos, int *vn, int *vcn, int *cvn, int *cv)
{
    int *tri = (int *)malloc(sizeof(int) * N * K);
    int nv = 0;
    /* triangles in the order of src/models/voronoiModelBase.cpp:380-423 (owner = smallest index) */
    for (int c = 0; c < N; ++c) {
        int z = nn[c];
        for (int n = 0; n < z; ++n) {
            int a = nbr[c * K + n], b = nbr[c * K + (n + 1) % z];
            tri[c * K + n] = -1;
            if (c < a && c < b) tri[c * K + n] = nv++;
        }
    }
    if (nv != 2 * N) { free(tri); return -3; }
    for (int c = 0; c < N; ++c) {
        int z = nn[c];
        for (int n = 0; n < z; ++n) {
            if (tri[c * K + n] >= 0) continue;
            int a = nbr[c * K + n], b = nbr[c * K + (n + 1) % z];
            int owner = a < b ? a : b;
            int nxt = (owner == a) ? b : c; /* the vertex following owner in (c,a,b) CCW */
            int s = slot_of(nbr + owner * K, nn[owner], nxt);
            if (s < 0) { free(tri); return -1; }
            tri[c * K + n] = tri[owner * K + s];
        }
    }
    for (int c = 0; c < N; ++c) {
        int z = nn[c];
        if (z > vmax) { free(tri); return -2; }
        cvn[c] = z;
        for (int n = 0; n < z; ++n) {
            int v = tri[c * K + n];
            cv[c * vmax + n] = v;
            int a = nbr[c * K + n], b = nbr[c * K + (n + 1) % z];
            if (c < a && c < b) {
                /* vertex of triangle (c,a,b): circumcentre, put in the box */
                double ra[2], rb[2], q[2];
                cgo_min_dist(box, pos + 2 * a, pos + 2 * c, ra);
                cgo_min_dist(box, pos + 2 * b, pos + 2 * c, rb);
                circumcenter0(ra, rb, q);
                vpos[2 * v] = pos[2 * c] + q[0];
                vpos[2 * v + 1] = pos[2 * c + 1] + q[1];
                cgo_put_in_box(box, vpos + 2 * v);
                int cells[3] = {c, a, b};
                for (int f = 0; f < 3; ++f) {
                    vcn[3 * v + f] = cells[f];
                    /* neighbour across the edge opposite cells[f]: triangle (q, x, r) */
                    int qc = cells[(f + 1) % 3], rc = cells[(f + 2) % 3];
                    int s = slot_of(nbr + qc * K, nn[qc], rc);
                    if (s < 0) { free(tri); return -1; }
                    int sp = (s - 1 + nn[qc]) % nn[qc];
                    vn[3 * v + f] = tri[qc * K + sp];
                }
            }
        }
    }
    free(tri);
    return nv;
}

/* vertexModelBase::computeGeometryCPU (src/models/vertexModelBase.cpp:248-297): positions relative
 * to the vertex at slot z-2, signed shoelace area and perimeter summed from slot z-1. */
void cgo_vertex_geometry(int Nc, const double *vpos, const double *box, int vmax, const int *cvn, const int *cv,
                         double *AP)
{
    for (int i = 0; i < Nc; ++i) {
        int z = cvn[i];
        const int *row = cv + i * vmax;
        const double *cp = vpos + 2 * row[z - 2];
        double vcur[2], vnext[2];
        cgo_min_dist(box, vpos + 2 * row[z - 1], cp, vcur);
        double A = 0.0, P = 0.0;
        for (int n = 0; n < z; ++n) {
            cgo_min_dist(box, vpos + 2 * row[n], cp, vnext);
            A += signed_area_part(vcur, vnext);
            double dx = vcur[0] - vnext[0], dy = vcur[1] - vnext[1];
            P += sqrt(dx * dx + dy * dy);
            vcur[0] = vnext[0];
            vcur[1] = vnext[1];
        }
        AP[2 * i] = A;
        AP[2 * i + 1] = P;
    }
}

/* computeForceSetVertexModel (inc/utility/functions.h:330-354) */
static void force_set_vm(const double *vcur, const double *vlast, const double *vnext, double Adiff,
                         double Pdiff, double *f)
{
    double dAx = 0.5 * (vlast[1] - vnext[1]);
    double dAy = -0.5 * (vlast[0] - vnext[0]);
    double dlx = vlast[0] - vcur[0], dly = vlast[1] - vcur[1];
    double dln = sqrt(dlx * dlx + dly * dly);
    double dnx = vcur[0] - vnext[0], dny = vcur[1] - vnext[1];
    double dnn = sqrt(dnx * dnx + dny * dny);
    double dPx = dlx / dln - dnx / dnn;
    double dPy = dly / dln - dny / dnn;
    f[0] = 2.0 * (Adiff * dAx + Pdiff * dPx);
    f[1] = 2.0 * (Adiff * dAy + Pdiff * dPy);
}


/* VertexQuadraticEnergy::computeForcesCPU (src/models/vertexQuadraticEnergy.cpp:71-113): the force
 * set of (vertex, cell) comes from the cell's (last, cur, next) vertices as stored by the geometry
 * pass at slot 3*v+f with vcn[3v+f] == cell (src/models/vertexModelBase.cpp:268-287); the force on a
 * vertex is the sum of its three sets in slot order. */
/* the cell other than `cell` among vertex v's three cells whose row holds vertex w (the cellIdx2
 * search of src/models/vertexQuadraticEnergyWithTension.cpp:108-119; the last match wins) */
static int cell_across(int v, int w, int cell, const int *vcn, const int *cvn, const int *cv, int vmax)
{
    int out = 0;
    for (int f = 0; f < 3; ++f) {
        int c2 = vcn[3 * v + f];
        if (c2 == cell) continue;
        for (int n = 0; n < cvn[c2]; ++n)
            if (cv[(size_t)c2 * vmax + n] == w) out = c2;
    }
    return out;
}

static void vertex_forces_impl(int Nc, int Nv, const double *vpos, const double *box, int vmax, const int *cvn,
                               const int *cv, const int *vcn, const double *AP, const double *APpref, double KA,
                               double KP, const tension_t *ten, double *F);

void cgo_vertex_forces(int Nc, int Nv, const double *vpos, const double *box, int vmax, const int *cvn,
                       const int *cv, const int *vcn, const double *AP, const double *APpref, double KA,
                       double KP, double *F)
{
    vertex_forces_impl(Nc, Nv, vpos, box, vmax, cvn, cv, vcn, AP, APpref, KA, KP, NULL, F);
}

/* VertexQuadraticEnergyWithTension::computeVertexTensionForcesCPU
 * (src/models/vertexQuadraticEnergyWithTension.cpp:65-151): each force set (vertex, cell) also gets
 * -gamma (vcur - vnext) / |vcur - vnext| for the edge to the cell's next vertex when the cell across
 * that edge has another type; gamma = the one value, or tensionMatrix[cellTypeIndexer(type of the
 * set's cell, type across)] = row (type across), column (own type). No norm clamp. */
void cgo_vertex_tension_forces(int Nc, int Nv, const double *vpos, const double *box, int vmax, const int *cvn,
                               const int *cv, const int *vcn, const double *AP, const double *APpref, double KA,
                               double KP, const int *ctype, int ntypes, double gamma, const double *tmat,
                               double *F)
{
    tension_t t = {ctype, ntypes, gamma, tmat};
    vertex_forces_impl(Nc, Nv, vpos, box, vmax, cvn, cv, vcn, AP, APpref, KA, KP, &t, F);
}

/* the quadratic energy plus gamma l over every edge between cells of different types, each edge
 * once (the reference leaves VertexQuadraticEnergyWithTension::computeEnergy unimplemented; this is
 * the energy whose gradient the forces above are) */
double cgo_vertex_tension_energy(int Nc, const double *vpos, const double *box, int vmax, const int *cvn,
                                 const int *cv, const int *vcn, const double *AP, const double *APpref, double KA,
                                 double KP, const int *ctype, int ntypes, double gamma, const double *tmat)
{
    tension_t t = {ctype, ntypes, gamma, tmat};
    double E = cgo_voronoi_energy(Nc, AP, APpref, KA, KP), ET = 0.0;
    for (int i = 0; i < Nc; ++i) {
        int z = cvn[i];
        const int *row = cv + (size_t)i * vmax;
        for (int n = 0; n < z; ++n) {
            int v = row[n], w = row[(n + 1) % z];
            double d[2];
            cgo_min_dist(box, vpos + 2 * w, vpos + 2 * v, d);
            ET += sqrt(d[0] * d[0] + d[1] * d[1]) * tension_w(&t, cell_across(v, w, i, vcn, cvn, cv, vmax), i);
        }
    }
    return E + 0.5 * ET;
}

static void vertex_forces_impl(int Nc, int Nv, const double *vpos, const double *box, int vmax, const int *cvn,
                               const int *cv, const int *vcn, const double *AP, const double *APpref, double KA,
                               double KP, const tension_t *ten, double *F)
{
    double *fs = (double *)calloc((size_t)6 * Nv, sizeof(double));
    for (int i = 0; i < Nc; ++i) {
        int z = cvn[i];
        const int *row = cv + (size_t)i * vmax;
        const double *cp = vpos + 2 * row[z - 2];
        double vlast[2] = {0.0, 0.0}, vcur[2], vnext[2];
        int vidx = row[z - 1];
        cgo_min_dist(box, vpos + 2 * vidx, cp, vcur);
        double Adiff = KA * (AP[2 * i] - APpref[2 * i]);
        double Pdiff = KP * (AP[2 * i + 1] - APpref[2 * i + 1]);
        for (int n = 0; n < z; ++n) {
            int fsidx = -1;
            for (int f = 0; f < 3; ++f)
                if (vcn[3 * vidx + f] == i) fsidx = 3 * vidx + f;
            int nv = row[n];
            cgo_min_dist(box, vpos + 2 * nv, cp, vnext);
            if (fsidx >= 0) force_set_vm(vcur, vlast, vnext, Adiff, Pdiff, fs + 2 * (size_t)fsidx);
            if (fsidx >= 0 && ten) {
                double g = tension_w(ten, cell_across(vidx, nv, i, vcn, cvn, cv, vmax), i);
                if (g != 0.0) {
                    double dx = vcur[0] - vnext[0], dy = vcur[1] - vnext[1];
                    double dn = sqrt(dx * dx + dy * dy);
                    fs[2 * (size_t)fsidx] -= g * dx / dn;
                    fs[2 * (size_t)fsidx + 1] -= g * dy / dn;
                }
            }
            vlast[0] = vcur[0]; vlast[1] = vcur[1];
            vcur[0] = vnext[0]; vcur[1] = vnext[1];
            vidx = nv;
        }
    }
    for (int v = 0; v < Nv; ++v) {
        double fx = 0.0, fy = 0.0;
        for (int f = 0; f < 3; ++f) {
            fx += fs[2 * (size_t)(3 * v + f)];
            fy += fs[2 * (size_t)(3 * v + f) + 1];
        }
        F[2 * v] = fx;
        F[2 * v + 1] = fy;
    }
    free(fs);
}

/* walk a cell's CCW vertex row until vcur == target: the loop shape of getCellVertexSetForT1
 * (src/models/vertexModelBase.cpp:536-546) */
static void find_in_cell(const int *row, int cneigh, int target, int *vlast, int *vcur, int *vnext)
{
    int l = row[cneigh - 2], c = row[cneigh - 1], nx = row[0];
    for (int cn = 0; cn < cneigh; ++cn) {
        nx = row[cn];
        if (c == target) break;
        l = c;
        c = nx;
    }
    *vlast = l;
    *vcur = c;
    *vnext = nx;
}

/* vertexModelBase::getCellVertexSetForT1 (src/models/vertexModelBase.cpp:507-625); the first
 * (dead) loop of the reference is omitted since its results are unused. */
static void t1_sets(int v1, int v2, const int *vcn, const int *cvn, const int *cv, int vmax, int cs[4],
                    int vs[4])
{
    int c1 = vcn[3 * v1], c2 = vcn[3 * v1 + 1], c3 = vcn[3 * v1 + 2];
    for (int f = 0; f < 3; ++f) {
        int t = vcn[3 * v2 + f];
        if (t != c1 && t != c2 && t != c3) cs[3] = t;
    }
    int cells[3] = {c1, c2, c3};
    for (int q = 0; q < 3; ++q) {
        int c = cells[q];
        int l, cur, nx;
        find_in_cell(cv + (size_t)c * vmax, cvn[c], v1, &l, &cur, &nx);
        if (l == v2) cs[0] = c;
        else if (nx == v2) cs[2] = c;
        else cs[1] = c;
    }
    int l, cur, nx;
    find_in_cell(cv + (size_t)cs[1] * vmax, cvn[cs[1]], v1, &l, &cur, &nx);
    vs[0] = l;
    vs[1] = nx;
    find_in_cell(cv + (size_t)cs[3] * vmax, cvn[cs[3]], v2, &l, &cur, &nx);
    vs[3] = l;
    vs[2] = nx;
}

/* vertexModelBase::testAndPerformT1TransitionsCPU (src/models/vertexModelBase.cpp:631-787): one
 * sequential sweep over vertex1 ascending and its three neighbour slots; each flip is applied at
 * once and later tests see the moved vertices and the rewired lists. */
int cgo_vertex_t1(int Nc, int Nv, double *vpos, const double *box, double threshold, int vmax, int *vn,
                  int *vcn, int *cvn, int *cv, int max_events, int *events)
{
    (void)Nc;
    int nflip = 0;
    int cs[4] = {0, 0, 0, 0}, vs[4] = {0, 0, 0, 0};
    int *copy = (int *)malloc(sizeof(int) * (vmax + 2));
    for (int vertex1 = 0; vertex1 < Nv; ++vertex1) {
        double v1[2] = {vpos[2 * vertex1], vpos[2 * vertex1 + 1]};
        for (int vv = 0; vv < 3; ++vv) {
            int vertex2 = vn[3 * vertex1 + vv];
            if (!(vertex1 < vertex2)) continue;
            double v2[2] = {vpos[2 * vertex2], vpos[2 * vertex2 + 1]};
            double e[2];
            cgo_min_dist(box, v1, v2, e);
            if (!(sqrt(e[0] * e[0] + e[1] * e[1]) < threshold)) continue;
            t1_sets(vertex1, vertex2, vcn, cvn, cv, vmax, cs, vs);
            if (cvn[cs[0]] == 3 || cvn[cs[2]] == 3) continue;
            if (cvn[cs[1]] + 1 > vmax || cvn[cs[3]] + 1 > vmax) { free(copy); return -2; }
            double mid[2] = {v2[0] + 0.5 * e[0], v2[1] + 0.5 * e[1]};
            v1[0] = mid[0] - e[1];
            v1[1] = mid[1] + e[0];
            v2[0] = mid[0] + e[1];
            v2[1] = mid[1] - e[0];
            cgo_put_in_box(box, v1);
            cgo_put_in_box(box, v2);
            vpos[2 * vertex1] = v1[0]; vpos[2 * vertex1 + 1] = v1[1];
            vpos[2 * vertex2] = v2[0]; vpos[2 * vertex2 + 1] = v2[1];
            if (nflip < max_events) {
                events[2 * nflip] = vertex1;
                events[2 * nflip + 1] = vertex2;
            }
            ++nflip;
            for (int vert = 0; vert < 3; ++vert) {
                if (vcn[3 * vertex1 + vert] == cs[2]) vcn[3 * vertex1 + vert] = cs[3];
                if (vcn[3 * vertex2 + vert] == cs[0]) vcn[3 * vertex2 + vert] = cs[1];
                if (vn[3 * vs[1] + vert] == vertex1) vn[3 * vs[1] + vert] = vertex2;
                if (vn[3 * vs[2] + vert] == vertex2) vn[3 * vs[2] + vert] = vertex1;
                if (vn[3 * vertex1 + vert] == vs[1]) vn[3 * vertex1 + vert] = vs[2];
                if (vn[3 * vertex2 + vert] == vs[2]) vn[3 * vertex2 + vert] = vs[1];
            }
            /* cell i loses vertex2 */
            int *row = cv + (size_t)cs[0] * vmax;
            int cneigh = cvn[cs[0]], cidx = 0;
            for (int cc = 0; cc < cneigh - 1; ++cc) {
                if (row[cc] == vertex2) cidx += 1;
                row[cc] = row[cidx];
                cidx += 1;
            }
            cvn[cs[0]] -= 1;
            /* cell j gains vertex2 after vertex1 */
            row = cv + (size_t)cs[1] * vmax;
            cneigh = cvn[cs[1]];
            cidx = 0;
            for (int cc = 0; cc < cneigh; ++cc) {
                int ci = row[cc];
                copy[cidx++] = ci;
                if (ci == vertex1) copy[cidx++] = vertex2;
            }
            for (int cc = 0; cc < cneigh + 1; ++cc) row[cc] = copy[cc];
            cvn[cs[1]] += 1;
            /* cell k loses vertex1 */
            row = cv + (size_t)cs[2] * vmax;
            cneigh = cvn[cs[2]];
            cidx = 0;
            for (int cc = 0; cc < cneigh - 1; ++cc) {
                if (row[cc] == vertex1) cidx += 1;
                row[cc] = row[cidx];
                cidx += 1;
            }
            cvn[cs[2]] -= 1;
            /* cell l gains vertex1 after vertex2 */
            row = cv + (size_t)cs[3] * vmax;
            cneigh = cvn[cs[3]];
            cidx = 0;
            for (int cc = 0; cc < cneigh; ++cc) {
                int ci = row[cc];
                copy[cidx++] = ci;
                if (ci == vertex2) copy[cidx++] = vertex1;
            }
            for (int cc = 0; cc < cneigh + 1; ++cc) row[cc] = copy[cc];
            cvn[cs[3]] = cneigh + 1;
        }
    }
    free(copy);
    return nflip;
}

int cgo_vertex_brownian_run(int Nc, int Nv, double *vpos, const double *box, int vmax, int *vn, int *vcn,
                            int *cvn, int *cv, const double *APpref, double KA, double KP, double dt,
                            double mu, double T, double t1_threshold, int n_steps, const double *noise,
                            double *F_out, double *AP_out, int *n_t1_out)
{
    double *AP = (double *)malloc(sizeof(double) * 2 * Nc);
    double *F = (double *)malloc(sizeof(double) * 2 * Nv);
    double *disp = (double *)malloc(sizeof(double) * 2 * Nv);
    int total = 0, st = 0;
    for (int s = 0; s < n_steps; ++s) {
        cgo_vertex_geometry(Nc, vpos, box, vmax, cvn, cv, AP);
        cgo_vertex_forces(Nc, Nv, vpos, box, vmax, cvn, cv, vcn, AP, APpref, KA, KP, F);
        if (F_out && s == n_steps - 1) memcpy(F_out, F, sizeof(double) * 2 * Nv);
        if (AP_out && s == n_steps - 1) memcpy(AP_out, AP, sizeof(double) * 2 * Nc);
        cgo_brownian_disp(Nv, F, noise + (size_t)s * 2 * Nv, dt, mu, T, disp);
        for (int v = 0; v < Nv; ++v) {
            vpos[2 * v] += disp[2 * v];
            vpos[2 * v + 1] += disp[2 * v + 1];
            cgo_put_in_box(box, vpos + 2 * v);
        }
        int nf = cgo_vertex_t1(Nc, Nv, vpos, box, t1_threshold, vmax, vn, vcn, cvn, cv, 0, NULL);
        if (nf < 0) { st = nf; break; }
        total += nf;
    }
    if (n_t1_out) *n_t1_out = total;
    free(AP);
    free(F);
    free(disp);
    return st;
}

/* ------------------------------------------------------------------------------------------ */
/* FIRE, CPU conventions: EnergyMinimizerFIRE::velocityVerletCPU (src/updaters/               */
/* EnergyMinimizerFIRE2D.cpp:120-151), fireStepCPU (:212-264), minimize (:269-284)             */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    int model; /* 0 Voronoi, 1 vertex */
    int Nc, Nv, N;
    double *pos;
    const double *box;
    int K, *nn, *nbr;
    int vmax, *vn, *vcn, *cvn, *cv;
    const double *APpref;
    double KA, KP, t1;
    double *AP;
} fire_sys;

static int fire_forces(fire_sys *s, double *F)
{
    if (s->model == 0) {
        cgo_voronoi_geometry(s->N, s->pos, s->box, s->K, s->nn, s->nbr, s->AP);
        return cgo_voronoi_forces(s->N, s->pos, s->box, s->K, s->nn, s->nbr, s->AP, s->APpref, s->KA,
                                  s->KP, F);
    }
    cgo_vertex_geometry(s->Nc, s->pos, s->box, s->vmax, s->cvn, s->cv, s->AP);
    cgo_vertex_forces(s->Nc, s->Nv, s->pos, s->box, s->vmax, s->cvn, s->cv, s->vcn, s->AP, s->APpref,
                      s->KA, s->KP, F);
    return 0;
}

static int fire_topology(fire_sys *s)
{
    if (s->model == 0) return cgo_periodic_delaunay(s->N, s->pos, s->box, s->K, s->nn, s->nbr);
    int nf = cgo_vertex_t1(s->Nc, s->Nv, s->pos, s->box, s->t1, s->vmax, s->vn, s->vcn, s->cvn, s->cv, 0,
                           NULL);
    return nf < 0 ? nf : 0;
}

static int fire_minimize(fire_sys *s, cgo_fire_params *p, double *v, double *F_out)
{
    int N = s->N;
    double *F = (double *)malloc(sizeof(double) * 2 * N);
    double *d = (double *)malloc(sizeof(double) * 2 * N);
    int st = fire_forces(s, F);
    p->force_max = 110.0;
    while (st == 0 && p->iterations < p->max_iterations && sqrt(p->force_max) > p->force_cutoff) {
        p->iterations += 1;
        /* velocity Verlet */
        double dt = p->dt;
        for (int i = 0; i < 2 * N; ++i) {
            d[i] = dt * v[i] + 0.5 * dt * dt * F[i];
            v[i] += 0.5 * dt * F[i];
        }
        for (int i = 0; i < N; ++i) {
            s->pos[2 * i] += d[2 * i];
            s->pos[2 * i + 1] += d[2 * i + 1];
            cgo_put_in_box(s->box, s->pos + 2 * i);
        }
        st = fire_topology(s);
        if (st) break;
        st = fire_forces(s, F);
        if (st) break;
        for (int i = 0; i < 2 * N; ++i) v[i] += 0.5 * dt * F[i];
        /* FIRE step */
        double power = 0.0, fnorm = 0.0, vnorm = 0.0;
        p->force_max = 0.0;
        for (int i = 0; i < N; ++i) {
            power += F[2 * i] * v[2 * i] + F[2 * i + 1] * v[2 * i + 1];
            double fdot = F[2 * i] * F[2 * i] + F[2 * i + 1] * F[2 * i + 1];
            if (fdot > p->force_max) p->force_max = fdot;
            fnorm += fdot;
            vnorm += v[2 * i] * v[2 * i] + v[2 * i + 1] * v[2 * i + 1];
        }
        p->power = power;
        double scaling = 0.0;
        if (fnorm > 0.) scaling = sqrt(vnorm / fnorm);
        for (int i = 0; i < 2 * N; ++i) v[i] = (1.0 - p->alpha) * v[i] + p->alpha * scaling * F[i];
        if (power > 0) {
            if (p->n_since_negative_power > p->n_min) {
                p->dt = fmin(p->dt * p->dt_inc, p->dt_max);
                p->alpha = p->alpha * p->alpha_dec;
            }
            p->n_since_negative_power += 1;
        } else {
            p->dt = p->dt * p->dt_dec;
            p->dt = fmax(p->dt, p->dt_min);
            p->alpha = p->alpha_start;
            for (int i = 0; i < 2 * N; ++i) v[i] = 0.0;
        }
    }
    if (F_out) memcpy(F_out, F, sizeof(double) * 2 * N);
    free(F);
    free(d);
    return st;
}

int cgo_fire_voronoi(int N, double *pos, const double *box, int K, int *nn, int *nbr, const double *APpref,
                     double KA, double KP, cgo_fire_params *prm, double *vel, double *F_out,
                     double *AP_out)
{
    fire_sys s;
    memset(&s, 0, sizeof(s));
    s.model = 0;
    s.N = s.Nc = N;
    s.pos = pos;
    s.box = box;
    s.K = K;
    s.nn = nn;
    s.nbr = nbr;
    s.APpref = APpref;
    s.KA = KA;
    s.KP = KP;
    s.AP = (double *)malloc(sizeof(double) * 2 * N);
    int st = fire_minimize(&s, prm, vel, F_out);
    if (AP_out) memcpy(AP_out, s.AP, sizeof(double) * 2 * N);
    free(s.AP);
    return st;
}

int cgo_fire_vertex(int Nc, int Nv, double *vpos, const double *box, int vmax, int *vn, int *vcn, int *cvn,
                    int *cv, const double *APpref, double KA, double KP, double t1_threshold,
                    cgo_fire_params *prm, double *vel, double *F_out, double *AP_out)
{
    fire_sys s;
    memset(&s, 0, sizeof(s));
    s.model = 1;
    s.Nc = Nc;
    s.Nv = Nv;
    s.N = Nv;
    s.pos = vpos;
    s.box = box;
    s.vmax = vmax;
    s.vn = vn;
    s.vcn = vcn;
    s.cvn = cvn;
    s.cv = cv;
    s.APpref = APpref;
    s.KA = KA;
    s.KP = KP;
    s.t1 = t1_threshold;
    s.AP = (double *)malloc(sizeof(double) * 2 * Nc);
    int st = fire_minimize(&s, prm, vel, F_out);
    if (AP_out) memcpy(AP_out, s.AP, sizeof(double) * 2 * Nc);
    free(s.AP);
    return st;
}

/* selfPropelledCellVertexDynamics::integrateEquationsOfMotionCPU
 * (src/updaters/selfPropelledCellVertexDynamics.cpp:81-122): vertex displacement from the mean of
 * its three cells' v0 (cos th, sin th) plus mu F, then the cells' directors advance by
 * xi sqrt(2 dt Dr) (one normal per cell, in index order); then move and T1 sweep. */
int cgo_vertex_spp_run(int Nc, int Nv, double *vpos, const double *box, int vmax, int *vn, int *vcn,
                       int *cvn, int *cv, const double *APpref, double KA, double KP, double *theta,
                       const double *motility, double dt, double mu, double t1_threshold, int n_steps,
                       const double *noise)
{
    double *AP = (double *)malloc(sizeof(double) * 2 * Nc);
    double *F = (double *)malloc(sizeof(double) * 2 * Nv);
    double *disp = (double *)malloc(sizeof(double) * 2 * Nv);
    int st = 0;
    for (int s = 0; s < n_steps; ++s) {
        cgo_vertex_geometry(Nc, vpos, box, vmax, cvn, cv, AP);
        cgo_vertex_forces(Nc, Nv, vpos, box, vmax, cvn, cv, vcn, AP, APpref, KA, KP, F);
        for (int i = 0; i < Nv; ++i) {
            int c0 = vcn[3 * i], c1 = vcn[3 * i + 1], c2 = vcn[3 * i + 2];
            double v1 = motility[2 * c0], v2 = motility[2 * c1], v3 = motility[2 * c2];
            double dx = v1 * cos(theta[c0]);
            dx += v2 * cos(theta[c1]);
            dx += v3 * cos(theta[c2]);
            dx /= 3.0;
            double dy = v1 * sin(theta[c0]);
            dy += v2 * sin(theta[c1]);
            dy += v3 * sin(theta[c2]);
            dy /= 3.0;
            disp[2 * i] = dt * (dx + mu * F[2 * i]);
            disp[2 * i + 1] = dt * (dy + mu * F[2 * i + 1]);
        }
        for (int c = 0; c < Nc; ++c) theta[c] += noise[(size_t)s * Nc + c] * sqrt(2.0 * dt * motility[2 * c + 1]);
        for (int v = 0; v < Nv; ++v) {
            vpos[2 * v] += disp[2 * v];
            vpos[2 * v + 1] += disp[2 * v + 1];
            cgo_put_in_box(box, vpos + 2 * v);
        }
        int nf = cgo_vertex_t1(Nc, Nv, vpos, box, t1_threshold, vmax, vn, vcn, cvn, cv, 0, NULL);
        if (nf < 0) { st = nf; break; }
    }
    free(AP);
    free(F);
    free(disp);
    return st;
}
