// cellgpu_b200 -- common device code: periodic box arithmetic, exact geometric predicates,
// counter-based RNG, warp helpers. sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cellgpu_b200.h"

#define CG_HD __host__ __device__ __forceinline__
#define CG_D __device__ __forceinline__

namespace cg {

constexpr int WARP = 32;

// ------------------------------------------------------------------------------------------
// Instance descriptor: one independent monolayer of the batch. A single-instance system is
// the drop-in for the reference's one-monolayer call path.
// ------------------------------------------------------------------------------------------
struct Inst {
    double Lx, Ly;      // periodic box sides (gpubox::setSquare(x,y), inc/utility/gpubox.h:83-93)
    double iLx, iLy;    // 1/L as gpubox stores xi11, xi22
    int off, n;         // first global cell (or vertex) and count
    int bin_off, nbx, nby;  // cell-list bins of this instance
    double bsx, bsy;    // bin sides
    int voff, nv;       // vertex-model vertices (off/n are cells)
    unsigned long long seed;  // Philox key of the instance's device noise (counters are local indices)
    unsigned step_off;  // added to the system's step counter in the noise counters: the instance's own
                        // step count when it joined this system (0 for an instance created here)
};

// SplitMix64 finaliser (G. Steele, D. Lea, C. Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014): decorrelated per-instance keys from one seed and the instance index.
CG_HD unsigned long long mix_seed(unsigned long long seed, unsigned long long index)
{
    unsigned long long z = seed + (index + 1ull) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// gpubox::minDist for a rectangular box (inc/utility/gpubox.h:154-165). The while loops and
// half-box thresholds are kept so the FP64 result is bit-identical to the reference's. Inputs far
// outside the box (or non-finite) are first reduced in one step, so no loop can run away on the
// device: for points inside the box the pre-reduction never triggers.
CG_HD double2 min_dist(double2 p1, double2 p2, double Lx, double Ly)
{
    double hx = Lx * 0.5, hy = Ly * 0.5;
    double x = p1.x - p2.x, y = p1.y - p2.y;
    if (!(fabs(x) <= 2.0 * Lx)) x -= Lx * rint(x / Lx);
    if (!(fabs(y) <= 2.0 * Ly)) y -= Ly * rint(y / Ly);
    while (x < -hx) x += Lx;
    while (y < -hy) y += Ly;
    while (x > hx) x -= Lx;
    while (y > hy) y -= Ly;
    return make_double2(x, y);
}

// min_dist with selects in place of the while loops, for warps whose lanes would take different
// paths through them (the thread-per-cell force pass gathers eight neighbours per lane): after the
// pre-reduction |x| <= 2 L, so each loop runs at most twice, and two conditional steps per loop give
// the same sequence of additions, hence the same bits
CG_D double wrap_sel(double x, double L, double h)
{
    if (!(fabs(x) <= 2.0 * L)) x -= L * rint(x / L);
    x = x < -h ? x + L : x;
    x = x < -h ? x + L : x;
    x = x > h ? x - L : x;
    x = x > h ? x - L : x;
    return x;
}

CG_D double2 min_dist_sel(double2 p1, double2 p2, double Lx, double Ly)
{
    return make_double2(wrap_sel(p1.x - p2.x, Lx, Lx * 0.5), wrap_sel(p1.y - p2.y, Ly, Ly * 0.5));
}

// gpubox::putInBoxReal (inc/utility/gpubox.h:131-152): v = xi*p, wrap v into [0,1) by +-1.0,
// p = L*v. Explicit round-to-nearest intrinsics keep the compiler from fusing anything.
CG_D double2 put_in_box(double2 p, double Lx, double Ly, double iLx, double iLy)
{
    double vx = __dmul_rn(iLx, p.x), vy = __dmul_rn(iLy, p.y);
    // one-step reduction for displacements of more than a box (or non-finite values), bounding
    // the loops below; a step that moves a point by less than one box never takes this branch
    if (!(vx >= -1.0 && vx < 2.0)) vx -= floor(vx);
    if (!(vy >= -1.0 && vy < 2.0)) vy -= floor(vy);
    while (vx < 0) vx = __dadd_rn(vx, 1.0);
    while (vy < 0) vy = __dadd_rn(vy, 1.0);
    while (vx >= 1.0) vx = __dsub_rn(vx, 1.0);
    while (vy >= 1.0) vy = __dsub_rn(vy, 1.0);
    return make_double2(__dmul_rn(Lx, vx), __dmul_rn(Ly, vy));
}

// ------------------------------------------------------------------------------------------
// Exact predicates (method of J. R. Shewchuk, Discrete Comput. Geom. 18, 1997): a floating-point
// filter and, when it cannot decide, exact evaluation with non-overlapping expansions. Points are
// relative to a centre at the origin, the form in which the reference feeds its local Delaunay
// construction (src/models/DelaunayLoc.cpp:171-273). Used for the Delaunay test and repair in both
// precision modes, so the topology is the same in FP64 and mixed mode.
// ------------------------------------------------------------------------------------------
CG_D void two_sum(double a, double b, double &x, double &y)
{
    double s = __dadd_rn(a, b);
    double bv = __dsub_rn(s, a);
    double av = __dsub_rn(s, bv);
    double br = __dsub_rn(b, bv);
    double ar = __dsub_rn(a, av);
    x = s;
    y = __dadd_rn(ar, br);
}

CG_D void two_prod(double a, double b, double &x, double &y)
{
    double p = __dmul_rn(a, b);
    x = p;
    y = __fma_rn(a, b, -p);
}

// h = e + b (grow with zero elimination); returns length
__device__ __noinline__ int exp_grow(int elen, const double *e, double b, double *h)
{
    double q = b, hh;
    int hidx = 0;
    for (int i = 0; i < elen; ++i) {
        double qn;
        two_sum(q, e[i], qn, hh);
        q = qn;
        if (hh != 0.0) h[hidx++] = hh;
    }
    if (q != 0.0 || hidx == 0) h[hidx++] = q;
    return hidx;
}

// h = e + f; scratch must hold elen+flen doubles. Repeated growth, ping-ponging between h and scratch.
__device__ __noinline__ int exp_sum(int elen, const double *e, int flen, const double *f, double *h,
                                    double *scratch)
{
    double *cur = scratch, *nxt = h;
    // make the final result land in h: choose the starting buffer by parity of flen
    if ((flen & 1) == 0) { cur = h; nxt = scratch; }
    for (int i = 0; i < elen; ++i) cur[i] = e[i];
    int n = elen;
    for (int j = 0; j < flen; ++j) {
        n = exp_grow(n, cur, f[j], nxt);
        double *t = cur; cur = nxt; nxt = t;
    }
    return n;
}

__device__ __noinline__ int exp_scale(int elen, const double *e, double b, double *h)
{
    double q, hh, p1, p0, sum;
    int hidx = 0;
    two_prod(e[0], b, q, hh);
    if (hh != 0.0) h[hidx++] = hh;
    for (int i = 1; i < elen; ++i) {
        two_prod(e[i], b, p1, p0);
        two_sum(q, p0, sum, hh);
        if (hh != 0.0) h[hidx++] = hh;
        two_sum(p1, sum, q, hh);
        if (hh != 0.0) h[hidx++] = hh;
    }
    if (q != 0.0 || hidx == 0) h[hidx++] = q;
    return hidx;
}

// product of two expansions of length <= 4: result <= 32 terms
__device__ __noinline__ int exp_mul4(int elen, const double *e, int flen, const double *f, double *h)
{
    double acc[32], tmp[8], scr[32];
    int n = 1;
    acc[0] = 0.0;
    for (int j = 0; j < flen; ++j) {
        int m = exp_scale(elen, e, f[j], tmp);
        double out[32];
        n = exp_sum(n, acc, m, tmp, out, scr);
        for (int i = 0; i < n; ++i) acc[i] = out[i];
    }
    for (int i = 0; i < n; ++i) h[i] = acc[i];
    return n;
}

CG_D int exp_sign(int n, const double *e)
{
    for (int i = n - 1; i >= 0; --i) {
        if (e[i] > 0.0) return 1;
        if (e[i] < 0.0) return -1;
    }
    return 0;
}

// a*b - c*d exactly, <= 4 terms
__device__ __noinline__ int exp_diff_prod(double a, double b, double c, double d, double *h)
{
    double p1, e1, p2, e2, scr[4];
    two_prod(a, b, p1, e1);
    two_prod(c, d, p2, e2);
    double x[2] = {e1, p1};
    double y[2] = {-e2, -p2};
    return exp_sum(2, x, 2, y, h, scr);
}

__device__ __noinline__ int exp_norm2(double a, double b, double *h)
{
    double p1, e1, p2, e2, scr[4];
    two_prod(a, a, p1, e1);
    two_prod(b, b, p2, e2);
    double x[2] = {e1, p1};
    double y[2] = {e2, p2};
    return exp_sum(2, x, 2, y, h, scr);
}

__device__ __noinline__ int orient0_exact(double ax, double ay, double bx, double by)
{
    double h[4];
    int n = exp_diff_prod(ax, by, ay, bx, h);
    return exp_sign(n, h);
}

__device__ __noinline__ int incircle0_exact(double ax, double ay, double bx, double by, double cx,
                                            double cy)
{
    double aa[4], bb[4], cc[4], bxc[4], axc[4], axb[4];
    int naa = exp_norm2(ax, ay, aa), nbb = exp_norm2(bx, by, bb), ncc = exp_norm2(cx, cy, cc);
    int nbxc = exp_diff_prod(bx, cy, by, cx, bxc);
    int naxc = exp_diff_prod(ax, cy, ay, cx, axc);
    int naxb = exp_diff_prod(ax, by, ay, bx, axb);
    double t1[32], t2[32], t3[32], s12[64], s[96], scr[96];
    int n1 = exp_mul4(naa, aa, nbxc, bxc, t1);
    int n2 = exp_mul4(nbb, bb, naxc, axc, t2);
    for (int i = 0; i < n2; ++i) t2[i] = -t2[i];
    int n3 = exp_mul4(ncc, cc, naxb, axb, t3);
    int n12 = exp_sum(n1, t1, n2, t2, s12, scr);
    int ns = exp_sum(n12, s12, n3, t3, s, scr);
    return exp_sign(ns, s);
}

// sign of a x b: +1 when b is counter-clockwise of a (as seen from the origin)
CG_D int orient0(double2 a, double2 b)
{
    double l = a.x * b.y, r = a.y * b.x;
    double det = l - r;
    double bound = 1.0e-15 * (fabs(l) + fabs(r));
    if (det > bound) return 1;
    if (-det > bound) return -1;
    return orient0_exact(a.x, a.y, b.x, b.y);
}

// sign of D(a,b,c) = |a|^2 (b x c) - |b|^2 (a x c) + |c|^2 (a x b). For (0,a,b) counter-clockwise,
// D < 0 iff c lies strictly inside the circle through 0, a and b.
CG_D int incircle0(double2 a, double2 b, double2 c)
{
    double aa = a.x * a.x + a.y * a.y, bb = b.x * b.x + b.y * b.y, cc = c.x * c.x + c.y * c.y;
    double bxc = b.x * c.y - b.y * c.x, axc = a.x * c.y - a.y * c.x, axb = a.x * b.y - a.y * b.x;
    double det = aa * bxc - bb * axc + cc * axb;
    double perm = aa * (fabs(b.x * c.y) + fabs(b.y * c.x)) + bb * (fabs(a.x * c.y) + fabs(a.y * c.x)) +
                  cc * (fabs(a.x * b.y) + fabs(a.y * b.x));
    double bound = 1.0e-14 * perm;
    if (det > bound) return 1;
    if (-det > bound) return -1;
    return incircle0_exact(a.x, a.y, b.x, b.y, c.x, c.y);
}

// ------------------------------------------------------------------------------------------
// The in-circle test of the triangulation, the same for every cell that asks it.
//
// Each cell evaluates predicates on positions relative to itself, formed by min_dist (one rounded
// difference and one rounded wrap: each coordinate is off the exact periodic difference by at most
// 1.5 u L, u = 2^-53, L = the larger box side). Exact arithmetic on those rounded inputs is exact
// for that cell only: when four cells are cocircular to within that rounding (relaxed fluid states
// drive Voronoi edges to zero length), two cells of the same quadrilateral can take opposite
// decisions and the rows stop matching. So:
//  * the floating-point filter decides only when its margin also covers the input rounding of this
//    cell's frame and of the canonical frame below; then its sign is the sign of the exact periodic
//    configuration, which every frame agrees on;
//  * otherwise the four points are re-expressed relative to the one with the smallest global index,
//    by min_dist from the absolute positions. Every cell computes the same doubles there, and the
//    exact determinant of those doubles decides;
//  * an exact zero (cocircular points) is resolved by simulation of simplicity (H. Edelsbrunner and
//    E. P. Mucke, ACM Trans. Graph. 9, 1990): the lifted coordinate |p|^2 of the point with the
//    smallest index is raised by an infinitesimal, so the sign is that of its cofactor, the
//    orientation of the other three points. The triangulation is then the unique Delaunay
//    triangulation of the perturbed set, whichever cell asks.
// incircle_g(c; a, b, t) keeps the sign convention of incircle0 in c's frame: negative iff t lies
// inside the circle through c, a and b (c, a, b counter-clockwise).
// ------------------------------------------------------------------------------------------

// sign of p x q + q x r + r x p (the orientation of p, q, r), exactly
__device__ __noinline__ int orient3_exact(double2 p, double2 q, double2 r)
{
    double e1[4], e2[4], e3[4], s12[8], s[12], scr[12];
    int n1 = exp_diff_prod(p.x, q.y, p.y, q.x, e1);
    int n2 = exp_diff_prod(q.x, r.y, q.y, r.x, e2);
    int n3 = exp_diff_prod(r.x, p.y, r.y, p.x, e3);
    int n12 = exp_sum(n1, e1, n2, e2, s12, scr);
    int ns = exp_sum(n12, s12, n3, e3, s, scr);
    return exp_sign(ns, s);
}

// canonical-frame exact evaluation with the simulation-of-simplicity tie break
__device__ __noinline__ int incircle_canonical(int ic, int ia, int ib, int it, const double2 *pos, double Lx,
                                               double Ly)
{
    const int id[4] = {ic, ia, ib, it};
    int j = 0;
    for (int k = 1; k < 4; ++k)
        if (id[k] < id[j]) j = k;
    const double2 pm = pos[id[j]];
    double2 q[3];
    int n = 0;
    for (int k = 0; k < 4; ++k)
        if (k != j) q[n++] = min_dist(pos[id[k]], pm, Lx, Ly);
    // D(c,a,b,t) as a 4x4 lifted determinant is alternating in its rows: moving the point of
    // position j to the front takes j transpositions
    const int par = (j & 1) ? -1 : 1;
    int s = incircle0_exact(q[0].x, q[0].y, q[1].x, q[1].y, q[2].x, q[2].y);
    if (s != 0) return par * s;
    return -par * orient3_exact(q[0], q[1], q[2]);
}

// filter with the input-rounding margin: +-1, or 0 when the canonical evaluation must decide.
// The derivative of D with respect to any coordinate is at most 4 M^3 (M = the largest |a|, |b|,
// |t|; the canonical frame's coordinates are at most 2M): six coordinates, both frames, each input
// off by at most 1.5 u L, doubled for safety -> 2 * (24 + 192) * 1.5 u L M^3 < 7.2e-14 L M^3, and
// M^3 <= M^2 (1 + M^2) / 2 avoids a square root.
// The arithmetic error of det is below 1e-14 times the sum of its terms' magnitudes, itself at
// most 6 M^4 (|b.x t.y| + |b.y t.x| <= 2 M^2 and so on).
CG_D int incircle_filter(double2 a, double2 b, double2 t, double Lmax)
{
    double aa = a.x * a.x + a.y * a.y, bb = b.x * b.x + b.y * b.y, tt = t.x * t.x + t.y * t.y;
    double bxt = b.x * t.y - b.y * t.x, axt = a.x * t.y - a.y * t.x, axb = a.x * b.y - a.y * b.x;
    double det = aa * bxt - bb * axt + tt * axb;
    double m2 = fmax(aa, fmax(bb, tt));
    double bound = m2 * (6.0e-14 * m2 + 3.6e-14 * Lmax * (1.0 + m2));
    if (det > bound) return 1;
    if (-det > bound) return -1;
    return 0;
}

CG_D int incircle_g(double2 a, double2 b, double2 t, int ic, int ia, int ib, int it, const double2 *pos,
                    double Lx, double Ly)
{
    int s = incircle_filter(a, b, t, fmax(Lx, Ly));
    return s ? s : incircle_canonical(ic, ia, ib, it, pos, Lx, Ly);
}

// ------------------------------------------------------------------------------------------
// Philox4x32-10 counter-based RNG (J. K. Salmon et al., "Parallel random numbers: as easy as
// 1, 2, 3", SC'11), and normal deviates by the Box-Muller transform. Counter = (cell, step,
// stream, 0), key = seed; a run can be resumed exactly from its step counter.
// ------------------------------------------------------------------------------------------
CG_D uint4 philox4x32_10(uint4 ctr, uint2 key)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(M0, ctr.x), lo0 = M0 * ctr.x;
        uint32_t hi1 = __umulhi(M1, ctr.z), lo1 = M1 * ctr.z;
        ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
        key.x += W0;
        key.y += W1;
    }
    return ctr;
}

// two standard normal deviates from one Philox block (53-bit uniforms, Box-Muller)
CG_D double2 normal2(uint64_t seed, uint32_t idx, uint32_t step, uint32_t stream)
{
    uint4 r = philox4x32_10(make_uint4(idx, step, stream, 0u),
                            make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    uint64_t a = ((uint64_t)r.x << 21) ^ (uint64_t)r.y;
    uint64_t b = ((uint64_t)r.z << 21) ^ (uint64_t)r.w;
    double u1 = ((double)(a & ((1ull << 53) - 1)) + 0.5) * (1.0 / 9007199254740992.0);
    double u2 = ((double)(b & ((1ull << 53) - 1)) + 0.5) * (1.0 / 9007199254740992.0);
    double rad = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    return make_double2(rad * c, rad * s);
}

// ------------------------------------------------------------------------------------------
// warp-aggregated append: one atomic per warp for all lanes with pred set
// ------------------------------------------------------------------------------------------
CG_D int warp_append(int *counter, bool pred)
{
    unsigned mask = __activemask();
    unsigned vote = __ballot_sync(mask, pred);
    if (!pred) return -1;
    int leader = __ffs(vote) - 1;
    int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(vote));
    base = __shfl_sync(vote, base, leader);
    return base + __popc(vote & ((1u << lane) - 1u));
}

}  // namespace cg
