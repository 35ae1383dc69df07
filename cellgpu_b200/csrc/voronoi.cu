// cellgpu_b200 -- Voronoi (SPV) model kernels for sm_100a.
//
// Design (B200-first, not a translation of the reference's kernels):
//  * One fused pass per cell computes the Voronoi polygon, A and P, and the force contributions
//    of that cell's energy to itself and to every neighbour (scatter form). A cell only needs its
//    own neighbour ring, so no per-slot voroCur / voroLastNext / forceSets / delSets / delOther
//    arrays are materialised in HBM (the reference writes and re-reads ~100 B per slot of those).
//  * The same pass runs the exact local-Delaunay test of the stored triangulation on the current
//    positions (every triangle counter-clockwise, every edge locally Delaunay). By Lawson's theorem
//    a valid triangulation whose edges are all locally Delaunay is the Delaunay triangulation, so
//    this test replaces the reference's cell-list circumcircle scan
//    (src/models/voronoiModelBase.cu:24-109) for the per-step check.
//  * Flagged cells and their neighbours (the reference's NeedsFixing set,
//    src/models/voronoiModelBase.cpp:632-646) get their Delaunay star recomputed exactly on the
//    device, one warp per cell; changed rows retract their old force contributions and add the new
//    ones, so forces always correspond to the repaired topology. Rounds continue until every
//    changed row is consistent with its partners; otherwise the step halts and the host runs the
//    device-side global triangulation (cell list + exact stars), the role of
//    globalTriangulationCGAL (src/models/voronoiModelBase.cpp:281-351).
#include "voronoi.cuh"

#include <cub/device/device_scan.cuh>

namespace cg {

// ------------------------------------------------------------------------------------------
// small vector helpers for FP64 / FP32 geometry
// ------------------------------------------------------------------------------------------
template <typename R>
struct Vec2;
template <>
struct Vec2<double> {
    using T = double2;
};
template <>
struct Vec2<float> {
    using T = float2;
};

template <typename R>
CG_D typename Vec2<R>::T mk(R x, R y)
{
    typename Vec2<R>::T v;
    v.x = x;
    v.y = y;
    return v;
}

template <typename R>
CG_D typename Vec2<R>::T cvt(double2 d)
{
    return mk<R>((R)d.x, (R)d.y);
}

// Circumcenter(x1,x2,xc) of (0, a, b) (inc/utility/functions.h:34-43)
template <typename R, typename V>
CG_D V circum0(V a, V b)
{
    R an = a.x * a.x + a.y * a.y;
    R bn = b.x * b.x + b.y * b.y;
    R den = R(0.5) / (a.x * b.y - a.y * b.x);
    return mk<R>(den * (an * b.y - a.y * bn), den * (a.x * bn - an * b.x));
}

// getdhdr (inc/utility/functions.h:234-287): d h / d r_0 for h = circumcentre(r_0, r_0+rij, r_0+rik),
// row = component of h, column = component of r_0.
template <typename R, typename V>
CG_D void dhdr(V rij, V rik, R &m11, R &m12, R &m21, R &m22)
{
    R cr = rij.y * rik.x - rij.x * rik.y;
    R den = R(0.5) / (cr * cr);
    R rik2 = rik.x * rik.x + rik.y * rik.y;
    R rij2 = rij.x * rij.x + rij.y * rij.y;
    R t1 = rik.y * rij2 - rij.y * rik2;
    R t2 = rik.x * rij2 - rij.x * rik2;
    m11 = den * (rik.y - rij.y) * t1;
    m12 = den * (rij.y - rik.y) * t2;
    m21 = den * (rij.x - rik.x) * t1;
    m22 = den * (rik.x - rij.x) * t2;
}

template <typename R>
CG_D void atomic_add2(void *F, int i, R x, R y);
template <>
CG_D void atomic_add2<double>(void *F, int i, double x, double y)
{
    double *f = reinterpret_cast<double *>(F) + 2 * (size_t)i;
    atomicAdd(f, x);
    atomicAdd(f + 1, y);
}
template <>
CG_D void atomic_add2<float>(void *F, int i, float x, float y)
{
    // forces are stored and summed in FP64 in every precision: the FP32 terms of the mixed mode
    // are added without FP32 rounding of the sum
    double *f = reinterpret_cast<double *>(F) + 2 * (size_t)i;
    atomicAdd(f, (double)x);
    atomicAdd(f + 1, (double)y);
}

// Order-independent sums (deterministic mode, VoroArgs::Ffix set). A value x is kept in FIXW = 3
// 64-bit integer words w[0..2] that hold x = w[0] 2^-20 + w[1] 2^-64 + w[2] 2^35 (w[0], w[2] signed,
// w[1] non-negative): |x| >= 2^35 first moves its nearest multiple of 2^35 to w[2] (the
// remainder, at most 2^34, is exact by Sterbenz's lemma), then hi = floor(x 2^20) goes to w[0] and
// lo = round((x 2^20 - hi) 2^44) to w[1]. Each part is added with a 64-bit integer atomic. Integer
// addition commutes exactly, so the sum does not depend on the order in which the parts arrive,
// and a retraction cancels its addition exactly. Resolution 2^-65 per value; any finite |x| < 2^98
// (the third word is touched only by |x| >= 2^35); a larger or non-finite x sets bit 62 of w[1]
// and the sum reads NaN.
constexpr int FIXW = 3;

CG_D void fix_add1(unsigned long long *w, double x)
{
    if (!(fabs(x) < 0x1p35)) {
        if (!(fabs(x) < 0x1p98)) {
            atomicOr(w + 1, 1ull << 62);
            return;
        }
        const double q = rint(x * 0x1p-35);
        atomicAdd(w + 2, (unsigned long long)(long long)q);
        x -= q * 0x1p35;
    }
    const double t = x * 0x1p20;
    const double h = floor(t);
    const long long hi = (long long)h;
    const long long lo = __double2ll_rn((t - h) * 0x1p44);
    if (hi) atomicAdd(w, (unsigned long long)hi);
    if (lo) atomicAdd(w + 1, (unsigned long long)lo);
}

CG_D double fix_value(unsigned long long hi, unsigned long long lo, unsigned long long top)
{
    if (lo >> 62) return __longlong_as_double(0x7ff8000000000000ll);
    return (double)(long long)top * 0x1p35 + ((double)(long long)hi + (double)lo * 0x1p-44) * 0x1p-20;
}

// Force components take FIXF = 4 words: w[0] counts 2^-56 and takes every |x| < 2 in one atomic
// (the common case; its resolution is FP64 rounding at 0.125), w[1..3] are the three-word form for
// the rest. w[0] cannot overflow: the integer sum equals the sum over the contributions of the
// cell's final rows (a retraction cancels its addition exactly), at most 33 terms below 2^57.
constexpr int FIXF = 4;

CG_D void fix_add_force(unsigned long long *w, double x)
{
    if (fabs(x) < 2.0) {
        const long long f = __double2ll_rn(x * 0x1p56);
        if (f) atomicAdd(w, (unsigned long long)f);
        return;
    }
    fix_add1(w + 1, x);
}

CG_D double fix_force_value(ulonglong2 a, ulonglong2 b)  // (w[0], w[1]), (w[2], w[3])
{
    return (double)(long long)a.x * 0x1p-56 + fix_value(a.y, b.x, b.y);
}

// add (x, y) to the force of cell i: F += (x, y), or to its fixed-point sums. FIX = -1 decides by
// Ffix at run time; the force pass is compiled for one mode (FIX = 0 atomics, 1 fixed point).
template <typename R, int FIX = -1>
CG_D void add_force(void *F, unsigned long long *Ffix, int i, R x, R y)
{
    if (FIX == 1 || (FIX == -1 && Ffix)) {
        unsigned long long *w = Ffix + 2 * FIXF * (size_t)i;
        fix_add_force(w, (double)x);
        fix_add_force(w + FIXF, (double)y);
    } else {
        atomic_add2<R>(F, i, x, y);
    }
}

template <typename R>
CG_D void store_ap(void *AP, int i, R A, R P)
{
    reinterpret_cast<typename Vec2<R>::T *>(AP)[i] = mk<R>(A, P);
}

CG_D const Inst &inst_of(const VoroArgs &a, int c)
{
    return a.inst ? a.inst[a.cell_inst ? a.cell_inst[c] : 0] : a.inst0;
}

// claim cell x for epoch e (first claimer wins) and append it to queue q; its slot is recorded in
// qslot[q & 1] (the round that reads it, q, and the round that writes the next claims, q + 1,
// use different halves)
CG_D void claim_enqueue(const VoroArgs &a, int x, int e, int q, int4 hint = make_int4(0, 0, 0, 0))
{
    if (q == 0 && a.nclaim) atomicAdd(&a.nclaim[x], 1);
    if (atomicMax(&a.mark[x], e) < e) {
        int slot = atomicAdd(&a.ctl->q_count[q], 1);
        a.queue[(size_t)q * a.N + slot] = x;
        if (a.qslot) a.qslot[(size_t)(q & 1) * a.N + x] = slot;
        if (q == 0 && a.qhint) a.qhint[slot] = hint;
    }
}

// The claims of an in-circle failure of edge (c, n), whose apexes are m (before n in c's row) and p
// (after it): the four cells, each with the edit of its row that flips the edge to (m, p) -- c and n
// drop each other, p gains m between c and n, m gains p between n and c (the hints of the first
// repair round's fast path, flip_edit)
CG_D void claim_flip(const VoroArgs &a, int e, int c, int n, int m, int p)
{
    claim_enqueue(a, c, e, 0, make_int4(1, n, 0, 0));
    claim_enqueue(a, n, e, 0, make_int4(1, c, 0, 0));
    claim_enqueue(a, p, e, 0, make_int4(2, m, c, n));
    claim_enqueue(a, m, e, 0, make_int4(2, p, n, c));
}

// ------------------------------------------------------------------------------------------
// The per-cell pass. Pass 1: Voronoi vertices h_k = circumcentre(0, r_{k-1}, r_k) relative to the
// cell (the CPU convention, src/models/voronoiModelBase.cpp:805-822), A = sum |h_k x h_{k+1}|/2,
// P = sum |h_k - h_{k+1}|, and (TEST) the exact local-Delaunay test. Pass 2 (SCATTER): with
// g_k = -dE_c/dh_k (E_c = KA (A-A0)^2 + KP (P-P0)^2; the derivatives of
// src/models/voronoiQuadraticEnergy.cpp:241-256 with the THRESHOLD clamp of :275-278), the force on
// cell x is the sum over the Voronoi vertices h of all cells of g . dh/dr_x; a vertex of c depends
// on c and the two neighbours that define it, with dh/dr_c = getdhdr(r_a, r_b),
// dh/dr_a = getdhdr(-r_a, r_b - r_a), dh/dr_b = I - dh/dr_c - dh/dr_a (translation invariance).
// sign = -1 retracts a stale row's contributions.
// Returns a test code: 0 ok, else (slot+1) of the first failing slot, negated for an orientation
// failure.
// ------------------------------------------------------------------------------------------
template <typename R, bool SCATTER, bool TEST>
CG_D int cell_pass(const VoroArgs &a, int c, const int *row, int z, double2 pc, double Lx, double Ly,
                   R sign, R &A_out, R &P_out)
{
    using V = typename Vec2<R>::T;
    const double2 *pos = a.pos;
    int fail = 0;
    if (z < 3) return -1;

    // ---- pass 1
    int nA = row[z - 1], nB = row[0];
    double2 dA = min_dist(pos[nA], pc, Lx, Ly);
    double2 dB = min_dist(pos[nB], pc, Lx, Ly);
    double2 hprev = circum0<double>(dA, dB);  // h_0 (vertex geometry and sums in FP64)
    double2 hfirst = hprev;
    double Asum = 0, Psum = 0;
    for (int k = 0; k < z; ++k) {
        int kn = (k + 1 == z) ? 0 : k + 1;
        int nC = row[kn];
        double2 dC = min_dist(pos[nC], pc, Lx, Ly);
        if (TEST && !fail) {
            if (orient0(dB, dC) <= 0) fail = -(k + 1);
            else if (c < nB && incircle_g(dA, dB, dC, c, nA, nB, nC, pos, Lx, Ly) < 0) fail = k + 1;
        }
        double2 hnext = (kn == 0) ? hfirst : circum0<double>(dB, dC);
        Asum += fabs(0.5 * (hprev.x * hnext.y - hprev.y * hnext.x));
        double dx = hprev.x - hnext.x, dy = hprev.y - hnext.y;
        Psum += sqrt(dx * dx + dy * dy);
        hprev = hnext;
        dA = dB;
        dB = dC;
        nA = nB;
        nB = nC;
    }
    A_out = (R)Asum;
    P_out = (R)Psum;

    if (SCATTER) {
        const R thr = R(1e-18);
        R Adiff = (R)(a.KA * (Asum - a.APpref[c].x));
        R Pdiff = (R)(a.KP * (Psum - a.APpref[c].y));
        // window: r_{k-1} = rA, r_k = rB, r_{k+1} = rC ; h_{k-1} = hP, h_k = hC, h_{k+1} = hN
        double2 rZ = min_dist(pos[row[z - 2]], pc, Lx, Ly);
        double2 rA = min_dist(pos[row[z - 1]], pc, Lx, Ly);
        double2 rB = min_dist(pos[row[0]], pc, Lx, Ly);
        double2 rC = min_dist(pos[row[1]], pc, Lx, Ly);
        V hP = cvt<R>(circum0<double>(rZ, rA));
        V hC = cvt<R>(circum0<double>(rA, rB));
        V hN = cvt<R>(circum0<double>(rB, rC));
        R sx = 0, sy = 0;          // self
        R pendx = 0, pendy = 0;    // slot k (b part), waiting for the a part of vertex k+1
        R fax = 0, fay = 0;        // a part of vertex 0, belongs to slot z-1
        for (int k = 0; k < z; ++k) {
            // g = -dE/dh_k
            R dAx = R(0.5) * (hN.y - hP.y), dAy = R(0.5) * (hP.x - hN.x);
            R dPx, dPy;
            if (sizeof(R) == sizeof(double)) {
                R lx = hC.x - hP.x, ly = hC.y - hP.y;
                R ln = sqrt(lx * lx + ly * ly);
                if (ln < thr) ln = thr;
                R nx = hC.x - hN.x, ny = hC.y - hN.y;
                R nnm = sqrt(nx * nx + ny * ny);
                if (nnm < thr) nnm = thr;
                dPx = lx / ln + nx / nnm;
                dPy = ly / ln + ny / nnm;
            } else {
                // exact tangent directions of the edges dual to r_{k-1} and r_k (see k_voro_groups)
                V fa = cvt<R>(rA), fb = cvt<R>(rB);
                R ia = R(1) / sqrt(fa.x * fa.x + fa.y * fa.y), ib = R(1) / sqrt(fb.x * fb.x + fb.y * fb.y);
                dPx = -fa.y * ia + fb.y * ib;
                dPy = fa.x * ia - fb.x * ib;
            }
            R gx = -R(2) * (Adiff * dAx + Pdiff * dPx);
            R gy = -R(2) * (Adiff * dAy + Pdiff * dPy);
            // Jacobians of h_k (FP64, see k_voro_groups)
            double d11, d12, d21, d22, e11, e12, e21, e22;
            dhdr<double>(rA, rB, d11, d12, d21, d22);
            dhdr<double>(make_double2(-rA.x, -rA.y), make_double2(rB.x - rA.x, rB.y - rA.y), e11, e12, e21, e22);
            R c11 = (R)d11, c12 = (R)d12, c21 = (R)d21, c22 = (R)d22;
            R a11 = (R)e11, a12 = (R)e12, a21 = (R)e21, a22 = (R)e22;
            R b11 = (R)(1.0 - d11 - e11), b12 = (R)(-d12 - e12), b21 = (R)(-d21 - e21), b22 = (R)(1.0 - d22 - e22);
            sx += gx * c11 + gy * c21;
            sy += gx * c12 + gy * c22;
            R cax = gx * a11 + gy * a21, cay = gx * a12 + gy * a22;
            R cbx = gx * b11 + gy * b21, cby = gx * b12 + gy * b22;
            if (k == 0) {
                fax = cax;
                fay = cay;
            } else {
                add_force<R>(a.F, a.Ffix, row[k - 1], sign * (pendx + cax), sign * (pendy + cay));
            }
            pendx = cbx;
            pendy = cby;
            // advance the window
            if (k + 1 < z) {
                int k2 = k + 2;
                if (k2 >= z) k2 -= z;
                hP = hC;
                hC = hN;
                rA = rB;
                rB = rC;
                rC = min_dist(pos[row[k2]], pc, Lx, Ly);
                hN = cvt<R>(circum0<double>(rB, rC));
            }
        }
        add_force<R>(a.F, a.Ffix, row[z - 1], sign * (pendx + fax), sign * (pendy + fay));
        add_force<R>(a.F, a.Ffix, c, sign * sx, sign * sy);
    }
    return fail;
}

// ------------------------------------------------------------------------------------------
// fused geometry + forces (+ exact test, + repair queue seeding)
// ------------------------------------------------------------------------------------------
template <typename R, bool SCATTER, bool TEST>
__global__ void __launch_bounds__(128) k_voro_cells(VoroArgs a)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.N) return;
    if (a.ctl && a.ctl->halt) return;
    const Inst &in = inst_of(a, c);
    double2 pc = a.pos[c];
    int z = a.nn[c];
    const int *row = a.nbr + (size_t)c * a.K;
    R A, P;
    int fail = cell_pass<R, SCATTER, TEST>(a, c, row, z, pc, in.Lx, in.Ly, R(1), A, P);
    if (a.AP) store_ap<R>(a.AP, c, A, P);
    if (TEST && fail && z < 3) {
        // degenerate row: only the cell itself can be queued
        if (a.ctl) {
            atomicAdd(&a.ctl->n_flagged, 1);
            claim_enqueue(a, c, a.ctl->epoch, 0);
        } else if (a.mark) {
            a.mark[c] = 1;
            a.queue[0] = 1;
        }
    } else if (TEST && fail) {
        if (a.ctl) {
            int e = a.ctl->epoch;
            atomicAdd(&a.ctl->n_flagged, 1);
            int k = (fail > 0 ? fail : -fail) - 1;
            // the cell, the edge's other end and the two apexes (or the triangle's corners)
            claim_enqueue(a, c, e, 0);
            claim_enqueue(a, row[k], e, 0);
            claim_enqueue(a, row[(k + 1) % z], e, 0);
            if (fail > 0) claim_enqueue(a, row[(k + z - 1) % z], e, 0);
        } else if (a.mark) {
            // raw test API: mark = flag array, queue[0] = any_fail word
            int k = (fail > 0 ? fail : -fail) - 1;
            a.mark[c] = 1;
            a.mark[row[k]] = 1;
            a.mark[row[(k + 1) % z]] = 1;
            if (fail > 0) a.mark[row[(k + z - 1) % z]] = 1;
            a.queue[0] = 1;
        }
    }
}

// ------------------------------------------------------------------------------------------
// Lane-per-Voronoi-vertex form of the same pass (the step's workhorse). A group of G = 8 lanes owns
// one cell; lane l handles vertices l and l+8 (rows up to 16). Ring neighbours (k-1, k+1) are
// exchanged through shared memory, A and P are reduced with group shuffles, and each vertex's
// three force contributions are formed once (no recomputation, no local arrays). One reciprocal of
// the cross product r_{k-1} x r_k serves the circumcentre and both Jacobians.
// In FP64 the perimeter derivative uses the unit vectors of h_{k+1}-h_k as the reference does
// (src/models/voronoiQuadraticEnergy.cpp:247-256). In mixed precision it uses their exact
// direction: both ends of the Voronoi edge dual to (c, n_k) lie on the perpendicular bisector of
// r_k, so the counter-clockwise unit tangent is (-r_k.y, r_k.x)/|r_k|; this removes the
// cancellation of nearly equal FP32 circumcentres on short edges.
// ------------------------------------------------------------------------------------------
constexpr int G = 8;
constexpr int GPW = 32 / G;  // cells per warp
constexpr int VG = 16;       // vertices per cell in the group kernels' fast form (K <= 16)
constexpr int VG_MAX = 32;   // their wide form, for systems whose rows grew to K = 32

template <typename R>
CG_D R group_sum(R v)
{
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    return v;
}

CG_D int group_min(int v)
{
    v = min(v, __shfl_xor_sync(0xffffffffu, v, 1));
    v = min(v, __shfl_xor_sync(0xffffffffu, v, 2));
    v = min(v, __shfl_xor_sync(0xffffffffu, v, 4));
    return v;
}

CG_D bool group_any(bool v)
{
    int x = v ? 1 : 0;
    x |= __shfl_xor_sync(0xffffffffu, x, 1);
    x |= __shfl_xor_sync(0xffffffffu, x, 2);
    x |= __shfl_xor_sync(0xffffffffu, x, 4);
    return x != 0;
}

// Shared-memory tile of one group's cell: relative neighbour positions r_k, Voronoi vertices h_k,
// the reciprocal 1 / (2 r_{k-1} x r_k) (shared by h_k and its Jacobians), unit tangents of the
// edges h_k -> h_{k+1}, and the dh_k/dr_{k-1} contraction consumed by the neighbouring lane.
template <typename R, int NS = VG>
struct GrpTile {
    double2 r[NS];
    double2 h[NS];
    double den[NS];
    typename Vec2<R>::T u[NS];
    typename Vec2<R>::T ca[NS];
    double w[NS];  // line-tension weight of the edge h_k -> h_{k+1} (dual to neighbour k)
};

// Phases A-C of one group's cell (called by the whole warp; `ok` switches a group off): relative
// neighbour positions (FP64, the exact Delaunay inputs), Voronoi vertices, A, P, the exact local
// test (TEST) and the edge unit vectors (SCATTER). nbk receives the neighbours of the lane's slots.
// pre0: row[gl] when the caller has already loaded it (padded rows, loaded beside the row length so
// that the neighbour gather waits for one load instead of two), else NO_PRE.
constexpr int NO_PRE = -2;

template <typename R, bool SCATTER, bool TEST, int NS = VG>
CG_D void grp_geometry(const VoroArgs &a, int c, const int *row, int z, bool ok, double2 pc, double Lx,
                       double Ly, int gl, GrpTile<R, NS> &T, int (&nbk)[NS / G], double &A, double &P, int &fail,
                       bool store_te = true, int pre0 = NO_PRE)
{
    using V = typename Vec2<R>::T;
#pragma unroll
    for (int r = 0; r < NS / G; ++r) {
        int k = gl + G * r;
        nbk[r] = -1;
        if (ok && k < z) {
            nbk[r] = (r == 0 && pre0 != NO_PRE) ? pre0 : row[k];
            T.r[k] = min_dist(a.pos[nbk[r]], pc, Lx, Ly);
        }
    }
    __syncwarp();
    // phase B: Voronoi vertices h_k = circumcentre(0, r_{k-1}, r_k) (inc/utility/functions.h:34-43);
    // exact local Delaunay test
    fail = 0x7fffffff;  // smallest failing slot (x2, +1 for orientation)
    int undecided = 0;  // slots whose in-circle sign the filter left to the canonical evaluation
#pragma unroll
    for (int r = 0; r < NS / G; ++r) {
        int k = gl + G * r;
        if (ok && k < z) {
            int km = k == 0 ? z - 1 : k - 1;
            double2 ra = T.r[km], rb = T.r[k];
            // Voronoi vertices are ill-conditioned (skinny triangles): always formed in FP64
            double an = ra.x * ra.x + ra.y * ra.y, bn = rb.x * rb.x + rb.y * rb.y;
            double den = 0.5 / (ra.x * rb.y - ra.y * rb.x);
            if (SCATTER) T.den[k] = den;
            T.h[k] = make_double2(den * (an * rb.y - ra.y * bn), den * (ra.x * bn - an * rb.x));
            if (TEST) {
                double2 rc = T.r[k + 1 == z ? 0 : k + 1];
                if (orient0(rb, rc) <= 0) {
                    fail = min(fail, 2 * k + 1);
                } else if (c < nbk[r]) {
                    int ic = incircle_filter(ra, rb, rc, fmax(Lx, Ly));
                    if (ic < 0) fail = min(fail, 2 * k);
                    if (ic == 0) undecided |= 1 << r;
                }
            }
        }
    }
    if (TEST && undecided) {
        // rare: the canonical evaluation runs in k_repair_begin (keeping this kernel's registers for
        // the common path); without a list, or when it is full, the edge counts as failing and the
        // repair recomputes the stars with the canonical predicate
        for (int r = 0; r < NS / G; ++r) {
            if (!(undecided & (1 << r))) continue;
            int k = gl + G * r;
            int idx = (a.undec && a.ctl) ? atomicAdd(&a.ctl->n_undec, 1) : a.N;
            if (idx < a.N) a.undec[idx] = c * KMAX + k;  // one encoding for every row width
            else fail = min(fail, 2 * k);
        }
    }
    __syncwarp();
    // phase C: edges h_k -> h_{k+1}: area, perimeter (FP64 sums in both modes: A - A0 and P - P0
    // are small differences), unit tangents
    double Ap = 0, Pp = 0;
#pragma unroll
    for (int r = 0; r < NS / G; ++r) {
        int k = gl + G * r;
        if (ok && k < z) {
            double2 h0 = T.h[k], h1 = T.h[k + 1 == z ? 0 : k + 1];
            double dx = h1.x - h0.x, dy = h1.y - h0.y;
            // one reciprocal square root gives the length and the unit vector; edges shorter than
            // the 1e-18 THRESHOLD take the clamped reciprocal as the reference does
            double l2 = dx * dx + dy * dy, len, il;
            if (l2 > 1e-36) {
                il = rsqrt(l2);
                len = l2 * il;
            } else {
                len = sqrt(l2);
                il = 1e18;
            }
            Ap += fabs(0.5 * (h0.x * h1.y - h0.y * h1.x));
            Pp += len;
            if (SCATTER) {
                V u;
                if (sizeof(R) == sizeof(double)) {
                    u = mk<R>((R)(dx * il), (R)(dy * il));
                } else {
                    V rk = cvt<R>(T.r[k]);
                    R ir = rsqrtf((float)(rk.x * rk.x + rk.y * rk.y));
                    u = mk<R>(-rk.y * ir, rk.x * ir);
                }
                T.u[k] = u;
            }
        }
    }
    A = group_sum<double>(Ap);
    P = group_sum<double>(Pp);
    if (TEST) fail = group_min(fail);
    if (a.tension_mode) {  // uniform across the grid
        // line tension: weight of every edge of the cell, and the cell's tension term sum w_k l_k
        double Tp = 0.0;
        const int tc = ok ? a.ctype[c] : 0;
#pragma unroll
        for (int r = 0; r < NS / G; ++r) {
            int k = gl + G * r;
            if (ok && k < z) {
                double w = tension_weight(a, tc, a.ctype[nbk[r]]);
                T.w[k] = w;
                double2 h0 = T.h[k], h1 = T.h[k + 1 == z ? 0 : k + 1];
                double dx = h1.x - h0.x, dy = h1.y - h0.y;
                Tp += w * sqrt(dx * dx + dy * dy);
            }
        }
        Tp = group_sum<double>(Tp);
        if (ok && store_te && gl == 0 && a.TE) a.TE[c] = Tp;
    }
}

// Phases D-E (called by the whole warp): g_k = -dE_c/dh_k, the three Jacobian contractions of every
// vertex, and the scatter of SIGN x (contribution) to the cell and its neighbours.
template <typename R, int SIGN, int NS = VG, int FIX = -1>
CG_D void grp_scatter(const VoroArgs &a, int c, int z, bool ok, int gl, GrpTile<R, NS> &T, const int (&nbk)[NS / G],
                      double A, double P, R sgn = R(SIGN), bool have_pref = false,
                      double2 pref = double2())
{
    using V = typename Vec2<R>::T;
    __syncwarp();
    R Adiff = 0, Pdiff = 0;
    if (ok) {
        const double2 pp = have_pref ? pref : a.APpref[c];  // (A0, P0): the force pass loads it early
        Adiff = (R)(a.KA * (A - pp.x));
        Pdiff = (R)(a.KP * (P - pp.y));
    }
    // the cell's own force and the pairs of contributions to each neighbour are summed in FP64 in
    // both precisions (mixed mode: FP32 terms, no FP32 rounding of their sums)
    using S = double;
    S sx = 0, sy = 0;
    V cb[NS / G];
#pragma unroll
    for (int r = 0; r < NS / G; ++r) {
        int k = gl + G * r;
        if (ok && k < z) {
            int km = k == 0 ? z - 1 : k - 1, kp = k + 1 == z ? 0 : k + 1;
            V hm = cvt<R>(T.h[km]), hp = cvt<R>(T.h[kp]);
            V um = T.u[km], uk = T.u[k];
            R dAx = R(0.5) * (hp.y - hm.y), dAy = R(0.5) * (hm.x - hp.x);
            R dPx = um.x - uk.x, dPy = um.y - uk.y;
            R gx = -R(2) * (Adiff * dAx + Pdiff * dPx);
            R gy = -R(2) * (Adiff * dAy + Pdiff * dPy);
            if (a.tension_mode) {
                // line tension of the cell's edges at h_k (VoronoiQuadraticEnergyWithTension:
                // each cell's force terms count its unlike edges, src/models/voronoiQuadraticEnergyWithTension.cpp:351-361)
                R wm = (R)T.w[km], wk = (R)T.w[k];
                gx -= wm * um.x - wk * uk.x;
                gy -= wm * um.y - wk * uk.y;
            }
            // Jacobians of h_k (getdhdr, inc/utility/functions.h:234-287; always FP64: their entries
            // scale as 1/|ra x rb|^2). dh/dr_c = getdhdr(ra, rb) and dh/dr_a = getdhdr(-ra, rb-ra)
            // share the denominator 2 (ra x rb)^2 = 1 / (2 den^2).
            double2 ra = T.r[km], rb = T.r[k];
            double den = T.den[k];
            double half_inv = 2.0 * den * den;
            double ra2 = ra.x * ra.x + ra.y * ra.y, rb2 = rb.x * rb.x + rb.y * rb.y;
            double t1 = rb.y * ra2 - ra.y * rb2, t2 = rb.x * ra2 - ra.x * rb2;
            double d11 = half_inv * (rb.y - ra.y) * t1, d12 = half_inv * (ra.y - rb.y) * t2;
            double d21 = half_inv * (ra.x - rb.x) * t1, d22 = half_inv * (rb.x - ra.x) * t2;
            double2 p = make_double2(-ra.x, -ra.y), q = make_double2(rb.x - ra.x, rb.y - ra.y);
            double q2 = q.x * q.x + q.y * q.y;
            double u1 = q.y * ra2 - p.y * q2, u2 = q.x * ra2 - p.x * q2;
            double e11 = half_inv * (q.y - p.y) * u1, e12 = half_inv * (p.y - q.y) * u2;
            double e21 = half_inv * (p.x - q.x) * u1, e22 = half_inv * (q.x - p.x) * u2;
            R c11 = (R)d11, c12 = (R)d12, c21 = (R)d21, c22 = (R)d22;
            R a11 = (R)e11, a12 = (R)e12, a21 = (R)e21, a22 = (R)e22;
            R b11 = (R)(1.0 - d11 - e11), b12 = (R)(-d12 - e12), b21 = (R)(-d21 - e21),
              b22 = (R)(1.0 - d22 - e22);
            if (sizeof(R) == sizeof(double)) {
                sx += gx * c11 + gy * c21;
                sy += gx * c12 + gy * c22;
            } else {
                sx += (S)(gx * c11) + (S)(gy * c21);
                sy += (S)(gx * c12) + (S)(gy * c22);
            }
            T.ca[k] = mk<R>(gx * a11 + gy * a21, gx * a12 + gy * a22);
            cb[r] = mk<R>(gx * b11 + gy * b21, gx * b12 + gy * b22);
        }
    }
    sx = group_sum<S>(sx);
    sy = group_sum<S>(sy);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < NS / G; ++r) {
        int k = gl + G * r;
        if (ok && k < z) {
            V ca = T.ca[k + 1 == z ? 0 : k + 1];
            if (sizeof(R) == sizeof(double))
                add_force<R, FIX>(a.F, a.Ffix, nbk[r], sgn * (cb[r].x + ca.x), sgn * (cb[r].y + ca.y));
            else
                add_force<S, FIX>(a.F, a.Ffix, nbk[r], (S)sgn * ((S)cb[r].x + (S)ca.x),
                                  (S)sgn * ((S)cb[r].y + (S)ca.y));
        }
    }
    if (ok && gl == 0) {
        add_force<S, FIX>(a.F, a.Ffix, c, (S)sgn * sx, (S)sgn * sy);
    }
}

// Cells whose row failed the exact test (fail: the smallest failing slot x 2, +1 for an
// orientation failure), or whose row is unusable (!ok: fewer than 3 or more than NS entries), are
// counted and queued for the repair with the cells of the failing edge (one thread per cell).
CG_D void flag_cell(const VoroArgs &a, int c, int z, bool ok, int fail, int ns)
{
    if (!ok) {
        if (a.ctl) {
            atomicAdd(&a.ctl->n_flagged, 1);
            claim_enqueue(a, c, a.ctl->epoch, 0);
            if (z > ns) {
                atomicExch(&a.ctl->status, CG_ERR_CAPACITY);
                atomicExch(&a.ctl->halt, 1);
            }
        } else if (a.mark) {
            a.mark[c] = 1;
            a.queue[0] = 1;
        }
    } else {
        int k = fail >> 1;
        bool orient_fail = fail & 1;
        const int *rw = a.nbr + (size_t)c * a.K;
        int nk = rw[k], nk1 = rw[k + 1 == z ? 0 : k + 1], nkm = rw[k == 0 ? z - 1 : k - 1];
        if (a.ctl) {
            int e = a.ctl->epoch;
            atomicAdd(&a.ctl->n_flagged, 1);
            if (orient_fail) {
                claim_enqueue(a, c, e, 0);
                claim_enqueue(a, nk, e, 0);
                claim_enqueue(a, nk1, e, 0);
            } else {
                claim_flip(a, e, c, nk, nkm, nk1);
            }
        } else if (a.mark) {
            a.mark[c] = 1;
            a.mark[nk] = 1;
            a.mark[nk1] = 1;
            if (!orient_fail) a.mark[nkm] = 1;
            a.queue[0] = 1;
        }
    }
}

// One cell per 8-lane group of the fused pass (called by the whole warp; live switches a group off)
template <typename R, bool SCATTER, bool TEST, int NS, int FIX>
CG_D void grp_cell(const VoroArgs &a, int c, bool live, int gl, GrpTile<R, NS> &tl)
{
    int z = 0, pre0 = NO_PRE;
    double2 pc = make_double2(0, 0), pref = make_double2(0, 0);
    double Lx = 1, Ly = 1;
    const int *row = nullptr;
    if (live) {
        // independent loads, issued together: position, row length, first row entry (rows of
        // the system are padded, so it needs no length), preferences
        row = a.nbr + (size_t)c * a.K;
        pc = a.pos[c];
        z = a.nn[c];
        if (CG_FP_PRE_ROW && a.rows_padded && gl < a.K) pre0 = row[gl];
        if (SCATTER && CG_FP_PRE_PREF) pref = a.APpref[c];
        const Inst &in = inst_of(a, c);
        Lx = in.Lx;
        Ly = in.Ly;
    }
    const bool ok = live && z >= 3 && z <= NS;
    // Rows of at most G entries (nearly every cell of a tissue): when all four cells of the warp
    // have them, the pass runs in its one-slot-per-lane form on the narrow tile (fewer live
    // registers, no second-slot code)
    const bool small = CG_FP_SMALL_PATH && NS > G && __all_sync(0xffffffffu, !live || z <= G);
    GrpTile<R, G> &tile8 = *reinterpret_cast<GrpTile<R, G> *>(&tl);
    int nbk[NS / G], nb8[1];
    double A, P;
    int fail;
    if (small)
        grp_geometry<R, SCATTER, TEST, G>(a, c, row, z, ok, pc, Lx, Ly, gl, tile8, nb8, A, P, fail, true, pre0);
    else
        grp_geometry<R, SCATTER, TEST, NS>(a, c, row, z, ok, pc, Lx, Ly, gl, tl, nbk, A, P, fail, true, pre0);
    if (ok && gl == 0 && a.AP) store_ap<R>(a.AP, c, (R)A, (R)P);
    // A cell whose own row fails the test holds its contributions back: the row is about to be
    // replaced, and a stale row can contain a nearly collinear triangle whose Jacobians (1/cross^2)
    // would swamp the forces. The repair commit adds the contributions of the new row.
    bool hold = SCATTER && TEST && a.held && ok && fail != 0x7fffffff;
    if (hold && gl == 0) a.held[c] = 1;
    if (SCATTER) {
        if (small)
            grp_scatter<R, 1, G, FIX>(a, c, z, ok && !hold, gl, tile8, nb8, A, P, R(1), CG_FP_PRE_PREF != 0, pref);
        else
            grp_scatter<R, 1, NS, FIX>(a, c, z, ok && !hold, gl, tl, nbk, A, P, R(1), CG_FP_PRE_PREF != 0, pref);
    }
    if (TEST && live && gl == 0 && (fail != 0x7fffffff || !ok)) flag_cell(a, c, z, ok, fail, NS);
    __syncwarp();
}

// A block takes a contiguous run of cpb cells (a multiple of its WPB * GPW groups), so that in a
// spatially sorted system the cells one SM works on are neighbours and their positions stay in L1.
template <typename R, bool SCATTER, bool TEST, int WPB, int MINB, int NS = VG, int FIX = 0>
__global__ void __launch_bounds__(WPB * 32, MINB) k_voro_groups(VoroArgs a, int cpb)
{
    __shared__ GrpTile<R, NS> tile[WPB * GPW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int gl = lane & (G - 1), gi = lane >> 3;
    const int sl = w * GPW + gi;
    const int c_end = min(a.N, (blockIdx.x + 1) * cpb);
    const bool halted = a.ctl && a.ctl->halt;  // uniform across the grid
    for (int base = blockIdx.x * cpb + w * GPW; base < c_end; base += WPB * GPW) {  // warp-uniform
        const int c = base + gi;
        grp_cell<R, SCATTER, TEST, NS, FIX>(a, c, c < c_end && !halted, gl, tile[sl]);
    }
}

// ------------------------------------------------------------------------------------------
// Thread-per-cell form of the fused pass (FP64, atomic force sums, no line tension, 16-slot padded
// rows). One thread walks its cell's ring: the row's first eight entries come in two 16-byte loads,
// the eight neighbour positions are gathered together, and the vertices, the exact test, A, P and
// the scatter run over the ring in the thread, with no shuffles.
// The group form spends most of its issue slots on exchanging ring neighbours between lanes
// (shared-memory tiles, shuffles); here a cell's ring never leaves its thread. The relative
// positions, vertices and reciprocals go to a shared-memory column of the thread's own (no
// exchange, no barrier) for the scatter pass, which forms the tangents u_k again (one reciprocal
// square root per vertex) instead of holding them for all eight vertices.
// Rows of 9-16 entries (about 1 % of the cells of a tissue) are run by the same warp afterwards, in
// the group form (four cells at a time, 8 lanes each).
// ------------------------------------------------------------------------------------------
constexpr int TC_Z = 8;  // rows of at most this many entries run in the thread form

// unit vector of the edge h0 -> h1 and its length, without a branch: the reciprocal square root
// of max(l2, 1e-36), so an edge shorter than 1e-18 (a degenerate Voronoi edge) gets the
// unit-vector scale 1e18 and a length of l2 * 1e18 (at most 1e-18)
CG_D double2 edge_unit(double2 h0, double2 h1, double &len)
{
    const double dx = h1.x - h0.x, dy = h1.y - h0.y;
    const double l2 = dx * dx + dy * dy;
    const double il = rsqrt(fmax(l2, 1e-36));
    len = l2 * il;
    return make_double2(dx * il, dy * il);
}

CG_D double2 vertex_h(double2 ra, double2 rb, double &den)
{
    const double an = ra.x * ra.x + ra.y * ra.y, bn = rb.x * rb.x + rb.y * rb.y;
    // 0.5 / x as the correctly rounded reciprocal halved: the same double (halving is exact), with a
    // shorter dependent chain than the division
    den = 0.5 * __drcp_rn(ra.x * rb.y - ra.y * rb.x);
    return make_double2(den * (an * rb.y - ra.y * bn), den * (ra.x * bn - an * rb.x));
}

// Per warp: the relative neighbour positions r_k, vertices h_k and reciprocals den_k of the lanes'
// cells ([slot][lane]: each lane reads and writes its own column, so no barrier), formed once in the
// geometry pass and read back by the scatter. Holding them here rather than in registers keeps the
// pass at 92 registers without spills (10 blocks of 2 warps per SM, as the 20 KB per block allows).
struct ThreadTile {
    double hx[TC_Z][WARP], hy[TC_Z][WARP], den[TC_Z][WARP], rx[TC_Z][WARP], ry[TC_Z][WARP];
};

// Returns true when the row is 9-16 entries long (the caller runs it in the group form).
template <bool TEST>
CG_D bool thread_cell(const VoroArgs &a, int c, ThreadTile &T, int lane)
{
    const int4 *r4 = reinterpret_cast<const int4 *>(a.nbr + (size_t)c * VG);
    const int4 q0 = r4[0], q1 = r4[1];
    const double2 pc = a.pos[c];
    const int z = a.nn[c];
    const double2 pref = a.APpref[c];
    const Inst &in = inst_of(a, c);
    const double Lx = in.Lx, Ly = in.Ly;
    if (z > TC_Z && z <= VG) return true;
    if (z < 3 || z > VG) {
        if (TEST) flag_cell(a, c, z, false, 0, VG);
        return false;
    }
    const int nb[TC_Z] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
    for (int k = 0; k < TC_Z; ++k) {
        if (k < z) {
            const double2 rk = min_dist_sel(a.pos[nb[k]], pc, Lx, Ly);
            T.rx[k][lane] = rk.x;
            T.ry[k][lane] = rk.y;
        }
    }
    auto R = [&](int k) { return make_double2(T.rx[k][lane], T.ry[k][lane]); };
    const double2 rl = R(z - 1);
    // vertices h_k = circumcentre(0, r_{k-1}, r_k), the exact local test, A and P
    const double Lmax = fmax(Lx, Ly);
    int fail = 0x7fffffff, undecided = 0;
    double Asum = 0.0, Psum = 0.0, len;
    double2 h0 = make_double2(0.0, 0.0), hprev = h0;
#pragma unroll
    for (int k = 0; k < TC_Z; ++k) {
        if (k < z) {
            const double2 ra = k == 0 ? rl : R(k == 0 ? 0 : k - 1), rb = R(k);
            const double2 rc = R(k + 1 < z ? k + 1 : 0);
            double den;
            const double2 h = vertex_h(ra, rb, den);
            T.hx[k][lane] = h.x;
            T.hy[k][lane] = h.y;
            T.den[k][lane] = den;
            if (TEST) {
                if (orient0(rb, rc) <= 0) {
                    fail = min(fail, 2 * k + 1);
                } else if (c < nb[k]) {
                    const int ic = incircle_filter(ra, rb, rc, Lmax);
                    if (ic < 0) fail = min(fail, 2 * k);
                    if (ic == 0) undecided |= 1 << k;
                }
            }
            if (k == 0) {
                h0 = h;
            } else {
                edge_unit(hprev, h, len);
                Asum += fabs(0.5 * (hprev.x * h.y - hprev.y * h.x));
                Psum += len;
            }
            hprev = h;
        }
    }
    const double2 hlast = hprev;
    const double2 ulast = edge_unit(hlast, h0, len);  // edge h_{z-1} -> h_0
    Asum += fabs(0.5 * (hlast.x * h0.y - hlast.y * h0.x));
    Psum += len;
    if (TEST && undecided) {
        // the canonical evaluation of these slots runs in the repair's first phase
        for (int k = 0; k < TC_Z; ++k) {
            if (!(undecided & (1 << k))) continue;
            int idx = (a.undec && a.ctl) ? atomicAdd(&a.ctl->n_undec, 1) : a.N;
            if (idx < a.N) a.undec[idx] = c * KMAX + k;
            else fail = min(fail, 2 * k);
        }
    }
    if (a.AP) store_ap<double>(a.AP, c, Asum, Psum);
    const bool hold = TEST && a.held && fail != 0x7fffffff;
    if (hold) a.held[c] = 1;
    if (!hold) {
        // g_k = -dE_c/dh_k and the three Jacobian contractions of every vertex, as in grp_scatter
        const double Adiff = a.KA * (Asum - pref.x), Pdiff = a.KP * (Psum - pref.y);
        double2 hm = hlast, hc = h0, um = ulast;
        double dc = T.den[0][lane];
        double sx = 0.0, sy = 0.0;
        double2 ca0 = make_double2(0.0, 0.0), cbp = ca0;
        int nprev = nb[0];
#pragma unroll
        for (int k = 0; k < TC_Z; ++k) {
            if (k < z) {
                double2 hn = h0;
                double dn = 0.0;
                if (k + 1 < TC_Z && k + 1 < z) {
                    hn = make_double2(T.hx[(k + 1) % TC_Z][lane], T.hy[(k + 1) % TC_Z][lane]);
                    dn = T.den[(k + 1) % TC_Z][lane];
                }
                const double2 uk = edge_unit(hc, hn, len);
                const double dAx = 0.5 * (hn.y - hm.y), dAy = 0.5 * (hm.x - hn.x);
                const double dPx = um.x - uk.x, dPy = um.y - uk.y;
                const double gx = -2.0 * (Adiff * dAx + Pdiff * dPx);
                const double gy = -2.0 * (Adiff * dAy + Pdiff * dPy);
                const double2 ra = k == 0 ? rl : R(k == 0 ? 0 : k - 1), rb = R(k);
                // the contractions of g with the three Jacobians of h = circumcentre(0, ra, rb) (getdhdr,
                // inc/utility/functions.h:234-287), written through h itself: with den = 1 / (2 ra x rb),
                // g.dh/dr_c = 2 den (g x (rb - ra)) h, g.dh/dr_a = -2 den (g x rb) (h - ra), and
                // g.dh/dr_b = g - both (translation invariance); g x v = gx v.y - gy v.x
                const double fc = 2.0 * dc * (gx * (rb.y - ra.y) - gy * (rb.x - ra.x));
                const double fa = -2.0 * dc * (gx * rb.y - gy * rb.x);
                const double scx = fc * hc.x, scy = fc * hc.y;
                sx += scx;
                sy += scy;
                const double2 ca = make_double2(fa * (hc.x - ra.x), fa * (hc.y - ra.y));
                const double2 cb = make_double2(gx - scx - ca.x, gy - scy - ca.y);
                // the contribution to neighbour k-1 is cb_{k-1} + ca_k
                if (k == 0) ca0 = ca;
                else atomic_add2<double>(a.F, nprev, cbp.x + ca.x, cbp.y + ca.y);
                cbp = cb;
                nprev = nb[k];
                hm = hc;
                hc = hn;
                um = uk;
                dc = dn;
            }
        }
        atomic_add2<double>(a.F, nprev, cbp.x + ca0.x, cbp.y + ca0.y);
        atomic_add2<double>(a.F, c, sx, sy);
    }
    if (TEST && fail != 0x7fffffff) flag_cell(a, c, z, true, fail, VG);
    return false;
}

union ThreadWarpSmem {
    ThreadTile t;                 // the thread form's vertices
    GrpTile<double, VG> g[GPW];   // then the group tiles of the warp's longer rows
};

template <bool TEST, int TPB, int MINB>
__global__ void __launch_bounds__(TPB, MINB) k_voro_thread(VoroArgs a)
{
    __shared__ ThreadWarpSmem wsm[TPB / WARP];
    const int c = blockIdx.x * TPB + threadIdx.x;
    const int lane = threadIdx.x & (WARP - 1), w = threadIdx.x / WARP;
    const bool halted = a.ctl && a.ctl->halt;  // uniform across the grid
    const bool defer = c < a.N && !halted && thread_cell<TEST>(a, c, wsm[w].t, lane);
    __syncwarp();  // the warp's vertex columns are free for its group tiles
    // the warp's rows of 9-16 entries, four at a time in its 8-lane groups
    unsigned left = __ballot_sync(0xffffffffu, defer);
    const int gl = lane & (G - 1), gi = lane >> 3;
    while (left) {  // warp-uniform
        int pick = -1;
        unsigned m = left;
        for (int i = 0; i <= gi && m; ++i) {
            pick = __ffs(m) - 1;
            m &= m - 1;
            if (i < gi) pick = -1;
        }
        grp_cell<double, true, TEST, VG, 0>(a, pick >= 0 ? c - lane + pick : 0, pick >= 0, gl, wsm[w].g[gi]);
        for (int i = 0; i < GPW && left; ++i) left &= left - 1;
    }
}

// Repair control. The exact test seeds queue 0 with the cells of every failing edge (its two ends
// and both apexes, or the corners of an inverted triangle). Their stars are recomputed exactly;
// rows that changed must agree with their partners' rows, and disagreeing partners are queued for
// the next round. A round's kernels take their round index from the control block, so the rounds
// can run inside a CUDA-graph WHILE node whose condition the device sets (cudaGraphSetConditional),
// and an empty round costs nothing.
// Start of the repair: first the slots the force pass's filter left undecided. Each is decided by
// the canonical evaluation (incircle_canonical); a failing one is handled as the force pass handles
// a failing edge: the cell's contributions, already scattered, are retracted and the cell is marked
// held (once per cell), and the cell, the edge's other end and both apexes are queued. Then the
// WHILE node is entered if queue 0 has cells.
// Decide the undecided slots t = base + (lane >> 3) (one per 8-lane group; whole warp, the warp's
// four group tiles in wt)
template <typename R, int NS>
CG_D void undec_groups(const VoroArgs &a, Ctl *ctl, int nu, int forces, int base, GrpTile<R, NS> *wt, int lane)
{
    const int gl = lane & (G - 1), gi = lane >> 3;
    const int e = ctl->epoch;
    const int t = base + gi;
    int c = 0, k = 0, z = 0;
    const int *row = a.nbr;
    double Lx = 1, Ly = 1;
    double2 pc = make_double2(0, 0);
    bool fails = false;
    if (t < nu) {
        const int en = a.undec[t];
        c = en / KMAX;
        k = en % KMAX;
        z = a.nn[c];
        row = a.nbr + (size_t)c * a.K;
        const Inst &in = inst_of(a, c);
        Lx = in.Lx;
        Ly = in.Ly;
        pc = a.pos[c];
        if (gl == 0)
            fails = incircle_canonical(c, row[k == 0 ? z - 1 : k - 1], row[k], row[k + 1 == z ? 0 : k + 1],
                                       a.pos, Lx, Ly) < 0;
    }
    fails = __shfl_sync(0xffffffffu, fails, lane & ~(G - 1));
    // retract the contributions once per cell (unless the force pass already held them)
    bool first = false;
    if (fails && gl == 0) {
        first = !forces || atomicExch(&a.held[c], 1) == 0;
        atomicAdd(&ctl->n_flagged, 1);
        claim_flip(a, e, c, row[k], row[k == 0 ? z - 1 : k - 1], row[k + 1 == z ? 0 : k + 1]);
    }
    first = __shfl_sync(0xffffffffu, first, lane & ~(G - 1));
    if (forces) {
        const bool ok = fails && first && z >= 3 && z <= NS;
        int nbk[NS / G];
        double A, P;
        int fl;
        grp_geometry<R, true, false, NS>(a, c, row, z, ok, pc, Lx, Ly, gl, wt[gi], nbk, A, P, fl);
        grp_scatter<R, -1, NS>(a, c, z, ok, gl, wt[gi], nbk, A, P);
    }
    __syncwarp();
}

template <typename R, int NS = VG>
__global__ void __launch_bounds__(256) k_repair_begin(VoroArgs a, unsigned long long cond, int use_cond,
                                                      int forces)
{
    constexpr int WPB = NS == VG ? 8 : 4;  // launched with WPB warps (shared tiles stay under 48 KB)
    __shared__ GrpTile<R, NS> tile[WPB * GPW];
    Ctl *ctl = a.ctl;
    const int nu = min(ctl->n_undec, a.N);
    if (!ctl->halt && nu > 0 && a.undec) {
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        for (int base = w * GPW; base < nu; base += WPB * GPW)  // warp-uniform
            undec_groups<R, NS>(a, ctl, nu, forces, base, tile + w * GPW, lane);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->n_undec = 0;
        ctl->round = 0;
        unsigned v = (!ctl->halt && ctl->q_count[0] > 0) ? 1u : 0u;
        if (use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, v);
    }
}

// end of a repair round (one thread): count it, advance to the next round, and decide whether the
// WHILE node runs another round; a queue that is still not empty after R_MAX rounds escalates to a
// global rebuild
CG_D void round_end(Ctl *ctl, unsigned long long cond, int use_cond)
{
    volatile Ctl *vc = ctl;
    int r = vc->round;
    unsigned v = 0;
    ctl->counters[7] += 1ull;  // executed repair rounds (2 kernels each)
    if (!vc->halt) {
        const int qr = vc->q_count[r];
        ctl->counters[1] += (unsigned long long)qr;
        if (qr > 0) ctl->counters[3] += 1ull;
        int nxt = r + 1;
        vc->round = nxt;
        if (nxt <= R_MAX && vc->q_count[nxt] > 0) {
            if (nxt >= R_MAX) {
                // the local repair did not converge: escalate to a global rebuild
                vc->need_global = 1;
                vc->status = CG_ERR_TOPOLOGY;
                vc->halt = 1;
            } else {
                v = 1;
            }
        }
    }
    if (use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, v);
}

// ------------------------------------------------------------------------------------------
// warp-cooperative exact Delaunay star of the origin among m candidates in shared memory.
// Gift wrapping: start from the nearest candidate (always a Delaunay neighbour); from neighbour a,
// the next counter-clockwise neighbour is the candidate strictly counter-clockwise of a whose circle
// through (0, a, b) is innermost in the pencil of circles through 0 and a (exact in-circle order,
// ties by index). Each step is a warp argmin under that order: a floating-point key with a rigorous
// error interval picks the minimum, and the exact predicate runs only among the candidates whose
// intervals reach below the smallest upper end. Writes global indices, CCW, rotated to start at the
// smallest index. Returns z, -1 (not enclosed), -2 (capacity).
// ------------------------------------------------------------------------------------------
struct StarFrame {
    int self;            // global index of the cell at the origin
    const double2 *pos;  // absolute positions, for the canonical-frame predicate
    double Lx, Ly;
};

// is c's circle through (0,a,c) strictly inside b's circle (0,a,b)?  <=> c inside circle(0,a,b);
// incircle_g never returns 0, so the order is strict
CG_D bool inner_than(const StarFrame &f, double2 pa, int ia, double2 pc, int ic, double2 pb, int ib)
{
    return incircle_g(pa, pb, pc, f.self, ia, ib, ic, f.pos, f.Lx, f.Ly) < 0;
}

// Position of the circle through 0, a and t in the pencil of circles through 0 and a: its centre is
// a/2 + s (-a.y, a.x) with s = t.(t - a) / (2 a x t). For t strictly counter-clockwise of a
// (a x t > 0), a point t' on that side lies strictly inside the circle of t exactly when
// s(t') < s(t), so the next Delaunay neighbour minimises s. [lo, hi] encloses the exact s: with
// u = 2^-53, the numerator's error is below 4u(|t.x dx| + |t.y dy|), the cross product's below
// ED = 3u(|a.x t.y| + |a.y t.x|), and for den > ED the quotient's below
// |num| ED / (den (den - ED)) + EN / (den - ED), plus u|s| for the division; the interval doubles
// the total. The interval must also hold the key of every frame the exact comparison may use (see
// incircle_g): inputs off by at most q = 4.5 u L per coordinate move num by at most
// q (3|t|_1 + |a|_1) and den by at most q (|t|_1 + |a|_1), which is added the same way.
// Near-collinear t (den <= 2 (ED + that)) gets an unbounded interval.
CG_D void pencil_key(double2 a, double2 t, double Lmax, double &lo, double &hi)
{
    const double u = 1.1102230246251565e-16;
    const double q = 5.0 * u * Lmax;
    double dx = t.x - a.x, dy = t.y - a.y;
    double n1 = t.x * dx, n2 = t.y * dy;
    double num = n1 + n2;
    double ta = fabs(t.x) + fabs(t.y), aa = fabs(a.x) + fabs(a.y);
    double EN = 4.0 * u * (fabs(n1) + fabs(n2)) + q * (3.0 * ta + aa);
    double d1 = a.x * t.y, d2 = a.y * t.x;
    double den = d1 - d2;
    double ED = 3.0 * u * (fabs(d1) + fabs(d2)) + q * (ta + aa);
    if (!(den > 2.0 * ED)) {
        lo = -HUGE_VAL;
        hi = HUGE_VAL;
        return;
    }
    // one reciprocal: with dm = den - ED >= den / 2, the quotient's error
    // 0.5 (|num| ED / (den dm) + EN / dm) is at most (|num| ED / den + EN) / den; forming s from the
    // reciprocal rounds twice (3u|s| covers it and the bound's own rounding)
    double id = 1.0 / den;
    double s = 0.5 * num * id;
    double err = (fabs(num) * ED * id + EN) * id + 3.0 * u * fabs(s);
    err *= 2.0;
    lo = s - err;
    hi = s + err;
}

// order-preserving map of a float onto an unsigned key (for the warp min reduction) and back
CG_D unsigned float_order_key(float f)
{
    unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
CG_D float float_from_order_key(unsigned k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__device__ int warp_star(const double2 *rel, const int *gidx, int m, int K, int *out, int lane,
                         const StarFrame &f)
{
    const double Lmax = fmax(f.Lx, f.Ly);
    const unsigned full = 0xffffffffu;
    // nearest candidate
    double best = 1e300;
    int bi = -1;
    for (int t = lane; t < m; t += WARP) {
        double d = rel[t].x * rel[t].x + rel[t].y * rel[t].y;
        if (d < best || (d == best && bi >= 0 && gidx[t] < gidx[bi])) {
            best = d;
            bi = t;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        double ob = __shfl_xor_sync(full, best, off);
        int oi = __shfl_xor_sync(full, bi, off);
        if (oi >= 0 && (bi < 0 || ob < best || (ob == best && gidx[oi] < gidx[bi]))) {
            best = ob;
            bi = oi;
        }
    }
    if (bi < 0) return -1;
    int start = bi, cur = bi, z = 0;
    for (int guard = 0; guard <= m; ++guard) {
        if (z >= K) return -2;
        if (lane == 0) out[z] = cur;
        ++z;
        double2 pa = rel[cur];
        // pass 1: key intervals of the counter-clockwise candidates (a lane keeps the lower ends of
        // its first two) and their smallest upper end U over the warp, rounded up to a float so
        // that one integer min reduction finds it (a U above the exact minimum only lets more
        // candidates through to the exact comparison)
        double klo0 = 0.0, klo1 = 0.0;
        unsigned ccw = 0u;
        unsigned ukey = 0xffffffffu;
        bool any = false;
        for (int j = 0, t = lane; t < m; ++j, t += WARP) {
            if (t == cur) continue;
            double2 pt = rel[t];
            if (orient0(pa, pt) <= 0) continue;
            double lo, hi;
            pencil_key(pa, pt, Lmax, lo, hi);
            if (j == 0) klo0 = lo;
            else if (j == 1) klo1 = lo;
            if (j < 2) ccw |= 1u << j;
            ukey = min(ukey, float_order_key(__double2float_ru(hi)));
            any = true;
        }
        if (!__any_sync(full, any)) return -1;
        ukey = __reduce_min_sync(full, ukey);
        const double U = (double)float_from_order_key(ukey);
        // pass 2: only candidates with lo <= U can be the minimum; order them exactly
        int b = -1, cnt = 0;
        for (int j = 0, t = lane; t < m; ++j, t += WARP) {
            if (t == cur) continue;
            double2 pt = rel[t];
            double lo;
            if (j < 2) {
                if (!(ccw & (1u << j))) continue;
                lo = j == 0 ? klo0 : klo1;
            } else {
                if (orient0(pa, pt) <= 0) continue;
                double hi;
                pencil_key(pa, pt, Lmax, lo, hi);
            }
            if (!(lo <= U)) continue;
            ++cnt;
            if (b < 0 || inner_than(f, pa, gidx[cur], pt, gidx[t], rel[b], gidx[b])) b = t;
        }
        unsigned has = __ballot_sync(full, cnt > 0);
        if (__reduce_add_sync(full, (unsigned)cnt) > 1u) {
            for (int off = 16; off > 0; off >>= 1) {
                int ob = __shfl_xor_sync(full, b, off);
                if (ob >= 0 && (b < 0 || inner_than(f, pa, gidx[cur], rel[ob], gidx[ob], rel[b], gidx[b]))) b = ob;
            }
        } else {
            b = __shfl_sync(full, b, __ffs(has) - 1);
        }
        if (b < 0) return -1;
        if (b == start) {
            __syncwarp();
            // map to global indices and rotate to the smallest
            int mn = 0x7fffffff, mpos = 0;
            for (int t = 0; t < z; ++t) {
                int g = gidx[out[t]];
                if (g < mn) {
                    mn = g;
                    mpos = t;
                }
            }
            __syncwarp();
            int tmp = 0;
            if (lane < z) tmp = gidx[out[(mpos + lane) % z]];
            __syncwarp();
            if (lane < z) out[lane] = tmp;
            __syncwarp();
            return z;
        }
        cur = b;
    }
    return -1;
}

// compact the candidate list in place, dropping `self` (no repeats possible)
CG_D int warp_remove(int *cand, int m, int self, int lane)
{
    int out = 0;
    for (int base = 0; base < m; base += WARP) {
        int t = base + lane;
        int v = (t < m) ? cand[t] : -1;
        bool keep = (t < m) && v != self;
        unsigned bal = __ballot_sync(0xffffffffu, keep);
        __syncwarp();
        if (keep) cand[out + __popc(bal & ((1u << lane) - 1u))] = v;
        out += __popc(bal);
        __syncwarp();
    }
    return out;
}

// Local repair star: candidates = the current 2-ring of the cell (its neighbours and theirs).
// One warp per queued cell; result goes to the staging row of the queue slot. Rows are expanded
// two at a time (16 lanes each, rows hold at most 16 entries), and candidates are deduplicated in a
// per-warp open-addressing table in shared memory, so collecting a ring costs a few parallel loads.
constexpr int CAND_HASH = 512;  // > CAND_LOCAL + 32: the table never fills
constexpr int STAR_MINB = 5;    // resident blocks of k_star_local per SM (its grid is one such wave)

CG_D void cand_insert(int *table, int *list, int *count, int v)
{
    unsigned h = ((unsigned)v * 2654435761u) >> 23;  // 9 bits
    for (int probe = 0; probe < CAND_HASH; ++probe) {
        int prev = atomicCAS(&table[h], -1, v);
        if (prev == -1) {
            int idx = atomicAdd(count, 1);
            if (idx < CAND_LOCAL) list[idx] = v;
            return;
        }
        if (prev == v) return;
        h = (h + 1) & (CAND_HASH - 1);
    }
}

// per-warp shared memory of the local star: candidate positions relative to the cell, their
// global indices, the deduplication table, the star and the candidate count
struct StarSmem {
    double2 rel[CAND_LOCAL];
    int cand[CAND_LOCAL];
    int hash[CAND_HASH];
    int out[KMAX];
    int m;
};

// First-round fast path: the row a single edge flip gives (whole warp). h is the hint the claim
// left: {1, v, -, -} drops v; {2, v, a, b} inserts v between the consecutive entries a and b. The
// row is rotated to start at its smallest entry and written to out. Returns the new length, or -1
// when the row does not have the shape the edit expects (v missing or already there, a and b not
// consecutive, fewer than 3 entries left, or no room), and the caller computes the star.
// The edit is used only for a cell that exactly one claim of the step named (nclaim), so it does
// not depend on the order of the claims; cells named by several failing edges get their stars. An
// edited row that the round's check finds wanting (a partner's row disagrees, or an edge fails the
// exact test: the cell had another failing edge, which only its first is reported for) queues the
// cell itself for the next round, whose stars are computed in full.
CG_D int flip_edit(const int *row, int z, int K, int4 h, int *out, int lane)
{
    const unsigned full = 0xffffffffu;
    const int v = lane < z ? row[lane] : -1;
    const unsigned has = __ballot_sync(full, lane < z && v == h.y);
    int nv, nz;
    if (h.x == 1) {
        if (__popc(has) != 1 || z - 1 < 3) return -1;
        const int pos = __ffs(has) - 1;
        nv = __shfl_sync(full, v, lane < pos ? lane : (lane + 1) & 31);
        nz = z - 1;
    } else {
        const int nxt = __shfl_sync(full, v, lane + 1 >= z ? 0 : lane + 1);
        const unsigned at = __ballot_sync(full, lane < z && v == h.z && nxt == h.w);
        if (has != 0u || __popc(at) != 1 || z + 1 > K) return -1;
        const int pos = __ffs(at) - 1;  // v goes after pos
        nv = __shfl_sync(full, v, lane <= pos ? lane : lane - 1);
        if (lane == pos + 1) nv = h.y;
        nz = z + 1;
    }
    const int mn = __reduce_min_sync(full, lane < nz ? (unsigned)nv : 0xffffffffu);
    const int r0 = __ffs(__ballot_sync(full, lane < nz && nv == mn)) - 1;
    int src = lane + r0;
    if (src >= nz) src -= nz;
    const int rv = __shfl_sync(full, nv, src & 31);
    if (lane < nz) out[lane] = rv;
    __syncwarp();
    return nz;
}

// exact star of the cell in queue slot q of `round` (whole warp); the result goes to the slot's
// staging row, a failure halts the step
CG_D void star_one(const VoroArgs &a, Ctl *ctl, int round, const int *queue, int q, StarSmem &S, int lane)
{
    volatile int *vm = &S.m;
    int c = queue[q];
    const Inst &in = inst_of(a, c);
    int z = a.nn[c];
    const int *row = a.nbr + (size_t)c * a.K;
    if (round == 0 && a.qhint) {
        const int4 h = a.qhint[q];
        const int claims = a.nclaim[c];
        __syncwarp();
        if (lane == 0) a.nclaim[c] = 0;  // every counted cell is in this queue: ready for the next step
        const int nz = (h.x != 0 && claims == 1) ? flip_edit(row, z, a.K, h, S.out, lane) : -1;
        if (nz > 0) {
            if (lane < nz) a.stage_nbr[(size_t)q * a.K + lane] = S.out[lane];
            if (lane == 0) a.stage_nn[q] = nz;
            __syncwarp();
            return;
        }
        if (lane == 0 && h.x != 0) a.qhint[q].x = 0;  // the check then knows the row is a star
    }
    for (int i = lane; i < CAND_HASH; i += WARP) S.hash[i] = -1;
    if (lane == 0) *vm = 0;
    __syncwarp();
    if (lane < z) cand_insert(S.hash, S.cand, &S.m, row[lane]);
    __syncwarp();
    // ring 1 expands the row's members; from round 1 on, ring 2 expands the new 2-ring members
    // too (3-ring), for cells whose new star reaches further
    int lo = 0, hi = min(*vm, CAND_LOCAL);
    for (int ring = 0; ring < (round == 0 ? 1 : 2); ++ring) {
        // rows are padded with -1 past their length, so whole rows are read without their
        // lengths; a lane takes slot (lane & 15) of members lane >> 4, +2, +4, +6 of each group
        // of 8 members, and the four loads are in flight together
        for (int base = lo; base < hi; base += 8) {
            for (int eb = 0; eb < a.K; eb += 16) {  // rows wider than 16 (K = 32) in two halves
                const int e = eb + (lane & 15);
                int v[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int j = base + (lane >> 4) + 2 * i;
                    v[i] = (j < hi && e < a.K) ? a.nbr[(size_t)S.cand[j] * a.K + e] : -1;
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (v[i] >= 0 && v[i] != c && *vm < CAND_LOCAL) cand_insert(S.hash, S.cand, &S.m, v[i]);
            }
        }
        __syncwarp();
        lo = hi;
        hi = min(*vm, CAND_LOCAL);
    }
    int m = min(*vm, CAND_LOCAL);
    double2 pc = a.pos[c];
    for (int t = lane; t < m; t += 2 * WARP) {
        const int t2 = t + WARP;
        double2 p1 = a.pos[S.cand[t]];
        double2 p2 = t2 < m ? a.pos[S.cand[t2]] : pc;
        S.rel[t] = min_dist(p1, pc, in.Lx, in.Ly);
        if (t2 < m) S.rel[t2] = min_dist(p2, pc, in.Lx, in.Ly);
    }
    __syncwarp();
    StarFrame fr = {c, a.pos, in.Lx, in.Ly};
    int zs = warp_star(S.rel, S.cand, m, a.K, S.out, lane, fr);
    if (zs < 0) {
        if (lane == 0) {
            atomicExch(&ctl->need_global, 1);
            atomicExch(&ctl->status, zs == -2 ? CG_ERR_CAPACITY : CG_ERR_TOPOLOGY);
            atomicExch(&ctl->halt, 1);
        }
        __syncwarp();
        return;
    }
    if (lane < zs) a.stage_nbr[(size_t)q * a.K + lane] = S.out[lane];
    if (lane == 0) a.stage_nn[q] = zs;
    __syncwarp();
}

template <int WPB>
__global__ void __launch_bounds__(WPB * 32, STAR_MINB) k_star_local(VoroArgs a)
{
    __shared__ StarSmem s_star[WPB];
    Ctl *ctl = a.ctl;
    if (ctl->halt) return;
    int round = ctl->round;
    if (round >= R_MAX) return;
    int nq = ctl->q_count[round];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int gw = blockIdx.x * WPB + w, nw = gridDim.x * WPB;
    const int *queue = a.queue + (size_t)round * a.N;
    for (int q = gw; q < nq; q += nw) star_one(a, ctl, round, queue, q, s_star[w], lane);
}

CG_D int row_find(const int *row, int z, int v)
{
    for (int k = 0; k < z; ++k)
        if (row[k] == v) return k;
    return -1;
}

// does row (length z) contain u immediately followed (cyclically) by v?
CG_D bool row_has_pair(const int *row, int z, int u, int v)
{
    int s = row_find(row, z, u);
    if (s < 0) return false;
    int t = s + 1;
    if (t == z) t = 0;
    return row[t] == v;
}

// does `row` (length z, capacity stride K) contain u immediately followed (cyclically) by v? Rows
// of 16-byte aligned capacity (K % 4 == 0) are read with independent 16-byte loads, so a lookup
// costs one memory latency.
template <int NS = VG>
CG_D bool pair_in(const int *row, int z, int K, int u, int v)
{
    if ((K & 3) != 0) return row_has_pair(row, z, u, v);
    int e[NS + 1];
    const int4 *r4 = reinterpret_cast<const int4 *>(row);
#pragma unroll
    for (int j = 0; j < NS / 4; ++j) {
        int4 t = (4 * j < K) ? r4[j] : make_int4(-1, -1, -1, -1);
        e[4 * j] = t.x;
        e[4 * j + 1] = t.y;
        e[4 * j + 2] = t.z;
        e[4 * j + 3] = t.w;
    }
    e[NS] = -1;
    bool found = false;
#pragma unroll
    for (int k = 0; k < NS; ++k)
        if (k < z && e[k] == u) found = (k + 1 < z ? e[k + 1] : e[0]) == v;
    return found;
}

// The row cell x has at the end of the current round: its staged star when x is queued in this
// round (queue slot from qslot, checked against the queue itself, so a stale entry from an earlier
// round is never taken), else its current row, which no thread writes during the round.
CG_D const int *future_row(const VoroArgs &a, int x, int round, int nq, const int *queue, int &z)
{
    const int s = a.qslot[(size_t)(round & 1) * a.N + x];
    if (s >= 0 && s < nq && queue[s] == x) {
        z = a.stage_nn[s];
        return a.stage_nbr + (size_t)s * a.K;
    }
    z = a.nn[x];
    return a.nbr + (size_t)x * a.K;
}

// Commit and check one repair round, 16 lanes per queue slot. Its first 8-lane group retracts the
// old row's force contributions while the second adds the new (staged) row's, with the same group
// code as the force pass; A/P are refreshed from the new row, which replaces the old one (padded
// with -1). Unchanged rows whose contributions the force pass held back add them now. Then the
// consistency check, against the rows every cell will have at the end of the round (future_row):
// every triangle (c,u,v) of the new row must appear in the rows of u and v, every dropped triangle
// must be gone from them, and a changed row must pass the exact local test (every edge). Offending
// cells are claimed for the next round. The last block to finish ends the round (round_end).
// Commit and check queue slots base and base + 1 of `round` (whole warp: 16 lanes per slot, the
// warp's four group tiles in wt)
template <typename R, bool FORCES, int NS>
CG_D void cc_pair(const VoroArgs &a, Ctl *ctl, int round, int nq, const int *queue, int e_next, int base,
                  GrpTile<R, NS> *wt, int lane)
{
    const unsigned full = 0xffffffffu;
    const int gl = lane & (G - 1), gi = lane >> 3;
    GrpTile<R, NS> &tl = wt[gi];
    const bool add = gi & 1;   // group 0 of a slot: old row (retract); group 1: new row (add)
    const int hl = lane & 15;  // lane within the slot's 16 lanes
    const int q = base + (gi >> 1);
    const bool live = q < nq;
    int c = 0, zo = 0, zn = 0;
    if (live) {
        c = queue[q];
        zo = a.nn[c];
        zn = a.stage_nn[q];
    }
    int *row = a.nbr + (size_t)c * a.K;
    const int *srow = a.stage_nbr + (size_t)(live ? q : 0) * a.K;
    bool diff = live && zo != zn;
#pragma unroll
    for (int e = hl; e < NS; e += 16)
        if (live && !diff && e < zn && row[e] != srow[e]) diff = true;
    int dv = diff ? 1 : 0;
    dv |= __shfl_xor_sync(full, dv, 1);
    dv |= __shfl_xor_sync(full, dv, 2);
    dv |= __shfl_xor_sync(full, dv, 4);
    dv |= __shfl_xor_sync(full, dv, 8);
    diff = dv != 0;
    const bool was_held = live && a.held && a.held[c];
    double2 pc = make_double2(0, 0);
    double Lx = 1, Ly = 1;
    if (live) {
        const Inst &in = inst_of(a, c);
        Lx = in.Lx;
        Ly = in.Ly;
        pc = a.pos[c];
    }
    // this group's row (old or new) in registers: slot k = gl + G r and its successor
    const int *grow = add ? srow : row;
    const int gz = add ? zn : zo;
    int ek[NS / G], ek1[NS / G];
#pragma unroll
    for (int r = 0; r < NS / G; ++r) {
        const int k = gl + G * r;
        ek[r] = -1;
        ek1[r] = -1;
        if (live && k < gz) {
            ek[r] = grow[k];
            ek1[r] = grow[k + 1 == gz ? 0 : k + 1];
        }
    }
    // forces: retract the old row (unless the force pass held it back) / add the new one
    const bool gok = add ? (live && (diff || (FORCES && was_held)) && zn >= 3 && zn <= NS)
                         : (FORCES && live && diff && !was_held && zo >= 3 && zo <= NS);
    int nbk[NS / G];
    double A, P;
    int fail;
    grp_geometry<R, FORCES, false, NS>(a, c, grow, gz, gok, pc, Lx, Ly, gl, tl, nbk, A, P, fail, add);
    if (FORCES) grp_scatter<R, 1, NS>(a, c, gz, gok, gl, tl, nbk, A, P, add ? R(1) : R(-1));
    if (add && gok && gl == 0 && a.AP) store_ap<R>(a.AP, c, (R)A, (R)P);
    __syncwarp();
    // the new row replaces the old one, padded with -1 (both were read above)
    if (live && diff) {
#pragma unroll
        for (int t = 0; t < KMAX / 16; ++t) {
            const int e = hl + 16 * t;
            if (e < a.K) row[e] = e < zn ? srow[e] : -1;
        }
    }
    if (live && hl == 0) {
        if (a.held) a.held[c] = 0;
        if (diff) {
            a.nn[c] = zn;
            atomicAdd(&ctl->counters[2], 1ull);
        }
    }
    // consistency against the end-of-round rows; a row from a first-round flip edit that a partner
    // disagrees with is queued again itself (it may be the wrong one)
    const bool edited = round == 0 && a.qhint && live && diff && a.qhint[q].x != 0;
    bool bad = false, disagree = false;
    if (add) {
        bad = live && diff && zn < 3;
#pragma unroll
        for (int r = 0; r < NS / G; ++r) {
            const int k = gl + G * r;
            if (live && k < zn) {
                const int u = ek[r], v = ek1[r];
                int zu, zv;
                const int *fu = future_row(a, u, round, nq, queue, zu);
                const int *fv = future_row(a, v, round, nq, queue, zv);
                if (!pair_in<NS>(fu, zu, a.K, v, c)) {
                    claim_enqueue(a, u, e_next, round + 1);
                    disagree = true;
                }
                if (!pair_in<NS>(fv, zv, a.K, c, u)) {
                    claim_enqueue(a, v, e_next, round + 1);
                    disagree = true;
                }
                if (diff && zn >= 3 && gok) {
                    // exact local test of the new row (every edge): relative positions from
                    // the group's tile (grp_geometry stored them)
                    const int km = k == 0 ? zn - 1 : k - 1, kp = k + 1 == zn ? 0 : k + 1;
                    const double2 dA = tl.r[km], dB = tl.r[k], dC = tl.r[kp];
                    const int um = srow[km];
                    if (orient0(dB, dC) <= 0 || incircle_g(dA, dB, dC, c, um, u, v, a.pos, Lx, Ly) < 0)
                        bad = true;
                }
            }
        }
    } else if (live && diff) {
        // dropped triangles of the old row must be gone from the partners' rows
#pragma unroll
        for (int r = 0; r < NS / G; ++r) {
            const int k = gl + G * r;
            if (k < zo) {
                const int u = ek[r], v = ek1[r];
                if (!pair_in<NS>(srow, zn, a.K, u, v)) {
                    int zu, zv;
                    const int *fu = future_row(a, u, round, nq, queue, zu);
                    const int *fv = future_row(a, v, round, nq, queue, zv);
                    if (pair_in<NS>(fu, zu, a.K, v, c)) {
                        claim_enqueue(a, u, e_next, round + 1);
                        disagree = true;
                    }
                    if (pair_in<NS>(fv, zv, a.K, c, u)) {
                        claim_enqueue(a, v, e_next, round + 1);
                        disagree = true;
                    }
                }
            }
        }
    }
    // both 8-lane groups of the slot (old row, new row) vote on the edited row
    int dv2 = edited && disagree ? 1 : 0;
    dv2 |= __shfl_xor_sync(0xffffffffu, dv2, 1);
    dv2 |= __shfl_xor_sync(0xffffffffu, dv2, 2);
    dv2 |= __shfl_xor_sync(0xffffffffu, dv2, 4);
    dv2 |= __shfl_xor_sync(0xffffffffu, dv2, 8);
    bad = bad || dv2 != 0;
    bad = group_any(bad);
    if (add && bad) {
        if (gl == 0) claim_enqueue(a, c, e_next, round + 1);
#pragma unroll
        for (int r = 0; r < NS / G; ++r)
            if (ek[r] >= 0) claim_enqueue(a, ek[r], e_next, round + 1);
    }
    __syncwarp();
}

template <typename R, bool FORCES, int WPB, int NS = VG>
__global__ void __launch_bounds__(WPB * 32) k_commit_check(VoroArgs a, unsigned long long cond, int use_cond)
{
    __shared__ GrpTile<R, NS> tile[WPB * GPW];
    __shared__ int s_last;
    Ctl *ctl = a.ctl;
    const int round = ctl->round;
    if (!ctl->halt && round < R_MAX) {
        const int nq = ctl->q_count[round];
        const int *queue = a.queue + (size_t)round * a.N;
        const int e_next = ctl->epoch + round + 1;  // claim epoch of the next round
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        const int step = gridDim.x * WPB * (GPW / 2);
        for (int base = (blockIdx.x * WPB + w) * (GPW / 2); base < nq; base += step)  // warp-uniform
            cc_pair<R, FORCES, NS>(a, ctl, round, nq, queue, e_next, base, tile + w * GPW, lane);
    }
    // the last block to finish ends the round (threadfence reduction: every block's claims are
    // visible before its count is)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&ctl->blocks_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        __threadfence();
        ctl->blocks_done = 0;
        round_end(ctl, cond, use_cond);
    }
}

// Particle exclusions (voronoiModelBase::setExclusions, src/models/voronoiModelBase.cpp:85-104, and
// the summation with exclusions, src/models/voronoiQuadraticEnergy.cpp:368-377 /
// gpu_sum_forces_with_exclusions_kernel, src/models/voronoiQuadraticEnergy.cu:59-93): once a force
// evaluation is complete, an excluded cell's net force is kept as the external force -F and its
// force is zeroed; other cells keep their external force at zero.
template <typename R>
__global__ void k_apply_exclusions(int N, const int *excl, void *F, double2 *ext)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N || !excl[c]) return;
    double2 *f = reinterpret_cast<double2 *>(F) + c;
    const double2 v = *f;
    ext[c] = make_double2(-v.x, -v.y);
    *f = make_double2(0.0, 0.0);
}

// end of a step: reset the per-step queue counters and advance the claim epoch
__global__ void k_step_done(Ctl *ctl, int advance_step)
{
    if (ctl->halt) return;
    ctl->step += advance_step;
    if (ctl->n_flagged) atomicAdd(&ctl->counters[0], (unsigned long long)ctl->n_flagged);
    ctl->n_flagged = 0;
    for (int r = 0; r <= R_MAX; ++r) ctl->q_count[r] = 0;
    ctl->round = 0;
    ctl->epoch += R_MAX + 2;
}

// ------------------------------------------------------------------------------------------
// cell list (counting sort, per-instance grids) and the global triangulation
// ------------------------------------------------------------------------------------------
CG_D int bin_of(const Inst &in, double2 p)
{
    int bx = (int)floor(p.x / in.bsx), by = (int)floor(p.y / in.bsy);
    bx = max(0, min(in.nbx - 1, bx));
    by = max(0, min(in.nby - 1, by));
    return in.bin_off + by * in.nbx + bx;
}

__global__ void k_bin_count(VoroArgs a)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.N) return;
    const Inst &in = inst_of(a, c);
    int b = bin_of(in, a.pos[c]);
    a.cell_bin[c] = b;
    a.cell_slot[c] = atomicAdd(&a.bin_count[b], 1);
}

__global__ void k_bin_scatter(VoroArgs a)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.N) return;
    int s = a.bin_start[a.cell_bin[c]] + a.cell_slot[c];
    a.bin_cells[s] = c;
    a.bin_pos[s] = a.pos[c];
}

// Global star of every cell from cell-list candidates in a (2w+1)^2 bin block. A star is accepted
// when every star triangle's circumcircle lies inside the covered disk of radius w*bin, which makes
// it the exact Delaunay star; otherwise the block grows.
template <int WPB>
__global__ void __launch_bounds__(WPB * 32) k_star_global(VoroArgs a, int *status)
{
    __shared__ int s_idx[WPB][CAND_GLOBAL];
    __shared__ double2 s_rel[WPB][CAND_GLOBAL];
    __shared__ int s_out[WPB][KMAX];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int c = blockIdx.x * WPB + w;
    if (c >= a.N) return;
    const Inst &in = inst_of(a, c);
    double2 pc = a.pos[c];
    int cbx = (int)floor(pc.x / in.bsx), cby = (int)floor(pc.y / in.bsy);
    cbx = max(0, min(in.nbx - 1, cbx));
    cby = max(0, min(in.nby - 1, cby));
    int wmaxx = (in.nbx - 1) / 2, wmaxy = (in.nby - 1) / 2;
    double bs = fmin(in.bsx, in.bsy);
    for (int wr = 2;; ++wr) {
        int wx = min(wr, wmaxx), wy = min(wr, wmaxy);
        int m = 0;
        bool overflow = false;
        for (int dy = -wy; dy <= wy && !overflow; ++dy)
            for (int dx = -wx; dx <= wx && !overflow; ++dx) {
                int bx = cbx + dx, by = cby + dy;
                if (bx < 0) bx += in.nbx;
                if (bx >= in.nbx) bx -= in.nbx;
                if (by < 0) by += in.nby;
                if (by >= in.nby) by -= in.nby;
                int b = in.bin_off + by * in.nbx + bx;
                int s0 = a.bin_start[b], cnt = a.bin_count[b];
                if (m + cnt > CAND_GLOBAL) {
                    overflow = true;
                    break;
                }
                for (int t = lane; t < cnt; t += WARP) s_idx[w][m + t] = a.bin_cells[s0 + t];
                m += cnt;
            }
        __syncwarp();
        if (overflow) {
            if (lane == 0) atomicCAS(status, 0, CG_ERR_CAPACITY);
            return;
        }
        __syncwarp();
        m = warp_remove(s_idx[w], m, c, lane);
        for (int t = lane; t < m; t += WARP) s_rel[w][t] = min_dist(a.pos[s_idx[w][t]], pc, in.Lx, in.Ly);
        __syncwarp();
        StarFrame fr = {c, a.pos, in.Lx, in.Ly};
        int z = warp_star(s_rel[w], s_idx[w], m, a.K, s_out[w], lane, fr);
        bool ok = z > 0;
        double R = (double)min(wx, wy) * bs;
        if (ok) {
            // containment: all triangle circumcircles inside the covered disk
            bool good = true;
            for (int t = lane; t < z; t += WARP) {
                int u = s_out[w][t], v = s_out[w][(t + 1) % z];
                double2 ru = min_dist(a.pos[u], pc, in.Lx, in.Ly);
                double2 rv = min_dist(a.pos[v], pc, in.Lx, in.Ly);
                double2 q = circum0<double>(ru, rv);
                double r = sqrt(q.x * q.x + q.y * q.y);
                if (!(2.0 * r < R * (1.0 - 1e-9))) good = false;
            }
            ok = __all_sync(0xffffffffu, good);
        }
        if (ok) {
            if (lane < a.K) a.nbr[(size_t)c * a.K + lane] = lane < z ? s_out[w][lane] : -1;  // padded
            if (lane == 0) a.nn[c] = z;
            return;
        }
        if (z == -2) {
            if (lane == 0) atomicCAS(status, 0, CG_ERR_CAPACITY);
            return;
        }
        if (wx >= wmaxx && wy >= wmaxy) {
            if (lane == 0) atomicCAS(status, 0, CG_ERR_TOPOLOGY);
            return;
        }
    }
}

// triangle-consistency and Euler check of a full triangulation: every triangle (c,u,v) of every row
// must appear in the rows of u and v; per instance, sum z = 6 N.
__global__ void k_validate(VoroArgs a, int *status, unsigned long long *zsum)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.N) return;
    const int *row = a.nbr + (size_t)c * a.K;
    int z = a.nn[c];
    atomicAdd(&zsum[a.cell_inst[c]], (unsigned long long)z);
    for (int k = 0; k < z; ++k) {
        int u = row[k], v = row[(k + 1) % z];
        if (!row_has_pair(a.nbr + (size_t)u * a.K, a.nn[u], v, c) ||
            !row_has_pair(a.nbr + (size_t)v * a.K, a.nn[v], c, u)) {
            atomicCAS(status, 0, CG_ERR_TOPOLOGY);
            return;
        }
    }
}

// ------------------------------------------------------------------------------------------
// integrators, fused with move-and-wrap
// ------------------------------------------------------------------------------------------

// selfPropelledParticleDynamics::integrateEquationsOfMotionCPU
// (src/updaters/selfPropelledParticleDynamics.cpp:67-101) + movePoints (Simple2DCell.cu:21-58):
// v from the current director, displacement dt (v + mu F), director <- atan2(v) + noise.
template <typename R>
CG_D void spp_cell(const VoroArgs &a, int c, double xi, double dt, double mu, int zero_force)
{
    const Inst &in = inst_of(a, c);
    const double2 f = reinterpret_cast<const double2 *>(a.F)[c];  // FP64 in every precision
    double fx = f.x, fy = f.y;
    double2 mot = a.motility[c];
    double th = a.theta[c];
    double s, co;
    sincos(th, &s, &co);
    double vx = __dmul_rn(mot.x, co), vy = __dmul_rn(mot.x, s);
    double dx = __dmul_rn(dt, __dadd_rn(vx, __dmul_rn(mu, fx)));
    double dy = __dmul_rn(dt, __dadd_rn(vy, __dmul_rn(mu, fy)));
    double thn = th;
    if (!(vx == 0. && vy == 0.)) thn = atan2(vy, vx);
    a.theta[c] = __dadd_rn(thn, __dmul_rn(xi, sqrt(__dmul_rn(__dmul_rn(2.0, dt), mot.y))));
    double2 p = a.pos[c];
    p.x = __dadd_rn(p.x, dx);
    p.y = __dadd_rn(p.y, dy);
    a.pos[c] = put_in_box(p, in.Lx, in.Ly, in.iLx, in.iLy);
    if (zero_force) reinterpret_cast<double2 *>(a.F)[c] = make_double2(0.0, 0.0);
}

// device noise of cell c: component (l & 1) of the Box-Muller pair with Philox counter
// (l >> 1, step + the instance's step offset), key = the instance's seed, l = the cell's index
// within its instance -- so a cell's noise does not depend on where its instance sits in a batch,
// nor on which system it has run in
CG_D double2 cell_pair_noise(const VoroArgs &a, int c, uint32_t step, int &local)
{
    const Inst &in = inst_of(a, c);
    local = c - in.off;
    return normal2(in.seed, (uint32_t)(local >> 1), step + in.step_off, 0u);
}

// Two cells per thread: one Box-Muller pair serves both when they are consecutive cells of one
// instance (the usual case) and the noise is generated on the device. step0 is the step counter
// when there is no control block (raw caller).
// the device normals of cells c0 and c0 + 1 at a step: one Box-Muller pair serves both when they
// are consecutive cells of one instance with c0 at an even local index, else each takes its own
CG_D double2 pair_draw(const VoroArgs &a, int c0, uint32_t step)
{
    const bool two = c0 + 1 < a.N;
    int l0, l1;
    double2 g0 = cell_pair_noise(a, c0, step, l0), xi;
    xi.x = (l0 & 1) ? g0.y : g0.x;
    xi.y = 0.0;
    if (two) {
        const Inst &i0 = inst_of(a, c0);
        if (!(l0 & 1) && c0 + 1 < i0.off + i0.n) {
            xi.y = g0.y;
        } else {
            double2 g1 = cell_pair_noise(a, c0 + 1, step, l1);
            xi.y = (l1 & 1) ? g1.y : g1.x;
        }
    }
    return xi;
}

// Deterministic mode: F of every cell from its fixed-point sums (after the step's force pass and
// repair rounds, before anything reads F).
template <typename R>
__global__ void k_fix_forces(VoroArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.N) return;
    const ulonglong2 *w = reinterpret_cast<const ulonglong2 *>(a.Ffix) + 4 * (size_t)i;  // 2 FIXF words
    const ulonglong2 w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3];
    reinterpret_cast<double2 *>(a.F)[i] = make_double2(fix_force_value(w0, w1), fix_force_value(w2, w3));
}

// The same normals for every cell of the current step, into out[N]. The step graph runs this
// beside the repair rounds (which leave most of the GPU idle), so k_spp reads them instead of
// drawing them on the step's critical path; the values are the ones k_spp would draw.
__global__ void k_draw_noise(VoroArgs a, double *out)
{
    const int c0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (c0 >= a.N) return;
    const double2 xi = pair_draw(a, c0, (uint32_t)a.ctl->step);
    out[c0] = xi.x;
    if (c0 + 1 < a.N) out[c0 + 1] = xi.y;
}

template <typename R>
__global__ void k_spp(VoroArgs a, const double *noise, double dt, double mu, uint32_t step0,
                      int zero_force)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    Ctl *ctl = a.ctl;
    if (ctl && ctl->halt) return;
    int c0 = 2 * t;
    if (c0 >= a.N) return;
    bool two = c0 + 1 < a.N;
    double2 xi;
    if (noise) xi = make_double2(noise[c0], two ? noise[c0 + 1] : 0.0);
    else xi = pair_draw(a, c0, ctl ? (uint32_t)ctl->step : step0);
    spp_cell<R>(a, c0, xi.x, dt, mu, zero_force);
    if (two) spp_cell<R>(a, c0 + 1, xi.y, dt, mu, zero_force);
}

// ------------------------------------------------------------------------------------------
// energies per instance (FP64 accumulation)
// ------------------------------------------------------------------------------------------
// Efix (deterministic mode): the sums go to FIXW fixed-point words per instance (fix_add1), which
// k_energy_from_fix converts into E
template <typename R>
__global__ void __launch_bounds__(256) k_energy(VoroArgs a, double *E, unsigned long long *Efix)
{
    __shared__ double s_part[8];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    int inst = 0;
    if (c < a.N) {
        typename Vec2<R>::T ap = reinterpret_cast<typename Vec2<R>::T *>(a.AP)[c];
        double da = (double)ap.x - a.APpref[c].x, dp = (double)ap.y - a.APpref[c].y;
        e = a.KA * da * da + a.KP * dp * dp;
        if (a.TE) e += 0.5 * a.TE[c];  // each unlike edge once, as computeEnergy counts it
        inst = a.cell_inst ? a.cell_inst[c] : 0;
    }
    // instances are contiguous: a block whose first and last cells share an instance reduces in
    // shared memory and adds once; a block across an instance boundary adds per cell
    const int c0 = blockIdx.x * blockDim.x, c1 = min(a.N, c0 + (int)blockDim.x) - 1;
    const int i0 = a.cell_inst ? a.cell_inst[c0] : 0, i1 = a.cell_inst ? a.cell_inst[c1] : 0;
    if (i0 == i1) {
        for (int off = 16; off > 0; off >>= 1) e += __shfl_down_sync(0xffffffffu, e, off);
        if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = e;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_part[w];
            if (Efix) fix_add1(Efix + FIXW * (size_t)i0, t);
            else atomicAdd(&E[i0], t);
        }
    } else if (c < a.N) {
        if (Efix) fix_add1(Efix + FIXW * (size_t)inst, e);
        else atomicAdd(&E[inst], e);
    }
}

// E[i] from the fixed-point sums of k_energy, which are left zeroed for the next call
__global__ void k_energy_from_fix(int n, unsigned long long *Efix, double *E)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned long long *w = Efix + FIXW * (size_t)i;
    E[i] = fix_value(w[0], w[1], w[2]);
    w[0] = w[1] = w[2] = 0ull;
}

// the energy of cell c from its A/P and preferences (half its line-tension sum: each unlike edge
// is counted by both of its cells)
template <typename R>
CG_D double cell_energy(const VoroArgs &a, int c)
{
    typename Vec2<R>::T ap = reinterpret_cast<typename Vec2<R>::T *>(a.AP)[c];
    double da = (double)ap.x - a.APpref[c].x, dp = (double)ap.y - a.APpref[c].y;
    double e = a.KA * da * da + a.KP * dp * dp;
    if (a.TE) e += 0.5 * a.TE[c];
    return e;
}

// The same sums written straight into page-locked host memory (host_out: its device address):
// block partials gather in acc (zero between calls); the last block to finish stores the totals
// to the host buffer and clears acc and its counter for the next call. One kernel replaces a
// memset, the reduction and a device-to-host copy, each a separate operation in the stream.
template <typename R>
__global__ void __launch_bounds__(256) k_energy_to_host(VoroArgs a, double *acc, unsigned *done, double *host_out)
{
    // deterministic mode (a.Ffix set): acc holds FIXW fixed-point words per instance (fix_add1)
    unsigned long long *afix = a.Ffix ? reinterpret_cast<unsigned long long *>(acc) : nullptr;
    __shared__ double s_part[8];
    __shared__ int s_last;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    int inst = 0;
    if (c < a.N) {
        e = cell_energy<R>(a, c);
        inst = a.cell_inst ? a.cell_inst[c] : 0;
    }
    const int c0 = blockIdx.x * blockDim.x, c1 = min(a.N, c0 + (int)blockDim.x) - 1;
    const int i0 = a.cell_inst ? a.cell_inst[c0] : 0, i1 = a.cell_inst ? a.cell_inst[c1] : 0;
    if (i0 == i1) {
        for (int off = 16; off > 0; off >>= 1) e += __shfl_down_sync(0xffffffffu, e, off);
        if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = e;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_part[w];
            if (afix) fix_add1(afix + FIXW * (size_t)i0, t);
            else atomicAdd(&acc[i0], t);
        }
    } else if (c < a.N) {
        if (afix) fix_add1(afix + FIXW * (size_t)inst, e);
        else atomicAdd(&acc[inst], e);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        for (int i = threadIdx.x; i < a.n_inst; i += blockDim.x) {
            if (afix) {
                unsigned long long *w = afix + FIXW * (size_t)i;
                const unsigned long long hi = atomicExch(w, 0ull), lo = atomicExch(w + 1, 0ull);
                const unsigned long long top = atomicExch(w + 2, 0ull);
                host_out[i] = fix_value(hi, lo, top);
            } else {
                unsigned long long v = atomicExch(reinterpret_cast<unsigned long long *>(&acc[i]), 0ull);
                host_out[i] = __longlong_as_double((long long)v);
            }
        }
        __threadfence_system();
        if (threadIdx.x == 0) *done = 0u;
    }
}

// The step's integration with its energy readout (host-energy steps with floating-point force
// sums): k_spp's two cells per thread, whose energies (of the configuration the forces were
// computed on: A/P are not changed by the move) are summed per block of 256 cells and per instance
// as k_energy_to_host sums them, the last block storing the totals to the host buffer. One kernel
// instead of the integrator and a separate readout after the step's epilogue.
template <typename R>
__global__ void __launch_bounds__(128) k_spp_energy(VoroArgs a, const double *noise, double dt, double mu, double *acc,
                                                    unsigned *done, double *host_out)
{
    __shared__ double s_part[4];
    __shared__ int s_last;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    Ctl *ctl = a.ctl;
    const int c0 = 2 * t;
    const bool one = c0 < a.N, two = c0 + 1 < a.N;
    double e0 = 0.0, e1 = 0.0;
    int n0 = 0, n1 = 0;
    if (one) {
        e0 = cell_energy<R>(a, c0);
        n0 = a.cell_inst ? a.cell_inst[c0] : 0;
    }
    if (two) {
        e1 = cell_energy<R>(a, c0 + 1);
        n1 = a.cell_inst ? a.cell_inst[c0 + 1] : 0;
    }
    if (one && !(ctl && ctl->halt)) {  // a halted step does not move (the host recovers it)
        double2 xi;
        if (noise) xi = make_double2(noise[c0], two ? noise[c0 + 1] : 0.0);
        else xi = pair_draw(a, c0, ctl ? (uint32_t)ctl->step : 0u);
        spp_cell<R>(a, c0, xi.x, dt, mu, 0);
        if (two) spp_cell<R>(a, c0 + 1, xi.y, dt, mu, 0);
    }
    const int b0 = 2 * blockIdx.x * blockDim.x, b1 = min(a.N, b0 + 2 * (int)blockDim.x) - 1;
    const int i0 = a.cell_inst ? a.cell_inst[b0] : 0, i1 = a.cell_inst ? a.cell_inst[b1] : 0;
    if (i0 == i1) {
        double e = e0 + e1;
        for (int off = 16; off > 0; off >>= 1) e += __shfl_down_sync(0xffffffffu, e, off);
        if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = e;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tsum = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tsum += s_part[w];
            atomicAdd(&acc[i0], tsum);
        }
    } else {
        if (one) atomicAdd(&acc[n0], e0);
        if (two) atomicAdd(&acc[n1], e1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        for (int i = threadIdx.x; i < a.n_inst; i += blockDim.x) {
            unsigned long long v = atomicExch(reinterpret_cast<unsigned long long *>(&acc[i]), 0ull);
            host_out[i] = __longlong_as_double((long long)v);
        }
        __threadfence_system();
        if (threadIdx.x == 0) *done = 0u;
    }
}

}  // namespace cg
