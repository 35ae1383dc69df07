// cellgpu_b200 -- vertex (AVM) model kernels for sm_100a: fused geometry + forces, Brownian and
// self-propelled integrators, the T1 edge test-and-flip, and the vertex initialisation from a
// Delaunay triangulation (the Voronoi dual). Included into system.cu after voronoi.cu.
#include "voronoi.cuh"

namespace cg {

// T1 candidate queue: one slot per edge of the instance (3 * its vertices), so neither the
// detection nor the keys queued during the replay can overflow

struct VertArgs {
    int Nc, Nv, vmax, n_inst;
    const Inst *inst;
    const int *cell_inst, *vert_inst;
    double2 *vpos;
    double2 *F;
    unsigned long long *Ffix;  // null, or 2 x 4 words per vertex: fixed-point sums of F (fix_add_force)
    double2 *AP;
    const double2 *APpref;
    double KA, KP;
    int *vn, *vcn, *cvn, *cv;
    double *theta;
    const double2 *motility;
    // T1
    double t1;
    int *cand;        // 3*Nv edge keys (3*v + slot), instance i at 3 * (its first vertex)
    int *cand_count;  // n_inst
    int *t1_resume;   // 2 * n_inst: keys of an interrupted sweep kept at the start of the instance's
                      // cand region, (sorted candidates, keys queued by flips); (0, 0) = none
    Ctl *ctl;
    // line tension (VertexQuadraticEnergyWithTension): per-cell types, one gamma (mode 1) or a
    // symmetric ntypes x ntypes matrix (mode 2); TE[c] = sum over the cell's unlike edges of gamma l
    int tension_mode, ntypes;
    double gamma;
    const int *ctype;
    const double *tmat;
    double *TE;
};

// Tension of the edge from vertex v to the next vertex w of cell c's row: the cell across that edge
// is the one of v's other two cells whose row holds w (the cellIdx2 search of
// VertexQuadraticEnergyWithTension::computeVertexTensionForcesCPU,
// src/models/vertexQuadraticEnergyWithTension.cpp:91-119); the weight is nonzero between types.
CG_D double vm_edge_weight(const VertArgs &a, int c, int v, int w)
{
    int across = 0;
    for (int f = 0; f < 3; ++f) {
        int c2 = a.vcn[3 * v + f];
        if (c2 == c) continue;
        const int *r2 = a.cv + (size_t)c2 * a.vmax;
        const int n2 = a.cvn[c2];
        for (int n = 0; n < n2; ++n)
            if (r2[n] == w) across = c2;
    }
    return tension_weight(a, a.ctype[c], a.ctype[across]);
}

// ------------------------------------------------------------------------------------------
// geometry + forces. Per cell: the polygon relative to its vertex at slot z-2, signed shoelace
// area and perimeter (vertexModelBase::computeGeometryCPU, src/models/vertexModelBase.cpp:248-297);
// then every vertex of the cell receives the force set computeForceSetVertexModel(vcur, vlast,
// vnext, KA(A-A0), KP(P-P0)) (inc/utility/functions.h:330-354) -- added directly to the vertex's
// force, which is the sum of its three sets (src/models/vertexQuadraticEnergy.cpp:100-112).
// ------------------------------------------------------------------------------------------
// add a force set to vertex v (the deterministic mode sums in fixed point, in any order exactly)
CG_D void vm_add_force(double2 *F, unsigned long long *Ffix, int v, double fx, double fy)
{
    if (Ffix) {
        fix_add_force(Ffix + 2 * FIXF * (size_t)v, fx);
        fix_add_force(Ffix + 2 * FIXF * (size_t)v + FIXF, fy);
    } else {
        atomicAdd(&F[v].x, fx);
        atomicAdd(&F[v].y, fy);
    }
}

// deterministic mode: F of every vertex from its fixed-point sums
__global__ void k_vm_fix_forces(VertArgs a)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.Nv) return;
    const ulonglong2 *w = reinterpret_cast<const ulonglong2 *>(a.Ffix) + 4 * (size_t)v;  // 2 FIXF words
    const ulonglong2 w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3];
    a.F[v] = make_double2(fix_force_value(w0, w1), fix_force_value(w2, w3));
}

__global__ void k_vm_forces(VertArgs a, int scatter)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.Nc) return;
    if (a.ctl && a.ctl->halt) return;
    const Inst &in = a.inst[a.cell_inst[c]];
    int z = a.cvn[c];
    const int *row = a.cv + (size_t)c * a.vmax;
    double2 cp = a.vpos[row[z - 2]];
    double2 vcur = min_dist(a.vpos[row[z - 1]], cp, in.Lx, in.Ly);
    double A = 0.0, P = 0.0;
    for (int n = 0; n < z; ++n) {
        double2 vnext = min_dist(a.vpos[row[n]], cp, in.Lx, in.Ly);
        A += 0.5 * (vcur.x + vnext.x) * (vnext.y - vcur.y);
        double dx = vcur.x - vnext.x, dy = vcur.y - vnext.y;
        P += sqrt(dx * dx + dy * dy);
        vcur = vnext;
    }
    a.AP[c] = make_double2(A, P);
    if (!scatter) return;
    double Adiff = a.KA * (A - a.APpref[c].x), Pdiff = a.KP * (P - a.APpref[c].y);
    double2 vlast = min_dist(a.vpos[row[z - 2]], cp, in.Lx, in.Ly);
    vcur = min_dist(a.vpos[row[z - 1]], cp, in.Lx, in.Ly);
    int vidx = row[z - 1];
    double te = 0.0;
    for (int n = 0; n < z; ++n) {
        int nv = row[n];
        double2 vnext = min_dist(a.vpos[nv], cp, in.Lx, in.Ly);
        double dAx = 0.5 * (vlast.y - vnext.y), dAy = -0.5 * (vlast.x - vnext.x);
        double lx = vlast.x - vcur.x, ly = vlast.y - vcur.y;
        double ln = sqrt(lx * lx + ly * ly);
        double nx = vcur.x - vnext.x, ny = vcur.y - vnext.y;
        double nnm = sqrt(nx * nx + ny * ny);
        double fx = 2.0 * (Adiff * dAx + Pdiff * (lx / ln - nx / nnm));
        double fy = 2.0 * (Adiff * dAy + Pdiff * (ly / ln - ny / nnm));
        if (a.tension_mode) {  // the edge to the next vertex (uniform across the grid)
            double wt = vm_edge_weight(a, c, vidx, nv);
            fx -= wt * nx / nnm;
            fy -= wt * ny / nnm;
            te += wt * nnm;
        }
        vm_add_force(a.F, a.Ffix, vidx, fx, fy);
        vlast = vcur;
        vcur = vnext;
        vidx = nv;
    }
    if (a.TE) a.TE[c] = te;
}

// The same pass with 8 lanes per cell (lane = vertex slot, rows up to VM_ROW_G vertices): the
// relative vertex positions and the per-vertex area and perimeter terms are formed in parallel,
// one lane adds the terms in the reference's vertex order (so A and P are summed as the CPU sums
// them), and every lane forms and scatters the force sets of its vertices.
constexpr int VM_G = 8;
constexpr int VM_ROW_G = 32;

template <int WPB>
__global__ void __launch_bounds__(WPB * 32) k_vm_forces_groups(VertArgs a, int scatter)
{
    constexpr int GPW_ = 32 / VM_G;
    __shared__ double2 sV[WPB * GPW_][VM_ROW_G];
    __shared__ double sA[WPB * GPW_][VM_ROW_G];
    __shared__ double sP[WPB * GPW_][VM_ROW_G];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int gl = lane & (VM_G - 1), gi = lane / VM_G;
    const int sl = w * GPW_ + gi;
    const int c = (blockIdx.x * WPB + w) * GPW_ + gi;
    bool live = c < a.Nc;
    if (a.ctl && a.ctl->halt) live = false;  // uniform across the grid
    // the row's entries (rows are allocated vmax wide), its length, the instance and the
    // preferences are loaded together; then the vertex positions: two dependent loads before the
    // arithmetic
    const int *row = a.cv + (size_t)(live ? c : 0) * a.vmax;
    int z = live ? a.cvn[c] : 0;
    int ent[VM_ROW_G / VM_G];
#pragma unroll
    for (int r = 0; r < VM_ROW_G / VM_G; ++r) {
        const int k = gl + VM_G * r;
        ent[r] = (live && k < a.vmax) ? row[k] : -1;
    }
    const double2 pref = live ? a.APpref[c] : make_double2(0.0, 0.0);
    const int ci = live ? a.cell_inst[c] : 0;
    const bool ok = live && z >= 3 && z <= VM_ROW_G;
    // the reference vertex (slot z - 2) from the lane of the group that holds it
    const int zz = ok ? z - 2 : 0;
    int mine = ent[0];
#pragma unroll
    for (int r = 1; r < VM_ROW_G / VM_G; ++r)
        if ((zz / VM_G) == r) mine = ent[r];
    const int vref = __shfl_sync(0xffffffffu, mine, (lane & ~(VM_G - 1)) + (zz & (VM_G - 1)));
    double Lx = 1.0, Ly = 1.0;
    double2 cp = make_double2(0.0, 0.0);
    if (ok) {
        const Inst &in = a.inst[ci];
        Lx = in.Lx;
        Ly = in.Ly;
        cp = a.vpos[vref];
    }
    int vid[VM_ROW_G / VM_G];
#pragma unroll
    for (int r = 0; r < VM_ROW_G / VM_G; ++r) {
        int k = gl + VM_G * r;
        vid[r] = -1;
        if (ok && k < z) {
            vid[r] = ent[r];
            sV[sl][k] = min_dist(a.vpos[vid[r]], cp, Lx, Ly);
        }
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < VM_ROW_G / VM_G; ++r) {
        int k = gl + VM_G * r;
        if (ok && k < z) {
            double2 vc = sV[sl][k == 0 ? z - 1 : k - 1], vn = sV[sl][k];
            sA[sl][k] = 0.5 * (vc.x + vn.x) * (vn.y - vc.y);
            double dx = vc.x - vn.x, dy = vc.y - vn.y;
            sP[sl][k] = sqrt(dx * dx + dy * dy);
        }
    }
    __syncwarp();
    double A = 0.0, P = 0.0;
    if (ok && gl == 0) {
        for (int n = 0; n < z; ++n) {
            A += sA[sl][n];
            P += sP[sl][n];
        }
        a.AP[c] = make_double2(A, P);
    }
    const int leader = lane & ~(VM_G - 1);
    A = __shfl_sync(0xffffffffu, A, leader);
    P = __shfl_sync(0xffffffffu, P, leader);
    if (!scatter) return;  // uniform
    double Adiff = 0.0, Pdiff = 0.0, te = 0.0;
    if (ok) {
        Adiff = a.KA * (A - pref.x);
        Pdiff = a.KP * (P - pref.y);
    }
#pragma unroll
    for (int r = 0; r < VM_ROW_G / VM_G; ++r) {
        int k = gl + VM_G * r;
        if (ok && k < z) {
            double2 vlast = sV[sl][k == 0 ? z - 1 : k - 1], vcur = sV[sl][k], vnext = sV[sl][k + 1 == z ? 0 : k + 1];
            double dAx = 0.5 * (vlast.y - vnext.y), dAy = -0.5 * (vlast.x - vnext.x);
            double lx = vlast.x - vcur.x, ly = vlast.y - vcur.y;
            double ln = sqrt(lx * lx + ly * ly);
            double nx = vcur.x - vnext.x, ny = vcur.y - vnext.y;
            double nnm = sqrt(nx * nx + ny * ny);
            double fx = 2.0 * (Adiff * dAx + Pdiff * (lx / ln - nx / nnm));
            double fy = 2.0 * (Adiff * dAy + Pdiff * (ly / ln - ny / nnm));
            if (a.tension_mode) {  // the edge to the next vertex (uniform across the grid)
                double wt = vm_edge_weight(a, c, vid[r], row[k + 1 == z ? 0 : k + 1]);
                fx -= wt * nx / nnm;
                fy -= wt * ny / nnm;
                te += wt * nnm;
            }
            vm_add_force(a.F, a.Ffix, vid[r], fx, fy);
        }
    }
    if (a.tension_mode) {
        te += __shfl_xor_sync(0xffffffffu, te, 1);
        te += __shfl_xor_sync(0xffffffffu, te, 2);
        te += __shfl_xor_sync(0xffffffffu, te, 4);
        if (ok && gl == 0 && a.TE) a.TE[c] = te;
    }
}

// brownianParticleDynamics::integrateEquationsOfMotionCPU (src/updaters/brownianParticleDynamics.cpp:92-109)
// + vertexModelBase::moveDegreesOfFreedom (src/models/vertexModelBase.cpp:11-47):
// d = xi sqrt(2 dt T mu) + dt mu F, two normals per vertex (x then y)
__global__ void k_vm_brownian(VertArgs a, const double *noise2, double dt, double mu, double T)
{
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.Nv) return;
    if (a.ctl && a.ctl->halt) return;
    const Inst &in = a.inst[a.vert_inst[v]];
    double r1, r2;
    if (noise2) {
        r1 = noise2[2 * (size_t)v];
        r2 = noise2[2 * (size_t)v + 1];
    } else {
        // counter = the vertex's index within its instance, key = the instance's seed
        double2 g = normal2(in.seed, (uint32_t)(v - in.voff), (a.ctl ? (uint32_t)a.ctl->step : 0u) + in.step_off, 1u);
        r1 = g.x;
        r2 = g.y;
    }
    double amp = sqrt(__dmul_rn(__dmul_rn(__dmul_rn(2.0, dt), T), mu));
    double2 f = a.F[v];
    double dx = __dadd_rn(__dmul_rn(r1, amp), __dmul_rn(__dmul_rn(dt, mu), f.x));
    double dy = __dadd_rn(__dmul_rn(r2, amp), __dmul_rn(__dmul_rn(dt, mu), f.y));
    double2 p = a.vpos[v];
    p.x = __dadd_rn(p.x, dx);
    p.y = __dadd_rn(p.y, dy);
    a.vpos[v] = put_in_box(p, in.Lx, in.Ly, in.iLx, in.iLy);
}

// selfPropelledCellVertexDynamics::integrateEquationsOfMotionCPU
// (src/updaters/selfPropelledCellVertexDynamics.cpp:81-122): vertex velocity = mean of its three
// cells' v0 n, displacement dt (v + mu F), then move; directors are advanced afterwards (below)
__global__ void k_vm_spp_vertices(VertArgs a, double dt, double mu)
{
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.Nv) return;
    if (a.ctl && a.ctl->halt) return;
    const Inst &in = a.inst[a.vert_inst[v]];
    double dx = 0.0, dy = 0.0;
    for (int f = 0; f < 3; ++f) {
        int c = a.vcn[3 * v + f];
        double s, co;
        sincos(a.theta[c], &s, &co);
        double v0 = a.motility[c].x;
        dx = __dadd_rn(dx, __dmul_rn(v0, co));
        dy = __dadd_rn(dy, __dmul_rn(v0, s));
    }
    dx = __ddiv_rn(dx, 3.0);
    dy = __ddiv_rn(dy, 3.0);
    double2 fo = a.F[v];
    double2 p = a.vpos[v];
    p.x = __dadd_rn(p.x, __dmul_rn(dt, __dadd_rn(dx, __dmul_rn(mu, fo.x))));
    p.y = __dadd_rn(p.y, __dmul_rn(dt, __dadd_rn(dy, __dmul_rn(mu, fo.y))));
    a.vpos[v] = put_in_box(p, in.Lx, in.Ly, in.iLx, in.iLy);
}

__global__ void k_vm_spp_directors(VertArgs a, const double *noise, double dt)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.Nc) return;
    if (a.ctl && a.ctl->halt) return;
    double xi;
    if (noise) {
        xi = noise[c];
    } else {
        const Inst &in = a.inst[a.cell_inst[c]];
        xi = normal2(in.seed, (uint32_t)(c - in.off), (a.ctl ? (uint32_t)a.ctl->step : 0u) + in.step_off, 2u).x;
    }
    a.theta[c] = __dadd_rn(a.theta[c], __dmul_rn(xi, sqrt(__dmul_rn(__dmul_rn(2.0, dt), a.motility[c].y))));
}

// ------------------------------------------------------------------------------------------
// T1 transitions. The reference's CPU sweep (vertexModelBase::testAndPerformT1TransitionsCPU,
// src/models/vertexModelBase.cpp:631-787) visits vertex1 ascending and its three neighbour slots,
// tests norm(edge) < threshold on the current state and flips at once, so later tests see moved
// vertices and rewired lists. Here: (1) every edge is tested in parallel on the state at the start
// of the sweep (edges that fail there and are not touched by a flip fail in the sweep too);
// (2) one thread per instance replays the sweep over the candidate keys (3*vertex1 + slot) in
// ascending order, and after each flip queues the keys of every edge the flip moved or rewired that
// lie ahead of the current key -- exactly the edges whose test could change. Equivalent to the
// full sequential sweep, at the cost of the candidates only.
// ------------------------------------------------------------------------------------------
CG_D double edge_len(double2 p1, double2 p2, const Inst &in)
{
    double2 e = min_dist(p1, p2, in.Lx, in.Ly);
    return __dsqrt_rn(__dadd_rn(__dmul_rn(e.x, e.x), __dmul_rn(e.y, e.y)));
}

__global__ void k_vm_t1_detect(VertArgs a)
{
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (a.ctl && a.ctl->halt) return;
    bool any[3] = {false, false, false};
    int inst = 0;
    if (v < a.Nv) {
        inst = a.vert_inst[v];
        const Inst &in = a.inst[inst];
        double2 p = a.vpos[v];
        for (int s = 0; s < 3; ++s) {
            int w = a.vn[3 * v + s];
            if (v < w && edge_len(p, a.vpos[w], in) < a.t1) any[s] = true;
        }
    }
    for (int s = 0; s < 3; ++s) {
        if (any[s]) {
            int slot = atomicAdd(&a.cand_count[inst], 1);
            a.cand[3 * (size_t)a.inst[inst].voff + slot] = 3 * v + s;
        }
    }
}

CG_D void find_in_cell_d(const int *row, int cneigh, int target, int &vlast, int &vcur, int &vnext)
{
    int l = row[cneigh - 2], c = row[cneigh - 1], nx = row[0];
    for (int cn = 0; cn < cneigh; ++cn) {
        nx = row[cn];
        if (c == target) break;
        l = c;
        c = nx;
    }
    vlast = l;
    vcur = c;
    vnext = nx;
}

// getCellVertexSetForT1 (src/models/vertexModelBase.cpp:507-625), without its unused first loop
CG_D void t1_sets_d(const VertArgs &a, int v1, int v2, int cs[4], int vs[4])
{
    int c1 = a.vcn[3 * v1], c2 = a.vcn[3 * v1 + 1], c3 = a.vcn[3 * v1 + 2];
    for (int f = 0; f < 3; ++f) {
        int t = a.vcn[3 * v2 + f];
        if (t != c1 && t != c2 && t != c3) cs[3] = t;
    }
    int cells[3] = {c1, c2, c3};
    for (int q = 0; q < 3; ++q) {
        int c = cells[q], l, cur, nx;
        find_in_cell_d(a.cv + (size_t)c * a.vmax, a.cvn[c], v1, l, cur, nx);
        if (l == v2) cs[0] = c;
        else if (nx == v2) cs[2] = c;
        else cs[1] = c;
    }
    int l, cur, nx;
    find_in_cell_d(a.cv + (size_t)cs[1] * a.vmax, a.cvn[cs[1]], v1, l, cur, nx);
    vs[0] = l;
    vs[1] = nx;
    find_in_cell_d(a.cv + (size_t)cs[3] * a.vmax, a.cvn[cs[3]], v2, l, cur, nx);
    vs[3] = l;
    vs[2] = nx;
}

// Start-of-sweep evaluation of the candidate edge `key` (read-only): vertex2, the cells of
// t1_sets_d (cs; vs is not formed) and the decision (0: rejected, 1: evaluate at its turn). The data
// are loaded in two batches instead of one dependent load per row entry: vn, the position and vcn of
// vertex1; then vertex2's position and vcn with the sizes and first eight entries of vertex1's three
// cell rows. The walk of find_in_cell_d then runs on registers in its own order (entry n-1 first,
// then 0, 1, ...), so the result is the same; rows longer than eight entries or shorter than three
// take the walk on global memory.
constexpr int T1_ROW_FAST = 8;
CG_D unsigned char t1_start_eval(const VertArgs &a, const Inst &in, int key, int &vertex2, int cs[4])
{
    const int v1 = key / 3;
    const int v2 = a.vn[3 * v1 + key % 3];
    vertex2 = v2;
    const double2 p1 = a.vpos[v1];
    int c3v1[3], c3v2[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) c3v1[f] = a.vcn[3 * v1 + f];
    if (!(v1 < v2)) return 0;
    const double2 p2 = a.vpos[v2];
#pragma unroll
    for (int f = 0; f < 3; ++f) c3v2[f] = a.vcn[3 * v2 + f];
    int n[3], r[3][T1_ROW_FAST];
    const int lim = a.vmax < T1_ROW_FAST ? a.vmax : T1_ROW_FAST;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const int *row = a.cv + (size_t)c3v1[q] * a.vmax;
        n[q] = a.cvn[c3v1[q]];
#pragma unroll
        for (int k = 0; k < T1_ROW_FAST; ++k) r[q][k] = k < lim ? row[k] : -1;
    }
    const double2 e = min_dist(p1, p2, in.Lx, in.Ly);
    if (!(__dsqrt_rn(__dadd_rn(__dmul_rn(e.x, e.x), __dmul_rn(e.y, e.y))) < a.t1)) return 0;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        const int t = c3v2[f];
        if (t != c3v1[0] && t != c3v1[1] && t != c3v1[2]) cs[3] = t;
    }
    int n0 = 0, n2 = 0;  // sizes of cs[0] and cs[2]
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const int c = c3v1[q], nq = n[q];
        int l, cur, nx;
        if (nq < 3 || nq > lim) {
            find_in_cell_d(a.cv + (size_t)c * a.vmax, nq, v1, l, cur, nx);
        } else {
            l = r[q][0];
            cur = r[q][0];
#pragma unroll
            for (int k = 1; k < T1_ROW_FAST; ++k) {
                if (k == nq - 2) l = r[q][k];
                if (k == nq - 1) cur = r[q][k];
            }
            nx = r[q][0];
            bool done = false;
#pragma unroll
            for (int cn = 0; cn < T1_ROW_FAST; ++cn) {
                if (!done && cn < nq) {
                    nx = r[q][cn];
                    if (cur == v1) {
                        done = true;
                    } else {
                        l = cur;
                        cur = nx;
                    }
                }
            }
        }
        if (l == v2) {
            cs[0] = c;
            n0 = nq;
        } else if (nx == v2) {
            cs[2] = c;
            n2 = nq;
        } else {
            cs[1] = c;
        }
    }
    return (n0 == 3 || n2 == 3) ? 0 : 1;
}

CG_D void row_remove(int *row, int &n, int v)
{
    int cidx = 0;
    for (int cc = 0; cc < n - 1; ++cc) {
        if (row[cc] == v) cidx += 1;
        row[cc] = row[cidx];
        cidx += 1;
    }
    n -= 1;
}

// insert w right after v
CG_D void row_insert_after(int *row, int &n, int v, int w)
{
    int k = 0;
    while (k < n && row[k] != v) ++k;
    for (int t = n; t > k + 1; --t) row[t] = row[t - 1];
    row[k + 1] = w;
    n += 1;
}

// Keys queued by flips ahead of the sweep: a binary min-heap h[0, n), kept by one thread. A key may
// be queued more than once; the sweep visits it once (it pops every copy together). Push and pop
// cost O(log n), where inserting into a sorted run moved every pending key above the new one.
CG_D void heap_push(int *h, int &n, int key)
{
    int i = n++;
    while (i > 0) {
        const int p = (i - 1) >> 1;
        const int hp = h[p];
        if (hp <= key) break;
        h[i] = hp;
        i = p;
    }
    h[i] = key;
}

CG_D int heap_pop(int *h, int &n)
{
    const int top = h[0];
    const int last = h[--n];
    int i = 0;
    while (true) {
        const int l = 2 * i + 1;
        if (l >= n) break;
        const int r = l + 1;
        const int c = (r < n && h[r] < h[l]) ? r : l;
        const int hc = h[c];
        if (last <= hc) break;
        h[i] = hc;
        i = c;
    }
    if (n > 0) h[i] = last;
    return top;
}

// the smallest key and all its copies
CG_D int heap_pop_unique(int *h, int &n)
{
    const int k = heap_pop(h, n);
    while (n > 0 && h[0] == k) heap_pop(h, n);
    return k;
}

// the heap's keys in ascending order, in place
CG_D void heap_sort_ascending(int *h, int n)
{
    for (int m = n; m > 1;) {
        const int k = heap_pop(h, m);
        h[m] = k;
    }
    for (int i = 0, j = n - 1; i < j; ++i, --j) {
        const int t = h[i];
        h[i] = h[j];
        h[j] = t;
    }
}

// One step of the sweep at edge key = 3*vertex1 + slot, on the current state (the body of the
// CPU sweep, src/models/vertexModelBase.cpp:653-787): 0 no flip, 1 flipped (cs, vs and vertex2
// filled), -1 a cell row would exceed vmax.
CG_D int t1_try_global(const VertArgs &a, const Inst &in, int key, int cs[4], int vs[4], int &vertex2)
{
    int vertex1 = key / 3, vv = key % 3;
    vertex2 = a.vn[3 * vertex1 + vv];
    if (!(vertex1 < vertex2)) return 0;
    double2 v1 = a.vpos[vertex1], v2 = a.vpos[vertex2];
    double2 e = min_dist(v1, v2, in.Lx, in.Ly);
    if (!(__dsqrt_rn(__dadd_rn(__dmul_rn(e.x, e.x), __dmul_rn(e.y, e.y))) < a.t1)) return 0;
    t1_sets_d(a, vertex1, vertex2, cs, vs);
    if (a.cvn[cs[0]] == 3 || a.cvn[cs[2]] == 3) return 0;
    if (a.cvn[cs[1]] + 1 > a.vmax || a.cvn[cs[3]] + 1 > a.vmax) return -1;
    // rotate the edge by 90 degrees about its midpoint
    double2 mid = make_double2(__dadd_rn(v2.x, __dmul_rn(0.5, e.x)), __dadd_rn(v2.y, __dmul_rn(0.5, e.y)));
    v1 = make_double2(__dsub_rn(mid.x, e.y), __dadd_rn(mid.y, e.x));
    v2 = make_double2(__dadd_rn(mid.x, e.y), __dsub_rn(mid.y, e.x));
    a.vpos[vertex1] = put_in_box(v1, in.Lx, in.Ly, in.iLx, in.iLy);
    a.vpos[vertex2] = put_in_box(v2, in.Lx, in.Ly, in.iLx, in.iLy);
    for (int vert = 0; vert < 3; ++vert) {
        if (a.vcn[3 * vertex1 + vert] == cs[2]) a.vcn[3 * vertex1 + vert] = cs[3];
        if (a.vcn[3 * vertex2 + vert] == cs[0]) a.vcn[3 * vertex2 + vert] = cs[1];
        if (a.vn[3 * vs[1] + vert] == vertex1) a.vn[3 * vs[1] + vert] = vertex2;
        if (a.vn[3 * vs[2] + vert] == vertex2) a.vn[3 * vs[2] + vert] = vertex1;
        if (a.vn[3 * vertex1 + vert] == vs[1]) a.vn[3 * vertex1 + vert] = vs[2];
        if (a.vn[3 * vertex2 + vert] == vs[2]) a.vn[3 * vertex2 + vert] = vs[1];
    }
    int *ri = a.cv + (size_t)cs[0] * a.vmax;
    row_remove(ri, a.cvn[cs[0]], vertex2);
    int *rj = a.cv + (size_t)cs[1] * a.vmax;
    row_insert_after(rj, a.cvn[cs[1]], vertex1, vertex2);
    int *rk = a.cv + (size_t)cs[2] * a.vmax;
    row_remove(rk, a.cvn[cs[2]], vertex1);
    int *rl = a.cv + (size_t)cs[3] * a.vmax;
    row_insert_after(rl, a.cvn[cs[3]], vertex2, vertex1);
    return 1;
}

// row walk of find_in_cell_d on a local copy of a cell's row
CG_D void find_in_row(const int *row, int cneigh, int target, int &vlast, int &vcur, int &vnext)
{
    int l = row[cneigh - 2], c = row[cneigh - 1], nx = row[0];
    for (int cn = 0; cn < cneigh; ++cn) {
        nx = row[cn];
        if (c == target) break;
        l = c;
        c = nx;
    }
    vlast = l;
    vcur = c;
    vnext = nx;
}

constexpr int T1_ROW_LOCAL = 32;  // cell rows up to this length are staged in local copies

// The same step as t1_try_global with the data it reads loaded in a few independent batches
// (the four cell rows and sizes at once, the four vertex rows at once) and the edits applied to
// local copies in the same order before being written back, so one sweeping thread waits for
// memory a handful of times per flip instead of once per access. Falls back to t1_try_global
// (before writing anything) when rows are longer than T1_ROW_LOCAL or the cells / vertices of
// the flip are not all distinct (where in-place edits of one row would be seen by the next).
CG_D int t1_try(const VertArgs &a, const Inst &in, int key, int cs[4], int vs[4], int &vertex2)
{
    if (a.vmax > T1_ROW_LOCAL) return t1_try_global(a, in, key, cs, vs, vertex2);
    const int vertex1 = key / 3, vv = key % 3;
    vertex2 = a.vn[3 * vertex1 + vv];
    if (!(vertex1 < vertex2)) return 0;
    double2 p1 = a.vpos[vertex1], p2 = a.vpos[vertex2];
    int c3v1[3], c3v2[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        c3v1[f] = a.vcn[3 * vertex1 + f];
        c3v2[f] = a.vcn[3 * vertex2 + f];
    }
    double2 e = min_dist(p1, p2, in.Lx, in.Ly);
    if (!(__dsqrt_rn(__dadd_rn(__dmul_rn(e.x, e.x), __dmul_rn(e.y, e.y))) < a.t1)) return 0;
    // cs[3]: the cell of vertex2 that vertex1 does not touch (left as given if there is none)
    int c4 = cs[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        int t = c3v2[f];
        if (t != c3v1[0] && t != c3v1[1] && t != c3v1[2]) c4 = t;
    }
    const int cid[4] = {c3v1[0], c3v1[1], c3v1[2], c4};
    int R[4][T1_ROW_LOCAL];
    int nr[4];
    // all four rows in flight at once (fully unrolled, predicated on vmax)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        nr[q] = a.cvn[cid[q]];
        const int *src = a.cv + (size_t)cid[q] * a.vmax;
#pragma unroll
        for (int k = 0; k < T1_ROW_LOCAL; ++k) R[q][k] = k < a.vmax ? src[k] : 0;
    }
    // classify vertex1's cells by the neighbours of vertex1 in their rows (t1_sets_d)
    int i0 = -1, i1 = -1, i2 = -1;
    for (int q = 0; q < 3; ++q) {
        int l, cur, nx;
        find_in_row(R[q], nr[q], vertex1, l, cur, nx);
        if (l == vertex2) i0 = q;
        else if (nx == vertex2) i2 = q;
        else i1 = q;
    }
    if (i0 < 0 || i1 < 0 || i2 < 0 || c4 == cid[0] || c4 == cid[1] || c4 == cid[2] || cid[0] == cid[1] ||
        cid[0] == cid[2] || cid[1] == cid[2])
        return t1_try_global(a, in, key, cs, vs, vertex2);
    cs[0] = cid[i0];
    cs[1] = cid[i1];
    cs[2] = cid[i2];
    cs[3] = c4;
    {
        int l, cur, nx;
        find_in_row(R[i1], nr[i1], vertex1, l, cur, nx);
        vs[0] = l;
        vs[1] = nx;
        find_in_row(R[3], nr[3], vertex2, l, cur, nx);
        vs[3] = l;
        vs[2] = nx;
    }
    if (nr[i0] == 3 || nr[i2] == 3) return 0;
    if (nr[i1] + 1 > a.vmax || nr[3] + 1 > a.vmax) return -1;
    const int vx[4] = {vertex1, vertex2, vs[1], vs[2]};
    if (vs[1] == vs[2] || vs[1] == vertex1 || vs[1] == vertex2 || vs[2] == vertex1 || vs[2] == vertex2)
        return t1_try_global(a, in, key, cs, vs, vertex2);
    int VN[4][3];
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int f = 0; f < 3; ++f) VN[t][f] = a.vn[3 * vx[t] + f];
    // rotate the edge by 90 degrees about its midpoint
    double2 mid = make_double2(__dadd_rn(p2.x, __dmul_rn(0.5, e.x)), __dadd_rn(p2.y, __dmul_rn(0.5, e.y)));
    double2 n1 = make_double2(__dsub_rn(mid.x, e.y), __dadd_rn(mid.y, e.x));
    double2 n2 = make_double2(__dadd_rn(mid.x, e.y), __dsub_rn(mid.y, e.x));
    a.vpos[vertex1] = put_in_box(n1, in.Lx, in.Ly, in.iLx, in.iLy);
    a.vpos[vertex2] = put_in_box(n2, in.Lx, in.Ly, in.iLx, in.iLy);
    // rewiring, in the order of the CPU sweep (rows are distinct here)
#pragma unroll
    for (int vert = 0; vert < 3; ++vert) {
        if (c3v1[vert] == cs[2]) c3v1[vert] = cs[3];
        if (c3v2[vert] == cs[0]) c3v2[vert] = cs[1];
        if (VN[2][vert] == vertex1) VN[2][vert] = vertex2;
        if (VN[3][vert] == vertex2) VN[3][vert] = vertex1;
        if (VN[0][vert] == vs[1]) VN[0][vert] = vs[2];
        if (VN[1][vert] == vs[2]) VN[1][vert] = vs[1];
    }
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        a.vcn[3 * vertex1 + f] = c3v1[f];
        a.vcn[3 * vertex2 + f] = c3v2[f];
    }
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int f = 0; f < 3; ++f) a.vn[3 * vx[t] + f] = VN[t][f];
    row_remove(R[i0], nr[i0], vertex2);
    row_insert_after(R[i1], nr[i1], vertex1, vertex2);
    row_remove(R[i2], nr[i2], vertex1);
    row_insert_after(R[3], nr[3], vertex2, vertex1);
    const int qi[4] = {i0, i1, i2, 3};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        int q = qi[t];
        int *dst = a.cv + (size_t)cid[q] * a.vmax;
        for (int k = 0; k < nr[q]; ++k) dst[k] = R[q][k];
        a.cvn[cid[q]] = nr[q];
    }
    return 1;
}

// after a flip at `key`: queue the edges that moved or were rewired (those of vertex1, vertex2,
// vs[1], vs[2]) ahead of the sweep position, into the pending part q[head, n) of an ascending queue.
// Only edges shorter than the threshold are queued: a longer edge can become short only when one of
// its ends moves, and the flip that moves it queues it again. The rows and positions are loaded
// up front so the single sweeping thread waits for memory once, not once per edge.
CG_D void t1_requeue(const VertArgs &a, const Inst &in, int key, int vertex2, const int vs[4], int *h, int &hn,
                     int hcap, bool &overflow)
{
    const int u4[4] = {key / 3, vertex2, vs[1], vs[2]};
    int w12[12];
    double2 pu[4], pw[12];
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int s = 0; s < 3; ++s) w12[3 * t + s] = a.vn[3 * u4[t] + s];
#pragma unroll
    for (int t = 0; t < 4; ++t) pu[t] = a.vpos[u4[t]];
#pragma unroll
    for (int i = 0; i < 12; ++i) pw[i] = a.vpos[w12[i]];
    for (int t = 0; t < 4; ++t) {
        const int u = u4[t];
        for (int s = 0; s < 3; ++s) {
            const int w = w12[3 * t + s];
            // the length exactly as the sweep computes it (from the smaller index to the larger)
            double2 e = u < w ? min_dist(pu[t], pw[3 * t + s], in.Lx, in.Ly)
                              : min_dist(pw[3 * t + s], pu[t], in.Lx, in.Ly);
            if (!(__dsqrt_rn(__dadd_rn(__dmul_rn(e.x, e.x), __dmul_rn(e.y, e.y))) < a.t1)) continue;
            int k2;
            if (u < w) {
                k2 = 3 * u + s;
            } else {
                int sw = 0;
                while (sw < 3 && a.vn[3 * w + sw] != u) ++sw;
                if (sw == 3) continue;
                k2 = 3 * w + sw;
            }
            if (k2 > key) {
                if (hn >= hcap) overflow = true;
                else heap_push(h, hn, k2);
            }
        }
    }
}

// the whole sweep by one thread over the candidate keys q[0, nc) (sorted here), the keys queued by
// flips in a min-heap at q[nc, 3 nv); used when the candidates do not fit the shared-memory path,
// and to resume an interrupted sweep. A flip that would overflow a cell row stops it before changing
// anything; the keys still to visit are then left in q as two ascending runs, the candidates (A) and
// the queued keys (B), with the interrupted key first in its run, and resume = {|A|, |B|}, so the
// sweep can continue once the rows have grown (the reference grows cellVertices at that point,
// src/models/vertexModelBase.cpp:474-500)
CG_D void t1_sweep_serial(const VertArgs &a, const Inst &in, int *q, int nc, int &flips, int &status,
                          int *resume)
{
    const int cap = 3 * in.nv;
    for (int i = 1; i < nc; ++i) {
        int key = q[i], j = i - 1;
        while (j >= 0 && q[j] > key) {
            q[j + 1] = q[j];
            --j;
        }
        q[j + 1] = key;
    }
    int *h = q + nc;
    const int hcap = cap - nc;
    int hm = 0, hn = 0;
    bool overflow = false;
    while (hm < nc || hn > 0) {
        int key;
        bool queued = false;
        if (hn > 0 && (hm >= nc || h[0] <= q[hm])) {
            key = heap_pop_unique(h, hn);
            if (hm < nc && q[hm] == key) ++hm;  // also a candidate: visited once
            queued = true;
        } else {
            key = q[hm++];
        }
        int cs[4] = {0, 0, 0, 0}, vs[4] = {0, 0, 0, 0}, vertex2 = 0;
        int r = t1_try(a, in, key, cs, vs, vertex2);
        if (r < 0) {
            // forward copies never overtake their sources: A moves down from q[hm - 1, nc), and a key
            // was queued only after a candidate was visited (hm >= 1), so B starts below q + nc
            int na = 0, nb = 0;
            if (!queued) q[na++] = key;
            for (int t = hm; t < nc; ++t) q[na++] = q[t];
            heap_sort_ascending(h, hn);
            if (queued) q[na + nb++] = key;
            for (int t = 0; t < hn; ++t) q[na + nb++] = h[t];
            if (resume) {
                resume[0] = na;
                resume[1] = nb;
            }
            status = CG_ERR_CAPACITY;
            return;
        }
        if (r == 0) continue;
        ++flips;
        t1_requeue(a, in, key, vertex2, vs, h, hn, hcap, overflow);
        if (overflow) {
            status = CG_ERR_CAPACITY;
            return;
        }
    }
}

// Shared-memory sweep state (dynamic shared memory; T1_CAP candidates at most)
constexpr int T1_CAP = 4096;
constexpr int T1_HASH = 4096;        // touched set as a hash: vertices and cells of larger instances
constexpr int T1_BITS = 1 << 19;     // touched set as a bitmap: instances whose ids fit (64 KB)
constexpr int T1_TOUCH_INTS = T1_BITS / 32 > T1_HASH ? T1_BITS / 32 : T1_HASH;
constexpr int T1_EXQ = 2048;         // keys queued by flips, in shared memory until they outgrow it
constexpr size_t T1_SMEM =
    (size_t)T1_CAP * (sizeof(int4) + 2 * sizeof(int) + 1) + (size_t)(T1_TOUCH_INTS + T1_EXQ) * sizeof(int);

CG_D unsigned t1_hash_slot(int id) { return ((unsigned)id * 2654435761u) >> 20; }  // 12 bits

CG_D bool t1_touched(const int *h, int id)
{
    unsigned sl = t1_hash_slot(id);
    for (int p = 0; p < T1_HASH; ++p) {
        int v = h[sl];
        if (v == id) return true;
        if (v < 0) return false;
        sl = (sl + 1) & (T1_HASH - 1);
    }
    return false;
}

// ---- warp-cooperative sweep helpers: a cell row is held one entry per lane (lane k: entry k) ----
constexpr unsigned T1_FULL = 0xffffffffu;

// position of the single occurrence of target among the first n entries, or -1 when it does not
// occur exactly once
CG_D int wrow_find(int rk, int n, int target, int lane)
{
    unsigned m = __ballot_sync(T1_FULL, lane < n && rk == target);
    return __popc(m) == 1 ? __ffs(m) - 1 : -1;
}

// returns false once the table is 3/4 full (the caller then stops trusting start-of-sweep results)
CG_D bool t1_touch_atomic(int *h, int id, int *count)
{
    unsigned sl = t1_hash_slot(id);
    for (int p = 0; p < T1_HASH; ++p) {
        int prev = atomicCAS(&h[sl], -1, id);
        if (prev == -1) return atomicAdd(count, 1) + 1 < (3 * T1_HASH) / 4;
        if (prev == id) return true;
        sl = (sl + 1) & (T1_HASH - 1);
    }
    return false;
}

// The sweep's touched set: the vertices (id 2 (v - voff)) and cells (id 2 (c - off) + 1) that its
// flips have written. Where the instance's ids fit T1_BITS it is an exact bitmap, so the
// start-of-sweep rejections stay usable for the whole sweep; otherwise the hash above. It is
// cleared when the sweep's first flip is made (nothing is touched before).
struct T1Touched {
    int *h;
    int *count;
    bool bits;
    int words;  // ints to clear
    CG_D bool has(int id) const
    {
        if (bits) return ((reinterpret_cast<const unsigned *>(h)[id >> 5] >> (id & 31)) & 1u) != 0;
        return t1_touched(h, id);
    }
    CG_D bool add(int id) const
    {
        if (bits) {
            atomicOr(reinterpret_cast<unsigned *>(h) + (id >> 5), 1u << (id & 31));
            return true;
        }
        return t1_touch_atomic(h, id, count);
    }
    CG_D void clear(int lane) const  // whole warp
    {
        const int fill = bits ? 0 : -1;
        for (int i = lane; i < words; i += 32) h[i] = fill;
        if (lane == 0) *count = 0;
        __syncwarp();
    }
};

// whether a flip of this sweep touched the data that candidate key's start-of-sweep evaluation read
CG_D bool t1_cand_touched(const T1Touched &T, const Inst &in, int key, int v2, int4 c4)
{
    if (T.has(2 * (key / 3 - in.voff)) || T.has(2 * (v2 - in.voff))) return true;
    if (c4.x < 0) return false;
    const int c[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (c[k] >= 0 && T.has(2 * (c[k] - in.off) + 1)) return true;
    return false;
}

// t1_try for a whole warp (every lane calls it; the result, cs, vs and vertex2 are the same in every
// lane). The four cell rows are loaded one entry per lane, found, cut and extended with ballots and
// shuffles, and written back by the lanes. Returns 2, before writing anything, where rows are not
// in the form that single-occurrence edits reproduce exactly (a target missing or repeated,
// cells or vertices of the flip not distinct, rows shorter than 3); the caller then runs
// t1_try_global in one lane. Needs vmax <= 32.
CG_D int t1_try_warp(const VertArgs &a, const Inst &in, int key, int cs[4], int vs[4], int &vertex2, int lane)
{
    const int vertex1 = key / 3, vv = key % 3;
    vertex2 = a.vn[3 * vertex1 + vv];
    if (!(vertex1 < vertex2)) return 0;
    double2 p1 = a.vpos[vertex1], p2 = a.vpos[vertex2];
    int c3v1[3], c3v2[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        c3v1[f] = a.vcn[3 * vertex1 + f];
        c3v2[f] = a.vcn[3 * vertex2 + f];
    }
    double2 e = min_dist(p1, p2, in.Lx, in.Ly);
    if (!(__dsqrt_rn(__dadd_rn(__dmul_rn(e.x, e.x), __dmul_rn(e.y, e.y))) < a.t1)) return 0;
    int c4 = cs[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        int t = c3v2[f];
        if (t != c3v1[0] && t != c3v1[1] && t != c3v1[2]) c4 = t;
    }
    const int cid[4] = {c3v1[0], c3v1[1], c3v1[2], c4};
    int nr[4];
    int R0, R1, R2, R3;
#pragma unroll
    for (int q = 0; q < 4; ++q) nr[q] = a.cvn[cid[q]];
    R0 = lane < a.vmax ? a.cv[(size_t)cid[0] * a.vmax + lane] : 0;
    R1 = lane < a.vmax ? a.cv[(size_t)cid[1] * a.vmax + lane] : 0;
    R2 = lane < a.vmax ? a.cv[(size_t)cid[2] * a.vmax + lane] : 0;
    R3 = lane < a.vmax ? a.cv[(size_t)cid[3] * a.vmax + lane] : 0;
    auto getR = [&](int q) { return q == 0 ? R0 : q == 1 ? R1 : q == 2 ? R2 : R3; };
    auto setR = [&](int q, int v) {
        if (q == 0) R0 = v;
        else if (q == 1) R1 = v;
        else if (q == 2) R2 = v;
        else R3 = v;
    };
    if (nr[0] < 3 || nr[1] < 3 || nr[2] < 3 || nr[3] < 3) return 2;
    // vertex1's cells by the neighbours of vertex1 in their rows (t1_sets_d)
    int i0 = -1, i1 = -1, i2 = -1, pos1[3], lq[3], nq[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        int rq = getR(q);
        int p = wrow_find(rq, nr[q], vertex1, lane);
        pos1[q] = p;
        if (p < 0) return 2;
        lq[q] = __shfl_sync(T1_FULL, rq, p == 0 ? nr[q] - 1 : p - 1);
        nq[q] = __shfl_sync(T1_FULL, rq, p + 1 == nr[q] ? 0 : p + 1);
        if (lq[q] == vertex2) i0 = q;
        else if (nq[q] == vertex2) i2 = q;
        else i1 = q;
    }
    if (i0 < 0 || i1 < 0 || i2 < 0 || c4 == cid[0] || c4 == cid[1] || c4 == cid[2] || cid[0] == cid[1] ||
        cid[0] == cid[2] || cid[1] == cid[2])
        return 2;
    const int p3 = wrow_find(R3, nr[3], vertex2, lane);
    if (p3 < 0) return 2;
    cs[0] = cid[i0];
    cs[1] = cid[i1];
    cs[2] = cid[i2];
    cs[3] = c4;
    vs[0] = lq[i1];
    vs[1] = nq[i1];
    vs[3] = __shfl_sync(T1_FULL, R3, p3 == 0 ? nr[3] - 1 : p3 - 1);
    vs[2] = __shfl_sync(T1_FULL, R3, p3 + 1 == nr[3] ? 0 : p3 + 1);
    if (nr[i0] == 3 || nr[i2] == 3) return 0;
    if (nr[i1] + 1 > a.vmax || nr[3] + 1 > a.vmax) return -1;
    if (vs[1] == vs[2] || vs[1] == vertex1 || vs[1] == vertex2 || vs[2] == vertex1 || vs[2] == vertex2) return 2;
    const int pa = wrow_find(getR(i0), nr[i0], vertex2, lane);  // vertex2 leaves cs[0]
    if (pa < 0) return 2;
    const int pb = pos1[i1], pc = pos1[i2];                      // after vertex1 in cs[1]; vertex1 leaves cs[2]
    // ---- no return below this line: the flip is written
    if (lane == 0) {
        double2 mid = make_double2(__dadd_rn(p2.x, __dmul_rn(0.5, e.x)), __dadd_rn(p2.y, __dmul_rn(0.5, e.y)));
        double2 n1 = make_double2(__dsub_rn(mid.x, e.y), __dadd_rn(mid.y, e.x));
        double2 n2 = make_double2(__dadd_rn(mid.x, e.y), __dsub_rn(mid.y, e.x));
        a.vpos[vertex1] = put_in_box(n1, in.Lx, in.Ly, in.iLx, in.iLy);
        a.vpos[vertex2] = put_in_box(n2, in.Lx, in.Ly, in.iLx, in.iLy);
    }
    // rewiring (rows distinct): vcn of vertex1 / vertex2, vn of vertex1, vertex2, vs[1], vs[2]
    if (lane < 3) {
        int c = c3v1[lane];
        a.vcn[3 * vertex1 + lane] = c == cs[2] ? cs[3] : c;
    } else if (lane < 6) {
        int c = c3v2[lane - 3];
        a.vcn[3 * vertex2 + lane - 3] = c == cs[0] ? cs[1] : c;
    }
    if (lane < 12) {
        const int t = lane / 3, f = lane % 3;
        const int x = t == 0 ? vertex1 : t == 1 ? vertex2 : t == 2 ? vs[1] : vs[2];
        int v = a.vn[3 * x + f];
        if (t == 0 && v == vs[1]) v = vs[2];
        else if (t == 1 && v == vs[2]) v = vs[1];
        else if (t == 2 && v == vertex1) v = vertex2;
        else if (t == 3 && v == vertex2) v = vertex1;
        a.vn[3 * x + f] = v;
    }
    // rows: the four edits of the CPU sweep (row_remove / row_insert_after on single occurrences)
    {
        int r = getR(i0), up = __shfl_down_sync(T1_FULL, r, 1);
        if (lane >= pa && lane < nr[i0] - 1) r = up;
        setR(i0, r);
        r = getR(i1);
        int prev = __shfl_up_sync(T1_FULL, r, 1);
        if (lane == pb + 1) r = vertex2;
        else if (lane > pb + 1 && lane <= nr[i1]) r = prev;
        setR(i1, r);
        r = getR(i2);
        up = __shfl_down_sync(T1_FULL, r, 1);
        if (lane >= pc && lane < nr[i2] - 1) r = up;
        setR(i2, r);
        prev = __shfl_up_sync(T1_FULL, R3, 1);
        if (lane == p3 + 1) R3 = vertex1;
        else if (lane > p3 + 1 && lane <= nr[3]) R3 = prev;
    }
    nr[i0] -= 1;
    nr[i1] += 1;
    nr[i2] -= 1;
    nr[3] += 1;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (lane < nr[q]) a.cv[(size_t)cid[q] * a.vmax + lane] = getR(q);
        if (lane == 0) a.cvn[cid[q]] = nr[q];
    }
    __syncwarp();
    return 1;
}

// t1_requeue for a whole warp: lanes 0-11 test one edge each, lane 0 queues the short ones
CG_D void t1_requeue_warp(const VertArgs &a, const Inst &in, int key, int vertex2, const int vs[4], int *q,
                          int &n, int cap, bool &overflow, int lane)
{
    int k2 = -1;
    if (lane < 12) {
        const int t = lane / 3, s = lane % 3;
        const int u = t == 0 ? key / 3 : t == 1 ? vertex2 : t == 2 ? vs[1] : vs[2];
        const int w = a.vn[3 * u + s];
        double2 pu = a.vpos[u], pw = a.vpos[w];
        double2 e = u < w ? min_dist(pu, pw, in.Lx, in.Ly) : min_dist(pw, pu, in.Lx, in.Ly);
        if (__dsqrt_rn(__dadd_rn(__dmul_rn(e.x, e.x), __dmul_rn(e.y, e.y))) < a.t1) {
            if (u < w) {
                k2 = 3 * u + s;
            } else {
                int sw = 0;
                while (sw < 3 && a.vn[3 * w + sw] != u) ++sw;
                if (sw < 3) k2 = 3 * w + sw;
            }
            if (k2 <= key) k2 = -1;
        }
    }
    unsigned m = __ballot_sync(T1_FULL, k2 >= 0);
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        const int kk = __shfl_sync(T1_FULL, k2, src);
        if (lane == 0) {
            if (n >= cap) overflow = true;
            else heap_push(q, n, kk);
        }
    }
    n = __shfl_sync(T1_FULL, n, 0);
    overflow = __shfl_sync(T1_FULL, (int)overflow, 0) != 0;
    __syncwarp();
}

// One block per instance. The candidates are sorted in parallel (bitonic, shared memory) and
// evaluated in parallel on the state at the start of the sweep; then warp 0 replays the sweep in
// ascending key order. A candidate rejected at the start stays rejected unless an earlier flip of
// this sweep touched one of its endpoints (positions, vn, vcn) or one of the four cells around it
// (rows, sizes), which are exactly the data the test reads; such candidates, and every candidate
// that was not rejected, are evaluated on the current state as the CPU sweep does. Touched-ness
// changes only at flips, so the warp decides the skips of 32 consecutive candidates at once, up to
// the first one it must evaluate or the next key queued by a flip.
__global__ void __launch_bounds__(256) k_vm_t1_replay(VertArgs a)
{
    extern __shared__ __align__(16) unsigned char t1_smem[];
    int4 *s_cs = reinterpret_cast<int4 *>(t1_smem);
    int *s_key = reinterpret_cast<int *>(s_cs + T1_CAP);
    int *s_v2 = s_key + T1_CAP;
    int *s_hash = s_v2 + T1_CAP;
    int *s_exq = s_hash + T1_TOUCH_INTS;
    unsigned char *s_dec = reinterpret_cast<unsigned char *>(s_exq + T1_EXQ);
    __shared__ int s_tn;  // entries of the touched set
    const int inst = blockIdx.x;
    Ctl *ctl = a.ctl;
    if (ctl && ctl->halt) return;  // uniform
    const int nc = a.cand_count[inst];
    __syncthreads();
    if (threadIdx.x == 0) a.cand_count[inst] = 0;
    if (nc == 0) return;
    const Inst &in = a.inst[inst];
    int *q = a.cand + 3 * (size_t)in.voff;
    int flips = 0, status = 0;
    if (nc > T1_CAP) {
        if (threadIdx.x == 0)
            t1_sweep_serial(a, in, q, nc, flips, status, a.t1_resume ? a.t1_resume + 2 * inst : nullptr);
    } else {
        // up to 32 candidates (the steady state): warp 0 alone sorts, evaluates and sweeps, with
        // warp barriers instead of block barriers; the other warps leave now
        const bool fast = nc <= 32;
        if (fast && threadIdx.x >= 32) return;
        const int nthr = fast ? 32 : blockDim.x;
        auto bsync = [fast]() {
            if (fast) __syncwarp();
            else __syncthreads();  // uniform across the block
        };
        int P = 1;
        while (P < nc) P <<= 1;
        for (int i = threadIdx.x; i < P; i += nthr) s_key[i] = i < nc ? q[i] : 0x7fffffff;
        bsync();
        for (int k = 2; k <= P; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < P; i += nthr) {
                    int ixj = i ^ j;
                    if (ixj > i) {
                        int x = s_key[i], y = s_key[ixj];
                        bool up = (i & k) == 0;
                        if ((x > y) == up) {
                            s_key[i] = y;
                            s_key[ixj] = x;
                        }
                    }
                }
                bsync();
            }
        }
        // start-of-sweep evaluation (read-only)
        for (int i = threadIdx.x; i < nc; i += nthr) {
            int v2, cs[4] = {-1, -1, -1, -1};
            const unsigned char dec = t1_start_eval(a, in, s_key[i], v2, cs);
            s_v2[i] = v2;
            s_cs[i] = make_int4(cs[0], cs[1], cs[2], cs[3]);
            s_dec[i] = dec;
        }
        bsync();
        if (threadIdx.x < 32) {
            // sweep by warp 0, all lanes in step: the sorted candidates merged with the keys queued
            // by flips (a min-heap popped by lane 0), kept in shared memory and moved to q[nc, 3 nv)
            // if they outgrow it
            const int lane = threadIdx.x;
            const bool warp_rows = a.vmax <= 32;
            const int nbits = 2 * max(in.nv, in.n);
            T1Touched T;
            T.h = s_hash;
            T.count = &s_tn;
            T.bits = nbits <= T1_BITS;
            T.words = T.bits ? (nbits + 31) / 32 : T1_HASH;
            bool touched_any = false;  // no flip yet: nothing touched, the set not yet cleared
            int *ex = s_exq;
            int ecap = T1_EXQ;
            const int gcap = 3 * in.nv - nc;
            int hm = 0, en = 0;
            bool trust = true, overflow = false;
            while (hm < nc || en > 0) {
                int key;
                int idx = -1;
                if (en > 0 && (hm >= nc || ex[0] <= s_key[hm])) {
                    int k = 0;
                    if (lane == 0) k = heap_pop_unique(ex, en);
                    key = __shfl_sync(T1_FULL, k, 0);
                    en = __shfl_sync(T1_FULL, en, 0);
                    __syncwarp();
                    if (hm < nc && s_key[hm] == key) ++hm;  // queued again by a flip: evaluate once
                } else {
                    if (trust) {
                        // skip the candidates rejected at the start and untouched since, up to the
                        // next queued key
                        const int bound = en > 0 ? ex[0] : 0x7fffffff;
                        unsigned stop;
                        while (true) {
                            const int i = hm + lane;
                            bool st = true;
                            if (i < nc && s_key[i] < bound && s_dec[i] == 0)
                                st = touched_any && t1_cand_touched(T, in, s_key[i], s_v2[i], s_cs[i]);
                            stop = __ballot_sync(T1_FULL, st);
                            if (stop) break;
                            hm += 32;
                        }
                        hm += __ffs(stop) - 1;
                        if (hm >= nc || (en > 0 && ex[0] <= s_key[hm])) continue;  // end of the list or a queued key
                    }
                    idx = hm++;
                    key = s_key[idx];
                }
                int cs[4] = {0, 0, 0, 0}, vs[4] = {0, 0, 0, 0}, vertex2 = 0;
                int r = warp_rows ? t1_try_warp(a, in, key, cs, vs, vertex2, lane) : 2;
                if (r == 2) {  // exact in-place edits by one lane
                    int rr = 0;
                    if (lane == 0) rr = t1_try_global(a, in, key, cs, vs, vertex2);
                    r = __shfl_sync(T1_FULL, rr, 0);
#pragma unroll
                    for (int t = 0; t < 4; ++t) {
                        cs[t] = __shfl_sync(T1_FULL, cs[t], 0);
                        vs[t] = __shfl_sync(T1_FULL, vs[t], 0);
                    }
                    vertex2 = __shfl_sync(T1_FULL, vertex2, 0);
                    __syncwarp();
                }
                if (r < 0) {
                    // a cell row would overflow: keep the keys still to visit for a resumed sweep
                    // once the rows have grown -- the sorted candidates from this one on (A), then
                    // the keys queued by flips, sorted (B); a key was queued only after a candidate
                    // was visited (hm >= 1), so B's forward copy from q[nc, ...) never overtakes
                    // its source
                    if (lane == 0 && a.t1_resume) {
                        const bool from_ex = idx < 0;
                        int na = 0, nb = 0;
                        for (int t = from_ex ? hm : hm - 1; t < nc; ++t) q[na++] = s_key[t];
                        heap_sort_ascending(ex, en);
                        if (from_ex) q[na + nb++] = key;
                        for (int t = 0; t < en; ++t) q[na + nb++] = ex[t];
                        a.t1_resume[2 * inst] = na;
                        a.t1_resume[2 * inst + 1] = nb;
                    }
                    status = CG_ERR_CAPACITY;
                    break;
                }
                if (r == 0) continue;
                ++flips;
                if (!touched_any) {
                    T.clear(lane);
                    touched_any = true;
                }
                int tid = -1;
                if (lane < 4) tid = 2 * ((lane == 0 ? key / 3 : lane == 1 ? vertex2 : lane == 2 ? vs[1] : vs[2]) - in.voff);
                else if (lane < 8) tid = 2 * (cs[lane - 4] - in.off) + 1;
                bool ok = tid < 0 || T.add(tid);
                if (!__all_sync(T1_FULL, ok)) trust = false;
                __syncwarp();
                if (ex == s_exq && en + 12 > ecap) {  // room for one flip's keys, else move to global
                    int *g = q + nc;
                    if (en + 12 > gcap) {
                        status = CG_ERR_CAPACITY;
                        break;
                    }
                    for (int t = lane; t < en; t += 32) g[t] = ex[t];  // a heap stays a heap
                    __syncwarp();
                    ex = g;
                    ecap = gcap;
                }
                t1_requeue_warp(a, in, key, vertex2, vs, ex, en, ecap, overflow, lane);
                if (overflow) {
                    status = CG_ERR_CAPACITY;
                    break;
                }
            }
        }
    }
    if (threadIdx.x == 0) {
        if (ctl) atomicAdd(&ctl->counters[5], (unsigned long long)flips);
        if (status && ctl) {
            atomicExch(&ctl->status, status);
            atomicExch(&ctl->halt, 1);
        }
    }
}

// Continue the sweeps that a row overflow interrupted, after the rows have grown: per instance with
// keys kept (t1_resume), one thread merges the two sorted runs (A then B, in cand) into one sorted
// list without repeats and runs the rest of the sweep on the current state, as the CPU sweep
// continues after growing its rows. Launched with T1_SMEM bytes of dynamic shared memory.
__global__ void k_vm_t1_resume(VertArgs a)
{
    extern __shared__ __align__(16) unsigned char t1_smem[];
    int *buf = reinterpret_cast<int *>(t1_smem);  // T1_SMEM / 4 >= 2 T1_CAP ints
    const int inst = blockIdx.x;
    if (threadIdx.x != 0) return;
    int *res = a.t1_resume + 2 * inst;
    const int na = res[0], nb = res[1];
    if (na + nb == 0) return;
    const Inst &in = a.inst[inst];
    int *q = a.cand + 3 * (size_t)in.voff;
    int flips = 0, status = 0;
    res[0] = res[1] = 0;
    if (na + nb > 2 * T1_CAP) {
        status = CG_ERR_CAPACITY;  // too many keys to merge here: the step fails as before
    } else {
        for (int t = 0; t < na + nb; ++t) buf[t] = q[t];
        int i = 0, j = na, m = 0;
        while (i < na || j < na + nb) {
            int k;
            if (j >= na + nb || (i < na && buf[i] <= buf[j])) k = buf[i++];
            else k = buf[j++];
            if (m == 0 || q[m - 1] != k) q[m++] = k;
        }
        t1_sweep_serial(a, in, q, m, flips, status, res);
    }
    if (a.ctl) {
        atomicAdd(&a.ctl->counters[5], (unsigned long long)flips);
        if (status) {
            atomicExch(&a.ctl->status, status);
            atomicExch(&a.ctl->halt, 1);
        }
    }
}

// ------------------------------------------------------------------------------------------
// vertex model from a Delaunay triangulation (vertexModelBase::setCellsVoronoiTesselation,
// src/models/vertexModelBase.cpp:115-229): one vertex per Delaunay triangle at its circumcentre.
// Triangles are numbered with their smallest cell as owner, in cell order then slot order; cell
// rows list their triangles counter-clockwise from (c, nbr[0], nbr[1]); vcn[3v+f] are the
// triangle's cells (owner first, counter-clockwise) and vn[3v+f] the triangle across from cell f.
// ------------------------------------------------------------------------------------------
struct DualArgs {
    int N, K, vmax;
    const Inst *inst;
    const int *cell_inst;
    const double2 *pos;
    const int *nn, *nbr;
    int *owned, *tri;  // owned[N] counts -> exclusive offsets; tri[N*K]
    double2 *vpos;
    int *vn, *vcn, *cvn, *cv;
    int *status;
};

__global__ void k_dual_count(DualArgs d)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.N) return;
    int z = d.nn[c], cnt = 0;
    for (int k = 0; k < z; ++k) {
        int a = d.nbr[(size_t)c * d.K + k], b = d.nbr[(size_t)c * d.K + (k + 1) % z];
        if (c < a && c < b) ++cnt;
    }
    d.owned[c] = cnt;
}

__global__ void k_dual_assign(DualArgs d)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.N) return;
    int z = d.nn[c], id = d.owned[c];  // exclusive offset after the scan
    for (int k = 0; k < z; ++k) {
        int a = d.nbr[(size_t)c * d.K + k], b = d.nbr[(size_t)c * d.K + (k + 1) % z];
        d.tri[(size_t)c * d.K + k] = (c < a && c < b) ? id++ : -1;
    }
}

CG_D int row_slot(const int *row, int z, int v)
{
    for (int k = 0; k < z; ++k)
        if (row[k] == v) return k;
    return -1;
}

__global__ void k_dual_resolve(DualArgs d)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.N) return;
    int z = d.nn[c];
    if (z > d.vmax) {
        atomicCAS(d.status, 0, CG_ERR_CAPACITY);
        return;
    }
    for (int k = 0; k < z; ++k) {
        int t = d.tri[(size_t)c * d.K + k];
        if (t < 0) {
            int a = d.nbr[(size_t)c * d.K + k], b = d.nbr[(size_t)c * d.K + (k + 1) % z];
            int o = a < b ? a : b, nxt = (o == a) ? b : c;
            int s = row_slot(d.nbr + (size_t)o * d.K, d.nn[o], nxt);
            if (s < 0) {
                atomicCAS(d.status, 0, CG_ERR_TOPOLOGY);
                return;
            }
            // the owner's entry is written by k_dual_assign only, so it is final here
            t = d.tri[(size_t)o * d.K + s];
        }
        d.cv[(size_t)c * d.vmax + k] = t;
    }
    d.cvn[c] = z;
}

__global__ void k_dual_vertices(DualArgs d)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.N) return;
    const Inst &in = d.inst[d.cell_inst[c]];
    int z = d.nn[c];
    for (int k = 0; k < z; ++k) {
        int a = d.nbr[(size_t)c * d.K + k], b = d.nbr[(size_t)c * d.K + (k + 1) % z];
        if (!(c < a && c < b)) continue;
        int v = d.tri[(size_t)c * d.K + k];
        double2 ra = min_dist(d.pos[a], d.pos[c], in.Lx, in.Ly), rb = min_dist(d.pos[b], d.pos[c], in.Lx, in.Ly);
        double an = ra.x * ra.x + ra.y * ra.y, bn = rb.x * rb.x + rb.y * rb.y;
        double den = 0.5 / (ra.x * rb.y - ra.y * rb.x);
        double2 q = make_double2(d.pos[c].x + den * (an * rb.y - ra.y * bn), d.pos[c].y + den * (ra.x * bn - an * rb.x));
        d.vpos[v] = put_in_box(q, in.Lx, in.Ly, in.iLx, in.iLy);
        int cells[3] = {c, a, b};
        for (int f = 0; f < 3; ++f) {
            d.vcn[3 * v + f] = cells[f];
            int qc = cells[(f + 1) % 3], rc = cells[(f + 2) % 3];
            int s = row_slot(d.nbr + (size_t)qc * d.K, d.nn[qc], rc);
            int zq = d.nn[qc];
            d.vn[3 * v + f] = d.cv[(size_t)qc * d.vmax + (s + zq - 1) % zq];
        }
    }
}

}  // namespace cg
