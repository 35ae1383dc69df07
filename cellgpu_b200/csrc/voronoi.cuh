// cellgpu_b200 -- Voronoi-model device state and kernel declarations.
#pragma once

#include "cg_common.cuh"

namespace cg {

constexpr int KMAX = 32;          // largest supported neighbour-row capacity
constexpr int R_MAX = 4;          // local repair rounds per step before escalating to a global rebuild
constexpr int CAND_LOCAL = 320;   // candidate slots per warp for the local (2-ring) star
constexpr int CAND_GLOBAL = 384;  // candidate slots per warp for the cell-list star

// launch shapes of the fused per-cell pass (warps per block, minimum resident blocks per SM for
// __launch_bounds__): shape 0 is the default, shape 1 the alternative the autotuner may pick;
// both cap registers at 64 per thread
#ifndef CG_FORCE_WPB
#define CG_FORCE_WPB 2
#endif
#ifndef CG_FORCE_MINB
#define CG_FORCE_MINB 16
#endif
#define CG_FORCE_WPB_ALT 4
#define CG_FORCE_MINB_ALT 8
// the fused pass loads a cell's first row entry (CG_FP_PRE_ROW) and its preferences
// (CG_FP_PRE_PREF) beside its position and row length, ahead of the geometry
#ifndef CG_FP_PRE_ROW
#define CG_FP_PRE_ROW 1
#endif
#ifndef CG_FP_PRE_PREF
#define CG_FP_PRE_PREF 1
#endif
// rows of at most 8 entries in all four cells of a warp take the pass's one-slot-per-lane form
#ifndef CG_FP_SMALL_PATH
#define CG_FP_SMALL_PATH 0
#endif

// device control block of one system
struct Ctl {
    int epoch;               // base claim epoch of the current step
    int halt;                // sticky: a step could not complete on the device
    int need_global;         // a global retriangulation is required
    int status;              // CG_* code explaining halt
    int n_flagged;           // cells flagged by the test of this step
    int n_undec;             // entries of VoroArgs::undec written by the test of this step
    int q_count[R_MAX + 1];  // per-round queue lengths
    int step;                // completed integrator steps since creation
    int round;               // current local-repair round of this step
    unsigned blocks_done;    // blocks of the current commit-and-check launch that have finished
    unsigned long long counters[8];  // 0 tests failed, 1 cells restarred, 2 rows changed, 3 rounds,
                                     // 4 global rebuilds, 5 T1 flips, 6 fire iterations,
                                     // 7 executed repair rounds (2 kernels each)
};

// everything a Voronoi kernel needs, passed by value
struct VoroArgs {
    int N, K, n_inst;
    Inst inst0;          // used when inst == nullptr (kernel callers on caller memory)
    const Inst *inst;
    const int *cell_inst;
    double2 *pos;
    double *theta;
    const double2 *motility;
    const double2 *APpref;
    double KA, KP;
    void *AP;       // double2 (FP64) or float2 (mixed)
    void *F;        // double2 (FP64) or float2 (mixed), accumulated with atomics
    unsigned long long *Ffix;  // null, or 2 x 4 words per cell: fixed-point sums of F (order-independent)
    int *nn, *nbr;
    int rows_padded;  // rows hold -1 past their length (system rows): a row can be read before its length
    int star_grid, commit_grid;  // blocks of the repair round's two launches (0: the defaults)
    // repair
    int *mark;
    int *queue;     // (R_MAX+1) * N
    int *stage_nn;  // N
    int *stage_nbr; // N * K
    int *qslot;     // 2 * N: queue slot of each cell claimed for a round, by round parity
    int4 *qhint;    // N: per slot of the first round's queue, the row edit of an edge flip, or 0
    int *nclaim;    // N: claims naming each cell for the first round of the current step
    int *held;      // N: 1 while a cell's contributions are held back (its own row failed the test)
    int *undec;     // N: slots (c * 16 + k) whose in-circle sign the filter left undecided, or null
    Ctl *ctl;
    // cell list
    int *bin_count, *bin_start, *bin_cells, *cell_bin, *cell_slot;
    double2 *bin_pos;
    int n_bins;
    // line tension (tension_mode 0 off, 1 one gamma for unlike types, 2 gamma matrix)
    int tension_mode, ntypes;
    double gamma;
    const int *ctype;
    const double *tmat;  // ntypes x ntypes, row = the cell's own type
    double *TE;          // per cell: sum over its unlike edges of gamma x length
};

// weight of the edge between a cell of type ta and a neighbour of type tb (Voronoi or vertex
// model arguments: both carry tension_mode, gamma, ntypes and tmat)
template <typename Args>
CG_D double tension_weight(const Args &a, int ta, int tb)
{
    if (ta == tb) return 0.0;
    return a.tension_mode == 1 ? a.gamma : a.tmat[ta * a.ntypes + tb];
}

}  // namespace cg
