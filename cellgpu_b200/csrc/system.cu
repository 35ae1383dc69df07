// cellgpu_b200 -- host side of the C ABI: kernel callers on caller memory, and the device-resident
// batched system (cg_system). Built as one translation unit with the kernel files.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "voronoi.cu"
#include "vertex.cu"
#include "fire.cu"

using namespace cg;

// ------------------------------------------------------------------------------------------
// errors
// ------------------------------------------------------------------------------------------
static thread_local std::string g_err;

static int set_err(int code, const char *msg)
{
    g_err = msg;
    return code;
}

#define CG_CUDA(call)                                                                           \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            g_err = std::string(#call) + ": " + cudaGetErrorString(e_);                         \
            return CG_ERR_CUDA;                                                                 \
        }                                                                                       \
    } while (0)

#define CG_TRY(call)                 \
    do {                             \
        int s_ = (call);             \
        if (s_ != CG_OK) return s_;  \
    } while (0)

extern "C" const char *cg_last_error_string(void) { return g_err.c_str(); }
extern "C" int cg_version(void) { return 100; }

static inline int nblk(int n, int b) { return (n + b - 1) / b; }

// integrate + move: two cells per thread; 128-thread blocks spread a 262144-cell pass over the 148
// SMs in about seven blocks each (its SPP step 118.7 -> 117.8 us against 256-thread blocks)
constexpr int SPP_BLOCK = 128;

// cells per block of the fused pass: two resident waves of blocks over the N cells (148 SMs x
// minb blocks each), in whole groups of cells. Against one group of cells per block this cut the
// force pass of a 262144-cell monolayer from 79.2 to 75.3 us (one wave: 75.6, four: 78.3) on the
// same B200.
static inline int cells_per_block(int N, int wpb, int minb)
{
    const int grp = wpb * GPW;
    const long long blocks = 148LL * minb * 2;
    int cpb = (int)((N + blocks - 1) / blocks);
    return std::max(grp, (cpb + grp - 1) / grp * grp);
}

// launch of the fused per-cell pass (groups of 8 lanes) in launch shape 0 or 1; rows of up to 16
// slots take the fast form, wider rows (K = 32) the form with four slots per lane; with forces,
// FIX = 1 is the form that sums them in fixed point (deterministic mode, VoroArgs::Ffix set)
template <typename R, bool SCATTER, bool TEST, int NS, int FIX>
static inline void launch_groups_ns(const VoroArgs &a, int N, cudaStream_t st, int shape)
{
    if (shape == 1) {
        int cpb = cells_per_block(N, CG_FORCE_WPB_ALT, CG_FORCE_MINB_ALT);
        k_voro_groups<R, SCATTER, TEST, CG_FORCE_WPB_ALT, CG_FORCE_MINB_ALT, NS, FIX>
            <<<nblk(N, cpb), CG_FORCE_WPB_ALT * 32, 0, st>>>(a, cpb);
    } else {
        int cpb = cells_per_block(N, CG_FORCE_WPB, CG_FORCE_MINB);
        k_voro_groups<R, SCATTER, TEST, CG_FORCE_WPB, CG_FORCE_MINB, NS, FIX>
            <<<nblk(N, cpb), CG_FORCE_WPB * 32, 0, st>>>(a, cpb);
    }
}

// the thread-per-cell form (launch shape 2): FP64 forces summed with atomics, no line tension,
// 16-slot padded rows; other systems run shape 0
// (blocks of 2 warps: a block's registers and shared memory are freed when its slower warp ends,
// which 4-warp blocks waited for longer; same occupancy, 48.1 against 48.5 us on a 262144-cell monolayer)
#ifndef CG_THREAD_TPB
#define CG_THREAD_TPB 64
#endif
#ifndef CG_THREAD_MINB
#define CG_THREAD_MINB 10
#endif
static inline bool thread_form_ok(const VoroArgs &a)
{
    return !a.Ffix && a.tension_mode == 0 && a.K == VG && a.rows_padded;
}

template <typename R, bool SCATTER, bool TEST>
static inline void launch_groups(const VoroArgs &a, int N, cudaStream_t st, int shape = 0)
{
    if constexpr (SCATTER && std::is_same<R, double>::value) {
        if (shape == 2 && thread_form_ok(a)) {
            k_voro_thread<TEST, CG_THREAD_TPB, CG_THREAD_MINB><<<nblk(N, CG_THREAD_TPB), CG_THREAD_TPB, 0, st>>>(a);
            return;
        }
    }
    if (shape == 2) shape = 0;
    if constexpr (SCATTER) {
        if (a.Ffix) {
            if (a.K > VG)
                launch_groups_ns<R, SCATTER, TEST, VG_MAX, 1>(a, N, st, shape);
            else
                launch_groups_ns<R, SCATTER, TEST, VG, 1>(a, N, st, shape);
            return;
        }
    }
    if (a.K > VG)
        launch_groups_ns<R, SCATTER, TEST, VG_MAX, 0>(a, N, st, shape);
    else
        launch_groups_ns<R, SCATTER, TEST, VG, 0>(a, N, st, shape);
}

static Inst make_inst(double Lx, double Ly, int off, int n, int bin_off, double bin_target)
{
    Inst in;
    memset(&in, 0, sizeof(in));
    in.Lx = Lx;
    in.Ly = Ly;
    in.iLx = 1.0 / Lx;
    in.iLy = 1.0 / Ly;
    in.off = off;
    in.n = n;
    in.bin_off = bin_off;
    in.nbx = std::max(1, (int)std::floor(Lx / bin_target));
    in.nby = std::max(1, (int)std::floor(Ly / bin_target));
    in.bsx = Lx / in.nbx;
    in.bsy = Ly / in.nby;
    return in;
}

static const double BIN_TARGET = 0.8;

// ------------------------------------------------------------------------------------------
// 1. kernel callers on caller-owned memory
// ------------------------------------------------------------------------------------------
static VoroArgs raw_args(const double *pos, const int *nn, const int *nbr, int K, int N, double Lx,
                         double Ly)
{
    VoroArgs a;
    memset(&a, 0, sizeof(a));
    a.N = N;
    a.K = K;
    a.n_inst = 1;
    a.inst0 = make_inst(Lx, Ly, 0, N, 0, BIN_TARGET);
    a.pos = (double2 *)pos;
    a.nn = (int *)nn;
    a.nbr = (int *)nbr;
    return a;
}

static int check_launch()
{
    CG_CUDA(cudaGetLastError());
    return CG_OK;
}

extern "C" int cg_voronoi_geometry(const double *pos, const int *nn, const int *nbr, int K, int N,
                                   double Lx, double Ly, double *AP, cudaStream_t stream)
{
    if (N <= 0 || K < 3 || K > KMAX || !pos || !nn || !nbr || !AP) return set_err(CG_ERR_ARG, "bad args");
    VoroArgs a = raw_args(pos, nn, nbr, K, N, Lx, Ly);
    a.AP = AP;
    if (K <= VG)
        launch_groups<double, false, false>(a, N, stream);
    else
        k_voro_cells<double, false, false><<<nblk(N, 128), 128, 0, stream>>>(a);
    return check_launch();
}

extern "C" int cg_voronoi_forces(const double *pos, const int *nn, const int *nbr, int K, int N,
                                 double Lx, double Ly, const double *APpref, double KA, double KP,
                                 double *AP, double *F, cudaStream_t stream)
{
    if (N <= 0 || K < 3 || K > KMAX || !pos || !nn || !nbr || !APpref || !F)
        return set_err(CG_ERR_ARG, "bad args");
    VoroArgs a = raw_args(pos, nn, nbr, K, N, Lx, Ly);
    a.APpref = (const double2 *)APpref;
    a.KA = KA;
    a.KP = KP;
    a.AP = AP;
    a.F = F;
    if (K <= VG)
        launch_groups<double, true, false>(a, N, stream);
    else
        k_voro_cells<double, true, false><<<nblk(N, 128), 128, 0, stream>>>(a);
    return check_launch();
}

extern "C" int cg_voronoi_test_triangulation(const double *pos, const int *nn, const int *nbr, int K,
                                             int N, double Lx, double Ly, int *flag, int *any_fail,
                                             cudaStream_t stream)
{
    if (N <= 0 || K < 3 || K > KMAX || !pos || !nn || !nbr || !flag || !any_fail)
        return set_err(CG_ERR_ARG, "bad args");
    VoroArgs a = raw_args(pos, nn, nbr, K, N, Lx, Ly);
    a.mark = flag;
    a.queue = any_fail;
    if (K <= VG)
        launch_groups<double, false, true>(a, N, stream);
    else
        k_voro_cells<double, false, true><<<nblk(N, 128), 128, 0, stream>>>(a);
    return check_launch();
}

extern "C" int cg_spp_step(double *pos, double *theta, const double *F, const double *motility,
                           const double *noise, int N, double Lx, double Ly, double dt, double mu,
                           uint64_t seed, uint32_t step, cudaStream_t stream)
{
    if (N <= 0 || !pos || !theta || !F || !motility) return set_err(CG_ERR_ARG, "bad args");
    VoroArgs a;
    memset(&a, 0, sizeof(a));
    a.N = N;
    a.inst0 = make_inst(Lx, Ly, 0, N, 0, BIN_TARGET);
    a.pos = (double2 *)pos;
    a.theta = theta;
    a.F = (void *)F;
    a.motility = (const double2 *)motility;
    a.inst0.seed = seed;
    k_spp<double><<<nblk((N + 1) / 2, SPP_BLOCK), SPP_BLOCK, 0, stream>>>(a, noise, dt, mu, step, 0);
    return check_launch();
}

// ------------------------------------------------------------------------------------------
// 2. systems
// ------------------------------------------------------------------------------------------
struct cg_system {
    int model = CG_MODEL_VORONOI;
    int precision = CG_FP64;
    int n_inst = 0, N = 0, K = 0, n_bins = 0, n_bins_cap = 0;
    std::vector<Inst> h_inst;
    std::vector<int> h_cell_inst;
    cudaStream_t stream = 0;
    uint64_t seed = 0x5eed;
    double KA = 1.0, KP = 1.0;
    size_t bytes = 0;
    std::vector<void *> allocs;
    // device
    Inst *inst = nullptr;
    int *cell_inst = nullptr;
    double2 *pos = nullptr, *motility = nullptr, *APpref = nullptr;
    double *theta = nullptr;
    void *AP = nullptr, *F = nullptr;
    int *nn = nullptr, *nbr = nullptr;
    int *mark = nullptr, *queue = nullptr, *stage_nn = nullptr, *stage_nbr = nullptr, *qslot = nullptr;
    int4 *qhint = nullptr;  // first-round row edits of edge flips, per queue slot
    int *nclaim = nullptr;  // first-round claims per cell in the current step (zero between steps)
    int *held = nullptr, *undec = nullptr;
    Ctl *ctl = nullptr;
    int *bin_count = nullptr, *bin_start = nullptr, *bin_cells = nullptr, *cell_bin = nullptr,
        *cell_slot = nullptr;
    double2 *bin_pos = nullptr;
    void *scan_tmp = nullptr;
    size_t scan_tmp_bytes = 0;
    int *d_status = nullptr;
    unsigned long long *d_zsum = nullptr;
    double *d_energy = nullptr;
    bool topology_valid = false;
    long long host_counters[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    cudaStream_t own_stream = nullptr;
    cudaStream_t body_stream = nullptr;  // captures the bodies of conditional graph nodes
    struct GraphEntry {
        int kind;  // 0 Voronoi SPP, 1 vertex Brownian, 2 vertex SPP, 3 FIRE iterations, 4 SPP + energy out
        int n;
        double dt, mu, T;
        const double *noise;
        cudaGraphExec_t exec;
        long long kernels;
        cg_fire_params fire;  // FIRE graphs: the parameters captured into the iteration kernels
        // host-energy step graphs (kind 4): the graph kept for updating its energy kernel node
        cudaGraph_t graph = nullptr;
        cudaGraphNode_t energy_node = nullptr;
    };
    std::vector<GraphEntry> graphs;
    long long kernels_enqueued = 0;  // kernels of this library launched for this system
    double *noise_buf = nullptr;     // staging for host-supplied noise (one step)
    double *draw_buf = nullptr;      // device normals of the step, drawn beside the repair rounds
    // deterministic force sums (cg_set_deterministic): fixed-point accumulator, 4 words per cell
    int det = 0;
    unsigned long long *Ffix = nullptr;
    unsigned long long *Efix = nullptr;  // fixed-point energy sums, FIXW words per instance
    // asynchronous host-buffer steps: copy stream, a second staging buffer, per-buffer events
    cudaStream_t copy_stream = nullptr;
    double *noise_buf2 = nullptr;
    double *e2e_acc = nullptr;       // energy partial sums of k_energy_to_host (zero between calls)
    unsigned *e2e_done = nullptr;    // its finished-block counter
    cudaEvent_t ev_copied[2] = {nullptr, nullptr}, ev_consumed[2] = {nullptr, nullptr};
    int host_slot = 0;
    // vertex model (model == CG_MODEL_VERTEX): pos/F are per vertex, AP/APpref/theta/motility per cell
    int Nv = 0, vmax = 0;
    int *vert_inst = nullptr, *vn = nullptr, *vcn = nullptr, *cvn = nullptr, *cv = nullptr;
    int *t1_cand = nullptr, *t1_count = nullptr, *t1_resume = nullptr;
    double t1 = 0.01;  // vertexModelBase default (src/models/vertexModelBase.cpp:59)
    // line tension (off until set): per-cell types, mode, gamma or gamma matrix, per-cell term
    int tension_mode = 0, ntypes = 0;
    double gamma = 0.0;
    int *ctype = nullptr;
    double *tmat = nullptr, *TE = nullptr;
    // autotuned launch choices: force-pass shape, cell-list bin side (in mean cell spacings)
    int tune_force = 2;  // the thread-per-cell form where it applies (launch_groups), else shape 0
    int tune_star_grid = 0, tune_commit_grid = 0;  // repair-round grids (0: the defaults)
    double bin_target = 0.8;
    // spatial sorting (allocated on first use): keys, order / inverse, staging, CUB scratch, tags
    unsigned long long *sort_key = nullptr;
    int *sort_idx = nullptr, *tags = nullptr;
    void *sort_tmp = nullptr, *sort_cub = nullptr;
    size_t sort_tmp_bytes = 0;
    // observables (allocated on first use): reference positions, per-instance sums and means
    double2 *obs_ref = nullptr;
    double *obs_acc = nullptr, *obs_mean = nullptr;
    // particle exclusions (off until set): per-cell flags, their count, external forces
    int *excl = nullptr;
    int n_excl = 0;
    double2 *ext_force = nullptr;
    // FIRE (allocated on first use)
    double2 *fire_vel = nullptr;
    void *fire_st = nullptr;
    int *fire_dofinst = nullptr;
    double *fire_part = nullptr;  // per-chunk partial sums of the deterministic FIRE reductions
    int2 *fire_chunk = nullptr;   // (instance, first dof) of every chunk
    int *fire_chunk_off = nullptr;
    int fire_nchunk = 0;
    unsigned *fire_blocks_done = nullptr;  // k_fire_vv2's finished-block count
};

static void release_graph(cg_system::GraphEntry &g)
{
    cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
}

static int ndof(const cg_system *s) { return s->model == CG_MODEL_VERTEX ? s->Nv : s->N; }

// Device memory of a system comes from the stream-ordered allocator on the system's stream, and
// is freed the same way: creating or destroying a system never synchronises the device, so
// systems served concurrently on other streams keep running.
template <typename T>
static int dalloc(cg_system *s, T **p, size_t count)
{
    size_t b = std::max<size_t>(count, 1) * sizeof(T);
    void *q = nullptr;
    CG_CUDA(cudaMallocAsync(&q, b, s->stream));
    s->allocs.push_back(q);
    s->bytes += b;
    CG_CUDA(cudaMemsetAsync(q, 0, b, s->stream));
    *p = (T *)q;
    return CG_OK;
}

// streams of a new system (before any allocation)
static int sys_streams(cg_system *s)
{
    CG_CUDA(cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking));
    CG_CUDA(cudaStreamCreateWithFlags(&s->body_stream, cudaStreamNonBlocking));
    s->stream = s->own_stream;
    return CG_OK;
}

// release everything a system holds (also on a failed creation)
static void sys_release(cg_system *s)
{
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto &g : s->graphs) release_graph(g);
    s->graphs.clear();
    cudaStream_t fs = s->own_stream;
    for (void *p : s->allocs) {
        if (fs) cudaFreeAsync(p, fs);
        else cudaFree(p);
    }
    s->allocs.clear();
    if (fs) cudaStreamSynchronize(fs);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    for (int i = 0; i < 2; ++i) {
        if (s->ev_copied[i]) cudaEventDestroy(s->ev_copied[i]);
        if (s->ev_consumed[i]) cudaEventDestroy(s->ev_consumed[i]);
    }
    if (s->body_stream) cudaStreamDestroy(s->body_stream);
    if (s->own_stream) cudaStreamDestroy(s->own_stream);
    delete s;
}

static VoroArgs sys_args(cg_system *s)
{
    VoroArgs a;
    memset(&a, 0, sizeof(a));
    a.rows_padded = 1;  // every writer of system rows pads them with -1
    a.star_grid = s->tune_star_grid;
    a.commit_grid = s->tune_commit_grid;
    a.N = s->N;
    a.K = s->K;
    a.n_inst = s->n_inst;
    a.inst = s->inst;
    a.cell_inst = s->cell_inst;
    a.pos = s->pos;
    a.theta = s->theta;
    a.motility = s->motility;
    a.APpref = s->APpref;
    a.KA = s->KA;
    a.KP = s->KP;
    a.AP = s->AP;
    a.F = s->F;
    a.Ffix = s->det ? s->Ffix : nullptr;
    a.nn = s->nn;
    a.nbr = s->nbr;
    a.mark = s->mark;
    a.queue = s->queue;
    a.stage_nn = s->stage_nn;
    a.stage_nbr = s->stage_nbr;
    a.qslot = s->qslot;
    a.qhint = s->qhint;
    a.nclaim = s->nclaim;
    a.held = s->held;
    a.undec = s->undec;
    a.ctl = s->ctl;
    a.bin_count = s->bin_count;
    a.bin_start = s->bin_start;
    a.bin_cells = s->bin_cells;
    a.cell_bin = s->cell_bin;
    a.cell_slot = s->cell_slot;
    a.bin_pos = s->bin_pos;
    a.n_bins = s->n_bins;
    a.tension_mode = s->tension_mode;
    a.ntypes = s->ntypes;
    a.gamma = s->gamma;
    a.ctype = s->ctype;
    a.tmat = s->tmat;
    a.TE = s->tension_mode ? s->TE : nullptr;
    return a;
}

static size_t voronoi_bytes(int N, int K, int n_bins, int n_inst, int precision)
{
    size_t real2 = precision == CG_FP64 ? 16 : 8;
    size_t per_cell = 4 /*cell_inst*/ + 4 /*held*/ + 4 /*undec*/ + 16 * 3 /*pos, motility, APpref*/ + 8 /*theta*/ + real2 /*AP*/ + 16 /*F*/ +
                      4 + 4 * (size_t)K /*nn, nbr*/ + 4 /*mark*/ + 4 * (R_MAX + 1) /*queue*/ + 4 +
                      4 * (size_t)K /*stage*/ + 4 * 2 /*qslot*/ + 16 /*qhint*/ + 4 /*nclaim*/ + 4 * 3 + 16 /*cell list*/ +
                      8 + 8 /*noise staging, device draw*/;
    return per_cell * (size_t)N + (size_t)n_bins * 8 + (size_t)n_inst * (sizeof(Inst) + 16) + 4096;
}

extern "C" size_t cg_voronoi_footprint(int n_inst, const int *N, int K)
{
    long long tot = 0, bins = 0;
    for (int i = 0; i < n_inst; ++i) {
        tot += N[i];
        double L = std::sqrt((double)N[i]);
        long long nb = std::max(1, (int)std::floor(L / BIN_TARGET));
        bins += nb * nb;
    }
    return voronoi_bytes((int)tot, K, (int)bins, n_inst, CG_FP64);
}

extern "C" int cg_voronoi_create(int n_inst, const int *N, const double *box, int K, int precision,
                                 cg_system **out)
{
    if (n_inst <= 0 || !N || !box || !out || K < 4 || K > VG_MAX || (K & 3) ||
        (precision != CG_FP64 && precision != CG_MIXED))
        return set_err(CG_ERR_ARG, "bad args");
    cg_system *s = new cg_system();
    s->model = CG_MODEL_VORONOI;
    s->precision = precision;
    if (const char *fs = getenv("CG_FORCE_SHAPE")) s->tune_force = atoi(fs);
    s->n_inst = n_inst;
    s->K = K;
    int off = 0, boff = 0;
    for (int i = 0; i < n_inst; ++i) {
        if (N[i] < 8 || !(box[2 * i] > 0) || !(box[2 * i + 1] > 0)) {
            delete s;
            return set_err(CG_ERR_ARG, "instance needs >= 8 cells and a positive box");
        }
        Inst in = make_inst(box[2 * i], box[2 * i + 1], off, N[i], boff, BIN_TARGET);
        in.seed = mix_seed(s->seed, (unsigned long long)i);
        s->h_inst.push_back(in);
        for (int c = 0; c < N[i]; ++c) s->h_cell_inst.push_back(i);
        off += N[i];
        boff += in.nbx * in.nby;
    }
    s->N = off;
    s->n_bins = boff;
    s->n_bins_cap = boff;
    int Nt = s->N;
    size_t r2 = precision == CG_FP64 ? sizeof(double2) : sizeof(float2);
    int st = sys_streams(s);
    if (st != CG_OK) {
        sys_release(s);
        return st;
    }
    do {
        if ((st = dalloc(s, &s->inst, n_inst))) break;
        if ((st = dalloc(s, &s->cell_inst, Nt))) break;
        if ((st = dalloc(s, &s->pos, Nt))) break;
        if ((st = dalloc(s, &s->motility, Nt))) break;
        if ((st = dalloc(s, &s->APpref, Nt))) break;
        if ((st = dalloc(s, &s->theta, Nt))) break;
        if ((st = dalloc(s, (char **)&s->AP, r2 * Nt))) break;
        if ((st = dalloc(s, (char **)&s->F, sizeof(double2) * Nt))) break;  // FP64 in every precision
        if ((st = dalloc(s, &s->nn, Nt))) break;
        if ((st = dalloc(s, &s->nbr, (size_t)Nt * K))) break;
        if ((st = dalloc(s, &s->mark, Nt))) break;
        if ((st = dalloc(s, &s->queue, (size_t)Nt * (R_MAX + 1)))) break;
        if ((st = dalloc(s, &s->stage_nn, Nt))) break;
        if ((st = dalloc(s, &s->stage_nbr, (size_t)Nt * K))) break;
        if ((st = dalloc(s, &s->qslot, (size_t)Nt * 2))) break;
        if ((st = dalloc(s, &s->qhint, Nt))) break;
        if ((st = dalloc(s, &s->nclaim, Nt))) break;
        if ((st = dalloc(s, &s->held, Nt))) break;
        if ((st = dalloc(s, &s->undec, Nt))) break;
        if ((st = dalloc(s, &s->ctl, 1))) break;
        if ((st = dalloc(s, &s->bin_count, s->n_bins + 1))) break;
        if ((st = dalloc(s, &s->bin_start, s->n_bins + 1))) break;
        if ((st = dalloc(s, &s->bin_cells, Nt))) break;
        if ((st = dalloc(s, &s->cell_bin, Nt))) break;
        if ((st = dalloc(s, &s->cell_slot, Nt))) break;
        if ((st = dalloc(s, &s->bin_pos, Nt))) break;
        if ((st = dalloc(s, &s->d_status, 4))) break;
        if ((st = dalloc(s, &s->d_zsum, n_inst))) break;
        if ((st = dalloc(s, &s->d_energy, n_inst))) break;
        if ((st = dalloc(s, &s->noise_buf, Nt))) break;
        if ((st = dalloc(s, &s->draw_buf, Nt))) break;
        size_t tmpb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tmpb, s->bin_count, s->bin_start, s->n_bins + 1);
        s->scan_tmp_bytes = tmpb;
        if ((st = dalloc(s, (char **)&s->scan_tmp, tmpb))) break;
    } while (0);
    if (st != CG_OK) {
        sys_release(s);
        return st;
    }
    cudaStream_t str = s->stream;
    cudaMemcpyAsync(s->inst, s->h_inst.data(), sizeof(Inst) * n_inst, cudaMemcpyHostToDevice, str);
    cudaMemcpyAsync(s->cell_inst, s->h_cell_inst.data(), sizeof(int) * Nt, cudaMemcpyHostToDevice, str);
    // defaults of the reference: A0 = 1, P0 = 3.8 (Simple2DCell::initializeSimple2DCell,
    // src/models/Simple2DCell.cpp:27), v0 = 0.05, Dr = 1 (VoronoiQuadraticEnergy(n,A0,P0,..),
    // src/models/voronoiQuadraticEnergy.cpp:34)
    std::vector<double2> pref(Nt, make_double2(1.0, 3.8)), mot(Nt, make_double2(0.05, 1.0));
    cudaMemcpyAsync(s->APpref, pref.data(), sizeof(double2) * Nt, cudaMemcpyHostToDevice, str);
    cudaMemcpyAsync(s->motility, mot.data(), sizeof(double2) * Nt, cudaMemcpyHostToDevice, str);
    Ctl c0;
    memset(&c0, 0, sizeof(c0));
    c0.epoch = 1;
    cudaMemcpyAsync(s->ctl, &c0, sizeof(Ctl), cudaMemcpyHostToDevice, str);
    cudaError_t e = cudaStreamSynchronize(str);  // host staging above must outlive the copies
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        sys_release(s);
        return set_err(CG_ERR_CUDA, cudaGetErrorString(e));
    }
    *out = s;
    return CG_OK;
}

extern "C" int cg_destroy(cg_system *s)
{
    if (!s) return CG_OK;
    sys_release(s);
    return CG_OK;
}

extern "C" int cg_num_cells(const cg_system *s) { return s ? s->N : 0; }
extern "C" int cg_num_dofs(const cg_system *s) { return s ? ndof(s) : 0; }
extern "C" int cg_num_instances(const cg_system *s) { return s ? s->n_inst : 0; }
extern "C" int cg_neighbor_capacity(const cg_system *s) { return s ? s->K : 0; }
extern "C" size_t cg_device_bytes(const cg_system *s) { return s ? s->bytes : 0; }

extern "C" int cg_device_memory(size_t *free_bytes, size_t *total_bytes)
{
    size_t f = 0, t = 0;
    CG_CUDA(cudaMemGetInfo(&f, &t));
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return CG_OK;
}

extern "C" int cg_set_stream(cg_system *s, cudaStream_t stream)
{
    if (!s) return set_err(CG_ERR_ARG, "null system");
    CG_CUDA(cudaStreamSynchronize(s->stream));
    s->stream = stream ? stream : s->own_stream;
    return CG_OK;
}

extern "C" cudaStream_t cg_get_stream(cg_system *s) { return s ? s->stream : nullptr; }

extern "C" int cg_synchronize(cg_system *s)
{
    if (!s) return set_err(CG_ERR_ARG, "null system");
    CG_CUDA(cudaStreamSynchronize(s->stream));
    return CG_OK;
}

static int h2d(cg_system *s, void *dst, const void *src, size_t b)
{
    CG_CUDA(cudaMemcpyAsync(dst, src, b, cudaMemcpyHostToDevice, s->stream));
    CG_CUDA(cudaStreamSynchronize(s->stream));
    return CG_OK;
}

static int d2h(cg_system *s, void *dst, const void *src, size_t b)
{
    CG_CUDA(cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToHost, s->stream));
    CG_CUDA(cudaStreamSynchronize(s->stream));
    return CG_OK;
}

extern "C" int cg_set_positions(cg_system *s, const double *pos)
{
    if (!s || !pos) return set_err(CG_ERR_ARG, "bad args");
    s->topology_valid = s->model == CG_MODEL_VERTEX ? s->topology_valid : false;
    return h2d(s, s->pos, pos, sizeof(double2) * ndof(s));
}
extern "C" int cg_get_positions(cg_system *s, double *pos)
{
    if (!s || !pos) return set_err(CG_ERR_ARG, "bad args");
    return d2h(s, pos, s->pos, sizeof(double2) * ndof(s));
}
extern "C" int cg_set_cell_preferences(cg_system *s, const double *p)
{
    if (!s || !p) return set_err(CG_ERR_ARG, "bad args");
    return h2d(s, s->APpref, p, sizeof(double2) * s->N);
}
extern "C" int cg_set_moduli(cg_system *s, double KA, double KP)
{
    if (!s) return set_err(CG_ERR_ARG, "bad args");
    s->KA = KA;
    s->KP = KP;
    return CG_OK;
}
extern "C" int cg_set_motility(cg_system *s, const double *m)
{
    if (!s || !m) return set_err(CG_ERR_ARG, "bad args");
    return h2d(s, s->motility, m, sizeof(double2) * s->N);
}
extern "C" int cg_set_directors(cg_system *s, const double *t)
{
    if (!s || !t) return set_err(CG_ERR_ARG, "bad args");
    return h2d(s, s->theta, t, sizeof(double) * s->N);
}
extern "C" int cg_get_directors(cg_system *s, double *t)
{
    if (!s || !t) return set_err(CG_ERR_ARG, "bad args");
    return d2h(s, t, s->theta, sizeof(double) * s->N);
}
// per-instance Philox keys live in the device instance table, so graphs never capture a seed
static int upload_inst(cg_system *s)
{
    CG_CUDA(cudaMemcpyAsync(s->inst, s->h_inst.data(), sizeof(Inst) * s->n_inst, cudaMemcpyHostToDevice,
                            s->stream));
    CG_CUDA(cudaStreamSynchronize(s->stream));
    return CG_OK;
}

extern "C" int cg_set_seed(cg_system *s, uint64_t seed)
{
    if (!s) return set_err(CG_ERR_ARG, "bad args");
    s->seed = seed;
    for (int i = 0; i < s->n_inst; ++i) s->h_inst[i].seed = mix_seed(seed, (unsigned long long)i);
    return upload_inst(s);
}

extern "C" int cg_set_instance_seeds(cg_system *s, const uint64_t *seeds)
{
    if (!s || !seeds) return set_err(CG_ERR_ARG, "bad args");
    for (int i = 0; i < s->n_inst; ++i) s->h_inst[i].seed = seeds[i];
    return upload_inst(s);
}

static int get_real2(cg_system *s, const void *src, double *dst, int n)
{
    if (s->precision == CG_FP64) return d2h(s, dst, src, sizeof(double2) * n);
    std::vector<float2> tmp(n);
    CG_TRY(d2h(s, tmp.data(), src, sizeof(float2) * n));
    for (int i = 0; i < n; ++i) {
        dst[2 * i] = tmp[i].x;
        dst[2 * i + 1] = tmp[i].y;
    }
    return CG_OK;
}

extern "C" int cg_get_forces(cg_system *s, double *F)
{
    if (!s || !F) return set_err(CG_ERR_ARG, "bad args");
    return d2h(s, F, s->F, sizeof(double2) * ndof(s));  // forces are FP64 in every precision
}
extern "C" int cg_get_area_perimeter(cg_system *s, double *AP)
{
    if (!s || !AP) return set_err(CG_ERR_ARG, "bad args");
    return get_real2(s, s->AP, AP, s->N);
}
extern "C" int cg_get_topology(cg_system *s, int *nn, int *nbr)
{
    if (!s || !nn || !nbr || s->model != CG_MODEL_VORONOI) return set_err(CG_ERR_ARG, "bad args");
    CG_TRY(d2h(s, nn, s->nn, sizeof(int) * s->N));
    return d2h(s, nbr, s->nbr, sizeof(int) * (size_t)s->N * s->K);
}
extern "C" int cg_set_topology(cg_system *s, const int *nn, const int *nbr)
{
    if (!s || !nn || !nbr || s->model != CG_MODEL_VORONOI) return set_err(CG_ERR_ARG, "bad args");
    for (int i = 0; i < s->N; ++i)
        if (nn[i] < 3 || nn[i] > s->K) return set_err(CG_ERR_ARG, "row length out of range");
    // rows on the device are padded with -1 past their length (the repair reads whole rows)
    std::vector<int> rows(nbr, nbr + (size_t)s->N * s->K);
    for (int i = 0; i < s->N; ++i)
        for (int k = nn[i]; k < s->K; ++k) rows[(size_t)i * s->K + k] = -1;
    CG_TRY(h2d(s, s->nn, nn, sizeof(int) * s->N));
    CG_TRY(h2d(s, s->nbr, rows.data(), sizeof(int) * (size_t)s->N * s->K));
    s->topology_valid = true;
    return CG_OK;
}

extern "C" int cg_counters(cg_system *s, long long *out, int n)
{
    if (!s || !out) return set_err(CG_ERR_ARG, "bad args");
    Ctl c;
    CG_TRY(d2h(s, &c, s->ctl, sizeof(Ctl)));
    for (int i = 0; i < n && i < 8; ++i) out[i] = (long long)c.counters[i] + s->host_counters[i];
    return CG_OK;
}

// ---- global triangulation on the device ---------------------------------------------------
static int build_cell_list(cg_system *s)
{
    VoroArgs a = sys_args(s);
    CG_CUDA(cudaMemsetAsync(s->bin_count, 0, sizeof(int) * (s->n_bins + 1), s->stream));
    k_bin_count<<<nblk(s->N, 256), 256, 0, s->stream>>>(a);
    CG_CUDA(cub::DeviceScan::ExclusiveSum(s->scan_tmp, s->scan_tmp_bytes, s->bin_count, s->bin_start,
                                          s->n_bins + 1, s->stream));
    k_bin_scatter<<<nblk(s->N, 256), 256, 0, s->stream>>>(a);
    return check_launch();
}

static int grow_rows(cg_system *s);

static int triangulate_sys(cg_system *s)
{
    CG_TRY(build_cell_list(s));
    VoroArgs a = sys_args(s);
    CG_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(int) * 4, s->stream));
    CG_CUDA(cudaMemsetAsync(s->d_zsum, 0, sizeof(unsigned long long) * s->n_inst, s->stream));
    constexpr int WPB = 4;
    k_star_global<WPB><<<nblk(s->N, WPB), WPB * 32, 0, s->stream>>>(a, s->d_status);
    CG_TRY(check_launch());
    int st = 0;
    CG_TRY(d2h(s, &st, s->d_status, sizeof(int)));
    if (st == CG_ERR_CAPACITY && s->K < VG_MAX) {  // a cell with more than K neighbours: widen, retry
        CG_TRY(grow_rows(s));
        return triangulate_sys(s);
    }
    if (st) return set_err(st, st == CG_ERR_CAPACITY ? "neighbour capacity exceeded in triangulation"
                                                      : "global triangulation failed");
    k_validate<<<nblk(s->N, 256), 256, 0, s->stream>>>(a, s->d_status, s->d_zsum);
    CG_TRY(check_launch());
    std::vector<unsigned long long> zs(s->n_inst);
    CG_TRY(d2h(s, &st, s->d_status, sizeof(int)));
    CG_TRY(d2h(s, zs.data(), s->d_zsum, sizeof(unsigned long long) * s->n_inst));
    if (st) return set_err(CG_ERR_TOPOLOGY, "triangulation is not consistent");
    for (int i = 0; i < s->n_inst; ++i)
        if (zs[i] != 6ull * (unsigned long long)s->h_inst[i].n)
            return set_err(CG_ERR_TOPOLOGY, "Euler check failed (sum of coordinations != 6N)");
    s->topology_valid = true;
    s->host_counters[4] += 1;
    return CG_OK;
}

extern "C" int cg_triangulate(cg_system *s)
{
    if (!s || s->model != CG_MODEL_VORONOI) return set_err(CG_ERR_ARG, "bad args");
    return triangulate_sys(s);
}

extern "C" int cg_voronoi_triangulate(const double *pos, int N, double Lx, double Ly, int K, int *nn,
                                      int *nbr, cudaStream_t stream)
{
    if (!pos || !nn || !nbr || N < 8 || K < 4 || K > KMAX) return set_err(CG_ERR_ARG, "bad args");
    cg_system *s = nullptr;
    double box[2] = {Lx, Ly};
    CG_TRY(cg_voronoi_create(1, &N, box, K, CG_FP64, &s));
    s->stream = stream;
    int st = CG_OK;
    do {
        if ((cudaMemcpyAsync(s->pos, pos, sizeof(double2) * N, cudaMemcpyDeviceToDevice, stream)) !=
            cudaSuccess) {
            st = set_err(CG_ERR_CUDA, "copy failed");
            break;
        }
        if ((st = triangulate_sys(s))) break;
        if (s->K != K) {  // rows widened past the caller's capacity: the caller's buffers cannot hold them
            st = set_err(CG_ERR_CAPACITY, "a cell has more neighbours than the row capacity K");
            break;
        }
        if (cudaMemcpyAsync(nn, s->nn, sizeof(int) * N, cudaMemcpyDeviceToDevice, stream) != cudaSuccess ||
            cudaMemcpyAsync(nbr, s->nbr, sizeof(int) * (size_t)N * K, cudaMemcpyDeviceToDevice, stream) !=
                cudaSuccess)
            st = set_err(CG_ERR_CUDA, "copy failed");
        cudaStreamSynchronize(stream);
    } while (0);
    cg_destroy(s);
    return st;
}

// ---- one step of the Voronoi model ---------------------------------------------------------
template <typename R>
static void launch_force_test(cg_system *s, const VoroArgs &a, bool test, bool clear_f = true)
{
    if (a.Ffix)
        cudaMemsetAsync(a.Ffix, 0, 2 * FIXF * sizeof(unsigned long long) * s->N, s->stream);
    else if (clear_f)
        cudaMemsetAsync(s->F, 0, sizeof(double2) * s->N, s->stream);
    if (test)
        launch_groups<R, true, true>(a, s->N, s->stream, s->tune_force);
    else
        launch_groups<R, true, false>(a, s->N, s->stream, s->tune_force);
    s->kernels_enqueued += 1;
}

// deterministic mode: F from the fixed-point sums, once the force pass (and repair) is complete
template <typename R>
static void finish_forces(cg_system *s, const VoroArgs &a, cudaStream_t st)
{
    if (a.Ffix) {
        k_fix_forces<R><<<nblk(s->N, 256), 256, 0, st>>>(a);
        s->kernels_enqueued += 1;
    }
    if (s->n_excl > 0) {  // excluded cells: F -> external force, F = 0
        k_apply_exclusions<R><<<nblk(s->N, 256), 256, 0, st>>>(s->N, s->excl, a.F, s->ext_force);
        s->kernels_enqueued += 1;
    }
}

// default grids of the repair round: one wave of k_star_local (STAR_MINB resident blocks per SM),
// 8 blocks of k_commit_check per SM; cg_autotune_repair can choose others
constexpr int STAR_GRID = 148 * STAR_MINB;
constexpr int COMMIT_GRID = 148 * 8;

template <typename R, int NS>
static void launch_round_ns(const VoroArgs &a, bool forces, cudaStream_t st, unsigned long long cond, int use_cond)
{
    constexpr int WPB = 4;
    // commit-and-check: 4 queue slots per 64-thread block, so a short queue still spreads over the SMs
    constexpr int WPB_C = 2;
    const int gs = a.star_grid > 0 ? a.star_grid : STAR_GRID, gc = a.commit_grid > 0 ? a.commit_grid : COMMIT_GRID;
    k_star_local<WPB><<<gs, WPB * 32, 0, st>>>(a);
    if (forces)
        k_commit_check<R, true, WPB_C, NS><<<gc, WPB_C * 32, 0, st>>>(a, cond, use_cond);
    else
        k_commit_check<R, false, WPB_C, NS><<<gc, WPB_C * 32, 0, st>>>(a, cond, use_cond);
}

template <typename R>
static void launch_round(cg_system *s, const VoroArgs &a, bool forces, cudaStream_t st, unsigned long long cond,
                         int use_cond)
{
    if (a.K > VG)
        launch_round_ns<R, VG_MAX>(a, forces, st, cond, use_cond);
    else
        launch_round_ns<R, VG>(a, forces, st, cond, use_cond);
}

// start of the repair (undecided in-circle slots of the force pass, then the WHILE condition)
template <typename R>
static void launch_repair_begin(const VoroArgs &a, cudaStream_t st, unsigned long long cond, int use_cond, int forces)
{
    if (a.K > VG)
        k_repair_begin<R, VG_MAX><<<1, 128, 0, st>>>(a, cond, use_cond, forces);
    else
        k_repair_begin<R, VG><<<1, 256, 0, st>>>(a, cond, use_cond, forces);
}

// repair rounds as plain launches (used outside graphs): every round is launched; empty rounds exit
template <typename R>
static void launch_repair(cg_system *s, const VoroArgs &a, bool forces)
{
    launch_repair_begin<R>(a, s->stream, 0ull, 0, forces ? 1 : 0);
    for (int r = 0; r < R_MAX; ++r) launch_round<R>(s, a, forces, s->stream, 0ull, 0);
    s->kernels_enqueued += 1;
    if (forces) finish_forces<R>(s, a, s->stream);
}

static int read_ctl(cg_system *s, Ctl &c) { return d2h(s, &c, s->ctl, sizeof(Ctl)); }

// clear a halted control block so the step can be re-run after the host-side fix
static int reset_ctl_after_halt(cg_system *s)
{
    Ctl c;
    CG_TRY(read_ctl(s, c));
    c.halt = 0;
    c.need_global = 0;
    c.status = 0;
    c.n_flagged = 0;
    for (int r = 0; r <= R_MAX; ++r) c.q_count[r] = 0;
    c.blocks_done = 0;
    c.epoch += R_MAX + 2;
    return h2d(s, s->ctl, &c, sizeof(Ctl));
}

// handle a halted step: global retriangulation (or report the error)
// Row capacity growth (the reference grows neighMax the same way, voronoiModelBase::
// allDelSets / resetLists): rows go from K to 32 slots, copied and padded with -1; the staging rows
// and the sort scratch are reallocated at the new width, and captured graphs (which hold the old
// width and pointers) are dropped. The group kernels then run in their 32-slot form.
__global__ void k_widen_rows(int N, int K, int K2, const int *src, int *dst)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    for (int k = 0; k < K2; ++k) dst[(size_t)c * K2 + k] = k < K ? src[(size_t)c * K + k] : -1;
}

static int grow_rows(cg_system *s)
{
    if (s->model != CG_MODEL_VORONOI || s->K >= VG_MAX)
        return set_err(CG_ERR_CAPACITY, "neighbour capacity exceeded (more than 32 neighbours)");
    const int K2 = VG_MAX;
    CG_CUDA(cudaStreamSynchronize(s->stream));
    for (auto &g : s->graphs) release_graph(g);
    s->graphs.clear();
    int *nbr2 = nullptr, *stage2 = nullptr;
    CG_TRY(dalloc(s, &nbr2, (size_t)s->N * K2));
    CG_TRY(dalloc(s, &stage2, (size_t)s->N * K2));
    k_widen_rows<<<nblk(s->N, 256), 256, 0, s->stream>>>(s->N, s->K, K2, s->nbr, nbr2);
    CG_TRY(check_launch());
    s->nbr = nbr2;  // (the old blocks stay in the arena until the system is destroyed)
    s->stage_nbr = stage2;
    if (s->sort_tmp)
        CG_TRY(dalloc(s, (char **)&s->sort_tmp, (size_t)s->N * std::max<size_t>(16, sizeof(int) * (size_t)(K2 + 1))));
    s->K = K2;
    return cg_synchronize(s);
}

static int recover(cg_system *s)
{
    Ctl c;
    CG_TRY(read_ctl(s, c));
    if (!c.halt) return CG_OK;
    if (c.status == CG_ERR_CAPACITY) CG_TRY(grow_rows(s));
    CG_TRY(reset_ctl_after_halt(s));
    if (s->held) CG_CUDA(cudaMemsetAsync(s->held, 0, sizeof(int) * s->N, s->stream));
    if (s->nclaim) CG_CUDA(cudaMemsetAsync(s->nclaim, 0, sizeof(int) * s->N, s->stream));
    return triangulate_sys(s);
}

template <typename R>
static int compute_forces_t(cg_system *s)
{
    VoroArgs a = sys_args(s);
    launch_force_test<R>(s, a, false);
    finish_forces<R>(s, a, s->stream);
    return check_launch();
}

static int vm_compute_forces(cg_system *s);
static int vm_enforce(cg_system *s);

extern "C" int cg_compute_forces(cg_system *s)
{
    if (!s) return set_err(CG_ERR_ARG, "null system");
    if (s->model == CG_MODEL_VERTEX) return vm_compute_forces(s);
    if (!s->topology_valid) CG_TRY(triangulate_sys(s));
    int st = s->precision == CG_FP64 ? compute_forces_t<double>(s) : compute_forces_t<float>(s);
    if (st) return st;
    return cg_synchronize(s);
}

template <typename R>
static int enforce_t(cg_system *s)
{
    VoroArgs a = sys_args(s);
    for (int attempt = 0; attempt < 3; ++attempt) {
        launch_groups<R, false, true>(a, s->N, s->stream, s->tune_force);
        launch_repair<R>(s, a, false);
        k_step_done<<<1, 1, 0, s->stream>>>(s->ctl, 0);
        CG_TRY(check_launch());
        Ctl c;
        CG_TRY(read_ctl(s, c));
        if (!c.halt) return CG_OK;
        CG_TRY(recover(s));
    }
    return set_err(CG_ERR_TOPOLOGY, "topology could not be enforced");
}

extern "C" int cg_enforce_topology(cg_system *s)
{
    if (!s) return set_err(CG_ERR_ARG, "null system");
    if (s->model == CG_MODEL_VERTEX) return vm_enforce(s);
    if (!s->topology_valid) return triangulate_sys(s);
    return s->precision == CG_FP64 ? enforce_t<double>(s) : enforce_t<float>(s);
}

template <typename R>
static void enqueue_spp_steps(cg_system *s, int n, double dt, double mu, const double *noise, bool noise_per_step)
{
    VoroArgs a = sys_args(s);
    for (int t = 0; t < n; ++t) {
        launch_force_test<R>(s, a, true);
        launch_repair<R>(s, a, true);
        const double *nz = noise ? (noise_per_step ? noise + (size_t)t * s->N : noise) : nullptr;
        k_spp<R><<<nblk((s->N + 1) / 2, SPP_BLOCK), SPP_BLOCK, 0, s->stream>>>(a, nz, dt, mu, 0u, 0);
        k_step_done<<<1, 1, 0, s->stream>>>(s->ctl, 1);
        s->kernels_enqueued += 2;
    }
}

// whether a host-energy step graph reads the energy out in its integrator (k_spp_energy): with
// floating-point force sums and outside the unrolled profiling form
static bool energy_in_spp(const cg_system *s, bool unrolled)
{
    return !s->det && !unrolled;
}

// Build a CUDA graph of n steps. Per step: zero F, fused force + exact test pass, then the local
// repair rounds inside a WHILE conditional node (the device decides whether another round runs),
// then integrate + move and the step epilogue. Kernels take queue lengths, epochs, rounds and the
// step counter from the device control block, so one graph serves every call.
// energy_node != null: the graph ends with k_energy_to_host writing to energy_dst, the graph
// template is kept (*keep) and *energy_node is that kernel's node, for per-call destination updates
template <typename R>
static int build_graph(cg_system *s, int n, double dt, double mu, const double *noise, cudaGraphExec_t *exec,
                       long long *static_kernels, double *energy_dst = nullptr,
                       cudaGraphNode_t *energy_node = nullptr, cudaGraph_t *keep = nullptr)
{
    VoroArgs a = sys_args(s);
    cudaGraph_t graph;
    CG_CUDA(cudaGraphCreate(&graph, 0));
    const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
    std::vector<cudaGraphNode_t> deps;
    long long k0 = s->kernels_enqueued;
    auto capture_deps = [&](cudaStream_t st) -> int {
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t *d = nullptr;
        size_t nd = 0;
        CG_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &d, &nd));
        deps.assign(d, d + nd);
        return CG_OK;
    };
    int st = CG_OK;
    // CG_GRAPH_UNROLLED=1 builds the same steps with the R_MAX rounds as plain kernel nodes (empty
    // rounds exit at once). Profilers that cannot see into conditional nodes need this form.
    const char *unrolled = getenv("CG_GRAPH_UNROLLED");
    if (unrolled && unrolled[0] == '1') {
        CG_CUDA(cudaStreamBeginCaptureToGraph(s->stream, graph, nullptr, nullptr, 0, mode));
        for (int t = 0; t < n; ++t) {
            launch_force_test<R>(s, a, true);
            launch_repair<R>(s, a, true);
            k_spp<R><<<nblk((s->N + 1) / 2, SPP_BLOCK), SPP_BLOCK, 0, s->stream>>>(a, noise, dt, mu, 0u, 0);
            k_step_done<<<1, 1, 0, s->stream>>>(s->ctl, 1);
            s->kernels_enqueued += 2;
        }
        if (energy_node) {
            k_energy_to_host<R><<<nblk(s->N, 256), 256, 0, s->stream>>>(a, s->e2e_acc, s->e2e_done, energy_dst);
            s->kernels_enqueued += 1;
            st = capture_deps(s->stream);
            if (st == CG_OK) *energy_node = deps.empty() ? nullptr : deps[0];
        }
        cudaGraph_t g2;
        CG_CUDA(cudaStreamEndCapture(s->stream, &g2));
    }
    for (int t = 0; t < n && st == CG_OK && !(unrolled && unrolled[0] == '1'); ++t) {
        cudaGraphConditionalHandle h;
        CG_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 0, 0));
        CG_CUDA(cudaStreamBeginCaptureToGraph(s->stream, graph, deps.empty() ? nullptr : deps.data(), nullptr,
                                              deps.size(), mode));
        launch_force_test<R>(s, a, true);
        launch_repair_begin<R>(a, s->stream, (unsigned long long)h, 1, 1);
        s->kernels_enqueued += 1;
        st = capture_deps(s->stream);
        cudaGraph_t g2;
        CG_CUDA(cudaStreamEndCapture(s->stream, &g2));
        if (st) break;
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cn;
        CG_CUDA(cudaGraphAddNode(&cn, graph, deps.data(), deps.size(), &cp));
        // device noise: drawn by a kernel node beside the WHILE node, read by k_spp
        cudaGraphNode_t dn = nullptr;
        if (!noise) {
            double *out = s->draw_buf;
            void *args[] = {&a, &out};
            cudaKernelNodeParams kp;
            memset(&kp, 0, sizeof(kp));
            kp.func = (void *)k_draw_noise;
            kp.gridDim = dim3(nblk((s->N + 1) / 2, SPP_BLOCK));
            kp.blockDim = dim3(SPP_BLOCK);
            kp.kernelParams = args;
            CG_CUDA(cudaGraphAddKernelNode(&dn, graph, deps.data(), deps.size(), &kp));
            s->kernels_enqueued += 1;
        }
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CG_CUDA(cudaStreamBeginCaptureToGraph(s->body_stream, body, nullptr, nullptr, 0, mode));
        launch_round<R>(s, a, true, s->body_stream, (unsigned long long)h, 1);  // counted on the device
        cudaGraph_t gb;
        CG_CUDA(cudaStreamEndCapture(s->body_stream, &gb));
        deps.assign(1, cn);
        if (dn) deps.push_back(dn);
        CG_CUDA(cudaStreamBeginCaptureToGraph(s->stream, graph, deps.data(), nullptr, deps.size(), mode));
        const double *nz = noise ? noise : s->draw_buf;
        finish_forces<R>(s, a, s->stream);
        // the last step's energy readout: inside its integrator with floating-point sums, else a
        // kernel after the step (fixed-point sums)
        const bool fuse_e = energy_node && t == n - 1 && energy_in_spp(s, false);
        if (fuse_e) {
            k_spp_energy<R><<<nblk((s->N + 1) / 2, SPP_BLOCK), SPP_BLOCK, 0, s->stream>>>(
                a, nz, dt, mu, s->e2e_acc, s->e2e_done, energy_dst);
            st = capture_deps(s->stream);
            if (st == CG_OK) *energy_node = deps.empty() ? nullptr : deps[0];
        } else {
            k_spp<R><<<nblk((s->N + 1) / 2, SPP_BLOCK), SPP_BLOCK, 0, s->stream>>>(a, nz, dt, mu, 0u, 0);
        }
        k_step_done<<<1, 1, 0, s->stream>>>(s->ctl, 1);
        s->kernels_enqueued += 2;
        if (energy_node && t == n - 1 && !fuse_e) {
            k_energy_to_host<R><<<nblk(s->N, 256), 256, 0, s->stream>>>(a, s->e2e_acc, s->e2e_done, energy_dst);
            s->kernels_enqueued += 1;
        }
        const int st2 = capture_deps(s->stream);
        if (st == CG_OK) st = st2;
        if (st == CG_OK && energy_node && t == n - 1 && !fuse_e) *energy_node = deps.empty() ? nullptr : deps[0];
        CG_CUDA(cudaStreamEndCapture(s->stream, &g2));
    }
    if (st == CG_OK && energy_node && !*energy_node) st = set_err(CG_ERR_CUDA, "energy node not captured");
    if (st == CG_OK) {
        cudaError_t e = cudaGraphInstantiate(exec, graph, 0);
        if (e != cudaSuccess) st = set_err(CG_ERR_CUDA, cudaGetErrorString(e));
    }
    if (st == CG_OK && keep)
        *keep = graph;  // its nodes name the exec's nodes for later parameter updates
    else
        cudaGraphDestroy(graph);
    *static_kernels = s->kernels_enqueued - k0;
    s->kernels_enqueued = k0;
    return st;
}

// Replay (building on first use) the n-step graph
template <typename R>
static int enqueue_graph(cg_system *s, int n, double dt, double mu, const double *noise)
{
    for (auto &g : s->graphs)
        if (g.kind == 0 && g.n == n && g.dt == dt && g.mu == mu && g.noise == noise) {
            CG_CUDA(cudaGraphLaunch(g.exec, s->stream));
            s->kernels_enqueued += g.kernels;
            return CG_OK;
        }
    cudaGraphExec_t exec;
    long long nk = 0;
    CG_TRY(build_graph<R>(s, n, dt, mu, noise, &exec, &nk));
    s->graphs.push_back({0, n, dt, mu, 0.0, noise, exec, nk});
    CG_CUDA(cudaGraphLaunch(exec, s->stream));
    s->kernels_enqueued += nk;
    return CG_OK;
}

static int read_status(cg_system *s, int *steps, int *halted)
{
    Ctl c;
    CG_TRY(read_ctl(s, c));
    if (steps) *steps = c.step;
    if (halted) *halted = c.halt;
    return CG_OK;
}

template <typename R>
static int spp_run_t(cg_system *s, int n_steps, double dt, double mu, const double *noise)
{
    int step0 = 0, step = 0, halted = 0;
    CG_TRY(read_status(s, &step0, nullptr));
    int done = 0, recoveries = 0;
    const int chunk = 32;  // graphs of 32, 16, ..., 1 steps: any n_steps reuses at most six graphs
    while (done < n_steps) {
        int todo = chunk;
        while (todo > n_steps - done) todo >>= 1;
        if (noise)
            enqueue_spp_steps<R>(s, todo, dt, mu, noise + (size_t)done * s->N, true);
        else
            CG_TRY(enqueue_graph<R>(s, todo, dt, mu, nullptr));
        CG_TRY(check_launch());
        CG_TRY(read_status(s, &step, &halted));
        done = step - step0;
        if (halted) {
            if (++recoveries > 8 + n_steps / 16) return set_err(CG_ERR_TOPOLOGY, "too many global rebuilds");
            CG_TRY(recover(s));
        }
    }
    return CG_OK;
}

// enqueue n RNG-driven steps without any host synchronisation (graph replay)
extern "C" int cg_spp_enqueue(cg_system *s, int n_steps, double dt, double mu)
{
    if (!s || s->model != CG_MODEL_VORONOI || n_steps <= 0) return set_err(CG_ERR_ARG, "bad args");
    if (!s->topology_valid) CG_TRY(triangulate_sys(s));
    return s->precision == CG_FP64 ? enqueue_graph<double>(s, n_steps, dt, mu, nullptr)
                                   : enqueue_graph<float>(s, n_steps, dt, mu, nullptr);
}

// per-instance energies into d_energy, enqueued (the deterministic mode sums in fixed point)
static int enqueue_energies(cg_system *s)
{
    VoroArgs a = sys_args(s);  // N = cells: A/P and preferences are per cell in both models
    unsigned long long *efix = a.Ffix ? s->Efix : nullptr;
    if (!efix) CG_CUDA(cudaMemsetAsync(s->d_energy, 0, sizeof(double) * s->n_inst, s->stream));
    if (s->precision == CG_FP64)
        k_energy<double><<<nblk(s->N, 256), 256, 0, s->stream>>>(a, s->d_energy, efix);
    else
        k_energy<float><<<nblk(s->N, 256), 256, 0, s->stream>>>(a, s->d_energy, efix);
    s->kernels_enqueued += 1;
    if (efix) {
        k_energy_from_fix<<<nblk(s->n_inst, 256), 256, 0, s->stream>>>(s->n_inst, efix, s->d_energy);
        s->kernels_enqueued += 1;
    }
    return CG_OK;
}

// one step with host-supplied noise (copied in) and the per-instance energies copied out
extern "C" int cg_spp_step_host(cg_system *s, const double *host_noise, double dt, double mu,
                                double *host_energy)
{
    if (!s || s->model != CG_MODEL_VORONOI || !host_noise) return set_err(CG_ERR_ARG, "bad args");
    if (!s->topology_valid) CG_TRY(triangulate_sys(s));
    CG_CUDA(cudaMemcpyAsync(s->noise_buf, host_noise, sizeof(double) * s->N, cudaMemcpyHostToDevice,
                            s->stream));
    int st = s->precision == CG_FP64 ? enqueue_graph<double>(s, 1, dt, mu, s->noise_buf)
                                     : enqueue_graph<float>(s, 1, dt, mu, s->noise_buf);
    if (st) return st;
    CG_TRY(enqueue_energies(s));
    if (host_energy)
        CG_CUDA(cudaMemcpyAsync(host_energy, s->d_energy, sizeof(double) * s->n_inst, cudaMemcpyDeviceToHost,
                                s->stream));
    CG_CUDA(cudaStreamSynchronize(s->stream));
    int halted = 0;
    CG_TRY(read_status(s, nullptr, &halted));
    if (halted) {
        CG_TRY(recover(s));
        return set_err(CG_ERR_STATE, "step halted for a global rebuild; state restored, step not taken");
    }
    return CG_OK;
}

// one host-buffer step whose graph ends with the energy kernel writing to page-locked host memory;
// the kernel node's destination is updated per call (cudaGraphExecKernelNodeSetParams), so the
// step and its energy readout are one graph launch
template <typename R>
static int enqueue_energy_graph(cg_system *s, double dt, double mu, const double *noise, double *dst)
{
    if (!s->e2e_acc) {
        CG_TRY(dalloc(s, &s->e2e_acc, FIXW * (size_t)s->n_inst));  // zeroed; the kernel leaves it zeroed
        CG_TRY(dalloc(s, &s->e2e_done, 1));
    }
    for (auto &g : s->graphs)
        if (g.kind == 4 && g.dt == dt && g.mu == mu && g.noise == noise) {
            VoroArgs a = sys_args(s);
            double *acc = s->e2e_acc, *d = dst;
            unsigned *done = s->e2e_done;
            const double *nz = noise ? noise : s->draw_buf;
            double dtv = dt, muv = mu;
            const char *unrolled = getenv("CG_GRAPH_UNROLLED");
            cudaKernelNodeParams kp;
            memset(&kp, 0, sizeof(kp));
            void *args_e[] = {&a, &acc, &done, &d};
            void *args_s[] = {&a, &nz, &dtv, &muv, &acc, &done, &d};
            if (energy_in_spp(s, unrolled && unrolled[0] == '1')) {
                kp.func = (void *)k_spp_energy<R>;
                kp.gridDim = dim3(nblk((s->N + 1) / 2, SPP_BLOCK));
                kp.blockDim = dim3(SPP_BLOCK);
                kp.kernelParams = args_s;
            } else {
                kp.func = (void *)k_energy_to_host<R>;
                kp.gridDim = dim3(nblk(s->N, 256));
                kp.blockDim = dim3(256);
                kp.kernelParams = args_e;
            }
            CG_CUDA(cudaGraphExecKernelNodeSetParams(g.exec, g.energy_node, &kp));
            CG_CUDA(cudaGraphLaunch(g.exec, s->stream));
            s->kernels_enqueued += g.kernels;
            return CG_OK;
        }
    cudaGraphExec_t exec;
    cudaGraph_t keep = nullptr;
    cudaGraphNode_t node = nullptr;
    long long nk = 0;
    CG_TRY(build_graph<R>(s, 1, dt, mu, noise, &exec, &nk, dst, &node, &keep));
    cg_system::GraphEntry e{4, 1, dt, mu, 0.0, noise, exec, nk};
    e.graph = keep;
    e.energy_node = node;
    s->graphs.push_back(e);
    CG_CUDA(cudaGraphLaunch(exec, s->stream));
    s->kernels_enqueued += nk;
    return CG_OK;
}

extern "C" int cg_spp_enqueue_host(cg_system *s, const double *host_noise, double dt, double mu,
                                   double *host_energy)
{
    if (!s || s->model != CG_MODEL_VORONOI || !host_noise) return set_err(CG_ERR_ARG, "bad args");
    if (!s->topology_valid) CG_TRY(triangulate_sys(s));
    if (!s->copy_stream) {
        CG_CUDA(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
        for (int i = 0; i < 2; ++i) {
            CG_CUDA(cudaEventCreateWithFlags(&s->ev_copied[i], cudaEventDisableTiming));
            CG_CUDA(cudaEventCreateWithFlags(&s->ev_consumed[i], cudaEventDisableTiming));
        }
        CG_TRY(dalloc(s, &s->noise_buf2, s->N));
    }
    // page-locked host memory (cudaHostAlloc / cudaHostRegister) for the energies is written by
    // the step graph's last kernel; other host memory takes a reduction and a device-to-host copy
    double *edst = nullptr;
    if (host_energy) {
        cudaPointerAttributes pa;
        if (cudaPointerGetAttributes(&pa, host_energy) != cudaSuccess) {
            cudaGetLastError();  // not a CUDA pointer: clear the error, copy instead
            pa.type = cudaMemoryTypeUnregistered;
        }
        if (pa.type == cudaMemoryTypeHost && pa.devicePointer) edst = static_cast<double *>(pa.devicePointer);
    }
    int slot = s->host_slot;
    s->host_slot ^= 1;
    double *buf = slot ? s->noise_buf2 : s->noise_buf;
    // the buffer is free once the step that last read it has run (no-op before its first use)
    CG_CUDA(cudaStreamWaitEvent(s->copy_stream, s->ev_consumed[slot], 0));
    CG_CUDA(cudaMemcpyAsync(buf, host_noise, sizeof(double) * s->N, cudaMemcpyHostToDevice, s->copy_stream));
    CG_CUDA(cudaEventRecord(s->ev_copied[slot], s->copy_stream));
    CG_CUDA(cudaStreamWaitEvent(s->stream, s->ev_copied[slot], 0));
    int st;
    if (edst)
        st = s->precision == CG_FP64 ? enqueue_energy_graph<double>(s, dt, mu, buf, edst)
                                     : enqueue_energy_graph<float>(s, dt, mu, buf, edst);
    else
        st = s->precision == CG_FP64 ? enqueue_graph<double>(s, 1, dt, mu, buf)
                                     : enqueue_graph<float>(s, 1, dt, mu, buf);
    if (st) return st;
    CG_CUDA(cudaEventRecord(s->ev_consumed[slot], s->stream));
    if (host_energy && !edst) {
        CG_TRY(enqueue_energies(s));
        CG_CUDA(cudaMemcpyAsync(host_energy, s->d_energy, sizeof(double) * s->n_inst, cudaMemcpyDeviceToHost,
                                s->stream));
    }
    return check_launch();
}

// poll: synchronise, report completed steps and whether the device halted; recover if asked
extern "C" int cg_poll(cg_system *s, int *steps_done, int *halted, int recover_if_halted)
{
    if (!s) return set_err(CG_ERR_ARG, "null system");
    CG_CUDA(cudaStreamSynchronize(s->stream));
    int h = 0;
    CG_TRY(read_status(s, steps_done, &h));
    if (halted) *halted = h;
    if (h && recover_if_halted) CG_TRY(recover(s));
    return CG_OK;
}

// the fused geometry+force(+test) pass alone, enqueued without synchronisation
extern "C" int cg_launch_force_pass(cg_system *s, int with_test)
{
    if (!s || s->model != CG_MODEL_VORONOI) return set_err(CG_ERR_ARG, "bad args");
    VoroArgs a = sys_args(s);
    a.undec = nullptr;  // no repair follows: undecided slots count as failing edges
    if (s->precision == CG_FP64) {
        launch_force_test<double>(s, a, with_test != 0);
        finish_forces<double>(s, a, s->stream);
    } else {
        launch_force_test<float>(s, a, with_test != 0);
        finish_forces<float>(s, a, s->stream);
    }
    return check_launch();
}

// kernels launched for this system: host-enqueued ones plus the 2 kernels of every repair round
// executed inside graph WHILE nodes (counted on the device); synchronises the stream
extern "C" long long cg_kernels_launched(cg_system *s)
{
    if (!s) return 0;
    Ctl c;
    if (read_ctl(s, c) != CG_OK) return -1;
    return s->kernels_enqueued + 2 * (long long)c.counters[7];
}

extern "C" int cg_spp_run(cg_system *s, int n_steps, double dt, double mu, const double *noise_dev)
{
    if (!s || s->model != CG_MODEL_VORONOI || n_steps < 0) return set_err(CG_ERR_ARG, "bad args");
    if (!s->topology_valid) CG_TRY(triangulate_sys(s));
    return s->precision == CG_FP64 ? spp_run_t<double>(s, n_steps, dt, mu, noise_dev)
                                   : spp_run_t<float>(s, n_steps, dt, mu, noise_dev);
}

extern "C" int cg_get_energies(cg_system *s, double *E)
{
    if (!s || !E) return set_err(CG_ERR_ARG, "bad args");
    CG_TRY(enqueue_energies(s));
    CG_TRY(check_launch());
    return d2h(s, E, s->d_energy, sizeof(double) * s->n_inst);
}

// Deterministic force sums. Off: forces are summed with floating-point atomics, whose order (and
// so the last bits of F, which a chaotic trajectory amplifies) varies from run to run. On: every
// contribution is added to a per-cell (Voronoi) or per-vertex (vertex model) fixed-point
// accumulator with integer atomics and F is converted from it once per force evaluation, so the
// same inputs give bit-identical forces and trajectories on every run (the reference's kernels sum
// each cell's force sets in a fixed order, src/models/voronoiQuadraticEnergy.cu:30-54). Costs
// 64 bytes per cell (or vertex) and one conversion kernel per force evaluation.
extern "C" int cg_set_deterministic(cg_system *s, int on)
{
    if (!s) return set_err(CG_ERR_ARG, "null system");
    on = on ? 1 : 0;
    if (on == s->det) return CG_OK;
    if (on && !s->Ffix) {
        CG_TRY(dalloc(s, &s->Ffix, 2 * FIXF * (size_t)ndof(s)));
        CG_TRY(dalloc(s, &s->Efix, FIXW * (size_t)s->n_inst));
    }
    CG_CUDA(cudaStreamSynchronize(s->stream));
    for (auto &g : s->graphs) release_graph(g);  // graphs captured the accumulation mode
    s->graphs.clear();
    s->det = on;
    return CG_OK;
}

extern "C" int cg_get_deterministic(cg_system *s) { return s ? s->det : 0; }

// allocation-free triangulation (file-scope device scratch)
#include "noalloc.cu"

// vertex model systems
#include "vertex_sys.cu"

// FIRE
#include "fire_sys.cu"

// line tension
#include "tension.cu"

// particle exclusions
#include "exclusions.cu"

// moving instances between systems (continuous batching)
#include "batching.cu"

// snapshots and exact resume
#include "snapshot.cu"

// observables
#include "observables.cu"

// spatial re-sorting
#include "spatial_sort.cu"

// autotuner
#include "autotune.cu"
