// cellgpu_b200 -- launch-parameter autotuner. Included by system.cu.
//
// cg_autotune times, on the system's current state, the runtime-selectable launch parameters and
// keeps the fastest: the launch shape of the fused force pass (8-lane groups with 2 warps per block
// and at least 16 blocks per SM, or 4 warps with at least 8, or one thread per cell) and the
// cell-list bin side of the global triangulation
// (0.8, 1.0 or 1.25 mean cell spacings; the bin arrays allocated at creation hold all three).
// cg_autotune_repair times the grids of the repair round's two launches on real SPP steps, which
// are the only way to get a representative repair load. The repair queues hold every cell of the
// system per round, so they cannot overflow and have no capacity to tune; the local star's
// candidate capacity is a compile-time shared-memory size. Cached step graphs are dropped so the
// next run captures the chosen shapes.

static int grid_bins(cg_system *s, double target)
{
    int boff = 0;
    std::vector<Inst> hi = s->h_inst;
    for (auto &in : hi) {
        in.nbx = std::max(1, (int)std::floor(in.Lx / target));
        in.nby = std::max(1, (int)std::floor(in.Ly / target));
        in.bsx = in.Lx / in.nbx;
        in.bsy = in.Ly / in.nby;
        in.bin_off = boff;
        boff += in.nbx * in.nby;
    }
    if (boff > s->n_bins_cap) return set_err(CG_ERR_CAPACITY, "bin grid larger than allocated");
    s->h_inst = hi;
    s->n_bins = boff;
    s->bin_target = target;
    return upload_inst(s);
}

extern "C" int cg_autotune(cg_system *s, double *times_ms, int *choice)
{
    if (!s) return set_err(CG_ERR_ARG, "null system");
    if (s->model != CG_MODEL_VORONOI) return CG_OK;  // the vertex-model kernels have one launch shape
    if (!s->topology_valid) CG_TRY(triangulate_sys(s));
    cudaEvent_t e0, e1;
    CG_CUDA(cudaEventCreate(&e0));
    CG_CUDA(cudaEventCreate(&e1));
    VoroArgs a = sys_args(s);
    const size_t fb = sizeof(double2) * (size_t)s->N;  // forces are FP64 in every precision
    float best = 1e30f;
    double t_force[3] = {0, 0, 0}, t_bins[3] = {0, 0, 0};
    // shape 2, the thread-per-cell form, only where it applies (FP64, atomic sums, no line
    // tension, 16-slot rows)
    const int n_shapes = (s->precision == CG_FP64 && thread_form_ok(a)) ? 3 : 2;
    for (int shape = 0; shape < n_shapes; ++shape) {
        for (int rep = 0; rep < 13; ++rep) {
            if (rep == 3) cudaEventRecord(e0, s->stream);
            if (a.Ffix) cudaMemsetAsync(a.Ffix, 0, 2 * FIXF * sizeof(unsigned long long) * s->N, s->stream);
            else cudaMemsetAsync(s->F, 0, fb, s->stream);
            if (s->precision == CG_FP64) launch_groups<double, true, false>(a, s->N, s->stream, shape);
            else launch_groups<float, true, false>(a, s->N, s->stream, shape);
        }
        cudaEventRecord(e1, s->stream);
        CG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        t_force[shape] = ms / 10.0;
        if (ms < best) {
            best = ms;
            s->tune_force = shape;
        }
    }
    if (s->precision == CG_FP64) finish_forces<double>(s, a, s->stream);  // F of the last timed pass
    else finish_forces<float>(s, a, s->stream);
    const double targets[3] = {0.8, 1.0, 1.25};
    int bbest = 0;
    best = 1e30f;
    for (int k = 0; k < 3; ++k) {
        CG_TRY(grid_bins(s, targets[k]));
        CG_TRY(triangulate_sys(s));  // warm-up
        cudaEventRecord(e0, s->stream);
        CG_TRY(triangulate_sys(s));
        cudaEventRecord(e1, s->stream);
        CG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        t_bins[k] = ms;
        if (ms < best) {
            best = ms;
            bbest = k;
        }
    }
    CG_TRY(grid_bins(s, targets[bbest]));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CG_CUDA(cudaStreamSynchronize(s->stream));
    for (auto &g : s->graphs) release_graph(g);
    s->graphs.clear();
    if (times_ms) {
        for (int k = 0; k < 3; ++k) times_ms[k] = t_force[k];
        for (int k = 0; k < 3; ++k) times_ms[3 + k] = t_bins[k];
    }
    if (choice) {
        choice[0] = s->tune_force;
        choice[1] = bbest;
    }
    return CG_OK;
}

// Repair-round grids: k_star_local with one wave of STAR_MINB or 2 blocks per SM, k_commit_check
// with 4, 8 or 16 blocks per SM. Each pair runs `steps` SPP steps (device noise) twice and keeps
// the faster window (a window with a halt pays for a global rebuild), timed with events around the
// whole call. The system advances by 2 x 6 x steps steps.
extern "C" int cg_autotune_repair(cg_system *s, int steps, double dt, double mu, double *times_ms, int *choice)
{
    if (!s || steps <= 0) return set_err(CG_ERR_ARG, "bad args");
    if (s->model != CG_MODEL_VORONOI) return CG_OK;
    if (!s->topology_valid) CG_TRY(triangulate_sys(s));
    const int star[2] = {148 * STAR_MINB, 148 * 2};
    const int commit[3] = {148 * 4, 148 * 8, 148 * 16};
    cudaEvent_t e0, e1;
    CG_CUDA(cudaEventCreate(&e0));
    CG_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int bs = 0, bc = 1;
    for (int i = 0; i < 2; ++i) {
        for (int j = 0; j < 3; ++j) {
            s->tune_star_grid = star[i];
            s->tune_commit_grid = commit[j];
            for (auto &g : s->graphs) release_graph(g);
            s->graphs.clear();
            float t = 1e30f;
            for (int rep = 0; rep < 2; ++rep) {
                CG_CUDA(cudaEventRecord(e0, s->stream));
                int st = s->precision == CG_FP64 ? spp_run_t<double>(s, steps, dt, mu, nullptr)
                                                 : spp_run_t<float>(s, steps, dt, mu, nullptr);
                if (st) {
                    cudaEventDestroy(e0);
                    cudaEventDestroy(e1);
                    return st;
                }
                CG_CUDA(cudaEventRecord(e1, s->stream));
                CG_CUDA(cudaEventSynchronize(e1));
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                t = std::min(t, ms / steps);
            }
            if (times_ms) times_ms[3 * i + j] = t;
            if (t < best) {
                best = t;
                bs = i;
                bc = j;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->tune_star_grid = star[bs];
    s->tune_commit_grid = commit[bc];
    for (auto &g : s->graphs) release_graph(g);
    s->graphs.clear();
    if (choice) {
        choice[0] = s->tune_star_grid;
        choice[1] = s->tune_commit_grid;
    }
    return CG_OK;
}
