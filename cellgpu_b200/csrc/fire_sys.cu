// cellgpu_b200 -- host side of FIRE minimisation (both models). Included by system.cu.

static int fire_alloc(cg_system *s)
{
    if (s->fire_vel) return CG_OK;
    CG_TRY(dalloc(s, &s->fire_vel, ndof(s)));
    FireInst *fs = nullptr;
    CG_TRY(dalloc(s, &fs, s->n_inst));
    s->fire_st = fs;
    CG_TRY(dalloc(s, &s->fire_dofinst, ndof(s)));
    // chunks of FIRE_BLOCK dofs counted from each instance's first dof (deterministic reductions)
    std::vector<int2> chunk;
    std::vector<int> chunk_off(s->n_inst + 1, 0);
    for (int i = 0; i < s->n_inst; ++i) {
        const Inst &in = s->h_inst[i];
        const int o = in.nv > 0 ? in.voff : in.off, n = in.nv > 0 ? in.nv : in.n;
        chunk_off[i] = (int)chunk.size();
        for (int d = 0; d < n; d += FIRE_BLOCK) chunk.push_back(make_int2(i, o + d));
    }
    chunk_off[s->n_inst] = (int)chunk.size();
    s->fire_nchunk = (int)chunk.size();
    CG_TRY(dalloc(s, &s->fire_part, 3 * (size_t)std::max(1, s->fire_nchunk)));
    CG_TRY(dalloc(s, &s->fire_chunk, (size_t)std::max(1, s->fire_nchunk)));
    CG_TRY(dalloc(s, &s->fire_chunk_off, (size_t)s->n_inst + 1));
    CG_TRY(dalloc(s, &s->fire_blocks_done, 1));
    if (s->fire_nchunk > 0)
        CG_CUDA(cudaMemcpyAsync(s->fire_chunk, chunk.data(), sizeof(int2) * chunk.size(), cudaMemcpyHostToDevice,
                                s->stream));
    CG_CUDA(cudaMemcpyAsync(s->fire_chunk_off, chunk_off.data(), sizeof(int) * chunk_off.size(),
                            cudaMemcpyHostToDevice, s->stream));
    CG_CUDA(cudaStreamSynchronize(s->stream));  // the host vectors go out of scope
    if (s->model == CG_MODEL_VORONOI) {
        CG_CUDA(cudaMemcpyAsync(s->fire_dofinst, s->cell_inst, sizeof(int) * s->N, cudaMemcpyDeviceToDevice,
                                s->stream));
    } else {
        CG_CUDA(cudaMemcpyAsync(s->fire_dofinst, s->vert_inst, sizeof(int) * s->Nv, cudaMemcpyDeviceToDevice,
                                s->stream));
    }
    return CG_OK;
}

static FireArgs fire_args(cg_system *s, const cg_fire_params &prm)
{
    FireArgs a;
    memset(&a, 0, sizeof(a));
    a.ndof = ndof(s);
    a.n_inst = s->n_inst;
    a.inst = s->inst;
    a.dof_inst = s->fire_dofinst;
    a.pos = s->pos;
    a.vel = s->fire_vel;
    a.F = reinterpret_cast<double2 *>(s->F);
    a.st = reinterpret_cast<FireInst *>(s->fire_st);
    a.part = s->det ? s->fire_part : nullptr;
    a.chunk = s->fire_chunk;
    a.chunk_off = s->fire_chunk_off;
    a.blocks_done = s->fire_blocks_done;
    a.iter_counter = &s->ctl->counters[6];
    a.zero_f = s->det ? 0 : 1;  // the deterministic mode sums into Ffix, which is cleared by memset
    a.prm = prm;
    a.ctl = s->ctl;
    return a;
}

// forces on the current topology (the loop head of minimize: computeForces before the loop).
// f_zeroed: F is already zero (k_fire_mix_vv1 cleared it), so its memset is left out.
static void fire_forces(cg_system *s, bool test_and_repair, bool f_zeroed = false)
{
    if (s->model == CG_MODEL_VORONOI) {
        VoroArgs a = sys_args(s);
        launch_force_test<double>(s, a, test_and_repair, !f_zeroed);
        if (test_and_repair)
            launch_repair<double>(s, a, true);
        else
            finish_forces<double>(s, a, s->stream);
        if (test_and_repair) {
            k_step_done<<<1, 1, 0, s->stream>>>(s->ctl, 0);
            s->kernels_enqueued += 1;
        }
    } else {
        VertArgs a = vm_args(s);
        if (test_and_repair) vm_launch_t1(s, a);
        launch_vm_forces(s, a, !f_zeroed);
        s->kernels_enqueued += 1;
    }
}

// second half-kick and the per-instance power / norm sums (deterministic mode: in an order fixed
// by each instance's dof count, so the same in any batch)
static void fire_vv2_reduce(cg_system *s, const FireArgs &f)
{
    if (f.part) {
        if (s->fire_nchunk > 0) k_fire_vv2_chunks<<<s->fire_nchunk, FIRE_BLOCK, 0, s->stream>>>(f);
        k_fire_reduce<<<s->n_inst, FIRE_BLOCK, 0, s->stream>>>(f);
        s->kernels_enqueued += 2;
    } else {
        k_fire_vv2<<<nblk(ndof(s), FIRE_BLOCK), FIRE_BLOCK, 0, s->stream>>>(f);
        s->kernels_enqueued += 1;
    }
}

// one FIRE iteration: the previous iteration's velocity mix and the first Verlet half (move),
// topology and forces, then the second half with the sums and the per-instance update
static void fire_enqueue_iteration(cg_system *s, const cg_fire_params &prm)
{
    FireArgs f = fire_args(s, prm);
    k_fire_mix_vv1<<<nblk(ndof(s), 256), 256, 0, s->stream>>>(f);
    s->kernels_enqueued += 1;
    fire_forces(s, true, f.zero_f != 0);
    fire_vv2_reduce(s, f);
}

// FIRE reads and moves FP64 positions and forces: mixed-precision Voronoi systems (FP32 forces)
// are refused
static int fire_check(cg_system *s)
{
    if (s->model == CG_MODEL_VORONOI && s->precision != CG_FP64)
        return set_err(CG_ERR_ARG, "FIRE needs an FP64 system");
    return CG_OK;
}

// Start a minimisation: per-instance FIRE state reset (EnergyMinimizerFIRE's initial dt, alpha and
// counters) and the forces of the current state (minimize's computeForces before the loop)
extern "C" int cg_fire_begin(cg_system *s, const cg_fire_params *prm)
{
    if (!s || !prm || prm->max_iterations < 0 || !(prm->dt > 0)) return set_err(CG_ERR_ARG, "bad args");
    CG_TRY(fire_check(s));
    if (!s->topology_valid) {
        if (s->model == CG_MODEL_VORONOI) CG_TRY(triangulate_sys(s));
        else return set_err(CG_ERR_STATE, "vertex topology not set");
    }
    CG_TRY(fire_alloc(s));
    FireArgs f = fire_args(s, *prm);
    k_fire_init<<<nblk(std::max(ndof(s), s->n_inst), 256), 256, 0, s->stream>>>(f, 0, s->n_inst);
    fire_forces(s, false);
    return check_launch();
}

// Fresh FIRE state for instances [first, first + count) only, the others keeping theirs, and the
// forces of the current state: instances admitted into a batch whose other instances are already
// minimising (serving). cg_fire_advance then continues all of them.
extern "C" int cg_fire_begin_instances(cg_system *s, const cg_fire_params *prm, int first, int count)
{
    if (!s || !prm || prm->max_iterations < 0 || !(prm->dt > 0) || first < 0 || count < 0 ||
        first + count > s->n_inst)
        return set_err(CG_ERR_ARG, "bad args");
    CG_TRY(fire_check(s));
    if (!s->topology_valid) {
        if (s->model == CG_MODEL_VORONOI) CG_TRY(triangulate_sys(s));
        else return set_err(CG_ERR_STATE, "vertex topology not set");
    }
    CG_TRY(fire_alloc(s));
    FireArgs f = fire_args(s, *prm);
    k_fire_init<<<nblk(std::max(ndof(s), s->n_inst), 256), 256, 0, s->stream>>>(f, first, first + count);
    fire_forces(s, false);
    return check_launch();
}

// Continue a minimisation started by cg_fire_begin for up to `iterations` more iterations of every
// instance (in graphs of 16; instances that have converged or reached max_iterations stay frozen),
// or until every instance has stopped. *n_stopped (may be NULL) receives the number of stopped
// instances. Calls with the same parameters continue the same trajectory, so running a
// minimisation in pieces gives the same result as one cg_fire_minimize call.
extern "C" int cg_fire_advance(cg_system *s, const cg_fire_params *prm, int iterations, int *n_stopped)
{
    if (!s || !prm || iterations < 0) return set_err(CG_ERR_ARG, "bad args");
    if (!s->fire_st) return set_err(CG_ERR_STATE, "cg_fire_begin first");
    FireArgs f = fire_args(s, *prm);
    std::vector<FireInst> st(s->n_inst);
    const int chunk = 16;
    int rounds = 0, stopped = 0;
    for (int done = 0;; done += chunk) {
        CG_TRY(d2h(s, st.data(), s->fire_st, sizeof(FireInst) * s->n_inst));
        stopped = 0;
        for (auto &x : st) stopped += x.converged ? 1 : 0;
        if (stopped == s->n_inst || done >= iterations) break;
        // a graph of `chunk` iterations
        cudaGraphExec_t exec = nullptr;
        long long nk = 0;
        for (auto &g : s->graphs)
            if (g.kind == 3 && g.n == chunk && memcmp(&g.fire, prm, sizeof(cg_fire_params)) == 0) {
                exec = g.exec;
                nk = g.kernels;
            }
        if (!exec) {
            cudaGraph_t graph;
            long long k0 = s->kernels_enqueued;
            CG_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
            for (int t = 0; t < chunk; ++t) fire_enqueue_iteration(s, *prm);
            CG_CUDA(cudaStreamEndCapture(s->stream, &graph));
            CG_CUDA(cudaGraphInstantiate(&exec, graph, 0));
            cudaGraphDestroy(graph);
            nk = s->kernels_enqueued - k0;
            s->kernels_enqueued = k0;
            cg_system::GraphEntry ge{3, chunk, prm->dt, prm->force_cutoff, prm->dt_max, nullptr, exec, nk, *prm};
            s->graphs.push_back(ge);
        }
        CG_CUDA(cudaGraphLaunch(exec, s->stream));
        s->kernels_enqueued += nk;
        CG_TRY(check_launch());
        Ctl c;
        CG_TRY(read_ctl(s, c));
        if (c.halt) {
            // a Voronoi step needed a global rebuild, or a vertex T1 sweep wider rows: fix it,
            // recompute forces and finish the halted iteration (its first half-kick and move
            // already happened)
            if (s->model == CG_MODEL_VORONOI) CG_TRY(recover(s));
            else CG_TRY(vm_recover(s, nullptr));
            fire_forces(s, false);
            fire_vv2_reduce(s, f);
            CG_TRY(check_launch());
        }
        if (++rounds > prm->max_iterations / chunk + 64) return set_err(CG_ERR_STATE, "FIRE did not stop");
    }
    if (n_stopped) *n_stopped = stopped;
    return CG_OK;
}

extern "C" int cg_fire_minimize(cg_system *s, const cg_fire_params *prm)
{
    CG_TRY(cg_fire_begin(s, prm));
    return cg_fire_advance(s, prm, prm->max_iterations + 16 * 64, nullptr);
}

extern "C" int cg_fire_state(cg_system *s, int *iterations, double *fmax_cpu, double *fnorm_gpu)
{
    if (!s || !s->fire_st) return set_err(CG_ERR_STATE, "no FIRE run on this system");
    std::vector<FireInst> st(s->n_inst);
    CG_TRY(d2h(s, st.data(), s->fire_st, sizeof(FireInst) * s->n_inst));
    for (int i = 0; i < s->n_inst; ++i) {
        if (iterations) iterations[i] = st[i].iterations;
        if (fmax_cpu) fmax_cpu[i] = sqrt(st[i].fmax);
        if (fnorm_gpu) fnorm_gpu[i] = st[i].ndof > 0 ? sqrt(st[i].fnorm_last / st[i].ndof) : 0.0;
    }
    return CG_OK;
}
