// cellgpu_b200 -- host side of the vertex (AVM) model systems. Included by system.cu.

static VertArgs vm_args(cg_system *s)
{
    VertArgs a;
    memset(&a, 0, sizeof(a));
    a.Nc = s->N;
    a.Nv = s->Nv;
    a.vmax = s->vmax;
    a.n_inst = s->n_inst;
    a.inst = s->inst;
    a.cell_inst = s->cell_inst;
    a.vert_inst = s->vert_inst;
    a.vpos = s->pos;
    a.F = reinterpret_cast<double2 *>(s->F);
    a.Ffix = s->det ? s->Ffix : nullptr;
    a.AP = reinterpret_cast<double2 *>(s->AP);
    a.APpref = s->APpref;
    a.KA = s->KA;
    a.KP = s->KP;
    a.vn = s->vn;
    a.vcn = s->vcn;
    a.cvn = s->cvn;
    a.cv = s->cv;
    a.theta = s->theta;
    a.motility = s->motility;
    a.t1 = s->t1;
    a.cand = s->t1_cand;
    a.cand_count = s->t1_count;
    a.t1_resume = s->t1_resume;
    a.ctl = s->ctl;
    a.tension_mode = s->tension_mode;
    a.ntypes = s->ntypes;
    a.gamma = s->gamma;
    a.ctype = s->ctype;
    a.tmat = s->tmat;
    a.TE = s->tension_mode ? s->TE : nullptr;
    return a;
}

// forces + geometry of every cell (F zeroed first): 8 lanes per cell for rows up to 32 vertices,
// else a thread per cell; the deterministic mode then converts its fixed-point sums into F
// clear_f = false: F is already zero (the caller's previous kernel cleared it)
static void launch_vm_forces(cg_system *s, const VertArgs &a, bool clear_f = true)
{
    if (a.Ffix)
        cudaMemsetAsync(a.Ffix, 0, 2 * FIXF * sizeof(unsigned long long) * s->Nv, s->stream);
    else if (clear_f)
        cudaMemsetAsync(s->F, 0, sizeof(double2) * s->Nv, s->stream);
    if (s->vmax <= VM_ROW_G)
        k_vm_forces_groups<4><<<nblk(s->N, 4 * (32 / VM_G)), 128, 0, s->stream>>>(a, 1);
    else
        k_vm_forces<<<nblk(s->N, 128), 128, 0, s->stream>>>(a, 1);
    if (a.Ffix) {
        k_vm_fix_forces<<<nblk(s->Nv, 256), 256, 0, s->stream>>>(a);
        s->kernels_enqueued += 1;
    }
}

static size_t vertex_bytes(long long Nc, int vmax, int n_inst)
{
    long long Nv = 2 * Nc;
    size_t per_cell = 4 /*cell_inst*/ + 16 * 4 /*AP, APpref, motility, +theta 8*/ + 8 + 4 + 4 * (size_t)vmax;
    size_t per_vert = 4 /*vert_inst*/ + 16 /*pos*/ + 16 /*F*/ + 12 + 12 /*vn, vcn*/ + 8 /*noise staging*/;
    return per_cell * Nc + (per_vert + 12 /*T1 queue*/) * Nv + (size_t)n_inst * (sizeof(Inst) + 16 + 4) + 4096;
}

extern "C" size_t cg_vertex_footprint(int n_inst, const int *Nc, int vmax)
{
    long long tot = 0;
    for (int i = 0; i < n_inst; ++i) tot += Nc[i];
    return vertex_bytes(tot, vmax, n_inst);
}

extern "C" int cg_vertex_create(int n_inst, const int *Nc, const double *box, int vmax, int precision,
                                cg_system **out)
{
    if (n_inst <= 0 || !Nc || !box || !out || vmax < 4 || precision != CG_FP64)
        return set_err(CG_ERR_ARG, "bad args (the vertex model runs in FP64)");
    cg_system *s = new cg_system();
    s->model = CG_MODEL_VERTEX;
    s->precision = CG_FP64;
    s->n_inst = n_inst;
    s->vmax = vmax;
    s->K = vmax;
    int off = 0;
    std::vector<int> vinst;
    for (int i = 0; i < n_inst; ++i) {
        if (Nc[i] < 8 || !(box[2 * i] > 0) || !(box[2 * i + 1] > 0)) {
            delete s;
            return set_err(CG_ERR_ARG, "instance needs >= 8 cells and a positive box");
        }
        Inst in = make_inst(box[2 * i], box[2 * i + 1], off, Nc[i], 0, BIN_TARGET);
        in.voff = 2 * off;
        in.nv = 2 * Nc[i];
        in.seed = mix_seed(s->seed, (unsigned long long)i);
        s->h_inst.push_back(in);
        for (int c = 0; c < Nc[i]; ++c) s->h_cell_inst.push_back(i);
        for (int v = 0; v < 2 * Nc[i]; ++v) vinst.push_back(i);
        off += Nc[i];
    }
    s->N = off;
    s->Nv = 2 * off;
    // the T1 sweep stages up to T1_CAP candidates per instance in dynamic shared memory
    cudaFuncSetAttribute(k_vm_t1_replay, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T1_SMEM);
    cudaFuncSetAttribute(k_vm_t1_resume, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T1_SMEM);
    int st = sys_streams(s);
    if (st != CG_OK) {
        sys_release(s);
        return st;
    }
    do {
        if ((st = dalloc(s, &s->inst, n_inst))) break;
        if ((st = dalloc(s, &s->cell_inst, s->N))) break;
        if ((st = dalloc(s, &s->vert_inst, s->Nv))) break;
        if ((st = dalloc(s, &s->pos, s->Nv))) break;
        if ((st = dalloc(s, (double2 **)&s->F, s->Nv))) break;
        if ((st = dalloc(s, (double2 **)&s->AP, s->N))) break;
        if ((st = dalloc(s, &s->APpref, s->N))) break;
        if ((st = dalloc(s, &s->motility, s->N))) break;
        if ((st = dalloc(s, &s->theta, s->N))) break;
        if ((st = dalloc(s, &s->vn, 3 * (size_t)s->Nv))) break;
        if ((st = dalloc(s, &s->vcn, 3 * (size_t)s->Nv))) break;
        if ((st = dalloc(s, &s->cvn, s->N))) break;
        if ((st = dalloc(s, &s->cv, (size_t)s->N * vmax))) break;
        if ((st = dalloc(s, &s->t1_cand, 3 * (size_t)s->Nv))) break;
        if ((st = dalloc(s, &s->t1_count, n_inst))) break;
        if ((st = dalloc(s, &s->t1_resume, 2 * (size_t)n_inst))) break;
        if ((st = dalloc(s, &s->ctl, 1))) break;
        if ((st = dalloc(s, &s->d_energy, n_inst))) break;
        if ((st = dalloc(s, &s->noise_buf, 2 * (size_t)s->Nv))) break;
    } while (0);
    if (st != CG_OK) {
        sys_release(s);
        return st;
    }
    cudaStream_t str = s->stream;
    cudaMemcpyAsync(s->inst, s->h_inst.data(), sizeof(Inst) * n_inst, cudaMemcpyHostToDevice, str);
    cudaMemcpyAsync(s->cell_inst, s->h_cell_inst.data(), sizeof(int) * s->N, cudaMemcpyHostToDevice, str);
    cudaMemcpyAsync(s->vert_inst, vinst.data(), sizeof(int) * s->Nv, cudaMemcpyHostToDevice, str);
    std::vector<double2> pref(s->N, make_double2(1.0, 3.8)), mot(s->N, make_double2(0.05, 1.0));
    cudaMemcpyAsync(s->APpref, pref.data(), sizeof(double2) * s->N, cudaMemcpyHostToDevice, str);
    cudaMemcpyAsync(s->motility, mot.data(), sizeof(double2) * s->N, cudaMemcpyHostToDevice, str);
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

extern "C" int cg_set_t1_threshold(cg_system *s, double threshold)
{
    if (!s || s->model != CG_MODEL_VERTEX || !(threshold >= 0)) return set_err(CG_ERR_ARG, "bad args");
    s->t1 = threshold;
    for (auto &g : s->graphs) release_graph(g);  // graphs bake the threshold in
    s->graphs.clear();
    return CG_OK;
}

extern "C" int cg_get_vertex_topology(cg_system *s, int *vn, int *vcn, int *cvn, int *cv)
{
    if (!s || s->model != CG_MODEL_VERTEX || !vn || !vcn || !cvn || !cv) return set_err(CG_ERR_ARG, "bad args");
    CG_TRY(d2h(s, vn, s->vn, sizeof(int) * 3 * (size_t)s->Nv));
    CG_TRY(d2h(s, vcn, s->vcn, sizeof(int) * 3 * (size_t)s->Nv));
    CG_TRY(d2h(s, cvn, s->cvn, sizeof(int) * s->N));
    return d2h(s, cv, s->cv, sizeof(int) * (size_t)s->N * s->vmax);
}

extern "C" int cg_set_vertex_topology(cg_system *s, const int *vn, const int *vcn, const int *cvn, const int *cv)
{
    if (!s || s->model != CG_MODEL_VERTEX || !vn || !vcn || !cvn || !cv) return set_err(CG_ERR_ARG, "bad args");
    for (int c = 0; c < s->N; ++c)
        if (cvn[c] < 3 || cvn[c] > s->vmax) return set_err(CG_ERR_ARG, "cell vertex count out of range");
    CG_TRY(h2d(s, s->vn, vn, sizeof(int) * 3 * (size_t)s->Nv));
    CG_TRY(h2d(s, s->vcn, vcn, sizeof(int) * 3 * (size_t)s->Nv));
    CG_TRY(h2d(s, s->cvn, cvn, sizeof(int) * s->N));
    CG_TRY(h2d(s, s->cv, cv, sizeof(int) * (size_t)s->N * s->vmax));
    s->topology_valid = true;
    return CG_OK;
}

// Initialise vertices and wiring from cell positions: Delaunay triangulation on the device (a
// temporary Voronoi batch with the same instances), then the dual.
extern "C" int cg_vertex_from_voronoi(cg_system *s, const double *cell_pos)
{
    if (!s || s->model != CG_MODEL_VERTEX || !cell_pos) return set_err(CG_ERR_ARG, "bad args");
    std::vector<int> Ns(s->n_inst);
    std::vector<double> boxes(2 * s->n_inst);
    for (int i = 0; i < s->n_inst; ++i) {
        Ns[i] = s->h_inst[i].n;
        boxes[2 * i] = s->h_inst[i].Lx;
        boxes[2 * i + 1] = s->h_inst[i].Ly;
    }
    cg_system *v = nullptr;
    const int K = 16;
    CG_TRY(cg_voronoi_create(s->n_inst, Ns.data(), boxes.data(), K, CG_FP64, &v));
    int st = cg_set_positions(v, cell_pos);
    if (st == CG_OK) st = triangulate_sys(v);
    int *owned = nullptr, *tri = nullptr;
    cudaStream_t str = s->stream;
    if (st == CG_OK) {
        if (cudaMallocAsync(&owned, sizeof(int) * (s->N + 1), str) != cudaSuccess ||
            cudaMallocAsync(&tri, sizeof(int) * (size_t)s->N * K, str) != cudaSuccess)
            st = set_err(CG_ERR_CUDA, "allocation failed");
    }
    if (st == CG_OK) {
        DualArgs d;
        memset(&d, 0, sizeof(d));
        d.N = s->N;
        d.K = K;
        d.vmax = s->vmax;
        d.inst = s->inst;
        d.cell_inst = s->cell_inst;
        d.pos = v->pos;
        d.nn = v->nn;
        d.nbr = v->nbr;
        d.owned = owned;
        d.tri = tri;
        d.vpos = s->pos;
        d.vn = s->vn;
        d.vcn = s->vcn;
        d.cvn = s->cvn;
        d.cv = s->cv;
        d.status = v->d_status;
        cudaMemsetAsync(v->d_status, 0, sizeof(int), str);
        k_dual_count<<<nblk(s->N, 256), 256, 0, str>>>(d);
        cudaMemsetAsync(owned + s->N, 0, sizeof(int), str);
        size_t tmpb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tmpb, owned, owned, s->N + 1);
        void *tmp = nullptr;
        if (cudaMallocAsync(&tmp, tmpb + 16, str) != cudaSuccess) st = set_err(CG_ERR_CUDA, "allocation failed");
        if (st == CG_OK) {
            cub::DeviceScan::ExclusiveSum(tmp, tmpb, owned, owned, s->N + 1, str);
            k_dual_assign<<<nblk(s->N, 256), 256, 0, str>>>(d);
            k_dual_resolve<<<nblk(s->N, 256), 256, 0, str>>>(d);
            k_dual_vertices<<<nblk(s->N, 256), 256, 0, str>>>(d);
            int h_status = 0, total = 0;
            cudaMemcpyAsync(&h_status, v->d_status, sizeof(int), cudaMemcpyDeviceToHost, str);
            cudaMemcpyAsync(&total, owned + s->N, sizeof(int), cudaMemcpyDeviceToHost, str);
            cudaError_t e = cudaStreamSynchronize(str);
            if (e != cudaSuccess) st = set_err(CG_ERR_CUDA, cudaGetErrorString(e));
            else if (h_status) st = set_err(h_status, "vertex initialisation failed");
            else if (total != s->Nv) st = set_err(CG_ERR_TOPOLOGY, "number of Delaunay triangles != 2N");
            cudaFreeAsync(tmp, str);
        }
    }
    if (owned) cudaFreeAsync(owned, str);
    if (tri) cudaFreeAsync(tri, str);
    cudaStreamSynchronize(str);
    cg_destroy(v);
    if (st == CG_OK) s->topology_valid = true;
    return st;
}

static int vm_compute_forces(cg_system *s)
{
    if (!s->topology_valid) return set_err(CG_ERR_STATE, "vertex topology not set");
    VertArgs a = vm_args(s);
    launch_vm_forces(s, a);
    s->kernels_enqueued += 1;
    CG_TRY(check_launch());
    return cg_synchronize(s);
}

static void vm_launch_t1(cg_system *s, const VertArgs &a)
{
    k_vm_t1_detect<<<nblk(s->Nv, 256), 256, 0, s->stream>>>(a);
    k_vm_t1_replay<<<s->n_inst, 256, T1_SMEM, s->stream>>>(a);
    s->kernels_enqueued += 2;
}

static int vm_check_halt(cg_system *s)
{
    Ctl c;
    CG_TRY(read_ctl(s, c));
    if (!c.halt) return CG_OK;
    int code = c.status ? c.status : CG_ERR_STATE;
    reset_ctl_after_halt(s);
    return set_err(code, code == CG_ERR_CAPACITY ? "vertex row capacity (vmax) exceeded"
                                                 : "vertex model step failed");
}

// Cell rows grow from vmax to vmax2 entries (copied, padded with -1); captured graphs, which hold
// the old rows and width, are dropped. The reference grows cellVertices the same way when a T1
// transition needs it (vertexModelBase::growCellVerticesList, src/models/vertexModelBase.cpp:474-500).
static int vm_grow_rows(cg_system *s, int vmax2)
{
    CG_CUDA(cudaStreamSynchronize(s->stream));
    for (auto &g : s->graphs) release_graph(g);
    s->graphs.clear();
    int *cv2 = nullptr;
    CG_TRY(dalloc(s, &cv2, (size_t)s->N * vmax2));
    k_widen_rows<<<nblk(s->N, 256), 256, 0, s->stream>>>(s->N, s->vmax, vmax2, s->cv, cv2);
    CG_TRY(check_launch());
    s->cv = cv2;  // (the old block stays in the arena until the system is destroyed)
    s->vmax = s->K = vmax2;
    return cg_synchronize(s);
}

// After a halt: a T1 sweep that stopped because a flip would overflow a cell row kept the keys it
// had still to visit; grow the rows and finish the sweep (repeatedly, if it stops again). Other
// halts are errors. Returns CG_OK when the system runs on.
static int vm_recover(cg_system *s, bool *recovered)
{
    if (recovered) *recovered = false;
    for (int attempt = 0; attempt < 16; ++attempt) {
        Ctl c;
        CG_TRY(read_ctl(s, c));
        if (!c.halt) return CG_OK;
        std::vector<int> res(2 * (size_t)s->n_inst);
        CG_TRY(d2h(s, res.data(), s->t1_resume, sizeof(int) * res.size()));
        bool pending = false;
        for (int v : res) pending = pending || v > 0;
        if (c.status != CG_ERR_CAPACITY || !pending) return vm_check_halt(s);
        CG_TRY(vm_grow_rows(s, s->vmax + 4));
        c.halt = 0;
        c.status = 0;
        CG_TRY(h2d(s, s->ctl, &c, sizeof(Ctl)));
        k_vm_t1_resume<<<s->n_inst, 32, T1_SMEM, s->stream>>>(vm_args(s));
        s->kernels_enqueued += 1;
        CG_TRY(check_launch());
        if (recovered) *recovered = true;
    }
    return set_err(CG_ERR_CAPACITY, "vertex rows kept overflowing after growing");
}

static int vm_enforce(cg_system *s)
{
    VertArgs a = vm_args(s);
    vm_launch_t1(s, a);
    CG_TRY(check_launch());
    return vm_recover(s, nullptr);
}

// one integrator step of the vertex model: forces, integrate + move, T1 sweep
static void vm_enqueue_step(cg_system *s, int kind, int t, double dt, double mu, double T, const double *noise,
                            bool per_step_noise)
{
    VertArgs a = vm_args(s);
    launch_vm_forces(s, a);
    if (kind == 0) {
        const double *nz = noise ? (per_step_noise ? noise + (size_t)t * 2 * s->Nv : noise) : nullptr;
        k_vm_brownian<<<nblk(s->Nv, 256), 256, 0, s->stream>>>(a, nz, dt, mu, T);
        s->kernels_enqueued += 2;
    } else {
        const double *nz = noise ? (per_step_noise ? noise + (size_t)t * s->N : noise) : nullptr;
        k_vm_spp_vertices<<<nblk(s->Nv, 256), 256, 0, s->stream>>>(a, dt, mu);
        k_vm_spp_directors<<<nblk(s->N, 256), 256, 0, s->stream>>>(a, nz, dt);
        s->kernels_enqueued += 3;
    }
    vm_launch_t1(s, a);
    k_step_done<<<1, 1, 0, s->stream>>>(s->ctl, 1);
    s->kernels_enqueued += 1;
}

static int vm_run(cg_system *s, int kind, int n_steps, double dt, double mu, double T, const double *noise)
{
    if (!s->topology_valid) return set_err(CG_ERR_STATE, "vertex topology not set");
    const int chunk = 32;  // graphs of 32, 16, ..., 1 steps: any n_steps reuses at most six graphs
    Ctl c0;
    CG_TRY(read_ctl(s, c0));
    int step_prev = c0.step;
    for (int done = 0; done < n_steps;) {
        int todo = chunk;
        while (todo > n_steps - done) todo >>= 1;
        if (noise) {
            for (int t = 0; t < todo; ++t) vm_enqueue_step(s, kind, done + t, dt, mu, T, noise, true);
        } else {
            // graph of `todo` steps (RNG noise), rebuilt only when the parameters change
            const int gkind = 1 + kind;
            cudaGraphExec_t exec = nullptr;
            long long nk = 0;
            for (auto &g : s->graphs)
                if (g.kind == gkind && g.n == todo && g.dt == dt && g.mu == mu && g.T == T) {
                    exec = g.exec;
                    nk = g.kernels;
                }
            if (!exec) {
                cudaGraph_t graph;
                long long k0 = s->kernels_enqueued;
                CG_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
                for (int t = 0; t < todo; ++t) vm_enqueue_step(s, kind, t, dt, mu, T, nullptr, false);
                CG_CUDA(cudaStreamEndCapture(s->stream, &graph));
                CG_CUDA(cudaGraphInstantiate(&exec, graph, 0));
                cudaGraphDestroy(graph);
                nk = s->kernels_enqueued - k0;
                s->kernels_enqueued = k0;
                s->graphs.push_back({gkind, todo, dt, mu, T, nullptr, exec, nk});
            }
            CG_CUDA(cudaGraphLaunch(exec, s->stream));
            s->kernels_enqueued += nk;
        }
        CG_TRY(check_launch());
        // a step whose T1 sweep stopped on a full cell row: grow the rows, finish its sweep and
        // the step; the later steps of the chunk did nothing and run again (done counts completed
        // steps only, so supplied noise stays aligned with the steps)
        bool recovered = false;
        CG_TRY(vm_recover(s, &recovered));
        if (recovered) {
            k_step_done<<<1, 1, 0, s->stream>>>(s->ctl, 1);
            s->kernels_enqueued += 1;
            CG_TRY(check_launch());
        }
        Ctl c;
        CG_TRY(read_ctl(s, c));
        done += c.step - step_prev;
        step_prev = c.step;
    }
    return CG_OK;
}

extern "C" int cg_brownian_run(cg_system *s, int n_steps, double dt, double mu, double T, const double *noise_dev)
{
    if (!s || s->model != CG_MODEL_VERTEX || n_steps < 0) return set_err(CG_ERR_ARG, "bad args");
    return vm_run(s, 0, n_steps, dt, mu, T, noise_dev);
}

extern "C" int cg_vertex_spp_run(cg_system *s, int n_steps, double dt, double mu, const double *noise_dev)
{
    if (!s || s->model != CG_MODEL_VERTEX || n_steps < 0) return set_err(CG_ERR_ARG, "bad args");
    return vm_run(s, 1, n_steps, dt, mu, 0.0, noise_dev);
}
