// cellgpu_b200 -- snapshots of a system's state and exact resume. Included by system.cu.
//
// A snapshot is one self-describing host byte buffer: a header (model, precision, sizes, moduli,
// T1 threshold, step counter, line tension), one record per instance (cells, box, noise key) and
// the per-cell (and, for the vertex model, per-vertex) state with the topology, the cell types and
// the tension matrix. The device noise of a step is
// Philox keyed by the instance seed with the step and the local index as counters, so a system
// restored from a snapshot draws the same noise as the original would have and continues the same
// trajectory: bit for bit when the system sums in the deterministic mode (cg_set_deterministic,
// which the snapshot records and the restore switches on), else up to the summation order of
// floating-point atomics. FIRE velocities and the
// derived quantities (forces, areas, perimeters) are not stored; they are recomputed.
// The reference's state files (netCDF, src/databases/DatabaseNetCDFSPV.cpp:32-46,
// DatabaseNetCDFAVM.cpp:33-52) hold positions and topology but no RNG state, so a run cannot be
// resumed exactly from them.

namespace {

struct SnapHeader {
    char magic[8];  // "CGB2SNP1"
    int version;
    int model, precision, n_inst;
    int N, Nv, K, vmax;
    int topology_valid, step;
    double KA, KP, t1;
    unsigned long long seed;
    int has_types, tension_mode, ntypes;  // line tension
    int flags;                            // bit 0: deterministic force sums (0 in older snapshots);
                                          // bit 1: particle exclusions (a block of N flags, last)
    double gamma;
};

struct SnapInst {
    int n;
    unsigned step_off;  // the instance's noise step offset (0 in older snapshots)
    double Lx, Ly;
    unsigned long long seed;
};

const char SNAP_MAGIC[8] = {'C', 'G', 'B', '2', 'S', 'N', 'P', '1'};

// byte size of every array block, in the order they are stored (the cell types and the tension
// matrix last, when present)
void snap_layout(const SnapHeader &h, size_t sizes[10], int &count)
{
    const size_t N = (size_t)h.N;
    if (h.model == CG_MODEL_VORONOI) {
        size_t s[] = {N * sizeof(double2), N * sizeof(double), N * sizeof(double2), N * sizeof(double2),
                      N * sizeof(int), N * (size_t)h.K * sizeof(int),
                      h.has_types ? N * sizeof(int) : 0,
                      h.tension_mode == 2 ? (size_t)h.ntypes * h.ntypes * sizeof(double) : 0,
                      (h.flags & 2) ? N * sizeof(int) : 0};
        count = 9;
        for (int i = 0; i < count; ++i) sizes[i] = s[i];
    } else {
        const size_t Nv = (size_t)h.Nv;
        size_t s[] = {Nv * sizeof(double2), N * sizeof(double), N * sizeof(double2), N * sizeof(double2),
                      3 * Nv * sizeof(int), 3 * Nv * sizeof(int), N * sizeof(int), N * (size_t)h.vmax * sizeof(int),
                      h.has_types ? N * sizeof(int) : 0,
                      h.tension_mode == 2 ? (size_t)h.ntypes * h.ntypes * sizeof(double) : 0};
        count = 10;
        for (int i = 0; i < count; ++i) sizes[i] = s[i];
    }
}

size_t snap_total(const SnapHeader &h)
{
    size_t sizes[10];
    int count = 0;
    snap_layout(h, sizes, count);
    size_t t = sizeof(SnapHeader) + (size_t)h.n_inst * sizeof(SnapInst);
    for (int i = 0; i < count; ++i) t += sizes[i];
    return t;
}

SnapHeader snap_header(const cg_system *s)
{
    SnapHeader h;
    memset(&h, 0, sizeof(h));
    memcpy(h.magic, SNAP_MAGIC, 8);
    h.version = 2;
    h.model = s->model;
    h.precision = s->precision;
    h.n_inst = s->n_inst;
    h.N = s->N;
    h.Nv = s->Nv;
    h.K = s->K;
    h.vmax = s->vmax;
    h.topology_valid = s->topology_valid ? 1 : 0;
    h.KA = s->KA;
    h.KP = s->KP;
    h.t1 = s->t1;
    h.seed = s->seed;
    h.has_types = s->ctype ? 1 : 0;
    h.tension_mode = s->tension_mode;
    h.ntypes = s->tension_mode == 2 ? s->ntypes : 0;
    h.gamma = s->gamma;
    h.flags = (s->det ? 1 : 0) | (s->n_excl > 0 ? 2 : 0);
    return h;
}

}  // namespace

extern "C" size_t cg_snapshot_size(cg_system *s)
{
    if (!s) return 0;
    return snap_total(snap_header(s));
}

extern "C" int cg_snapshot(cg_system *s, void *buf, size_t bytes)
{
    if (!s || !buf) return set_err(CG_ERR_ARG, "bad args");
    SnapHeader h = snap_header(s);
    if (bytes < snap_total(h)) return set_err(CG_ERR_ARG, "snapshot buffer too small (see cg_snapshot_size)");
    Ctl c;
    CG_TRY(read_ctl(s, c));
    h.step = c.step;
    unsigned char *p = static_cast<unsigned char *>(buf);
    memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    for (int i = 0; i < s->n_inst; ++i) {
        SnapInst r;
        memset(&r, 0, sizeof(r));
        r.n = s->h_inst[i].n;
        r.Lx = s->h_inst[i].Lx;
        r.Ly = s->h_inst[i].Ly;
        r.seed = s->h_inst[i].seed;
        r.step_off = s->h_inst[i].step_off;
        memcpy(p, &r, sizeof(r));
        p += sizeof(r);
    }
    size_t sizes[10];
    int count = 0;
    snap_layout(h, sizes, count);
    const void *src_v[] = {s->pos, s->theta, s->motility, s->APpref, s->nn, s->nbr, s->ctype, s->tmat, s->excl};
    const void *src_m[] = {s->pos, s->theta, s->motility, s->APpref, s->vn, s->vcn, s->cvn, s->cv, s->ctype, s->tmat};
    const void *const *src = s->model == CG_MODEL_VORONOI ? src_v : src_m;
    for (int i = 0; i < count; ++i) {
        if (sizes[i]) CG_TRY(d2h(s, p, src[i], sizes[i]));
        p += sizes[i];
    }
    return CG_OK;
}

extern "C" int cg_restore(const void *buf, size_t bytes, cg_system **out)
{
    if (!buf || !out || bytes < sizeof(SnapHeader)) return set_err(CG_ERR_ARG, "bad args");
    SnapHeader h;
    memcpy(&h, buf, sizeof(h));
    if (memcmp(h.magic, SNAP_MAGIC, 8) != 0 || h.version != 2) return set_err(CG_ERR_ARG, "not a cellgpu_b200 snapshot");
    if (h.n_inst <= 0 || h.N <= 0 || (h.model != CG_MODEL_VORONOI && h.model != CG_MODEL_VERTEX) ||
        h.tension_mode < 0 || h.tension_mode > 2 || h.ntypes < 0 || (h.tension_mode == 2 && h.ntypes < 1) ||
        (h.tension_mode && !h.has_types) || (h.flags & ~3) ||
        ((h.flags & 2) && h.model != CG_MODEL_VORONOI) || bytes < snap_total(h))
        return set_err(CG_ERR_ARG, "corrupt or truncated snapshot");
    const unsigned char *p = static_cast<const unsigned char *>(buf) + sizeof(h);
    std::vector<int> Ns(h.n_inst);
    std::vector<double> boxes(2 * (size_t)h.n_inst);
    std::vector<uint64_t> seeds(h.n_inst);
    std::vector<unsigned> step_offs(h.n_inst);
    long long total = 0;
    for (int i = 0; i < h.n_inst; ++i) {
        SnapInst r;
        memcpy(&r, p, sizeof(r));
        p += sizeof(r);
        Ns[i] = r.n;
        boxes[2 * i] = r.Lx;
        boxes[2 * i + 1] = r.Ly;
        seeds[i] = r.seed;
        step_offs[i] = r.step_off;
        total += r.n;
    }
    if (total != h.N) return set_err(CG_ERR_ARG, "corrupt snapshot (instance sizes)");
    cg_system *s = nullptr;
    if (h.model == CG_MODEL_VORONOI)
        CG_TRY(cg_voronoi_create(h.n_inst, Ns.data(), boxes.data(), h.K, h.precision, &s));
    else
        CG_TRY(cg_vertex_create(h.n_inst, Ns.data(), boxes.data(), h.vmax, h.precision, &s));
    int st = CG_OK;
    do {
        s->seed = h.seed;
        for (int i = 0; i < h.n_inst; ++i) s->h_inst[i].step_off = step_offs[i];
        if ((st = cg_set_instance_seeds(s, seeds.data()))) break;
        s->KA = h.KA;
        s->KP = h.KP;
        s->t1 = h.t1;
        size_t sizes[10];
        int count = 0;
        snap_layout(h, sizes, count);
        if (h.has_types && (st = tension_alloc(s))) break;
        if (h.tension_mode == 2 && (st = dalloc(s, &s->tmat, (size_t)h.ntypes * h.ntypes))) break;
        if ((h.flags & 2) && ((st = dalloc(s, &s->excl, s->N)) || (st = dalloc(s, &s->ext_force, s->N)))) break;
        void *dst_v[] = {s->pos, s->theta, s->motility, s->APpref, s->nn, s->nbr, s->ctype, s->tmat, s->excl};
        void *dst_m[] = {s->pos, s->theta, s->motility, s->APpref, s->vn, s->vcn, s->cvn, s->cv, s->ctype, s->tmat};
        void **dst = h.model == CG_MODEL_VORONOI ? dst_v : dst_m;
        for (int i = 0; i < count && st == CG_OK; ++i) {
            if (sizes[i]) st = h2d(s, dst[i], p, sizes[i]);
            p += sizes[i];
        }
        if (st) break;
        if (h.flags & 2) {  // the exclusion flags are the last block
            std::vector<int> fl(s->N);
            memcpy(fl.data(), p - sizes[count - 1], sizeof(int) * (size_t)s->N);
            s->n_excl = 0;
            for (int f : fl) s->n_excl += f != 0;
        }
        s->tension_mode = h.tension_mode;
        s->ntypes = h.ntypes;
        s->gamma = h.gamma;
        s->topology_valid = h.topology_valid != 0;
        if ((h.flags & 1) && (st = cg_set_deterministic(s, 1))) break;
        Ctl c;
        if ((st = read_ctl(s, c))) break;
        c.step = h.step;
        st = h2d(s, s->ctl, &c, sizeof(Ctl));
    } while (0);
    if (st != CG_OK) {
        cg_destroy(s);
        return st;
    }
    *out = s;
    return CG_OK;
}

extern "C" int cg_get_instances(cg_system *s, int *N, double *box)
{
    if (!s) return set_err(CG_ERR_ARG, "bad args");
    for (int i = 0; i < s->n_inst; ++i) {
        if (N) N[i] = s->h_inst[i].n;
        if (box) {
            box[2 * i] = s->h_inst[i].Lx;
            box[2 * i + 1] = s->h_inst[i].Ly;
        }
    }
    return CG_OK;
}

extern "C" int cg_model_kind(cg_system *s) { return s ? s->model : -1; }
extern "C" int cg_precision(cg_system *s) { return s ? s->precision : -1; }
