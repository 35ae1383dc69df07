// cellgpu_b200 -- on-device observables per instance. Included by system.cu.
//
// Shape statistics from the stored areas and perimeters, as Simple2DCell::reportq, reportVarq,
// reportMeanP and reportVarAP compute them (src/models/Simple2DCell.cpp:699-765: mean of
// q = P / sqrt(A), and two-pass variances about the means), and the dynamical features of
// dynamicalFeatures (src/analysis/dynamicalFeatures.cpp:17-50): mean squared displacement and the
// overlap function (fraction of degrees of freedom whose minimum-image displacement from the
// reference positions is below a cutoff) against positions captured by
// cg_set_reference_positions. Every reduction is per instance, so a batch needs no host loop.

namespace cg {

struct ObsArgs {
    int n, n_inst;
    const int *inst_of;  // instance of each element (cells or degrees of freedom)
    const Inst *inst;
    const void *AP;
    int fp64;
    const double2 *pos, *ref;
    double cutoff;
    const double *mean;  // per instance: mean q, mean A, mean P (pass 2)
    double *acc;         // per instance: OBS_ACC sums
};
constexpr int OBS_ACC = 8;

// add v[0..k) to acc[inst * OBS_ACC + slot0 + j]: blocks inside one instance (elements of an
// instance are contiguous) reduce in shared memory and add once, others add per element
template <int KV>
CG_D void obs_block_add(const ObsArgs &o, int e, int inst, double (&v)[KV], int slot0)
{
    __shared__ double s_part[KV][8];
    const int e0 = blockIdx.x * blockDim.x, e1 = min(o.n, e0 + (int)blockDim.x) - 1;
    const int i0 = o.inst_of[e0], i1 = o.inst_of[e1];
    if (i0 == i1) {
#pragma unroll
        for (int j = 0; j < KV; ++j) {
            double x = v[j];
            for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
            if ((threadIdx.x & 31) == 0) s_part[j][threadIdx.x >> 5] = x;
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (int j = 0; j < KV; ++j) {
                double t = 0.0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_part[j][w];
                atomicAdd(&o.acc[(size_t)i0 * OBS_ACC + slot0 + j], t);
            }
    } else if (e < o.n) {
        for (int j = 0; j < KV; ++j) atomicAdd(&o.acc[(size_t)inst * OBS_ACC + slot0 + j], v[j]);
    }
}

CG_D double2 obs_ap(const ObsArgs &o, int c)
{
    if (o.fp64) return reinterpret_cast<const double2 *>(o.AP)[c];
    float2 f = reinterpret_cast<const float2 *>(o.AP)[c];
    return make_double2(f.x, f.y);
}

// pass 1 over cells: sums of q, A, P (slots 0-2)
__global__ void __launch_bounds__(256) k_obs_shape(ObsArgs o)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    int inst = 0;
    if (c < o.n) {
        double2 ap = obs_ap(o, c);
        v[0] = ap.y / sqrt(ap.x);
        v[1] = ap.x;
        v[2] = ap.y;
        inst = o.inst_of[c];
    }
    obs_block_add<3>(o, c, inst, v, 0);
}

// pass 2 over cells: squared deviations of q, A, P from their instance means (slots 3-5)
__global__ void __launch_bounds__(256) k_obs_shape_var(ObsArgs o)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    int inst = 0;
    if (c < o.n) {
        inst = o.inst_of[c];
        double2 ap = obs_ap(o, c);
        const double *m = o.mean + 3 * (size_t)inst;
        double dq = ap.y / sqrt(ap.x) - m[0], da = ap.x - m[1], dp = ap.y - m[2];
        v[0] = dq * dq;
        v[1] = da * da;
        v[2] = dp * dp;
    }
    obs_block_add<3>(o, c, inst, v, 3);
}

// over degrees of freedom: squared minimum-image displacement and the overlap count (slots 6-7)
__global__ void __launch_bounds__(256) k_obs_dynamics(ObsArgs o)
{
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    double v[2] = {0.0, 0.0};
    int inst = 0;
    if (d < o.n) {
        inst = o.inst_of[d];
        const Inst &in = o.inst[inst];
        double2 disp = min_dist(o.ref[d], o.pos[d], in.Lx, in.Ly);  // Box->minDist(init, cur, disp)
        double r2 = disp.x * disp.x + disp.y * disp.y;
        v[0] = r2;
        v[1] = sqrt(r2) < o.cutoff ? 1.0 : 0.0;
    }
    obs_block_add<2>(o, d, inst, v, 6);
}

}  // namespace cg

static double2 *obs_ref(cg_system *s, bool alloc)
{
    static_assert(sizeof(double2) == 16, "layout");
    if (!s->obs_ref && alloc) {
        if (dalloc(s, &s->obs_ref, ndof(s)) != CG_OK) return nullptr;
    }
    return s->obs_ref;
}

extern "C" int cg_set_reference_positions(cg_system *s)
{
    if (!s) return set_err(CG_ERR_ARG, "bad args");
    double2 *ref = obs_ref(s, true);
    if (!ref) return CG_ERR_CUDA;
    CG_CUDA(cudaMemcpyAsync(ref, s->pos, sizeof(double2) * ndof(s), cudaMemcpyDeviceToDevice, s->stream));
    return cg_synchronize(s);
}

extern "C" int cg_observables(cg_system *s, double cutoff, double *out)
{
    if (!s || !out) return set_err(CG_ERR_ARG, "bad args");
    if (!s->obs_acc) {
        CG_TRY(dalloc(s, &s->obs_acc, (size_t)s->n_inst * OBS_ACC));
        CG_TRY(dalloc(s, &s->obs_mean, (size_t)s->n_inst * 3));
    }
    const int nI = s->n_inst;
    CG_CUDA(cudaMemsetAsync(s->obs_acc, 0, sizeof(double) * nI * OBS_ACC, s->stream));
    ObsArgs o;
    memset(&o, 0, sizeof(o));
    o.n_inst = nI;
    o.inst = s->inst;
    o.AP = s->AP;
    o.fp64 = s->precision == CG_FP64;
    o.acc = s->obs_acc;
    o.n = s->N;
    o.inst_of = s->cell_inst;
    k_obs_shape<<<nblk(s->N, 256), 256, 0, s->stream>>>(o);
    std::vector<double> acc((size_t)nI * OBS_ACC), mean(3 * (size_t)nI);
    CG_TRY(d2h(s, acc.data(), s->obs_acc, sizeof(double) * acc.size()));
    for (int i = 0; i < nI; ++i)
        for (int j = 0; j < 3; ++j) mean[3 * i + j] = acc[(size_t)i * OBS_ACC + j] / s->h_inst[i].n;
    CG_TRY(h2d(s, s->obs_mean, mean.data(), sizeof(double) * mean.size()));
    o.mean = s->obs_mean;
    k_obs_shape_var<<<nblk(s->N, 256), 256, 0, s->stream>>>(o);
    if (s->obs_ref) {
        o.n = ndof(s);
        o.inst_of = s->model == CG_MODEL_VERTEX ? s->vert_inst : s->cell_inst;
        o.pos = s->pos;
        o.ref = s->obs_ref;
        o.cutoff = cutoff;
        k_obs_dynamics<<<nblk(o.n, 256), 256, 0, s->stream>>>(o);
    }
    s->kernels_enqueued += s->obs_ref ? 3 : 2;
    CG_TRY(check_launch());
    CG_TRY(d2h(s, acc.data(), s->obs_acc, sizeof(double) * acc.size()));
    for (int i = 0; i < nI; ++i) {
        const double n = s->h_inst[i].n;
        const double nd = s->model == CG_MODEL_VERTEX ? 2.0 * n : n;
        const double *a = &acc[(size_t)i * OBS_ACC];
        double *r = out + (size_t)i * CG_OBS_FIELDS;
        r[0] = mean[3 * i];           // mean q
        r[1] = a[3] / n;              // var q
        r[2] = mean[3 * i + 1];       // mean A
        r[3] = mean[3 * i + 2];       // mean P
        r[4] = a[4] / n;              // var A
        r[5] = a[5] / n;              // var P
        r[6] = s->obs_ref ? a[6] / nd : NAN;  // MSD
        r[7] = s->obs_ref ? a[7] / nd : NAN;  // overlap
    }
    return CG_OK;
}
