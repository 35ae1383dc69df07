// cellgpu_b200 -- particle exclusions of the Voronoi model (voronoiModelBase::setExclusions,
// src/models/voronoiModelBase.cpp:85-104). Included by system.cu.
//
// An excluded cell gets zero motility (v0 = Dr = 0) when the exclusions are set, and after every
// force evaluation its net force is moved to the external force (-F) and F is zeroed, as the
// reference's force summation with exclusions does (src/models/voronoiQuadraticEnergy.cpp:119-135,
// 368-377). The flags travel with the cells through spatial sorting (reIndexCellArray(exclusions),
// src/models/voronoiModelBase.cpp:679) and are stored in snapshots.

__global__ void k_exclusion_motility(int N, const int *excl, double2 *motility)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < N && excl[c]) motility[c] = make_double2(0.0, 0.0);
}

extern "C" int cg_set_exclusions(cg_system *s, const int *excluded)
{
    if (!s || s->model != CG_MODEL_VORONOI) return set_err(CG_ERR_ARG, "exclusions need a Voronoi system");
    if (!s->excl) {
        CG_TRY(dalloc(s, &s->excl, s->N));  // zeroed
        CG_TRY(dalloc(s, &s->ext_force, s->N));
    }
    std::vector<int> flags(s->N, 0);
    int n = 0;
    if (excluded)
        for (int i = 0; i < s->N; ++i) {
            flags[i] = excluded[i] != 0;
            n += flags[i];
        }
    CG_TRY(h2d(s, s->excl, flags.data(), sizeof(int) * s->N));
    CG_CUDA(cudaMemsetAsync(s->ext_force, 0, sizeof(double2) * s->N, s->stream));
    if (n > 0) {
        k_exclusion_motility<<<nblk(s->N, 256), 256, 0, s->stream>>>(s->N, s->excl, s->motility);
        CG_TRY(check_launch());
    }
    s->n_excl = n;
    drop_graphs(s);  // step graphs hold (or lack) the exclusion kernel
    return cg_synchronize(s);
}

extern "C" int cg_get_external_forces(cg_system *s, double *out)
{
    if (!s || !out || s->model != CG_MODEL_VORONOI) return set_err(CG_ERR_ARG, "bad args");
    if (!s->ext_force) {
        memset(out, 0, sizeof(double) * 2 * (size_t)s->N);
        return CG_OK;
    }
    return d2h(s, out, s->ext_force, sizeof(double2) * s->N);
}
