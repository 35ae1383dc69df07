// cellgpu_b200 -- spatial re-sorting of the cells of a Voronoi batch. Included by system.cu.
//
// Simple2DCell::spatiallySortCells (src/models/Simple2DCell.cpp:438-477) reorders the cells along a
// 2D Hilbert curve so that neighbours sit near each other in memory, and keeps idxToTag /
// tagToIdx to relate the current indices to the original ones. Here every instance is sorted on
// its own (cells stay inside their instance's index range): key = (instance, Hilbert index of
// the cell's position on a 2^16 x 2^16 grid over its box, current index), one device radix sort;
// then every per-cell array is gathered into the new order, neighbour rows are relabelled and
// rotated to start at their smallest neighbour again, and the index -> tag map is updated.
#include <cub/device/device_radix_sort.cuh>

namespace cg {

// Hilbert-curve index of (x, y) on an n x n grid, n a power of two (the classic rotate-and-reflect
// construction: at each scale, the quadrant gives two bits and the frame is turned so the
// sub-curve starts where the previous one ended)
CG_D unsigned hilbert_d(unsigned n, unsigned x, unsigned y)
{
    unsigned d = 0;
    for (unsigned s = n >> 1; s > 0; s >>= 1) {
        unsigned rx = (x & s) ? 1u : 0u, ry = (y & s) ? 1u : 0u;
        d += s * s * ((3u * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) {
                x = n - 1 - x;
                y = n - 1 - y;
            }
            unsigned t = x;
            x = y;
            y = t;
        }
    }
    return d;
}

__global__ void k_sort_keys(int N, const double2 *pos, const Inst *inst, const int *cell_inst,
                            unsigned long long *key, int *idx)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int i = cell_inst[c];
    const Inst &in = inst[i];
    const unsigned n = 1u << 16;
    double fx = pos[c].x * in.iLx, fy = pos[c].y * in.iLy;
    unsigned x = (unsigned)fmin(fmax(fx * n, 0.0), (double)(n - 1));
    unsigned y = (unsigned)fmin(fmax(fy * n, 0.0), (double)(n - 1));
    key[c] = ((unsigned long long)i << 32) | hilbert_d(n, x, y);
    idx[c] = c;
}

// tti[old] = new
__global__ void k_sort_inverse(int N, const int *order, int *tti)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < N) tti[order[c]] = c;
}

template <typename T>
__global__ void k_gather(int N, const int *order, const T *src, T *dst)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < N) dst[c] = src[order[c]];
}

// new row of cell c: the old row of order[c], relabelled through tti and rotated to start at its
// smallest entry (the stored convention)
__global__ void k_gather_rows(int N, int K, const int *order, const int *tti, const int *nn_old,
                              const int *nbr_old, int *nn, int *nbr)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int o = order[c];
    const int z = nn_old[o];
    const int *src = nbr_old + (size_t)o * K;
    int mn = 0x7fffffff, mpos = 0;
    for (int k = 0; k < z; ++k) {
        int v = tti[src[k]];
        if (v < mn) {
            mn = v;
            mpos = k;
        }
    }
    int *dst = nbr + (size_t)c * K;
    for (int k = 0; k < z; ++k) dst[k] = tti[src[(mpos + k) % z]];
    for (int k = z; k < K; ++k) dst[k] = -1;
    nn[c] = z;
}

__global__ void k_iota(int N, int *a)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < N) a[c] = c;
}

}  // namespace cg

// gather a per-cell array of `elem` bytes into the new order through the staging buffer
static int sort_gather(cg_system *s, void *arr, size_t elem, const int *order)
{
    if (!arr) return CG_OK;
    const int N = s->N;
    CG_CUDA(cudaMemcpyAsync(s->sort_tmp, arr, elem * N, cudaMemcpyDeviceToDevice, s->stream));
    if (elem == 16)
        k_gather<double2><<<nblk(N, 256), 256, 0, s->stream>>>(N, order, (const double2 *)s->sort_tmp, (double2 *)arr);
    else if (elem == 8)
        k_gather<double><<<nblk(N, 256), 256, 0, s->stream>>>(N, order, (const double *)s->sort_tmp, (double *)arr);
    else if (elem == 4)
        k_gather<int><<<nblk(N, 256), 256, 0, s->stream>>>(N, order, (const int *)s->sort_tmp, (int *)arr);
    else
        return set_err(CG_ERR_ARG, "unsupported element size");
    s->kernels_enqueued += 1;
    return CG_OK;
}

static int sort_alloc(cg_system *s)
{
    if (s->sort_key) return CG_OK;
    const int N = s->N;
    CG_TRY(dalloc(s, &s->sort_key, 2 * (size_t)N));  // keys in, keys out
    CG_TRY(dalloc(s, &s->sort_idx, 3 * (size_t)N));  // values in, order (values out), tti
    CG_TRY(dalloc(s, (char **)&s->sort_tmp, (size_t)N * std::max<size_t>(16, sizeof(int) * (size_t)(s->K + 1))));
    CG_TRY(dalloc(s, &s->tags, N));
    k_iota<<<nblk(N, 256), 256, 0, s->stream>>>(N, s->tags);
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, s->sort_key, s->sort_key + N, s->sort_idx, s->sort_idx + N, N, 0,
                                    64, s->stream);
    s->sort_tmp_bytes = tb;
    CG_TRY(dalloc(s, (char **)&s->sort_cub, tb));
    return CG_OK;
}

extern "C" int cg_spatial_sort(cg_system *s)
{
    if (!s) return set_err(CG_ERR_ARG, "null system");
    if (s->model != CG_MODEL_VORONOI) return set_err(CG_ERR_STATE, "spatial sorting is for the Voronoi model");
    if (!s->topology_valid) CG_TRY(triangulate_sys(s));
    CG_TRY(sort_alloc(s));
    const int N = s->N;
    int *vals_in = s->sort_idx, *order = s->sort_idx + N, *tti = s->sort_idx + 2 * (size_t)N;
    k_sort_keys<<<nblk(N, 256), 256, 0, s->stream>>>(N, s->pos, s->inst, s->cell_inst, s->sort_key, vals_in);
    CG_CUDA(cub::DeviceRadixSort::SortPairs(s->sort_cub, s->sort_tmp_bytes, s->sort_key, s->sort_key + N, vals_in,
                                            order, N, 0, 64, s->stream));
    k_sort_inverse<<<nblk(N, 256), 256, 0, s->stream>>>(N, order, tti);
    s->kernels_enqueued += 2;
    const size_t r2 = s->precision == CG_FP64 ? sizeof(double2) : sizeof(float2);
    CG_TRY(sort_gather(s, s->pos, sizeof(double2), order));
    CG_TRY(sort_gather(s, s->theta, sizeof(double), order));
    CG_TRY(sort_gather(s, s->motility, sizeof(double2), order));
    CG_TRY(sort_gather(s, s->APpref, sizeof(double2), order));
    CG_TRY(sort_gather(s, s->AP, r2, order));
    CG_TRY(sort_gather(s, s->F, sizeof(double2), order));  // forces are FP64 in every precision
    CG_TRY(sort_gather(s, s->tags, sizeof(int), order));
    if (s->obs_ref) CG_TRY(sort_gather(s, s->obs_ref, sizeof(double2), order));
    if (s->ctype) CG_TRY(sort_gather(s, s->ctype, sizeof(int), order));
    if (s->TE) CG_TRY(sort_gather(s, s->TE, sizeof(double), order));
    if (s->excl) {  // exclusions move with their cells (reIndexCellArray, voronoiModelBase.cpp:679)
        CG_TRY(sort_gather(s, s->excl, sizeof(int), order));
        CG_TRY(sort_gather(s, s->ext_force, sizeof(double2), order));
    }
    // rows: old rows staged in sort_tmp (nn first, then nbr), new rows written in place
    int *nn_old = (int *)s->sort_tmp, *nbr_old = nn_old + N;
    CG_CUDA(cudaMemcpyAsync(nn_old, s->nn, sizeof(int) * N, cudaMemcpyDeviceToDevice, s->stream));
    CG_CUDA(cudaMemcpyAsync(nbr_old, s->nbr, sizeof(int) * (size_t)N * s->K, cudaMemcpyDeviceToDevice, s->stream));
    k_gather_rows<<<nblk(N, 128), 128, 0, s->stream>>>(N, s->K, order, tti, nn_old, nbr_old, s->nn, s->nbr);
    s->kernels_enqueued += 1;
    CG_TRY(check_launch());
    return cg_synchronize(s);
}

extern "C" int cg_get_tags(cg_system *s, int *idx_to_tag)
{
    if (!s || !idx_to_tag) return set_err(CG_ERR_ARG, "bad args");
    if (!s->tags) {
        for (int i = 0; i < s->N; ++i) idx_to_tag[i] = i;
        return CG_OK;
    }
    return d2h(s, idx_to_tag, s->tags, sizeof(int) * s->N);
}
