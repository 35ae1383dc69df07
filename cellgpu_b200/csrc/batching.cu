// cellgpu_b200 -- moving running instances between systems, for continuous batching. Included by
// system.cu. No counterpart in the reference (one monolayer per process there).
//
// A serving batch is one system holding many instances. When some of them finish and requests
// wait, the server builds a new system of the still-running instances plus the new ones: the
// running instances move with cg_copy_instances (their whole state: positions, directors,
// preferences, motility, forces, topology, FIRE state, line-tension and exclusion data, noise key
// and step count) and continue exactly where they were, while the new ones start fresh.

// dst[i] = src[i] + delta for entries >= 0 (row padding and "none" markers stay negative)
__global__ void k_copy_shift(long long n, const int *src, int *dst, int delta)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int v = src[i];
    dst[i] = v >= 0 ? v + delta : v;
}

// rows of width Ks into rows of width Kd (Kd >= Ks, padded with -1), entries shifted by delta
__global__ void k_copy_rows(int rows, int Ks, int Kd, const int *src, int *dst, int delta)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    for (int k = 0; k < Kd; ++k) {
        const int v = k < Ks ? src[(size_t)r * Ks + k] : -1;
        dst[(size_t)r * Kd + k] = v >= 0 ? v + delta : v;
    }
}

template <typename T>
static int dd_copy(cg_system *d, T *dst, const T *src, size_t count)
{
    if (count == 0) return CG_OK;
    CG_CUDA(cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyDeviceToDevice, d->stream));
    return CG_OK;
}

extern "C" int cg_copy_instances(cg_system *dst, int dst_first, cg_system *src, int src_first, int count)
{
    if (!dst || !src || dst == src || count <= 0 || dst_first < 0 || src_first < 0 ||
        dst_first + count > dst->n_inst || src_first + count > src->n_inst)
        return set_err(CG_ERR_ARG, "bad instance range");
    if (dst->model != src->model || dst->precision != src->precision || dst->det != src->det)
        return set_err(CG_ERR_ARG, "systems differ in model, precision or summation mode");
    if (dst->model == CG_MODEL_VERTEX && dst->vmax != src->vmax)
        return set_err(CG_ERR_ARG, "vertex systems differ in vmax");
    for (int i = 0; i < count; ++i) {
        const Inst &a = src->h_inst[src_first + i], &b = dst->h_inst[dst_first + i];
        if (a.n != b.n || a.Lx != b.Lx || a.Ly != b.Ly) return set_err(CG_ERR_ARG, "instance sizes or boxes differ");
    }
    if (dst->model == CG_MODEL_VORONOI && src->K > dst->K) CG_TRY(grow_rows(dst));
    // the source's state must be complete before the copies (which run on dst's stream) read it
    CG_CUDA(cudaStreamSynchronize(src->stream));
    Ctl cs, cd;
    CG_TRY(read_ctl(src, cs));
    CG_TRY(read_ctl(dst, cd));
    const Inst &s0 = src->h_inst[src_first], &d0 = dst->h_inst[dst_first];
    int nc = 0, nv = 0;
    for (int i = 0; i < count; ++i) {
        nc += src->h_inst[src_first + i].n;
        nv += src->h_inst[src_first + i].nv;
    }
    const int cs0 = s0.off, cd0 = d0.off, dc = cd0 - cs0;
    const size_t r2 = dst->precision == CG_FP64 ? sizeof(double2) : sizeof(float2);
    CG_TRY(dd_copy(dst, dst->APpref + cd0, src->APpref + cs0, nc));
    CG_TRY(dd_copy(dst, dst->motility + cd0, src->motility + cs0, nc));
    CG_TRY(dd_copy(dst, dst->theta + cd0, src->theta + cs0, nc));
    CG_TRY(dd_copy(dst, (char *)dst->AP + r2 * cd0, (const char *)src->AP + r2 * cs0, r2 * nc));
    if (dst->model == CG_MODEL_VORONOI) {
        CG_TRY(dd_copy(dst, dst->pos + cd0, src->pos + cs0, nc));
        CG_TRY(dd_copy(dst, (char *)dst->F + 16 * cd0, (const char *)src->F + 16 * cs0, 16 * nc));  // FP64
        CG_TRY(dd_copy(dst, dst->nn + cd0, src->nn + cs0, nc));
        k_copy_rows<<<nblk(nc, 256), 256, 0, dst->stream>>>(nc, src->K, dst->K, src->nbr + (size_t)cs0 * src->K,
                                                          dst->nbr + (size_t)cd0 * dst->K, dc);
        CG_TRY(check_launch());
        if (src->excl) {
            if (!dst->excl) {
                CG_TRY(dalloc(dst, &dst->excl, dst->N));
                CG_TRY(dalloc(dst, &dst->ext_force, dst->N));
            }
            CG_TRY(dd_copy(dst, dst->excl + cd0, src->excl + cs0, nc));
            CG_TRY(dd_copy(dst, dst->ext_force + cd0, src->ext_force + cs0, nc));
            std::vector<int> fl(dst->N);
            CG_TRY(d2h(dst, fl.data(), dst->excl, sizeof(int) * dst->N));
            dst->n_excl = 0;
            for (int f : fl) dst->n_excl += f != 0;
        }
    } else {
        const int vs0 = s0.voff, vd0 = d0.voff, dv = vd0 - vs0;
        CG_TRY(dd_copy(dst, dst->pos + vd0, src->pos + vs0, nv));
        CG_TRY(dd_copy(dst, (char *)dst->F + 16 * vd0, (const char *)src->F + 16 * vs0, 16 * nv));
        k_copy_shift<<<nblk(3 * nv, 256), 256, 0, dst->stream>>>(3ll * nv, src->vn + 3 * (size_t)vs0,
                                                                  dst->vn + 3 * (size_t)vd0, dv);
        k_copy_shift<<<nblk(3 * nv, 256), 256, 0, dst->stream>>>(3ll * nv, src->vcn + 3 * (size_t)vs0,
                                                                  dst->vcn + 3 * (size_t)vd0, dc);
        k_copy_shift<<<nblk((long long)nc * src->vmax, 256), 256, 0, dst->stream>>>(
            (long long)nc * src->vmax, src->cv + (size_t)cs0 * src->vmax, dst->cv + (size_t)cd0 * dst->vmax, dv);
        CG_TRY(check_launch());
        CG_TRY(dd_copy(dst, dst->cvn + cd0, src->cvn + cs0, nc));
    }
    if (src->ctype) {
        CG_TRY(tension_alloc(dst));
        CG_TRY(dd_copy(dst, dst->ctype + cd0, src->ctype + cs0, nc));
    }
    if (src->fire_st) {
        CG_TRY(fire_alloc(dst));
        const int f0 = dst->model == CG_MODEL_VORONOI ? cd0 : d0.voff;
        const int g0 = src->model == CG_MODEL_VORONOI ? cs0 : s0.voff;
        CG_TRY(dd_copy(dst, dst->fire_vel + f0, src->fire_vel + g0, dst->model == CG_MODEL_VORONOI ? nc : nv));
        CG_TRY(dd_copy(dst, reinterpret_cast<FireInst *>(dst->fire_st) + dst_first,
                       reinterpret_cast<const FireInst *>(src->fire_st) + src_first, count));
    }
    // noise keys, and step offsets that keep each instance's noise counters running on
    for (int i = 0; i < count; ++i) {
        const Inst &a = src->h_inst[src_first + i];
        Inst &b = dst->h_inst[dst_first + i];
        b.seed = a.seed;
        b.step_off = (unsigned)cs.step + a.step_off - (unsigned)cd.step;
    }
    CG_TRY(upload_inst(dst));
    return cg_synchronize(dst);
}
