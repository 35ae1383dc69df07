// cellgpu_b200 -- FIRE minimisation on the device, every instance of a batch independently.
// EnergyMinimizerFIRE::minimize (src/updaters/EnergyMinimizerFIRE2D.cpp:269-284) with the CPU
// conventions of velocityVerletCPU (:120-151) and fireStepCPU (:212-264): forceMax = max |F|^2,
// dt clamped below by dt_min, the mix uses the forces just computed. Per-instance dt, alpha,
// counters and the power / norm reductions live in device memory; an iteration is a handful of
// kernels with no host round trip, and converged instances stop moving. An iteration's kernels:
// k_fire_mix_vv1 (the previous iteration's velocity mix, the first Verlet half, F zeroed), the
// model's topology and force kernels, k_fire_vv2 (second half, sums, and in its last block the
// per-instance update that decides the next mix).

namespace cg {

struct FireInst {
    double dt, alpha;
    double power, fnorm, vnorm;
    unsigned long long fmax_bits;  // max |F|^2 as the bit pattern of a non-negative double
    double fmax;                   // max |F|^2 of the last completed iteration
    double fnorm_last;             // sum |F|^2 of the last completed iteration
    // the FIRE velocity mix that an iteration's update decided, applied by the next iteration's
    // first kernel while mix_seq != mix_done: v <- 0 (mix_zero), else v <- (1 - mix_a) v +
    // mix_a mix_s F (mix_a: alpha before the update, mix_s = sqrt(|v|^2 / |F|^2))
    double mix_a, mix_s;
    int mix_zero, mix_seq, mix_done;
    int n_since, iterations, converged, ndof;
};

constexpr int FIRE_BLOCK = 256;  // threads (= dofs) per block of the per-dof FIRE kernels

struct FireArgs {
    int ndof, n_inst;
    const Inst *inst;
    const int *dof_inst;
    double2 *pos, *vel;
    double2 *F;
    FireInst *st;
    // deterministic mode: the dofs of every instance in chunks of FIRE_BLOCK counted from the
    // instance's first dof (chunk[j] = (instance, first dof); the chunks of instance i are
    // [chunk_off[i], chunk_off[i+1])), and part[3 j ..] = (power, |F|^2, |v|^2) of chunk j, which
    // k_fire_reduce sums per instance in a fixed order; null: atomic sums
    double *part;
    const int2 *chunk;
    const int *chunk_off;
    unsigned *blocks_done;              // finished blocks of k_fire_vv2 (zero between launches)
    unsigned long long *iter_counter;   // executed FIRE iterations (a device counter)
    int zero_f;                         // k_fire_mix_vv1 zeroes F after reading it
    cg_fire_params prm;
    const Ctl *ctl;  // a halted step (pending global rebuild) freezes the iteration
};

// Start of an iteration: the velocity mix that the previous iteration's update decided (with that
// iteration's forces, which F still holds), then the first velocity Verlet half: d = dt v +
// dt^2/2 F ; v += dt/2 F ; move and wrap. With zero_f, F is then zeroed for the force kernels that
// accumulate into it (every dof: the forces of stopped instances are recomputed too).
__global__ void k_fire_mix_vv1(FireArgs a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.ndof) return;
    if (a.ctl && a.ctl->halt) return;
    int inst = a.dof_inst[i];
    const FireInst &st = a.st[inst];
    double2 v = a.vel[i], f = a.F[i];
    bool store_v = false;
    if (st.mix_seq != st.mix_done) {
        if (st.mix_zero) {
            v = make_double2(0.0, 0.0);
        } else {
            double scaling = st.mix_s;
            double al = st.mix_a;
            v.x = (1.0 - al) * v.x + al * scaling * f.x;
            v.y = (1.0 - al) * v.y + al * scaling * f.y;
        }
        store_v = true;
    }
    if (!st.converged) {
        const Inst &in = a.inst[inst];
        double dt = st.dt;
        double dx = __dadd_rn(__dmul_rn(dt, v.x), __dmul_rn(__dmul_rn(__dmul_rn(0.5, dt), dt), f.x));
        double dy = __dadd_rn(__dmul_rn(dt, v.y), __dmul_rn(__dmul_rn(__dmul_rn(0.5, dt), dt), f.y));
        v.x = __dadd_rn(v.x, __dmul_rn(__dmul_rn(0.5, dt), f.x));
        v.y = __dadd_rn(v.y, __dmul_rn(__dmul_rn(0.5, dt), f.y));
        store_v = true;
        double2 p = a.pos[i];
        p.x = __dadd_rn(p.x, dx);
        p.y = __dadd_rn(p.y, dy);
        a.pos[i] = put_in_box(p, in.Lx, in.Ly, in.iLx, in.iLy);
    }
    if (store_v) a.vel[i] = v;
    if (a.zero_f) a.F[i] = make_double2(0.0, 0.0);
}

// End of an iteration for one instance whose sums are complete (fireStepCPU's decisions): the mix
// for the next iteration's first kernel, with the alpha before this update; dt / alpha / N_since;
// the iteration count and the convergence test of the loop head; the sums are cleared for the next
// iteration. The mix that the previous update decided has been applied by now (mix_done).
// The state is read with L2 loads issued together (the last block of k_fire_vv2 reads sums that
// other blocks added, which its L1 may hold stale), updated in registers and stored back.
CG_D void fire_update(FireInst *sp, const cg_fire_params &p, unsigned long long *iter_counter)
{
    FireInst st;
    st.dt = __ldcg(&sp->dt);
    st.alpha = __ldcg(&sp->alpha);
    st.power = __ldcg(&sp->power);
    st.fnorm = __ldcg(&sp->fnorm);
    st.vnorm = __ldcg(&sp->vnorm);
    st.fmax_bits = __ldcg(&sp->fmax_bits);
    st.fmax = __ldcg(&sp->fmax);
    st.fnorm_last = __ldcg(&sp->fnorm_last);
    st.mix_a = __ldcg(&sp->mix_a);
    st.mix_s = __ldcg(&sp->mix_s);
    st.mix_zero = __ldcg(&sp->mix_zero);
    st.mix_seq = __ldcg(&sp->mix_seq);
    st.mix_done = __ldcg(&sp->mix_done);
    st.n_since = __ldcg(&sp->n_since);
    st.iterations = __ldcg(&sp->iterations);
    st.converged = __ldcg(&sp->converged);
    st.ndof = __ldcg(&sp->ndof);
    st.mix_done = st.mix_seq;
    if (!st.converged) {
        st.mix_zero = !(st.power > 0) ? 1 : 0;
        st.mix_s = st.fnorm > 0. ? sqrt(st.vnorm / st.fnorm) : 0.0;
        st.mix_a = st.alpha;
        st.mix_seq += 1;
        st.iterations += 1;
        atomicAdd(iter_counter, 1ull);
        if (st.power > 0) {
            if (st.n_since > p.n_min) {
                st.dt = fmin(st.dt * p.dt_inc, p.dt_max);
                st.alpha = st.alpha * p.alpha_dec;
            }
            st.n_since += 1;
        } else {
            st.dt = st.dt * p.dt_dec;
            st.dt = fmax(st.dt, p.dt_min);
            st.alpha = p.alpha_start;
        }
        st.fmax = __longlong_as_double((long long)st.fmax_bits);
        st.fnorm_last = st.fnorm;
        st.converged = !(st.iterations < p.max_iterations && sqrt(st.fmax) > p.force_cutoff);
        st.power = 0;
        st.fnorm = 0;
        st.vnorm = 0;
        st.fmax_bits = 0;
    }
    *sp = st;
}

// second half-kick with the new forces, then the FIRE reductions per instance. Degrees of freedom
// of one instance are contiguous: a block that lies inside one (unconverged) instance reduces in
// shared memory and adds once per quantity; other blocks reduce per warp where the warp is uniform
// and per lane otherwise. (Launched with 256 threads.)
__global__ void __launch_bounds__(256) k_fire_vv2(FireArgs a)
{
    __shared__ double s_red[4][8];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (a.ctl && a.ctl->halt) return;  // uniform across the grid
    int inst = -1;
    double P = 0, ff = 0, vv = 0, fm = 0;
    if (i < a.ndof) {
        inst = a.dof_inst[i];
        const FireInst &st = a.st[inst];
        if (!st.converged) {
            double dt = st.dt;
            double2 v = a.vel[i], f = a.F[i];
            v.x = __dadd_rn(v.x, __dmul_rn(__dmul_rn(0.5, dt), f.x));
            v.y = __dadd_rn(v.y, __dmul_rn(__dmul_rn(0.5, dt), f.y));
            a.vel[i] = v;
            P = f.x * v.x + f.y * v.y;
            ff = f.x * f.x + f.y * f.y;
            vv = v.x * v.x + v.y * v.y;
            fm = ff;
        } else {
            inst = -1;
        }
    }
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int d0 = blockIdx.x * blockDim.x, d1 = min(a.ndof, d0 + (int)blockDim.x) - 1;
    const int b0 = a.dof_inst[d0], b1 = a.dof_inst[d1];
    if (b0 == b1 && !a.st[b0].converged) {  // uniform across the block
        for (int off = 16; off > 0; off >>= 1) {
            P += __shfl_down_sync(full, P, off);
            ff += __shfl_down_sync(full, ff, off);
            vv += __shfl_down_sync(full, vv, off);
            fm = fmax(fm, __shfl_down_sync(full, fm, off));
        }
        if (lane == 0) {
            s_red[0][w] = P;
            s_red[1][w] = ff;
            s_red[2][w] = vv;
            s_red[3][w] = fm;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double tp = 0, tf = 0, tv = 0, tm = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
                tp += s_red[0][k];
                tf += s_red[1][k];
                tv += s_red[2][k];
                tm = fmax(tm, s_red[3][k]);
            }
            atomicAdd(&a.st[b0].power, tp);
            atomicAdd(&a.st[b0].fnorm, tf);
            atomicAdd(&a.st[b0].vnorm, tv);
            atomicMax(&a.st[b0].fmax_bits, (unsigned long long)__double_as_longlong(tm));
        }
    } else if (__all_sync(full, inst == __shfl_sync(full, inst, 0))) {
        // warp-level segmented reduction (lanes of one instance are contiguous)
        for (int off = 16; off > 0; off >>= 1) {
            P += __shfl_down_sync(full, P, off);
            ff += __shfl_down_sync(full, ff, off);
            vv += __shfl_down_sync(full, vv, off);
            fm = fmax(fm, __shfl_down_sync(full, fm, off));
        }
        if (lane == 0 && inst >= 0) {
            atomicAdd(&a.st[inst].power, P);
            atomicAdd(&a.st[inst].fnorm, ff);
            atomicAdd(&a.st[inst].vnorm, vv);
            atomicMax(&a.st[inst].fmax_bits, (unsigned long long)__double_as_longlong(fm));
        }
    } else if (inst >= 0) {
        atomicAdd(&a.st[inst].power, P);
        atomicAdd(&a.st[inst].fnorm, ff);
        atomicAdd(&a.st[inst].vnorm, vv);
        atomicMax(&a.st[inst].fmax_bits, (unsigned long long)__double_as_longlong(fm));
    }
    // the last block to finish updates every instance (threadfence reduction: each block's sums
    // are visible before its count is)
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(a.blocks_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int k = threadIdx.x; k < a.n_inst; k += blockDim.x) fire_update(a.st + k, a.prm, a.iter_counter);
    if (threadIdx.x == 0) *a.blocks_done = 0;
}

// Deterministic mode, second half-kick: one block per chunk (FireArgs::chunk), so a block holds
// the same dofs of its instance wherever the instance sits in the batch, and its partial sums
// (a fixed shuffle tree, then the warps in order) depend on the instance alone. max |F|^2 is an
// integer maximum of bit patterns, exact in any order.
__global__ void __launch_bounds__(FIRE_BLOCK) k_fire_vv2_chunks(FireArgs a)
{
    __shared__ double s_red[3][FIRE_BLOCK / 32];
    if (a.ctl && a.ctl->halt) return;  // uniform across the grid
    const int2 ch = a.chunk[blockIdx.x];
    const FireInst &st = a.st[ch.x];
    if (st.converged) return;  // uniform across the block
    const Inst &in = a.inst[ch.x];
    const int end = in.nv > 0 ? in.voff + in.nv : in.off + in.n;
    const int i = ch.y + threadIdx.x;
    double P = 0, ff = 0, vv = 0, fm = 0;
    if (i < end) {
        const double dt = st.dt;
        double2 v = a.vel[i], f = a.F[i];
        v.x = __dadd_rn(v.x, __dmul_rn(__dmul_rn(0.5, dt), f.x));
        v.y = __dadd_rn(v.y, __dmul_rn(__dmul_rn(0.5, dt), f.y));
        a.vel[i] = v;
        P = f.x * v.x + f.y * v.y;
        ff = f.x * f.x + f.y * f.y;
        vv = v.x * v.x + v.y * v.y;
        fm = ff;
    }
    const unsigned full = 0xffffffffu;
    for (int off = 16; off > 0; off >>= 1) {
        P += __shfl_down_sync(full, P, off);
        ff += __shfl_down_sync(full, ff, off);
        vv += __shfl_down_sync(full, vv, off);
        fm = fmax(fm, __shfl_down_sync(full, fm, off));
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        s_red[0][w] = P;
        s_red[1][w] = ff;
        s_red[2][w] = vv;
        atomicMax(&a.st[ch.x].fmax_bits, (unsigned long long)__double_as_longlong(fm));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tp = 0, tf = 0, tv = 0;
        for (int k = 0; k < FIRE_BLOCK / 32; ++k) {
            tp += s_red[0][k];
            tf += s_red[1][k];
            tv += s_red[2][k];
        }
        a.part[3 * (size_t)blockIdx.x] = tp;
        a.part[3 * (size_t)blockIdx.x + 1] = tf;
        a.part[3 * (size_t)blockIdx.x + 2] = tv;
    }
}

// Deterministic mode: the power and norm sums of every unconverged instance (one block per
// instance) from its chunks' partial sums, thread t taking chunks t, t + FIRE_BLOCK, ... in order,
// then the fixed tree. The order depends on the instance's dof count alone, so the sums are
// bit-identical on every run and in every batch that holds the instance.
__global__ void __launch_bounds__(FIRE_BLOCK) k_fire_reduce(FireArgs a)
{
    __shared__ double s_red[3][FIRE_BLOCK / 32];
    if (a.ctl && a.ctl->halt) return;  // uniform across the grid
    FireInst &st = a.st[blockIdx.x];
    if (st.converged) {  // uniform across the block
        if (threadIdx.x == 0) fire_update(&st, a.prm, a.iter_counter);  // (acknowledges the last mix)
        return;
    }
    const int j0 = a.chunk_off[blockIdx.x], j1 = a.chunk_off[blockIdx.x + 1];
    double P = 0, ff = 0, vv = 0;
    for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        const double *q = a.part + 3 * (size_t)j;
        P += q[0];
        ff += q[1];
        vv += q[2];
    }
    const unsigned full = 0xffffffffu;
    for (int off = 16; off > 0; off >>= 1) {
        P += __shfl_down_sync(full, P, off);
        ff += __shfl_down_sync(full, ff, off);
        vv += __shfl_down_sync(full, vv, off);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        s_red[0][w] = P;
        s_red[1][w] = ff;
        s_red[2][w] = vv;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tp = 0, tf = 0, tv = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            tp += s_red[0][k];
            tf += s_red[1][k];
            tv += s_red[2][k];
        }
        st.power = tp;
        st.fnorm = tf;
        st.vnorm = tv;
        fire_update(&st, a.prm, a.iter_counter);
    }
}

__global__ void k_fire_init(FireArgs a, int lo, int hi)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.ndof) {
        const int d = a.dof_inst[i];
        if (d >= lo && d < hi) a.vel[i] = make_double2(0.0, 0.0);
    }
    if (i >= lo && i < hi) {
        FireInst s;
        s.dt = a.prm.dt;
        s.alpha = a.prm.alpha_start;
        s.power = s.fnorm = s.vnorm = 0;
        s.fmax_bits = 0;
        s.fmax = 110.0;  // minimize() starts the loop with forceMax = 110
        s.fnorm_last = 0;
        s.mix_a = s.mix_s = 0;
        s.mix_zero = s.mix_seq = s.mix_done = 0;
        s.n_since = 0;
        s.iterations = 0;
        s.converged = !(0 < a.prm.max_iterations && sqrt(110.0) > a.prm.force_cutoff);
        s.ndof = a.inst[i].nv > 0 ? a.inst[i].nv : a.inst[i].n;
        a.st[i] = s;
    }
}

}  // namespace cg
