// cellgpu_b200 -- periodic Delaunay triangulation without any allocation.
//
// cg_voronoi_triangulate() builds a temporary system and therefore calls cudaMalloc/cudaFree. Some
// callers cannot do that: host applications that hand the library a fixed device-memory budget up
// front (pre-partitioned memory, or another framework's caching allocator that owns the heap),
// loops where cudaFree's implicit device synchronisation stalls every stream, and threads that run
// while another thread captures a CUDA graph in global mode (allocation is an illegal call for every
// thread then). cg_voronoi_triangulate_noalloc() serves them: its scratch (the cell list, the
// prefix-sum workspace and the status words) is one file-scope __device__ array of fixed size that
// every GPU which loads this library reserves until the process exits.
//
// Limits: at most CG_NOALLOC_MAX_CELLS cells and CG_NOALLOC_MAX_BINS cell-list bins (bins are
// about 0.8 x 0.8 in box units, so a box of area A uses about 1.56 A bins).
//
// Rules for callers:
//  * The call is synchronous: it reads the status words back on `stream` and waits for them, so it
//    cannot be captured into a graph. Beside another thread's global-mode capture, pass a
//    cudaStreamNonBlocking stream (the legacy default stream synchronises with capturing streams).
//  * The first call on a device resolves the array's device address with cudaGetSymbolAddress
//    (with that device current) and sizes the scan workspace.
//  * Every call uses the same array and leaves the previous call's contents in it; each call
//    clears what has to start at zero. Calls that overlap on the GPU (two streams, two threads, or
//    two devices' worth of work aimed at the same device) race on the array: serialise them.
#include <mutex>

namespace cg_noalloc {

constexpr int MAX_CELLS = CG_NOALLOC_MAX_CELLS;
constexpr int MAX_BINS = CG_NOALLOC_MAX_BINS;
constexpr size_t SCAN_BYTES = 64 << 10;  // prefix-sum workspace reserved for MAX_BINS + 1 counts

// byte layout of the array (every piece 256-byte aligned)
constexpr size_t al(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t OFF_BIN_COUNT = 0;
constexpr size_t OFF_BIN_START = OFF_BIN_COUNT + al(sizeof(int) * (MAX_BINS + 1));
constexpr size_t OFF_BIN_CELLS = OFF_BIN_START + al(sizeof(int) * (MAX_BINS + 1));
constexpr size_t OFF_CELL_BIN = OFF_BIN_CELLS + al(sizeof(int) * MAX_CELLS);
constexpr size_t OFF_CELL_SLOT = OFF_CELL_BIN + al(sizeof(int) * MAX_CELLS);
constexpr size_t OFF_BIN_POS = OFF_CELL_SLOT + al(sizeof(int) * MAX_CELLS);
constexpr size_t OFF_STATUS = OFF_BIN_POS + al(sizeof(double2) * MAX_CELLS);
constexpr size_t OFF_ZSUM = OFF_STATUS + al(sizeof(int) * 4);
constexpr size_t OFF_SCAN = OFF_ZSUM + al(sizeof(unsigned long long));
constexpr size_t TOTAL = OFF_SCAN + al(SCAN_BYTES);

static __device__ __align__(256) unsigned char g_tri_scratch[TOTAL];

constexpr int MAX_DEVICES = 64;
static void *g_dev_addr[MAX_DEVICES];
static std::mutex g_setup_mutex;

// triangle-consistency and Euler count of one triangulation. status[0] is the star kernel's word:
// when it reports a failure, rows may be missing or still hold the caller's old contents, so no row
// is read. bad is set on an inconsistency. Every length and index is checked before it is used, so
// rows that hold arbitrary values cannot send a read outside the caller's buffers.
__global__ void k_validate_one(cg::VoroArgs a, const int *status, int *bad, unsigned long long *zsum)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.N || *status != 0) return;
    const int *row = a.nbr + (size_t)c * a.K;
    int z = a.nn[c];
    if (z < 3 || z > a.K) {
        atomicCAS(bad, 0, CG_ERR_TOPOLOGY);
        return;
    }
    atomicAdd(zsum, (unsigned long long)z);
    for (int k = 0; k < z; ++k) {
        int u = row[k], v = row[(k + 1) % z];
        bool ok = u >= 0 && u < a.N && v >= 0 && v < a.N;
        if (ok) {
            int zu = a.nn[u], zv = a.nn[v];
            ok = zu >= 3 && zu <= a.K && zv >= 3 && zv <= a.K &&
                 cg::row_has_pair(a.nbr + (size_t)u * a.K, zu, v, c) &&
                 cg::row_has_pair(a.nbr + (size_t)v * a.K, zv, c, u);
        }
        if (!ok) {
            atomicCAS(bad, 0, CG_ERR_TOPOLOGY);
            return;
        }
    }
}

// once per device, with that device current
static int setup(void **addr)
{
    int dev = 0;
    CG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return set_err(CG_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_dev_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_tri_scratch);
        if (e != cudaSuccess)
            return set_err(CG_ERR_CUDA, (std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)).c_str());
        size_t need = 0;
        int *dummy = reinterpret_cast<int *>(p);
        e = cub::DeviceScan::ExclusiveSum(nullptr, need, dummy, dummy, MAX_BINS + 1);
        if (e != cudaSuccess) return set_err(CG_ERR_CUDA, cudaGetErrorString(e));
        if (need > SCAN_BYTES) return set_err(CG_ERR_CAPACITY, "scan workspace larger than reserved");
        g_dev_addr[dev] = p;
    }
    *addr = g_dev_addr[dev];
    return CG_OK;
}

}  // namespace cg_noalloc

static int triangulate_noalloc(const double *pos, int N, double Lx, double Ly, int K, int *nn, int *nbr,
                               cudaStream_t stream)
{
    using namespace cg_noalloc;
    if (!pos || !nn || !nbr || N < 8 || K < 4 || K > KMAX || !(Lx > 0) || !(Ly > 0))
        return set_err(CG_ERR_ARG, "bad args");
    if (N > MAX_CELLS) return set_err(CG_ERR_CAPACITY, "N exceeds CG_NOALLOC_MAX_CELLS");
    Inst in = make_inst(Lx, Ly, 0, N, 0, BIN_TARGET);
    if ((long long)in.nbx * in.nby > MAX_BINS)
        return set_err(CG_ERR_CAPACITY, "the box needs more cell-list bins than CG_NOALLOC_MAX_BINS");
    void *base = nullptr;
    CG_TRY(setup(&base));
    unsigned char *b = reinterpret_cast<unsigned char *>(base);
    VoroArgs a;
    memset(&a, 0, sizeof(a));
    a.N = N;
    a.K = K;
    a.n_inst = 1;
    a.inst0 = in;
    a.pos = (double2 *)pos;
    a.nn = nn;
    a.nbr = nbr;
    a.bin_count = reinterpret_cast<int *>(b + OFF_BIN_COUNT);
    a.bin_start = reinterpret_cast<int *>(b + OFF_BIN_START);
    a.bin_cells = reinterpret_cast<int *>(b + OFF_BIN_CELLS);
    a.cell_bin = reinterpret_cast<int *>(b + OFF_CELL_BIN);
    a.cell_slot = reinterpret_cast<int *>(b + OFF_CELL_SLOT);
    a.bin_pos = reinterpret_cast<double2 *>(b + OFF_BIN_POS);
    a.n_bins = in.nbx * in.nby;
    int *status = reinterpret_cast<int *>(b + OFF_STATUS);
    unsigned long long *zsum = reinterpret_cast<unsigned long long *>(b + OFF_ZSUM);
    void *scan_tmp = b + OFF_SCAN;
    size_t scan_bytes = SCAN_BYTES;
    // what must start at zero: bin counts, status words, the coordination sum
    CG_CUDA(cudaMemsetAsync(a.bin_count, 0, sizeof(int) * (a.n_bins + 1), stream));
    CG_CUDA(cudaMemsetAsync(status, 0, sizeof(int) * 4, stream));
    CG_CUDA(cudaMemsetAsync(zsum, 0, sizeof(unsigned long long), stream));
    k_bin_count<<<nblk(N, 256), 256, 0, stream>>>(a);
    CG_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, a.bin_count, a.bin_start, a.n_bins + 1, stream));
    k_bin_scatter<<<nblk(N, 256), 256, 0, stream>>>(a);
    constexpr int WPB = 4;
    k_star_global<WPB><<<nblk(N, WPB), WPB * 32, 0, stream>>>(a, status);
    k_validate_one<<<nblk(N, 256), 256, 0, stream>>>(a, status, status + 1, zsum);
    CG_TRY(check_launch());
    int h_status[2] = {0, 0};
    unsigned long long h_zsum = 0;
    CG_CUDA(cudaMemcpyAsync(h_status, status, sizeof(int) * 2, cudaMemcpyDeviceToHost, stream));
    CG_CUDA(cudaMemcpyAsync(&h_zsum, zsum, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream));
    CG_CUDA(cudaStreamSynchronize(stream));
    if (h_status[0]) return set_err(h_status[0], h_status[0] == CG_ERR_CAPACITY ? "neighbour capacity exceeded"
                                                                                 : "triangulation failed");
    if (h_status[1]) return set_err(CG_ERR_TOPOLOGY, "triangulation is not consistent");
    if (h_zsum != 6ull * (unsigned long long)N)
        return set_err(CG_ERR_TOPOLOGY, "Euler check failed (sum of coordinations != 6N)");
    return CG_OK;
}

extern "C" int cg_voronoi_triangulate_noalloc(const double *pos, int N, double Lx, double Ly, int K, int *nn,
                                              int *nbr, cudaStream_t stream)
{
    // This thread's calls (the status read-back waits on `stream`) would otherwise count as unsafe
    // while another thread captures in global mode, and invalidate that capture; in thread-local
    // mode other threads' captures are ignored. `stream` must then not be the legacy default stream,
    // which synchronises with capturing streams. The caller's mode is restored on return.
    cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
    CG_CUDA(cudaThreadExchangeStreamCaptureMode(&mode));
    const int st = triangulate_noalloc(pos, N, Lx, Ly, K, nn, nbr, stream);
    cudaThreadExchangeStreamCaptureMode(&mode);
    return st;
}
