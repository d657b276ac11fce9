// Persistent multigrid: V-cycles (or a whole solve to tolerance) in one
// cooperative launch.
//
// The per-level schedule is the one of the launch-per-kernel path in mg.cu
// (mac/mg_workspace.py:85-102 with the gauge carried as pending shifts), but
// every kernel boundary becomes a grid barrier inside one kernel, so a
// V-cycle on 64^3 costs about 22 barriers instead of 22 launches, and in solve
// mode the residual-norm checks of mac/multigrid.py:75-98 run on the device,
// leaving one host read per solve.
//
// Launch: cooperative, one 1024-thread block per SM, so every block is
// resident and the barrier can wait.  Each barrier waits with a clock-bounded
// spin (about one second); a barrier that times out sets the error word, every
// later barrier returns at once, the kernel exits and the host raises.  The
// levels with at most kCoarseCells cells run in block 0's shared memory
// (coarse_cycle) while the other blocks wait at the next barrier.
//
// Reductions (means of the gauge, the residual norm) travel with the barrier:
// each block deposits its partial, the last block to arrive sums the partials
// in block order and publishes the total before releasing the others, so
// every block reads the same deterministic value.
#include <algorithm>
#include "mg_ops.cuh"

namespace afsi {

constexpr int kPThreads = 1024;

struct Tiling {  // a 1024-thread block covers bx * by * bz cells (powers of two)
    int bxl, byl, bzl;
    int gx, gy, gz;
};

constexpr int kNormSlot = AFSI_MG_MAX_LEVELS * 3;

template <class T, class TC>
struct PersistentArgs {
    Lv<T> lv[AFSI_MG_MAX_LEVELS];
    Tiling tl[AFSI_MG_MAX_LEVELS];
    T* P[AFSI_MG_MAX_LEVELS];
    T* Q[AFSI_MG_MAX_LEVELS];
    T* R[AFSI_MG_MAX_LEVELS];
    CoarseLevels<T> coarse;
    const TC* cinv;
    GridSync gs;
    int levels, first_coarse, smooth;
    int solve;        // 0: run `cycles` V-cycles; 1: solve to `tol` (at most `cycles`)
    int cycles, check_every;
    double tol;
    double* info;     // solve: {cycles, residual norm, status}
};


// Cells of this block in virtual-block order; f(x, y, z, i).
template <int BC, class T, class F>
__device__ __forceinline__ void for_cells(const Tiling& t, const Lv<T>& L, F f) {
    const int tx = threadIdx.x & ((1 << t.bxl) - 1);
    const int ty = (threadIdx.x >> t.bxl) & ((1 << t.byl) - 1);
    const int tz = threadIdx.x >> (t.bxl + t.byl);
    const int nv = t.gx * t.gy * t.gz;
    for (int v = blockIdx.x; v < nv; v += gridDim.x) {
        const int vx = v % t.gx, r = v / t.gx, vy = r % t.gy, vz = r / t.gy;
        const int fast = (vx << t.bxl) + tx, mid = (vy << t.byl) + ty, slow = (vz << t.bzl) + tz;
        int x, y, z;
        if (is3d(BC)) {
            z = fast; y = mid; x = slow;
            if (z >= L.nz || y >= L.ny || x >= L.nx) continue;
        } else {
            y = fast; x = mid; z = 0;
            if (y >= L.ny || x >= L.nx || slow > 0) continue;
        }
        f(x, y, z, index_of(x, y, z, L));
    }
}

__device__ __forceinline__ double block_total(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    if (warp == 0) v = warp_sum(v);
    __syncthreads();
    return v;
}

template <int BC, class T, class TC>
__global__ void __launch_bounds__(kPThreads, 1) mg_persistent(PersistentArgs<T, TC> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[32];
    constexpr bool singular = singular_bc(BC);
    const GridSync& gs = a.gs;
    const int fc = a.first_coarse;
    T* down[AFSI_MG_MAX_LEVELS];
    bool ok = true;
    int done = 0;
    double residual = -1.0;
    for (int cycle = 0; cycle < a.cycles && ok; ++cycle) {
        // ---- down legs of the grid levels
        for (int l = 0; l < fc && ok; ++l) {
            const Lv<T>& L = a.lv[l];
            T* cur = a.P[l];
            T* oth = a.Q[l];
            for (int s = 0; s < a.smooth && ok; ++s) {
                const bool first = s == 0, last = s == a.smooth - 1;
                const bool zero = first && l > 0;
                const T mr = (zero && singular) ? T(read_mean(gs.slot + l * 3 + 2, L.n)) : T(0);
                double local = 0.0;
                T* rhs = a.R[l];
                const T* src = cur;
                T* dst = oth;
                for_cells<BC>(a.tl[l], L, [&](int x, int y, int z, int64_t i) {
                    T r = rhs[i];
                    if (zero && singular) {
                        r = r - mr;
                        rhs[i] = r;
                    }
                    T v;
                    if (zero) {
                        v = T(0) + (omega<T>() * r) / diag_at<BC>(x, y, z, L);
                    } else {
                        const T pc = src[i];
                        v = pc + (omega<T>() * (r - neg_lap<BC, false>(src, i, x, y, z, L, T(0), pc))) /
                                     diag_at<BC>(x, y, z, L);
                    }
                    dst[i] = v;
                    local += double(v);
                });
                const bool emit = last && singular;
                const double tot = emit ? block_total(local, red) : 0.0;
                ok = grid_sync(gs, tot, emit ? gs.slot + l * 3 + 0 : nullptr);
                T* t = cur; cur = oth; oth = t;
            }
            down[l] = cur;
            const Lv<T>& C = a.lv[l + 1];
            const T m = singular ? T(read_mean(gs.slot + l * 3 + 0, L.n)) : T(0);
            double local = 0.0;
            T* coarse = a.R[l + 1];
            const T* rhs = a.R[l];
            const T* src = cur;
            for_cells<BC>(a.tl[l + 1], C, [&](int x, int y, int z, int64_t c) {
                const T v = restrict_residual_at<BC, false>(src, rhs, x, y, z, L, m);
                coarse[c] = v;
                local += double(v);
            });
            const double tot = singular ? block_total(local, red) : 0.0;
            if (ok) ok = grid_sync(gs, tot, singular ? gs.slot + (l + 1) * 3 + 2 : nullptr);
        }
        if (!ok) break;
        // ---- coarse levels in block 0
        if (blockIdx.x == 0)
            coarse_cycle<BC, T, TC>(reinterpret_cast<T*>(smem_raw), a.R[fc],
                                    (fc > 0 && singular) ? gs.slot + fc * 3 + 2 : nullptr, fc == 0 ? a.P[0] : nullptr,
                                    a.P[fc], a.cinv, a.coarse, a.smooth);
        ok = grid_sync(gs, 0.0, nullptr);
        const T* corr = a.P[fc];
        T corr_mean = T(0);
        // ---- up legs
        for (int l = fc - 1; l >= 0 && ok; --l) {
            const Lv<T>& L = a.lv[l];
            const Lv<T>& C = a.lv[l + 1];
            const T md = singular ? T(read_mean(gs.slot + l * 3 + 0, L.n)) : T(0);
            T* dstp = a.P[l];
            const T* srcd = down[l];
            for_cells<BC>(a.tl[l], L, [&](int x, int y, int z, int64_t i) {
                dstp[i] = (srcd[i] - md) + prolong_at<BC>(corr, x, y, z, C, corr_mean);
            });
            ok = grid_sync(gs, 0.0, nullptr);
            T* cur = a.P[l];
            T* oth = a.Q[l];
            for (int s = 0; s < a.smooth && ok; ++s) {
                const bool last = s == a.smooth - 1;
                double local = 0.0;
                const T* src = cur;
                T* dst = oth;
                const T* rhs = a.R[l];
                for_cells<BC>(a.tl[l], L, [&](int x, int y, int z, int64_t i) {
                    const T pc = src[i];
                    const T v = pc + (omega<T>() * (rhs[i] - neg_lap<BC, false>(src, i, x, y, z, L, T(0), pc))) /
                                         diag_at<BC>(x, y, z, L);
                    dst[i] = v;
                    local += double(v);
                });
                const bool emit = last && singular;
                const double tot = emit ? block_total(local, red) : 0.0;
                ok = grid_sync(gs, tot, emit ? gs.slot + l * 3 + 1 : nullptr);
                T* t = cur; cur = oth; oth = t;
            }
            corr = cur;
            corr_mean = singular ? T(read_mean(gs.slot + l * 3 + 1, L.n)) : T(0);
        }
        if (!ok) break;
        // ---- level-0 iterate back in p[0], mean removed
        if (fc > 0 && (corr != a.P[0] || singular)) {
            T* p0 = a.P[0];
            const T* src = corr;
            const T m = corr_mean;
            for_cells<BC>(a.tl[0], a.lv[0], [&](int, int, int, int64_t i) { p0[i] = src[i] - m; });
            ok = grid_sync(gs, 0.0, nullptr);
        }
        done = cycle + 1;
        // ---- device-side convergence check (solve mode)
        if (a.solve && ok && (done % a.check_every == 0 || done == a.cycles)) {
            const Lv<T>& L = a.lv[0];
            const T* p = a.P[0];
            const T* rhs = a.R[0];
            double local = 0.0;
            for_cells<BC>(a.tl[0], L, [&](int x, int y, int z, int64_t i) {
                const T pc = p[i];
                const T r = rhs[i] - neg_lap<BC, true>(p, i, x, y, z, L, T(0), pc);
                local += double(r) * double(r);
            });
            const double tot = block_total(local, red);
            ok = grid_sync(gs, tot, gs.slot + kNormSlot);
            residual = sqrt(__ldcg(gs.slot + kNormSlot));
            if (!(residual > a.tol)) break;  // converged (or NaN: reported, host decides)
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && a.info) {
        a.info[0] = double(done);
        a.info[1] = residual;
        a.info[2] = ok ? 0.0 : 1.0;
    }
}

}  // namespace afsi

using namespace afsi;

namespace {

int log2i(int v) {
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}

template <class T>
Tiling tiling_for(const Lv<T>& L, int bc) {
    const bool three = is3d(bc);
    const int fast = three ? L.nz : L.ny, mid = three ? L.ny : L.nx, slow = three ? L.nx : 1;
    Tiling t;
    t.bxl = std::min(5, log2i(fast));
    t.byl = std::min(10 - t.bxl, log2i(mid));
    t.bzl = 10 - t.bxl - t.byl;
    t.gx = (fast + (1 << t.bxl) - 1) >> t.bxl;
    t.gy = (mid + (1 << t.byl) - 1) >> t.byl;
    t.gz = (slow + (1 << t.bzl) - 1) >> t.bzl;
    return t;
}

template <class T>
Lv<T> level_of(const afsi_mg_plan* plan, int l) {
    const afsi_mg_level& s = plan->level[l];
    Lv<T> L;
    L.nx = int(s.shape[0]);
    L.ny = int(s.shape[1]);
    L.nz = plan->dim == 3 ? int(s.shape[2]) : 1;
    L.n = int64_t(L.nx) * L.ny * L.nz;
    for (int a = 0; a < 3; ++a) {
        L.h2[a] = T(a < plan->dim ? s.h2[a] : 1.0);
        L.ih2[a] = T(a < plan->dim ? s.inv_h2[a] : 1.0);
    }
    return L;
}

template <int BC, class T, class TC>
int32_t run_persistent(const afsi_mg_plan* plan, int cycles, int solve, int check_every, double tol, double* info,
                       void* sync_scratch, cudaStream_t stream) {
    PersistentArgs<T, TC> a;
    a.levels = plan->levels;
    a.smooth = plan->smooth;
    for (int l = 0; l < plan->levels; ++l) {
        a.lv[l] = level_of<T>(plan, l);
        a.tl[l] = tiling_for(a.lv[l], BC);
        a.P[l] = static_cast<T*>(plan->level[l].p);
        a.Q[l] = static_cast<T*>(plan->level[l].ping);
        a.R[l] = static_cast<T*>(plan->level[l].rhs);
    }
    a.first_coarse = plan->levels - 1;
    for (int l = 0; l < plan->levels; ++l) {
        int64_t cells = 0;
        for (int k = l; k < plan->levels; ++k) cells += a.lv[k].n;
        if (a.lv[l].n <= kCoarseCells && (cells * 3 + 64 * (plan->levels - l)) * int64_t(sizeof(T)) <= 200 * 1024) {
            a.first_coarse = l;
            break;
        }
    }
    for (int k = 0; k < plan->levels; ++k) a.coarse.lv[k] = a.lv[k];
    a.coarse.first = a.first_coarse;
    a.coarse.last = plan->levels - 1;
    int64_t cells = 0;
    for (int k = a.first_coarse; k < plan->levels; ++k) cells += a.lv[k].n;
    const size_t smem = (size_t(cells) * 3 + 64 * size_t(plan->levels - a.first_coarse)) * sizeof(T);
    a.cinv = static_cast<const TC*>(plan->coarse_inverse);
    a.solve = solve;
    a.cycles = cycles;
    a.check_every = check_every;
    a.tol = tol;
    a.info = info;
    // barrier words and reduction slots
    unsigned char* b = static_cast<unsigned char*>(sync_scratch);
    a.gs.count = reinterpret_cast<unsigned int*>(b);
    a.gs.gen = reinterpret_cast<unsigned int*>(b + 4);
    a.gs.error = reinterpret_cast<int*>(b + 8);
    a.gs.slot = reinterpret_cast<double*>(b + 64);
    a.gs.partial = reinterpret_cast<double*>(b + 64 + 8 * (kNormSlot + 8));

    auto kernel = mg_persistent<BC, T, TC>;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024);
        configured = true;
    }
    int device = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPThreads, smem);
    AFSI_REQUIRE(per_sm >= 1 && sms >= 1, "persistent multigrid kernel does not fit on this device");
    int grid = a.first_coarse == 0 ? 1 : sms;  // one block per SM (co-residency)
    AFSI_REQUIRE(grid <= 4096, "too many blocks for the barrier scratch");
    cudaMemsetAsync(a.gs.error, 0, sizeof(int), stream);
    void* args[] = {&a};
    cudaError_t err = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(grid),
                                                  dim3(kPThreads), args, smem, stream);
    if (err != cudaSuccess) return fail(AFSI_ERR_CUDA, "persistent multigrid launch: %s", cudaGetErrorString(err));
    return launched("persistent multigrid");
}

int32_t check(const afsi_mg_plan* plan) {
    AFSI_REQUIRE(plan && plan->levels >= 1 && plan->levels <= AFSI_MG_MAX_LEVELS, "invalid plan");
    AFSI_REQUIRE((plan->dim == 3 && (plan->bc == AFSI_BC_NEUMANN || plan->bc == AFSI_BC_DIRICHLET)) ||
                     (plan->dim == 2 && (plan->bc == AFSI_BC_CHANNEL || plan->bc == AFSI_BC_PERIODIC)),
                 "unsupported dim/boundary combination");
    AFSI_REQUIRE(plan->smooth >= 1 && plan->coarse_inverse, "invalid plan");
    for (int l = 0; l < plan->levels; ++l)
        AFSI_REQUIRE(plan->level[l].p && plan->level[l].ping && plan->level[l].rhs, "null level buffer");
    return AFSI_OK;
}

}  // namespace

extern "C" int64_t afsi_b200_mg_sync_bytes(void) { return 64 + 8 * (kNormSlot + 8) + 8 * 4096; }

extern "C" int32_t afsi_b200_mg_persistent(const afsi_mg_plan* plan, int32_t cycles, int32_t solve,
                                           int32_t check_every, double tol, double* info, void* sync_scratch,
                                           afsi_stream_t stream) {
    int32_t rc = check(plan);
    if (rc) return rc;
    AFSI_REQUIRE(cycles >= 0 && check_every >= 1 && sync_scratch, "invalid persistent multigrid arguments");
    AFSI_REQUIRE(!solve || info, "solve mode needs an info buffer");
    AFSI_REQUIRE(plan->smoother == AFSI_MG_JACOBI, "the persistent multigrid runs the Jacobi smoother only");
    if (cycles == 0) return AFSI_OK;
    AFSI_REQUIRE(plan->coarse_dtype == AFSI_F64 || plan->coarse_dtype == plan->dtype, "unsupported coarse dtype");
    switch (plan->bc) {
#define AFSI_PERSIST(BCV)                                                                                    \
    case BCV:                                                                                                \
        AFSI_DISPATCH(plan->dtype, {                                                                         \
            if (plan->coarse_dtype == AFSI_F64)                                                              \
                return run_persistent<BCV, T, double>(plan, cycles, solve, check_every, tol, info, sync_scratch, \
                                                      stream);                                               \
            return run_persistent<BCV, T, T>(plan, cycles, solve, check_every, tol, info, sync_scratch, stream); \
        });                                                                                                  \
        break;
        AFSI_PERSIST(AFSI_BC_NEUMANN)
        AFSI_PERSIST(AFSI_BC_CHANNEL)
        AFSI_PERSIST(AFSI_BC_PERIODIC)
        AFSI_PERSIST(AFSI_BC_DIRICHLET)
#undef AFSI_PERSIST
    default:
        return fail(AFSI_ERR_ARG, "unknown boundary condition");
    }
    return AFSI_OK;
}
