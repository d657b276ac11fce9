// MAC geometric multigrid on the B200: elementwise level kernels and a fused
// V-cycle.
//
// Operators (per-axis accumulation order of the reference):
//   Neumann 3D   mac/grid.py:86-93, mac/_triton_mg.py:12-34
//   channel 2D   mac2d/grid.py:61-71, mac2d/_triton_mg.py:7-22 (p=0 outlet ghost)
//   periodic 2D  x-wrapped differences, one-sided y rows (no reference solver)
// Jacobi p + ((2/3)*(rhs-Ap))/diag with diag rebuilt in the kernel in the
// order of mac/multigrid.py:38-42 (no diagonal array is read); restriction by
// child averaging (children summed x-major, z fastest); cell-centred
// prolongation of mac/_triton_mg.py:89-118 and mac2d/_triton_mg.py:55-75.
//
// Fused V-cycle: the schedule of mac/mg_workspace.py:85-102 with three
// changes in how it is executed, none in what is computed:
//  * the mean-zero gauge (p -= mean after each smoothing block, rhs -= mean
//    after restriction) is carried as a pending shift: the kernel that writes
//    a field also reduces its sum (deterministic per-block partials, summed
//    in index order by the last block to finish), and the next kernel that
//    reads the field subtracts sum/n on load, so no separate mean or subtract
//    launches exist;
//  * zeroing the coarse iterate is folded into the first sweep (p_in = 0);
//  * every level with at most kCoarseCells cells, the dense coarsest solve
//    included, runs inside one thread block in shared memory.
#include "common.cuh"

namespace afsi {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 4096;        // grid-stride cap, fixed => deterministic partials
constexpr int kCoarseThreads = 1024;
constexpr int64_t kCoarseCells = 4096;  // levels at or below this size run in one CTA

template <class T>
struct Lv {
    int64_t nx, ny, nz, n;
    T h2[3], ih2[3];
};

// One reduction site: per-block partials, completion counter, result.
struct Site {
    double* partial;
    unsigned int* counter;
    double* result;
};

template <int BC, class T>
__device__ __forceinline__ T diag_at(int64_t x, int64_t y, int64_t z, const Lv<T>& L) {
    T d = T(0);
    if (BC == AFSI_BC_NEUMANN) {
        if (x < L.nx - 1) d += L.ih2[0];
        if (x > 0) d += L.ih2[0];
        if (y < L.ny - 1) d += L.ih2[1];
        if (y > 0) d += L.ih2[1];
        if (z < L.nz - 1) d += L.ih2[2];
        if (z > 0) d += L.ih2[2];
    } else {
        if (BC == AFSI_BC_CHANNEL) {
            if (x < L.nx - 1) d += L.ih2[0];
            if (x > 0) d += L.ih2[0];
        } else {
            d += L.ih2[0];
            d += L.ih2[0];
        }
        if (y < L.ny - 1) d += L.ih2[1];
        if (y > 0) d += L.ih2[1];
        if (BC == AFSI_BC_CHANNEL && x == L.nx - 1) d += T(2) * L.ih2[0];
    }
    return d;
}

// (A p)_i with every load shifted by m (pc = p_i - m already loaded).
template <int BC, class T>
__device__ __forceinline__ T neg_lap(const T* __restrict__ p, int64_t i, int64_t x, int64_t y, int64_t z,
                                     const Lv<T>& L, T m, T pc) {
    T a = T(0);
    if (BC == AFSI_BC_NEUMANN) {
        const int64_t sx = L.ny * L.nz, sy = L.nz;
        if (x + 1 < L.nx) a = a - ((p[i + sx] - m) - pc) / L.h2[0];
        if (x > 0) a = a + (pc - (p[i - sx] - m)) / L.h2[0];
        if (y + 1 < L.ny) a = a - ((p[i + sy] - m) - pc) / L.h2[1];
        if (y > 0) a = a + (pc - (p[i - sy] - m)) / L.h2[1];
        if (z + 1 < L.nz) a = a - ((p[i + 1] - m) - pc) / L.h2[2];
        if (z > 0) a = a + (pc - (p[i - 1] - m)) / L.h2[2];
    } else {
        const int64_t sx = L.ny;
        if (BC == AFSI_BC_CHANNEL) {
            if (x + 1 < L.nx) a = a - ((p[i + sx] - m) - pc) / L.h2[0];
            if (x > 0) a = a + (pc - (p[i - sx] - m)) / L.h2[0];
        } else {
            const int64_t right = x + 1 < L.nx ? i + sx : i - (L.nx - 1) * sx;
            const int64_t left = x > 0 ? i - sx : i + (L.nx - 1) * sx;
            a = a - ((p[right] - m) - pc) / L.h2[0];
            a = a + (pc - (p[left] - m)) / L.h2[0];
        }
        if (y + 1 < L.ny) a = a - ((p[i + 1] - m) - pc) / L.h2[1];
        if (y > 0) a = a + (pc - (p[i - 1] - m)) / L.h2[1];
        if (BC == AFSI_BC_CHANNEL && x == L.nx - 1) a = a + T(2) * pc / L.h2[0];
    }
    return a;
}

template <class T>
__device__ __forceinline__ void coords(int64_t i, const Lv<T>& L, int64_t& x, int64_t& y, int64_t& z) {
    z = i % L.nz;
    const int64_t r = i / L.nz;
    y = r % L.ny;
    x = r / L.ny;
}

template <class T>
__device__ __forceinline__ T omega() { return T(2.0 / 3.0); }

__device__ __forceinline__ double site_mean(const double* result, int64_t n) {
    return result ? *result / double(n) : 0.0;
}

// Block partial + last-block completion for a grid reduction of `v`.
__device__ __forceinline__ void site_finish(const Site& s, double v) {
    __shared__ double warp_sums[32];
    __shared__ bool last;
    v = block_sum(v, warp_sums);
    if (threadIdx.x == 0) s.partial[blockIdx.x] = v;
    if (grid_reduce_arrive(s.counter, &last)) {
        double t = sum_partials(s.partial, gridDim.x, 1, 0, warp_sums);
        if (threadIdx.x == 0) {
            *s.result = t;
            *s.counter = 0u;
        }
    }
}

// ------------------------------------------------------------------ sweeps

// out = p + (2/3)(rhs - A p)/diag, p read with shift m_p (p_in == nullptr: p=0).
// fix_rhs: rhs -= mean(rhs) (pending from the restriction) and write it back.
// emit: reduce sum(out) into the site.
template <int BC, class T>
__global__ void __launch_bounds__(kThreads) sweep_kernel(const T* __restrict__ p, T* __restrict__ rhs, T* __restrict__ out,
                                                         Lv<T> L, const double* p_sum, const double* rhs_sum,
                                                         Site emit, int fix_rhs, int do_emit) {
    const T m = T(site_mean(p_sum, L.n));
    const T mr = T(site_mean(rhs_sum, L.n));
    double local = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < L.n; i += int64_t(gridDim.x) * blockDim.x) {
        int64_t x, y, z;
        coords(i, L, x, y, z);
        T r = rhs[i];
        if (fix_rhs) {
            r = r - mr;
            rhs[i] = r;
        }
        T v;
        if (p) {
            const T pc = p[i] - m;
            const T a = neg_lap<BC>(p, i, x, y, z, L, m, pc);
            v = pc + (omega<T>() * (r - a)) / diag_at<BC>(x, y, z, L);
        } else {
            v = T(0) + (omega<T>() * r) / diag_at<BC>(x, y, z, L);
        }
        out[i] = v;
        local += double(v);
    }
    if (do_emit) site_finish(emit, local);
}

// coarse[c] = mean of children of (rhs - A p), p shifted by m_p.
template <int BC, class T>
__global__ void __launch_bounds__(kThreads) residual_restrict_kernel(const T* __restrict__ p, const T* __restrict__ rhs,
                                                                     T* __restrict__ coarse, Lv<T> L, Lv<T> C,
                                                                     const double* p_sum, Site emit, int do_emit) {
    const T m = T(site_mean(p_sum, L.n));
    double local = 0.0;
    for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < C.n; c += int64_t(gridDim.x) * blockDim.x) {
        int64_t cx, cy, cz;
        coords(c, C, cx, cy, cz);
        T v = T(0);
        if (BC == AFSI_BC_NEUMANN) {
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int d = 0; d < 2; ++d) {
                        const int64_t x = 2 * cx + a, y = 2 * cy + b, z = 2 * cz + d;
                        const int64_t i = (x * L.ny + y) * L.nz + z;
                        const T pc = p[i] - m;
                        v = v + (rhs[i] - neg_lap<BC>(p, i, x, y, z, L, m, pc));
                    }
            v = v * T(.125);
        } else {
            T r[4];
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    const int64_t x = 2 * cx + a, y = 2 * cy + b;
                    const int64_t i = x * L.ny + y;
                    const T pc = p[i] - m;
                    r[a * 2 + b] = rhs[i] - neg_lap<BC>(p, i, x, y, 0, L, m, pc);
                }
            v = ((r[0] + r[1]) + r[2] + r[3]) * T(.25);
        }
        coarse[c] = v;
        local += double(v);
    }
    if (do_emit) site_finish(emit, local);
}

// Coarse value with the boundary ghosts of each BC (coarse lattice C).
template <int BC, class T>
__device__ __forceinline__ T coarse_at(const T* __restrict__ c, int64_t x, int64_t y, int64_t z, const Lv<T>& C, T m) {
    if (BC == AFSI_BC_NEUMANN) {
        x = x < 0 ? 0 : (x > C.nx - 1 ? C.nx - 1 : x);
        y = y < 0 ? 0 : (y > C.ny - 1 ? C.ny - 1 : y);
        z = z < 0 ? 0 : (z > C.nz - 1 ? C.nz - 1 : z);
        return c[(x * C.ny + y) * C.nz + z] - m;
    }
    T sign = T(1);
    if (BC == AFSI_BC_CHANNEL) {
        if (x >= C.nx) sign = T(-1);
        x = x < 0 ? 0 : (x > C.nx - 1 ? C.nx - 1 : x);
    } else {
        x = x < 0 ? x + C.nx : (x >= C.nx ? x - C.nx : x);
    }
    y = y < 0 ? 0 : (y > C.ny - 1 ? C.ny - 1 : y);
    return sign * (c[x * C.ny + y] - m);
}

template <int BC, class T>
__device__ __forceinline__ T prolong_at(const T* __restrict__ c, int64_t x, int64_t y, int64_t z, const Lv<T>& C, T m) {
    const int64_t ax = x / 2 - 1 + x % 2, ay = y / 2 - 1 + y % 2;
    const T wx = (x % 2 == 0) ? T(.75) : T(.25), wy = (y % 2 == 0) ? T(.75) : T(.25);
    if (BC == AFSI_BC_NEUMANN) {
        const int64_t az = z / 2 - 1 + z % 2;
        const T wz = (z % 2 == 0) ? T(.75) : T(.25);
        const int64_t x0 = ax < 0 ? 0 : ax, x1 = ax + 1 < C.nx - 1 ? ax + 1 : C.nx - 1;
        const int64_t y0 = ay < 0 ? 0 : ay, y1 = ay + 1 < C.ny - 1 ? ay + 1 : C.ny - 1;
        const int64_t z0 = az < 0 ? 0 : az, z1 = az + 1 < C.nz - 1 ? az + 1 : C.nz - 1;
        auto at = [&](int64_t i, int64_t j, int64_t k) { return c[(i * C.ny + j) * C.nz + k] - m; };
        const T c00 = at(x0, y0, z0) * (T(1) - wz) + at(x0, y0, z1) * wz;
        const T c01 = at(x0, y1, z0) * (T(1) - wz) + at(x0, y1, z1) * wz;
        const T c10 = at(x1, y0, z0) * (T(1) - wz) + at(x1, y0, z1) * wz;
        const T c11 = at(x1, y1, z0) * (T(1) - wz) + at(x1, y1, z1) * wz;
        return (c00 * (T(1) - wy) + c01 * wy) * (T(1) - wx) + (c10 * (T(1) - wy) + c11 * wy) * wx;
    }
    const T c00 = coarse_at<BC>(c, ax, ay, 0, C, m), c01 = coarse_at<BC>(c, ax, ay + 1, 0, C, m);
    const T c10 = coarse_at<BC>(c, ax + 1, ay, 0, C, m), c11 = coarse_at<BC>(c, ax + 1, ay + 1, 0, C, m);
    return (c00 * (T(1) - wy) + c01 * wy) * (T(1) - wx) + (c10 * (T(1) - wy) + c11 * wy) * wx;
}

// dst = (src - m_src) + P(corr - m_corr); src may alias dst (own cell only).
template <int BC, class T>
__global__ void __launch_bounds__(kThreads) prolong_kernel(const T* src, const T* __restrict__ corr, T* dst, Lv<T> L,
                                                           Lv<T> C, const double* src_sum, const double* corr_sum) {
    const T ms = T(site_mean(src_sum, L.n)), mc = T(site_mean(corr_sum, C.n));
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < L.n; i += int64_t(gridDim.x) * blockDim.x) {
        int64_t x, y, z;
        coords(i, L, x, y, z);
        dst[i] = (src[i] - ms) + prolong_at<BC>(corr, x, y, z, C, mc);
    }
}

// dst = src - mean (or a copy).
template <class T>
__global__ void __launch_bounds__(kThreads) shift_kernel(const T* src, T* dst, int64_t n, const double* sum) {
    const T m = T(site_mean(sum, n));
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        dst[i] = src[i] - m;
}

// ----------------------------------------------------------- coarse block

template <class T>
struct CoarseLevels {
    Lv<T> lv[AFSI_MG_MAX_LEVELS];
    int first, last;  // level indices handled here
};

// Block-wide mean (deterministic) of smem array a[0..n).
template <class T>
__device__ double block_mean(const T* a, int64_t n, double* red) {
    double v = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) v += double(a[i]);
    v = block_sum(v, red);
    __shared__ double bcast;
    if (threadIdx.x == 0) bcast = v / double(n);
    __syncthreads();
    return bcast;
}

// Levels first..last of one V-cycle in one CTA.  rhs of level `first` comes
// from global memory (shifted by rhs_sum/n); p[first] starts from p_global
// (first==0) or zero; the final p[first] is written to p_out.
template <int BC, class T, class TC>
__global__ void __launch_bounds__(kCoarseThreads) coarse_kernel(const T* __restrict__ rhs_global, const double* rhs_sum,
                                                               const T* p_global, T* p_out, const TC* __restrict__ cinv,
                                                               CoarseLevels<T> cl, int smooth) {
    extern __shared__ unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    __shared__ double red[32];
    constexpr bool singular = BC != AFSI_BC_CHANNEL;
    T* P[AFSI_MG_MAX_LEVELS];
    T* Q[AFSI_MG_MAX_LEVELS];
    T* R[AFSI_MG_MAX_LEVELS];
    {
        T* cur = smem;
        for (int l = cl.first; l <= cl.last; ++l) {
            const int64_t n = cl.lv[l].n;
            P[l] = cur;
            Q[l] = cur + n;
            R[l] = cur + 2 * n;
            cur += 3 * n;
        }
    }
    const int f = cl.first;
    {
        const T mr = T(site_mean(rhs_sum, cl.lv[f].n));
        for (int64_t i = threadIdx.x; i < cl.lv[f].n; i += blockDim.x) {
            R[f][i] = rhs_global[i] - mr;
            P[f][i] = p_global ? p_global[i] : T(0);
        }
    }
    __syncthreads();
    // down
    for (int l = f; l <= cl.last; ++l) {
        const Lv<T>& L = cl.lv[l];
        if (l == cl.last) {
            // dense coarsest solve p = inv * rhs (mac/mg_workspace.py:86-90)
            for (int64_t r = threadIdx.x; r < L.n; r += blockDim.x) {
                double s = 0.0;
                for (int64_t j = 0; j < L.n; ++j) s += double(cinv[r * L.n + j]) * double(R[l][j]);
                P[l][r] = T(s);
            }
            __syncthreads();
            if (singular) {
                const T m = T(block_mean(P[l], L.n, red));
                for (int64_t i = threadIdx.x; i < L.n; i += blockDim.x) P[l][i] = P[l][i] - m;
                __syncthreads();
            }
            break;
        }
        T* cur = P[l];
        T* oth = Q[l];
        for (int s = 0; s < smooth; ++s) {
            for (int64_t i = threadIdx.x; i < L.n; i += blockDim.x) {
                int64_t x, y, z;
                coords(i, L, x, y, z);
                const T pc = cur[i];
                const T a = neg_lap<BC>(cur, i, x, y, z, L, T(0), pc);
                oth[i] = pc + (omega<T>() * (R[l][i] - a)) / diag_at<BC>(x, y, z, L);
            }
            __syncthreads();
            T* t = cur; cur = oth; oth = t;
        }
        if (cur != P[l]) {
            for (int64_t i = threadIdx.x; i < L.n; i += blockDim.x) P[l][i] = cur[i];
            __syncthreads();
        }
        if (singular) {
            const T m = T(block_mean(P[l], L.n, red));
            for (int64_t i = threadIdx.x; i < L.n; i += blockDim.x) P[l][i] = P[l][i] - m;
            __syncthreads();
        }
        const Lv<T>& C = cl.lv[l + 1];
        for (int64_t c = threadIdx.x; c < C.n; c += blockDim.x) {
            int64_t cx, cy, cz;
            coords(c, C, cx, cy, cz);
            T v = T(0);
            if (BC == AFSI_BC_NEUMANN) {
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2; ++b)
                        for (int d = 0; d < 2; ++d) {
                            const int64_t x = 2 * cx + a, y = 2 * cy + b, z = 2 * cz + d;
                            const int64_t i = (x * L.ny + y) * L.nz + z;
                            v = v + (R[l][i] - neg_lap<BC>(P[l], i, x, y, z, L, T(0), P[l][i]));
                        }
                v = v * T(.125);
            } else {
                T r[4];
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2; ++b) {
                        const int64_t x = 2 * cx + a, y = 2 * cy + b, i = x * L.ny + y;
                        r[a * 2 + b] = R[l][i] - neg_lap<BC>(P[l], i, x, y, 0, L, T(0), P[l][i]);
                    }
                v = ((r[0] + r[1]) + r[2] + r[3]) * T(.25);
            }
            R[l + 1][c] = v;
            P[l + 1][c] = T(0);
        }
        __syncthreads();
        if (singular) {
            const T m = T(block_mean(R[l + 1], C.n, red));
            for (int64_t i = threadIdx.x; i < C.n; i += blockDim.x) R[l + 1][i] = R[l + 1][i] - m;
            __syncthreads();
        }
    }
    // up
    for (int l = cl.last - 1; l >= f; --l) {
        const Lv<T>& L = cl.lv[l];
        const Lv<T>& C = cl.lv[l + 1];
        for (int64_t i = threadIdx.x; i < L.n; i += blockDim.x) {
            int64_t x, y, z;
            coords(i, L, x, y, z);
            P[l][i] = P[l][i] + prolong_at<BC>(P[l + 1], x, y, z, C, T(0));
        }
        __syncthreads();
        T* cur = P[l];
        T* oth = Q[l];
        for (int s = 0; s < smooth; ++s) {
            for (int64_t i = threadIdx.x; i < L.n; i += blockDim.x) {
                int64_t x, y, z;
                coords(i, L, x, y, z);
                const T pc = cur[i];
                const T a = neg_lap<BC>(cur, i, x, y, z, L, T(0), pc);
                oth[i] = pc + (omega<T>() * (R[l][i] - a)) / diag_at<BC>(x, y, z, L);
            }
            __syncthreads();
            T* t = cur; cur = oth; oth = t;
        }
        if (cur != P[l]) {
            for (int64_t i = threadIdx.x; i < L.n; i += blockDim.x) P[l][i] = cur[i];
            __syncthreads();
        }
        if (singular) {
            const T m = T(block_mean(P[l], L.n, red));
            for (int64_t i = threadIdx.x; i < L.n; i += blockDim.x) P[l][i] = P[l][i] - m;
            __syncthreads();
        }
    }
    for (int64_t i = threadIdx.x; i < cl.lv[f].n; i += blockDim.x) p_out[i] = P[f][i];
}

// ------------------------------------------------------- residual norm

template <int BC, class T>
__global__ void __launch_bounds__(kThreads) residual_norm_kernel(const T* __restrict__ p, const T* __restrict__ rhs,
                                                                 Lv<T> L, Site s, double* norm_out) {
    double local = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < L.n; i += int64_t(gridDim.x) * blockDim.x) {
        int64_t x, y, z;
        coords(i, L, x, y, z);
        const T pc = p[i];
        const T r = rhs[i] - neg_lap<BC>(p, i, x, y, z, L, T(0), pc);
        local += double(r) * double(r);
    }
    __shared__ double warp_sums[32];
    __shared__ bool last;
    local = block_sum(local, warp_sums);
    if (threadIdx.x == 0) s.partial[blockIdx.x] = local;
    if (grid_reduce_arrive(s.counter, &last)) {
        const double t = sum_partials(s.partial, gridDim.x, 1, 0, warp_sums);
        if (threadIdx.x == 0) {
            *norm_out = sqrt(t);
            *s.counter = 0u;
        }
    }
}

// sum, sum|x|, sum x^2, finite flag
template <class T>
__global__ void __launch_bounds__(kThreads) stats_kernel(const T* __restrict__ x, int64_t n, double* partial,
                                                         unsigned int* counter, double* out) {
    double s = 0.0, a = 0.0, q = 0.0, bad = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const double v = double(x[i]);
        if (!isfinite(v)) bad = 1.0;
        s += v;
        a += fabs(v);
        q += v * v;
    }
    __shared__ double warp_sums[32];
    __shared__ bool last;
    s = block_sum(s, warp_sums);
    a = block_sum(a, warp_sums);
    q = block_sum(q, warp_sums);
    bad = block_sum(bad, warp_sums);
    if (threadIdx.x == 0) {
        partial[blockIdx.x * 4 + 0] = s;
        partial[blockIdx.x * 4 + 1] = a;
        partial[blockIdx.x * 4 + 2] = q;
        partial[blockIdx.x * 4 + 3] = bad;
    }
    if (grid_reduce_arrive(counter, &last)) {
        double r[4];
        for (int k = 0; k < 4; ++k) r[k] = sum_partials(partial, gridDim.x, 4, k, warp_sums);
        if (threadIdx.x == 0) {
            out[0] = r[0];
            out[1] = r[1];
            out[2] = r[2];
            out[3] = r[3] > 0.0 ? 0.0 : 1.0;
            *counter = 0u;
        }
    }
}

// ------------------------------------------------------ standalone kernels

template <int BC, class T>
__global__ void __launch_bounds__(kThreads) restrict_kernel(const T* __restrict__ fine, T* __restrict__ coarse,
                                                            Lv<T> L, Lv<T> C) {
    for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < C.n; c += int64_t(gridDim.x) * blockDim.x) {
        int64_t cx, cy, cz;
        coords(c, C, cx, cy, cz);
        T v;
        if (BC == AFSI_BC_NEUMANN) {
            const int64_t j = ((2 * cx) * L.ny + 2 * cy) * L.nz + 2 * cz;
            const int64_t sy = L.nz, sx = L.ny * L.nz;
            v = fine[j];
            v = v + fine[j + 1];
            v = v + fine[j + sy];
            v = v + fine[j + sy + 1];
            v = v + fine[j + sx];
            v = v + fine[j + sx + 1];
            v = v + fine[j + sx + sy];
            v = v + fine[j + sx + sy + 1];
            v = v * T(.125);
        } else {
            const int64_t j = 2 * cx * L.ny + 2 * cy;
            v = ((fine[j] + fine[j + 1]) + fine[j + L.ny] + fine[j + L.ny + 1]) * T(.25);
        }
        coarse[c] = v;
    }
}

}  // namespace afsi

using namespace afsi;

namespace {

int grid_for(int64_t n) {
    int64_t b = (n + kThreads - 1) / kThreads;
    return int(b < kMaxBlocks ? (b > 0 ? b : 1) : kMaxBlocks);
}

template <class T>
Lv<T> make_level(const int64_t* shape, const double* h2, const double* ih2, int dim) {
    Lv<T> L;
    L.nx = shape[0];
    L.ny = shape[1];
    L.nz = dim == 3 ? shape[2] : 1;
    L.n = L.nx * L.ny * L.nz;
    for (int a = 0; a < 3; ++a) {
        L.h2[a] = T(a < dim ? h2[a] : 1.0);
        L.ih2[a] = T(ih2 && a < dim ? ih2[a] : 1.0);
    }
    return L;
}

template <class T>
Lv<T> coarser(const Lv<T>& L) {
    Lv<T> C = L;
    C.nx = L.nx / 2;
    C.ny = L.ny / 2;
    C.nz = L.nz > 1 ? L.nz / 2 : 1;
    C.n = C.nx * C.ny * C.nz;
    return C;
}

int32_t check_bc(int32_t dim, int32_t bc) {
    AFSI_REQUIRE((dim == 3 && bc == AFSI_BC_NEUMANN) || (dim == 2 && (bc == AFSI_BC_CHANNEL || bc == AFSI_BC_PERIODIC)),
                 "unsupported dim/boundary combination (%d, %d)", dim, bc);
    return AFSI_OK;
}

#define AFSI_BC_DISPATCH(bc, ...)                                                   \
    switch (bc) {                                                                   \
    case AFSI_BC_NEUMANN: { constexpr int BC = AFSI_BC_NEUMANN; __VA_ARGS__; } break; \
    case AFSI_BC_CHANNEL: { constexpr int BC = AFSI_BC_CHANNEL; __VA_ARGS__; } break; \
    case AFSI_BC_PERIODIC: { constexpr int BC = AFSI_BC_PERIODIC; __VA_ARGS__; } break; \
    default: return fail(AFSI_ERR_ARG, "unknown boundary condition %d", (int)(bc)); \
    }

int32_t check_shape(const int64_t* shape, int dim) {
    AFSI_REQUIRE(shape, "null shape");
    for (int a = 0; a < dim; ++a) AFSI_REQUIRE(shape[a] > 0, "non-positive grid extent");
    return AFSI_OK;
}

// ---- fused V-cycle plan execution ----

struct SiteTable {
    Site s[AFSI_MG_MAX_LEVELS][3];  // 0: p after down sweeps, 1: p after up sweeps, 2: rhs
    Site norm;
};

constexpr int64_t kSiteBytes = int64_t(kMaxBlocks) * 8 * 4 + 64;  // partial (x4 for stats) + result + counter

SiteTable sites_for(const afsi_mg_plan* plan) {
    SiteTable t;
    unsigned char* base = static_cast<unsigned char*>(plan->scratch);
    int k = 0;
    auto make = [&](int idx) {
        unsigned char* b = base + int64_t(idx) * kSiteBytes;
        Site s;
        s.partial = reinterpret_cast<double*>(b);
        s.result = reinterpret_cast<double*>(b + int64_t(kMaxBlocks) * 8 * 4);
        s.counter = reinterpret_cast<unsigned int*>(b + int64_t(kMaxBlocks) * 8 * 4 + 8);
        return s;
    };
    for (int l = 0; l < AFSI_MG_MAX_LEVELS; ++l)
        for (int j = 0; j < 3; ++j) t.s[l][j] = make(k++);
    t.norm = make(k++);
    return t;
}

template <int BC, class T, class TC>
struct Runner {
    const afsi_mg_plan* plan;
    cudaStream_t stream;
    SiteTable st;
    Lv<T> lv[AFSI_MG_MAX_LEVELS];
    int first_coarse;

    T* P(int l) const { return static_cast<T*>(plan->level[l].p); }
    T* Q(int l) const { return static_cast<T*>(plan->level[l].ping); }
    T* R(int l) const { return static_cast<T*>(plan->level[l].rhs); }
    static constexpr bool singular = BC != AFSI_BC_CHANNEL;

    int32_t coarse(int l, const double* rhs_sum, T** out) {
        CoarseLevels<T> cl;
        for (int k = 0; k < plan->levels; ++k) cl.lv[k] = lv[k];
        cl.first = l;
        cl.last = plan->levels - 1;
        int64_t cells = 0;
        for (int k = l; k < plan->levels; ++k) cells += lv[k].n;
        const size_t bytes = size_t(cells) * 3 * sizeof(T);
        static bool configured = false;  // once per instantiation, before any graph capture of it
        if (!configured) {
            cudaFuncSetAttribute(coarse_kernel<BC, T, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024);
            configured = true;
        }
        coarse_kernel<BC, T, TC><<<1, kCoarseThreads, bytes, stream>>>(
            R(l), rhs_sum, l == 0 ? P(0) : nullptr, P(l), static_cast<const TC*>(plan->coarse_inverse), cl,
            plan->smooth);
        *out = P(l);
        return launched("mg coarse block");
    }

    // Returns the buffer holding the level's final iterate and the site whose
    // sum is its pending mean (nullptr: exact).
    int32_t level(int l, T** out, const double** out_sum) {
        int32_t rc;
        if (l >= first_coarse) {
            rc = coarse(l, (l > 0 && singular) ? st.s[l][2].result : nullptr, out);
            *out_sum = nullptr;
            return rc;
        }
        const Lv<T>& L = lv[l];
        const int g = grid_for(L.n);
        T* cur = P(l);
        T* oth = Q(l);
        for (int s = 0; s < plan->smooth; ++s) {
            const bool first = s == 0;
            const bool last = s == plan->smooth - 1;
            sweep_kernel<BC, T><<<g, kThreads, 0, stream>>>(
                (first && l > 0) ? nullptr : cur, R(l), oth, L, nullptr,
                (first && l > 0 && singular) ? st.s[l][2].result : nullptr, st.s[l][0],
                (first && l > 0 && singular) ? 1 : 0, (last && singular) ? 1 : 0);
            if ((rc = launched("mg sweep"))) return rc;
            T* t = cur; cur = oth; oth = t;
        }
        const double* down_sum = singular ? st.s[l][0].result : nullptr;
        const Lv<T>& C = lv[l + 1];
        residual_restrict_kernel<BC, T><<<grid_for(C.n), kThreads, 0, stream>>>(
            cur, R(l), R(l + 1), L, C, down_sum, st.s[l + 1][2], singular ? 1 : 0);
        if ((rc = launched("mg residual_restrict"))) return rc;
        T* corr;
        const double* corr_sum;
        if ((rc = level(l + 1, &corr, &corr_sum))) return rc;
        prolong_kernel<BC, T><<<g, kThreads, 0, stream>>>(cur, corr, P(l), L, C, down_sum, corr_sum);
        if ((rc = launched("mg prolong_add"))) return rc;
        cur = P(l);
        oth = Q(l);
        for (int s = 0; s < plan->smooth; ++s) {
            const bool last = s == plan->smooth - 1;
            sweep_kernel<BC, T><<<g, kThreads, 0, stream>>>(cur, R(l), oth, L, nullptr, nullptr, st.s[l][1], 0,
                                                            (last && singular) ? 1 : 0);
            if ((rc = launched("mg sweep"))) return rc;
            T* t = cur; cur = oth; oth = t;
        }
        *out = cur;
        *out_sum = singular ? st.s[l][1].result : nullptr;
        return AFSI_OK;
    }

    int32_t cycles(int count) {
        for (int c = 0; c < count; ++c) {
            T* out;
            const double* sum;
            int32_t rc = level(0, &out, &sum);
            if (rc) return rc;
            if (out != P(0) || sum) {
                shift_kernel<T><<<grid_for(lv[0].n), kThreads, 0, stream>>>(out, P(0), lv[0].n, sum);
                if ((rc = launched("mg finalize"))) return rc;
            }
        }
        return AFSI_OK;
    }
};

int32_t validate_plan(const afsi_mg_plan* plan) {
    AFSI_REQUIRE(plan, "null plan");
    int32_t rc = check_bc(plan->dim, plan->bc);
    if (rc) return rc;
    AFSI_REQUIRE(plan->levels >= 1 && plan->levels <= AFSI_MG_MAX_LEVELS, "invalid level count");
    AFSI_REQUIRE(plan->smooth >= 1, "smooth must be >= 1");
    AFSI_REQUIRE(plan->scratch, "null scratch");
    AFSI_REQUIRE(plan->coarse_inverse, "null coarse inverse");
    for (int l = 0; l < plan->levels; ++l) {
        const afsi_mg_level& L = plan->level[l];
        if ((rc = check_shape(L.shape, plan->dim))) return rc;
        AFSI_REQUIRE(L.p && L.ping && L.rhs, "null level buffer at level %d", l);
        if (l + 1 < plan->levels) {
            const afsi_mg_level& C = plan->level[l + 1];
            for (int a = 0; a < plan->dim; ++a)
                AFSI_REQUIRE(L.shape[a] % 2 == 0 && C.shape[a] == L.shape[a] / 2,
                             "level %d is not a 2x coarsening of level %d", l + 1, l);
        }
    }
    int64_t nc = 1;
    for (int a = 0; a < plan->dim; ++a) nc *= plan->level[plan->levels - 1].shape[a];
    AFSI_REQUIRE(nc <= 512, "coarsest level must have <= 512 cells");
    return AFSI_OK;
}

template <int BC, class T, class TC>
int32_t run_plan(const afsi_mg_plan* plan, int cycles, cudaStream_t stream) {
    Runner<BC, T, TC> r;
    r.plan = plan;
    r.stream = stream;
    r.st = sites_for(plan);
    for (int l = 0; l < plan->levels; ++l)
        r.lv[l] = make_level<T>(plan->level[l].shape, plan->level[l].h2, plan->level[l].inv_h2, plan->dim);
    // first level that fits the single-block path (shared memory for 3 arrays
    // of it and every coarser level)
    r.first_coarse = plan->levels - 1;
    for (int l = 0; l < plan->levels; ++l) {
        int64_t cells = 0;
        for (int k = l; k < plan->levels; ++k) cells += r.lv[k].n;
        if (r.lv[l].n <= kCoarseCells && cells * 3 * int64_t(sizeof(T)) <= 200 * 1024) {
            r.first_coarse = l;
            break;
        }
    }
    return r.cycles(cycles);
}

}  // namespace

extern "C" int64_t afsi_b200_mg_scratch_bytes(const afsi_mg_plan* plan) {
    (void)plan;
    return (int64_t(AFSI_MG_MAX_LEVELS) * 3 + 1) * kSiteBytes;
}

extern "C" int32_t afsi_b200_mg_vcycles(const afsi_mg_plan* plan, int32_t cycles, afsi_stream_t stream) {
    int32_t rc = validate_plan(plan);
    if (rc) return rc;
    AFSI_REQUIRE(cycles >= 0, "negative cycle count");
    AFSI_REQUIRE(plan->coarse_dtype == AFSI_F64 || plan->coarse_dtype == plan->dtype, "unsupported coarse dtype");
    AFSI_BC_DISPATCH(plan->bc, {
        AFSI_DISPATCH(plan->dtype, {
            if (plan->coarse_dtype == AFSI_F64)
                return run_plan<BC, T, double>(plan, cycles, stream);
            return run_plan<BC, T, T>(plan, cycles, stream);
        });
    });
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_mg_residual_norm(const afsi_mg_plan* plan, double* norm_out, afsi_stream_t stream) {
    int32_t rc = validate_plan(plan);
    if (rc) return rc;
    AFSI_REQUIRE(norm_out, "null output");
    SiteTable st = sites_for(plan);
    AFSI_BC_DISPATCH(plan->bc, {
        AFSI_DISPATCH(plan->dtype, {
            Lv<T> L = make_level<T>(plan->level[0].shape, plan->level[0].h2, plan->level[0].inv_h2, plan->dim);
            residual_norm_kernel<BC, T><<<grid_for(L.n), kThreads, 0, stream>>>(
                static_cast<const T*>(plan->level[0].p), static_cast<const T*>(plan->level[0].rhs), L, st.norm,
                norm_out);
        });
    });
    return launched("mg residual_norm");
}

extern "C" int32_t afsi_b200_vector_stats(const void* x, int64_t n, double* stats_out, void* scratch, int32_t dtype,
                                          afsi_stream_t stream) {
    AFSI_REQUIRE(n > 0 && x && stats_out && scratch, "invalid stats arguments");
    unsigned char* b = static_cast<unsigned char*>(scratch);
    double* partial = reinterpret_cast<double*>(b);
    unsigned int* counter = reinterpret_cast<unsigned int*>(b + int64_t(kMaxBlocks) * 8 * 4 + 8);
    AFSI_DISPATCH(dtype, {
        stats_kernel<T><<<grid_for(n), kThreads, 0, stream>>>(static_cast<const T*>(x), n, partial, counter,
                                                              stats_out);
    });
    return launched("vector_stats");
}

extern "C" int32_t afsi_b200_subtract_mean(void* x, int64_t n, const double* stats, int32_t dtype,
                                           afsi_stream_t stream) {
    AFSI_REQUIRE(n > 0 && x && stats, "invalid subtract_mean arguments");
    AFSI_DISPATCH(dtype, {
        shift_kernel<T><<<grid_for(n), kThreads, 0, stream>>>(static_cast<const T*>(x), static_cast<T*>(x), n,
                                                              stats);
    });
    return launched("subtract_mean");
}

// ---- standalone kernel-object entry points ----

extern "C" int32_t afsi_b200_mg_smooth(const void* p, const void* rhs, void* out, const int64_t* shape,
                                       const double* h2, const double* inv_h2, int32_t dim, int32_t bc,
                                       int32_t dtype, afsi_stream_t stream) {
    int32_t rc = check_bc(dim, bc);
    if (rc || (rc = check_shape(shape, dim))) return rc;
    AFSI_REQUIRE(p && rhs && out && h2 && inv_h2, "null argument");
    AFSI_BC_DISPATCH(bc, {
        AFSI_DISPATCH(dtype, {
            Lv<T> L = make_level<T>(shape, h2, inv_h2, dim);
            Site none{nullptr, nullptr, nullptr};
            sweep_kernel<BC, T><<<grid_for(L.n), kThreads, 0, stream>>>(
                static_cast<const T*>(p), const_cast<T*>(static_cast<const T*>(rhs)), static_cast<T*>(out), L,
                nullptr, nullptr, none, 0, 0);
        });
    });
    return launched("mg_smooth");
}

namespace afsi {
template <int BC, class T>
__global__ void __launch_bounds__(kThreads) residual_kernel(const T* __restrict__ p, const T* __restrict__ rhs,
                                                            T* __restrict__ out, Lv<T> L) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < L.n; i += int64_t(gridDim.x) * blockDim.x) {
        int64_t x, y, z;
        coords(i, L, x, y, z);
        const T pc = p[i];
        out[i] = rhs[i] - neg_lap<BC>(p, i, x, y, z, L, T(0), pc);
    }
}
}  // namespace afsi

extern "C" int32_t afsi_b200_mg_residual(const void* p, const void* rhs, void* out, const int64_t* shape,
                                         const double* h2, int32_t dim, int32_t bc, int32_t dtype,
                                         afsi_stream_t stream) {
    int32_t rc = check_bc(dim, bc);
    if (rc || (rc = check_shape(shape, dim))) return rc;
    AFSI_REQUIRE(p && rhs && out && h2, "null argument");
    AFSI_BC_DISPATCH(bc, {
        AFSI_DISPATCH(dtype, {
            Lv<T> L = make_level<T>(shape, h2, nullptr, dim);
            residual_kernel<BC, T><<<grid_for(L.n), kThreads, 0, stream>>>(
                static_cast<const T*>(p), static_cast<const T*>(rhs), static_cast<T*>(out), L);
        });
    });
    return launched("mg_residual");
}

extern "C" int32_t afsi_b200_mg_restrict(const void* fine, void* coarse, const int64_t* shape, int32_t dim,
                                         int32_t dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(dim == 2 || dim == 3, "dim must be 2 or 3");
    int32_t rc = check_shape(shape, dim);
    if (rc) return rc;
    AFSI_REQUIRE(fine && coarse, "null argument");
    for (int a = 0; a < dim; ++a) AFSI_REQUIRE(shape[a] % 2 == 0, "restriction needs even extents");
    const double one[3] = {1, 1, 1};
    AFSI_DISPATCH(dtype, {
        Lv<T> L = make_level<T>(shape, one, one, dim);
        Lv<T> C = coarser(L);
        if (dim == 3)
            restrict_kernel<AFSI_BC_NEUMANN, T><<<grid_for(C.n), kThreads, 0, stream>>>(
                static_cast<const T*>(fine), static_cast<T*>(coarse), L, C);
        else
            restrict_kernel<AFSI_BC_CHANNEL, T><<<grid_for(C.n), kThreads, 0, stream>>>(
                static_cast<const T*>(fine), static_cast<T*>(coarse), L, C);
    });
    return launched("mg_restrict");
}

extern "C" int32_t afsi_b200_mg_residual_restrict(const void* p, const void* rhs, void* coarse, const int64_t* shape,
                                                  const double* h2, int32_t dim, int32_t bc, int32_t dtype,
                                                  afsi_stream_t stream) {
    int32_t rc = check_bc(dim, bc);
    if (rc || (rc = check_shape(shape, dim))) return rc;
    AFSI_REQUIRE(p && rhs && coarse && h2, "null argument");
    for (int a = 0; a < dim; ++a) AFSI_REQUIRE(shape[a] % 2 == 0, "restriction needs even extents");
    AFSI_BC_DISPATCH(bc, {
        AFSI_DISPATCH(dtype, {
            Lv<T> L = make_level<T>(shape, h2, nullptr, dim);
            Lv<T> C = coarser(L);
            Site none{nullptr, nullptr, nullptr};
            residual_restrict_kernel<BC, T><<<grid_for(C.n), kThreads, 0, stream>>>(
                static_cast<const T*>(p), static_cast<const T*>(rhs), static_cast<T*>(coarse), L, C, nullptr, none, 0);
        });
    });
    return launched("mg_residual_restrict");
}

extern "C" int32_t afsi_b200_mg_prolong_add(const void* coarse, void* fine, const int64_t* shape, int32_t dim,
                                            int32_t bc, int32_t dtype, afsi_stream_t stream) {
    int32_t rc = check_bc(dim, bc);
    if (rc || (rc = check_shape(shape, dim))) return rc;
    AFSI_REQUIRE(coarse && fine, "null argument");
    for (int a = 0; a < dim; ++a) AFSI_REQUIRE(shape[a] % 2 == 0, "prolongation needs even extents");
    const double one[3] = {1, 1, 1};
    AFSI_BC_DISPATCH(bc, {
        AFSI_DISPATCH(dtype, {
            Lv<T> L = make_level<T>(shape, one, one, dim);
            Lv<T> C = coarser(L);
            prolong_kernel<BC, T><<<grid_for(L.n), kThreads, 0, stream>>>(
                static_cast<const T*>(fine), static_cast<const T*>(coarse), static_cast<T*>(fine), L, C, nullptr,
                nullptr);
        });
    });
    return launched("mg_prolong_add");
}
