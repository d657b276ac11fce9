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
// Two arithmetic modes (template flag Exact):
//   Exact  stencil differences divided by h*h, as the reference kernels do:
//          the level kernels are bit-exact with the reference FP64 results;
//   fast   differences multiplied by 1/h**2 (identical when h is a power of
//          two, otherwise within one rounding per term); used by the fused
//          V-cycle, where the FP64 divisions would dominate the single-block
//          coarse levels.  The Jacobi division by the diagonal is kept.
//
// Launch geometry: block (bx,by) over the two fastest axes, grid z over the
// slowest, so cell coordinates come from the block/thread indices with no
// integer division.
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
#include <algorithm>
#include <atomic>
#include <cstring>
#include <type_traits>
#include <vector>
#include "mg_cluster.cuh"

namespace afsi {

// ------------------------------------------------------------------ sweeps

// out = p + (2/3)(rhs - A p)/diag, p read with shift m_p (p_in == nullptr: p=0).
// fix_rhs: rhs -= mean(rhs) (pending from the restriction) and write it back.
// emit: reduce sum(out) into the site.
// Exact: the reference's operation order, (2/3)(rhs - A p) divided by the
// diagonal; fast: the update p + (rhs - A p)(omega/diag) with omega/diag from a
// 64-entry boundary-class table each block builds before waiting on its
// predecessor (the single-CTA coarse levels use the same update).
template <int BC, bool Exact, class T>
__global__ void __launch_bounds__(kThreads) sweep_kernel(const T* __restrict__ p, T* __restrict__ rhs, T* __restrict__ out,
                                                         Lv<T> L, const double* p_sum, const double* rhs_sum,
                                                         Site emit, int fix_rhs, int do_emit) {
    __shared__ T wtab[64];
    if (!Exact) {
        const unsigned t = thread_linear();
        if (t < 64) wtab[t] = omega_of_class<BC>(int(t), L);
        __syncthreads();
    }
    pdl_enter();
    double local = 0.0;
    const T m = T(site_mean(p_sum, L.n));
    const T mr = T(site_mean(rhs_sum, L.n));
    for_my_cells<BC>(L, [&](int x, int y, int z) {
        const int64_t i = index_of(x, y, z, L);
        T r = rhs[i];
        if (fix_rhs) {
            r = r - mr;
            rhs[i] = r;
        }
        T v;
        if (Exact) {
            if (p) {
                const T pc = p[i] - m;
                const T a = neg_lap<BC, Exact>(p, i, x, y, z, L, m, pc);
                v = pc + (omega<T>() * (r - a)) / diag_at<BC>(x, y, z, L);
            } else {
                v = T(0) + (omega<T>() * r) / diag_at<BC>(x, y, z, L);
            }
        } else {
            const T w = wtab[boundary_class(x, y, z, L.nx, L.ny, L.nz)];
            if (p) {
                const T pc = p[i] - m;
                v = jacobi_update(pc, r, neg_lap<BC, Exact>(p, i, x, y, z, L, m, pc), w);
            } else {
                v = r * w;
            }
        }
        out[i] = v;
        local += double(v);
    });
    if (do_emit) site_finish(emit, local);
}

// (A p) of the z-adjacent cells (x,y,z) and (x,y,z+1), z even, of a 3D
// level (Neumann or Dirichlet), every load shifted by m: neg_lap's fast-form
// terms in neg_lap's order for each cell, with the pair and its x and y
// neighbours read as 16-byte vectors and the two outer z neighbours as
// scalars.  Returns the shifted centre values in pc0, pc1.
template <int BC, class T>
__device__ __forceinline__ void pair_neg_lap(const T* __restrict__ p, int64_t i, int x, int y, int z, const Lv<T>& L,
                                             T m, T& pc0, T& pc1, T& a0, T& a1) {
    using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    const int64_t sx = int64_t(L.ny) * L.nz, sy = L.nz;
    const bool xp_in = x + 1 < L.nx, xm_in = x > 0, yp_in = y + 1 < L.ny, ym_in = y > 0, zm_in = z > 0,
               zp_in = z + 2 < L.nz;
    const V c = *reinterpret_cast<const V*>(p + i);
    pc0 = c.x - m;
    pc1 = c.y - m;
    V xp, xm, yp, ym;
    if (xp_in) xp = *reinterpret_cast<const V*>(p + i + sx);
    if (xm_in) xm = *reinterpret_cast<const V*>(p + i - sx);
    if (yp_in) yp = *reinterpret_cast<const V*>(p + i + sy);
    if (ym_in) ym = *reinterpret_cast<const V*>(p + i - sy);
    const T zm = zm_in ? p[i - 1] - m : T(0), zq = zp_in ? p[i + 2] - m : T(0);
    a0 = T(0);
    a1 = T(0);
    if (BC == AFSI_BC_DIRICHLET) {
        a0 = xp_in ? a0 - ((xp.x - m) - pc0) * L.ih2[0] : a0 + (pc0 + pc0) * L.ih2[0];
        a1 = xp_in ? a1 - ((xp.y - m) - pc1) * L.ih2[0] : a1 + (pc1 + pc1) * L.ih2[0];
        a0 = xm_in ? a0 + (pc0 - (xm.x - m)) * L.ih2[0] : a0 + (pc0 + pc0) * L.ih2[0];
        a1 = xm_in ? a1 + (pc1 - (xm.y - m)) * L.ih2[0] : a1 + (pc1 + pc1) * L.ih2[0];
        a0 = yp_in ? a0 - ((yp.x - m) - pc0) * L.ih2[1] : a0 + (pc0 + pc0) * L.ih2[1];
        a1 = yp_in ? a1 - ((yp.y - m) - pc1) * L.ih2[1] : a1 + (pc1 + pc1) * L.ih2[1];
        a0 = ym_in ? a0 + (pc0 - (ym.x - m)) * L.ih2[1] : a0 + (pc0 + pc0) * L.ih2[1];
        a1 = ym_in ? a1 + (pc1 - (ym.y - m)) * L.ih2[1] : a1 + (pc1 + pc1) * L.ih2[1];
        a0 = a0 - (pc1 - pc0) * L.ih2[2];
        a1 = zp_in ? a1 - (zq - pc1) * L.ih2[2] : a1 + (pc1 + pc1) * L.ih2[2];
        a0 = zm_in ? a0 + (pc0 - zm) * L.ih2[2] : a0 + (pc0 + pc0) * L.ih2[2];
        a1 = a1 + (pc1 - pc0) * L.ih2[2];
    } else {
        if (xp_in) {
            a0 = a0 - ((xp.x - m) - pc0) * L.ih2[0];
            a1 = a1 - ((xp.y - m) - pc1) * L.ih2[0];
        }
        if (xm_in) {
            a0 = a0 + (pc0 - (xm.x - m)) * L.ih2[0];
            a1 = a1 + (pc1 - (xm.y - m)) * L.ih2[0];
        }
        if (yp_in) {
            a0 = a0 - ((yp.x - m) - pc0) * L.ih2[1];
            a1 = a1 - ((yp.y - m) - pc1) * L.ih2[1];
        }
        if (ym_in) {
            a0 = a0 + (pc0 - (ym.x - m)) * L.ih2[1];
            a1 = a1 + (pc1 - (ym.y - m)) * L.ih2[1];
        }
        a0 = a0 - (pc1 - pc0) * L.ih2[2];
        if (zp_in) a1 = a1 - (zq - pc1) * L.ih2[2];
        if (zm_in) a0 = a0 + (pc0 - zm) * L.ih2[2];
        a1 = a1 + (pc1 - pc0) * L.ih2[2];
    }
}

// The fast-form Jacobi sweep of a 3D level (Neumann or Dirichlet) with two
// z-adjacent cells per thread, z = 2k and 2k+1 (nz even): the pair's p and
// rhs and its x and y neighbours are 16-byte loads, the outer z neighbours
// two 8-byte loads, and the pair shares its address and x/y tests.  No
// pending shift of p (the launched sweeps take none); fix_rhs subtracts the
// rhs mean and writes it back.  Per cell the same operations in the same
// order as sweep_kernel's fast form, so out is bitwise equal; the emitted sum
// is added per block in this kernel's cell order.
template <int BC, class T>
__global__ void __launch_bounds__(kThreads) sweep_zpair_kernel(const T* __restrict__ p, T* __restrict__ rhs,
                                                               T* __restrict__ out, Lv<T> L, const double* rhs_sum,
                                                               Site emit, int fix_rhs, int do_emit) {
    using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    __shared__ T wtab[64];
    {
        const unsigned t = thread_linear();
        if (t < 64) wtab[t] = omega_of_class<BC>(int(t), L);
        __syncthreads();
    }
    pdl_enter();
    double local = 0.0;
    const T mr = T(site_mean(rhs_sum, L.n));
    const int zp = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = 2 * zp;
    if (z < L.nz && y < L.ny) {
        for (int x = blockIdx.z; x < L.nx; x += gridDim.z) {
            const int64_t i = (int64_t(x) * L.ny + y) * L.nz + z;
            const V rv = *reinterpret_cast<const V*>(rhs + i);
            T r0 = rv.x, r1 = rv.y;
            if (fix_rhs) {
                r0 = r0 - mr;
                r1 = r1 - mr;
                V w;
                w.x = r0;
                w.y = r1;
                *reinterpret_cast<V*>(rhs + i) = w;
            }
            const T w0 = wtab[boundary_class(x, y, z, L.nx, L.ny, L.nz)];
            const T w1 = wtab[boundary_class(x, y, z + 1, L.nx, L.ny, L.nz)];
            T v0, v1;
            if (p) {
                T pc0, pc1, a0, a1;
                pair_neg_lap<BC>(p, i, x, y, z, L, T(0), pc0, pc1, a0, a1);
                v0 = jacobi_update(pc0, r0, a0, w0);
                v1 = jacobi_update(pc1, r1, a1, w1);
            } else {
                v0 = r0 * w0;
                v1 = r1 * w1;
            }
            V o;
            o.x = v0;
            o.y = v1;
            *reinterpret_cast<V*>(out + i) = o;
            local += double(v0);
            local += double(v1);
        }
    }
    if (do_emit) site_finish(emit, local);
}

// residual_restrict_kernel's fast form for 3D levels (Neumann or Dirichlet)
// with the fine z pairs of each coarse cell read by pair_neg_lap: the eight
// children summed in the same order (x, y, then z), so coarse is bitwise
// equal.
template <int BC, class T>
__global__ void __launch_bounds__(kThreads) residual_restrict_zpair_kernel(const T* __restrict__ p,
                                                                          const T* __restrict__ rhs,
                                                                          T* __restrict__ coarse, Lv<T> L, Lv<T> C,
                                                                          const double* p_sum, Site emit,
                                                                          int do_emit) {
    using V = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    pdl_enter();
    double local = 0.0;
    const T m = T(site_mean(p_sum, L.n));
    for_my_cells<BC>(C, [&](int cx, int cy, int cz) {
        T v = T(0);
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const int x = 2 * cx + a, y = 2 * cy + b, z = 2 * cz;
                const int64_t i = index_of(x, y, z, L);
                T pc0, pc1, a0, a1;
                pair_neg_lap<BC>(p, i, x, y, z, L, m, pc0, pc1, a0, a1);
                const V r = *reinterpret_cast<const V*>(rhs + i);
                v = v + (r.x - a0);
                v = v + (r.y - a1);
            }
        v = v * T(.125);
        coarse[index_of(cx, cy, cz, C)] = v;
        local += double(v);
    });
    if (do_emit) site_finish(emit, local);
}

// coarse[c] = mean of children of (rhs - A p), p shifted by m_p.  Launched
// over the coarse lattice C.
template <int BC, bool Exact, class T>
__global__ void __launch_bounds__(kThreads) residual_restrict_kernel(const T* __restrict__ p, const T* __restrict__ rhs,
                                                                     T* __restrict__ coarse, Lv<T> L, Lv<T> C,
                                                                     const double* p_sum, Site emit, int do_emit) {
    pdl_enter();
    double local = 0.0;
    const T m = T(site_mean(p_sum, L.n));
    for_my_cells<BC>(C, [&](int cx, int cy, int cz) {
        const T v = restrict_residual_at<BC, Exact>(p, rhs, cx, cy, cz, L, m);
        coarse[index_of(cx, cy, cz, C)] = v;
        local += double(v);
    });
    if (do_emit) site_finish(emit, local);
}

// dst = (src - m_src) + P(corr - m_corr); src may alias dst (own cell only).
template <int BC, class T>
__global__ void __launch_bounds__(kThreads) prolong_kernel(const T* src, const T* __restrict__ corr, T* dst, Lv<T> L,
                                                           Lv<T> C, const double* src_sum, const double* corr_sum) {
    pdl_enter();
    const T ms = T(site_mean(src_sum, L.n)), mc = T(site_mean(corr_sum, C.n));
    for_my_cells<BC>(L, [&](int x, int y, int z) {
        const int64_t i = index_of(x, y, z, L);
        dst[i] = (src[i] - ms) + prolong_at<BC>(corr, x, y, z, C, mc);
    });
}

// The end of a check block of the solve loop in one launch: the last V-cycle's
// finalize (dst = src - m, the pending mean m of src; no write when src is
// dst and there is no mean) fused with the residual norm of the finalized
// iterate (residual_norm_kernel's exact form and geometry on the values
// src - m, which are the finalized values bit for bit, so the norm is the
// same) and, in the last block, the loop decision of mg_decide_kernel.
template <int BC, class T>
__global__ void __launch_bounds__(kThreads) finalize_check_kernel(const T* src, T* dst, const T* __restrict__ rhs,
                                                                  Lv<T> L, const double* sum, Site s, double* norm,
                                                                  double* loop, int check_every, int max_cycles,
                                                                  cudaGraphConditionalHandle handle) {
    pdl_enter();
    const T m = T(site_mean(sum, L.n));
    const bool write = src != dst;
    double local = 0.0;
    for_my_cells<BC>(L, [&](int x, int y, int z) {
        const int64_t i = index_of(x, y, z, L);
        const T pc = src[i] - m;
        if (write) dst[i] = pc;
        const T r = rhs[i] - neg_lap<BC, true>(src, i, x, y, z, L, m, pc);
        local += double(r) * double(r);
    });
    site_finish_then(s, local, norm, [&](double r) {
        const double cycles = loop[1] + check_every;
        loop[1] = cycles;
        loop[2] = r;
        const bool finite = isfinite(r);
        if (!finite) loop[3] = 1.0;
        const bool again = finite && r > loop[0] && cycles + check_every <= max_cycles;
        cudaGraphSetConditional(handle, again ? 1u : 0u);
    });
}

// dst = src - sum/n (or a copy when sum is null); flat grid-stride.
template <class T>
__global__ void __launch_bounds__(kThreads) shift_kernel(const T* src, T* dst, int64_t n, const double* sum) {
    pdl_enter();
    const T m = T(site_mean(sum, n));
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        dst[i] = src[i] - m;
}

template <int BC, bool Exact, class T>
__global__ void __launch_bounds__(kThreads) residual_kernel(const T* __restrict__ p, const T* __restrict__ rhs,
                                                            T* __restrict__ out, Lv<T> L) {
    pdl_enter();
    for_my_cells<BC>(L, [&](int x, int y, int z) {
        const int64_t i = index_of(x, y, z, L);
        const T pc = p[i];
        out[i] = rhs[i] - neg_lap<BC, Exact>(p, i, x, y, z, L, T(0), pc);
    });
}

template <int BC, bool Exact, class T>
__global__ void __launch_bounds__(kThreads) residual_norm_kernel(const T* __restrict__ p, const T* __restrict__ rhs,
                                                                 Lv<T> L, Site s, double* norm_out) {
    pdl_enter();
    double local = 0.0;
    for_my_cells<BC>(L, [&](int x, int y, int z) {
        const int64_t i = index_of(x, y, z, L);
        const T pc = p[i];
        const T r = rhs[i] - neg_lap<BC, Exact>(p, i, x, y, z, L, T(0), pc);
        local += double(r) * double(r);
    });
    site_finish(s, local, norm_out);
}

template <int BC, class T>
__global__ void __launch_bounds__(kThreads) restrict_kernel(const T* __restrict__ fine, T* __restrict__ coarse,
                                                            Lv<T> L, Lv<T> C) {
    pdl_enter();
    for_my_cells<BC>(C, [&](int cx, int cy, int cz) {
    T v;
    if (is3d(BC)) {
        const int64_t j = index_of(2 * cx, 2 * cy, 2 * cz, L);
        const int64_t sy = L.nz, sx = int64_t(L.ny) * L.nz;
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
        const int64_t j = int64_t(2 * cx) * L.ny + 2 * cy;
        v = ((fine[j] + fine[j + 1]) + fine[j + L.ny] + fine[j + L.ny + 1]) * T(.25);
    }
    coarse[index_of(cx, cy, cz, C)] = v;
    });
}

// sum, sum|x|, sum x^2, finite flag over a flat vector
template <class T>
__global__ void __launch_bounds__(kThreads) stats_kernel(const T* __restrict__ x, int64_t n, double* partial,
                                                         unsigned int* counter, double* out) {
    pdl_enter();
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

// Levels of one 3D V-cycle from `first` down, in one thread-block cluster
// (cluster_cycle).
template <int BC, class T, class TC>
__global__ void __launch_bounds__(kCoarseThreads) cluster_kernel(const T* __restrict__ rhs_global,
                                                                const double* rhs_sum, const T* p_global, T* p_out,
                                                                const TC* __restrict__ cinv, ClusterLevels<T> cl,
                                                                int smooth) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cluster_tables<BC, T>(reinterpret_cast<T*>(smem_raw), cl);
    pdl_enter();
    cluster_cycle<BC, T, TC>(reinterpret_cast<T*>(smem_raw), rhs_global, rhs_sum, p_global, p_out, cinv, cl, smooth);
}

// Levels of one V-cycle from `first` down, in one CTA (coarse_cycle).
template <int BC, class T, class TC>
__global__ void __launch_bounds__(kCoarseThreads) coarse_kernel(const T* __restrict__ rhs_global, const double* rhs_sum,
                                                               const T* p_global, T* p_out, const TC* __restrict__ cinv,
                                                               CoarseLevels<T> cl, int smooth) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    coarse_cycle<BC, T, TC>(reinterpret_cast<T*>(smem_raw), rhs_global, rhs_sum, p_global, p_out, cinv, cl, smooth);
}

template <int BC, class T, class TC>
__global__ void __launch_bounds__(kCoarseThreads) coarse_rb_kernel(const T* __restrict__ rhs_global,
                                                                  const T* p_global, T* p_out,
                                                                  const TC* __restrict__ cinv, CoarseLevels<T> cl,
                                                                  int smooth) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    coarse_cycle_rb<BC, T, TC>(reinterpret_cast<T*>(smem_raw), rhs_global, p_global, p_out, cinv, cl, smooth);
}

// ---- red-black Gauss-Seidel V-cycle (selectable smoother) ----
//
// A method change beside the reference's weighted Jacobi (mac/multigrid.py:
// 107-110): each sweep updates the cells with (x+y+z) even, then the odd ones,
// in place with omega 1, p += (rhs - A p)/diag, so every update reads only
// cells of the other colour (7- or 5-point stencil) and the half-sweep is
// race-free.  Periodic x needs even extents for the colouring to wrap, which
// the plan check enforces on every smoothed level.

template <int BC, class T>
__global__ void __launch_bounds__(kThreads) rb_kernel(T* p, const T* __restrict__ rhs, Lv<T> L, int color) {
    pdl_enter();
    for_my_cells<BC>(L, [&](int x, int y, int z) {
        if (((x + y + z) & 1) != color) return;
        const int64_t i = index_of(x, y, z, L);
        const T pc = p[i];
        const T a = neg_lap<BC, true>(p, i, x, y, z, L, T(0), pc);
        p[i] = pc + (rhs[i] - a) / diag_at<BC>(x, y, z, L);
    });
}

// Sum of a level into the site (for the mean gauge of singular problems).
template <int BC, class T>
__global__ void __launch_bounds__(kThreads) level_sum_kernel(const T* __restrict__ x, Lv<T> L, Site s) {
    pdl_enter();
    double local = 0.0;
    for_my_cells<BC>(L, [&](int cx, int cy, int cz) { local += double(x[index_of(cx, cy, cz, L)]); });
    site_finish(s, local);
}

// Coarsest level: p = inv (rhs) with the dense inverse of the (regularised)
// operator, accumulated in TC; singular problems then subtract the mean of p
// (summed in index order by thread 0: at most 512 cells).
constexpr int kDenseThreads = 512;

template <int BC, class T, class TC>
__global__ void __launch_bounds__(kDenseThreads) rb_dense_kernel(const T* __restrict__ rhs, T* __restrict__ p,
                                                                 const TC* __restrict__ inv, int n) {
    pdl_enter();
    __shared__ TC r[kDenseThreads];
    __shared__ T out[kDenseThreads];
    __shared__ double mean;
    for (int i = threadIdx.x; i < n; i += kDenseThreads) r[i] = TC(rhs[i]);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += kDenseThreads) {
        TC acc = TC(0);
        for (int j = 0; j < n; ++j) acc = fma(inv[int64_t(i) * n + j], r[j], acc);
        out[i] = T(acc);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sum = 0.0;
        if (singular_bc(BC))
            for (int i = 0; i < n; ++i) sum += double(out[i]);
        mean = sum / n;
    }
    __syncthreads();
    const T m = T(mean);
    for (int i = threadIdx.x; i < n; i += kDenseThreads) p[i] = out[i] - m;
}

// Iterative refinement (precision form): the residual of the FP64 iterate in
// FP64, handed to the FP32 V-cycles as float, with the norm of the FP64
// residual; then the FP32 correction added to the FP64 iterate.
template <int BC>
__global__ void __launch_bounds__(kThreads) refine_residual_kernel(const double* __restrict__ p,
                                                                   const double* __restrict__ rhs,
                                                                   float* __restrict__ out, Lv<double> L, Site s,
                                                                   double* norm_out) {
    pdl_enter();
    double local = 0.0;
    for_my_cells<BC>(L, [&](int x, int y, int z) {
        const int64_t i = index_of(x, y, z, L);
        const double pc = p[i];
        const double r = rhs[i] - neg_lap<BC, true>(p, i, x, y, z, L, 0.0, pc);
        out[i] = float(r);
        local += r * r;
    });
    site_finish(s, local, norm_out);
}

__global__ void __launch_bounds__(kThreads) refine_correct_kernel(double* __restrict__ p, const float* __restrict__ e,
                                                                  int64_t n) {
    pdl_enter();
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        p[i] = p[i] + double(e[i]);
}

}  // namespace afsi

using namespace afsi;

namespace {

struct Geometry {
    dim3 grid, block;
    int64_t blocks;
};

// Block over the two fastest axes (z,y in 3D; y,x in 2D), grid z over x (3D).
template <class T>
Geometry launch_for(const Lv<T>& L, int bc) {
    const bool three = is3d(bc);
    const int fast = three ? L.nz : L.ny;
    const int mid = three ? L.ny : L.nx;
    const int slow = three ? L.nx : 1;
    int bx = 1;
    while (bx < fast && bx < 32) bx <<= 1;
    int by = kThreads / bx;
    // shrink toward the middle extent, keeping whole warps per block
    while (by > 1 && (by >> 1) >= mid && bx * (by >> 1) >= 32) by >>= 1;
    Geometry g;
    g.block = dim3(bx, by, 1);
    const int gx = (fast + bx - 1) / bx, gy = (mid + by - 1) / by;
    // cap the blocks at 16 per SM of a B200 (x slabs beyond are strided inside
    // the kernel), which bounds the arrivals at a reducing launch's completion
    // counter; up to 64^3 every thread owns one cell
    const int cap = std::max(1, 2368 / std::max(1, gx * gy));
    g.grid = dim3(gx, gy, std::min(slow, cap));
    g.blocks = int64_t(g.grid.x) * g.grid.y * g.grid.z;
    return g;
}

// Geometry of sweep_zpair_kernel: launch_for with the z extent halved.
template <class T>
Geometry launch_for_zpairs(Lv<T> L) {
    L.nz /= 2;
    return launch_for(L, AFSI_BC_NEUMANN);
}

int flat_grid(int64_t n) {
    int64_t b = (n + kThreads - 1) / kThreads;
    return int(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

template <class T>
Lv<T> make_level(const int64_t* shape, const double* h2, const double* ih2, int dim) {
    Lv<T> L;
    L.nx = int(shape[0]);
    L.ny = int(shape[1]);
    L.nz = dim == 3 ? int(shape[2]) : 1;
    L.n = int64_t(L.nx) * L.ny * L.nz;
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
    C.n = int64_t(C.nx) * C.ny * C.nz;
    return C;
}

int32_t check_bc(int32_t dim, int32_t bc) {
    AFSI_REQUIRE((dim == 3 && (bc == AFSI_BC_NEUMANN || bc == AFSI_BC_DIRICHLET)) ||
                     (dim == 2 && (bc == AFSI_BC_CHANNEL || bc == AFSI_BC_PERIODIC)),
                 "unsupported dim/boundary combination (%d, %d)", dim, bc);
    return AFSI_OK;
}

#define AFSI_BC_DISPATCH(bc, ...)                                                   \
    switch (bc) {                                                                   \
    case AFSI_BC_NEUMANN: { constexpr int BC = AFSI_BC_NEUMANN; __VA_ARGS__; } break; \
    case AFSI_BC_CHANNEL: { constexpr int BC = AFSI_BC_CHANNEL; __VA_ARGS__; } break; \
    case AFSI_BC_PERIODIC: { constexpr int BC = AFSI_BC_PERIODIC; __VA_ARGS__; } break; \
    case AFSI_BC_DIRICHLET: { constexpr int BC = AFSI_BC_DIRICHLET; __VA_ARGS__; } break; \
    default: return fail(AFSI_ERR_ARG, "unknown boundary condition %d", (int)(bc)); \
    }

int32_t check_shape(const int64_t* shape, int dim) {
    AFSI_REQUIRE(shape, "null shape");
    for (int a = 0; a < dim; ++a)
        AFSI_REQUIRE(shape[a] > 0 && shape[a] <= (int64_t(1) << 20), "grid extent out of range");
    int64_t n = 1;
    for (int a = 0; a < dim; ++a) n *= shape[a];
    AFSI_REQUIRE(n < (int64_t(1) << 31), "grid too large for one level");
    if (dim == 3) AFSI_REQUIRE(shape[0] <= 65535, "x extent exceeds the launch grid");
    return AFSI_OK;
}

// Loop decision of the solve graph: count the block's cycles, keep the norm,
// flag a nonfinite norm, and continue while the norm is above loop[0] and
// another block fits max_cycles.
__global__ void mg_decide_kernel(double* loop, const double* norm, int check_every, int max_cycles,
                                 cudaGraphConditionalHandle handle) {
    pdl_enter();
    const double cycles = loop[1] + check_every;
    const double r = *norm;
    loop[1] = cycles;
    loop[2] = r;
    const bool finite = isfinite(r);
    if (!finite) loop[3] = 1.0;
    const bool again = finite && r > loop[0] && cycles + check_every <= max_cycles;
    cudaGraphSetConditional(handle, again ? 1u : 0u);
}

// ---- fused V-cycle plan execution ----

// Scratch layout: kSites reduction sites, each `width` partial doubles (the
// largest block count of the finest level, x4 for the stats kernel), then a
// result double and a counter.
constexpr int kSites = AFSI_MG_MAX_LEVELS * 3 + 1;

int64_t partial_width(const afsi_mg_plan* plan) {
    int64_t blocks = 4096;
    if (plan && plan->levels >= 1) {
        Lv<double> L = make_level<double>(plan->level[0].shape, plan->level[0].h2, plan->level[0].inv_h2, plan->dim);
        blocks = std::max<int64_t>(blocks, launch_for(L, plan->bc).blocks);
    }
    return blocks;
}

int64_t site_bytes(int64_t width) { return width * 8 * 4 + 64; }

struct SiteTable {
    Site s[AFSI_MG_MAX_LEVELS][3];  // 0: p after down sweeps, 1: p after up sweeps, 2: rhs
    Site norm;
};

SiteTable sites_for(const afsi_mg_plan* plan) {
    const int64_t width = partial_width(plan), bytes = site_bytes(width);
    SiteTable t;
    unsigned char* base = static_cast<unsigned char*>(plan->scratch);
    auto make = [&](int idx) {
        unsigned char* b = base + int64_t(idx) * bytes;
        Site s;
        s.partial = reinterpret_cast<double*>(b);
        s.result = reinterpret_cast<double*>(b + width * 8 * 4);
        s.counter = reinterpret_cast<unsigned int*>(b + width * 8 * 4 + 8);
        return s;
    };
    int k = 0;
    for (int l = 0; l < AFSI_MG_MAX_LEVELS; ++l)
        for (int j = 0; j < 3; ++j) t.s[l][j] = make(k++);
    t.norm = make(k++);
    return t;
}

constexpr int64_t kClusterCells = 512;  // cells per CTA of the first cluster level

template <int BC, class T, class TC>
struct Runner {
    const afsi_mg_plan* plan;
    cudaStream_t stream;
    SiteTable st;
    Lv<T> lv[AFSI_MG_MAX_LEVELS];
    int first_coarse;
    int first_cluster = AFSI_MG_MAX_LEVELS;  // levels from here run in the cluster kernel (3D)
    int cluster_size = 0;
    size_t cluster_bytes = 0;
    ClusterLevels<T> ccl;

    T* P(int l) const { return static_cast<T*>(plan->level[l].p); }
    T* Q(int l) const { return static_cast<T*>(plan->level[l].ping); }
    T* R(int l) const { return static_cast<T*>(plan->level[l].rhs); }
    static constexpr bool singular = singular_bc(BC);

    // Two z cells per thread (sweep_zpair_kernel) on 3D levels with even nz
    // whose buffers are 16-byte aligned.
    bool zpairs(int l) const {
        if constexpr (BC == AFSI_BC_NEUMANN || BC == AFSI_BC_DIRICHLET) {
            const auto a16 = [](const void* q) { return reinterpret_cast<uintptr_t>(q) % 16 == 0; };
            return lv[l].nz % 2 == 0 && a16(P(l)) && a16(Q(l)) && a16(R(l));
        } else {
            return false;
        }
    }

    int32_t coarse(int l, const double* rhs_sum, T** out) {
        CoarseLevels<T> cl;
        for (int k = 0; k < plan->levels; ++k) cl.lv[k] = lv[k];
        cl.first = l;
        cl.last = plan->levels - 1;
        int64_t cells = 0;
        for (int k = l; k < plan->levels; ++k) cells += lv[k].n;
        const size_t bytes = (size_t(cells) * 3 + 64 * size_t(plan->levels - l)) * sizeof(T);
        static bool configured = false;  // once per instantiation, before any graph capture of it
        if (!configured) {
            cudaFuncSetAttribute(coarse_kernel<BC, T, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024);
            configured = true;
        }
        *out = P(l);
        return launch_pdl("mg coarse block", coarse_kernel<BC, T, TC>, dim3(1), dim3(kCoarseThreads), bytes, stream,
                          R(l), rhs_sum, l == 0 ? P(0) : nullptr, P(l), static_cast<const TC*>(plan->coarse_inverse),
                          cl, plan->smooth);
    }

    int32_t cluster(int l, const double* rhs_sum, T** out) {
        *out = P(l);
        if constexpr (is3d(BC)) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(cluster_size);
            cfg.blockDim = dim3(kCoarseThreads);
            cfg.dynamicSmemBytes = cluster_bytes;
            cfg.stream = stream;
            // programmatic dependent launch as for the level kernels: the cluster's
            // CTAs may start while the restriction drains and wait in pdl_enter
            cudaLaunchAttribute attr[2];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = cluster_size;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attr[1].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 2;
            const cudaError_t err =
                cudaLaunchKernelEx(&cfg, cluster_kernel<BC, T, TC>, static_cast<const T*>(R(l)), rhs_sum,
                                   static_cast<const T*>(l == 0 ? P(0) : nullptr), P(l),
                                   static_cast<const TC*>(plan->coarse_inverse), ccl, plan->smooth);
            if (err != cudaSuccess) return fail(AFSI_ERR_CUDA, "mg cluster block: %s", cudaGetErrorString(err));
            return launched("mg cluster block");
        } else {
            return fail(AFSI_ERR_ARG, "cluster path is 3D only");
        }
    }

    // Cluster plan for the 3D BCs: the first level whose x extent splits into
    // 16 slabs of at most kClusterCells cells, distributed while nx is a
    // multiple of 16 (at least 16), then replicated; used when it starts no
    // coarser than the single-CTA block and leaves the coarsest level
    // replicated.  Measured on the B200: a 16-CTA cluster beats the single CTA
    // on 16^3 -> 4^3 (33 vs 38 us per cycle); with the 32^3 level inside
    // (2048 cells per CTA) it loses to launched 32^3 kernels, and an 8-CTA
    // cluster loses to the single CTA.
    void plan_cluster() {
        if constexpr (is3d(BC)) {
            const int C = cluster_capacity();
            if (C != kClusterMax) return;
            const int last = plan->levels - 1;
            for (int l = 0; l < last && l <= first_coarse; ++l) {
                const Lv<T>& L = lv[l];
                if (L.nx % C || L.nx < C || L.n / C > kClusterCells) continue;
                int64_t off = 0;
                bool distributed = true;
                for (int k = l; k <= last; ++k) {
                    ClusterLevel<T>& c = ccl.lv[k];
                    c.L = lv[k];
                    distributed = distributed && k < last && lv[k].nx % C == 0 && lv[k].nx >= C;
                    c.ppc = distributed ? lv[k].nx / C : 0;
                    c.cells = int(distributed ? lv[k].n / C : lv[k].n);
                    c.off = int(off);
                    off += 3 * int64_t(c.cells);
                }
                ccl.tables = int(off);
                const size_t bytes = size_t(off + 64 * (last - l + 1)) * sizeof(T);
                if (bytes > 200 * 1024) continue;
                ccl.first = l;
                ccl.last = last;
                first_cluster = l;
                cluster_size = C;
                cluster_bytes = bytes;
                return;
            }
        }
    }

    // Largest cluster (16, else 8) that this device runs with 1024-thread
    // CTAs and 200 KB of shared memory each; 0 if none.  Queried once per
    // instantiation, on the first (uncaptured) run.
    static int cluster_capacity() {
        static int capacity = -1;
        if constexpr (is3d(BC)) {
            if (capacity < 0) {
                capacity = 0;
                auto kernel = cluster_kernel<BC, T, TC>;
                cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
                for (int C : {16, 8}) {
                    if (C > 8 && cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                                     cudaSuccess) {
                        cudaGetLastError();
                        continue;
                    }
                    cudaLaunchConfig_t cfg = {};
                    cfg.gridDim = dim3(C);
                    cfg.blockDim = dim3(kCoarseThreads);
                    cfg.dynamicSmemBytes = 200 * 1024;
                    cudaLaunchAttribute attr;
                    attr.id = cudaLaunchAttributeClusterDimension;
                    attr.val.clusterDim.x = C;
                    attr.val.clusterDim.y = 1;
                    attr.val.clusterDim.z = 1;
                    cfg.attrs = &attr;
                    cfg.numAttrs = 1;
                    int clusters = 0;
                    if (cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg) == cudaSuccess && clusters > 0) {
                        capacity = C;
                        break;
                    }
                    cudaGetLastError();
                }
            }
        }
        return capacity < 0 ? 0 : capacity;
    }

    // Returns the buffer holding the level's final iterate and the site whose
    // sum is its pending mean (nullptr: exact).
    int32_t level(int l, T** out, const double** out_sum) {
        int32_t rc;
        if (l >= first_cluster) {
            rc = cluster(l, (l > 0 && singular) ? st.s[l][2].result : nullptr, out);
            *out_sum = nullptr;
            return rc;
        }
        if (l >= first_coarse) {
            rc = coarse(l, (l > 0 && singular) ? st.s[l][2].result : nullptr, out);
            *out_sum = nullptr;
            return rc;
        }
        const Lv<T>& L = lv[l];
        const Geometry g = launch_for(L, BC);
        const Geometry gz = launch_for_zpairs(L);
        T* cur = P(l);
        T* oth = Q(l);
        for (int s = 0; s < plan->smooth; ++s) {
            const bool first = s == 0;
            const bool last = s == plan->smooth - 1;
            if (zpairs(l))
                rc = launch_pdl("mg sweep", sweep_zpair_kernel<BC, T>, gz.grid, gz.block, 0, stream,
                                static_cast<const T*>((first && l > 0) ? nullptr : cur), R(l), oth, L,
                                (first && l > 0 && singular) ? st.s[l][2].result : nullptr, st.s[l][0],
                                (first && l > 0 && singular) ? 1 : 0, (last && singular) ? 1 : 0);
            else
                rc = launch_pdl("mg sweep", sweep_kernel<BC, false, T>, g.grid, g.block, 0, stream,
                                (first && l > 0) ? nullptr : cur, R(l), oth, L, static_cast<const double*>(nullptr),
                                (first && l > 0 && singular) ? st.s[l][2].result : nullptr, st.s[l][0],
                                (first && l > 0 && singular) ? 1 : 0, (last && singular) ? 1 : 0);
            if (rc) return rc;
            T* t = cur; cur = oth; oth = t;
        }
        const double* down_sum = singular ? st.s[l][0].result : nullptr;
        const Lv<T>& C = lv[l + 1];
        const Geometry gc = launch_for(C, BC);
        if (zpairs(l))
            rc = launch_pdl("mg residual_restrict", residual_restrict_zpair_kernel<BC, T>, gc.grid, gc.block, 0, stream,
                            cur, R(l), R(l + 1), L, C, down_sum, st.s[l + 1][2], singular ? 1 : 0);
        else
            rc = launch_pdl("mg residual_restrict", residual_restrict_kernel<BC, false, T>, gc.grid, gc.block, 0, stream,
                            cur, R(l), R(l + 1), L, C, down_sum, st.s[l + 1][2], singular ? 1 : 0);
        if (rc) return rc;
        T* corr;
        const double* corr_sum;
        if ((rc = level(l + 1, &corr, &corr_sum))) return rc;
        // the finest level of a singular operator prolongs into the buffer the
        // pre-smoothing left free, so its post-smoothing ends in Q(0) and the
        // finalize (and the fused check of the solve loop) never shifts in place
        T* pdst = (l == 0 && singular && cur == P(l)) ? Q(l) : P(l);
        rc = launch_pdl("mg prolong_add", prolong_kernel<BC, T>, g.grid, g.block, 0, stream, cur,
                        static_cast<const T*>(corr), pdst, L, C, down_sum, corr_sum);
        if (rc) return rc;
        cur = pdst;
        oth = pdst == P(l) ? Q(l) : P(l);
        for (int s = 0; s < plan->smooth; ++s) {
            const bool last = s == plan->smooth - 1;
            if (zpairs(l))
                rc = launch_pdl("mg sweep", sweep_zpair_kernel<BC, T>, gz.grid, gz.block, 0, stream,
                                static_cast<const T*>(cur), R(l), oth, L, static_cast<const double*>(nullptr),
                                st.s[l][1], 0, (last && singular) ? 1 : 0);
            else
                rc = launch_pdl("mg sweep", sweep_kernel<BC, false, T>, g.grid, g.block, 0, stream, cur, R(l), oth,
                                L, static_cast<const double*>(nullptr), static_cast<const double*>(nullptr),
                                st.s[l][1], 0, (last && singular) ? 1 : 0);
            if (rc) return rc;
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
                rc = launch_pdl("mg finalize", shift_kernel<T>, dim3(flat_grid(lv[0].n)), dim3(kThreads), 0, stream,
                                static_cast<const T*>(out), P(0), lv[0].n, sum);
                if (rc) return rc;
            }
        }
        return AFSI_OK;
    }

    // One check block of the solve loop: `count` V-cycles, the residual norm
    // into norm and the loop decision; the last cycle's finalize, the norm and
    // the decision are one launch (finalize_check_kernel) unless the finalize
    // would shift in place.
    int32_t checked_block(int count, double* norm, double* loop, int check_every, int max_cycles,
                          cudaGraphConditionalHandle handle) {
        int32_t rc = cycles(count - 1);
        if (rc) return rc;
        T* out;
        const double* sum;
        if ((rc = level(0, &out, &sum))) return rc;
        const Geometry g = launch_for(lv[0], BC);
        if (out == P(0) && sum) {
            rc = launch_pdl("mg finalize", shift_kernel<T>, dim3(flat_grid(lv[0].n)), dim3(kThreads), 0, stream,
                            static_cast<const T*>(out), P(0), lv[0].n, sum);
            if (!rc)
                rc = launch_pdl("mg residual_norm", residual_norm_kernel<BC, true, T>, g.grid, g.block, 0, stream,
                                static_cast<const T*>(P(0)), static_cast<const T*>(R(0)), lv[0], st.norm, norm);
            if (!rc)
                rc = launch_pdl("mg solve decide", mg_decide_kernel, dim3(1), dim3(1), 0, stream, loop,
                                static_cast<const double*>(norm), check_every, max_cycles, handle);
            return rc;
        }
        return launch_pdl("mg finalize check", finalize_check_kernel<BC, T>, g.grid, g.block, 0, stream,
                          static_cast<const T*>(out), P(0), static_cast<const T*>(R(0)), lv[0], sum, st.norm, norm,
                          loop, check_every, max_cycles, handle);
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
    AFSI_REQUIRE(plan->smoother == AFSI_MG_JACOBI || plan->smoother == AFSI_MG_RED_BLACK, "unknown smoother %d",
                 int(plan->smoother));
    if (plan->smoother == AFSI_MG_RED_BLACK && plan->bc == AFSI_BC_PERIODIC)
        for (int l = 0; l + 1 < plan->levels; ++l)
            AFSI_REQUIRE(plan->level[l].shape[0] % 2 == 0,
                         "red-black smoothing with periodic x needs an even x extent on every smoothed level");
    return AFSI_OK;
}

// First level that fits the single-block path: at most kCoarseCells cells,
// and shared memory for 3 arrays of it and of every coarser level plus the
// per-level tables.
template <class T>
int coarse_start(const Lv<T>* lv, int levels) {
    for (int l = 0; l < levels; ++l) {
        int64_t cells = 0;
        for (int k = l; k < levels; ++k) cells += lv[k].n;
        if (lv[l].n <= kCoarseCells && (cells * 3 + 64 * (levels - l)) * int64_t(sizeof(T)) <= 200 * 1024) return l;
    }
    return levels - 1;
}

template <class T>
size_t coarse_smem_bytes(const Lv<T>* lv, int first, int levels) {
    int64_t cells = 0;
    for (int k = first; k < levels; ++k) cells += lv[k].n;
    return (size_t(cells) * 3 + 64 * size_t(levels - first)) * sizeof(T);
}

template <int BC, class T, class TC>
void setup_runner(Runner<BC, T, TC>& r, const afsi_mg_plan* plan, cudaStream_t stream) {
    r.plan = plan;
    r.stream = stream;
    r.st = sites_for(plan);
    for (int l = 0; l < plan->levels; ++l)
        r.lv[l] = make_level<T>(plan->level[l].shape, plan->level[l].h2, plan->level[l].inv_h2, plan->dim);
    r.first_coarse = coarse_start(r.lv, plan->levels);
    r.plan_cluster();
}

template <int BC, class T, class TC>
int32_t run_plan(const afsi_mg_plan* plan, int cycles, cudaStream_t stream) {
    Runner<BC, T, TC> r;
    setup_runner(r, plan, stream);
    return r.cycles(cycles);
}

template <int BC, class T, class TC>
int32_t run_plan_checked(const afsi_mg_plan* plan, int cycles, cudaStream_t stream, double* norm, double* loop,
                         int max_cycles, cudaGraphConditionalHandle handle) {
    Runner<BC, T, TC> r;
    setup_runner(r, plan, stream);
    return r.checked_block(cycles, norm, loop, cycles, max_cycles, handle);
}

}  // namespace

extern "C" int64_t afsi_b200_mg_scratch_bytes(const afsi_mg_plan* plan) {
    return int64_t(kSites) * site_bytes(partial_width(plan));
}

// V-cycles with the red-black smoother: per level `smooth` sweeps of two
// half-sweeps before and after the coarse correction, the fused residual
// restriction (coarse right-hand side shifted to mean zero for singular
// problems), a zero coarse start, the dense coarsest solve and the
// prolongation of mac/multigrid.py:112-123; the finest iterate is shifted to
// mean zero after every cycle for singular problems.
template <int BC, class T, class TC>
struct RbRunner {
    const afsi_mg_plan* plan;
    cudaStream_t stream;
    SiteTable st;
    Lv<T> lv[AFSI_MG_MAX_LEVELS];
    int first_coarse;  // levels from here run in one CTA (coarse_rb_kernel)
    static constexpr bool singular = singular_bc(BC);

    int32_t coarse(int l) {
        CoarseLevels<T> cl;
        for (int k = 0; k < plan->levels; ++k) cl.lv[k] = lv[k];
        cl.first = l;
        cl.last = plan->levels - 1;
        int64_t cells = 0;
        for (int k = l; k < plan->levels; ++k) cells += lv[k].n;
        const size_t bytes = (size_t(cells) * 3 + 64 * size_t(plan->levels - l)) * sizeof(T);
        static bool configured = false;  // once per instantiation, before any graph capture of it
        if (!configured) {
            cudaFuncSetAttribute(coarse_rb_kernel<BC, T, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 210 * 1024);
            configured = true;
        }
        return launch_pdl("mg red-black coarse block", coarse_rb_kernel<BC, T, TC>, dim3(1), dim3(kCoarseThreads),
                          bytes, stream, static_cast<const T*>(R(l)), static_cast<const T*>(l == 0 ? P(0) : nullptr),
                          P(l), static_cast<const TC*>(plan->coarse_inverse), cl, plan->smooth);
    }

    T* P(int l) const { return static_cast<T*>(plan->level[l].p); }
    T* R(int l) const { return static_cast<T*>(plan->level[l].rhs); }

    int32_t smooth(int l) {
        const Geometry g = launch_for(lv[l], BC);
        for (int k = 0; k < plan->smooth; ++k)
            for (int color = 0; color < 2; ++color) {
                const int32_t rc = launch_pdl("mg red-black sweep", rb_kernel<BC, T>, g.grid, g.block, 0, stream, P(l),
                                              static_cast<const T*>(R(l)), lv[l], color);
                if (rc) return rc;
            }
        return AFSI_OK;
    }

    int32_t shift_to_mean_zero(T* x, int l, const Site& site) {
        const Geometry g = launch_for(lv[l], BC);
        int32_t rc = launch_pdl("mg level sum", level_sum_kernel<BC, T>, g.grid, g.block, 0, stream,
                                static_cast<const T*>(x), lv[l], site);
        if (rc) return rc;
        return launch_pdl("mg mean shift", shift_kernel<T>, dim3(flat_grid(lv[l].n)), dim3(kThreads), 0, stream,
                          static_cast<const T*>(x), x, lv[l].n, static_cast<const double*>(site.result));
    }

    int32_t level(int l) {
        const int last = plan->levels - 1;
        int32_t rc;
        if (l == first_coarse && l < last) return coarse(l);
        if (l == last)
            return launch_pdl("mg dense coarse solve", rb_dense_kernel<BC, T, TC>, dim3(1), dim3(kDenseThreads), 0,
                              stream, static_cast<const T*>(R(l)), P(l),
                              static_cast<const TC*>(plan->coarse_inverse), int(lv[l].n));
        if ((rc = smooth(l))) return rc;
        const Geometry gc = launch_for(lv[l + 1], BC);
        rc = launch_pdl("mg residual restrict", residual_restrict_kernel<BC, true, T>, gc.grid, gc.block, 0, stream,
                        static_cast<const T*>(P(l)), static_cast<const T*>(R(l)), R(l + 1), lv[l], lv[l + 1],
                        static_cast<const double*>(nullptr), st.s[l + 1][2], int(singular));
        if (rc) return rc;
        if (singular) {
            rc = launch_pdl("mg mean shift", shift_kernel<T>, dim3(flat_grid(lv[l + 1].n)), dim3(kThreads), 0, stream,
                            static_cast<const T*>(R(l + 1)), R(l + 1), lv[l + 1].n,
                            static_cast<const double*>(st.s[l + 1][2].result));
            if (rc) return rc;
        }
        if (l + 1 < last && l + 1 != first_coarse) {
            const cudaError_t err = cudaMemsetAsync(P(l + 1), 0, size_t(lv[l + 1].n) * sizeof(T), stream);
            if (err != cudaSuccess) return fail(AFSI_ERR_CUDA, "mg zero start: %s", cudaGetErrorString(err));
        }
        if ((rc = level(l + 1))) return rc;
        const Geometry g = launch_for(lv[l], BC);
        rc = launch_pdl("mg prolong add", prolong_kernel<BC, T>, g.grid, g.block, 0, stream,
                        static_cast<const T*>(P(l)), static_cast<const T*>(P(l + 1)), P(l), lv[l], lv[l + 1],
                        static_cast<const double*>(nullptr), static_cast<const double*>(nullptr));
        if (rc) return rc;
        return smooth(l);
    }

    int32_t run(int cycles) {
        for (int l = 0; l < plan->levels; ++l)
            lv[l] = make_level<T>(plan->level[l].shape, plan->level[l].h2, plan->level[l].inv_h2, plan->dim);
        first_coarse = coarse_start(lv, plan->levels);
        for (int c = 0; c < cycles; ++c) {
            int32_t rc = level(0);
            if (!rc && singular) rc = shift_to_mean_zero(P(0), 0, st.s[0][0]);
            if (rc) return rc;
        }
        return AFSI_OK;
    }
};

template <int BC, class T, class TC>
int32_t run_red_black(const afsi_mg_plan* plan, int cycles, cudaStream_t stream) {
    RbRunner<BC, T, TC> r;
    r.plan = plan;
    r.stream = stream;
    r.st = sites_for(plan);
    return r.run(cycles);
}

extern "C" int32_t afsi_b200_mg_vcycles(const afsi_mg_plan* plan, int32_t cycles, afsi_stream_t stream) {
    int32_t rc = validate_plan(plan);
    if (rc) return rc;
    AFSI_REQUIRE(cycles >= 0, "negative cycle count");
    AFSI_REQUIRE(plan->coarse_dtype == AFSI_F64 || plan->coarse_dtype == plan->dtype, "unsupported coarse dtype");
    AFSI_BC_DISPATCH(plan->bc, {
        AFSI_DISPATCH(plan->dtype, {
            if (plan->smoother == AFSI_MG_RED_BLACK) {
                if (plan->coarse_dtype == AFSI_F64) return run_red_black<BC, T, double>(plan, cycles, stream);
                return run_red_black<BC, T, T>(plan, cycles, stream);
            }
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
            const Geometry g = launch_for(L, BC);
            return launch_pdl("mg residual_norm", residual_norm_kernel<BC, true, T>, g.grid, g.block, 0, stream,
                              static_cast<const T*>(plan->level[0].p), static_cast<const T*>(plan->level[0].rhs), L,
                              st.norm, norm_out);
        });
    });
    return AFSI_OK;
}

// ------------------------------------------------------------ solve graph
//
// The solve loop of mac/multigrid.py:88-97 (check_every V-cycles, residual
// norm, stop at tol or max_cycles) as one CUDA graph: a WHILE conditional
// node whose body holds check_every V-cycles, the residual norm and a decide
// kernel that updates the loop state and sets the condition.  One graph
// launch replaces check_every-sized host round trips.  The body stops before
// a block of check_every cycles would pass max_cycles; the caller runs any
// tail on the host path.
//
// loop (device double[4]): [0] tol (written by the caller before each
// launch), [1] cycles run, [2] last residual norm, [3] 1 when the norm was
// nonfinite.

namespace {


struct SolveGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t capture = nullptr;
};

void release(SolveGraph* sg) {
    if (!sg) return;
    if (sg->exec) cudaGraphExecDestroy(sg->exec);
    if (sg->graph) cudaGraphDestroy(sg->graph);
    if (sg->capture) cudaStreamDestroy(sg->capture);
    delete sg;
}

}  // namespace

// Start of a solve in the started loop graph: the tolerance
// max(atol, rtol ||b||) from the shifted right-hand side's sum of squares,
// the compatibility screen of a singular operator, and the WHILE condition
// (the initial residual above the tolerance, every input finite and
// compatible).  params: [rtol, atol, rel, n] (rel: the screen's relative
// bound); stats: vector_stats of the raw rhs [0:4], of the initial iterate
// [4:8] and of the shifted rhs [8:12].
__global__ void mg_loop_start_kernel(double* loop, const double* norm, const double* stats, const double* params,
                                     int singular, int check_every, int max_cycles,
                                     cudaGraphConditionalHandle handle) {
    pdl_enter();
    const double rhs_norm = sqrt(stats[10]);
    const double tol = fmax(params[1], params[0] * rhs_norm);
    const double r = *norm, n = params[3];
    const bool compatible = !singular || fabs(stats[0] / n) <= 1e-12 + params[2] * (stats[1] / n);
    loop[0] = tol;
    loop[1] = 0.0;
    loop[2] = r;
    loop[3] = isfinite(r) ? 0.0 : 1.0;
    const bool go = stats[3] != 0.0 && stats[7] != 0.0 && compatible && isfinite(rhs_norm) && isfinite(r) && r > tol &&
                    check_every <= max_cycles;
    cudaGraphSetConditional(handle, go ? 1u : 0u);
}

// Body of the solve loop: check_every V-cycles, the residual norm and the
// decision (fused into one launch for the Jacobi schedule).
int32_t check_block(const afsi_mg_plan* plan, int check_every, int max_cycles, double* loop, double* norm,
                    cudaGraphConditionalHandle handle, cudaStream_t stream) {
    if (plan->smoother == AFSI_MG_JACOBI) {
        AFSI_BC_DISPATCH(plan->bc, {
            AFSI_DISPATCH(plan->dtype, {
                if (plan->coarse_dtype == AFSI_F64)
                    return run_plan_checked<BC, T, double>(plan, check_every, stream, norm, loop, max_cycles, handle);
                return run_plan_checked<BC, T, T>(plan, check_every, stream, norm, loop, max_cycles, handle);
            });
        });
    }
    int32_t rc = afsi_b200_mg_vcycles(plan, check_every, stream);
    if (!rc) rc = afsi_b200_mg_residual_norm(plan, norm, stream);
    if (!rc)
        rc = launch_pdl("mg solve decide", mg_decide_kernel, dim3(1), dim3(1), 0, stream, loop,
                        static_cast<const double*>(norm), check_every, max_cycles, handle);
    return rc;
}

extern "C" int32_t afsi_b200_mg_solve_graph_create(const afsi_mg_plan* plan, int32_t check_every,
                                                   int32_t max_cycles, double* loop, double* norm,
                                                   void** graph_out) {
    int32_t rc = validate_plan(plan);
    if (rc) return rc;
    AFSI_REQUIRE(graph_out && loop && norm, "null solve-graph argument");
    AFSI_REQUIRE(check_every >= 1 && max_cycles >= check_every, "solve graph needs 1 <= check_every <= max_cycles");
    AFSI_REQUIRE(plan->coarse_dtype == AFSI_F64 || plan->coarse_dtype == plan->dtype, "unsupported coarse dtype");
    *graph_out = nullptr;
    SolveGraph* sg = new SolveGraph;
    cudaGraphConditionalHandle handle;
    cudaGraphNodeParams np = {};
    cudaGraphNode_t node;
    if (cudaStreamCreateWithFlags(&sg->capture, cudaStreamNonBlocking) != cudaSuccess ||
        cudaGraphCreate(&sg->graph, 0) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&handle, sg->graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
        release(sg);
        return fail(AFSI_ERR_CUDA, "solve graph setup failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    if (cudaGraphAddNode(&node, sg->graph, nullptr, 0, &np) != cudaSuccess) {
        release(sg);
        return fail(AFSI_ERR_CUDA, "solve graph conditional node failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    cudaGraph_t body = np.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(sg->capture, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) !=
        cudaSuccess) {
        release(sg);
        return fail(AFSI_ERR_CUDA, "solve graph capture failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    rc = check_block(plan, check_every, max_cycles, loop, norm, handle, sg->capture);
    cudaGraph_t captured = nullptr;
    const cudaError_t end = cudaStreamEndCapture(sg->capture, &captured);
    if (rc) {
        release(sg);
        return rc;
    }
    if (end != cudaSuccess || cudaGraphInstantiate(&sg->exec, sg->graph, 0) != cudaSuccess) {
        release(sg);
        return fail(AFSI_ERR_CUDA, "solve graph instantiation failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    *graph_out = sg;
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_vector_stats(const void* x, int64_t n, double* stats_out, void* scratch, int32_t dtype,
                                          afsi_stream_t stream);
extern "C" int32_t afsi_b200_subtract_mean(void* x, int64_t n, const double* stats, int32_t dtype,
                                          afsi_stream_t stream);

extern "C" int32_t afsi_b200_mg_solve_graph_create_started(const afsi_mg_plan* plan, int32_t check_every,
                                                           int32_t max_cycles, double* loop, double* norm,
                                                           double* stats, void* stat_scratch, const double* params,
                                                           void** graph_out) {
    int32_t rc = validate_plan(plan);
    if (rc) return rc;
    AFSI_REQUIRE(graph_out && loop && norm && stats && stat_scratch && params, "null solve-graph argument");
    AFSI_REQUIRE(check_every >= 1 && max_cycles >= check_every, "solve graph needs 1 <= check_every <= max_cycles");
    AFSI_REQUIRE(plan->coarse_dtype == AFSI_F64 || plan->coarse_dtype == plan->dtype, "unsupported coarse dtype");
    *graph_out = nullptr;
    const int singular = plan->bc == AFSI_BC_NEUMANN || plan->bc == AFSI_BC_PERIODIC ? 1 : 0;
    int64_t n = 1;
    for (int a = 0; a < plan->dim; ++a) n *= plan->level[0].shape[a];
    SolveGraph* sg = new SolveGraph;
    cudaGraphConditionalHandle handle;
    if (cudaStreamCreateWithFlags(&sg->capture, cudaStreamNonBlocking) != cudaSuccess ||
        cudaGraphCreate(&sg->graph, 0) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&handle, sg->graph, 0, cudaGraphCondAssignDefault) != cudaSuccess) {
        release(sg);
        return fail(AFSI_ERR_CUDA, "solve graph setup failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    // the start: statistics, gauge shift, initial residual, tolerance and condition
    if (cudaStreamBeginCaptureToGraph(sg->capture, sg->graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) !=
        cudaSuccess) {
        release(sg);
        return fail(AFSI_ERR_CUDA, "solve graph capture failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    void* rhs = plan->level[0].rhs;
    void* p0 = plan->level[0].p;
    rc = afsi_b200_vector_stats(rhs, n, stats, stat_scratch, plan->dtype, sg->capture);
    if (!rc) rc = afsi_b200_vector_stats(p0, n, stats + 4, stat_scratch, plan->dtype, sg->capture);
    if (!rc && singular) {
        rc = afsi_b200_subtract_mean(rhs, n, stats, plan->dtype, sg->capture);
        if (!rc) rc = afsi_b200_subtract_mean(p0, n, stats + 4, plan->dtype, sg->capture);
        if (!rc) rc = afsi_b200_vector_stats(rhs, n, stats + 8, stat_scratch, plan->dtype, sg->capture);
    } else if (!rc && cudaMemcpyAsync(stats + 8, stats, 4 * sizeof(double), cudaMemcpyDeviceToDevice, sg->capture) !=
                          cudaSuccess) {
        rc = fail(AFSI_ERR_CUDA, "solve graph statistics copy failed");
    }
    if (!rc) rc = afsi_b200_mg_residual_norm(plan, norm, sg->capture);
    if (!rc)
        rc = launch_pdl("mg solve start", mg_loop_start_kernel, dim3(1), dim3(1), 0, sg->capture, loop,
                        static_cast<const double*>(norm), static_cast<const double*>(stats), params, singular,
                        check_every, max_cycles, handle);
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaStreamCaptureStatus status;
    if (!rc && cudaStreamGetCaptureInfo(sg->capture, &status, nullptr, nullptr, &deps, &ndeps) != cudaSuccess)
        rc = fail(AFSI_ERR_CUDA, "solve graph capture info failed");
    std::vector<cudaGraphNode_t> start_leaves(deps, deps + (rc ? 0 : ndeps));
    cudaGraph_t captured = nullptr;
    cudaError_t end = cudaStreamEndCapture(sg->capture, &captured);
    if (rc || end != cudaSuccess) {
        release(sg);
        return rc ? rc : fail(AFSI_ERR_CUDA, "solve graph capture failed: %s", cudaGetErrorString(end));
    }
    // the loop, after the start
    cudaGraphNodeParams np = {};
    cudaGraphNode_t node;
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    if (cudaGraphAddNode(&node, sg->graph, start_leaves.data(), start_leaves.size(), &np) != cudaSuccess) {
        release(sg);
        return fail(AFSI_ERR_CUDA, "solve graph conditional node failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    cudaGraph_t body = np.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(sg->capture, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) !=
        cudaSuccess) {
        release(sg);
        return fail(AFSI_ERR_CUDA, "solve graph capture failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    rc = check_block(plan, check_every, max_cycles, loop, norm, handle, sg->capture);
    end = cudaStreamEndCapture(sg->capture, &captured);
    if (rc) {
        release(sg);
        return rc;
    }
    if (end != cudaSuccess || cudaGraphInstantiate(&sg->exec, sg->graph, 0) != cudaSuccess) {
        release(sg);
        return fail(AFSI_ERR_CUDA, "solve graph instantiation failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    *graph_out = sg;
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_mg_solve_graph_launch(void* graph, afsi_stream_t stream) {
    AFSI_REQUIRE(graph, "null solve graph");
    if (cudaGraphLaunch(static_cast<SolveGraph*>(graph)->exec, stream) != cudaSuccess)
        return fail(AFSI_ERR_CUDA, "solve graph launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_mg_solve_graph_destroy(void* graph) {
    release(static_cast<SolveGraph*>(graph));
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_vector_stats(const void* x, int64_t n, double* stats_out, void* scratch, int32_t dtype,
                                          afsi_stream_t stream) {
    AFSI_REQUIRE(n > 0 && x && stats_out && scratch, "invalid stats arguments");
    unsigned char* b = static_cast<unsigned char*>(scratch);
    double* partial = reinterpret_cast<double*>(b);
    unsigned int* counter = reinterpret_cast<unsigned int*>(b + int64_t(4096) * 8 * 4 + 8);
    AFSI_DISPATCH(dtype, {
        stats_kernel<T><<<flat_grid(n), kThreads, 0, stream>>>(static_cast<const T*>(x), n, partial, counter,
                                                               stats_out);
    });
    return launched("vector_stats");
}

extern "C" int32_t afsi_b200_subtract_mean(void* x, int64_t n, const double* stats, int32_t dtype,
                                           afsi_stream_t stream) {
    AFSI_REQUIRE(n > 0 && x && stats, "invalid subtract_mean arguments");
    AFSI_DISPATCH(dtype, {
        shift_kernel<T><<<flat_grid(n), kThreads, 0, stream>>>(static_cast<const T*>(x), static_cast<T*>(x), n,
                                                               stats);
    });
    return launched("subtract_mean");
}

// ---- iterative refinement (precision form) ----

extern "C" int64_t afsi_b200_mg_refine_scratch_bytes(const int64_t* shape, int32_t dim, int32_t bc) {
    if (check_bc(dim, bc) || check_shape(shape, dim)) return -1;
    const double one[3] = {1, 1, 1};
    const Geometry g = launch_for(make_level<double>(shape, one, one, dim), bc);
    return g.blocks * 8 + 64;
}

extern "C" int32_t afsi_b200_mg_refine_residual(const double* p, const double* rhs, float* r32, const int64_t* shape,
                                                const double* h2, int32_t dim, int32_t bc, double* norm_out,
                                                void* scratch, afsi_stream_t stream) {
    int32_t rc = check_bc(dim, bc);
    if (rc || (rc = check_shape(shape, dim))) return rc;
    AFSI_REQUIRE(p && rhs && r32 && h2 && norm_out && scratch, "null argument");
    AFSI_REQUIRE(reinterpret_cast<uintptr_t>(scratch) % 16 == 0, "refinement scratch must be 16-byte aligned");
    const double one[3] = {1, 1, 1};
    Lv<double> L = make_level<double>(shape, h2, one, dim);
    const Geometry g = launch_for(L, bc);
    unsigned char* b = static_cast<unsigned char*>(scratch);
    const Site site{reinterpret_cast<double*>(b), reinterpret_cast<unsigned int*>(b + g.blocks * 8 + 8),
                    reinterpret_cast<double*>(b + g.blocks * 8)};
    AFSI_BC_DISPATCH(bc, {
        return launch_pdl("mg refine residual", refine_residual_kernel<BC>, g.grid, g.block, 0, stream, p, rhs, r32,
                          L, site, norm_out);
    });
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_mg_refine_correct(double* p, const float* e, int64_t n, afsi_stream_t stream) {
    AFSI_REQUIRE(p && e && n > 0, "invalid refinement correction arguments");
    return launch_pdl("mg refine correct", refine_correct_kernel, dim3(flat_grid(n)), dim3(kThreads), 0, stream, p,
                      e, n);
}

// ---- standalone kernel-object entry points (exact arithmetic) ----

extern "C" int32_t afsi_b200_mg_smooth(const void* p, const void* rhs, void* out, const int64_t* shape,
                                       const double* h2, const double* inv_h2, int32_t dim, int32_t bc,
                                       int32_t dtype, afsi_stream_t stream) {
    int32_t rc = check_bc(dim, bc);
    if (rc || (rc = check_shape(shape, dim))) return rc;
    AFSI_REQUIRE(p && rhs && out && h2 && inv_h2, "null argument");
    AFSI_BC_DISPATCH(bc, {
        AFSI_DISPATCH(dtype, {
            Lv<T> L = make_level<T>(shape, h2, inv_h2, dim);
            const Geometry g = launch_for(L, BC);
            Site none{nullptr, nullptr, nullptr};
            sweep_kernel<BC, true, T><<<g.grid, g.block, 0, stream>>>(
                static_cast<const T*>(p), const_cast<T*>(static_cast<const T*>(rhs)), static_cast<T*>(out), L,
                nullptr, nullptr, none, 0, 0);
        });
    });
    return launched("mg_smooth");
}

extern "C" int32_t afsi_b200_mg_residual(const void* p, const void* rhs, void* out, const int64_t* shape,
                                         const double* h2, int32_t dim, int32_t bc, int32_t dtype,
                                         afsi_stream_t stream) {
    int32_t rc = check_bc(dim, bc);
    if (rc || (rc = check_shape(shape, dim))) return rc;
    AFSI_REQUIRE(p && rhs && out && h2, "null argument");
    AFSI_BC_DISPATCH(bc, {
        AFSI_DISPATCH(dtype, {
            Lv<T> L = make_level<T>(shape, h2, nullptr, dim);
            const Geometry g = launch_for(L, BC);
            residual_kernel<BC, true, T><<<g.grid, g.block, 0, stream>>>(
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
        if (dim == 3) {
            const Geometry g = launch_for(C, AFSI_BC_NEUMANN);
            restrict_kernel<AFSI_BC_NEUMANN, T><<<g.grid, g.block, 0, stream>>>(
                static_cast<const T*>(fine), static_cast<T*>(coarse), L, C);
        } else {
            const Geometry g = launch_for(C, AFSI_BC_CHANNEL);
            restrict_kernel<AFSI_BC_CHANNEL, T><<<g.grid, g.block, 0, stream>>>(
                static_cast<const T*>(fine), static_cast<T*>(coarse), L, C);
        }
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
            const Geometry g = launch_for(C, BC);
            Site none{nullptr, nullptr, nullptr};
            residual_restrict_kernel<BC, true, T><<<g.grid, g.block, 0, stream>>>(
                static_cast<const T*>(p), static_cast<const T*>(rhs), static_cast<T*>(coarse), L, C, nullptr, none,
                0);
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
            const Geometry g = launch_for(L, BC);
            prolong_kernel<BC, T><<<g.grid, g.block, 0, stream>>>(static_cast<const T*>(fine),
                                                                  static_cast<const T*>(coarse), static_cast<T*>(fine),
                                                                  L, C, nullptr, nullptr);
        });
    });
    return launched("mg_prolong_add");
}

// ---- residual norm without any device allocation ----
//
// Some callers cannot allocate device memory at the moment they need a
// residual norm: a solver driven from inside a region where the CUDA
// allocator must not be called (for example while a CUDA graph is being
// captured, where cudaMalloc would break the capture), a host application that
// hands this library only its own fixed buffers (a Fortran/C code with a
// preallocated pool, a real-time loop that forbids allocation after start-up),
// or an embedding that has no PyTorch caching allocator to lend scratch.
// afsi_b200_mg_residual_norm needs caller-provided reduction scratch; this
// variant keeps its per-block partial sums in a file-scope device array
// instead, so the caller passes only the inputs and the output.
//
// The array is sized for kNoAllocBlocks blocks (4096 partial sums plus a
// result and a completion counter, about 32 KB); every GPU that loads the
// library holds it until the process exits.  Grids whose launch needs more
// blocks (2D grids above about 2^20 cells, 3D grids whose y-z section exceeds
// about 2^20 cells) are rejected.  All calls share the one array: calls that overlap on
// the GPU (different streams, no ordering between them) race and must not be
// issued.

namespace {

constexpr int kNoAllocBlocks = 4096;

struct NoAllocScratch {
    double partial[kNoAllocBlocks];
    double result;
    unsigned int counter;
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of g_noalloc_scratch per device (the host-side symbol is only
// a stand-in; the address is looked up once per device, with it current).
std::atomic<NoAllocScratch*> g_noalloc_address[64];

int32_t noalloc_scratch(NoAllocScratch** out) {
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return fail(AFSI_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(err));
    AFSI_REQUIRE(device >= 0 && device < 64, "device index %d out of range", device);
    NoAllocScratch* p = g_noalloc_address[device].load(std::memory_order_acquire);
    if (!p) {
        void* addr = nullptr;
        err = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
        if (err != cudaSuccess)
            return fail(AFSI_ERR_CUDA, "cudaGetSymbolAddress(no-allocation scratch): %s", cudaGetErrorString(err));
        p = static_cast<NoAllocScratch*>(addr);
        g_noalloc_address[device].store(p, std::memory_order_release);
    }
    *out = p;
    return AFSI_OK;
}

}  // namespace

extern "C" int32_t afsi_b200_mg_residual_norm_noalloc(const void* p, const void* rhs, const int64_t* shape,
                                                      const double* h2, int32_t dim, int32_t bc, double* norm_out,
                                                      int32_t dtype, afsi_stream_t stream) {
    int32_t rc = check_bc(dim, bc);
    if (rc || (rc = check_shape(shape, dim))) return rc;
    AFSI_REQUIRE(p && rhs && h2 && norm_out, "null argument");
    AFSI_REQUIRE(dtype == AFSI_F32 || dtype == AFSI_F64, "unsupported dtype code %d", (int)dtype);
    const double one[3] = {1, 1, 1};
    const Geometry probe = launch_for(make_level<double>(shape, h2, one, dim), bc);
    AFSI_REQUIRE(probe.blocks <= kNoAllocBlocks,
                 "grid needs %lld blocks; the no-allocation residual norm serves at most %d "
                 "(use afsi_b200_mg_residual_norm with caller scratch)",
                 (long long)probe.blocks, kNoAllocBlocks);
    NoAllocScratch* scratch = nullptr;
    if ((rc = noalloc_scratch(&scratch))) return rc;
    // the completion counter must start at zero for every call
    cudaError_t err = cudaMemsetAsync(&scratch->counter, 0, sizeof(unsigned int), stream);
    if (err != cudaSuccess) return fail(AFSI_ERR_CUDA, "clearing no-allocation scratch: %s", cudaGetErrorString(err));
    const Site site{scratch->partial, &scratch->counter, &scratch->result};
    AFSI_BC_DISPATCH(bc, {
        AFSI_DISPATCH(dtype, {
            Lv<T> L = make_level<T>(shape, h2, one, dim);
            const Geometry g = launch_for(L, BC);
            residual_norm_kernel<BC, true, T><<<g.grid, g.block, 0, stream>>>(
                static_cast<const T*>(p), static_cast<const T*>(rhs), L, site, norm_out);
        });
    });
    return launched("mg_residual_norm_noalloc");
}

// ---- batched V-cycles (batching form) ----
//
// Many independent channel plans advanced together.  Each level operation of
// Runner (a Jacobi sweep, the residual restriction, the prolongation) runs
// for every instance that has a launched level at that depth in ONE launch,
// and the single-CTA coarse levels of all instances run in one launch with a
// CTA per instance, so a cycle costs 2*smooth+2 launches per launched depth
// plus one, whatever the instance count.  Each instance's sequence of
// operations and every cell's arithmetic are Runner's (the same device
// functions, compiled with --fmad=false), so the iterates are bitwise those
// of afsi_b200_mg_vcycles on each plan alone.  Channel (non-singular) Jacobi
// plans only: there are no gauge sites to batch.
//
// A launch over a depth covers its instances' levels in 32 x 32 cell tiles
// (y fastest, four cells per thread); a block map gives each block its
// instance entry and tile.

namespace afsi {

constexpr int kBatchTileY = 32, kBatchTileX = 32;                // cells per tile (y fastest)
constexpr int kBatchRowStep = kThreads / kBatchTileY;             // x rows apart of a thread's cells
constexpr int kBatchRows = kBatchTileX / kBatchRowStep;           // cells per thread
constexpr int kBatchEntryBits = 11;  // block map word: entry << kBatchLocalBits | tile
constexpr int kBatchLocalBits = 32 - kBatchEntryBits;

template <class T>
struct BatchLevel {
    T w[64];           // omega/diag per boundary class of L (the fast sweep's table)
    Lv<T> L, C;        // the level and its coarser level
    T *p, *q, *r;      // iterate, Jacobi partner, right-hand side
    T* rc;             // coarser right-hand side
    const T* down;     // where the pre-smoothing leaves the iterate (p or q)
    const T* corr;     // the coarser level's final iterate
};

template <class T, class TC>
struct BatchCoarse {
    CoarseLevels<T> cl;
    const T* rhs;      // right-hand side of level cl.first
    const T* p_start;  // initial iterate (level 0) or null (zero start)
    T* p_out;
    const TC* cinv;
};

template <class T>
struct BatchStart {
    const T* src;  // the instance's right-hand side, or null
    T *r, *p;      // its finest rhs (copied into) and iterate (zeroed)
    int nx, ny;
};

// Entry and tile of a block map word.
__device__ __forceinline__ int batch_word(uint32_t w, int& tile) {
    tile = int(w & ((1u << kBatchLocalBits) - 1));
    return int(w >> kBatchLocalBits);
}

// Column y and first row x0 of thread `tid` (of kThreads) in the tile; its
// cells are (x0 + m * kBatchRowStep, y), m < kBatchRows.
__device__ __forceinline__ void batch_tile(int tile, int ny, int tid, int& x0, int& y) {
    const int gy = (ny + kBatchTileY - 1) / kBatchTileY;
    y = (tile % gy) * kBatchTileY + tid % kBatchTileY;
    x0 = (tile / gy) * kBatchTileX + tid / kBatchTileY;
}

// The tile operations below compute all of a thread's cells before storing
// any, so the loads of the cells are in flight together (the outputs never
// alias another cell's inputs).  They are shared by the per-operation
// launches and the persistent kernel.

// One Jacobi sweep of an entry's tile: p -> q (odd == 0) or q -> p (odd == 1);
// zero_in: the iterate is zero (first sweep below the finest level).  The
// arithmetic of sweep_kernel with no pending shifts.
template <int BC, class T>
__device__ __forceinline__ void sweep_tile(const BatchLevel<T>& e, int tile, int tid, int odd, int zero_in) {
    const Lv<T> L = e.L;
    int x0, y;
    batch_tile(tile, L.ny, tid, x0, y);
    if (y >= L.ny) return;
    const T* p = odd ? e.q : e.p;
    T* out = odd ? e.p : e.q;
    const T* rhs = e.r;
    T v[kBatchRows];
#pragma unroll
    for (int m = 0; m < kBatchRows; ++m) {
        const int x = x0 + m * kBatchRowStep;
        if (x >= L.nx) break;
        const int64_t i = index_of(x, y, 0, L);
        const T r = rhs[i];
        const T w = e.w[boundary_class(x, y, 0, L.nx, L.ny, L.nz)];
        if (!zero_in) {
            const T pc = p[i];
            v[m] = jacobi_update(pc, r, neg_lap<BC, false>(p, i, x, y, 0, L, T(0), pc), w);
        } else {
            v[m] = r * w;
        }
    }
#pragma unroll
    for (int m = 0; m < kBatchRows; ++m) {
        const int x = x0 + m * kBatchRowStep;
        if (x >= L.nx) break;
        out[index_of(x, y, 0, L)] = v[m];
    }
}

// rc = restricted residual of the pre-smoothed iterate (residual_restrict_kernel).
template <int BC, class T>
__device__ __forceinline__ void restrict_tile(const BatchLevel<T>& e, int tile, int tid) {
    const Lv<T> C = e.C;
    int cx0, cy;
    batch_tile(tile, C.ny, tid, cx0, cy);
    if (cy >= C.ny) return;
    const Lv<T> L = e.L;
    T v[kBatchRows];
#pragma unroll
    for (int m = 0; m < kBatchRows; ++m) {
        const int cx = cx0 + m * kBatchRowStep;
        if (cx >= C.nx) break;
        v[m] = restrict_residual_at<BC, false>(e.down, e.r, cx, cy, 0, L, T(0));
    }
#pragma unroll
    for (int m = 0; m < kBatchRows; ++m) {
        const int cx = cx0 + m * kBatchRowStep;
        if (cx >= C.nx) break;
        e.rc[index_of(cx, cy, 0, C)] = v[m];
    }
}

// p = down + P(corr) (prolong_kernel; down may be p itself, own cell only).
template <int BC, class T>
__device__ __forceinline__ void prolong_tile(const BatchLevel<T>& e, int tile, int tid) {
    const Lv<T> L = e.L;
    int x0, y;
    batch_tile(tile, L.ny, tid, x0, y);
    if (y >= L.ny) return;
    const Lv<T> C = e.C;
    T v[kBatchRows];
#pragma unroll
    for (int m = 0; m < kBatchRows; ++m) {
        const int x = x0 + m * kBatchRowStep;
        if (x >= L.nx) break;
        v[m] = e.down[index_of(x, y, 0, L)] + prolong_at<BC>(e.corr, x, y, 0, C, T(0));
    }
#pragma unroll
    for (int m = 0; m < kBatchRows; ++m) {
        const int x = x0 + m * kBatchRowStep;
        if (x >= L.nx) break;
        e.p[index_of(x, y, 0, L)] = v[m];
    }
}

// p = q after an odd number of post-sweeps on the finest level (the finalize copy).
template <class T>
__device__ __forceinline__ void finalize_tile(const BatchLevel<T>& e, int tile, int tid) {
    int x0, y;
    batch_tile(tile, e.L.ny, tid, x0, y);
    if (y >= e.L.ny) return;
#pragma unroll
    for (int m = 0; m < kBatchRows; ++m) {
        const int x = x0 + m * kBatchRowStep;
        if (x >= e.L.nx) break;
        const int64_t i = index_of(x, y, 0, e.L);
        e.p[i] = e.q[i];
    }
}

// Cycle start of an instance: finest rhs = its source (when the table has
// one), iterate = 0.
template <class T>
__device__ __forceinline__ void start_tile(const BatchStart<T>& j, int tile, int tid) {
    int x0, y;
    batch_tile(tile, j.ny, tid, x0, y);
    if (y >= j.ny) return;
#pragma unroll
    for (int m = 0; m < kBatchRows; ++m) {
        const int x = x0 + m * kBatchRowStep;
        if (x >= j.nx) break;
        const int64_t i = int64_t(x) * j.ny + y;
        if (j.src) j.r[i] = j.src[i];
        j.p[i] = T(0);
    }
}

template <int BC, class T>
__global__ void __launch_bounds__(kThreads) batch_sweep_kernel(const BatchLevel<T>* __restrict__ lv,
                                                               const uint32_t* __restrict__ map, int odd,
                                                               int zero_in) {
    pdl_enter();
    int tile;
    const int ent = batch_word(map[blockIdx.x], tile);
    sweep_tile<BC>(lv[ent], tile, threadIdx.x, odd, zero_in);
}

template <int BC, class T>
__global__ void __launch_bounds__(kThreads) batch_restrict_kernel(const BatchLevel<T>* __restrict__ lv,
                                                                  const uint32_t* __restrict__ map) {
    pdl_enter();
    int tile;
    const int ent = batch_word(map[blockIdx.x], tile);
    restrict_tile<BC>(lv[ent], tile, threadIdx.x);
}

template <int BC, class T>
__global__ void __launch_bounds__(kThreads) batch_prolong_kernel(const BatchLevel<T>* __restrict__ lv,
                                                                 const uint32_t* __restrict__ map) {
    pdl_enter();
    int tile;
    const int ent = batch_word(map[blockIdx.x], tile);
    prolong_tile<BC>(lv[ent], tile, threadIdx.x);
}

template <class T>
__global__ void __launch_bounds__(kThreads) batch_finalize_kernel(const BatchLevel<T>* __restrict__ lv,
                                                                  const uint32_t* __restrict__ map) {
    pdl_enter();
    int tile;
    const int ent = batch_word(map[blockIdx.x], tile);
    finalize_tile(lv[ent], tile, threadIdx.x);
}

template <class T>
__global__ void __launch_bounds__(kThreads) batch_start_kernel(const BatchStart<T>* __restrict__ jobs,
                                                               const uint32_t* __restrict__ map) {
    pdl_enter();
    int tile;
    const int ent = batch_word(map[blockIdx.x], tile);
    start_tile(jobs[ent], tile, threadIdx.x);
}

// The single-CTA levels of every instance, one CTA each (coarse_cycle).
template <int BC, class T, class TC>
__global__ void __launch_bounds__(kCoarseThreads) batch_coarse_kernel(const BatchCoarse<T, TC>* __restrict__ jobs,
                                                                     int smooth) {
    pdl_enter();
    __shared__ CoarseLevels<T> cl;
    static_assert(sizeof(CoarseLevels<T>) % 4 == 0, "word copy");
    const BatchCoarse<T, TC>& j = jobs[blockIdx.x];
    const unsigned* src = reinterpret_cast<const unsigned*>(&j.cl);
    unsigned* dst = reinterpret_cast<unsigned*>(&cl);
    for (int k = threadIdx.x; k < int(sizeof(cl) / 4); k += blockDim.x) dst[k] = src[k];
    const T* rhs = j.rhs;
    const T* p_start = j.p_start;
    T* p_out = j.p_out;
    const TC* cinv = j.cinv;
    __syncthreads();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    coarse_cycle<BC, T, TC>(reinterpret_cast<T*>(smem_raw), rhs, nullptr, p_start, p_out, cinv, cl, smooth);
}

// ---- persistent batched V-cycles: every level operation of every cycle in
// one cooperative launch, the launches of batch_cycles replaced by grid
// barriers (bounded waits; a timed-out barrier sets the error word and the
// kernel returns).  Each 1024-thread CTA works as four 256-thread virtual
// blocks over the block maps; the coarse jobs go to CTAs in turn.

constexpr int kBatchPThreads = 1024;
constexpr int kBatchVirtual = kBatchPThreads / kThreads;

template <class T, class TC>
struct BatchPersistArgs {
    const unsigned char* table;
    int64_t level_off[AFSI_MG_MAX_LEVELS], map_l_off[AFSI_MG_MAX_LEVELS], map_c_off[AFSI_MG_MAX_LEVELS];
    int64_t blocks_l[AFSI_MG_MAX_LEVELS], blocks_c[AFSI_MG_MAX_LEVELS];
    int64_t start_off, start_map_off, blocks_start, coarse_off;
    int depths, smooth, count, cycles, start;
    GridSync gs;
};

template <int BC, class T, class TC>
__global__ void __launch_bounds__(kBatchPThreads, 1) batch_persistent_kernel(BatchPersistArgs<T, TC> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ CoarseLevels<T> cl;
    const int tid = threadIdx.x % kThreads;
    const int64_t vb0 = int64_t(blockIdx.x) * kBatchVirtual + threadIdx.x / kThreads;
    const int64_t vstride = int64_t(gridDim.x) * kBatchVirtual;
    auto lv = [&](int d) { return reinterpret_cast<const BatchLevel<T>*>(a.table + a.level_off[d]); };
    auto ml = [&](int d) { return reinterpret_cast<const uint32_t*>(a.table + a.map_l_off[d]); };
    auto mc = [&](int d) { return reinterpret_cast<const uint32_t*>(a.table + a.map_c_off[d]); };
    // f(entry, tile) for the blocks of a map, virtual block by virtual block
    auto over = [&](int64_t blocks, const uint32_t* map, auto f) {
        for (int64_t b = vb0; b < blocks; b += vstride) {
            int tile;
            const int ent = batch_word(map[b], tile);
            f(ent, tile);
        }
    };
    bool ok = true;
    if (a.start) {
        const BatchStart<T>* jobs = reinterpret_cast<const BatchStart<T>*>(a.table + a.start_off);
        over(a.blocks_start, reinterpret_cast<const uint32_t*>(a.table + a.start_map_off),
             [&](int ent, int tile) { start_tile(jobs[ent], tile, tid); });
        ok = grid_barrier(a.gs);
    }
    for (int c = 0; c < a.cycles && ok; ++c) {
        for (int d = 0; d < a.depths && ok; ++d) {
            const BatchLevel<T>* L = lv(d);
            for (int s = 0; s < a.smooth && ok; ++s) {
                const int zero = (s == 0 && d > 0) ? 1 : 0;
                over(a.blocks_l[d], ml(d), [&](int ent, int tile) { sweep_tile<BC>(L[ent], tile, tid, s & 1, zero); });
                ok = grid_barrier(a.gs);
            }
            if (!ok) break;
            over(a.blocks_c[d], mc(d), [&](int ent, int tile) { restrict_tile<BC>(L[ent], tile, tid); });
            ok = grid_barrier(a.gs);
        }
        if (!ok) break;
        const BatchCoarse<T, TC>* jobs = reinterpret_cast<const BatchCoarse<T, TC>*>(a.table + a.coarse_off);
        for (int j = blockIdx.x; j < a.count; j += gridDim.x) {
            const unsigned* src = reinterpret_cast<const unsigned*>(&jobs[j].cl);
            unsigned* dst = reinterpret_cast<unsigned*>(&cl);
            for (int k = threadIdx.x; k < int(sizeof(cl) / 4); k += blockDim.x) dst[k] = src[k];
            __syncthreads();
            coarse_cycle<BC, T, TC>(reinterpret_cast<T*>(smem_raw), jobs[j].rhs, nullptr, jobs[j].p_start,
                                    jobs[j].p_out, jobs[j].cinv, cl, a.smooth);
            __syncthreads();
        }
        ok = grid_barrier(a.gs);
        for (int d = a.depths - 1; d >= 0 && ok; --d) {
            const BatchLevel<T>* L = lv(d);
            over(a.blocks_l[d], ml(d), [&](int ent, int tile) { prolong_tile<BC>(L[ent], tile, tid); });
            ok = grid_barrier(a.gs);
            for (int s = 0; s < a.smooth && ok; ++s) {
                over(a.blocks_l[d], ml(d), [&](int ent, int tile) { sweep_tile<BC>(L[ent], tile, tid, s & 1, 0); });
                ok = grid_barrier(a.gs);
            }
        }
        if (ok && a.depths > 0 && a.smooth % 2 == 1) {
            const BatchLevel<T>* L = lv(0);
            over(a.blocks_l[0], ml(0), [&](int ent, int tile) { finalize_tile(L[ent], tile, tid); });
            ok = grid_barrier(a.gs);
        }
    }
}

}  // namespace afsi

namespace {

constexpr int kBatchMaxInstances = 1 << kBatchEntryBits;

int64_t align16(int64_t v) { return (v + 15) & ~int64_t(15); }

// Table layout derived from the plans alone (so the cycles entry recomputes it).
struct BatchLayout {
    int depths = 0;  // launched depths: max over instances of the coarse start
    int64_t entries[AFSI_MG_MAX_LEVELS] = {};
    int64_t blocks_l[AFSI_MG_MAX_LEVELS] = {}, blocks_c[AFSI_MG_MAX_LEVELS] = {};
    int64_t level_off[AFSI_MG_MAX_LEVELS] = {}, map_l_off[AFSI_MG_MAX_LEVELS] = {},
            map_c_off[AFSI_MG_MAX_LEVELS] = {};
    int64_t blocks_start = 0, start_off = 0, start_map_off = 0;
    int64_t coarse_off = 0, bytes = 0;
    size_t coarse_smem = 0;
};

int64_t tiles_of(int nx, int ny) {
    return int64_t((ny + kBatchTileY - 1) / kBatchTileY) * ((nx + kBatchTileX - 1) / kBatchTileX);
}

int32_t validate_batch(const afsi_mg_plan* const* plans, int32_t count) {
    AFSI_REQUIRE(plans && count >= 1 && count <= kBatchMaxInstances, "batch needs 1..%d plans", kBatchMaxInstances);
    const afsi_mg_plan* a = plans[0];
    AFSI_REQUIRE(a, "null plan 0");
    for (int i = 0; i < count; ++i) {
        const afsi_mg_plan* p = plans[i];
        int32_t rc = validate_plan(p);
        if (rc) return rc;
        AFSI_REQUIRE(p->bc == AFSI_BC_CHANNEL && p->smoother == AFSI_MG_JACOBI,
                     "batched V-cycles take channel plans with the Jacobi smoother (plan %d)", i);
        AFSI_REQUIRE(p->smooth == a->smooth && p->dtype == a->dtype && p->coarse_dtype == a->coarse_dtype,
                     "plan %d differs from plan 0 in smooth count or dtypes", i);
        AFSI_REQUIRE(p->coarse_dtype == AFSI_F64 || p->coarse_dtype == p->dtype, "unsupported coarse dtype");
    }
    return AFSI_OK;
}

template <class T>
void load_levels(const afsi_mg_plan* p, Lv<T>* lv) {
    for (int l = 0; l < p->levels; ++l)
        lv[l] = make_level<T>(p->level[l].shape, p->level[l].h2, p->level[l].inv_h2, p->dim);
}

// Layout, and with host != null the table itself.  Entries of a depth are the
// instances (in plan order) with a launched level there; coarse jobs are
// ordered by decreasing shared-memory size so that the largest start first.
template <class T, class TC>
int32_t batch_table(const afsi_mg_plan* const* plans, int count, const void* const* sources, BatchLayout& lay,
                    unsigned char* host) {
    std::vector<int> start(count);
    std::vector<size_t> smem(count);
    lay = BatchLayout();
    for (int i = 0; i < count; ++i) {
        Lv<T> lv[AFSI_MG_MAX_LEVELS];
        load_levels<T>(plans[i], lv);
        start[i] = coarse_start(lv, plans[i]->levels);
        smem[i] = coarse_smem_bytes(lv, start[i], plans[i]->levels);
        lay.depths = std::max(lay.depths, start[i]);
        lay.coarse_smem = std::max(lay.coarse_smem, smem[i]);
        AFSI_REQUIRE(tiles_of(lv[0].nx, lv[0].ny) < (int64_t(1) << kBatchLocalBits), "plan %d: level too large", i);
        for (int d = 0; d < start[i]; ++d) {
            lay.entries[d] += 1;
            lay.blocks_l[d] += tiles_of(lv[d].nx, lv[d].ny);
            lay.blocks_c[d] += tiles_of(lv[d + 1].nx, lv[d + 1].ny);
        }
        lay.blocks_start += tiles_of(lv[0].nx, lv[0].ny);
    }
    AFSI_REQUIRE(lay.blocks_start < (int64_t(1) << 31), "batch too large for one launch");
    int64_t off = 0;
    for (int d = 0; d < lay.depths; ++d) {
        lay.level_off[d] = off;
        off = align16(off + lay.entries[d] * int64_t(sizeof(BatchLevel<T>)));
        lay.map_l_off[d] = off;
        off = align16(off + lay.blocks_l[d] * 4);
        lay.map_c_off[d] = off;
        off = align16(off + lay.blocks_c[d] * 4);
    }
    lay.start_off = off;
    off = align16(off + int64_t(count) * int64_t(sizeof(BatchStart<T>)));
    lay.start_map_off = off;
    off = align16(off + lay.blocks_start * 4);
    lay.coarse_off = off;
    off = align16(off + int64_t(count) * int64_t(sizeof(BatchCoarse<T, TC>)));
    lay.bytes = off;
    if (!host) return AFSI_OK;

    std::memset(host, 0, size_t(lay.bytes));
    auto word = [](int entry, int64_t tile) { return (uint32_t(entry) << kBatchLocalBits) | uint32_t(tile); };
    int64_t fill[AFSI_MG_MAX_LEVELS] = {}, bl[AFSI_MG_MAX_LEVELS] = {}, bc[AFSI_MG_MAX_LEVELS] = {};
    int64_t bs = 0;
    for (int i = 0; i < count; ++i) {
        const afsi_mg_plan* pl = plans[i];
        Lv<T> lv[AFSI_MG_MAX_LEVELS];
        load_levels<T>(pl, lv);
        auto P = [&](int l) { return static_cast<T*>(pl->level[l].p); };
        auto Q = [&](int l) { return static_cast<T*>(pl->level[l].ping); };
        auto R = [&](int l) { return static_cast<T*>(pl->level[l].rhs); };
        // the final iterate of level l: the coarse block writes p; launched
        // levels end on p after an even number of post-sweeps, else on q
        auto final_of = [&](int l) { return (l >= start[i] || pl->smooth % 2 == 0) ? P(l) : Q(l); };
        for (int d = 0; d < start[i]; ++d) {
            const int k = int(fill[d]++);
            BatchLevel<T> e;
            std::memset(&e, 0, sizeof(e));
            e.L = lv[d];
            e.C = lv[d + 1];
            for (int k = 0; k < 64; ++k) e.w[k] = omega_of_class<AFSI_BC_CHANNEL>(k, e.L);
            e.p = P(d);
            e.q = Q(d);
            e.r = R(d);
            e.rc = R(d + 1);
            e.down = pl->smooth % 2 == 0 ? P(d) : Q(d);
            e.corr = final_of(d + 1);
            std::memcpy(host + lay.level_off[d] + int64_t(k) * int64_t(sizeof(e)), &e, sizeof(e));
            uint32_t* ml = reinterpret_cast<uint32_t*>(host + lay.map_l_off[d]);
            for (int64_t t = 0; t < tiles_of(lv[d].nx, lv[d].ny); ++t) ml[bl[d]++] = word(k, t);
            uint32_t* mc = reinterpret_cast<uint32_t*>(host + lay.map_c_off[d]);
            for (int64_t t = 0; t < tiles_of(lv[d + 1].nx, lv[d + 1].ny); ++t) mc[bc[d]++] = word(k, t);
        }
        BatchStart<T> s;
        std::memset(&s, 0, sizeof(s));
        s.src = static_cast<const T*>(sources ? sources[i] : nullptr);
        s.r = R(0);
        s.p = P(0);
        s.nx = lv[0].nx;
        s.ny = lv[0].ny;
        std::memcpy(host + lay.start_off + int64_t(i) * int64_t(sizeof(s)), &s, sizeof(s));
        uint32_t* ms = reinterpret_cast<uint32_t*>(host + lay.start_map_off);
        for (int64_t t = 0; t < tiles_of(lv[0].nx, lv[0].ny); ++t) ms[bs++] = word(i, t);
    }
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return smem[a] > smem[b]; });
    for (int k = 0; k < count; ++k) {
        const int i = order[k];
        const afsi_mg_plan* pl = plans[i];
        BatchCoarse<T, TC> j;
        std::memset(&j, 0, sizeof(j));
        load_levels<T>(pl, j.cl.lv);
        j.cl.first = start[i];
        j.cl.last = pl->levels - 1;
        j.rhs = static_cast<const T*>(pl->level[start[i]].rhs);
        j.p_start = start[i] == 0 ? static_cast<const T*>(pl->level[0].p) : nullptr;
        j.p_out = static_cast<T*>(pl->level[start[i]].p);
        j.cinv = static_cast<const TC*>(pl->coarse_inverse);
        std::memcpy(host + lay.coarse_off + int64_t(k) * int64_t(sizeof(j)), &j, sizeof(j));
    }
    return AFSI_OK;
}

template <class T, class TC>
int32_t batch_cycles(const afsi_mg_plan* const* plans, int count, const unsigned char* table, int cycles, int start,
                     cudaStream_t stream) {
    constexpr int BC = AFSI_BC_CHANNEL;
    BatchLayout lay;
    int32_t rc = batch_table<T, TC>(plans, count, nullptr, lay, nullptr);
    if (rc) return rc;
    static bool configured = false;  // once per instantiation, before any graph capture of it
    if (!configured) {
        cudaFuncSetAttribute(batch_coarse_kernel<BC, T, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             210 * 1024);
        configured = true;
    }
    const int smooth = plans[0]->smooth;
    auto lv = [&](int d) { return reinterpret_cast<const BatchLevel<T>*>(table + lay.level_off[d]); };
    auto ml = [&](int d) { return reinterpret_cast<const uint32_t*>(table + lay.map_l_off[d]); };
    auto mc = [&](int d) { return reinterpret_cast<const uint32_t*>(table + lay.map_c_off[d]); };
    const dim3 block(kThreads);
    if (start) {
        rc = launch_pdl("mg batch start", batch_start_kernel<T>, dim3(unsigned(lay.blocks_start)), block, 0, stream,
                        reinterpret_cast<const BatchStart<T>*>(table + lay.start_off),
                        reinterpret_cast<const uint32_t*>(table + lay.start_map_off));
        if (rc) return rc;
    }
    for (int c = 0; c < cycles; ++c) {
        for (int d = 0; d < lay.depths; ++d) {
            const dim3 gl(unsigned(lay.blocks_l[d])), gc(unsigned(lay.blocks_c[d]));
            for (int s = 0; s < smooth; ++s)
                if ((rc = launch_pdl("mg batch sweep", batch_sweep_kernel<BC, T>, gl, block, 0, stream, lv(d), ml(d),
                                     s & 1, (s == 0 && d > 0) ? 1 : 0)))
                    return rc;
            if ((rc = launch_pdl("mg batch residual_restrict", batch_restrict_kernel<BC, T>, gc, block, 0, stream,
                                 lv(d), mc(d))))
                return rc;
        }
        if ((rc = launch_pdl("mg batch coarse blocks", batch_coarse_kernel<BC, T, TC>, dim3(unsigned(count)),
                             dim3(kCoarseThreads), lay.coarse_smem, stream,
                             reinterpret_cast<const BatchCoarse<T, TC>*>(table + lay.coarse_off), smooth)))
            return rc;
        for (int d = lay.depths - 1; d >= 0; --d) {
            const dim3 gl(unsigned(lay.blocks_l[d]));
            if ((rc = launch_pdl("mg batch prolong_add", batch_prolong_kernel<BC, T>, gl, block, 0, stream, lv(d),
                                 ml(d))))
                return rc;
            for (int s = 0; s < smooth; ++s)
                if ((rc = launch_pdl("mg batch sweep", batch_sweep_kernel<BC, T>, gl, block, 0, stream, lv(d), ml(d),
                                     s & 1, 0)))
                    return rc;
        }
        if (lay.depths > 0 && smooth % 2 == 1 &&
            (rc = launch_pdl("mg batch finalize", batch_finalize_kernel<T>, dim3(unsigned(lay.blocks_l[0])), block, 0,
                             stream, lv(0), ml(0))))
            return rc;
    }
    return AFSI_OK;
}

// The persistent form of batch_cycles: one cooperative launch, one CTA per
// SM; `sync` is afsi_b200_mg_sync_bytes() of zero-initialised barrier words
// (its error word is cleared here).
template <class T, class TC>
int32_t batch_persistent(const afsi_mg_plan* const* plans, int count, const unsigned char* table, int cycles,
                         int start, void* sync, cudaStream_t stream) {
    constexpr int BC = AFSI_BC_CHANNEL;
    BatchLayout lay;
    int32_t rc = batch_table<T, TC>(plans, count, nullptr, lay, nullptr);
    if (rc) return rc;
    BatchPersistArgs<T, TC> a;
    a.table = table;
    for (int d = 0; d < AFSI_MG_MAX_LEVELS; ++d) {
        a.level_off[d] = lay.level_off[d];
        a.map_l_off[d] = lay.map_l_off[d];
        a.map_c_off[d] = lay.map_c_off[d];
        a.blocks_l[d] = lay.blocks_l[d];
        a.blocks_c[d] = lay.blocks_c[d];
    }
    a.start_off = lay.start_off;
    a.start_map_off = lay.start_map_off;
    a.blocks_start = lay.blocks_start;
    a.coarse_off = lay.coarse_off;
    a.depths = lay.depths;
    a.smooth = plans[0]->smooth;
    a.count = count;
    a.cycles = cycles;
    a.start = start;
    unsigned char* b = static_cast<unsigned char*>(sync);
    a.gs.count = reinterpret_cast<unsigned int*>(b);
    a.gs.gen = reinterpret_cast<unsigned int*>(b + 4);
    a.gs.error = reinterpret_cast<int*>(b + 8);
    a.gs.slot = reinterpret_cast<double*>(b + 64);
    a.gs.partial = reinterpret_cast<double*>(b + 64 + 8 * (AFSI_MG_MAX_LEVELS * 3 + 8));
    auto kernel = batch_persistent_kernel<BC, T, TC>;
    static int per_sm = -1;  // once per instantiation, before any graph capture of it
    if (per_sm < 0) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBatchPThreads, 200 * 1024);
    }
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    AFSI_REQUIRE(per_sm >= 1 && sms >= 1 && sms <= 4096, "persistent batched V-cycles do not fit on this device");
    // counter, generation and error word start from zero (a run whose barrier
    // timed out may have left the counter part-way)
    if (cudaMemsetAsync(sync, 0, 12, stream) != cudaSuccess)
        return fail(AFSI_ERR_CUDA, "clearing the barrier words failed");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(sms);
    cfg.blockDim = dim3(kBatchPThreads);
    cfg.dynamicSmemBytes = lay.coarse_smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeCooperative;
    attr.val.cooperative = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    const cudaError_t err = cudaLaunchKernelEx(&cfg, kernel, a);
    if (err != cudaSuccess) return fail(AFSI_ERR_CUDA, "persistent batched V-cycles: %s", cudaGetErrorString(err));
    return launched("mg batch persistent");
}

#define AFSI_BATCH_DISPATCH(plans, ...)      \
    AFSI_DISPATCH((plans)[0]->dtype, {        \
        if ((plans)[0]->coarse_dtype == AFSI_F64) { \
            using TC = double;                \
            __VA_ARGS__;                      \
        } else {                              \
            using TC = T;                     \
            __VA_ARGS__;                      \
        }                                     \
    })

}  // namespace

extern "C" int64_t afsi_b200_mg_batch_table_bytes(const afsi_mg_plan* const* plans, int32_t count) {
    if (validate_batch(plans, count)) return -1;
    BatchLayout lay;
    int32_t rc = AFSI_OK;
    AFSI_BATCH_DISPATCH(plans, rc = batch_table<T, TC>(plans, count, nullptr, lay, nullptr));
    return rc ? -1 : lay.bytes;
}

extern "C" int32_t afsi_b200_mg_batch_table(const afsi_mg_plan* const* plans, int32_t count,
                                            const void* const* rhs_sources, void* host_table, int64_t bytes) {
    int32_t rc = validate_batch(plans, count);
    if (rc) return rc;
    AFSI_REQUIRE(host_table, "null table");
    if (rhs_sources)
        for (int i = 0; i < count; ++i) AFSI_REQUIRE(rhs_sources[i], "null rhs source %d", i);
    BatchLayout lay;
    AFSI_BATCH_DISPATCH(plans, {
        if ((rc = batch_table<T, TC>(plans, count, nullptr, lay, nullptr))) return rc;
        AFSI_REQUIRE(bytes >= lay.bytes, "table needs %lld bytes", (long long)lay.bytes);
        return batch_table<T, TC>(plans, count, rhs_sources, lay, static_cast<unsigned char*>(host_table));
    });
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_mg_batch_vcycles(const afsi_mg_plan* const* plans, int32_t count, const void* table,
                                              int32_t cycles, int32_t start, afsi_stream_t stream) {
    int32_t rc = validate_batch(plans, count);
    if (rc) return rc;
    AFSI_REQUIRE(table && reinterpret_cast<uintptr_t>(table) % 16 == 0, "device table must be 16-byte aligned");
    AFSI_REQUIRE(cycles >= 0, "negative cycle count");
    AFSI_BATCH_DISPATCH(plans, {
        return batch_cycles<T, TC>(plans, count, static_cast<const unsigned char*>(table), cycles, start ? 1 : 0,
                                   static_cast<cudaStream_t>(stream));
    });
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_mg_batch_persistent(const afsi_mg_plan* const* plans, int32_t count, const void* table,
                                                 int32_t cycles, int32_t start, void* sync_scratch,
                                                 afsi_stream_t stream) {
    int32_t rc = validate_batch(plans, count);
    if (rc) return rc;
    AFSI_REQUIRE(table && reinterpret_cast<uintptr_t>(table) % 16 == 0, "device table must be 16-byte aligned");
    AFSI_REQUIRE(sync_scratch, "null barrier scratch");
    AFSI_REQUIRE(cycles >= 0, "negative cycle count");
    AFSI_BATCH_DISPATCH(plans, {
        return batch_persistent<T, TC>(plans, count, static_cast<const unsigned char*>(table), cycles, start ? 1 : 0,
                                       sync_scratch, static_cast<cudaStream_t>(stream));
    });
    return AFSI_OK;
}
