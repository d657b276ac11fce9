// The coarse part of a 3D V-cycle in one thread-block cluster.
//
// The single-CTA coarse block (mg_ops.cuh) puts every level below ~4096
// cells on one SM.  Here a cluster of C CTAs (C = 8 or 16, 1024 threads
// each) takes the levels from `first` down:
//  * "distributed" levels (extent nx a multiple of C, at least C) are cut into
//    x-slabs of ppc = nx/C planes, one per CTA, at the same shared-memory
//    offset in every CTA; a cell on a slab face reads its x-neighbour in the
//    next CTA's shared memory through the cluster's distributed shared memory
//    (mapa / ld.shared::cluster), and each phase ends with a cluster barrier;
//  * "replicated" levels (nx < C) are held and computed in full by every CTA,
//    with the single-CTA routines of mg_ops.cuh and no communication; the
//    transition into them reads the distributed fine level across the
//    cluster, and every CTA computes the same values in the same order.
// Means of the singular (Neumann) problem are summed per CTA, published in a
// shared slot and added over the ranks in rank order by every CTA: the same
// total everywhere, deterministic.  The arithmetic is the coarse block's
// (fast mode: branch-free stencil, omega/diag tables, pending gauge shifts).
// Every CTA executes every cluster barrier (uniform control flow), and the
// last barrier precedes the exit so no CTA leaves while another may still
// read its shared memory.
#pragma once
#include <cooperative_groups.h>
#include "mg_ops.cuh"

namespace afsi {

namespace cg = cooperative_groups;

constexpr int kClusterMax = 16;

template <class T>
struct ClusterLevel {
    Lv<T> L;    // the whole level
    int ppc;    // planes per CTA; 0 = replicated
    int cells;  // cells held by each CTA
    int off;    // P at arena + off, Q at + cells, R at + 2*cells
};

template <class T>
struct ClusterLevels {
    ClusterLevel<T> lv[AFSI_MG_MAX_LEVELS];
    int first, last, tables;  // tables: offset of the omega/diag tables (64 per level)
};

template <class T>
struct Slab {
    const T* prev;  // the same array in the CTA holding the previous slab (nullptr at x = 0)
    const T* next;  // ... the next slab (nullptr at the last)
};

template <class T>
__device__ __forceinline__ Slab<T> slab_of(const T* local, int rank, int ranks) {
    Slab<T> s;
    s.prev = rank > 0 ? static_cast<const T*>(__cluster_map_shared_rank(const_cast<T*>(local), rank - 1)) : nullptr;
    s.next = rank + 1 < ranks ? static_cast<const T*>(__cluster_map_shared_rank(const_cast<T*>(local), rank + 1))
                              : nullptr;
    return s;
}

// Cluster-wide sum, identical in every CTA: the CTA sums are added in rank
// order.  One block barrier, one cluster barrier, then warp 0 reads the
// ranks' sums (lane r from rank r, one distributed-shared-memory round trip
// per CTA instead of one per thread and rank) and publishes the total.
// slot: two doubles per CTA (alternating), bcast: two doubles (alternating),
// red: block scratch.
__device__ __forceinline__ double cluster_sum(double v, double* slot, double* bcast, int& parity, double (*red)[32],
                                              int& rt, int ranks) {
    const double mine = block_sum_all(v, red[rt]);
    rt ^= 1;
    if (threadIdx.x == 0) slot[parity] = mine;
    cg::this_cluster().sync();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        const double x =
            lane < ranks ? static_cast<const double*>(__cluster_map_shared_rank(slot, lane))[parity] : 0.0;
        double total = 0.0;
        for (int r = 0; r < ranks; ++r) total += __shfl_sync(0xffffffffu, x, r);
        if (lane == 0) bcast[parity] = total;
    }
    __syncthreads();
    const double total = bcast[parity];
    parity ^= 1;
    return total;
}

// Ghost of a missing wall neighbour: the cell itself (closed box) or its
// negative (open box, zero pressure half a cell outside).
template <int BC, class T>
__device__ __forceinline__ T wall_ghost(T pc) {
    return BC == AFSI_BC_DIRICHLET ? -pc : pc;
}

// (A p)_i for local cell i = (xl, y, z) of a distributed slab.
template <int BC, class T>
__device__ __forceinline__ T dist_apply(const T* __restrict__ p, const Slab<T>& s, int i, int xl, int y, int z, int ppc,
                                        const Lv<T>& L, T pc) {
    const int sy = L.nz, sx = L.ny * L.nz;
    const T g = wall_ghost<BC>(pc);
    const T xm = xl > 0 ? p[i - sx] : (s.prev ? s.prev[i + (ppc - 1) * sx] : g);
    const T xp = xl + 1 < ppc ? p[i + sx] : (s.next ? s.next[i - (ppc - 1) * sx] : g);
    const T ym = y > 0 ? p[i - sy] : g, yp = y + 1 < L.ny ? p[i + sy] : g;
    const T zm = z > 0 ? p[i - 1] : g, zp = z + 1 < L.nz ? p[i + 1] : g;
    return __fma_rn((pc - xm) + (pc - xp), L.ih2[0],
                    __fma_rn((pc - ym) + (pc - yp), L.ih2[1], ((pc - zm) + (pc - zp)) * L.ih2[2]));
}

// Local coordinates of cell i of a slab (ppc x ny x nz, z fastest).
template <class T>
__device__ __forceinline__ void slab_coords(int i, const Lv<T>& L, int& xl, int& y, int& z) {
    z = i % L.nz;
    const int r = i / L.nz;
    y = r % L.ny;
    xl = r / L.ny;
}

// `smooth` Jacobi sweeps of a distributed level; returns the final buffer and
// the pending mean (singular BCs) of the level's iterate over the cluster.
template <int BC, class T>
__device__ T* dist_smooth(T* cur, T* oth, T* R, const ClusterLevel<T>& lv, const T* wrd, int smooth, bool zero,
                          T rhs_shift, int rank, int ranks, double* slot, double* bcast, int& parity, double (*red)[32],
                          int& rt, T* mean) {
    constexpr bool singular = singular_bc(BC);
    const Lv<T>& L = lv.L;
    const int x0 = rank * lv.ppc;
    for (int s = 0; s < smooth; ++s) {
        const bool last = s == smooth - 1;
        const bool z0 = s == 0 && zero;
        const Slab<T> h = slab_of<T>(cur, rank, ranks);
        double acc = 0.0;
        for (int i = threadIdx.x; i < lv.cells; i += blockDim.x) {
            int xl, y, z;
            slab_coords(i, L, xl, y, z);
            const T w = wrd[boundary_class(x0 + xl, y, z, L.nx, L.ny, L.nz)];
            T v;
            if (z0) {
                const T r = R[i] - rhs_shift;
                if (rhs_shift != T(0)) R[i] = r;
                v = r * w;
            } else {
                const T pc = cur[i];
                v = __fma_rn(R[i] - dist_apply<BC>(cur, h, i, xl, y, z, lv.ppc, L, pc), w, pc);
            }
            oth[i] = v;
            if (last) acc += double(v);
        }
        if (last && singular) {
            *mean = T(cluster_sum(acc, slot, bcast, parity, red, rt, ranks) / double(L.n));
        } else {
            cg::this_cluster().sync();
        }
        T* t = cur;
        cur = oth;
        oth = t;
    }
    if (!singular) *mean = T(0);
    return cur;
}

// omega/diag tables of levels first..last (cluster_cycle's arena): no input
// of the predecessor kernel is read, so the kernel builds them before its
// programmatic-dependent-launch wait.
template <int BC, class T>
__device__ void cluster_tables(T* arena, const ClusterLevels<T>& cl) {
    for (int l = cl.first; l <= cl.last; ++l) omega_table<BC>(cl.lv[l].L, arena + cl.tables + 64 * (l - cl.first));
}

// Levels first..last of one V-cycle in a cluster (3D BCs).  As coarse_cycle:
// rhs of level `first` from global memory (shifted by rhs_sum/n), p from
// p_global (first == 0) or zero; the final p of level `first`, mean removed
// for the singular operator, written to p_out.  Level `first` is distributed.
template <int BC, class T, class TC>
__device__ void cluster_cycle(T* arena, const T* __restrict__ rhs_global, const double* rhs_sum, const T* p_global,
                              T* p_out, const TC* __restrict__ cinv, const ClusterLevels<T>& cl, int smooth) {
    __shared__ double red[2][32];
    __shared__ double slot[2], bcast[2];
    __shared__ T down_mean[AFSI_MG_MAX_LEVELS];
    constexpr bool singular = singular_bc(BC);
    int rt = 0, parity = 0;
    const int rank = int(cg::this_cluster().block_rank());
    const int ranks = int(cg::this_cluster().num_blocks());
    const int f = cl.first, last = cl.last;
    auto P_of = [&](int l) { return arena + cl.lv[l].off; };
    T* tables = arena + cl.tables;  // filled by cluster_tables before the kernel waits on its predecessor
    {
        const ClusterLevel<T>& lv = cl.lv[f];
        const T mr = T(site_mean(rhs_sum, lv.L.n));
        T* P = P_of(f);
        T* R = P + 2 * lv.cells;
        const int64_t g0 = int64_t(rank) * lv.cells;
        for (int i = threadIdx.x; i < lv.cells; i += blockDim.x) {
            R[i] = rhs_global[g0 + i] - mr;
            if (p_global) P[i] = p_global[g0 + i];
        }
    }
    cg::this_cluster().sync();
    // down
    T rhs_shift = T(0);
    for (int l = f; l < last; ++l) {
        const ClusterLevel<T>& F = cl.lv[l];
        const ClusterLevel<T>& C = cl.lv[l + 1];
        T* P = P_of(l);
        T* R = P + 2 * F.cells;
        T* Rc = P_of(l + 1) + 2 * C.cells;
        const T* wrd = tables + 64 * (l - f);
        T m;
        const T* cur;
        if (F.ppc) {
            cur = dist_smooth<BC>(P, P + F.cells, R, F, wrd, smooth, l > f || !p_global, rhs_shift, rank, ranks, slot,
                                  bcast, parity, red, rt, &m);
        } else {
            FastCoords<T> fcF;
            fcF.init(F.L);
            cur = block_smooth<BC>(P, P + F.cells, R, F.L, fcF, wrd, smooth, true, rhs_shift, red, rt, &m);
        }
        if (threadIdx.x == 0) down_mean[l] = m;
        double acc = 0.0;
        FastCoords<T> fcC;
        fcC.init(C.L);
        if (F.ppc && C.ppc) {
            // both distributed: the coarse slab's fine planes are local
            const Slab<T> h = slab_of<T>(cur, rank, ranks);
            for (int c = threadIdx.x; c < C.cells; c += blockDim.x) {
                int cxl, cy, cz;
                slab_coords(c, C.L, cxl, cy, cz);
                T v = T(0);
#pragma unroll
                for (int a = 0; a < 2; ++a)
#pragma unroll
                    for (int b = 0; b < 2; ++b)
#pragma unroll
                        for (int d = 0; d < 2; ++d) {
                            const int xl = 2 * cxl + a, y = 2 * cy + b, z = 2 * cz + d;
                            const int i = (xl * F.L.ny + y) * F.L.nz + z;
                            v = v + (R[i] - dist_apply<BC>(cur, h, i, xl, y, z, F.ppc, F.L, cur[i]));
                        }
                v = v * T(.125);
                Rc[c] = v;
                acc += double(v);
            }
            if (singular) {
                rhs_shift = T(cluster_sum(acc, slot, bcast, parity, red, rt, ranks) / double(C.L.n));
            } else {
                cg::this_cluster().sync();
            }
        } else if (F.ppc) {
            // distributed -> replicated.  Each CTA sums, per coarse cell, the
            // residuals of the four children in each of its own fine planes
            // (partials in the buffer the smoothing left free); after a cluster
            // barrier every CTA adds the two partials of each coarse cell.
            T* part = cur == P ? P + F.cells : P;
            const Slab<T> h = slab_of<T>(cur, rank, ranks);
            const int nzc = C.L.nz, plane = C.L.ny * nzc;
            for (int j = threadIdx.x; j < F.ppc * plane; j += blockDim.x) {
                const int xl = j / plane, rem = j - xl * plane, cy = rem / nzc, cz = rem - cy * nzc;
                T v = T(0);
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int d = 0; d < 2; ++d) {
                        const int y = 2 * cy + b, z = 2 * cz + d;
                        const int i = (xl * F.L.ny + y) * F.L.nz + z;
                        v = v + (R[i] - dist_apply<BC>(cur, h, i, xl, y, z, F.ppc, F.L, cur[i]));
                    }
                part[j] = v;
            }
            cg::this_cluster().sync();
            for (int c = threadIdx.x; c < C.cells; c += blockDim.x) {
                int cx, cy, cz;
                fcC.get(c, C.L, cx, cy, cz);
                const int rem = cy * nzc + cz;
                T v = T(0);
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const int x = 2 * cx + a, owner = x / F.ppc;
                    const T* pr = static_cast<const T*>(__cluster_map_shared_rank(part, owner));
                    v = v + pr[(x - owner * F.ppc) * plane + rem];
                }
                v = v * T(.125);
                Rc[c] = v;
                acc += double(v);
            }
            if (singular) {
                rhs_shift = T(block_sum_all(acc, red[rt]) / double(C.L.n));
                rt ^= 1;
            }
            // every CTA has read the partials before any CTA writes the fine
            // level again (prolongation on the way up)
            cg::this_cluster().sync();
        } else {
            for (int c = threadIdx.x; c < C.cells; c += blockDim.x) {
                int cx, cy, cz;
                fcC.get(c, C.L, cx, cy, cz);
                const T v = block_restrict<BC>(cur, R, cx, cy, cz, F.L);
                Rc[c] = v;
                acc += double(v);
            }
            if (singular) {
                rhs_shift = T(block_sum_all(acc, red[rt]) / double(C.L.n));
                rt ^= 1;
            } else {
                __syncthreads();
            }
        }
    }
    // dense coarsest solve, replicated in every CTA (mac/mg_workspace.py:86-90)
    T coarse_shift;
    {
        const ClusterLevel<T>& lv = cl.lv[last];
        T* P = P_of(last);
        const T* R = P + 2 * lv.cells;
        const int n = lv.cells;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
        double acc = 0.0;
        for (int r = warp; r < n; r += warps) {
            double s = 0.0;
            for (int j = lane; j < n; j += 32) s += double(cinv[int64_t(r) * n + j]) * double(R[j] - rhs_shift);
            s = warp_sum(s);
            const T v = T(s);
            if (lane == 0) {
                P[r] = v;
                acc += double(v);
            }
        }
        if (singular) {
            coarse_shift = T(block_sum_all(acc, red[rt]) / double(n));
            rt ^= 1;
        } else {
            coarse_shift = T(0);
            __syncthreads();
        }
    }
    // up
    const T* corr = P_of(last);
    bool corr_distributed = false;
    for (int l = last - 1; l >= f; --l) {
        const ClusterLevel<T>& F = cl.lv[l];
        const ClusterLevel<T>& C = cl.lv[l + 1];
        T* P = P_of(l);
        T* Q = P + F.cells;
        T* R = Q + F.cells;
        T* down = (smooth & 1) ? Q : P;
        const T dm = down_mean[l];
        const T* wrd = tables + 64 * (l - f);
        T m;
        if (F.ppc) {
            const int x0 = rank * F.ppc;
            // coarse planes next to this CTA's coarse slab, copied from the
            // neighbouring CTAs into the coarse level's free buffers (its rhs
            // and its other Jacobi buffer), so the prolongation reads locally
            const int nzc = C.L.nz, plane = C.L.ny * nzc;
            const int xc0 = rank * C.ppc;
            T* ghost_prev = P_of(l + 1) + 2 * C.cells;
            T* ghost_next = corr == P_of(l + 1) ? P_of(l + 1) + C.cells : P_of(l + 1);
            if (corr_distributed) {
                const Slab<T> hc = slab_of<T>(corr, rank, ranks);
                for (int j = threadIdx.x; j < plane; j += blockDim.x) {
                    ghost_prev[j] = hc.prev ? hc.prev[(C.ppc - 1) * plane + j] : T(0);
                    ghost_next[j] = hc.next ? hc.next[j] : T(0);
                }
                __syncthreads();
            }
            auto coarse = [&](int cx, int cy, int cz) {
                const int r = cy * nzc + cz;
                return cx < xc0 ? ghost_prev[r] : cx >= xc0 + C.ppc ? ghost_next[r] : corr[(cx - xc0) * plane + r];
            };
            for (int i = threadIdx.x; i < F.cells; i += blockDim.x) {
                int xl, y, z;
                slab_coords(i, F.L, xl, y, z);
                T add;
                if (corr_distributed) {
                    // coarse values by global coordinates (the clamped and ghost rules of prolong_at)
                    const int x = x0 + xl;
                    const int ax = x / 2 - 1 + (x & 1), ay = y / 2 - 1 + (y & 1), az = z / 2 - 1 + (z & 1);
                    const T wx = (x & 1) ? T(.25) : T(.75), wy = (y & 1) ? T(.25) : T(.75),
                            wz = (z & 1) ? T(.25) : T(.75);
                    const Lv<T>& Cl = C.L;
                    const int cx0 = ax < 0 ? 0 : ax, cx1 = ax + 1 < Cl.nx - 1 ? ax + 1 : Cl.nx - 1;
                    const int cy0 = ay < 0 ? 0 : ay, cy1 = ay + 1 < Cl.ny - 1 ? ay + 1 : Cl.ny - 1;
                    const int cz0 = az < 0 ? 0 : az, cz1 = az + 1 < Cl.nz - 1 ? az + 1 : Cl.nz - 1;
                    const bool odd = BC == AFSI_BC_DIRICHLET;
                    const bool gx0 = odd && ax < 0, gx1 = odd && ax + 1 > Cl.nx - 1, gy0 = odd && ay < 0,
                               gy1 = odd && ay + 1 > Cl.ny - 1, gz0 = odd && az < 0, gz1 = odd && az + 1 > Cl.nz - 1;
                    auto at = [&](int i2, int j2, int k2, bool fi, bool fj, bool fk) {
                        const T v = coarse(i2, j2, k2) - coarse_shift;
                        return (fi != fj) != fk ? -v : v;
                    };
                    const T c00 = at(cx0, cy0, cz0, gx0, gy0, gz0) * (T(1) - wz) + at(cx0, cy0, cz1, gx0, gy0, gz1) * wz;
                    const T c01 = at(cx0, cy1, cz0, gx0, gy1, gz0) * (T(1) - wz) + at(cx0, cy1, cz1, gx0, gy1, gz1) * wz;
                    const T c10 = at(cx1, cy0, cz0, gx1, gy0, gz0) * (T(1) - wz) + at(cx1, cy0, cz1, gx1, gy0, gz1) * wz;
                    const T c11 = at(cx1, cy1, cz0, gx1, gy1, gz0) * (T(1) - wz) + at(cx1, cy1, cz1, gx1, gy1, gz1) * wz;
                    add = (c00 * (T(1) - wy) + c01 * wy) * (T(1) - wx) + (c10 * (T(1) - wy) + c11 * wy) * wx;
                } else {
                    add = prolong_at<BC>(corr, x0 + xl, y, z, C.L, coarse_shift);
                }
                P[i] = (down[i] - dm) + add;
            }
            cg::this_cluster().sync();
            corr = dist_smooth<BC>(P, Q, R, F, wrd, smooth, false, T(0), rank, ranks, slot, bcast, parity, red, rt,
                                   &m);
            corr_distributed = true;
        } else {
            FastCoords<T> fcL;
            fcL.init(F.L);
            for (int i = threadIdx.x; i < F.cells; i += blockDim.x) {
                int x, y, z;
                fcL.get(i, F.L, x, y, z);
                P[i] = (down[i] - dm) + prolong_at<BC>(corr, x, y, z, C.L, coarse_shift);
            }
            __syncthreads();
            corr = block_smooth<BC>(P, Q, R, F.L, fcL, wrd, smooth, false, T(0), red, rt, &m);
        }
        coarse_shift = m;
    }
    {
        const ClusterLevel<T>& lv = cl.lv[f];
        const int64_t g0 = int64_t(rank) * lv.cells;
        for (int i = threadIdx.x; i < lv.cells; i += blockDim.x) p_out[g0 + i] = corr[i] - coarse_shift;
    }
    cg::this_cluster().sync();  // no CTA leaves while another may read its shared memory
}

}  // namespace afsi
