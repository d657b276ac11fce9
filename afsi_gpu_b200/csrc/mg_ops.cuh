// Device operators of the MAC multigrid shared by the per-level kernels
// (mg.cu) and the persistent V-cycle (mg_persistent.cu).  See mg.cu for the
// operators, arithmetic modes and launch geometry.
#pragma once
#include "common.cuh"

namespace afsi {


constexpr int kThreads = 256;
constexpr int kCoarseThreads = 1024;
constexpr int64_t kCoarseCells = 4096;  // levels at or below this size run in one CTA

template <class T>
struct Lv {
    int nx, ny, nz;  // cells per axis; nz == 1 in 2D (index x*ny + y)
    int64_t n;
    T h2[3], ih2[3];
};

// One reduction site: per-block partials, completion counter, result.
struct Site {
    double* partial;
    unsigned int* counter;
    double* result;
};

template <int BC, class T>
__device__ __forceinline__ T diag_at(int x, int y, int z, const Lv<T>& L) {
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

template <bool Exact, class T>
__device__ __forceinline__ T scale(T diff, const Lv<T>& L, int a) {
    return Exact ? diff / L.h2[a] : diff * L.ih2[a];
}

// (A p)_i with every load shifted by m (pc = p_i - m already loaded).
template <int BC, bool Exact, class T>
__device__ __forceinline__ T neg_lap(const T* __restrict__ p, int64_t i, int x, int y, int z, const Lv<T>& L, T m,
                                     T pc) {
    T a = T(0);
    if (BC == AFSI_BC_NEUMANN) {
        const int64_t sx = int64_t(L.ny) * L.nz, sy = L.nz;
        if (x + 1 < L.nx) a = a - scale<Exact>((p[i + sx] - m) - pc, L, 0);
        if (x > 0) a = a + scale<Exact>(pc - (p[i - sx] - m), L, 0);
        if (y + 1 < L.ny) a = a - scale<Exact>((p[i + sy] - m) - pc, L, 1);
        if (y > 0) a = a + scale<Exact>(pc - (p[i - sy] - m), L, 1);
        if (z + 1 < L.nz) a = a - scale<Exact>((p[i + 1] - m) - pc, L, 2);
        if (z > 0) a = a + scale<Exact>(pc - (p[i - 1] - m), L, 2);
    } else {
        const int64_t sx = L.ny;
        if (BC == AFSI_BC_CHANNEL) {
            if (x + 1 < L.nx) a = a - scale<Exact>((p[i + sx] - m) - pc, L, 0);
            if (x > 0) a = a + scale<Exact>(pc - (p[i - sx] - m), L, 0);
        } else {
            const int64_t right = x + 1 < L.nx ? i + sx : i - int64_t(L.nx - 1) * sx;
            const int64_t left = x > 0 ? i - sx : i + int64_t(L.nx - 1) * sx;
            a = a - scale<Exact>((p[right] - m) - pc, L, 0);
            a = a + scale<Exact>(pc - (p[left] - m), L, 0);
        }
        if (y + 1 < L.ny) a = a - scale<Exact>((p[i + 1] - m) - pc, L, 1);
        if (y > 0) a = a + scale<Exact>(pc - (p[i - 1] - m), L, 1);
        if (BC == AFSI_BC_CHANNEL && x == L.nx - 1) a = a + scale<Exact>(T(2) * pc, L, 0);
    }
    return a;
}

template <class T>
__device__ __forceinline__ int64_t index_of(int x, int y, int z, const Lv<T>& L) {
    return (int64_t(x) * L.ny + y) * L.nz + z;
}

// Cell of this thread in the 3D launch geometry (see launch_for); false if
// the thread is padding.
template <int BC, class T>
__device__ __forceinline__ bool my_cell(const Lv<T>& L, int& x, int& y, int& z) {
    const int fast = blockIdx.x * blockDim.x + threadIdx.x;
    const int mid = blockIdx.y * blockDim.y + threadIdx.y;
    if (BC == AFSI_BC_NEUMANN) {
        z = fast;
        y = mid;
        x = blockIdx.z;
        return z < L.nz && y < L.ny;
    }
    y = fast;
    x = mid;
    z = 0;
    return y < L.ny && x < L.nx;
}

// Coordinates of flat index i (single-block code only; 32-bit division).
template <class T>
__device__ __forceinline__ void coords32(int i, const Lv<T>& L, int& x, int& y, int& z) {
    z = i % L.nz;
    const int r = i / L.nz;
    y = r % L.ny;
    x = r / L.ny;
}

template <class T>
__device__ __forceinline__ T omega() { return T(2.0 / 3.0); }

__device__ __forceinline__ double site_mean(const double* result, int64_t n) {
    return result ? *result / double(n) : 0.0;
}

__device__ __forceinline__ unsigned block_linear() {
    return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
}

__device__ __forceinline__ unsigned thread_linear() { return threadIdx.x + blockDim.x * threadIdx.y; }

// Block-wide sum for 2D blocks (result valid in linear thread 0).
__device__ __forceinline__ double block_sum2(double v, double* shared) {
    const unsigned t = thread_linear();
    const unsigned lane = t & 31, warp = t >> 5;
    v = warp_sum(v);
    if (lane == 0) shared[warp] = v;
    __syncthreads();
    const unsigned warps = (blockDim.x * blockDim.y + 31) >> 5;
    v = t < warps ? shared[t] : 0.0;
    if (warp == 0) v = warp_sum(v);
    __syncthreads();
    return v;
}

// Block partial + last-block completion for a grid reduction of `v`.
__device__ __forceinline__ void site_finish(const Site& s, double v, double* sqrt_out = nullptr) {
    __shared__ double warp_sums[32];
    __shared__ bool last;
    v = block_sum2(v, warp_sums);
    const unsigned t = thread_linear();
    const unsigned blocks = gridDim.x * gridDim.y * gridDim.z;
    if (t == 0) s.partial[block_linear()] = v;
    __threadfence();
    __syncthreads();
    if (t == 0) last = atomicAdd(s.counter, 1u) == blocks - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc = 0.0;
    const unsigned threads = blockDim.x * blockDim.y;
    for (unsigned i = t; i < blocks; i += threads) acc += __ldcg(s.partial + i);
    acc = block_sum2(acc, warp_sums);
    if (t == 0) {
        if (sqrt_out) *sqrt_out = sqrt(acc);
        else *s.result = acc;
        *s.counter = 0u;
    }
}

template <int BC, bool Exact, class T>
__device__ __forceinline__ T restrict_residual_at(const T* __restrict__ p, const T* __restrict__ rhs, int cx, int cy,
                                                  int cz, const Lv<T>& L, T m) {
    if (BC == AFSI_BC_NEUMANN) {
        T v = T(0);
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int d = 0; d < 2; ++d) {
                    const int x = 2 * cx + a, y = 2 * cy + b, z = 2 * cz + d;
                    const int64_t i = index_of(x, y, z, L);
                    const T pc = p[i] - m;
                    v = v + (rhs[i] - neg_lap<BC, Exact>(p, i, x, y, z, L, m, pc));
                }
        return v * T(.125);
    }
    T r[4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int x = 2 * cx + a, y = 2 * cy + b;
            const int64_t i = int64_t(x) * L.ny + y;
            const T pc = p[i] - m;
            r[a * 2 + b] = rhs[i] - neg_lap<BC, Exact>(p, i, x, y, 0, L, m, pc);
        }
    return ((r[0] + r[1]) + r[2] + r[3]) * T(.25);
}

// Coarse value with the boundary ghosts of each BC (coarse lattice C).
template <int BC, class T>
__device__ __forceinline__ T coarse_at(const T* __restrict__ c, int x, int y, const Lv<T>& C, T m) {
    T sign = T(1);
    if (BC == AFSI_BC_CHANNEL) {
        if (x >= C.nx) sign = T(-1);
        x = x < 0 ? 0 : (x > C.nx - 1 ? C.nx - 1 : x);
    } else {
        x = x < 0 ? x + C.nx : (x >= C.nx ? x - C.nx : x);
    }
    y = y < 0 ? 0 : (y > C.ny - 1 ? C.ny - 1 : y);
    return sign * (c[int64_t(x) * C.ny + y] - m);
}

template <int BC, class T>
__device__ __forceinline__ T prolong_at(const T* __restrict__ c, int x, int y, int z, const Lv<T>& C, T m) {
    const int ax = x / 2 - 1 + (x & 1), ay = y / 2 - 1 + (y & 1);
    const T wx = (x & 1) ? T(.25) : T(.75), wy = (y & 1) ? T(.25) : T(.75);
    if (BC == AFSI_BC_NEUMANN) {
        const int az = z / 2 - 1 + (z & 1);
        const T wz = (z & 1) ? T(.25) : T(.75);
        const int x0 = ax < 0 ? 0 : ax, x1 = ax + 1 < C.nx - 1 ? ax + 1 : C.nx - 1;
        const int y0 = ay < 0 ? 0 : ay, y1 = ay + 1 < C.ny - 1 ? ay + 1 : C.ny - 1;
        const int z0 = az < 0 ? 0 : az, z1 = az + 1 < C.nz - 1 ? az + 1 : C.nz - 1;
        auto at = [&](int i, int j, int k) { return c[index_of(i, j, k, C)] - m; };
        const T c00 = at(x0, y0, z0) * (T(1) - wz) + at(x0, y0, z1) * wz;
        const T c01 = at(x0, y1, z0) * (T(1) - wz) + at(x0, y1, z1) * wz;
        const T c10 = at(x1, y0, z0) * (T(1) - wz) + at(x1, y0, z1) * wz;
        const T c11 = at(x1, y1, z0) * (T(1) - wz) + at(x1, y1, z1) * wz;
        return (c00 * (T(1) - wy) + c01 * wy) * (T(1) - wx) + (c10 * (T(1) - wy) + c11 * wy) * wx;
    }
    const T c00 = coarse_at<BC>(c, ax, ay, C, m), c01 = coarse_at<BC>(c, ax, ay + 1, C, m);
    const T c10 = coarse_at<BC>(c, ax + 1, ay, C, m), c11 = coarse_at<BC>(c, ax + 1, ay + 1, C, m);
    return (c00 * (T(1) - wy) + c01 * wy) * (T(1) - wx) + (c10 * (T(1) - wy) + c11 * wy) * wx;
}

// ----------------------------------------------------------- coarse block

template <class T>
struct CoarseLevels {
    Lv<T> lv[AFSI_MG_MAX_LEVELS];
    int first, last;  // level indices handled here
};

// Block-wide mean (deterministic) of smem array a[0..n).
template <class T>
__device__ T block_mean(const T* a, int n, double* red) {
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += double(a[i]);
    v = block_sum(v, red);
    __shared__ double bcast;
    if (threadIdx.x == 0) bcast = v / double(n);
    __syncthreads();
    return T(bcast);
}

template <int BC, class T>
__device__ void block_smooth(T*& cur, T*& oth, const T* R, const Lv<T>& L, int smooth) {
    for (int s = 0; s < smooth; ++s) {
        for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
            int x, y, z;
            coords32(i, L, x, y, z);
            const T pc = cur[i];
            const T a = neg_lap<BC, false>(cur, i, x, y, z, L, T(0), pc);
            oth[i] = pc + (omega<T>() * (R[i] - a)) / diag_at<BC>(x, y, z, L);
        }
        __syncthreads();
        T* t = cur;
        cur = oth;
        oth = t;
    }
}

// Levels first..last of one V-cycle in one CTA (fast arithmetic).  rhs of
// level `first` comes from global memory (shifted by rhs_sum/n); p[first]
// starts from p_global (first==0) or zero; the final p[first] is written to
// p_out.
template <int BC, class T, class TC>
__device__ void coarse_cycle(T* smem, const T* __restrict__ rhs_global, const double* rhs_sum, const T* p_global,
                             T* p_out, const TC* __restrict__ cinv, const CoarseLevels<T>& cl, int smooth) {
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
        for (int i = threadIdx.x; i < cl.lv[f].n; i += blockDim.x) {
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
            for (int r = threadIdx.x; r < L.n; r += blockDim.x) {
                double s = 0.0;
                for (int j = 0; j < L.n; ++j) s += double(cinv[int64_t(r) * L.n + j]) * double(R[l][j]);
                P[l][r] = T(s);
            }
            __syncthreads();
            if (singular) {
                const T m = block_mean(P[l], int(L.n), red);
                for (int i = threadIdx.x; i < L.n; i += blockDim.x) P[l][i] = P[l][i] - m;
                __syncthreads();
            }
            break;
        }
        T* cur = P[l];
        T* oth = Q[l];
        block_smooth<BC>(cur, oth, R[l], L, smooth);
        const T m = singular ? block_mean(cur, int(L.n), red) : T(0);
        for (int i = threadIdx.x; i < L.n; i += blockDim.x) P[l][i] = cur[i] - m;
        __syncthreads();
        const Lv<T>& C = cl.lv[l + 1];
        for (int c = threadIdx.x; c < C.n; c += blockDim.x) {
            int cx, cy, cz;
            coords32(c, C, cx, cy, cz);
            R[l + 1][c] = restrict_residual_at<BC, false>(P[l], R[l], cx, cy, cz, L, T(0));
            P[l + 1][c] = T(0);
        }
        __syncthreads();
        if (singular) {
            const T mc = block_mean(R[l + 1], int(C.n), red);
            for (int i = threadIdx.x; i < C.n; i += blockDim.x) R[l + 1][i] = R[l + 1][i] - mc;
            __syncthreads();
        }
    }
    // up
    for (int l = cl.last - 1; l >= f; --l) {
        const Lv<T>& L = cl.lv[l];
        const Lv<T>& C = cl.lv[l + 1];
        for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
            int x, y, z;
            coords32(i, L, x, y, z);
            P[l][i] = P[l][i] + prolong_at<BC>(P[l + 1], x, y, z, C, T(0));
        }
        __syncthreads();
        T* cur = P[l];
        T* oth = Q[l];
        block_smooth<BC>(cur, oth, R[l], L, smooth);
        const T m = singular ? block_mean(cur, int(L.n), red) : T(0);
        for (int i = threadIdx.x; i < L.n; i += blockDim.x) P[l][i] = cur[i] - m;
        __syncthreads();
    }
    for (int i = threadIdx.x; i < cl.lv[f].n; i += blockDim.x) p_out[i] = P[f][i];
    __syncthreads();
}

}  // namespace afsi
