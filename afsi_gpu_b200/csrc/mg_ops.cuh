// Device operators of the MAC multigrid shared by the per-level kernels
// (mg.cu) and the persistent V-cycle (mg_persistent.cu).  See mg.cu for the
// operators, arithmetic modes and launch geometry.
#pragma once
#include "common.cuh"

namespace afsi {


constexpr int kThreads = 256;
constexpr int kCoarseThreads = 1024;
constexpr int64_t kCoarseCells = 4096;  // levels at or below this size run in one CTA

// 3D levels (z fastest) for the closed and the open box; 2D (y fastest) otherwise.
__host__ __device__ constexpr bool is3d(int bc) { return bc == AFSI_BC_NEUMANN || bc == AFSI_BC_DIRICHLET; }
// Singular operators (constants in the null space): mean-zero gauge.
__host__ __device__ constexpr bool singular_bc(int bc) { return bc == AFSI_BC_NEUMANN || bc == AFSI_BC_PERIODIC; }

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

// Grid barrier of a cooperative launch (every block resident): arrival
// counter, generation word, error word (a barrier that waits longer than
// about a second sets it, and every later barrier returns at once), one
// partial per block and reduction result slots.
struct GridSync {
    unsigned int* count;
    unsigned int* gen;
    int* error;
    double* partial;  // one per block
    double* slot;     // reduction results: [level*3 + {0: p down, 1: p up, 2: rhs}], [kNormSlot]
};


// Barrier with an optional deterministic sum of one double per block
// (valid in thread 0).  Returns false if any barrier of this launch failed.
__device__ inline bool grid_sync(const GridSync& g, double v, double* slot) {
    __shared__ int s_ok;
    __shared__ bool s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_last = false;
        const int failed = *reinterpret_cast<volatile int*>(g.error);
        if (failed) {
            s_ok = 0;
        } else {
            const unsigned my_gen = *reinterpret_cast<volatile unsigned*>(g.gen);
            if (slot) g.partial[blockIdx.x] = v;
            __threadfence();
            const unsigned arrived = atomicAdd(g.count, 1u);
            if (arrived == gridDim.x - 1) {
                s_last = true;  // release after the reduction below
            } else {
                const long long t0 = clock64();
                while (*reinterpret_cast<volatile unsigned*>(g.gen) == my_gen) {
                    if (clock64() - t0 > 2000000000LL) {
                        atomicOr(g.error, 1);
                        break;
                    }
                    __nanosleep(32);
                }
            }
            s_ok = 1;
        }
    }
    __syncthreads();
    if (s_last) {
        if (threadIdx.x < 32) {
            double t = 0.0;
            if (slot)
                for (unsigned i = threadIdx.x; i < gridDim.x; i += 32) t += __ldcg(g.partial + i);
            t = warp_sum(t);
            if (threadIdx.x == 0) {
                if (slot) *slot = t;
                *g.count = 0u;
                __threadfence();
                atomicAdd(g.gen, 1u);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (*reinterpret_cast<volatile int*>(g.error)) s_ok = 0;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ double read_mean(const double* slot, int64_t n) { return __ldcg(slot) / double(n); }

// Grid barrier without a reduction: the block's threads meet at the CTA
// barrier, then thread 0 arrives with an acquire-release add on the counter;
// the last block to arrive resets the counter and releases the generation
// word, the others spin on it with acquire loads (bounded as grid_sync).  The
// release by thread 0 is cumulative over the writes its CTA barrier ordered
// before it, so every block's writes are visible to every block afterwards.
// Returns false if any barrier of the launch failed.
__device__ inline bool grid_barrier(const GridSync& g) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned gen0, arrived;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(gen0) : "l"(g.gen) : "memory");
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(arrived) : "l"(g.count) : "memory");
        if (arrived == gridDim.x - 1) {
            asm volatile("st.relaxed.gpu.global.u32 [%0], 0;" ::"l"(g.count) : "memory");
            asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(g.gen) : "memory");
        } else {
            const long long t0 = clock64();
            unsigned gen;
            do {
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(gen) : "l"(g.gen) : "memory");
                if (gen == gen0 && clock64() - t0 > 2000000000LL) {
                    atomicOr(g.error, 1);
                    break;
                }
            } while (gen == gen0);
        }
        int err;
        asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(err) : "l"(g.error) : "memory");
        if (err) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <int BC, class T>
__host__ __device__ __forceinline__ T diag_at(int x, int y, int z, const Lv<T>& L) {
    T d = T(0);
    if (BC == AFSI_BC_DIRICHLET) {
        // mac/open_boundary.py:47-52: 2·Σ h^-2, plus h^-2 on each boundary face
        d = T(2) * ((L.ih2[0] + L.ih2[1]) + L.ih2[2]);
        if (x == 0) d += L.ih2[0];
        if (x == L.nx - 1) d += L.ih2[0];
        if (y == 0) d += L.ih2[1];
        if (y == L.ny - 1) d += L.ih2[1];
        if (z == 0) d += L.ih2[2];
        if (z == L.nz - 1) d += L.ih2[2];
    } else if (BC == AFSI_BC_NEUMANN) {
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
    if (BC == AFSI_BC_DIRICHLET) {
        // zero pressure half a cell outside: the missing neighbour is the ghost -p
        const int64_t sx = int64_t(L.ny) * L.nz, sy = L.nz;
        a = x + 1 < L.nx ? a - scale<Exact>((p[i + sx] - m) - pc, L, 0) : a + scale<Exact>(pc + pc, L, 0);
        a = x > 0 ? a + scale<Exact>(pc - (p[i - sx] - m), L, 0) : a + scale<Exact>(pc + pc, L, 0);
        a = y + 1 < L.ny ? a - scale<Exact>((p[i + sy] - m) - pc, L, 1) : a + scale<Exact>(pc + pc, L, 1);
        a = y > 0 ? a + scale<Exact>(pc - (p[i - sy] - m), L, 1) : a + scale<Exact>(pc + pc, L, 1);
        a = z + 1 < L.nz ? a - scale<Exact>((p[i + 1] - m) - pc, L, 2) : a + scale<Exact>(pc + pc, L, 2);
        a = z > 0 ? a + scale<Exact>(pc - (p[i - 1] - m), L, 2) : a + scale<Exact>(pc + pc, L, 2);
    } else if (BC == AFSI_BC_NEUMANN) {
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

// Cells of this thread in the launch geometry of launch_for: the block covers
// the two fastest axes; in 3D the grid's z dimension strides over x slabs
// (the grid is capped, so one block may own several slabs).  f(x, y, z).
template <int BC, class T, class F>
__device__ __forceinline__ void for_my_cells(const Lv<T>& L, F f) {
    const int fast = blockIdx.x * blockDim.x + threadIdx.x;
    const int mid = blockIdx.y * blockDim.y + threadIdx.y;
    if (is3d(BC)) {
        if (fast >= L.nz || mid >= L.ny) return;
        for (int x = blockIdx.z; x < L.nx; x += gridDim.z) f(x, mid, fast);
    } else {
        if (fast < L.ny && mid < L.nx) f(mid, fast, 0);
    }
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
__host__ __device__ __forceinline__ T omega() { return T(2.0 / 3.0); }

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

// site_finish, then tail(result) in thread 0 of the last block, after the
// result is written.
template <class Tail>
__device__ __forceinline__ void site_finish_then(const Site& s, double v, double* sqrt_out, Tail tail) {
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
        tail(sqrt_out ? sqrt(acc) : acc);
    }
}

template <int BC, bool Exact, class T>
__device__ __forceinline__ T restrict_residual_at(const T* __restrict__ p, const T* __restrict__ rhs, int cx, int cy,
                                                  int cz, const Lv<T>& L, T m) {
    if constexpr (is3d(BC)) {
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
    } else {
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
    if (is3d(BC)) {
        const int az = z / 2 - 1 + (z & 1);
        const T wz = (z & 1) ? T(.25) : T(.75);
        const int x0 = ax < 0 ? 0 : ax, x1 = ax + 1 < C.nx - 1 ? ax + 1 : C.nx - 1;
        const int y0 = ay < 0 ? 0 : ay, y1 = ay + 1 < C.ny - 1 ? ay + 1 : C.ny - 1;
        const int z0 = az < 0 ? 0 : az, z1 = az + 1 < C.nz - 1 ? az + 1 : C.nz - 1;
        // ghost one cell outside the coarse grid: the edge value (closed box)
        // or its negative (open box, odd extension: mac/dirichlet_mg.py:52-62)
        const bool odd = BC == AFSI_BC_DIRICHLET;
        const bool gx0 = odd && ax < 0, gx1 = odd && ax + 1 > C.nx - 1, gy0 = odd && ay < 0,
                   gy1 = odd && ay + 1 > C.ny - 1, gz0 = odd && az < 0, gz1 = odd && az + 1 > C.nz - 1;
        auto at = [&](int i, int j, int k, bool fi, bool fj, bool fk) {
            const T v = c[index_of(i, j, k, C)] - m;
            return (fi != fj) != fk ? -v : v;  // one sign flip per ghost axis
        };
        const T c00 = at(x0, y0, z0, gx0, gy0, gz0) * (T(1) - wz) + at(x0, y0, z1, gx0, gy0, gz1) * wz;
        const T c01 = at(x0, y1, z0, gx0, gy1, gz0) * (T(1) - wz) + at(x0, y1, z1, gx0, gy1, gz1) * wz;
        const T c10 = at(x1, y0, z0, gx1, gy0, gz0) * (T(1) - wz) + at(x1, y0, z1, gx1, gy0, gz1) * wz;
        const T c11 = at(x1, y1, z0, gx1, gy1, gz0) * (T(1) - wz) + at(x1, y1, z1, gx1, gy1, gz1) * wz;
        return (c00 * (T(1) - wy) + c01 * wy) * (T(1) - wx) + (c10 * (T(1) - wy) + c11 * wy) * wx;
    }
    const T c00 = coarse_at<BC>(c, ax, ay, C, m), c01 = coarse_at<BC>(c, ax, ay + 1, C, m);
    const T c10 = coarse_at<BC>(c, ax + 1, ay, C, m), c11 = coarse_at<BC>(c, ax + 1, ay + 1, C, m);
    return (c00 * (T(1) - wy) + c01 * wy) * (T(1) - wx) + (c10 * (T(1) - wy) + c11 * wy) * wx;
}

// ----------------------------------------------------------- coarse block
//
// All levels from `first` down run inside one thread block in shared memory.
// The block works with fast arithmetic and keeps the single SM's instruction
// count low:
//  * cell coordinates come from shifts when a level's extents are powers of
//    two (division otherwise);
//  * the stencil is branch-free: a missing Neumann neighbour reads as the
//    cell itself (zero flux), the channel outlet ghost as its negative, the
//    periodic neighbour through the wrapped index; the axis terms are
//    combined with fused multiply-adds;
//  * the Jacobi update multiplies by omega/diag looked up in a per-level
//    table of the 64 boundary classes (first/last cell per axis), built once
//    per launch;
//  * the mean-zero gauge of the singular operators is carried as pending
//    shifts: the mean of a level's iterate is summed inside its last sweep
//    (one barrier per reduction, every thread adds the 32 warp partials in the
//    same order) and subtracted where the iterate is next read — in the
//    prolongation, the next level's first sweep or the final copy — instead of
//    in passes of their own.  A(p - m·1) = A p for these operators, so the
//    restriction reads the unshifted iterate;
//  * a zero initial iterate is folded into the first sweep;
//  * the dense coarsest solve is warp-cooperative (lanes over a row).

template <class T>
struct CoarseLevels {
    Lv<T> lv[AFSI_MG_MAX_LEVELS];
    int first, last;  // level indices handled here
};

// Sum of v over the block, returned to every thread: one barrier.  Warp
// partials go to red (32 slots); every warp then reduces the slots with the
// same butterfly, so all threads get the same value.  The caller alternates
// between two red buffers so that a slot is rewritten only after a later
// barrier.
__device__ __forceinline__ double block_sum_all(double v, double* red) {
#pragma unroll
    for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    const int lane = threadIdx.x & 31;
    if (lane == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = lane < int(blockDim.x >> 5) ? red[lane] : 0.0;
#pragma unroll
    for (int d = 16; d; d >>= 1) t += __shfl_xor_sync(0xffffffffu, t, d);
    return t;
}

template <class T>
struct FastCoords {
    int lz, ly, mz, my;
    bool pow2;
    __device__ void init(const Lv<T>& L) {
        pow2 = !(L.nz & (L.nz - 1)) && !(L.ny & (L.ny - 1));
        lz = __ffs(L.nz) - 1;
        ly = __ffs(L.ny) - 1;
        mz = L.nz - 1;
        my = L.ny - 1;
    }
    __device__ __forceinline__ void get(int i, const Lv<T>& L, int& x, int& y, int& z) const {
        if (pow2) {
            z = i & mz;
            y = (i >> lz) & my;
            x = i >> (lz + ly);
        } else {
            coords32(i, L, x, y, z);
        }
    }
};

__host__ __device__ __forceinline__ int boundary_class(int x, int y, int z, int nx, int ny, int nz) {
    return (x == 0) | ((x == nx - 1) << 1) | ((y == 0) << 2) | ((y == ny - 1) << 3) | ((z == 0) << 4) |
           ((z == nz - 1) << 5);
}

// omega/diag of boundary class k of level L (diag_at order, one IEEE
// division), the same bits on the host and the device; classes that cannot
// occur (first and last both set on an axis longer than one cell) get an
// unused value.
template <int BC, class T>
__host__ __device__ __forceinline__ T omega_of_class(int k, const Lv<T>& L) {
    const int x = (k & 1) ? 0 : ((k & 2) ? L.nx - 1 : (L.nx > 2 ? 1 : 0));
    const int y = (k & 4) ? 0 : ((k & 8) ? L.ny - 1 : (L.ny > 2 ? 1 : 0));
    const int z = (k & 16) ? 0 : ((k & 32) ? L.nz - 1 : (L.nz > 2 ? 1 : 0));
    return omega<T>() / diag_at<BC>(x, y, z, L);
}

// omega/diag for each of the 64 boundary classes of level L.
template <int BC, class T>
__device__ void omega_table(const Lv<T>& L, T* table) {
    for (int k = threadIdx.x; k < 64; k += blockDim.x) table[k] = omega_of_class<BC>(k, L);
}

// The weighted-Jacobi update of the fast arithmetic, shared by the launched,
// batched and single-CTA sweeps: p + (rhs - A p) * (omega/diag) as one fused
// multiply-add; from a zero iterate rhs * (omega/diag).
template <class T>
__device__ __forceinline__ T jacobi_update(T pc, T r, T a, T w) { return __fma_rn(r - a, w, pc); }

// (A p)_i of the block path, pc = p_i.
template <int BC, class T>
__device__ __forceinline__ T block_apply(const T* __restrict__ p, int i, int x, int y, int z, const Lv<T>& L, T pc) {
    if (is3d(BC)) {
        const int sx = L.ny * L.nz, sy = L.nz;
        const T g = BC == AFSI_BC_DIRICHLET ? -pc : pc;  // wall ghost: open box -p, closed box p
        const T xm = x > 0 ? p[i - sx] : g, xp = x + 1 < L.nx ? p[i + sx] : g;
        const T ym = y > 0 ? p[i - sy] : g, yp = y + 1 < L.ny ? p[i + sy] : g;
        const T zm = z > 0 ? p[i - 1] : g, zp = z + 1 < L.nz ? p[i + 1] : g;
        return __fma_rn((pc - xm) + (pc - xp), L.ih2[0],
                        __fma_rn((pc - ym) + (pc - yp), L.ih2[1], ((pc - zm) + (pc - zp)) * L.ih2[2]));
    } else {
        const int sx = L.ny;
        T xm, xp;
        if (BC == AFSI_BC_CHANNEL) {
            xm = x > 0 ? p[i - sx] : pc;
            xp = x + 1 < L.nx ? p[i + sx] : -pc;  // outlet ghost: p = 0 on the face
        } else {
            xm = p[x > 0 ? i - sx : i + (L.nx - 1) * sx];
            xp = p[x + 1 < L.nx ? i + sx : i - (L.nx - 1) * sx];
        }
        const T ym = y > 0 ? p[i - 1] : pc, yp = y + 1 < L.ny ? p[i + 1] : pc;
        return __fma_rn((pc - xm) + (pc - xp), L.ih2[0], ((pc - ym) + (pc - yp)) * L.ih2[1]);
    }
}

// Full-weighting restriction of the residual rhs - A p at coarse cell (cx,cy,cz).
template <int BC, class T>
__device__ __forceinline__ T block_restrict(const T* __restrict__ p, const T* __restrict__ rhs, int cx, int cy, int cz,
                                            const Lv<T>& L) {
    if constexpr (is3d(BC)) {
        T v = T(0);
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int d = 0; d < 2; ++d) {
                    const int x = 2 * cx + a, y = 2 * cy + b, z = 2 * cz + d;
                    const int i = (x * L.ny + y) * L.nz + z;
                    v = v + (rhs[i] - block_apply<BC>(p, i, x, y, z, L, p[i]));
                }
        return v * T(.125);
    } else {
        T r[4];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const int x = 2 * cx + a, y = 2 * cy + b;
                const int i = x * L.ny + y;
                r[a * 2 + b] = rhs[i] - block_apply<BC>(p, i, x, y, 0, L, p[i]);
            }
        return ((r[0] + r[1]) + r[2] + r[3]) * T(.25);
    }
}

// `smooth` Jacobi sweeps of level L in ping-pong buffers cur/oth.  zero: the
// iterate starts at 0 (the first sweep reads no neighbours); rhs_shift: a
// pending mean of R, subtracted in the first sweep and written back.
// Returns the buffer of the final iterate; *mean gets its mean (singular BCs).
template <int BC, class T>
__device__ T* block_smooth(T* cur, T* oth, T* R, const Lv<T>& L, const FastCoords<T>& fc, const T* wrd, int smooth,
                           bool zero, T rhs_shift, double (*red)[32], int& rt, T* mean) {
    constexpr bool singular = singular_bc(BC);
    const int n = int(L.n);
    for (int s = 0; s < smooth; ++s) {
        const bool last = s == smooth - 1;
        double acc = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            int x, y, z;
            fc.get(i, L, x, y, z);
            const T w = wrd[boundary_class(x, y, z, L.nx, L.ny, L.nz)];
            T v;
            if (s == 0 && zero) {
                const T r = R[i] - rhs_shift;
                if (rhs_shift != T(0)) R[i] = r;
                v = r * w;
            } else {
                const T pc = cur[i];
                v = jacobi_update(pc, R[i], block_apply<BC>(cur, i, x, y, z, L, pc), w);
            }
            oth[i] = v;
            if (last) acc += double(v);
        }
        if (last && singular) {
            *mean = T(block_sum_all(acc, red[rt]) / double(n));
            rt ^= 1;
        } else {
            __syncthreads();
        }
        T* t = cur;
        cur = oth;
        oth = t;
    }
    if (!singular) *mean = T(0);
    return cur;
}

// Levels first..last of one V-cycle in one CTA (fast arithmetic).  rhs of
// level `first` comes from global memory (shifted by rhs_sum/n); p[first]
// starts from p_global (first==0) or zero; the final p[first], mean removed
// for the singular operators, is written to p_out.  smem holds, per level, p,
// its Jacobi partner and rhs, then the omega/diag tables.
template <int BC, class T, class TC>
__device__ void coarse_cycle(T* smem, const T* __restrict__ rhs_global, const double* rhs_sum, const T* p_global,
                             T* p_out, const TC* __restrict__ cinv, const CoarseLevels<T>& cl, int smooth) {
    __shared__ double red[2][32];
    __shared__ T down_mean[AFSI_MG_MAX_LEVELS];  // pending mean of each level's pre-smoothed iterate
    constexpr bool singular = singular_bc(BC);
    int rt = 0;
    const int f = cl.first, last = cl.last;
    // layout: [P_f Q_f R_f][P_f+1 ...]...[tables]
    auto level_base = [&](int l) {
        int64_t off = 0;
        for (int k = f; k < l; ++k) off += 3 * cl.lv[k].n;
        return smem + off;
    };
    T* tables = level_base(last + 1);
    for (int l = f; l <= last; ++l) omega_table<BC>(cl.lv[l], tables + 64 * (l - f));
    {
        const T mr = T(site_mean(rhs_sum, cl.lv[f].n));
        T* P = level_base(f);
        T* R = P + 2 * cl.lv[f].n;
        for (int i = threadIdx.x; i < cl.lv[f].n; i += blockDim.x) {
            R[i] = rhs_global[i] - mr;
            if (p_global) P[i] = p_global[i];
        }
    }
    __syncthreads();
    // down: pre-smooth, restrict the residual; the restricted rhs mean is
    // pending into the next level's first sweep
    T rhs_shift = T(0);
    for (int l = f; l < last; ++l) {
        const Lv<T>& L = cl.lv[l];
        const Lv<T>& C = cl.lv[l + 1];
        T* P = level_base(l);
        T* R = P + 2 * L.n;
        T* Rc = level_base(l + 1) + 2 * C.n;
        FastCoords<T> fcL, fcC;
        fcL.init(L);
        fcC.init(C);
        T m;
        const T* cur = block_smooth<BC>(P, P + L.n, R, L, fcL, tables + 64 * (l - f), smooth,
                                        l > f || !p_global, rhs_shift, red, rt, &m);
        if (threadIdx.x == 0) down_mean[l] = m;
        double acc = 0.0;
        for (int c = threadIdx.x; c < C.n; c += blockDim.x) {
            int cx, cy, cz;
            fcC.get(c, C, cx, cy, cz);
            const T v = block_restrict<BC>(cur, R, cx, cy, cz, L);
            Rc[c] = v;
            acc += double(v);
        }
        if (singular) {
            rhs_shift = T(block_sum_all(acc, red[rt]) / double(C.n));
            rt ^= 1;
        } else {
            __syncthreads();
        }
    }
    // dense coarsest solve p = inv * (rhs - shift) (mac/mg_workspace.py:86-90), warp per row
    T coarse_shift;
    {
        const Lv<T>& L = cl.lv[last];
        T* P = level_base(last);
        const T* R = P + 2 * L.n;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
        double acc = 0.0;
        for (int r = warp; r < L.n; r += warps) {
            double s = 0.0;
            for (int j = lane; j < L.n; j += 32) s += double(cinv[int64_t(r) * L.n + j]) * double(R[j] - rhs_shift);
            s = warp_sum(s);
            const T v = T(s);
            if (lane == 0) {
                P[r] = v;
                acc += double(v);
            }
        }
        if (singular) {
            coarse_shift = T(block_sum_all(acc, red[rt]) / double(L.n));
            rt ^= 1;
        } else {
            coarse_shift = T(0);
            __syncthreads();
        }
    }
    // up: add the prolonged correction to the shifted pre-smoothed iterate,
    // post-smooth; the level's mean is pending into the level above
    const T* corr = level_base(last);
    for (int l = last - 1; l >= f; --l) {
        const Lv<T>& L = cl.lv[l];
        const Lv<T>& C = cl.lv[l + 1];
        T* P = level_base(l);
        T* Q = P + L.n;
        T* R = Q + L.n;
        T* down = (smooth & 1) ? Q : P;  // where the pre-smoothing left the iterate
        const T dm = down_mean[l];
        FastCoords<T> fcL;
        fcL.init(L);
        for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
            int x, y, z;
            fcL.get(i, L, x, y, z);
            P[i] = (down[i] - dm) + prolong_at<BC>(corr, x, y, z, C, coarse_shift);
        }
        __syncthreads();
        T m;
        corr = block_smooth<BC>(P, Q, R, L, fcL, tables + 64 * (l - f), smooth, false, T(0), red, rt, &m);
        coarse_shift = m;
    }
    for (int i = threadIdx.x; i < cl.lv[f].n; i += blockDim.x) p_out[i] = corr[i] - coarse_shift;
    __syncthreads();
}

// Red-black Gauss-Seidel sweeps of level L in place (omega 1): cells with
// (x+y+z) even, then odd, p += (R - A p)/diag (fast block arithmetic).
template <int BC, class T>
__device__ void block_smooth_rb(T* P, const T* R, const Lv<T>& L, const FastCoords<T>& fc, int smooth) {
    const int n = int(L.n);
    for (int s = 0; s < smooth; ++s) {
        for (int color = 0; color < 2; ++color) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                int x, y, z;
                fc.get(i, L, x, y, z);
                if (((x + y + z) & 1) != color) continue;
                const T pc = P[i];
                P[i] = pc + (R[i] - block_apply<BC>(P, i, x, y, z, L, pc)) / diag_at<BC>(x, y, z, L);
            }
            __syncthreads();
        }
    }
}

// Levels first..last of one red-black V-cycle in one CTA: rhs of level
// `first` from global memory (already mean-free for singular problems), p
// from p_global or zero; coarse right-hand sides shifted to mean zero, zero
// coarse starts, the dense coarsest solve (mean removed for singular
// problems), prolongation and post-smoothing; the final p[first] goes to p_out.
template <int BC, class T, class TC>
__device__ void coarse_cycle_rb(T* smem, const T* __restrict__ rhs_global, const T* p_global, T* p_out,
                                const TC* __restrict__ cinv, const CoarseLevels<T>& cl, int smooth) {
    __shared__ double red[2][32];
    constexpr bool singular = singular_bc(BC);
    int rt = 0;
    const int f = cl.first, last = cl.last;
    auto level_base = [&](int l) {
        int64_t off = 0;
        for (int k = f; k < l; ++k) off += 3 * cl.lv[k].n;
        return smem + off;
    };
    {
        T* P = level_base(f);
        T* R = P + 2 * cl.lv[f].n;
        for (int i = threadIdx.x; i < cl.lv[f].n; i += blockDim.x) {
            R[i] = rhs_global[i];
            P[i] = p_global ? p_global[i] : T(0);
        }
    }
    __syncthreads();
    for (int l = f; l < last; ++l) {
        const Lv<T>& L = cl.lv[l];
        const Lv<T>& C = cl.lv[l + 1];
        T* P = level_base(l);
        const T* R = P + 2 * L.n;
        T* Pc = level_base(l + 1);
        T* Rc = Pc + 2 * C.n;
        FastCoords<T> fcL, fcC;
        fcL.init(L);
        fcC.init(C);
        block_smooth_rb<BC>(P, R, L, fcL, smooth);
        double acc = 0.0;
        for (int c = threadIdx.x; c < C.n; c += blockDim.x) {
            int cx, cy, cz;
            fcC.get(c, C, cx, cy, cz);
            const T v = block_restrict<BC>(P, R, cx, cy, cz, L);
            Rc[c] = v;
            Pc[c] = T(0);
            acc += double(v);
        }
        if (singular) {
            const T m = T(block_sum_all(acc, red[rt]) / double(C.n));
            rt ^= 1;
            for (int c = threadIdx.x; c < C.n; c += blockDim.x) Rc[c] = Rc[c] - m;
        }
        __syncthreads();
    }
    {
        const Lv<T>& L = cl.lv[last];
        T* P = level_base(last);
        const T* R = P + 2 * L.n;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
        double acc = 0.0;
        for (int r = warp; r < L.n; r += warps) {
            double s = 0.0;
            for (int j = lane; j < L.n; j += 32) s += double(cinv[int64_t(r) * L.n + j]) * double(R[j]);
            s = warp_sum(s);
            if (lane == 0) {
                P[r] = T(s);
                acc += double(T(s));
            }
        }
        if (singular) {
            const T m = T(block_sum_all(acc, red[rt]) / double(L.n));
            rt ^= 1;
            for (int r = threadIdx.x; r < L.n; r += blockDim.x) P[r] = P[r] - m;
        }
        __syncthreads();
    }
    for (int l = last - 1; l >= f; --l) {
        const Lv<T>& L = cl.lv[l];
        const Lv<T>& C = cl.lv[l + 1];
        T* P = level_base(l);
        const T* R = P + 2 * L.n;
        const T* corr = level_base(l + 1);
        FastCoords<T> fcL;
        fcL.init(L);
        for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
            int x, y, z;
            fcL.get(i, L, x, y, z);
            P[i] = P[i] + prolong_at<BC>(corr, x, y, z, C, T(0));
        }
        __syncthreads();
        block_smooth_rb<BC>(P, R, L, fcL, smooth);
    }
    const T* P = level_base(f);
    for (int i = threadIdx.x; i < cl.lv[f].n; i += blockDim.x) p_out[i] = P[i];
    __syncthreads();
}

}  // namespace afsi
