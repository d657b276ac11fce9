// Run-merged accumulation of an element's spread into a shared-memory box.
//
// The interaction points of one element are few lattice cells apart: on the
// P2 shells of the transfer workloads the 64 points of an order-4 element
// fall on about five distinct support origins per component, and consecutive
// points of the rule share their origin four times out of five.  The warp
// therefore sums the 4x4x4 contributions of each run of consecutive points
// with the same support origin in registers and adds the sum to the box once
// per run instead of once per point, with plain read-modify-writes in a fixed
// order: deterministic, no atomics.
//
// Box layout (padded_strides): entry (x,y,z) at x*sx + y*sy + z with sy odd
// and sx = 4 (mod 8); the 16 offsets li*sx + lj*sy (li, lj in 0..3) are 16
// distinct values mod 16, so a half-warp's 16 lanes meet 16 different 8-byte
// bank pairs.
#pragma once
#include <type_traits>
#include "common.cuh"

namespace afsi {

// Padded strides for a box of y extent ey and z extent ez.
__device__ __forceinline__ void padded_strides(int ey, int ez, int& sx, int& sy) {
    sy = ez | 1;
    sx = ey * sy;
    sx += (12 - (sx & 7)) & 7;
}

// Run key of a support origin (dx, dy, dz) relative to the box corner
// (each in [0, 1024)); -1 marks a point that takes no part.
__device__ __forceinline__ int run_key(int dx, int dy, int dz) { return dx | (dy << 10) | (dz << 20); }

// Accumulate points 0..n-1 (n <= C) of one component into `box` (padded
// strides sx, sy).  key[q]: run_key of point q's support origin in the box,
// or -1; f[q]: its force factor; wx/wy/wz: its x, y and z weight rows at q*12
// (four each).  The warp takes the runs of consecutive points with one key
// in order; within a run, half h takes points h, h+2, ... and lane (i,j)
// accumulates ((wx[i] * wy[j]) * f) * wz[k] for k = 0..3 in registers.  At
// the end of the run the halves exchange two sums each (half 0 keeps z links
// 0-1, half 1 links 2-3) and every lane adds two values to the box: one
// read-modify-write pass of the whole warp per run, in a fixed order.
template <class T, int C>
__device__ __forceinline__ void spread_runs(T* box, const int* key, const T* f, const T* wx, const T* wy,
                                            const T* wz, int n, int sx, int sy) {
    const int lane = threadIdx.x & 31, half = lane >> 4, li = (lane >> 2) & 3, lj = lane & 3;
    unsigned long long heads = 0;
#pragma unroll
    for (int j = 0; j < C / 32; ++j) {
        const int q = lane + 32 * j;
        const bool h = q < n && (q == 0 || key[q] != key[q - 1]);
        heads |= static_cast<unsigned long long>(__ballot_sync(0xffffffffu, h)) << (32 * j);
    }
    using P = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    while (heads) {
        const int s0 = __ffsll(static_cast<long long>(heads)) - 1;
        heads &= heads - 1;
        const int e0 = heads ? __ffsll(static_cast<long long>(heads)) - 1 : n;
        const int k = key[s0];
        if (k < 0) continue;
        T acc[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll 2
        for (int q = s0 + half; q < e0; q += 2) {
            const T a = (wx[q * 12 + li] * wy[q * 12 + lj]) * f[q];
            const P za = reinterpret_cast<const P*>(wz + q * 12)[0];
            const P zb = reinterpret_cast<const P*>(wz + q * 12)[1];
            acc[0] = fma(a, za.x, acc[0]);
            acc[1] = fma(a, za.y, acc[1]);
            acc[2] = fma(a, zb.x, acc[2]);
            acc[3] = fma(a, zb.y, acc[3]);
        }
        const T r0 = __shfl_xor_sync(0xffffffffu, half ? acc[0] : acc[2], 16);
        const T r1 = __shfl_xor_sync(0xffffffffu, half ? acc[1] : acc[3], 16);
        const T t0 = (half ? acc[2] : acc[0]) + r0, t1 = (half ? acc[3] : acc[1]) + r1;
        T* dst = box + ((k & 1023) + li) * sx + (((k >> 10) & 1023) + lj) * sy + (k >> 20) + 2 * half;
        dst[0] += t0;
        dst[1] += t1;
        __syncwarp();
    }
}

// Groups points 0..n-1 (n <= C) by key, 32 points at a time (one per
// lane, __match_any_sync): perm lists, run by run, the points of one key
// among points j*32 .. j*32+31 in index order, padded with `zero` (the index of
// an all-zero row) to a multiple of four; run r spans perm[rs[r] .. rs[r+1])
// and has key rk[r].  Points with key < 0 take no part.  perm needs room for
// 4 n entries.  Returns the number of runs.
template <int C>
__device__ __forceinline__ int group_runs(const int* key, int n, int* perm, int* rs, int* rk, int zero) {
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    int pos = 0, r = 0;
#pragma unroll
    for (int j = 0; j < C / 32; ++j) {
        const int q = lane + 32 * j;
        const int k = q < n ? key[q] : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, k);
        unsigned leaders = __ballot_sync(0xffffffffu, k >= 0 && (peers & below) == 0u);
        while (leaders) {
            const int l = __ffs(leaders) - 1;
            leaders &= leaders - 1u;
            const unsigned grp = __shfl_sync(0xffffffffu, peers, l);
            const int kl = __shfl_sync(0xffffffffu, k, l);
            const int cnt = __popc(grp), padded = (cnt + 3) & ~3;
            if ((grp >> lane) & 1u) perm[pos + __popc(grp & below)] = q;
            if (lane < padded - cnt) perm[pos + cnt + lane] = zero;
            if (lane == 0) {
                rs[r] = pos;
                rk[r] = kl;
            }
            pos += padded;
            ++r;
        }
    }
    if (lane == 0) rs[r] = pos;
    __syncwarp();
    return r;
}

// D = A * B + D for one 8x8x4 FP64 tensor-core step (mma.m8n8k4, A row-major
// 8x4, B column-major 4x8): lane t holds A[t/4][t%4], B[t%4][t/4] and
// D[t/4][2(t%4)], D[t/4][2(t%4)+1].
__device__ __forceinline__ void mma884(double d[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// FP64 form of spread_runs on the tensor cores.  The points are grouped by key
// (group_runs); for a run with support origin K the 4x4x4 sum
// S[i][j][k] = sum_p X_p[i] (f_p Y_p[j] Z_p[k]) is the product of the 4 x L
// matrix of x weights and the L x 16 matrix of (f Y (x) Z) rows, taken four
// points at a time by two m8n8k4 steps (j = 0-1 and j = 2-3; rows 4-7 of A
// read the zero row).  Lanes 0-15 then add their two pairs of z links to the
// box.  Row `zero` (index C) of wx/wy/wz and f must be all zero; perm, rs and
// rk are group_runs' scratch.
template <int C>
__device__ __forceinline__ void spread_runs_mma(double* box, const int* key, const double* f, const double* wx,
                                                const double* wy, const double* wz, int n, int sx, int sy,
                                                int* perm, int* rs, int* rk) {
    const int lane = threadIdx.x & 31;
    const int runs = group_runs<C>(key, n, perm, rs, rk, C);
    const int slot = lane & 3, row = lane >> 2;     // A: x offset `row`, point `slot`
    const int jb = lane >> 4, kb = (lane >> 2) & 3;  // B column lane/4 = (j, k) = (jb [+2], kb)
    const int ax = row & 3;
    for (int r = 0; r < runs; ++r) {
        const int s0 = rs[r], e0 = rs[r + 1], K = rk[r];
        double d0[2] = {0.0, 0.0}, d1[2] = {0.0, 0.0};
#pragma unroll 2
        for (int b = s0 + slot; b < e0; b += 4) {
            const int q = perm[b];
            const int qa = row < 4 ? q : C;
            const double a = wx[qa * 12 + ax];
            const double fz = f[q] * wz[q * 12 + kb];
            mma884(d0, a, wy[q * 12 + jb] * fz);
            mma884(d1, a, wy[q * 12 + jb + 2] * fz);
        }
        if (row < 4) {
            const int j0 = slot >> 1, k0 = 2 * (slot & 1);
            double* dst = box + ((K & 1023) + row) * sx + (((K >> 10) & 1023) + j0) * sy + (K >> 20) + k0;
            dst[0] += d0[0];
            dst[1] += d0[1];
            dst += 2 * sy;
            dst[0] += d1[0];
            dst[1] += d1[1];
        }
        __syncwarp();
    }
}

// The element spread of one component: the FP64 tensor-core form for double,
// the register-run form otherwise.
template <class T, int C>
__device__ __forceinline__ void spread_element(T* box, const int* key, const T* f, const T* wx, const T* wy,
                                               const T* wz, int n, int sx, int sy, int* perm, int* rs, int* rk) {
    if constexpr (sizeof(T) == 8)
        spread_runs_mma<C>(box, key, f, wx, wy, wz, n, sx, sy, perm, rs, rk);
    else
        spread_runs<T, C>(box, key, f, wx, wy, wz, n, sx, sy);
}

// ------------------------------------------------------------------ gather
//
// Face patch of one component for the lane-per-point gathers: entry (x,y,z)
// at x*kGSX + y*kGSY + z with fixed strides, so the 64 loads of a support
// have immediate offsets; kGSX = 68 (4 mod 16) and kGSY = 8 put the support
// origins of nearby points in different bank pairs, and lanes whose points
// share an origin read the same words.  Extents up to kGExt per axis.
constexpr int kGSX = 68, kGSY = 8, kGExt = 8;
constexpr int kGPatch = kGExt * kGSX;

// sum_ijk wx[i] wy[j] wz[k] p[i*sx + j*sy + k]
template <class T, class I>
__device__ __forceinline__ T support_dot(const T* p, I sx, I sy, const T wx[4], const T wy[4], const T wz[4]) {
    T u = T(0);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        T ti = T(0);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const T* r = p + i * sx + j * sy;
            T tz = r[0] * wz[0];
            tz = fma(r[1], wz[1], tz);
            tz = fma(r[2], wz[2], tz);
            tz = fma(r[3], wz[3], tz);
            ti = fma(wy[j], tz, ti);
        }
        u = fma(wx[i], ti, u);
    }
    return u;
}

}  // namespace afsi
