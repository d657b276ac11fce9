// P2 element transfers (spread, gather-assemble) for the B200.
//
// One warp owns one P2 element at a time (grid-stride over elements) and
// works on two quadrature points at once: each half-warp takes one point and
// its 16 lanes own the (i,j) columns of the point's 4x4x4 support, with the
// four z links of a column handled by that lane.
//
// Spread: the element's contributions are accumulated into a shared-memory
// box covering all its supports.  Each half-warp has a private copy of the
// box, so the adds are plain read-modify-writes with a fixed order (points
// h, h+2, h+4, ... in half h): no atomics.  The two copies are summed and
// flushed to the face arrays with one L2 reduction per non-zero face — about
// 400 per element instead of 192 per point.
// Gather: the face values of the box are staged in shared memory once per
// element; each point reads its 64 links from there and the 16 lanes reduce
// with four shuffles.  The nodal sums Σ_q N[q,a] W U(x_q) are accumulated in
// registers and added to the right-hand side (or written per element for the
// deterministic node reduction).
// Point forces F = (Σ_a N[q,a] value[a]) * W (mac/compact_transfer.py:29-35)
// are computed once per point by a lanes-over-points pass; the spread
// contribution is (φx·φy)·φz · (F/volume), one division per point instead of
// per link as in the reference kernel (one rounding of difference).
// An element whose box does not fit the shared-memory copies is processed
// with direct L2 reductions / global loads, checking each point's support
// against the grid (a point outside sets AFSI_FLAG_INDEX and is skipped).
#include <climits>
#include "common.cuh"
#include "p2.cuh"

namespace afsi {

constexpr int kWarps = 4;       // warps per block
constexpr int kChunk = 64;      // points whose forces are held at once
template <class T> struct BoxCap { static constexpr int value = 5120 / sizeof(T); };  // per copy (640 doubles)

template <class T>
struct SpreadStage {
    T f[3][kChunk];
    T coef[32];
    T copy[2][BoxCap<T>::value];
};

template <class T>
struct GatherStage {
    T patch[BoxCap<T>::value];
};

struct Box {
    int lo[3][3], ext[3][3], off[4];
};

__device__ __forceinline__ int64_t table_row(int64_t total, int64_t row, int c, int a) {
    return ((int64_t(a != c) * total) + row) * 3 + a;
}

// Box of all supports of element e, per component.
__device__ __forceinline__ void element_box(const int64_t* __restrict__ base, const P2Dims& g, int64_t e, Box& bx) {
    int mn[3][3], mx[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mn[c][a] = INT_MAX;
            mx[c][a] = INT_MIN;
        }
    for (int64_t q = threadIdx.x & 31; q < g.nq; q += 32) {
        const int64_t row = g.offset + e * g.nq + q;
        int b0[3], b1[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            b0[a] = int(base[row * 3 + a]);
            b1[a] = int(base[(g.total + row) * 3 + a]);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const int v = a == c ? b0[a] : b1[a];
                mn[c][a] = min(mn[c][a], v);
                mx[c][a] = max(mx[c][a], v);
            }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
#pragma unroll
            for (int d = 16; d; d >>= 1) {
                mn[c][a] = min(mn[c][a], __shfl_xor_sync(0xffffffffu, mn[c][a], d));
                mx[c][a] = max(mx[c][a], __shfl_xor_sync(0xffffffffu, mx[c][a], d));
            }
            bx.lo[c][a] = mn[c][a];
            bx.ext[c][a] = mx[c][a] - mn[c][a] + 4;
        }
    bx.off[0] = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) bx.off[c + 1] = bx.off[c] + bx.ext[c][0] * bx.ext[c][1] * bx.ext[c][2];
}

template <class T>
__device__ __forceinline__ bool box_fits(const Box& bx, const P2Dims& g) {
    const int64_t fe[3][3] = {{g.nx + 1, g.ny, g.nz}, {g.nx, g.ny + 1, g.nz}, {g.nx, g.ny, g.nz + 1}};
    bool inside = true;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) inside = inside && bx.lo[c][a] >= 0 && bx.lo[c][a] + bx.ext[c][a] <= fe[c][a];
    return inside && bx.off[3] <= BoxCap<T>::value;
}

__device__ __forceinline__ int64_t face_index(const P2Dims& g, int c, int x, int y, int z) {
    return (int64_t(x) * (g.ny + (c == 1)) + y) * (g.nz + (c == 2)) + z;
}

// The 4x4x4 box of component c starting at (x,y,z) lies inside its face array.
__device__ __forceinline__ bool point_inside(const P2Dims& g, int c, int x, int y, int z) {
    return x >= 0 && y >= 0 && z >= 0 && x + 3 < g.nx + (c == 0) && y + 3 < g.ny + (c == 1) &&
           z + 3 < g.nz + (c == 2);
}

// ------------------------------------------------------------------ spread

template <class T>
__global__ void __launch_bounds__(kWarps * 32) p2_spread_kernel(const T* __restrict__ value,
                                                                const int64_t* __restrict__ cells,
                                                                const T* __restrict__ N, const T* __restrict__ W,
                                                                const int64_t* __restrict__ base,
                                                                const T* __restrict__ phi, T* __restrict__ u0,
                                                                T* __restrict__ u1, T* __restrict__ u2, P2Dims g,
                                                                T volume, int32_t* status) {
    __shared__ SpreadStage<T> stage_all[kWarps];
    SpreadStage<T>& s = stage_all[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31, half = lane >> 4, li = (lane >> 2) & 3, lj = lane & 3;
    const int64_t warps = int64_t(gridDim.x) * kWarps;
    T* fields[3] = {u0, u1, u2};
    for (int64_t e = int64_t(blockIdx.x) * kWarps + (threadIdx.x >> 5); e < g.elements; e += warps) {
        const int64_t node = lane < 10 ? cells[e * 10 + lane] : 0;
        if (__any_sync(0xffffffffu, lane < 10 && (node < 0 || node >= g.nodes))) {
            if (lane == 0) flag(status, AFSI_FLAG_INDEX);
            continue;
        }
        const int64_t mine = __shfl_sync(0xffffffffu, node, lane < 30 ? lane / 3 : 0);
        if (lane < 30) s.coef[lane] = value[mine * 3 + lane % 3];
        Box bx;
        element_box(base, g, e, bx);
        const bool fits = box_fits<T>(bx, g);
        if (fits)
            for (int t = lane; t < 2 * BoxCap<T>::value; t += 32) (&s.copy[0][0])[t] = T(0);
        for (int64_t q0 = 0; q0 < g.nq; q0 += kChunk) {
            const int n = int(g.nq - q0 < kChunk ? g.nq - q0 : kChunk);
            __syncwarp();
            for (int q = lane; q < n; q += 32) {  // forces, lanes over points
                T F[3] = {T(0), T(0), T(0)};
#pragma unroll
                for (int a = 0; a < 10; ++a) {
                    const T nv = N[(q0 + q) * 10 + a];
#pragma unroll
                    for (int c = 0; c < 3; ++c) F[c] += nv * s.coef[a * 3 + c];
                }
                const T wq = W[e * g.nq + q0 + q];
#pragma unroll
                for (int c = 0; c < 3; ++c) s.f[c][q] = (F[c] * wq) / volume;
            }
            __syncwarp();
            T* copy = s.copy[half];
            // unrolled so that several points' table loads are in flight per warp
#pragma unroll 4
            for (int q = half; q < n; q += 2) {
                const int64_t row = g.offset + e * g.nq + q0 + q;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int64_t rx = table_row(g.total, row, c, 0), ry = table_row(g.total, row, c, 1),
                                  rz = table_row(g.total, row, c, 2);
                    const int gx = int(base[rx]), gy = int(base[ry]), gz = int(base[rz]);
                    const T w = (phi[rx * 4 + li] * phi[ry * 4 + lj]);
                    const T fq = s.f[c][q];
                    T v[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) v[k] = (w * phi[rz * 4 + k]) * fq;
                    if (fits) {
                        T* dst = copy + bx.off[c] +
                                 ((gx - bx.lo[c][0] + li) * bx.ext[c][1] + (gy - bx.lo[c][1] + lj)) * bx.ext[c][2] +
                                 (gz - bx.lo[c][2]);
#pragma unroll
                        for (int k = 0; k < 4; ++k) dst[k] += v[k];
                    } else if (point_inside(g, c, gx, gy, gz)) {
                        T* dst = fields[c] + face_index(g, c, gx + li, gy + lj, gz);
#pragma unroll
                        for (int k = 0; k < 4; ++k) atomicAdd(dst + k, v[k]);
                    } else if ((lane & 15) == 0) {
                        flag(status, AFSI_FLAG_INDEX);
                    }
                }
            }
        }
        __syncwarp();
        if (fits) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int ey = bx.ext[c][1], ez = bx.ext[c][2];
                const int n = bx.ext[c][0] * ey * ez;
                for (int t = lane; t < n; t += 32) {
                    const T v = s.copy[0][bx.off[c] + t] + s.copy[1][bx.off[c] + t];
                    if (v != T(0)) {
                        const int z = t % ez, r = t / ez;
                        atomicAdd(fields[c] + face_index(g, c, bx.lo[c][0] + r / ey, bx.lo[c][1] + r % ey,
                                                         bx.lo[c][2] + z), v);
                    }
                }
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------ gather

template <class T, bool Local>
__global__ void __launch_bounds__(kWarps * 32) p2_gather_kernel(const T* __restrict__ u0, const T* __restrict__ u1,
                                                                const T* __restrict__ u2,
                                                                const int64_t* __restrict__ cells,
                                                                const T* __restrict__ N, const T* __restrict__ W,
                                                                const int64_t* __restrict__ base,
                                                                const T* __restrict__ phi, T* __restrict__ out,
                                                                P2Dims g, int32_t* status) {
    __shared__ GatherStage<T> stage_all[kWarps];
    GatherStage<T>& s = stage_all[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31, half = lane >> 4, li = (lane >> 2) & 3, lj = lane & 3;
    const int64_t warps = int64_t(gridDim.x) * kWarps;
    const T* fields[3] = {u0, u1, u2};
    for (int64_t e = int64_t(blockIdx.x) * kWarps + (threadIdx.x >> 5); e < g.elements; e += warps) {
        const int64_t node = lane < 10 ? cells[e * 10 + lane] : 0;
        if (__any_sync(0xffffffffu, lane < 10 && (node < 0 || node >= g.nodes))) {
            if (lane == 0) flag(status, AFSI_FLAG_INDEX);
            continue;
        }
        Box bx;
        element_box(base, g, e, bx);
        const bool fits = box_fits<T>(bx, g);
        __syncwarp();
        if (fits) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int ey = bx.ext[c][1], ez = bx.ext[c][2];
                const int n = bx.ext[c][0] * ey * ez;
                for (int t = lane; t < n; t += 32) {
                    const int z = t % ez, r = t / ez;
                    s.patch[bx.off[c] + t] =
                        fields[c][face_index(g, c, bx.lo[c][0] + r / ey, bx.lo[c][1] + r % ey, bx.lo[c][2] + z)];
                }
            }
        }
        __syncwarp();
        // lanes 0..9 of each half accumulate node a = lane&15 over that half's points
        T acc[3] = {T(0), T(0), T(0)};
        const int a_node = lane & 15;
#pragma unroll 4
        for (int64_t qb = 0; qb < g.nq; qb += 2) {
            const int64_t q = qb + half;
            const bool active = q < g.nq;
            const int64_t row = g.offset + e * g.nq + (active ? q : 0);
            T U[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int64_t rx = table_row(g.total, row, c, 0), ry = table_row(g.total, row, c, 1),
                              rz = table_row(g.total, row, c, 2);
                const int gx = int(base[rx]), gy = int(base[ry]), gz = int(base[rz]);
                const T w = phi[rx * 4 + li] * phi[ry * 4 + lj];
                T sum = T(0);
                if (active) {
                    if (fits) {
                        const T* src = s.patch + bx.off[c] +
                                       ((gx - bx.lo[c][0] + li) * bx.ext[c][1] + (gy - bx.lo[c][1] + lj)) *
                                           bx.ext[c][2] +
                                       (gz - bx.lo[c][2]);
#pragma unroll
                        for (int k = 0; k < 4; ++k) sum = fma(src[k], phi[rz * 4 + k], sum);
                    } else if (point_inside(g, c, gx, gy, gz)) {
                        const T* src = fields[c] + face_index(g, c, gx + li, gy + lj, gz);
#pragma unroll
                        for (int k = 0; k < 4; ++k) sum = fma(src[k], phi[rz * 4 + k], sum);
                    } else if ((lane & 15) == 0) {
                        flag(status, AFSI_FLAG_INDEX);
                    }
                }
                sum *= w;
#pragma unroll
                for (int d = 8; d; d >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, d);
                U[c] = sum;
            }
            if (active && a_node < 10) {
                const T nw = N[q * 10 + a_node] * W[e * g.nq + q];
#pragma unroll
                for (int c = 0; c < 3; ++c) acc[c] = fma(nw, U[c], acc[c]);
            }
        }
        // combine the two halves: node a sums lane a and lane a+16
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 16);
        const int64_t nd = __shfl_sync(0xffffffffu, node, a_node < 10 ? a_node : 0);
        if (lane < 10) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                if (Local)
                    out[(e * 10 + lane) * 3 + c] = acc[c];
                else
                    atomicAdd(out + nd * 3 + c, acc[c]);
            }
        }
        __syncwarp();
    }
}

template <class T>
int32_t launch_spread_staged(const T* value, const int64_t* cells, const T* N, const T* W, const int64_t* base,
                             const T* phi, T* u0, T* u1, T* u2, const P2Dims& g, T volume, int32_t* status,
                             int blocks, cudaStream_t stream) {
    p2_spread_kernel<T><<<blocks, kWarps * 32, 0, stream>>>(value, cells, N, W, base, phi, u0, u1, u2, g, volume,
                                                            status);
    return launched("p2_spread");
}

template <class T, bool Local>
int32_t launch_gather_staged(const T* u0, const T* u1, const T* u2, const int64_t* cells, const T* N, const T* W,
                             const int64_t* base, const T* phi, T* out, const P2Dims& g, int32_t* status,
                             int blocks, cudaStream_t stream) {
    p2_gather_kernel<T, Local><<<blocks, kWarps * 32, 0, stream>>>(u0, u1, u2, cells, N, W, base, phi, out, g,
                                                                  status);
    return launched(Local ? "p2_gather_local" : "p2_gather_assemble");
}

// explicit instantiations used by transfer.cu
template int32_t launch_spread_staged<double>(const double*, const int64_t*, const double*, const double*,
                                              const int64_t*, const double*, double*, double*, double*, const P2Dims&,
                                              double, int32_t*, int, cudaStream_t);
template int32_t launch_spread_staged<float>(const float*, const int64_t*, const float*, const float*, const int64_t*,
                                             const float*, float*, float*, float*, const P2Dims&, float, int32_t*,
                                             int, cudaStream_t);
template int32_t launch_gather_staged<double, false>(const double*, const double*, const double*, const int64_t*,
                                                     const double*, const double*, const int64_t*, const double*,
                                                     double*, const P2Dims&, int32_t*, int, cudaStream_t);
template int32_t launch_gather_staged<double, true>(const double*, const double*, const double*, const int64_t*,
                                                    const double*, const double*, const int64_t*, const double*,
                                                    double*, const P2Dims&, int32_t*, int, cudaStream_t);
template int32_t launch_gather_staged<float, false>(const float*, const float*, const float*, const int64_t*,
                                                    const float*, const float*, const int64_t*, const float*, float*,
                                                    const P2Dims&, int32_t*, int, cudaStream_t);
template int32_t launch_gather_staged<float, true>(const float*, const float*, const float*, const int64_t*,
                                                   const float*, const float*, const int64_t*, const float*, float*,
                                                   const P2Dims&, int32_t*, int, cudaStream_t);

}  // namespace afsi
