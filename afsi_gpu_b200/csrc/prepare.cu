// Binning and IB_4 weight tables (compact 3D, reflected 2D, P2 quadrature).
//
// One thread per point: the point's coordinates are read once and all of its
// lattices and axes are produced from registers, so the only HBM traffic is
// the point read and the table write.  Arithmetic follows the reference
// operation order (library built with --fmad=false, IEEE division and sqrt),
// which makes the integer bases bit-exact and the weights equal to rounding.
#include "common.cuh"
#include "peskin.cuh"

namespace afsi {

template <class T>
__device__ __forceinline__ void store4(T* dst, const T w[4]);
template <>
__device__ __forceinline__ void store4<double>(double* dst, const double w[4]) {
    reinterpret_cast<double2*>(dst)[0] = make_double2(w[0], w[1]);
    reinterpret_cast<double2*>(dst)[1] = make_double2(w[2], w[3]);
}
template <>
__device__ __forceinline__ void store4<float>(float* dst, const float w[4]) {
    *reinterpret_cast<float4*>(dst) = make_float4(w[0], w[1], w[2], w[3]);
}

template <class T>
struct CompactParams {
    T origins[3][3];
    T spacing[3];
    T grid_origin[3];
    T limits[3];
    int lattices;
    int form;
};

template <class T>
__global__ void __launch_bounds__(256) compact_prepare_kernel(const T* __restrict__ points, int64_t count,
                                                              CompactParams<T> prm, int64_t* __restrict__ base,
                                                              T* __restrict__ phi, int32_t* status) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= count) return;
    T x[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) x[a] = points[p * 3 + a];
    bool valid = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const T s = (x[a] - prm.grid_origin[a]) / prm.spacing[a];
        valid = valid && isfinite(s) && s >= T(2) && s < prm.limits[a];
    }
    if (!valid) flag(status, AFSI_FLAG_SUPPORT);
    for (int l = 0; l < prm.lattices; ++l) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const T scaled = (x[a] - prm.origins[l][a]) / prm.spacing[a];
            const T lo = floor(scaled - T(1));
            const int64_t lower = static_cast<int64_t>(lo);
            const int64_t row = (l * count + p) * 3 + a;
            base[row] = lower;
            T w[4];
            if (prm.form == AFSI_PHI_RADICAL) {
                peskin_radical(scaled - T(lower) - T(1), w);
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k) w[k] = peskin_clamped(scaled - T(lower + k));
            }
            store4(phi + row * 4, w);
        }
    }
}

template <class T>
struct Prepare2dParams {
    T hx, hy;
    T xmin, xmax, ymin, ymax;
    int64_t ny;
};

// Reflected 4x4 stencils of u (faces (nx+1,ny)) and v (faces (nx,ny+1)),
// mac2d/transfer.py:61-81.  Offsets k=i*4+j, j (y) fastest.  One thread per
// point; a warp's 32 points own 32 consecutive rows of 16 ids and 16 weights
// per component, so each warp stages its rows in shared memory and writes
// them as one contiguous run (coalesced stores).
constexpr int kPrep2dThreads = 256;
constexpr int kPrep2dRow = 17;  // int64 words per staged row (16 taps + 1 pad against bank conflicts)

template <class T>
__global__ void __launch_bounds__(kPrep2dThreads) prepare2d_kernel(const T* __restrict__ points, int64_t count,
                                                                   Prepare2dParams<T> prm, int64_t* __restrict__ ids,
                                                                   T* __restrict__ weights, int32_t* status) {
    __shared__ int64_t s_rows[kPrep2dThreads / 32][32 * kPrep2dRow];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t p0 = int64_t(blockIdx.x) * blockDim.x + (threadIdx.x & ~31);
    if (p0 >= count) return;  // whole warp
    const int n_valid = count - p0 < 32 ? int(count - p0) : 32;
    const int64_t p = p0 + lane;
    const bool live = lane < n_valid;
    int64_t* row = s_rows[warp] + lane * kPrep2dRow;
    T* wrow = reinterpret_cast<T*>(s_rows[warp]) + lane * kPrep2dRow;
    T px = T(0), py = T(0);
    if (live) {
        px = points[p * 2];
        py = points[p * 2 + 1];
        const bool valid = isfinite(px) && isfinite(py) && px >= prm.xmin && px <= prm.xmax && py >= prm.ymin &&
                           py <= prm.ymax;
        if (!valid) flag(status, AFSI_FLAG_SUPPORT);
    }
    const int64_t ny = prm.ny;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        T wx[4], wy[4];
        int64_t by = 0;
        if (live) {
            const T ox = prm.hx * (c == 0 ? T(0) : T(.5));
            const T oy = prm.hy * (c == 1 ? T(0) : T(.5));
            const T sx = (px - ox) / prm.hx, sy = (py - oy) / prm.hy;
            const int64_t bx = static_cast<int64_t>(floor(sx - T(1)));
            by = static_cast<int64_t>(floor(sy - T(1)));
            const int64_t face_ny = ny + (c == 1);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                wx[k] = peskin_clamped(sx - T(bx + k));
                wy[k] = peskin_clamped(sy - T(by + k));
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int64_t y = by + j;
                    const int64_t r = c == 0 ? (y < 0 ? -y - 1 : (y >= ny ? 2 * ny - y - 1 : y))
                                             : (y < 0 ? -y : (y > ny ? 2 * ny - y : y));
                    row[i * 4 + j] = (bx + i) * face_ny + r;
                }
        }
        __syncwarp();
        const int64_t out0 = (c * count + p0) * 16;
        for (int k = lane; k < 16 * n_valid; k += 32) ids[out0 + k] = s_rows[warp][(k >> 4) * kPrep2dRow + (k & 15)];
        __syncwarp();
        if (live) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int64_t y = by + j;
                    const bool outside = c == 0 ? (y < 0 || y >= ny) : (y < 0 || y > ny);
                    const T w = wx[i] * wy[j];
                    wrow[i * 4 + j] = outside ? -w : w;
                }
        }
        __syncwarp();
        const T* sw = reinterpret_cast<const T*>(s_rows[warp]);
        for (int k = lane; k < 16 * n_valid; k += 32) weights[out0 + k] = sw[(k >> 4) * kPrep2dRow + (k & 15)];
        __syncwarp();
    }
}

template <class T>
struct P2Params {
    T origin[3], spacing[3], limits[3];
    int64_t nodes, elements, nq, total, offset;
};

// P2 positions + shared tables, mac/csrc/p2_transfer.cu:12-45.  One thread per
// quadrature point (element-major, q fastest); each axis has its own validity
// as in the reference, and an invalid axis is binned from scaled=0.
template <class T> struct Vec16;
template <> struct Vec16<double> { using type = double2; static constexpr int n = 2; };
template <> struct Vec16<float> { using type = float4; static constexpr int n = 4; };

constexpr int kPrepThreads = 128;

// The tables of a block's points are staged in shared memory and written out
// as two contiguous ranges per lattice (bases: 3 int64 per point, weights: 12
// values per point) with coalesced stores, instead of 18 scattered stores per
// point.  A point with a node id out of range flags AFSI_FLAG_INDEX and gets
// zero tables.  Positions, bases and weights are computed in T; the weights
// are stored in TW (T, or float beside FP64 positions in the precision form).
template <class T, int NPC, class TW = T>
__global__ void __launch_bounds__(kPrepThreads) fe_prepare_kernel(const T* __restrict__ x,
                                                                  const int64_t* __restrict__ cells,
                                                                  const T* __restrict__ N, P2Params<T> prm,
                                                                  int64_t* __restrict__ base, TW* __restrict__ phi,
                                                                  int32_t* status) {
    __shared__ __align__(16) TW s_phi[2][kPrepThreads * 12];
    __shared__ int64_t s_base[2][kPrepThreads * 3];
    const int64_t first = int64_t(blockIdx.x) * kPrepThreads;
    const int64_t points = prm.elements * prm.nq;
    const int n = int(points - first < kPrepThreads ? points - first : kPrepThreads);
    const int t = threadIdx.x;
    if (t < n) {
        const int64_t p = first + t;
        const int64_t e = p / prm.nq, q = p % prm.nq;
        int64_t node[NPC];
        bool ok = true;
#pragma unroll
        for (int a = 0; a < NPC; ++a) {
            node[a] = cells[e * NPC + a];
            ok = ok && node[a] >= 0 && node[a] < prm.nodes;
        }
        T pos[3] = {T(0), T(0), T(0)};
        if (ok) {
#pragma unroll
            for (int a = 0; a < NPC; ++a) {
                const T nv = N[q * NPC + a];
#pragma unroll
                for (int d = 0; d < 3; ++d) pos[d] += nv * x[node[a] * 3 + d];
            }
        } else {
            flag(status, AFSI_FLAG_INDEX);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const T physical = (pos[a] - prm.origin[a]) / prm.spacing[a];
            const bool valid = ok && isfinite(physical) && physical >= T(2) && physical < prm.limits[a];
            if (ok && !valid) flag(status, AFSI_FLAG_SUPPORT);
#pragma unroll
            for (int lattice = 0; lattice < 2; ++lattice) {
                const T start = lattice ? prm.origin[a] + T(.5) * prm.spacing[a] : prm.origin[a];
                const T scaled = valid ? (pos[a] - start) / prm.spacing[a] : T(0);
                const int64_t lower = static_cast<int64_t>(floor(scaled - T(1)));
                T w[4];
                peskin_radical(scaled - T(lower) - T(1), w);
                s_base[lattice][t * 3 + a] = ok ? lower : 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) s_phi[lattice][(t * 3 + a) * 4 + k] = ok ? TW(w[k]) : TW(0);
            }
        }
    }
    __syncthreads();
    using V = typename Vec16<TW>::type;
    constexpr int per = Vec16<TW>::n;
#pragma unroll
    for (int lattice = 0; lattice < 2; ++lattice) {
        const int64_t row = (lattice * prm.total + prm.offset + first) * 3;
        for (int i = t; i < n * 3; i += kPrepThreads) base[row + i] = s_base[lattice][i];
        // weights start at row*4 values: a multiple of 12, so 16-byte aligned
        V* dst = reinterpret_cast<V*>(phi + row * 4);
        const V* src = reinterpret_cast<const V*>(s_phi[lattice]);
        for (int i = t; i < n * 12 / per; i += kPrepThreads) dst[i] = src[i];
    }
}

// Adaptive quadrature order of each element (mac/adaptive_transfer.py:167-187):
// ceil(density * D / dx), at least min_order.  P2 (NPC = 10): D is the
// diameter of the element's ten Bernstein control points (the four corners
// and, per edge (i,j) of the tetrahedron, 2 x_mid - (x_i + x_j)/2).  P1
// (NPC = 4): D is the longest edge, the diameter of the four corners.  D is
// the square root of the largest squared pair distance ((dx^2+dy^2)+dz^2); the
// square root is monotone, so this equals the maximum of the pair norms.
// The launch also counts the elements whose order differs from `last`, the
// largest order, and a histogram of orders < bins, all into `summary`
// (changed, max, flags, hist[bins]).  Nonfinite positions set
// AFSI_FLAG_SUPPORT, node ids outside [0, nodes) AFSI_FLAG_INDEX; those
// elements get order 0.
// ends of tetrahedron edge k: (0,1) (0,2) (0,3) (1,2) (1,3) (2,3)
__host__ __device__ constexpr int edge_from(int k) { return k < 3 ? 0 : k < 5 ? 1 : 2; }
__host__ __device__ constexpr int edge_to(int k) { return k < 3 ? k + 1 : k < 5 ? k - 1 : 3; }
constexpr int kOrderBins = 64;

template <class T, int NPC>
__global__ void __launch_bounds__(256) fe_orders_kernel(const T* __restrict__ x, const int64_t* __restrict__ cells,
                                                        int64_t elements, int64_t nodes, T dx, T density,
                                                        int64_t min_order, int64_t* __restrict__ orders,
                                                        const int64_t* __restrict__ last, int32_t* summary,
                                                        int bins) {
    __shared__ int hist[kOrderBins];
    for (int t = threadIdx.x; t < kOrderBins; t += blockDim.x) hist[t] = 0;
    __syncthreads();
    const int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    int64_t order = 0;
    bool changed = false;
    int32_t flags = 0;
    if (e < elements) {
        int64_t node[NPC];
        bool ok = true;
#pragma unroll
        for (int a = 0; a < NPC; ++a) {
            node[a] = cells[e * NPC + a];
            ok = ok && node[a] >= 0 && node[a] < nodes;
        }
        if (!ok) {
            flags |= AFSI_FLAG_INDEX;
        } else {
            constexpr int H = NPC == 10 ? 10 : 4;  // P2: corners + edge controls; P1: corners
            T hull[H][3];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int d = 0; d < 3; ++d) hull[a][d] = x[node[a] * 3 + d];
#pragma unroll
            for (int k = 0; k < H - 4; ++k)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    hull[4 + k][d] = T(2) * x[node[4 + k] * 3 + d] -
                                     T(.5) * (hull[edge_from(k)][d] + hull[edge_to(k)][d]);
            T best = T(0);
            bool finite = true;
#pragma unroll
            for (int a = 0; a < H; ++a)
#pragma unroll
                for (int b = a + 1; b < H; ++b) {
                    const T d0 = hull[a][0] - hull[b][0], d1 = hull[a][1] - hull[b][1], d2 = hull[a][2] - hull[b][2];
                    const T s = (d0 * d0 + d1 * d1) + d2 * d2;
                    finite = finite && isfinite(s);
                    best = s > best ? s : best;
                }
            const T v = ceil(density * sqrt(best) / dx);
            if (!finite || !isfinite(v)) {
                flags |= AFSI_FLAG_SUPPORT;
            } else {
                const T capped = v < T(1e15) ? v : T(1e15);
                order = int64_t(capped);
                if (order < min_order) order = min_order;
            }
        }
        orders[e] = order;
        changed = last == nullptr || last[e] != order;
        if (order < bins) atomicAdd(&hist[order], 1);
    }
    const int lane = threadIdx.x & 31;
    const unsigned moved = __ballot_sync(0xffffffffu, changed);
    int32_t top = int32_t(order < INT32_MAX ? order : INT32_MAX);
#pragma unroll
    for (int d = 16; d; d >>= 1) {
        top = max(top, __shfl_xor_sync(0xffffffffu, top, d));
        flags |= __shfl_xor_sync(0xffffffffu, flags, d);
    }
    if (lane == 0) {
        if (moved) atomicAdd(&summary[0], __popc(moved));
        if (top > 0) atomicMax(&summary[1], top);
        if (flags) atomicOr(&summary[2], flags);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < bins; t += blockDim.x)
        if (hist[t]) atomicAdd(&summary[3 + t], hist[t]);
}

}  // namespace afsi

using namespace afsi;

extern "C" int32_t afsi_b200_compact_prepare(const void* points, int64_t count, int32_t lattices,
                                             const double* origins, const double* spacing,
                                             const double* grid_origin, const int64_t* shape,
                                             int32_t phi_form, int64_t* base, void* phi, int32_t* status,
                                             int32_t dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(count >= 0, "negative point count");
    AFSI_REQUIRE(lattices >= 1 && lattices <= 3, "lattices must be 1..3");
    AFSI_REQUIRE(origins && spacing && grid_origin && shape, "null host parameter array");
    AFSI_REQUIRE(phi_form == AFSI_PHI_CLAMPED || phi_form == AFSI_PHI_RADICAL, "unknown phi form");
    if (count == 0) return AFSI_OK;
    AFSI_REQUIRE(points && base && phi, "null device pointer");
    AFSI_DISPATCH(dtype, {
        CompactParams<T> prm;
        for (int l = 0; l < 3; ++l)
            for (int a = 0; a < 3; ++a) prm.origins[l][a] = T(l < lattices ? origins[l * 3 + a] : 0.0);
        for (int a = 0; a < 3; ++a) {
            AFSI_REQUIRE(spacing[a] > 0 && shape[a] > 0, "invalid grid spacing/shape");
            prm.spacing[a] = T(spacing[a]);
            prm.grid_origin[a] = T(grid_origin[a]);
            prm.limits[a] = T(shape[a]) - T(2);
        }
        prm.lattices = lattices;
        prm.form = phi_form;
        compact_prepare_kernel<T><<<blocks_for(count, 256), 256, 0, stream>>>(
            static_cast<const T*>(points), count, prm, base, static_cast<T*>(phi), status);
    });
    return launched("compact_prepare");
}

extern "C" int32_t afsi_b200_indexed_prepare2d(const void* points, int64_t count, int64_t nx, int64_t ny,
                                               double hx, double hy, double lx, double ly, int64_t* ids,
                                               void* weights, int32_t* status, int32_t dtype,
                                               afsi_stream_t stream) {
    AFSI_REQUIRE(count >= 0 && nx > 0 && ny > 0 && hx > 0 && hy > 0, "invalid 2D grid or point count");
    if (count == 0) return AFSI_OK;
    AFSI_REQUIRE(points && ids && weights, "null device pointer");
    AFSI_DISPATCH(dtype, {
        Prepare2dParams<T> prm;
        prm.hx = T(hx);
        prm.hy = T(hy);
        prm.xmin = T(2 * hx);
        prm.xmax = T(lx - 2 * hx);
        prm.ymin = T(-hy);
        prm.ymax = T(ly + hy);
        prm.ny = ny;
        prepare2d_kernel<T><<<blocks_for(count, kPrep2dThreads), kPrep2dThreads, 0, stream>>>(
            static_cast<const T*>(points), count, prm, ids, static_cast<T*>(weights), status);
    });
    return launched("indexed_prepare2d");
}

template <int NPC>
static int32_t fe_prepare(const void* x, int64_t nodes, const int64_t* cells, int64_t elements, const void* N,
                          int64_t nq, const double* origin, const double* spacing, const double* limits,
                          int64_t* base, void* phi, int64_t total, int64_t offset, int32_t* status, int32_t dtype,
                          afsi_stream_t stream, int32_t weight_dtype = -1) {
    if (weight_dtype < 0) weight_dtype = dtype;
    AFSI_REQUIRE(weight_dtype == dtype || (dtype == AFSI_F64 && weight_dtype == AFSI_F32),
                 "weights may be stored in FP32 beside FP64 positions only");
    AFSI_REQUIRE(elements >= 0 && nq > 0 && nodes >= 0, "invalid IB group sizes");
    AFSI_REQUIRE(offset >= 0 && offset <= total && elements * nq <= total - offset, "IB group exceeds table bounds");
    AFSI_REQUIRE(origin && spacing && limits, "null host parameter array");
    if (elements == 0) return AFSI_OK;
    AFSI_REQUIRE(x && cells && N && base && phi, "null device pointer");
    AFSI_REQUIRE(reinterpret_cast<uintptr_t>(phi) % 16 == 0, "IB weight table must be 16-byte aligned");
    AFSI_DISPATCH(dtype, {
        P2Params<T> prm;
        for (int a = 0; a < 3; ++a) {
            prm.origin[a] = T(origin[a]);
            prm.spacing[a] = T(spacing[a]);
            prm.limits[a] = T(limits[a]);
        }
        prm.nodes = nodes;
        prm.elements = elements;
        prm.nq = nq;
        prm.total = total;
        prm.offset = offset;
        if (weight_dtype != dtype) {
            if constexpr (sizeof(T) == 8)
                fe_prepare_kernel<T, NPC, float><<<blocks_for(elements * nq, kPrepThreads), kPrepThreads, 0, stream>>>(
                    static_cast<const T*>(x), cells, static_cast<const T*>(N), prm, base, static_cast<float*>(phi),
                    status);
        } else {
            fe_prepare_kernel<T, NPC><<<blocks_for(elements * nq, kPrepThreads), kPrepThreads, 0, stream>>>(
                static_cast<const T*>(x), cells, static_cast<const T*>(N), prm, base, static_cast<T*>(phi), status);
        }
    });
    return launched(NPC == 10 ? "p2_prepare" : "p1_prepare");
}

extern "C" int32_t afsi_b200_p2_prepare(const void* x, int64_t nodes, const int64_t* cells, int64_t elements,
                                        const void* N, int64_t nq, const double* origin, const double* spacing,
                                        const double* limits, int64_t* base, void* phi, int64_t total,
                                        int64_t offset, int32_t* status, int32_t dtype, afsi_stream_t stream) {
    return fe_prepare<10>(x, nodes, cells, elements, N, nq, origin, spacing, limits, base, phi, total, offset, status,
                          dtype, stream);
}

extern "C" int32_t afsi_b200_fe_prepare_mixed(int32_t nodes_per_cell, const double* x, int64_t nodes,
                                              const int64_t* cells, int64_t elements, const double* N, int64_t nq,
                                              const double* origin, const double* spacing, const double* limits,
                                              int64_t* base, void* phi, int64_t total, int64_t offset,
                                              int32_t* status, int32_t weight_dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(nodes_per_cell == 10 || nodes_per_cell == 4, "nodes per cell must be 10 (P2) or 4 (P1)");
    if (nodes_per_cell == 10)
        return fe_prepare<10>(x, nodes, cells, elements, N, nq, origin, spacing, limits, base, phi, total, offset,
                              status, AFSI_F64, stream, weight_dtype);
    return fe_prepare<4>(x, nodes, cells, elements, N, nq, origin, spacing, limits, base, phi, total, offset, status,
                         AFSI_F64, stream, weight_dtype);
}

extern "C" int32_t afsi_b200_p1_prepare(const void* x, int64_t nodes, const int64_t* cells, int64_t elements,
                                        const void* N, int64_t nq, const double* origin, const double* spacing,
                                        const double* limits, int64_t* base, void* phi, int64_t total,
                                        int64_t offset, int32_t* status, int32_t dtype, afsi_stream_t stream) {
    return fe_prepare<4>(x, nodes, cells, elements, N, nq, origin, spacing, limits, base, phi, total, offset, status,
                         dtype, stream);
}

template <int NPC>
static int32_t fe_orders(const void* x, int64_t nodes, const int64_t* cells, int64_t elements, double dx,
                         double density, int64_t min_order, int64_t* orders, const int64_t* last_orders,
                         int32_t* summary, int32_t bins, int32_t dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(elements >= 0 && nodes >= 0, "invalid element or node count");
    AFSI_REQUIRE(bins >= 1 && bins <= kOrderBins, "order histogram needs 1..%d bins, got %d", kOrderBins, bins);
    AFSI_REQUIRE(dx > 0 && density > 0, "element orders need a positive spacing and point density");
    AFSI_REQUIRE(summary, "null summary pointer");
    if (cudaMemsetAsync(summary, 0, sizeof(int32_t) * (3 + bins), stream) != cudaSuccess)
        return fail(AFSI_ERR_CUDA, "summary clear failed");
    if (elements == 0) return AFSI_OK;
    AFSI_REQUIRE(x && cells && orders, "null device pointer");
    AFSI_DISPATCH(dtype, {
        fe_orders_kernel<T, NPC><<<blocks_for(elements, 256), 256, 0, stream>>>(
            static_cast<const T*>(x), cells, elements, nodes, T(dx), T(density), min_order, orders, last_orders,
            summary, bins);
    });
    return launched(NPC == 10 ? "p2_orders" : "p1_orders");
}

extern "C" int32_t afsi_b200_p2_orders(const void* x, int64_t nodes, const int64_t* cells, int64_t elements,
                                       double dx, double density, int64_t min_order, int64_t* orders,
                                       const int64_t* last_orders, int32_t* summary, int32_t bins, int32_t dtype,
                                       afsi_stream_t stream) {
    return fe_orders<10>(x, nodes, cells, elements, dx, density, min_order, orders, last_orders, summary, bins, dtype,
                         stream);
}

extern "C" int32_t afsi_b200_p1_orders(const void* x, int64_t nodes, const int64_t* cells, int64_t elements,
                                       double dx, double density, int64_t min_order, int64_t* orders,
                                       const int64_t* last_orders, int32_t* summary, int32_t bins, int32_t dtype,
                                       afsi_stream_t stream) {
    return fe_orders<4>(x, nodes, cells, elements, dx, density, min_order, orders, last_orders, summary, bins, dtype,
                        stream);
}
