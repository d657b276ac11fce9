// Batched 2D IB transfers: many independent channel instances of different
// grid and point counts in one launch per operation (the batching form).
//
// The batch keeps every instance's points back to back and every instance's
// u and v face arrays back to back; an instance table gives each instance's
// grid, first point, point count and first u / v face.  Stencil ids are
// written as batch-global face ids, so the gather needs no table at all, and
// the spread looks its point's instance up (binary search over the first
// points, the table staged in shared memory) only for the cell area.
//
// Per instance the arithmetic is that of the single-instance kernels, which
// follow mac2d/transfer.py:61-81 (reflected 4x4 stencils) and :108-127
// (spread divided by the cell area, gather): positions, bases and weights are
// formed in FP64 and the weights stored in the transfer type TW (float in
// the precision form), so ids equal the single-instance FP64 ids exactly.
#include <algorithm>
#include "common.cuh"
#include "peskin.cuh"

namespace afsi {

constexpr int kMaxBatch = 1024;  // instances per batch (table staged in shared memory)

struct BatchTable {
    const afsi_batch2d_instance* inst;
    int count;
};

// Index of the instance owning point p (the last instance whose first point
// is <= p); s_first holds the first points in order.
__device__ __forceinline__ int owner(const int64_t* s_first, int count, int64_t p) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_first[mid] <= p)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void stage_firsts(const BatchTable& t, int64_t* s_first) {
    for (int i = threadIdx.x; i < t.count; i += blockDim.x) s_first[i] = t.inst[i].point_offset;
    __syncthreads();
}

constexpr int kPrepThreads = 256;
constexpr int kStageRow = 17;  // int64 words per staged point row (16 taps + 1 pad against bank conflicts)

// One thread per point.  A warp's 32 points own 32 consecutive rows of 16 ids
// (and 16 weights) per component, so each warp stages its rows in shared
// memory and writes them out as one contiguous run (coalesced stores).
template <class TW>
__global__ void __launch_bounds__(kPrepThreads) batch_prepare2d_kernel(const double* __restrict__ points,
                                                                       int64_t total, BatchTable t,
                                                                       int64_t* __restrict__ ids,
                                                                       TW* __restrict__ weights, int32_t* status) {
    __shared__ int64_t s_first[kMaxBatch];
    __shared__ int64_t s_rows[kPrepThreads / 32][32 * kStageRow];
    stage_firsts(t, s_first);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t p0 = int64_t(blockIdx.x) * blockDim.x + (threadIdx.x & ~31);
    if (p0 >= total) return;  // whole warp
    const int n_valid = total - p0 < 32 ? int(total - p0) : 32;
    const int64_t p = p0 + lane;
    const bool live = lane < n_valid;
    int64_t* row = s_rows[warp] + lane * kStageRow;
    TW* wrow = reinterpret_cast<TW*>(s_rows[warp]) + lane * kStageRow;
    afsi_batch2d_instance I{};
    double px = 0.0, py = 0.0;
    if (live) {
        I = t.inst[owner(s_first, t.count, p)];
        px = points[p * 2];
        py = points[p * 2 + 1];
        const bool valid = p < I.point_offset + I.point_count && isfinite(px) && isfinite(py) &&
                           px >= 2 * I.hx && px <= I.lx - 2 * I.hx && py >= -I.hy && py <= I.ly + I.hy;
        if (!valid) flag(status, AFSI_FLAG_SUPPORT);
    }
    const double hx = I.hx, hy = I.hy;
    const int64_t ny = I.ny;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        double wx[4], wy[4];
        int64_t bx = 0, by = 0;
        if (live) {
            const double ox = hx * (c == 0 ? 0.0 : .5);
            const double oy = hy * (c == 1 ? 0.0 : .5);
            const double sx = (px - ox) / hx, sy = (py - oy) / hy;
            bx = static_cast<int64_t>(floor(sx - 1.0));
            by = static_cast<int64_t>(floor(sy - 1.0));
            const int64_t face_ny = ny + (c == 1);
            const int64_t face_base = c == 0 ? I.u_offset : I.v_offset;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                wx[k] = peskin_clamped(sx - double(bx + k));
                wy[k] = peskin_clamped(sy - double(by + k));
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int64_t y = by + j;
                    const int64_t r = c == 0 ? (y < 0 ? -y - 1 : (y >= ny ? 2 * ny - y - 1 : y))
                                             : (y < 0 ? -y : (y > ny ? 2 * ny - y : y));
                    row[i * 4 + j] = face_base + (bx + i) * face_ny + r;
                }
        }
        __syncwarp();
        const int64_t out0 = (c * total + p0) * 16;
        for (int k = lane; k < 16 * n_valid; k += 32) ids[out0 + k] = s_rows[warp][(k >> 4) * kStageRow + (k & 15)];
        __syncwarp();
        if (live) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int64_t y = by + j;
                    const bool outside = c == 0 ? (y < 0 || y >= ny) : (y < 0 || y > ny);
                    const double w = wx[i] * wy[j];
                    wrow[i * 4 + j] = TW(outside ? -w : w);
                }
        }
        __syncwarp();
        const TW* sw = reinterpret_cast<const TW*>(s_rows[warp]);
        for (int k = lane; k < 16 * n_valid; k += 32) weights[out0 + k] = sw[(k >> 4) * kStageRow + (k & 15)];
        __syncwarp();
    }
}

// Transfers: 16 lanes per (point, component) task, each lane one stencil
// tap.  A 16-lane group takes kTaskUnroll consecutive tasks per iteration of
// a grid-stride loop and issues all their loads before it uses them, so a
// thread keeps several loads in flight; the grid is capped at a few blocks
// per SM.
constexpr int kTaskUnroll = 4;
constexpr int kTransferThreads = 256;

// u_c[id] += F_c * w / (hx hy) of the point's instance.
template <class T>
__global__ void __launch_bounds__(kTransferThreads) batch_spread2d_kernel(const T* __restrict__ force,
                                                                          const int64_t* __restrict__ ids,
                                                                          const T* __restrict__ w, int64_t total,
                                                                          BatchTable t, T* __restrict__ u,
                                                                          T* __restrict__ v, int64_t nu, int64_t nv,
                                                                          int32_t* status) {
    __shared__ int64_t s_first[kMaxBatch];
    stage_firsts(t, s_first);
    const int sub = threadIdx.x % 16;
    const int64_t tasks = total * 2;
    const int64_t groups = (int64_t(gridDim.x) * blockDim.x) / 16;
    for (int64_t g = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 16; g * kTaskUnroll < tasks; g += groups) {
        int64_t j[kTaskUnroll];
        T fw[kTaskUnroll];
#pragma unroll
        for (int k = 0; k < kTaskUnroll; ++k) {
            const int64_t task = g * kTaskUnroll + k;
            if (task < tasks) {
                const int64_t p = task >> 1;
                const int c = int(task & 1);
                const int64_t row = (c * total + p) * 16 + sub;
                j[k] = ids[row];
                fw[k] = force[p * 2 + c] * w[row];
            }
        }
        int64_t owner_p = -1;
        int inst = 0;
#pragma unroll
        for (int k = 0; k < kTaskUnroll; ++k) {
            const int64_t task = g * kTaskUnroll + k;
            if (task >= tasks) break;
            const int64_t p = task >> 1;
            const int c = int(task & 1);
            if (p != owner_p) {  // both components of a point share the lookup
                inst = owner(s_first, t.count, p);
                owner_p = p;
            }
            const afsi_batch2d_instance& I = t.inst[inst];
            const T volume = T(I.hx * I.hy);
            const int64_t lo = c == 0 ? I.u_offset : I.v_offset;
            const int64_t hi = lo + (c == 0 ? (I.nx + 1) * I.ny : I.nx * (I.ny + 1));
            if (j[k] < lo || j[k] >= hi || j[k] >= (c == 0 ? nu : nv)) {
                flag(status, AFSI_FLAG_INDEX);
                continue;
            }
            atomicAdd((c == 0 ? u : v) + j[k], fw[k] / volume);
        }
    }
}

// U_c[p] = sum of u_c[id] * w (ids are batch-global, so no instance lookup);
// the 16 taps summed by the shuffle tree of the single-instance gather.
template <class T>
__global__ void __launch_bounds__(kTransferThreads) batch_gather2d_kernel(const T* __restrict__ u,
                                                                          const T* __restrict__ v,
                                                                          const int64_t* __restrict__ ids,
                                                                          const T* __restrict__ w, int64_t total,
                                                                          int64_t nu, int64_t nv,
                                                                          T* __restrict__ out, int32_t* status) {
    const int sub = threadIdx.x % 16;
    const int64_t tasks = total * 2;
    const int64_t groups = (int64_t(gridDim.x) * blockDim.x) / 16;
    // uniform trip count per warp (both half-warps run every shuffle)
    const int64_t first = (int64_t(blockIdx.x) * blockDim.x + (threadIdx.x & ~31)) / 16;
    for (int64_t g0 = first; g0 * kTaskUnroll < tasks; g0 += groups) {
        const int64_t g = g0 + (threadIdx.x & 16 ? 1 : 0);
        int64_t j[kTaskUnroll];
        T wt[kTaskUnroll];
#pragma unroll
        for (int k = 0; k < kTaskUnroll; ++k) {
            const int64_t task = g * kTaskUnroll + k;
            j[k] = -1;
            wt[k] = T(0);
            if (task < tasks) {
                const int64_t row = ((task & 1) * total + (task >> 1)) * 16 + sub;
                j[k] = ids[row];
                wt[k] = w[row];
            }
        }
        T sum[kTaskUnroll];
#pragma unroll
        for (int k = 0; k < kTaskUnroll; ++k) {
            const int64_t task = g * kTaskUnroll + k;
            sum[k] = T(0);
            if (task < tasks) {
                const int c = int(task & 1);
                if (j[k] < 0 || j[k] >= (c == 0 ? nu : nv))
                    flag(status, AFSI_FLAG_INDEX);
                else
                    sum[k] = (c == 0 ? u : v)[j[k]] * wt[k];
            }
        }
#pragma unroll
        for (int k = 0; k < kTaskUnroll; ++k) {
#pragma unroll
            for (int d = 8; d; d >>= 1) sum[k] += __shfl_down_sync(0xffffffffu, sum[k], d, 16);
            const int64_t task = g * kTaskUnroll + k;
            if (task < tasks && sub == 0) out[(task >> 1) * 2 + (task & 1)] = sum[k];
        }
    }
}

}  // namespace afsi

using namespace afsi;

namespace {

// Blocks for a transfer over `total` points: one 16-lane group per
// kTaskUnroll tasks, at most 8 blocks per SM (grid-stride beyond).
unsigned transfer_blocks(int64_t total) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    const int64_t groups = (total * 2 + kTaskUnroll - 1) / kTaskUnroll;
    const int64_t blocks = (groups * 16 + kTransferThreads - 1) / kTransferThreads;
    return unsigned(std::max<int64_t>(1, std::min<int64_t>(blocks, int64_t(sms) * 8)));
}

int32_t check_table(const afsi_batch2d_instance* inst, int32_t count) {
    AFSI_REQUIRE(inst && count >= 1 && count <= kMaxBatch, "batch needs 1..%d instances and a device table",
                 kMaxBatch);
    return AFSI_OK;
}

}  // namespace

extern "C" int32_t afsi_b200_batch2d_prepare(const double* points, int64_t total,
                                             const afsi_batch2d_instance* instances, int32_t count, int64_t* ids,
                                             void* weights, int32_t* status, int32_t weight_dtype,
                                             afsi_stream_t stream) {
    int32_t rc = check_table(instances, count);
    if (rc) return rc;
    AFSI_REQUIRE(total >= 0, "negative point count");
    if (total == 0) return AFSI_OK;
    AFSI_REQUIRE(points && ids && weights, "null device pointer");
    const BatchTable t{instances, count};
    AFSI_DISPATCH(weight_dtype, {
        batch_prepare2d_kernel<T><<<blocks_for(total, kPrepThreads), kPrepThreads, 0, stream>>>(points, total, t, ids,
                                                                              static_cast<T*>(weights), status);
    });
    return launched("batch2d prepare");
}

extern "C" int32_t afsi_b200_batch2d_spread(const void* force, const int64_t* ids, const void* weights, int64_t total,
                                            const afsi_batch2d_instance* instances, int32_t count, void* u, void* v,
                                            int64_t nu, int64_t nv, int32_t* status, int32_t dtype,
                                            afsi_stream_t stream) {
    int32_t rc = check_table(instances, count);
    if (rc) return rc;
    AFSI_REQUIRE(total >= 0 && nu > 0 && nv > 0, "invalid batch sizes");
    if (total == 0) return AFSI_OK;
    AFSI_REQUIRE(force && ids && weights && u && v, "null device pointer");
    const BatchTable t{instances, count};
    AFSI_DISPATCH(dtype, {
        batch_spread2d_kernel<T><<<transfer_blocks(total), kTransferThreads, 0, stream>>>(
            static_cast<const T*>(force), ids, static_cast<const T*>(weights), total, t, static_cast<T*>(u),
            static_cast<T*>(v), nu, nv, status);
    });
    return launched("batch2d spread");
}

extern "C" int32_t afsi_b200_batch2d_gather(const void* u, const void* v, int64_t nu, int64_t nv, const int64_t* ids,
                                            const void* weights, int64_t total, void* out, int32_t* status,
                                            int32_t dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(total >= 0 && nu > 0 && nv > 0, "invalid batch sizes");
    if (total == 0) return AFSI_OK;
    AFSI_REQUIRE(u && v && ids && weights && out, "null device pointer");
    AFSI_DISPATCH(dtype, {
        batch_gather2d_kernel<T><<<transfer_blocks(total), kTransferThreads, 0, stream>>>(
            static_cast<const T*>(u), static_cast<const T*>(v), ids, static_cast<const T*>(weights), total, nu, nv,
            static_cast<T*>(out), status);
    });
    return launched("batch2d gather");
}
