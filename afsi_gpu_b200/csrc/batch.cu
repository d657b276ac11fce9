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

template <class TW>
__global__ void __launch_bounds__(256) batch_prepare2d_kernel(const double* __restrict__ points, int64_t total,
                                                              BatchTable t, int64_t* __restrict__ ids,
                                                              TW* __restrict__ weights, int32_t* status) {
    __shared__ int64_t s_first[kMaxBatch];
    stage_firsts(t, s_first);
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= total) return;
    const afsi_batch2d_instance I = t.inst[owner(s_first, t.count, p)];
    const double px = points[p * 2], py = points[p * 2 + 1];
    const double hx = I.hx, hy = I.hy;
    const bool valid = p < I.point_offset + I.point_count && isfinite(px) && isfinite(py) && px >= 2 * hx &&
                       px <= I.lx - 2 * hx && py >= -hy && py <= I.ly + hy;
    if (!valid) flag(status, AFSI_FLAG_SUPPORT);
    const int64_t ny = I.ny;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const double ox = hx * (c == 0 ? 0.0 : .5);
        const double oy = hy * (c == 1 ? 0.0 : .5);
        const double sx = (px - ox) / hx, sy = (py - oy) / hy;
        const int64_t bx = static_cast<int64_t>(floor(sx - 1.0));
        const int64_t by = static_cast<int64_t>(floor(sy - 1.0));
        const int64_t face_ny = ny + (c == 1);
        const int64_t face_base = c == 0 ? I.u_offset : I.v_offset;
        double wx[4], wy[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            wx[k] = peskin_clamped(sx - double(bx + k));
            wy[k] = peskin_clamped(sy - double(by + k));
        }
        int64_t* out_ids = ids + (c * total + p) * 16;
        TW* out_w = weights + (c * total + p) * 16;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t y = by + j;
                bool outside;
                int64_t r;
                if (c == 0) {
                    outside = y < 0 || y >= ny;
                    r = y < 0 ? -y - 1 : (y >= ny ? 2 * ny - y - 1 : y);
                } else {
                    outside = y < 0 || y > ny;
                    r = y < 0 ? -y : (y > ny ? 2 * ny - y : y);
                }
                const double w = wx[i] * wy[j];
                out_ids[i * 4 + j] = face_base + (bx + i) * face_ny + r;
                out_w[i * 4 + j] = TW(outside ? -w : w);
            }
        }
    }
}

// 16 lanes per (point, component): u_c[id] += F_c * w / (hx hy) of the point's instance.
template <class T>
__global__ void __launch_bounds__(256) batch_spread2d_kernel(const T* __restrict__ force, const int64_t* __restrict__ ids,
                                                             const T* __restrict__ w, int64_t total, BatchTable t,
                                                             T* __restrict__ u, T* __restrict__ v, int64_t nu,
                                                             int64_t nv, int32_t* status) {
    __shared__ int64_t s_first[kMaxBatch];
    stage_firsts(t, s_first);
    const int64_t task = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 16;
    const int sub = threadIdx.x % 16;
    if (task >= total * 2) return;
    const int64_t p = task >> 1;
    const int c = int(task & 1);
    const afsi_batch2d_instance& I = t.inst[owner(s_first, t.count, p)];
    const T volume = T(I.hx * I.hy);
    const int64_t j = ids[(c * total + p) * 16 + sub];
    T* out = c == 0 ? u : v;
    const int64_t lo = c == 0 ? I.u_offset : I.v_offset;
    const int64_t hi = lo + (c == 0 ? (I.nx + 1) * I.ny : I.nx * (I.ny + 1));
    if (j < lo || j >= hi || j >= (c == 0 ? nu : nv)) {
        flag(status, AFSI_FLAG_INDEX);
        return;
    }
    atomicAdd(out + j, (force[p * 2 + c] * w[(c * total + p) * 16 + sub]) / volume);
}

// 16 lanes per (point, component): U_c[p] = sum of u_c[id] * w (ids are
// batch-global, so no instance lookup); xor-free shuffle tree as in the
// single-instance gather.
template <class T>
__global__ void __launch_bounds__(256) batch_gather2d_kernel(const T* __restrict__ u, const T* __restrict__ v,
                                                             const int64_t* __restrict__ ids, const T* __restrict__ w,
                                                             int64_t total, int64_t nu, int64_t nv,
                                                             T* __restrict__ out, int32_t* status) {
    const int64_t task = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 16;
    const int sub = threadIdx.x % 16;
    const bool active = task < total * 2;
    const int64_t p = active ? task >> 1 : 0;
    const int c = int(task & 1);
    T sum = T(0);
    if (active) {
        const int64_t j = ids[(c * total + p) * 16 + sub];
        const int64_t n = c == 0 ? nu : nv;
        if (j < 0 || j >= n)
            flag(status, AFSI_FLAG_INDEX);
        else
            sum = (c == 0 ? u : v)[j] * w[(c * total + p) * 16 + sub];
    }
#pragma unroll
    for (int d = 8; d; d >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, d, 16);
    if (active && sub == 0) out[p * 2 + c] = sum;
}

}  // namespace afsi

using namespace afsi;

namespace {

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
        batch_prepare2d_kernel<T><<<blocks_for(total, 256), 256, 0, stream>>>(points, total, t, ids,
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
        batch_spread2d_kernel<T><<<blocks_for(total * 2 * 16, 256), 256, 0, stream>>>(
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
        batch_gather2d_kernel<T><<<blocks_for(total * 2 * 16, 256), 256, 0, stream>>>(
            static_cast<const T*>(u), static_cast<const T*>(v), ids, static_cast<const T*>(weights), total, nu, nv,
            static_cast<T*>(out), status);
    });
    return launched("batch2d gather");
}
