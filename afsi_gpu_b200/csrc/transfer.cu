// IB_4 spread / gather kernels: indexed (explicit ids) and compact separable
// 3D (one component), plus the C-ABI of the fused P2 element transfers whose
// kernels live in p2.cu.
//
// Gather kernels are atomic-free and deterministic.  The compact gather gives
// each point a group of four lanes (one x-offset i per lane, 16 (j,k) links
// each) so the L2-resident face field is read by four times more threads in
// flight than points, and combines the lanes with shuffles.  Spreads add into
// the caller's pre-zeroed fields with fire-and-forget L2 reductions.
#include "common.cuh"
#include "p2.cuh"

namespace afsi {

// ----------------------------------------------------------------- indexed

// G lanes per (point, component); G = 16 for the 2D 4x4 stencils.
template <class T, bool Spread, int G>
__global__ void __launch_bounds__(256) indexed_kernel(const T* __restrict__ f, const int64_t* __restrict__ ids,
                                                      const T* __restrict__ w, T* __restrict__ out, int64_t points,
                                                      int64_t neighbors, int64_t components, int64_t nodes,
                                                      T volume, int32_t* status) {
    const int64_t task = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / G;
    const int sub = threadIdx.x % G;
    const bool active = task < points * components;
    const int64_t p = active ? task / components : 0, c = active ? task % components : 0;
    T sum = T(0);
    if (active) {
        for (int64_t k = sub; k < neighbors; k += G) {
            const int64_t j = ids[p * neighbors + k];
            if (j < 0 || j >= nodes) {
                flag(status, AFSI_FLAG_INDEX);
                continue;
            }
            const T weight = w[p * neighbors + k];
            if (Spread)
                atomicAdd(out + j * components + c, (f[p * components + c] * weight) / volume);
            else
                sum += f[j * components + c] * weight;
        }
    }
    if (!Spread) {
#pragma unroll
        for (int d = G / 2; d; d >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, d, G);
        if (active && sub == 0) out[p * components + c] = sum;
    }
}

// ----------------------------------------------------------------- compact

// Four lanes per point; lane i owns x-offset i.  Returns false (and flags) if
// the 4x4x4 box leaves [0,n).
__device__ __forceinline__ bool box_inside(int64_t bx, int64_t by, int64_t bz, int64_t nx, int64_t ny, int64_t nz) {
    return bx >= 0 && by >= 0 && bz >= 0 && bx + 3 < nx && by + 3 < ny && bz + 3 < nz;
}

template <class T, bool Spread>
__global__ void __launch_bounds__(256) compact_kernel(const T* __restrict__ f, const int64_t* __restrict__ base,
                                                      const T* __restrict__ phi, T* __restrict__ out, int64_t points,
                                                      int64_t nx, int64_t ny, int64_t nz, T volume,
                                                      int32_t* status) {
    const int64_t p = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 2;
    const int i = threadIdx.x & 3;
    const bool active = p < points;
    T sum = T(0);
    if (active) {
        const int64_t bx = base[p * 3], by = base[p * 3 + 1], bz = base[p * 3 + 2];
        if (!box_inside(bx, by, bz, nx, ny, nz)) {
            if (i == 0) flag(status, AFSI_FLAG_INDEX);
        } else {
            const T* ph = phi + p * 12;
            const T px = ph[i];
            T py[4], pz[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                py[k] = ph[4 + k];
                pz[k] = ph[8 + k];
            }
            const int64_t row = (bx + i) * ny;
            if (Spread) {
                const T fv = f[p];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    T* dst = out + (row + by + j) * nz + bz;
                    const T wxy = px * py[j];
#pragma unroll
                    for (int k = 0; k < 4; ++k) atomicAdd(dst + k, ((wxy * pz[k]) * fv) / volume);
                }
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const T* src = f + (row + by + j) * nz + bz;
                    const T wxy = px * py[j];
#pragma unroll
                    for (int k = 0; k < 4; ++k) sum = fma(src[k], wxy * pz[k], sum);
                }
            }
        }
    }
    if (!Spread) {
        sum += __shfl_xor_sync(0xffffffffu, sum, 1);
        sum += __shfl_xor_sync(0xffffffffu, sum, 2);
        if (active && i == 0) out[p] = sum;
    }
}

// rhs[n] (+)= sum over the node's (element, slot) entries in CSR order.
template <class T>
__global__ void __launch_bounds__(256) node_reduce_kernel(const T* __restrict__ local, int64_t slots,
                                                          const int64_t* __restrict__ crow,
                                                          const int64_t* __restrict__ slot, int64_t nodes,
                                                          T* __restrict__ rhs, int accumulate, int32_t* status) {
    const int64_t n = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n >= nodes) return;
    T s[3] = {T(0), T(0), T(0)};
    for (int64_t k = crow[n]; k < crow[n + 1]; ++k) {
        const int64_t s_ = slot[k];
        if (s_ < 0 || s_ >= slots) {
            flag(status, AFSI_FLAG_INDEX);
            continue;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) s[c] += local[s_ * 3 + c];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) rhs[n * 3 + c] = accumulate ? rhs[n * 3 + c] + s[c] : s[c];
}

}  // namespace afsi

using namespace afsi;

extern "C" int32_t afsi_b200_indexed_gather(const void* field, int64_t nodes, int64_t components,
                                            const int64_t* ids, const void* weights, int64_t points,
                                            int64_t neighbors, void* out, int32_t* status, int32_t dtype,
                                            afsi_stream_t stream) {
    AFSI_REQUIRE(nodes > 0 && components > 0 && neighbors > 0 && points >= 0, "invalid indexed gather sizes");
    if (points == 0) return AFSI_OK;
    AFSI_REQUIRE(field && ids && weights && out, "null device pointer");
    const int64_t tasks = points * components;
    AFSI_DISPATCH(dtype, {
        if (neighbors <= 16)
            indexed_kernel<T, false, 16><<<blocks_for(tasks * 16, 256), 256, 0, stream>>>(
                static_cast<const T*>(field), ids, static_cast<const T*>(weights), static_cast<T*>(out), points,
                neighbors, components, nodes, T(1), status);
        else
            indexed_kernel<T, false, 32><<<blocks_for(tasks * 32, 256), 256, 0, stream>>>(
                static_cast<const T*>(field), ids, static_cast<const T*>(weights), static_cast<T*>(out), points,
                neighbors, components, nodes, T(1), status);
    });
    return launched("indexed_gather");
}

extern "C" int32_t afsi_b200_indexed_spread(const void* field, int64_t points, int64_t components,
                                            const int64_t* ids, const void* weights, int64_t neighbors,
                                            int64_t size, double volume, void* out, int32_t* status, int32_t dtype,
                                            afsi_stream_t stream) {
    AFSI_REQUIRE(size > 0 && components > 0 && neighbors > 0 && points >= 0, "invalid indexed spread sizes");
    AFSI_REQUIRE(isfinite(volume) && volume > 0, "invalid IB output size/volume");
    if (points == 0) return AFSI_OK;
    AFSI_REQUIRE(field && ids && weights && out, "null device pointer");
    const int64_t tasks = points * components;
    AFSI_DISPATCH(dtype, {
        if (neighbors <= 16)
            indexed_kernel<T, true, 16><<<blocks_for(tasks * 16, 256), 256, 0, stream>>>(
                static_cast<const T*>(field), ids, static_cast<const T*>(weights), static_cast<T*>(out), points,
                neighbors, components, size, T(volume), status);
        else
            indexed_kernel<T, true, 32><<<blocks_for(tasks * 32, 256), 256, 0, stream>>>(
                static_cast<const T*>(field), ids, static_cast<const T*>(weights), static_cast<T*>(out), points,
                neighbors, components, size, T(volume), status);
    });
    return launched("indexed_spread");
}

extern "C" int32_t afsi_b200_compact_gather(const void* field, const int64_t* base, const void* phi,
                                            int64_t points, int64_t nx, int64_t ny, int64_t nz, void* out,
                                            int32_t* status, int32_t dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(nx > 0 && ny > 0 && nz > 0 && points >= 0, "invalid compact grid");
    if (points == 0) return AFSI_OK;
    AFSI_REQUIRE(field && base && phi && out, "null device pointer");
    AFSI_DISPATCH(dtype, {
        compact_kernel<T, false><<<blocks_for(points * 4, 256), 256, 0, stream>>>(
            static_cast<const T*>(field), base, static_cast<const T*>(phi), static_cast<T*>(out), points, nx, ny,
            nz, T(1), status);
    });
    return launched("compact_gather");
}

extern "C" int32_t afsi_b200_compact_spread(const void* field, const int64_t* base, const void* phi,
                                            int64_t points, int64_t nx, int64_t ny, int64_t nz, double volume,
                                            void* out, int32_t* status, int32_t dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(nx > 0 && ny > 0 && nz > 0 && points >= 0, "invalid compact grid");
    AFSI_REQUIRE(isfinite(volume) && volume > 0, "invalid compact grid/volume");
    if (points == 0) return AFSI_OK;
    AFSI_REQUIRE(field && base && phi && out, "null device pointer");
    AFSI_DISPATCH(dtype, {
        compact_kernel<T, true><<<blocks_for(points * 4, 256), 256, 0, stream>>>(
            static_cast<const T*>(field), base, static_cast<const T*>(phi), static_cast<T*>(out), points, nx, ny,
            nz, T(volume), status);
    });
    return launched("compact_spread");
}

static int32_t p2_check(int64_t elements, int64_t nq, int64_t total, int64_t offset, int64_t nx, int64_t ny,
                        int64_t nz) {
    AFSI_REQUIRE(elements >= 0 && nq > 0, "invalid P2 group sizes");
    AFSI_REQUIRE(offset >= 0 && offset <= total && elements * nq <= total - offset,
                 "P2 IB group exceeds table bounds");
    AFSI_REQUIRE(nx > 0 && ny > 0 && nz > 0, "invalid P2 MAC grid");
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_p2_spread(const void* value, int64_t nodes, const int64_t* cells, int64_t elements,
                                       const void* N, int64_t nq, const void* W, const int64_t* base,
                                       const void* phi, int64_t total, int64_t offset, void* u0, void* u1, void* u2,
                                       int64_t nx, int64_t ny, int64_t nz, double volume, int32_t* status,
                                       int32_t dtype, afsi_stream_t stream) {
    int32_t rc = p2_check(elements, nq, total, offset, nx, ny, nz);
    if (rc) return rc;
    AFSI_REQUIRE(isfinite(volume) && volume > 0, "invalid P2 MAC grid");
    if (elements == 0) return AFSI_OK;
    AFSI_REQUIRE(value && cells && N && W && base && phi && u0 && u1 && u2, "null device pointer");
    P2Dims g{nx, ny, nz, total, offset, nq, nodes, elements};
    AFSI_DISPATCH(dtype, {
        return launch_spread_staged<T>(static_cast<const T*>(value), cells, static_cast<const T*>(N),
                                       static_cast<const T*>(W), base, static_cast<const T*>(phi),
                                       static_cast<T*>(u0), static_cast<T*>(u1), static_cast<T*>(u2), g, T(volume),
                                       status, staged_blocks(elements), stream);
    });
    return AFSI_OK;
}

template <bool Local>
static int32_t p2_gather(const void* u0, const void* u1, const void* u2, const int64_t* cells, int64_t elements,
                         const void* N, int64_t nq, const void* W, const int64_t* base, const void* phi,
                         int64_t total, int64_t offset, void* out, int64_t nodes, int64_t nx, int64_t ny,
                         int64_t nz, int32_t* status, int32_t dtype, afsi_stream_t stream) {
    int32_t rc = p2_check(elements, nq, total, offset, nx, ny, nz);
    if (rc) return rc;
    if (elements == 0) return AFSI_OK;
    AFSI_REQUIRE(u0 && u1 && u2 && cells && N && W && base && phi && out, "null device pointer");
    P2Dims g{nx, ny, nz, total, offset, nq, nodes, elements};
    AFSI_DISPATCH(dtype, {
        return launch_gather_staged<T, Local>(static_cast<const T*>(u0), static_cast<const T*>(u1),
                                              static_cast<const T*>(u2), cells, static_cast<const T*>(N),
                                              static_cast<const T*>(W), base, static_cast<const T*>(phi),
                                              static_cast<T*>(out), g, status, staged_blocks(elements), stream);
    });
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_p2_gather_assemble(const void* u0, const void* u1, const void* u2,
                                                const int64_t* cells, int64_t elements, const void* N, int64_t nq,
                                                const void* W, const int64_t* base, const void* phi, int64_t total,
                                                int64_t offset, void* rhs, int64_t nodes, int64_t nx, int64_t ny,
                                                int64_t nz, int32_t* status, int32_t dtype, afsi_stream_t stream) {
    return p2_gather<false>(u0, u1, u2, cells, elements, N, nq, W, base, phi, total, offset, rhs, nodes, nx, ny, nz,
                            status, dtype, stream);
}

extern "C" int32_t afsi_b200_p2_gather_local(const void* u0, const void* u1, const void* u2, const int64_t* cells,
                                             int64_t elements, const void* N, int64_t nq, const void* W,
                                             const int64_t* base, const void* phi, int64_t total, int64_t offset,
                                             void* local, int64_t nx, int64_t ny, int64_t nz, int32_t* status,
                                             int32_t dtype, afsi_stream_t stream) {
    return p2_gather<true>(u0, u1, u2, cells, elements, N, nq, W, base, phi, total, offset, local, INT64_MAX, nx,
                           ny, nz, status, dtype, stream);
}

extern "C" int32_t afsi_b200_node_reduce(const void* local, int64_t slots, const int64_t* crow, const int64_t* slot,
                                         int64_t nodes, void* rhs, int32_t accumulate, int32_t* status,
                                         int32_t dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(nodes >= 0 && slots >= 0, "invalid node reduction sizes");
    if (nodes == 0) return AFSI_OK;
    AFSI_REQUIRE(local && crow && slot && rhs, "null device pointer");
    AFSI_DISPATCH(dtype, {
        node_reduce_kernel<T><<<blocks_for(nodes, 256), 256, 0, stream>>>(
            static_cast<const T*>(local), slots, crow, slot, nodes, static_cast<T*>(rhs), accumulate, status);
    });
    return launched("node_reduce");
}
