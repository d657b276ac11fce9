// P2 element transfers (spread, gather-assemble) for the B200.
//
// One warp owns one P2 element at a time (grid-stride over elements).
//
// Spread: for each velocity component in turn, the element's contributions
// are accumulated into a shared-memory box covering the supports of that
// component.  The warp works on two quadrature points at once: each half-warp
// takes one point and its 16 lanes own the (i,j) columns of the point's 4x4x4
// support, with the four z links of a column handled by that lane.  Each
// half-warp has a private copy of the box, so the adds are plain
// read-modify-writes in a fixed order (points h, h+2, h+4, ... in half h): no
// atomics.  The box strides are padded (y stride odd, x stride = 4 mod 8) so
// that the 16 lanes of a half-warp always address 16 different 8-byte bank
// pairs: the read-modify-writes are free of bank conflicts wherever the point
// lies.  The two copies are summed and flushed to the face array with one L2
// reduction per non-zero face — about 130 per element and component instead
// of 64 per point.
// Gather: one lane per point reads the point's table rows and sums its
// support over the component's face patch, staged in shared memory once per
// element and component; the nodal sums Σ_q N[q,a] W U(x_q) are formed by
// lanes (a, c) in point order and added to the right-hand side (or written
// per element for the deterministic node reduction).
// Rules of at most 64 points per element take a spread variant that stages the
// element's stencil rows in shared memory with bulk copies first and merges
// runs of points with the same support origin in registers before adding them
// to a single box copy (p2_spread_rows_kernel, runs.cuh).
// Point forces F = (Σ_a N[q,a] value[a]) * W (mac/compact_transfer.py:29-35)
// are computed once per point and component by a lanes-over-points pass; the
// spread contribution is (φx·φy)·φz · (F/volume), one division per point
// instead of per link as in the reference kernel (one rounding of difference).
// An element whose box does not fit the shared-memory copies is processed
// with direct L2 reductions / global loads, checking each point's support
// against the grid (a point outside sets AFSI_FLAG_INDEX and is skipped).
#include <climits>
#include "common.cuh"
#include "p2.cuh"
#include "runs.cuh"

namespace afsi {

constexpr int kWarps = 4;       // warps per block
constexpr int kChunk = 64;      // points whose forces are held at once
constexpr int kSpreadCap = 288;   // spread: entries of one component's padded box per copy

// f(t, x, y, z) for the cells t = lane, lane + 32, ... of an ex x ey x ez box
// (z fastest); the coordinates advance by mixed-radix addition of 32 (one
// carry per axis at most) instead of two divisions per cell.
template <class F>
__device__ __forceinline__ void box_walk(int lane, int ex, int ey, int ez, F f) {
    const int n = ex * ey * ez;
    if (lane >= n) return;
    const int qz = 32 % ez, q = 32 / ez, qy = q % ey, qx = q / ey;
    int z = lane % ez, r = lane / ez, y = r % ey, x = r / ey;
    for (int t = lane; t < n; t += 32) {
        f(t, x, y, z);
        z += qz;
        int carry = z >= ez ? 1 : 0;
        z -= carry * ez;
        y += qy + carry;
        carry = y >= ey ? 1 : 0;
        y -= carry * ey;
        x += qx + carry;
    }
}
constexpr int kSpreadBlocks = 6;  // resident blocks per SM the spread is compiled for
constexpr int kGatherBlocks = 6;  // same for the gather

struct Box {
    int lo[3][3], ext[3][3];
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
}

__device__ __forceinline__ bool component_inside(const Box& bx, const P2Dims& g, int c) {
    const int64_t fe[3] = {g.nx + (c == 0), g.ny + (c == 1), g.nz + (c == 2)};
    bool inside = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) inside = inside && bx.lo[c][a] >= 0 && int64_t(bx.lo[c][a]) + bx.ext[c][a] <= fe[a];
    return inside;
}


// Padded strides of component c's box in a spread copy: sy = ez|1 (odd) and
// sx = 4 (mod 8), sx >= ey*sy.  Entry (x,y,z) sits at x*sx + y*sy + z, and the
// offsets li*sx + lj*sy (li, lj in 0..3) are 16 distinct values mod 16: the
// 16 lanes of a half-warp meet 16 different 8-byte bank pairs.  False when the
// box leaves the face array or does not fit kSpreadCap entries.
__device__ __forceinline__ bool spread_layout(const Box& bx, const P2Dims& g, int c, int& sx, int& sy) {
    const int ey = bx.ext[c][1], ez = bx.ext[c][2];
    sy = sx = 0;
    if (!component_inside(bx, g, c) || ey > 64 || ez > 64) return false;
    padded_strides(ey, ez, sx, sy);
    return int64_t(bx.ext[c][0]) * sx <= kSpreadCap;
}

__device__ __forceinline__ int64_t face_index(const P2Dims& g, int c, int x, int y, int z) {
    return (int64_t(x) * (g.ny + (c == 1)) + y) * (g.nz + (c == 2)) + z;
}

// The 4x4x4 box of component c starting at (x,y,z) lies inside its face array.
__device__ __forceinline__ bool point_inside(const P2Dims& g, int c, int x, int y, int z) {
    return x >= 0 && y >= 0 && z >= 0 && x + 3 < g.nx + (c == 0) && y + 3 < g.ny + (c == 1) &&
           z + 3 < g.nz + (c == 2);
}

// Rows of four weights are read as one 32-byte pair of vector loads.

template <class T> struct Pair;
template <> struct Pair<double> { using type = double2; };
template <> struct Pair<float> { using type = float2; };

template <class T>
__device__ __forceinline__ void load_row4(const T* __restrict__ w, T out[4]) {
    using P = typename Pair<T>::type;
    const P a = reinterpret_cast<const P*>(w)[0];
    const P b = reinterpret_cast<const P*>(w)[1];
    out[0] = a.x;
    out[1] = a.y;
    out[2] = b.x;
    out[3] = b.y;
}

// ------------------------------------------------------------------ spread

template <class T>
struct SpreadStage {
    T f[kChunk];
    T coef[32];
    T copy[2][kSpreadCap];
};

template <class T>
__global__ void __launch_bounds__(kWarps * 32, kSpreadBlocks) p2_spread_kernel(
    const T* __restrict__ value, const int64_t* __restrict__ cells, const T* __restrict__ N, const T* __restrict__ W,
    const int64_t* __restrict__ base, const T* __restrict__ phi, T* __restrict__ u0, T* __restrict__ u1,
    T* __restrict__ u2, P2Dims g, T volume, int32_t* status) {
    __shared__ SpreadStage<T> stage_all[kWarps];
    SpreadStage<T>& s = stage_all[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31, half = lane >> 4, li = (lane >> 2) & 3, lj = lane & 3;
    const int64_t warps = int64_t(gridDim.x) * kWarps;
    const T inv_volume = exact_reciprocal(volume);
    for (int64_t e = int64_t(blockIdx.x) * kWarps + (threadIdx.x >> 5); e < g.elements; e += warps) {
        const int64_t node = lane < 10 ? cells[e * 10 + lane] : 0;
        if (__any_sync(0xffffffffu, lane < 10 && (node < 0 || node >= g.nodes))) {
            if (lane == 0) flag(status, AFSI_FLAG_INDEX);
            continue;
        }
        const int64_t mine = __shfl_sync(0xffffffffu, node, lane < 30 ? lane / 3 : 0);
        __syncwarp();
        if (lane < 30) s.coef[lane] = value[mine * 3 + lane % 3];
        Box bx;
        element_box(base, g, e, bx);
        T* copy = s.copy[half];
#pragma unroll
        for (int c = 0; c < 3; ++c) {  // unrolled: the box and field of c stay in registers
            T* field = c == 0 ? u0 : c == 1 ? u1 : u2;
            int sx, sy;
            const bool fits = spread_layout(bx, g, c, sx, sy);
            __syncwarp();
            if (fits)
                for (int t = lane; t < 2 * kSpreadCap; t += 32) (&s.copy[0][0])[t] = T(0);
            for (int64_t q0 = 0; q0 < g.nq; q0 += kChunk) {
                const int n = int(g.nq - q0 < kChunk ? g.nq - q0 : kChunk);
                __syncwarp();
                for (int q = lane; q < n; q += 32) {  // component c of the forces, lanes over points
                    T F = T(0);
#pragma unroll
                    for (int a = 0; a < 10; ++a) F += N[(q0 + q) * 10 + a] * s.coef[a * 3 + c];
                    const T fw = F * W[e * g.nq + q0 + q];
                    s.f[q] = inv_volume != T(0) ? fw * inv_volume : fw / volume;
                }
                __syncwarp();
#pragma unroll 2
                for (int q = half; q < n; q += 2) {
                    const int64_t row = g.offset + e * g.nq + q0 + q;
                    const int64_t rx = table_row(g.total, row, c, 0), ry = table_row(g.total, row, c, 1),
                                  rz = table_row(g.total, row, c, 2);
                    const int gx = int(base[rx]), gy = int(base[ry]), gz = int(base[rz]);
                    const T w = phi[rx * 4 + li] * phi[ry * 4 + lj];
                    T wz[4];
                    load_row4(phi + rz * 4, wz);
                    const T fq = s.f[q];
                    if (fits) {
                        T* dst = copy + (gx - bx.lo[c][0] + li) * sx + (gy - bx.lo[c][1] + lj) * sy +
                                 (gz - bx.lo[c][2]);
#pragma unroll
                        for (int k = 0; k < 4; ++k) dst[k] += (w * wz[k]) * fq;
                    } else if (point_inside(g, c, gx, gy, gz)) {
                        T* dst = field + face_index(g, c, gx + li, gy + lj, gz);
#pragma unroll
                        for (int k = 0; k < 4; ++k) atomicAdd(dst + k, (w * wz[k]) * fq);
                    } else if ((lane & 15) == 0) {
                        flag(status, AFSI_FLAG_INDEX);
                    }
                }
            }
            __syncwarp();
            if (fits) {
                box_walk(lane, bx.ext[c][0], bx.ext[c][1], bx.ext[c][2], [&](int, int x, int y, int z) {
                    const int o = x * sx + y * sy + z;
                    const T v = s.copy[0][o] + s.copy[1][o];
                    if (v != T(0))
                        atomicAdd(field + face_index(g, c, bx.lo[c][0] + x, bx.lo[c][1] + y, bx.lo[c][2] + z), v);
                });
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------- spread, staged rows
//
// For rules of at most kRowPoints points per element (the common adaptive
// orders) the element's stencil rows — both lattices' bases (3 int64 per
// point) and weights (12 per point), about 15 KB for 64 points in FP64 — are
// contiguous in the tables, and are brought into shared memory by the bulk
// copy engine (cp.async.bulk, one copy per lattice's weights and, when
// 16-byte aligned, per lattice's bases), completing on a per-warp mbarrier,
// instead of one chain of dependent global loads per point; the element's
// boxes come from the staged bases.  The wait on the mbarrier is bounded by
// a clock budget: a copy that does not complete flags AFSI_FLAG_TIMEOUT and
// the element is skipped.  The accumulation is spread_runs (runs.cuh): each
// run of consecutive points with one support origin is summed in registers
// and added to the padded box once.

constexpr int kRowPoints = 64;
constexpr int kRowWarps = 2;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from
// global to this CTA's shared memory, completing on mbarrier `bar`.
__device__ __forceinline__ void bulk_copy(void* smem, const void* gmem, unsigned bytes, unsigned long long* bar) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    const unsigned b = static_cast<unsigned>(__cvta_generic_to_shared(bar));
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(d), "l"(gmem), "r"(bytes), "r"(b) : "memory");
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
    const unsigned b = static_cast<unsigned>(__cvta_generic_to_shared(bar));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect(unsigned long long* bar, unsigned bytes) {
    const unsigned b = static_cast<unsigned>(__cvta_generic_to_shared(bar));
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
}

// Wait for phase `parity` of `bar` to complete, for at most about a second.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    const unsigned b = static_cast<unsigned>(__cvta_generic_to_shared(bar));
    const long long t0 = clock64();
    while (true) {
        unsigned done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}" : "=r"(done) : "r"(b), "r"(parity) : "memory");
        if (done) return true;
        if (clock64() - t0 > 2000000000LL) return false;
    }
}

template <class T>
struct __align__(16) RowStage {  // size a multiple of 16: every warp's copy targets start 16-byte aligned
    T phi[2][(kRowPoints + 1) * 12];  // row kRowPoints stays zero (spread_element's padding row)
    int64_t base[2][kRowPoints * 3];
    T f[kRowPoints + 1];
    T coef[32];
    T box[kSpreadCap];
    int key[kRowPoints];
    int perm[4 * kRowPoints];   // points grouped by key (spread_element)
    int rs[kRowPoints + 1], rk[kRowPoints];
    unsigned long long bar;  // completion of this warp's bulk copies
};

template <class T>
__global__ void __launch_bounds__(kRowWarps * 32, 6) p2_spread_rows_kernel(
    const T* __restrict__ value, const int64_t* __restrict__ cells, const T* __restrict__ N, const T* __restrict__ W,
    const int64_t* __restrict__ base, const T* __restrict__ phi, T* __restrict__ u0, T* __restrict__ u1,
    T* __restrict__ u2, P2Dims g, T volume, int32_t* status) {
    __shared__ __align__(16) RowStage<T> stage_all[kRowWarps];
    RowStage<T>& s = stage_all[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31, half = lane >> 4, li = (lane >> 2) & 3, lj = lane & 3;
    const int64_t warps = int64_t(gridDim.x) * kRowWarps;
    const int n = int(g.nq);
    const T inv_volume = exact_reciprocal(volume);
    // weights: n*12*sizeof(T) bytes per lattice, a multiple of 16 (n even for T=float)
    const unsigned phi_bytes = unsigned(n * 12 * int(sizeof(T)));
    const bool phi_bulk = phi_bytes % 16 == 0;
    if (lane == 0) mbar_init(&s.bar);
    if (lane < 24) s.phi[lane / 12][kRowPoints * 12 + lane % 12] = T(0);
    if (lane == 0) s.f[kRowPoints] = T(0);
    __syncwarp();
    unsigned parity = 0;
    for (int64_t e = int64_t(blockIdx.x) * kRowWarps + (threadIdx.x >> 5); e < g.elements; e += warps) {
        const int64_t node = lane < 10 ? cells[e * 10 + lane] : 0;
        if (__any_sync(0xffffffffu, lane < 10 && (node < 0 || node >= g.nodes))) {
            if (lane == 0) flag(status, AFSI_FLAG_INDEX);
            continue;
        }
        __syncwarp();
        const int64_t row0 = g.offset + e * g.nq;
        // bases: bulk when both lattices' rows start 16-byte aligned (row0 and total even)
        const bool base_bulk = ((row0 | g.total) & 1) == 0 && (n * 3 * 8) % 16 == 0 &&
                               reinterpret_cast<uintptr_t>(base) % 16 == 0;
        if (lane == 0) {
            // order this warp's earlier shared-memory reads before the bulk writes
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            const unsigned bytes = (phi_bulk ? 2 * phi_bytes : 0) + (base_bulk ? 2 * unsigned(n * 3 * 8) : 0);
            mbar_expect(&s.bar, bytes);
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                if (phi_bulk) bulk_copy(s.phi[t], phi + (int64_t(t) * g.total + row0) * 12, phi_bytes, &s.bar);
                if (base_bulk)
                    bulk_copy(s.base[t], base + (int64_t(t) * g.total + row0) * 3, unsigned(n * 3 * 8), &s.bar);
            }
        }
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            if (!phi_bulk) {
                const unsigned char* src =
                    reinterpret_cast<const unsigned char*>(phi + (int64_t(t) * g.total + row0) * 12);
                for (int i = lane; i < n * 12 * int(sizeof(T)) / 8; i += 32)
                    cp_async8(reinterpret_cast<unsigned char*>(s.phi[t]) + i * 8, src + i * 8);
            }
            if (!base_bulk) {
                const int64_t* bsrc = base + (int64_t(t) * g.total + row0) * 3;
                for (int i = lane; i < n * 3; i += 32) cp_async8(&s.base[t][i], bsrc + i);
            }
        }
        const int64_t mine = __shfl_sync(0xffffffffu, node, lane < 30 ? lane / 3 : 0);
        if (lane < 30) s.coef[lane] = value[mine * 3 + lane % 3];
        cp_async_wait_all();
        const bool arrived = mbar_wait(&s.bar, parity);
        parity ^= 1u;
        if (!__all_sync(0xffffffffu, arrived)) {
            // a copy that never completed: flag it; this warp's later bulk copies
            // would land in the same buffers, so the warp stops here
            if (lane == 0) flag(status, AFSI_FLAG_TIMEOUT);
            return;
        }
        __syncwarp();
        Box bx;
        {
            int mn[3][3], mx[3][3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    mn[c][a] = INT_MAX;
                    mx[c][a] = INT_MIN;
                }
            for (int q = lane; q < n; q += 32) {
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const int v = int(s.base[a != c][q * 3 + a]);
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
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {  // unrolled: the box, tables and field of c stay in registers
            T* field = c == 0 ? u0 : c == 1 ? u1 : u2;
            int sx, sy;
            const bool fits = spread_layout(bx, g, c, sx, sy);
            const int tx = c != 0, ty = c != 1, tz = c != 2;
            __syncwarp();
            if (fits)
                for (int t = lane; t < kSpreadCap; t += 32) s.box[t] = T(0);
            for (int q = lane; q < n; q += 32) {  // component c of the forces and the run keys, lanes over points
                T F = T(0);
#pragma unroll
                for (int a = 0; a < 10; ++a) F += N[q * 10 + a] * s.coef[a * 3 + c];
                const T fw = F * W[e * g.nq + q];
                s.f[q] = inv_volume != T(0) ? fw * inv_volume : fw / volume;
                if (fits)
                    s.key[q] = run_key(int(s.base[tx][q * 3]) - bx.lo[c][0], int(s.base[ty][q * 3 + 1]) - bx.lo[c][1],
                                       int(s.base[tz][q * 3 + 2]) - bx.lo[c][2]);
            }
            __syncwarp();
            if (fits) {
                spread_element<T, kRowPoints>(s.box, s.key, s.f, s.phi[tx], s.phi[ty] + 4, s.phi[tz] + 8, n, sx, sy, s.perm, s.rs, s.rk);
                __syncwarp();
                box_walk(lane, bx.ext[c][0], bx.ext[c][1], bx.ext[c][2], [&](int, int x, int y, int z) {
                    const T v = s.box[x * sx + y * sy + z];
                    if (v != T(0))
                        atomicAdd(field + face_index(g, c, bx.lo[c][0] + x, bx.lo[c][1] + y, bx.lo[c][2] + z), v);
                });
            } else {
                for (int q = half; q < n; q += 2) {
                    const int gx = int(s.base[tx][q * 3]), gy = int(s.base[ty][q * 3 + 1]),
                              gz = int(s.base[tz][q * 3 + 2]);
                    if (point_inside(g, c, gx, gy, gz)) {
                        const T w = (s.phi[tx][q * 12 + li] * s.phi[ty][q * 12 + 4 + lj]) * s.f[q];
                        T* dst = field + face_index(g, c, gx + li, gy + lj, gz);
#pragma unroll
                        for (int k = 0; k < 4; ++k) atomicAdd(dst + k, w * s.phi[tz][q * 12 + 8 + k]);
                    } else if ((lane & 15) == 0) {
                        flag(status, AFSI_FLAG_INDEX);
                    }
                }
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------ gather
//
// One lane per point: the lane reads its point's three table rows of the
// component (bases and four weights per axis, one 32-byte row each) and sums
// the 64 links over the component's face patch in shared memory (fixed
// strides, runs.cuh), or over the face array where the element's box does
// not fit.  The velocities U_c(x_q) of up to 64 points are kept in shared
// memory and assembled by lanes (a, c) in point order:
// rhs[a][c] = sum_q N[q,a] W_q U_c(x_q) (mac/csrc/p2_transfer.cu:150-188).

constexpr int kGatherPoints = 64;

template <class T>
struct GatherStage {
    T patch[kGPatch];
    T u[3][kGatherPoints];
    T w[kGatherPoints];
};

template <class T, bool Local>
__global__ void __launch_bounds__(kWarps * 32, kGatherBlocks) p2_gather_kernel(const T* __restrict__ u0, const T* __restrict__ u1,
                                                                const T* __restrict__ u2,
                                                                const int64_t* __restrict__ cells,
                                                                const T* __restrict__ N, const T* __restrict__ W,
                                                                const int64_t* __restrict__ base,
                                                                const T* __restrict__ phi, T* __restrict__ out,
                                                                P2Dims g, int32_t* status) {
    __shared__ __align__(16) GatherStage<T> stage_all[kWarps];
    GatherStage<T>& s = stage_all[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * kWarps;
    using P = typename Pair<T>::type;
    for (int64_t e = int64_t(blockIdx.x) * kWarps + (threadIdx.x >> 5); e < g.elements; e += warps) {
        const int64_t node = lane < 10 ? cells[e * 10 + lane] : 0;
        if (__any_sync(0xffffffffu, lane < 10 && (node < 0 || node >= g.nodes))) {
            if (lane == 0) flag(status, AFSI_FLAG_INDEX);
            continue;
        }
        Box bx;
        element_box(base, g, e, bx);
        T acc = T(0);  // lane (a, cc) = (lane / 3, lane % 3), lane < 30
        for (int64_t q0 = 0; q0 < g.nq; q0 += kGatherPoints) {
            const int n = int(g.nq - q0 < kGatherPoints ? g.nq - q0 : kGatherPoints);
            __syncwarp();
            for (int q = lane; q < n; q += 32) s.w[q] = W[e * g.nq + q0 + q];
#pragma unroll 1
            for (int c = 0; c < 3; ++c) {
                const T* field = c == 0 ? u0 : c == 1 ? u1 : u2;
                bool fits = component_inside(bx, g, c);
#pragma unroll
                for (int a = 0; a < 3; ++a) fits = fits && bx.ext[c][a] <= kGExt;
                __syncwarp();  // the previous component's patch reads are done
                if (fits)
                    box_walk(lane, bx.ext[c][0], bx.ext[c][1], bx.ext[c][2], [&](int, int x, int y, int z) {
                        s.patch[x * kGSX + y * kGSY + z] =
                            field[face_index(g, c, bx.lo[c][0] + x, bx.lo[c][1] + y, bx.lo[c][2] + z)];
                    });
                __syncwarp();
#pragma unroll
                for (int j = 0; j < kGatherPoints / 32; ++j) {
                    const int q = lane + 32 * j;
                    if (q >= n) continue;
                    const int64_t row = g.offset + e * g.nq + q0 + q;
                    int b[3];
                    T wr[3][4];
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const int64_t ra = table_row(g.total, row, c, a);
                        b[a] = int(base[ra]);
                        const P w01 = reinterpret_cast<const P*>(phi + ra * 4)[0];
                        const P w23 = reinterpret_cast<const P*>(phi + ra * 4)[1];
                        wr[a][0] = w01.x;
                        wr[a][1] = w01.y;
                        wr[a][2] = w23.x;
                        wr[a][3] = w23.y;
                    }
                    T U = T(0);
                    if (fits) {
                        const T* p0 =
                            s.patch + (b[0] - bx.lo[c][0]) * kGSX + (b[1] - bx.lo[c][1]) * kGSY + (b[2] - bx.lo[c][2]);
                        U = support_dot(p0, kGSX, kGSY, wr[0], wr[1], wr[2]);
                    } else if (point_inside(g, c, b[0], b[1], b[2])) {
                        const int64_t sz = g.nz + (c == 2), sy = (g.ny + (c == 1)) * sz;
                        U = support_dot(field + face_index(g, c, b[0], b[1], b[2]), sy, sz, wr[0], wr[1], wr[2]);
                    } else {
                        flag(status, AFSI_FLAG_INDEX);
                    }
                    s.u[c][q] = U;
                }
            }
            __syncwarp();
            if (lane < 30) {
                const int a = lane / 3, cc = lane - 3 * (lane / 3);
                for (int q = 0; q < n; ++q) acc = fma(N[(q0 + q) * 10 + a] * s.w[q], s.u[cc][q], acc);
            }
        }
        const int64_t nd = __shfl_sync(0xffffffffu, node, lane < 30 ? lane / 3 : 0);
        if (lane < 30) {
            const int a = lane / 3, cc = lane - 3 * (lane / 3);
            if (Local)
                out[(e * 10 + a) * 3 + cc] = acc;
            else
                atomicAdd(out + nd * 3 + cc, acc);
        }
        __syncwarp();
    }
}

template <class T>
int32_t launch_spread_staged(const T* value, const int64_t* cells, const T* N, const T* W, const int64_t* base,
                             const T* phi, T* u0, T* u1, T* u2, const P2Dims& g, T volume, int32_t* status,
                             int blocks, cudaStream_t stream) {
    if (g.nq <= kRowPoints && reinterpret_cast<uintptr_t>(phi) % 16 == 0) {
        const int64_t want = (g.elements + kRowWarps - 1) / kRowWarps;
        p2_spread_rows_kernel<T><<<unsigned(want), kRowWarps * 32, 0, stream>>>(value, cells, N, W, base, phi, u0, u1,
                                                                              u2, g, volume, status);
    } else {
        p2_spread_kernel<T><<<blocks, kWarps * 32, 0, stream>>>(value, cells, N, W, base, phi, u0, u1, u2, g, volume,
                                                                status);
    }
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
