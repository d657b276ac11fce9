// Table-free element transfers: the spread and the gather-assemble of P2
// (10-node) and P1 (4-node) tetrahedra with each interaction point's
// position, lattice bases and Peskin weights formed inside the transfer
// kernel, instead of being written to (2,P,3) / (2,P,3,4) tables by a prepare
// and read back by the transfer.
//
// Reference semantics: the P2 transfer (mac/csrc/p2_transfer.cu:12-45 prepare,
// :98-188 spread / gather-assemble) and the matrix-free P1 element transfer
// (mac/adaptive_cell.py:22-83 -> mac/_triton_adaptive.py:25-128,
// mac/_triton_shared_fe.py:14-40): x_q = sum_a N[q,a] x[cell_a]; per axis a the
// support check 2 <= (x_q - origin)/h < n - 2; per lattice (faces along the
// axis: origin; cell centres: origin + h/2) scaled = (x_q - start)/h,
// base = floor(scaled - 1), weights = IB_4 of scaled - base - 1 in the
// shared-radical form.  Component c reads axis a on lattice (a != c).
// spread: f_c[face] += phi_x phi_y phi_z (F_q / volume), F_q = (N coef) W;
// gather-assemble: rhs[cell_a] += N[q,a] W_q U_c(x_q).
//
// Arithmetic: positions, validity, bases and weights use exactly the
// operations of fe_prepare_kernel (prepare.cu) in the position type TP, so the
// bases are bit-exact with the tables and the weights are the tables'
// weights (rounded once to T in the precision form); the accumulation is the
// staged-row kernels' (p2.cu), so a transfer equals the table-based one up to
// the order of its global atomic additions.
//
// Layout: one warp per element.  A first pass over the element's points
// (lanes over points) forms the positions and the six (axis, lattice) bases
// and reduces the element's support box per component.  Points are then
// taken in chunks of 64: lanes over points form the rows a chunk needs in
// shared memory (the spread: the three rows of one component and its
// forces; the gather: all six rows); the accumulation half-warp per point
// (spread, padded private boxes) or four points in flight (gather, staged face
// patch) follows.  A point whose support leaves the grid sets
// AFSI_FLAG_SUPPORT and is skipped; an element with a node id outside
// [0, nodes) sets AFSI_FLAG_INDEX and is skipped.
#include <climits>
#include "common.cuh"
#include "peskin.cuh"

namespace afsi {
namespace {

constexpr int kFSpreadWarps = 2;  // warps per spread block (about 19 KB of rows and boxes each)
constexpr int kFGatherWarps = 4;  // warps per gather block
// Points whose rows are held at once: 64 for P2 (the common adaptive orders
// have 15 or 64 points), 32 for P1 (orders 2 and 3 have 8 and 27 points), so a
// P1 warp's staging is half the size and twice as many warps fit an SM.
template <int NPC> struct FChunk { static constexpr int value = NPC == 10 ? 64 : 32; };
constexpr int kFSpreadCap = 288;  // entries of one component's padded box per copy
template <class T> struct FPatch { static constexpr int value = 4608 / sizeof(T); };

struct FusedDims {
    int64_t nx, ny, nz, nodes, elements, nq;
};

template <class TP>
struct Geo {
    TP origin[3], spacing[3], limits[3];
};

struct FBox {
    int lo[3][3], ext[3][3], off[4];
};

template <class T> struct FPair;
template <> struct FPair<double> { using type = double2; };
template <> struct FPair<float> { using type = float2; };

template <class TP, int NPC>
struct ElementNodes {
    TP x[NPC * 3];
};

// Position of point q (fe_prepare_kernel: pos[d] += N[q,a] * x[a][d], a in
// order, from zero), then per axis and lattice its base and, with w != null,
// its four weights; the lattice-0 quotient (x - origin)/h is also the
// prepare's support coordinate.  Returns the point's validity (every axis
// finite with 2 <= (x - origin)/h < n - 2).
template <class TP, class T, int NPC>
__device__ __forceinline__ bool point_rows(const TP* __restrict__ Npos, const TP* xs, int64_t q, const Geo<TP>& geo,
                                           int b[2][3], T* w0, T* w1) {
    TP pos[3] = {TP(0), TP(0), TP(0)};
#pragma unroll
    for (int a = 0; a < NPC; ++a) {
        const TP nv = Npos[q * NPC + a];
#pragma unroll
        for (int d = 0; d < 3; ++d) pos[d] += nv * xs[a * 3 + d];
    }
    bool valid = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const TP start = l ? geo.origin[a] + TP(.5) * geo.spacing[a] : geo.origin[a];
            const TP scaled = (pos[a] - start) / geo.spacing[a];
            if (l == 0) valid = valid && isfinite(scaled) && scaled >= TP(2) && scaled < geo.limits[a];
            const int64_t lower = static_cast<int64_t>(floor(scaled - TP(1)));
            b[l][a] = int(lower);
            T* w = l ? w1 : w0;
            if (w) {
                TP r[4];
                peskin_radical(scaled - TP(lower) - TP(1), r);
#pragma unroll
                for (int k = 0; k < 4; ++k) w[a * 4 + k] = T(r[k]);
            }
        }
    }
    return valid;
}

// Rows of points q0 .. q0+n-1 into shared memory (lanes over points):
// w[l][q*12 + a*4 + k], b[l][q*3 + a]; an invalid point is marked by
// b[0][q*3] = INT_MIN.  Returns true in every lane if any point was invalid.
template <class TP, class T, int NPC>
__device__ __forceinline__ bool fill_rows(const TP* __restrict__ Npos, const TP* xs, int64_t q0, int n,
                                          const Geo<TP>& geo, T* w0, T* w1, int* b0, int* b1) {
    bool bad = false;
    for (int q = threadIdx.x & 31; q < n; q += 32) {
        int b[2][3];
        const bool valid = point_rows<TP, T, NPC>(Npos, xs, q0 + q, geo, b, &w0[q * 12], &w1[q * 12]);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            b0[q * 3 + a] = b[0][a];
            b1[q * 3 + a] = b[1][a];
        }
        if (!valid) {
            b0[q * 3] = INT_MIN;
            bad = true;
        }
    }
    return __any_sync(0xffffffffu, bad);
}

__device__ __forceinline__ void box_init(int mn[3][3], int mx[3][3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mn[c][a] = INT_MAX;
            mx[c][a] = INT_MIN;
        }
}

__device__ __forceinline__ void box_add(int mn[3][3], int mx[3][3], const int b[2][3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int v = b[a != c][a];
            mn[c][a] = min(mn[c][a], v);
            mx[c][a] = max(mx[c][a], v);
        }
}

// Warp-reduce the per-lane bounds into the box; false when no point was valid.
__device__ __forceinline__ bool box_finish(int mn[3][3], int mx[3][3], FBox& bx) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int d = 16; d; d >>= 1) {
                mn[c][a] = min(mn[c][a], __shfl_xor_sync(0xffffffffu, mn[c][a], d));
                mx[c][a] = max(mx[c][a], __shfl_xor_sync(0xffffffffu, mx[c][a], d));
            }
    if (mn[0][0] == INT_MAX) return false;  // no valid point
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            bx.lo[c][a] = mn[c][a];
            bx.ext[c][a] = mx[c][a] - mn[c][a] + 4;
        }
    bx.off[0] = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        bx.off[c + 1] = bx.off[c] + int(min(int64_t(bx.ext[c][0]) * bx.ext[c][1] * bx.ext[c][2], int64_t(1) << 20));
    return true;
}

// Box of the n rows held in shared memory.
__device__ __forceinline__ bool box_from_rows(const int* b0, const int* b1, int n, FBox& bx) {
    int mn[3][3], mx[3][3];
    box_init(mn, mx);
    for (int q = threadIdx.x & 31; q < n; q += 32) {
        if (b0[q * 3] == INT_MIN) continue;
        int b[2][3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            b[0][a] = b0[q * 3 + a];
            b[1][a] = b1[q * 3 + a];
        }
        box_add(mn, mx, b);
    }
    return box_finish(mn, mx, bx);
}

// Box of all nq points, bases only (rules larger than one chunk); invalid
// points set AFSI_FLAG_SUPPORT.
template <class TP, class T, int NPC>
__device__ __forceinline__ bool box_from_points(const TP* __restrict__ Npos, const TP* xs, int64_t nq,
                                                const Geo<TP>& geo, FBox& bx, int32_t* status) {
    int mn[3][3], mx[3][3];
    box_init(mn, mx);
    bool bad = false;
    for (int64_t q = threadIdx.x & 31; q < nq; q += 32) {
        int b[2][3];
        if (!point_rows<TP, T, NPC>(Npos, xs, q, geo, b, nullptr, nullptr)) {
            bad = true;
            continue;
        }
        box_add(mn, mx, b);
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) flag(status, AFSI_FLAG_SUPPORT);
    return box_finish(mn, mx, bx);
}

__device__ __forceinline__ int64_t ffield_index(const FusedDims& g, int c, int x, int y, int z) {
    return (int64_t(x) * (g.ny + (c == 1)) + y) * (g.nz + (c == 2)) + z;
}

__device__ __forceinline__ bool fcomponent_inside(const FBox& bx, const FusedDims& g, int c) {
    const int64_t fe[3] = {g.nx + (c == 0), g.ny + (c == 1), g.nz + (c == 2)};
    bool inside = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) inside = inside && bx.lo[c][a] >= 0 && int64_t(bx.lo[c][a]) + bx.ext[c][a] <= fe[a];
    return inside;
}

__device__ __forceinline__ bool fpoint_inside(const FusedDims& g, int c, int x, int y, int z) {
    return x >= 0 && y >= 0 && z >= 0 && x + 3 < g.nx + (c == 0) && y + 3 < g.ny + (c == 1) &&
           z + 3 < g.nz + (c == 2);
}

// Stage the element's node positions (TP) and, optionally, its nodal values
// (T, three per node).  Returns false (and flags) for a node id out of range.
template <class TP, class T, int NPC>
__device__ __forceinline__ bool stage_element(const TP* __restrict__ x, const int64_t* __restrict__ cells,
                                              const T* __restrict__ value, int64_t e, int64_t nodes, TP* xs,
                                              T* coef, int64_t& node, int32_t* status) {
    const int lane = threadIdx.x & 31;
    node = lane < NPC ? cells[e * NPC + lane] : 0;
    if (__any_sync(0xffffffffu, lane < NPC && (node < 0 || node >= nodes))) {
        if (lane == 0) flag(status, AFSI_FLAG_INDEX);
        return false;
    }
    __syncwarp();
    const int64_t mine = __shfl_sync(0xffffffffu, node, lane < NPC * 3 ? lane / 3 : 0);
    if (lane < NPC * 3) {
        xs[lane] = x[mine * 3 + lane % 3];
        if (value) coef[lane] = value[mine * 3 + lane % 3];
    }
    __syncwarp();
    return true;
}

// ------------------------------------------------------------------ spread

template <class TP, class T, int NPC>
struct __align__(16) FSpreadStage {
    T w[2][FChunk<NPC>::value * 12];    // rows of both lattices: axis a weights at q*12 + a*4
    int b[2][FChunk<NPC>::value * 3];   // bases; b[0][q*3] == INT_MIN marks an invalid point
    T f[FChunk<NPC>::value];
    T coef[32];
    TP xs[32];
    T copy[2][kFSpreadCap];
};

// Padded strides of component c's box (p2.cu spread_layout).
__device__ __forceinline__ bool fspread_layout(const FBox& bx, const FusedDims& g, int c, int& sx, int& sy) {
    const int ey = bx.ext[c][1], ez = bx.ext[c][2];
    sy = sx = 0;
    if (!fcomponent_inside(bx, g, c) || ey > 64 || ez > 64) return false;
    sy = ez | 1;
    sx = ey * sy;
    sx += (12 - (sx & 7)) & 7;
    return int64_t(bx.ext[c][0]) * sx <= kFSpreadCap;
}

template <class F>
__device__ __forceinline__ void fbox_walk(int lane, int ex, int ey, int ez, F f) {
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

// Element boxes: from the resident rows when the rule fits one chunk (the
// rows are then formed once per element), else from a bases-only pass.
template <class TP, class T, int NPC, class Stage>
__device__ __forceinline__ bool element_rows_and_box(Stage& s, const TP* __restrict__ Npos, const FusedDims& g,
                                                     const Geo<TP>& geo, FBox& bx, int32_t* status) {
    if (g.nq <= FChunk<NPC>::value) {
        if (fill_rows<TP, T, NPC>(Npos, s.xs, 0, int(g.nq), geo, s.w[0], s.w[1], s.b[0], s.b[1]) &&
            (threadIdx.x & 31) == 0)
            flag(status, AFSI_FLAG_SUPPORT);
        __syncwarp();
        return box_from_rows(s.b[0], s.b[1], int(g.nq), bx);
    }
    return box_from_points<TP, T, NPC>(Npos, s.xs, g.nq, geo, bx, status);
}

template <class TP, class T, int NPC>
__global__ void __launch_bounds__(kFSpreadWarps * 32) fused_spread_kernel(
    const TP* __restrict__ x, const int64_t* __restrict__ cells, const TP* __restrict__ Npos,
    const T* __restrict__ N, const T* __restrict__ W, const T* __restrict__ value, Geo<TP> geo, T* __restrict__ u0,
    T* __restrict__ u1, T* __restrict__ u2, FusedDims g, T volume, int32_t* status) {
    extern __shared__ __align__(16) unsigned char fused_smem[];
    FSpreadStage<TP, T, NPC>& s = reinterpret_cast<FSpreadStage<TP, T, NPC>*>(fused_smem)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31, half = lane >> 4, li = (lane >> 2) & 3, lj = lane & 3;
    const int64_t warps = int64_t(gridDim.x) * kFSpreadWarps;
    const bool resident = g.nq <= FChunk<NPC>::value;
    for (int64_t e = int64_t(blockIdx.x) * kFSpreadWarps + (threadIdx.x >> 5); e < g.elements; e += warps) {
        int64_t node;
        if (!stage_element<TP, T, NPC>(x, cells, value, e, g.nodes, s.xs, s.coef, node, status)) continue;
        FBox bx;
        if (!element_rows_and_box<TP, T, NPC>(s, Npos, g, geo, bx, status)) continue;
        T* copy = s.copy[half];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            T* field = c == 0 ? u0 : c == 1 ? u1 : u2;
            const int tx = c != 0, ty = c != 1, tz = c != 2;
            int sx, sy;
            const bool fits = fspread_layout(bx, g, c, sx, sy);
            __syncwarp();
            if (fits)
                for (int t = lane; t < 2 * kFSpreadCap; t += 32) (&s.copy[0][0])[t] = T(0);
            for (int64_t q0 = 0; q0 < g.nq; q0 += FChunk<NPC>::value) {
                const int n = int(g.nq - q0 < FChunk<NPC>::value ? g.nq - q0 : FChunk<NPC>::value);
                __syncwarp();
                if (!resident) fill_rows<TP, T, NPC>(Npos, s.xs, q0, n, geo, s.w[0], s.w[1], s.b[0], s.b[1]);
                for (int q = lane; q < n; q += 32) {  // component c of the forces, lanes over points
                    if (s.b[0][q * 3] == INT_MIN) continue;
                    T F = T(0);
#pragma unroll
                    for (int a = 0; a < NPC; ++a) F += N[(q0 + q) * NPC + a] * s.coef[a * 3 + c];
                    s.f[q] = (F * W[e * g.nq + q0 + q]) / volume;
                }
                __syncwarp();
#pragma unroll 4
                for (int q = half; q < n; q += 2) {
                    if (s.b[0][q * 3] == INT_MIN) continue;
                    const int gx = s.b[tx][q * 3], gy = s.b[ty][q * 3 + 1], gz = s.b[tz][q * 3 + 2];
                    const T w = s.w[tx][q * 12 + li] * s.w[ty][q * 12 + 4 + lj];
                    using P = typename FPair<T>::type;
                    const P za = reinterpret_cast<const P*>(&s.w[tz][q * 12 + 8])[0];
                    const P zb = reinterpret_cast<const P*>(&s.w[tz][q * 12 + 8])[1];
                    const T wz[4] = {za.x, za.y, zb.x, zb.y};
                    const T fq = s.f[q];
                    if (fits) {
                        T* dst = copy + (gx - bx.lo[c][0] + li) * sx + (gy - bx.lo[c][1] + lj) * sy + (gz - bx.lo[c][2]);
#pragma unroll
                        for (int k = 0; k < 4; ++k) dst[k] += (w * wz[k]) * fq;
                    } else if (fpoint_inside(g, c, gx, gy, gz)) {
                        T* dst = field + ffield_index(g, c, gx + li, gy + lj, gz);
#pragma unroll
                        for (int k = 0; k < 4; ++k) atomicAdd(dst + k, (w * wz[k]) * fq);
                    } else if ((lane & 15) == 0) {
                        flag(status, AFSI_FLAG_INDEX);
                    }
                }
            }
            __syncwarp();
            if (fits) {
                fbox_walk(lane, bx.ext[c][0], bx.ext[c][1], bx.ext[c][2], [&](int, int xx, int yy, int zz) {
                    const int o = xx * sx + yy * sy + zz;
                    const T v = s.copy[0][o] + s.copy[1][o];
                    if (v != T(0))
                        atomicAdd(field + ffield_index(g, c, bx.lo[c][0] + xx, bx.lo[c][1] + yy, bx.lo[c][2] + zz), v);
                });
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------ gather

template <class TP, class T, int NPC>
struct __align__(16) FGatherStage {
    T w[2][FChunk<NPC>::value * 12];    // both lattices' rows: axis a at q*12 + a*4
    int b[2][FChunk<NPC>::value * 3];
    T patch[FPatch<T>::value];
    TP xs[32];
};

template <class TP, class T, int NPC, bool Local>
__global__ void __launch_bounds__(kFGatherWarps * 32) fused_gather_kernel(
    const T* __restrict__ u0, const T* __restrict__ u1, const T* __restrict__ u2, const TP* __restrict__ x,
    const int64_t* __restrict__ cells, const TP* __restrict__ Npos, const T* __restrict__ N, const T* __restrict__ W,
    Geo<TP> geo, T* __restrict__ out, FusedDims g, int32_t* status) {
    extern __shared__ __align__(16) unsigned char fused_smem[];
    FGatherStage<TP, T, NPC>& s = reinterpret_cast<FGatherStage<TP, T, NPC>*>(fused_smem)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31, grp = lane >> 3, li = (lane >> 1) & 3, ljp = lane & 1, sub = lane & 7;
    const int64_t warps = int64_t(gridDim.x) * kFGatherWarps;
    const bool resident = g.nq <= FChunk<NPC>::value;
    const T* fields[3] = {u0, u1, u2};
    for (int64_t e = int64_t(blockIdx.x) * kFGatherWarps + (threadIdx.x >> 5); e < g.elements; e += warps) {
        int64_t node;
        if (!stage_element<TP, T, NPC>(x, cells, static_cast<const T*>(nullptr), e, g.nodes, s.xs, nullptr, node,
                                        status))
            continue;
        FBox bx;
        const bool any = element_rows_and_box<TP, T, NPC>(s, Npos, g, geo, bx, status);
        int64_t cells_all = 0;
        bool fits = any;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            fits = fits && fcomponent_inside(bx, g, c);
            cells_all += int64_t(bx.ext[c][0]) * bx.ext[c][1] * bx.ext[c][2];
        }
        fits = fits && cells_all <= FPatch<T>::value;
        __syncwarp();
        if (fits) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
                fbox_walk(lane, bx.ext[c][0], bx.ext[c][1], bx.ext[c][2], [&](int t, int xx, int yy, int zz) {
                    s.patch[bx.off[c] + t] =
                        fields[c][ffield_index(g, c, bx.lo[c][0] + xx, bx.lo[c][1] + yy, bx.lo[c][2] + zz)];
                });
        }
        T acc[2][3] = {{T(0), T(0), T(0)}, {T(0), T(0), T(0)}};
        for (int64_t q0 = 0; q0 < g.nq && any; q0 += FChunk<NPC>::value) {
            const int n = int(g.nq - q0 < FChunk<NPC>::value ? g.nq - q0 : FChunk<NPC>::value);
            if (!resident) {
                __syncwarp();
                fill_rows<TP, T, NPC>(Npos, s.xs, q0, n, geo, s.w[0], s.w[1], s.b[0], s.b[1]);
            }
            __syncwarp();
#pragma unroll 2
            for (int qb = 0; qb < n; qb += 4) {
                const int q = qb + grp;
                const bool active = q < n && s.b[0][q * 3] != INT_MIN;
                const int qq = active ? q : 0;
                T U[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int tx = c != 0, ty = c != 1, tz = c != 2;
                    const int gx = s.b[tx][qq * 3], gy = s.b[ty][qq * 3 + 1], gz = s.b[tz][qq * 3 + 2];
                    const T wx = s.w[tx][qq * 12 + li];
                    using P = typename FPair<T>::type;
                    const P wy = reinterpret_cast<const P*>(&s.w[ty][qq * 12 + 4])[ljp];
                    const P za = reinterpret_cast<const P*>(&s.w[tz][qq * 12 + 8])[0];
                    const P zb = reinterpret_cast<const P*>(&s.w[tz][qq * 12 + 8])[1];
                    const T wz[4] = {za.x, za.y, zb.x, zb.y};
                    T s0 = T(0), s1 = T(0);
                    if (active) {
                        const T* src = nullptr;
                        int64_t sy = 0;
                        if (fits) {
                            src = s.patch + bx.off[c] +
                                  ((gx - bx.lo[c][0] + li) * bx.ext[c][1] + (gy - bx.lo[c][1] + 2 * ljp)) * bx.ext[c][2] +
                                  (gz - bx.lo[c][2]);
                            sy = bx.ext[c][2];
                        } else if (fpoint_inside(g, c, gx, gy, gz)) {
                            src = fields[c] + ffield_index(g, c, gx + li, gy + 2 * ljp, gz);
                            sy = g.nz + (c == 2);
                        } else if (sub == 0) {
                            flag(status, AFSI_FLAG_INDEX);
                        }
                        if (src) {
#pragma unroll
                            for (int k = 0; k < 4; ++k) {
                                s0 = fma(src[k], wz[k], s0);
                                s1 = fma(src[sy + k], wz[k], s1);
                            }
                        }
                    }
                    T sum = wx * (wy.x * s0 + wy.y * s1);
                    sum += __shfl_xor_sync(0xffffffffu, sum, 1);
                    sum += __shfl_xor_sync(0xffffffffu, sum, 2);
                    sum += __shfl_xor_sync(0xffffffffu, sum, 4);
                    U[c] = sum;
                }
                if (active) {
                    const T wq = W[e * g.nq + q0 + q];
#pragma unroll
                    for (int m = 0; m < 2; ++m) {
                        const int a = sub + 8 * m;
                        if (a < NPC) {
                            const T nw = N[(q0 + q) * NPC + a] * wq;
#pragma unroll
                            for (int c = 0; c < 3; ++c) acc[m][c] = fma(nw, U[c], acc[m][c]);
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int m = 0; m < 2; ++m)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                T v = acc[m][c];
                v += __shfl_xor_sync(0xffffffffu, v, 8);
                v += __shfl_xor_sync(0xffffffffu, v, 16);
                acc[m][c] = v;
            }
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const int a = sub + 8 * m;
            const int64_t nd = __shfl_sync(0xffffffffu, node, a < NPC ? a : 0);
            if (grp == 0 && a < NPC) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    if (Local)
                        out[(e * NPC + a) * 3 + c] = acc[m][c];
                    else
                        atomicAdd(out + nd * 3 + c, acc[m][c]);
                }
            }
        }
        __syncwarp();
    }
}

template <class TP>
Geo<TP> make_geo(const double* origin, const double* spacing, const double* limits) {
    Geo<TP> geo;
    for (int a = 0; a < 3; ++a) {
        geo.origin[a] = TP(origin[a]);
        geo.spacing[a] = TP(spacing[a]);
        geo.limits[a] = TP(limits[a]);
    }
    return geo;
}

int32_t check_fused(int32_t npc, int64_t nodes, int64_t elements, int64_t nq, int64_t nx, int64_t ny, int64_t nz,
                    const double* origin, const double* spacing, const double* limits, int32_t pos_dtype,
                    int32_t dtype) {
    AFSI_REQUIRE(npc == 10 || npc == 4, "nodes per cell must be 10 (P2) or 4 (P1)");
    AFSI_REQUIRE(nodes >= 0 && elements >= 0 && nq >= 1 && nq <= (int64_t(1) << 20), "invalid element counts");
    AFSI_REQUIRE(nx >= 4 && ny >= 4 && nz >= 4 && nx < (1 << 28) && ny < (1 << 28) && nz < (1 << 28),
                 "invalid MAC grid");
    AFSI_REQUIRE(origin && spacing && limits, "null geometry");
    AFSI_REQUIRE((pos_dtype == AFSI_F64 && (dtype == AFSI_F64 || dtype == AFSI_F32)) ||
                     (pos_dtype == AFSI_F32 && dtype == AFSI_F32),
                 "positions FP64 with FP64/FP32 transfers, or FP32 throughout");
    return AFSI_OK;
}

int fused_blocks(int64_t elements, int warps) {
    const int64_t b = (elements + warps - 1) / warps;
    return int(b < (int64_t(1) << 30) ? b : (int64_t(1) << 30));
}

#define AFSI_FUSED_DISPATCH(npc, pos_dtype, dtype, ...)                              \
    do {                                                                              \
        if ((pos_dtype) == AFSI_F64 && (dtype) == AFSI_F64) {                         \
            using TP = double; using T = double;                                      \
            if ((npc) == 10) { constexpr int NPC = 10; __VA_ARGS__; }                 \
            else { constexpr int NPC = 4; __VA_ARGS__; }                              \
        } else if ((pos_dtype) == AFSI_F64) {                                         \
            using TP = double; using T = float;                                       \
            if ((npc) == 10) { constexpr int NPC = 10; __VA_ARGS__; }                 \
            else { constexpr int NPC = 4; __VA_ARGS__; }                              \
        } else {                                                                      \
            using TP = float; using T = float;                                        \
            if ((npc) == 10) { constexpr int NPC = 10; __VA_ARGS__; }                 \
            else { constexpr int NPC = 4; __VA_ARGS__; }                              \
        }                                                                             \
    } while (0)

}  // namespace
}  // namespace afsi

using namespace afsi;

extern "C" int32_t afsi_b200_fe_fused_spread(int32_t nodes_per_cell, const void* x, int64_t nodes,
                                             const int64_t* cells, int64_t elements, const void* N_pos,
                                             const void* N, int64_t nq, const void* W, const void* value,
                                             const double* origin, const double* spacing, const double* limits,
                                             void* u0, void* u1, void* u2, int64_t nx, int64_t ny, int64_t nz,
                                             double volume, int32_t* status, int32_t pos_dtype, int32_t dtype,
                                             afsi_stream_t stream) {
    int32_t rc = check_fused(nodes_per_cell, nodes, elements, nq, nx, ny, nz, origin, spacing, limits, pos_dtype,
                             dtype);
    if (rc) return rc;
    AFSI_REQUIRE(isfinite(volume) && volume > 0, "invalid cell volume");
    if (elements == 0) return AFSI_OK;
    AFSI_REQUIRE(x && cells && N_pos && N && W && value && u0 && u1 && u2, "null device pointer");
    const FusedDims g{nx, ny, nz, nodes, elements, nq};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    AFSI_FUSED_DISPATCH(nodes_per_cell, pos_dtype, dtype, {
        const size_t smem = sizeof(FSpreadStage<TP, T, NPC>) * kFSpreadWarps;
        static bool configured = false;  // once per instantiation, before any graph capture of it
        if (!configured) {
            cudaFuncSetAttribute(fused_spread_kernel<TP, T, NPC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem));
            configured = true;
        }
        fused_spread_kernel<TP, T, NPC><<<fused_blocks(elements, kFSpreadWarps), kFSpreadWarps * 32, smem, s>>>(
            static_cast<const TP*>(x), cells, static_cast<const TP*>(N_pos), static_cast<const T*>(N),
            static_cast<const T*>(W), static_cast<const T*>(value), make_geo<TP>(origin, spacing, limits),
            static_cast<T*>(u0), static_cast<T*>(u1), static_cast<T*>(u2), g, T(volume), status);
    });
    return launched(nodes_per_cell == 10 ? "p2_fused_spread" : "p1_fused_spread");
}

template <bool Local>
static int32_t fused_gather(int32_t nodes_per_cell, const void* x, int64_t nodes, const int64_t* cells,
                            int64_t elements, const void* N_pos, const void* N, int64_t nq, const void* W,
                            const void* u0, const void* u1, const void* u2, const double* origin,
                            const double* spacing, const double* limits, void* out, int64_t nx, int64_t ny,
                            int64_t nz, int32_t* status, int32_t pos_dtype, int32_t dtype, afsi_stream_t stream) {
    int32_t rc = check_fused(nodes_per_cell, nodes, elements, nq, nx, ny, nz, origin, spacing, limits, pos_dtype,
                             dtype);
    if (rc) return rc;
    if (elements == 0) return AFSI_OK;
    AFSI_REQUIRE(x && cells && N_pos && N && W && u0 && u1 && u2 && out, "null device pointer");
    const FusedDims g{nx, ny, nz, nodes, elements, nq};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    AFSI_FUSED_DISPATCH(nodes_per_cell, pos_dtype, dtype, {
        const size_t smem = sizeof(FGatherStage<TP, T, NPC>) * kFGatherWarps;
        static bool configured = false;  // once per instantiation, before any graph capture of it
        if (!configured) {
            cudaFuncSetAttribute(fused_gather_kernel<TP, T, NPC, Local>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem));
            configured = true;
        }
        fused_gather_kernel<TP, T, NPC, Local><<<fused_blocks(elements, kFGatherWarps), kFGatherWarps * 32, smem, s>>>(
            static_cast<const T*>(u0), static_cast<const T*>(u1), static_cast<const T*>(u2),
            static_cast<const TP*>(x), cells, static_cast<const TP*>(N_pos), static_cast<const T*>(N),
            static_cast<const T*>(W), make_geo<TP>(origin, spacing, limits), static_cast<T*>(out), g, status);
    });
    return launched(Local ? "fe_fused_gather_local" : (nodes_per_cell == 10 ? "p2_fused_gather" : "p1_fused_gather"));
}

extern "C" int32_t afsi_b200_fe_fused_gather(int32_t nodes_per_cell, const void* x, int64_t nodes,
                                             const int64_t* cells, int64_t elements, const void* N_pos,
                                             const void* N, int64_t nq, const void* W, const void* u0,
                                             const void* u1, const void* u2, const double* origin,
                                             const double* spacing, const double* limits, void* rhs, int64_t nx,
                                             int64_t ny, int64_t nz, int32_t* status, int32_t pos_dtype,
                                             int32_t dtype, afsi_stream_t stream) {
    return fused_gather<false>(nodes_per_cell, x, nodes, cells, elements, N_pos, N, nq, W, u0, u1, u2, origin,
                               spacing, limits, rhs, nx, ny, nz, status, pos_dtype, dtype, stream);
}

extern "C" int32_t afsi_b200_fe_fused_gather_local(int32_t nodes_per_cell, const void* x, int64_t nodes,
                                                   const int64_t* cells, int64_t elements, const void* N_pos,
                                                   const void* N, int64_t nq, const void* W, const void* u0,
                                                   const void* u1, const void* u2, const double* origin,
                                                   const double* spacing, const double* limits, void* local,
                                                   int64_t nx, int64_t ny, int64_t nz, int32_t* status,
                                                   int32_t pos_dtype, int32_t dtype, afsi_stream_t stream) {
    return fused_gather<true>(nodes_per_cell, x, nodes, cells, elements, N_pos, N, nq, W, u0, u1, u2, origin,
                              spacing, limits, local, nx, ny, nz, status, pos_dtype, dtype, stream);
}
