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
// weights (rounded once to T in the precision form).  Where the spacing of an
// axis is a power of two, (x - start) / h is formed as (x - start) * (1/h),
// which is the same correctly rounded value.
//
// Layout: one warp per element, the three components in turn.  The element's
// point positions are formed once (lanes over points, kept in shared memory
// for rules of at most one chunk); per component, lanes over points form the
// three weight rows the component reads (x, y, z: 12 values per point), its
// support origins and, for the spread, its force factors; the warp reduces
// the component's box.  The spread then accumulates runs of points with one
// support origin in registers and adds each run to a padded shared-memory box
// once (spread_runs, runs.cuh), flushed to the face array with one L2
// reduction per non-zero face.  The gather stages the component's face patch
// in the same padded layout, and four lane groups of eight walk contiguous
// quarters of the points, reloading their eight patch values only when the
// support origin changes.  A point whose support leaves the grid sets
// AFSI_FLAG_SUPPORT and is skipped; an element with a node id outside
// [0, nodes) sets AFSI_FLAG_INDEX and is skipped.
#include <climits>
#include <cmath>
#include <cub/device/device_radix_sort.cuh>
#include "common.cuh"
#include "peskin.cuh"
#include "runs.cuh"

namespace afsi {
namespace {

constexpr int kFWarps = 2;        // warps per block (spread and gather)
// Points whose rows are held at once: 64 for P2 (the common adaptive orders
// have 15 or 64 points), 32 for P1 (orders 2 and 3 have 8 and 27 points).
template <int NPC> struct FChunk { static constexpr int value = NPC == 10 ? 64 : 32; };
constexpr int kFBoxCap = 288;     // entries of one component's padded box (spread) or patch (gather)
constexpr int kDetBoxCap = 640;   // padded box of the deterministic spread (extents up to 8 x 8 x 8)
constexpr int kDetExt = 8;        // largest box extent per axis of the deterministic spread

struct FusedDims {
    int64_t nx, ny, nz, nodes, elements, nq;
};

template <class TP>
struct Geo {
    TP origin[3], spacing[3], limits[3], inv[3];
    int pow2;  // bit a: spacing[a] is a power of two (inv[a] = 1 / spacing[a] exactly)
};

// One component's box: lower corner and extents of the supports.
struct FBox {
    int lo[3], ext[3];
};

template <class T> struct FPair;
template <> struct FPair<double> { using type = double2; };
template <> struct FPair<float> { using type = float2; };

// (x - start) / h on lattice l of axis a.
template <class TP>
__device__ __forceinline__ TP lattice_scaled(const Geo<TP>& geo, TP x, int a, int l) {
    const TP start = l ? geo.origin[a] + TP(.5) * geo.spacing[a] : geo.origin[a];
    return ((geo.pow2 >> a) & 1) ? (x - start) * geo.inv[a] : (x - start) / geo.spacing[a];
}

// x_q = sum_a N[q,a] x[a] (fe_prepare_kernel: a in order, from zero) and its
// validity (every axis finite with 2 <= (x - origin)/h < n - 2).
template <class TP, int NPC>
__device__ __forceinline__ bool point_position(const TP* __restrict__ Npos, const TP* xs, int64_t q,
                                               const Geo<TP>& geo, TP pos[3]) {
    pos[0] = pos[1] = pos[2] = TP(0);
#pragma unroll
    for (int a = 0; a < NPC; ++a) {
        const TP nv = Npos[q * NPC + a];
#pragma unroll
        for (int d = 0; d < 3; ++d) pos[d] += nv * xs[a * 3 + d];
    }
    bool valid = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const TP s0 = lattice_scaled(geo, pos[a], a, 0);
        valid = valid && isfinite(s0) && s0 >= TP(2) && s0 < geo.limits[a];
    }
    return valid;
}

// Component c's support origins of a point (axis a on lattice a != c) and,
// with w != null, its weight rows w[a*4 + k].
template <class TP, class T>
__device__ __forceinline__ void component_rows(const Geo<TP>& geo, const TP pos[3], int c, int b[3], T* w) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const TP scaled = lattice_scaled(geo, pos[a], a, a != c);
        const int64_t lower = static_cast<int64_t>(floor(scaled - TP(1)));
        b[a] = int(lower);
        if (w) {
            TP r[4];
            peskin_radical(scaled - TP(lower) - TP(1), r);
#pragma unroll
            for (int k = 0; k < 4; ++k) w[a * 4 + k] = T(r[k]);
        }
    }
}

__device__ __forceinline__ void bounds_init(int mn[3], int mx[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        mn[a] = INT_MAX;
        mx[a] = INT_MIN;
    }
}

__device__ __forceinline__ void bounds_add(int mn[3], int mx[3], const int b[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        mn[a] = min(mn[a], b[a]);
        mx[a] = max(mx[a], b[a]);
    }
}

// Warp-reduce the per-lane bounds into the box; false when no point was valid.
__device__ __forceinline__ bool bounds_finish(int mn[3], int mx[3], FBox& bx) {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int d = 16; d; d >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], d));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], d));
        }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        bx.lo[a] = mn[a];
        bx.ext[a] = mx[a] == INT_MIN ? 0 : mx[a] - mn[a] + 4;
    }
    return mn[0] != INT_MAX;
}

__device__ __forceinline__ int64_t ffield_index(const FusedDims& g, int c, int x, int y, int z) {
    return (int64_t(x) * (g.ny + (c == 1)) + y) * (g.nz + (c == 2)) + z;
}

__device__ __forceinline__ bool fpoint_inside(const FusedDims& g, int c, int x, int y, int z) {
    return x >= 0 && y >= 0 && z >= 0 && x + 3 < g.nx + (c == 0) && y + 3 < g.ny + (c == 1) &&
           z + 3 < g.nz + (c == 2);
}

// Padded strides of component c's box; false when the box leaves the face
// array or does not fit `cap` entries (the element then takes the direct
// L2 path).
__device__ __forceinline__ bool fbox_layout(const FBox& bx, const FusedDims& g, int c, int& sx, int& sy, int cap) {
    const int64_t fe[3] = {g.nx + (c == 0), g.ny + (c == 1), g.nz + (c == 2)};
    bool inside = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) inside = inside && bx.lo[a] >= 0 && int64_t(bx.lo[a]) + bx.ext[a] <= fe[a];
    sx = sy = 0;
    if (!inside || bx.ext[1] > 64 || bx.ext[2] > 64) return false;
    padded_strides(bx.ext[1], bx.ext[2], sx, sy);
    return int64_t(bx.ext[0]) * sx <= cap;
}

template <class F>
__device__ __forceinline__ void fbox_walk(int lane, int ex, int ey, int ez, F f) {
    const int n = ex * ey * ez;
    if (lane >= n) return;
    const int qz = 32 % ez, q = 32 / ez, qy = q % ey, qx = q / ey;
    int z = lane % ez, r = lane / ez, y = r % ey, x = r / ey;
    for (int t = lane; t < n; t += 32) {
        f(x, y, z);
        z += qz;
        int carry = z >= ez ? 1 : 0;
        z -= carry * ez;
        y += qy + carry;
        carry = y >= ey ? 1 : 0;
        y -= carry * ey;
        x += qx + carry;
    }
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

// Per-warp shared memory of both kernels.
template <class TP, class T, int NPC, int Cap = kFBoxCap>
struct __align__(16) FStage {
    T w[(FChunk<NPC>::value + 1) * 12];  // one component's rows: x at q*12, y at q*12+4, z at q*12+8; the last stays zero
    TP pos[FChunk<NPC>::value * 3];    // positions of a resident rule
    int b[FChunk<NPC>::value * 3];     // support origins (absolute) of the component
    int key[FChunk<NPC>::value];       // run keys in the box, -1 for an invalid point
    T f[FChunk<NPC>::value + 1];       // spread: force factors of the component; the last stays zero
    T box[Cap];                        // padded box
    T coef[32];
    TP xs[32];
    int perm[4 * FChunk<NPC>::value];  // points grouped by key (spread_element)
    int rs[FChunk<NPC>::value + 1], rk[FChunk<NPC>::value];
};

// Positions of a resident rule (all nq <= chunk points) into s.pos; returns
// the validity bits in every lane (bit q) and flags an invalid point.
template <class TP, int NPC, class S>
__device__ __forceinline__ unsigned long long resident_positions(S& s, const TP* __restrict__ Npos, int n,
                                                                 const Geo<TP>& geo, int32_t* status) {
    const int lane = threadIdx.x & 31;
    unsigned long long valid = 0;
#pragma unroll
    for (int j = 0; j < FChunk<NPC>::value / 32; ++j) {
        const int q = lane + 32 * j;
        bool v = false;
        if (q < n) {
            TP pos[3];
            v = point_position<TP, NPC>(Npos, s.xs, q, geo, pos);
#pragma unroll
            for (int d = 0; d < 3; ++d) s.pos[q * 3 + d] = pos[d];
        }
        valid |= static_cast<unsigned long long>(__ballot_sync(0xffffffffu, v)) << (32 * j);
    }
    const unsigned long long all = n >= 64 ? ~0ull : ((1ull << n) - 1);
    if (valid != all && lane == 0) flag(status, AFSI_FLAG_SUPPORT);
    __syncwarp();
    return valid;
}

// Box of component c over all nq points (rules larger than one chunk),
// support origins only; invalid points set AFSI_FLAG_SUPPORT.
template <class TP, int NPC>
__device__ __forceinline__ bool component_box_all(const TP* __restrict__ Npos, const TP* xs, int64_t nq,
                                                  const Geo<TP>& geo, int c, FBox& bx, int32_t* status) {
    int mn[3], mx[3];
    bounds_init(mn, mx);
    bool bad = false;
    for (int64_t q = threadIdx.x & 31; q < nq; q += 32) {
        TP pos[3];
        if (!point_position<TP, NPC>(Npos, xs, q, geo, pos)) {
            bad = true;
            continue;
        }
        int b[3];
        component_rows<TP, float>(geo, pos, c, b, nullptr);
        bounds_add(mn, mx, b);
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) flag(status, AFSI_FLAG_SUPPORT);
    return bounds_finish(mn, mx, bx);
}

// Rows pass of component c over points q0 .. q0+n-1 (lanes over points):
// weight rows and absolute support origins into shared memory, the spread's
// force factors when coef != null; the bounds of the valid points' origins
// are added to mn/mx.  Invalid points get b[q*3] = INT_MIN.
template <class TP, class T, int NPC, int Cap>
__device__ __forceinline__ void component_pass(FStage<TP, T, NPC, Cap>& s, const TP* __restrict__ Npos,
                                               const T* __restrict__ N, const T* __restrict__ W, bool resident,
                                               unsigned long long valid_bits, int64_t e, int64_t nq, int64_t q0,
                                               int n, const Geo<TP>& geo, int c, const T* coef, T volume, T inv_volume, int mn[3],
                                               int mx[3]) {
    const int lane = threadIdx.x & 31;
#pragma unroll 1
    for (int j = 0; j < FChunk<NPC>::value / 32; ++j) {
        const int q = lane + 32 * j;
        if (q >= n) continue;
        TP pos[3];
        bool v;
        if (resident) {
#pragma unroll
            for (int d = 0; d < 3; ++d) pos[d] = s.pos[q * 3 + d];
            v = (valid_bits >> q) & 1;
        } else {
            v = point_position<TP, NPC>(Npos, s.xs, q0 + q, geo, pos);
        }
        if (!v) {
            s.b[q * 3] = INT_MIN;
            continue;
        }
        int b[3];
        component_rows<TP, T>(geo, pos, c, b, &s.w[q * 12]);
#pragma unroll
        for (int a = 0; a < 3; ++a) s.b[q * 3 + a] = b[a];
        bounds_add(mn, mx, b);
        if (coef) {
            T F = T(0);
#pragma unroll
            for (int a = 0; a < NPC; ++a) F += N[(q0 + q) * NPC + a] * coef[a * 3 + c];
            const T fw = F * W[e * nq + q0 + q];
            s.f[q] = inv_volume != T(0) ? fw * inv_volume : fw / volume;
        }
    }
}

// Run keys of points 0..n-1 in box bx (-1 for invalid points, or all -1 when
// the box does not fit).
template <class TP, class T, int NPC, int Cap>
__device__ __forceinline__ void component_keys(FStage<TP, T, NPC, Cap>& s, int n, const FBox& bx, bool fits) {
    for (int q = threadIdx.x & 31; q < n; q += 32) {
        const int bx0 = s.b[q * 3];
        s.key[q] = (fits && bx0 != INT_MIN)
                       ? run_key(bx0 - bx.lo[0], s.b[q * 3 + 1] - bx.lo[1], s.b[q * 3 + 2] - bx.lo[2])
                       : -1;
    }
}

// ------------------------------------------------------------------ spread

// Element boxes of the deterministic form: box b = e * 3 + c is component
// c's box of element e, stored dense (ext0 x ext1 x ext2, z fastest) in slot
// b of kDetSlot entries, with meta[b * 8 + 0..5] = lo0, lo1, lo2, ext0, ext1,
// ext2 (zeroed by the caller: ext0 == 0 is no box).
constexpr int kDetSlot = kDetExt * kDetExt * kDetExt;
constexpr int kDetMeta = 8;

// Mode 0: each element's box is added to the face arrays with L2
// reductions.  Modes 1 and 2 write it to its slot instead (plain stores), with
// extents up to kDetExt: mode 1 with the padded box of mode 0 (kFBoxCap
// entries, the same occupancy), queueing each (element, component) box that
// does not fit as e * 3 + c in `queue`; mode 2 takes only the queued boxes,
// with kDetBoxCap entries, and a box that still does not fit sets
// AFSI_FLAG_OVERFLOW and contributes nothing.
template <class TP, class T, int NPC, int Mode>
__global__ void __launch_bounds__(kFWarps * 32, 8) fused_spread_kernel(
    const TP* __restrict__ x, const int64_t* __restrict__ cells, const TP* __restrict__ Npos,
    const T* __restrict__ N, const T* __restrict__ W, const T* __restrict__ value, Geo<TP> geo, T* __restrict__ u0,
    T* __restrict__ u1, T* __restrict__ u2, FusedDims g, T volume, int32_t* status, T* __restrict__ slots,
    int32_t* __restrict__ meta, int32_t* __restrict__ queue, int32_t* __restrict__ queued) {
    extern __shared__ __align__(16) unsigned char fused_smem[];
    constexpr bool Boxes = Mode != 0;
    constexpr int Cap = Mode == 2 ? kDetBoxCap : kFBoxCap;
    FStage<TP, T, NPC, Cap>& s = reinterpret_cast<FStage<TP, T, NPC, Cap>*>(fused_smem)[threadIdx.x >> 5];
    constexpr int C = FChunk<NPC>::value;
    const int lane = threadIdx.x & 31, half = lane >> 4, li = (lane >> 2) & 3, lj = lane & 3;
    const int64_t warps = int64_t(gridDim.x) * kFWarps;
    const bool resident = g.nq <= C;
    const T inv_volume = exact_reciprocal(volume);
    if (lane < 12) s.w[C * 12 + lane] = T(0);
    if (lane == 0) s.f[C] = T(0);
    __syncwarp();
    const int64_t items = Mode == 2 ? int64_t(*queued) : g.elements;
    for (int64_t it = int64_t(blockIdx.x) * kFWarps + (threadIdx.x >> 5); it < items; it += warps) {
        const int64_t e = Mode == 2 ? int64_t(queue[it]) / 3 : it;
        const int only = Mode == 2 ? queue[it] % 3 : -1;
        int64_t node;
        if (!stage_element<TP, T, NPC>(x, cells, value, e, g.nodes, s.xs, s.coef, node, status)) continue;
        const unsigned long long valid =
            resident ? resident_positions<TP, NPC>(s, Npos, int(g.nq), geo, status) : 0ull;
#pragma unroll 1
        for (int c = 0; c < 3; ++c) {
            if (Mode == 2 && c != only) continue;
            T* field = c == 0 ? u0 : c == 1 ? u1 : u2;
            FBox bx;
            bool any = true;
            if (!resident) any = component_box_all<TP, NPC>(Npos, s.xs, g.nq, geo, c, bx, status);
            int sx = 0, sy = 0;
            bool fits = false;
            for (int64_t q0 = 0; q0 < g.nq && any; q0 += C) {
                const int n = int(g.nq - q0 < C ? g.nq - q0 : C);
                __syncwarp();
                int mn[3], mx[3];
                bounds_init(mn, mx);
                component_pass(s, Npos, N, W, resident, valid, e, g.nq, q0, n, geo, c, s.coef, volume,
                                           inv_volume, mn, mx);
                if (resident) {
                    any = bounds_finish(mn, mx, bx);
                    if (!any) break;
                }
                if (q0 == 0) {
                    fits = fbox_layout(bx, g, c, sx, sy, Cap) &&
                           (!Boxes || (bx.ext[0] <= kDetExt && bx.ext[1] <= kDetExt && bx.ext[2] <= kDetExt));
                    if (fits)
                        for (int t = lane; t < Cap; t += 32) s.box[t] = T(0);
                }
                __syncwarp();
                component_keys(s, n, bx, fits);
                __syncwarp();
                if (fits) {
                    spread_element<T, C>(s.box, s.key, s.f, s.w, s.w + 4, s.w + 8, n, sx, sy, s.perm, s.rs, s.rk);
                } else if (Mode == 1) {
                    if (lane == 0) queue[atomicAdd(queued, 1)] = int32_t(e * 3 + c);
                    break;
                } else if (Mode == 2) {
                    if (lane == 0) flag(status, AFSI_FLAG_OVERFLOW);
                    break;
                } else {
                    for (int q = half; q < n; q += 2) {
                        const int gx = s.b[q * 3], gy = s.b[q * 3 + 1], gz = s.b[q * 3 + 2];
                        if (gx == INT_MIN) continue;
                        if (fpoint_inside(g, c, gx, gy, gz)) {
                            const T w = (s.w[q * 12 + li] * s.w[q * 12 + 4 + lj]) * s.f[q];
                            T* dst = field + ffield_index(g, c, gx + li, gy + lj, gz);
#pragma unroll
                            for (int k = 0; k < 4; ++k) atomicAdd(dst + k, w * s.w[q * 12 + 8 + k]);
                        } else if ((lane & 15) == 0) {
                            flag(status, AFSI_FLAG_INDEX);
                        }
                    }
                }
            }
            __syncwarp();
            if (any && fits) {
                if (Boxes) {
                    const int64_t b = e * 3 + c;
                    T* slot = slots + b * kDetSlot;
                    const int ey = bx.ext[1], ez = bx.ext[2];
                    fbox_walk(lane, bx.ext[0], ey, ez, [&](int xx, int yy, int zz) {
                        slot[(xx * ey + yy) * ez + zz] = s.box[xx * sx + yy * sy + zz];
                    });
                    const int mv = lane == 0   ? bx.lo[0]
                                   : lane == 1 ? bx.lo[1]
                                   : lane == 2 ? bx.lo[2]
                                   : lane == 3 ? bx.ext[0]
                                   : lane == 4 ? ey
                                               : ez;
                    if (lane < 6) meta[b * kDetMeta + lane] = mv;
                } else {
                    fbox_walk(lane, bx.ext[0], bx.ext[1], bx.ext[2], [&](int xx, int yy, int zz) {
                        const T v = s.box[xx * sx + yy * sy + zz];
                        if (v != T(0))
                            atomicAdd(field + ffield_index(g, c, bx.lo[0] + xx, bx.lo[1] + yy, bx.lo[2] + zz), v);
                    });
                }
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------- deterministic reduction
//
// The element boxes (fused_spread_kernel modes 1 and 2) are added to the
// face arrays in a fixed order per face: every box names the 4x4x4 face
// tiles it overlaps (at most three per axis), the (tile, box) pairs are
// sorted by tile with a stable radix sort (a tile's boxes stay in the order
// of their key slots, a function of the boxes alone), and one CTA per tile
// adds, face by face, the covering boxes' entries in an order fixed by that
// list (det_box_reduce_kernel).  Small tiles keep the box list short: on a
// shell, 8x8x8 tiles put up to about 5000 boxes in one tile.  No atomics:
// the result is bitwise the same on every run, and equals the L2-reduction
// spread to rounding.

constexpr int kDetTile = 4;
constexpr int kDetKeys = 27;  // tile keys per box

struct DetTiles {
    int64_t n[3][3];  // tiles per axis of each component's face array
    int64_t first[4]; // first tile id of each component; first[3] = all tiles
};

inline DetTiles det_tiles(int64_t nx, int64_t ny, int64_t nz) {
    DetTiles t;
    int64_t acc = 0;
    for (int c = 0; c < 3; ++c) {
        const int64_t fe[3] = {nx + (c == 0), ny + (c == 1), nz + (c == 2)};
        for (int a = 0; a < 3; ++a) t.n[c][a] = (fe[a] + kDetTile - 1) / kDetTile;
        t.first[c] = acc;
        acc += t.n[c][0] * t.n[c][1] * t.n[c][2];
    }
    t.first[3] = acc;
    return t;
}

// Keys of box b: the ids of the tiles it overlaps, then `none`, stored
// slot-major (key j of box b at j * boxes + b, so the stores of a warp are
// contiguous); a box that spans more than three tiles along an axis sets
// AFSI_FLAG_OVERFLOW.
__global__ void det_box_keys_kernel(const int32_t* __restrict__ meta, int64_t boxes, DetTiles t, uint32_t none,
                                    uint32_t* __restrict__ keys, int32_t* __restrict__ vals, int32_t* status) {
    for (int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; b < boxes; b += int64_t(gridDim.x) * blockDim.x) {
        const int32_t* m = meta + b * kDetMeta;
        const int c = int(b % 3);
        const int64_t first = c == 2 ? t.first[2] : c == 1 ? t.first[1] : t.first[0];
        const int64_t n1 = c == 2 ? t.n[2][1] : c == 1 ? t.n[1][1] : t.n[0][1];
        const int64_t n2 = c == 2 ? t.n[2][2] : c == 1 ? t.n[1][2] : t.n[0][2];
        int j = 0;
        if (m[3] > 0) {
            int lo[3], hi[3];
            bool ok = true;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                lo[a] = m[a] / kDetTile;
                hi[a] = (m[a] + m[3 + a] - 1) / kDetTile;
                ok = ok && hi[a] - lo[a] <= 2;
            }
            if (ok) {
                for (int i = lo[0]; i <= hi[0]; ++i)
                    for (int jy = lo[1]; jy <= hi[1]; ++jy)
                        for (int kz = lo[2]; kz <= hi[2]; ++kz) {
                            keys[j * boxes + b] = uint32_t(first + (int64_t(i) * n1 + jy) * n2 + kz);
                            vals[j * boxes + b] = int32_t(b);
                            ++j;
                        }
            } else {
                flag(status, AFSI_FLAG_OVERFLOW);
            }
        }
        for (; j < kDetKeys; ++j) {
            keys[j * boxes + b] = none;
            vals[j * boxes + b] = int32_t(b);
        }
    }
}

// [start, end) of every tile's pairs in the sorted keys (zeroed by the
// caller: an absent tile keeps an empty range).
__global__ void det_box_ranges_kernel(const uint32_t* __restrict__ keys, int64_t n, uint32_t none,
                                      int32_t* __restrict__ start, int32_t* __restrict__ end) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const uint32_t k = keys[i];
        if (k == none) continue;
        if (i == 0 || keys[i - 1] != k) start[k] = int32_t(i);
        if (i + 1 == n || keys[i + 1] != k) end[k] = int32_t(i + 1);
    }
}

constexpr int kDetBatch = 64;   // boxes staged per step of the reduction
constexpr int kDetParts = 4;    // threads per face, each over its quarter of every staged batch
constexpr int kDetAhead = kDetBatch / kDetParts;  // loads a thread issues before adding them

// One CTA of 256 threads per tile: thread t takes face f = t % 64 of the
// tile ((f/16, f/4 % 4, f % 4)) and part q = t / 64.  The tile's boxes are
// staged 64 at a time; part q reads the entries of boxes 16q .. 16q+15 of
// each batch that cover its face (all 16 loads issued before the adds, so one
// memory round trip per batch rather than per box) and adds them in order to
// its partial sum; the face then adds the four partials in part order.  The
// association is fixed by the tile's box list alone: bitwise reproducible.
template <class T>
__global__ void __launch_bounds__(kDetBatch * kDetParts) det_box_reduce_kernel(
    const T* __restrict__ slots, const int32_t* __restrict__ meta, const int32_t* __restrict__ vals,
    const int32_t* __restrict__ start, const int32_t* __restrict__ end, DetTiles t, FusedDims g, T* __restrict__ u0,
    T* __restrict__ u1, T* __restrict__ u2) {
    __shared__ int4 s_lo[kDetBatch], s_ext[kDetBatch];
    __shared__ T part[kDetParts][kDetBatch];
    const int64_t tile = blockIdx.x;
    const int s0 = start[tile], e0 = end[tile];
    if (s0 >= e0) return;
    const int c = tile >= t.first[2] ? 2 : tile >= t.first[1] ? 1 : 0;
    const int64_t r = tile - (c == 2 ? t.first[2] : c == 1 ? t.first[1] : t.first[0]);
    const int64_t n1 = c == 2 ? t.n[2][1] : c == 1 ? t.n[1][1] : t.n[0][1];
    const int64_t n2 = c == 2 ? t.n[2][2] : c == 1 ? t.n[1][2] : t.n[0][2];
    const int64_t tz = r % n2, ty = (r / n2) % n1, tx = r / (n2 * n1);
    const int th = threadIdx.x, f = th % kDetBatch, q = th / kDetBatch;
    const int fx = int(tx) * kDetTile + (f >> 4), fy = int(ty) * kDetTile + ((f >> 2) & 3),
              fz = int(tz) * kDetTile + (f & 3);
    const int64_t fe0 = g.nx + (c == 0), fe1 = g.ny + (c == 1), fe2 = g.nz + (c == 2);
    T acc = T(0);
    for (int i0 = s0; i0 < e0; i0 += kDetBatch) {
        const int n = min(kDetBatch, e0 - i0);
        __syncthreads();
        if (th < n) {
            const int b = vals[i0 + th];
            const int32_t* m = meta + int64_t(b) * kDetMeta;
            s_lo[th] = make_int4(m[0], m[1], m[2], b);
            s_ext[th] = make_int4(m[3], m[4], m[5], 0);
        }
        __syncthreads();
        T v[kDetAhead];
#pragma unroll
        for (int u = 0; u < kDetAhead; ++u) {
            const int j = q * kDetAhead + u;
            v[u] = T(0);
            if (j < n) {
                const int4 lo = s_lo[j], ex = s_ext[j];
                const int dx = fx - lo.x, dy = fy - lo.y, dz = fz - lo.z;
                if (unsigned(dx) < unsigned(ex.x) && unsigned(dy) < unsigned(ex.y) && unsigned(dz) < unsigned(ex.z))
                    v[u] = slots[int64_t(lo.w) * kDetSlot + (dx * ex.y + dy) * ex.z + dz];
            }
        }
#pragma unroll
        for (int u = 0; u < kDetAhead; ++u) acc += v[u];
    }
    part[q][f] = acc;
    __syncthreads();
    if (q == 0 && fx < fe0 && fy < fe1 && fz < fe2) {
        T* field = c == 0 ? u0 : c == 1 ? u1 : u2;
        T* out = field + (int64_t(fx) * fe1 + fy) * fe2 + fz;
        T sum = part[0][f];
#pragma unroll
        for (int k = 1; k < kDetParts; ++k) sum += part[k][f];
        *out = *out + sum;
    }
}

// Scratch of the deterministic table-free spread of `elements` elements:
// slots, meta, keys and values (in and out), tile ranges, sort temporary.
struct DetBoxLayout {
    int64_t slots, meta, keys_in, keys_out, vals_in, vals_out, start, end, queue, queued, temp, temp_bytes, bytes;
    int bits;
};

inline int64_t det_align(int64_t v) { return (v + 255) / 256 * 256; }

inline int det_key_bits(int64_t limit) {
    int bits = 1;
    while (bits < 32 && (int64_t(1) << bits) <= limit) ++bits;
    return bits;
}

inline DetBoxLayout det_box_layout(int64_t elements, const DetTiles& t, int64_t esize) {
    DetBoxLayout L;
    const int64_t boxes = elements * 3, pairs = boxes * kDetKeys;
    int64_t off = 0;
    L.slots = off;
    off = det_align(off + boxes * kDetSlot * esize);
    L.meta = off;
    off = det_align(off + boxes * kDetMeta * 4);
    L.keys_in = off;
    off = det_align(off + pairs * 4);
    L.keys_out = off;
    off = det_align(off + pairs * 4);
    L.vals_in = off;
    off = det_align(off + pairs * 4);
    L.vals_out = off;
    off = det_align(off + pairs * 4);
    L.start = off;
    off = det_align(off + t.first[3] * 4);
    L.end = off;
    off = det_align(off + t.first[3] * 4);
    L.queue = off;
    off = det_align(off + boxes * 4);
    L.queued = off;
    off = det_align(off + 4);
    L.bits = det_key_bits(t.first[3]);
    size_t temp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, temp, static_cast<const uint32_t*>(nullptr),
                                    static_cast<uint32_t*>(nullptr), static_cast<const int32_t*>(nullptr),
                                    static_cast<int32_t*>(nullptr), int(pairs > 0 ? pairs : 1), 0, L.bits);
    L.temp = off;
    L.temp_bytes = int64_t(temp);
    L.bytes = det_align(off + L.temp_bytes);
    return L;
}

// ------------------------------------------------------------------ gather
//
// One lane per point: the lane forms the point's three weight rows of the
// component in registers and sums the 64 links over the component's face
// patch (support_dot over the fixed-stride patch of runs.cuh).  The
// velocities U_c(x_q) of a chunk are kept in shared memory and assembled by
// lanes (a, c) in point order: rhs[a][c] = sum_q N[q,a] W_q U_c(x_q).

constexpr int kGWarps = 4;

template <class TP, class T, int NPC>
struct __align__(16) FGStage {
    T patch[kGPatch];
    T u[3][FChunk<NPC>::value];
    T w[FChunk<NPC>::value];
    TP pos[FChunk<NPC>::value * 3];
    TP xs[32];
};

template <class TP, class T, int NPC, bool Local>
__global__ void __launch_bounds__(kGWarps * 32, 4) fused_gather_kernel(
    const T* __restrict__ u0, const T* __restrict__ u1, const T* __restrict__ u2, const TP* __restrict__ x,
    const int64_t* __restrict__ cells, const TP* __restrict__ Npos, const T* __restrict__ N, const T* __restrict__ W,
    Geo<TP> geo, T* __restrict__ out, FusedDims g, int32_t* status) {
    extern __shared__ __align__(16) unsigned char fused_smem[];
    FGStage<TP, T, NPC>& s = reinterpret_cast<FGStage<TP, T, NPC>*>(fused_smem)[threadIdx.x >> 5];
    constexpr int C = FChunk<NPC>::value, J = C / 32;
    const int lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * kGWarps;
    const bool resident = g.nq <= C;
    for (int64_t e = int64_t(blockIdx.x) * kGWarps + (threadIdx.x >> 5); e < g.elements; e += warps) {
        int64_t node;
        if (!stage_element<TP, T, NPC>(x, cells, static_cast<const T*>(nullptr), e, g.nodes, s.xs, nullptr, node,
                                        status))
            continue;
        const unsigned long long valid = resident ? resident_positions<TP, NPC>(s, Npos, int(g.nq), geo, status) : 0ull;
        FBox boxes[3];
        bool anys[3] = {true, true, true};
        if (!resident)
#pragma unroll 1
            for (int c = 0; c < 3; ++c) anys[c] = component_box_all<TP, NPC>(Npos, s.xs, g.nq, geo, c, boxes[c], status);
        T acc = T(0);  // lane (a, cc) = (lane / 3, lane % 3), lane < NPC * 3
        for (int64_t q0 = 0; q0 < g.nq; q0 += C) {
            const int n = int(g.nq - q0 < C ? g.nq - q0 : C);
            __syncwarp();
            for (int q = lane; q < n; q += 32) s.w[q] = W[e * g.nq + q0 + q];
#pragma unroll 1
            for (int c = 0; c < 3; ++c) {
                const T* field = c == 0 ? u0 : c == 1 ? u1 : u2;
                TP sc[J][3];
                int bb[J][3];
                bool vv[J];
                int mn[3], mx[3];
                bounds_init(mn, mx);
#pragma unroll
                for (int j = 0; j < J; ++j) {
                    const int q = lane + 32 * j;
                    vv[j] = false;
                    if (q < n) {
                        TP pos[3];
                        if (resident) {
#pragma unroll
                            for (int d = 0; d < 3; ++d) pos[d] = s.pos[q * 3 + d];
                            vv[j] = (valid >> q) & 1;
                        } else {
                            vv[j] = point_position<TP, NPC>(Npos, s.xs, q0 + q, geo, pos);
                        }
                        if (vv[j]) {
#pragma unroll
                            for (int a = 0; a < 3; ++a) {
                                sc[j][a] = lattice_scaled(geo, pos[a], a, a != c);
                                bb[j][a] = int(static_cast<int64_t>(floor(sc[j][a] - TP(1))));
                            }
                            bounds_add(mn, mx, bb[j]);
                        }
                    }
                }
                FBox bx;
                bool any;
                if (resident) {
                    any = bounds_finish(mn, mx, bx);
                } else {
                    bx = boxes[c];
                    any = anys[c];
                }
                const int64_t fe[3] = {g.nx + (c == 0), g.ny + (c == 1), g.nz + (c == 2)};
                bool fits = any;
#pragma unroll
                for (int a = 0; a < 3; ++a)
                    fits = fits && bx.lo[a] >= 0 && int64_t(bx.lo[a]) + bx.ext[a] <= fe[a] && bx.ext[a] <= kGExt;
                __syncwarp();  // the previous component's patch reads are done
                if (fits)
                    fbox_walk(lane, bx.ext[0], bx.ext[1], bx.ext[2], [&](int xx, int yy, int zz) {
                        s.patch[xx * kGSX + yy * kGSY + zz] =
                            field[ffield_index(g, c, bx.lo[0] + xx, bx.lo[1] + yy, bx.lo[2] + zz)];
                    });
                __syncwarp();
#pragma unroll
                for (int j = 0; j < J; ++j) {
                    const int q = lane + 32 * j;
                    if (q >= n) continue;
                    T U = T(0);
                    if (vv[j]) {
                        T wr[3][4];
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            TP r[4];
                            peskin_radical(sc[j][a] - TP(bb[j][a]) - TP(1), r);
#pragma unroll
                            for (int k = 0; k < 4; ++k) wr[a][k] = T(r[k]);
                        }
                        if (fits) {
                            const T* p0 = s.patch + (bb[j][0] - bx.lo[0]) * kGSX + (bb[j][1] - bx.lo[1]) * kGSY +
                                          (bb[j][2] - bx.lo[2]);
                            U = support_dot(p0, kGSX, kGSY, wr[0], wr[1], wr[2]);
                        } else if (fpoint_inside(g, c, bb[j][0], bb[j][1], bb[j][2])) {
                            const int64_t sz = g.nz + (c == 2), sy = (g.ny + (c == 1)) * sz;
                            U = support_dot(field + ffield_index(g, c, bb[j][0], bb[j][1], bb[j][2]), sy, sz, wr[0],
                                            wr[1], wr[2]);
                        } else {
                            flag(status, AFSI_FLAG_INDEX);
                        }
                    }
                    s.u[c][q] = U;
                }
            }
            __syncwarp();
            if (lane < NPC * 3) {
                const int a = lane / 3, cc = lane - 3 * (lane / 3);
                for (int q = 0; q < n; ++q) acc = fma(N[(q0 + q) * NPC + a] * s.w[q], s.u[cc][q], acc);
            }
        }
        const int64_t nd = __shfl_sync(0xffffffffu, node, lane < NPC * 3 ? lane / 3 : 0);
        if (lane < NPC * 3) {
            const int a = lane / 3, cc = lane - 3 * (lane / 3);
            if (Local)
                out[(e * NPC + a) * 3 + cc] = acc;
            else
                atomicAdd(out + nd * 3 + cc, acc);
        }
        __syncwarp();
    }
}

template <class TP>
Geo<TP> make_geo(const double* origin, const double* spacing, const double* limits) {
    Geo<TP> geo;
    geo.pow2 = 0;
    for (int a = 0; a < 3; ++a) {
        geo.origin[a] = TP(origin[a]);
        geo.spacing[a] = TP(spacing[a]);
        geo.limits[a] = TP(limits[a]);
        int ex = 0;
        const TP h = geo.spacing[a];
        // a power of two: its reciprocal is exact and x * (1/h) rounds as x / h
        const bool pow2 = std::isfinite(double(h)) && h > TP(0) && std::frexp(double(h), &ex) == 0.5 &&
                          TP(1) / h == TP(std::ldexp(1.0, 1 - ex)) && std::isnormal(double(TP(1) / h));
        geo.inv[a] = pow2 ? TP(1) / h : TP(0);
        if (pow2) geo.pow2 |= 1 << a;
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
        const size_t smem = sizeof(FStage<TP, T, NPC>) * kFWarps;
        static bool configured = false;  // once per instantiation, before any graph capture of it
        if (!configured) {
            cudaFuncSetAttribute(fused_spread_kernel<TP, T, NPC, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem));
            configured = true;
        }
        fused_spread_kernel<TP, T, NPC, 0><<<fused_blocks(elements, kFWarps), kFWarps * 32, smem, s>>>(
            static_cast<const TP*>(x), cells, static_cast<const TP*>(N_pos), static_cast<const T*>(N),
            static_cast<const T*>(W), static_cast<const T*>(value), make_geo<TP>(origin, spacing, limits),
            static_cast<T*>(u0), static_cast<T*>(u1), static_cast<T*>(u2), g, T(volume), status,
            static_cast<T*>(nullptr), static_cast<int32_t*>(nullptr), static_cast<int32_t*>(nullptr),
            static_cast<int32_t*>(nullptr));
    });
    return launched(nodes_per_cell == 10 ? "p2_fused_spread" : "p1_fused_spread");
}

extern "C" int64_t afsi_b200_fe_det_spread_bytes(int64_t elements, int64_t nx, int64_t ny, int64_t nz,
                                                 int32_t dtype) {
    if (elements < 0 || elements * 3 * kDetKeys >= (int64_t(1) << 31)) return -1;  // sort items are int
    if (nx < 4 || ny < 4 || nz < 4 || nx >= (1 << 28) || ny >= (1 << 28) || nz >= (1 << 28)) return -1;
    if (dtype != AFSI_F32 && dtype != AFSI_F64) return -1;
    const DetTiles t = det_tiles(nx, ny, nz);
    if (t.first[3] >= (int64_t(1) << 31)) return -1;
    return det_box_layout(elements, t, dtype == AFSI_F64 ? 8 : 4).bytes;
}

extern "C" int32_t afsi_b200_fe_det_spread(int32_t nodes_per_cell, const void* x, int64_t nodes,
                                           const int64_t* cells, int64_t elements, const void* N_pos,
                                           const void* N, int64_t nq, const void* W, const void* value,
                                           const double* origin, const double* spacing, const double* limits,
                                           void* u0, void* u1, void* u2, int64_t nx, int64_t ny, int64_t nz,
                                           double volume, void* scratch, int64_t scratch_bytes, int32_t* status,
                                           int32_t pos_dtype, int32_t dtype, afsi_stream_t stream) {
    int32_t rc = check_fused(nodes_per_cell, nodes, elements, nq, nx, ny, nz, origin, spacing, limits, pos_dtype,
                             dtype);
    if (rc) return rc;
    AFSI_REQUIRE(isfinite(volume) && volume > 0, "invalid cell volume");
    if (elements == 0) return AFSI_OK;
    AFSI_REQUIRE(x && cells && N_pos && N && W && value && u0 && u1 && u2 && scratch, "null device pointer");
    const int64_t need = afsi_b200_fe_det_spread_bytes(elements, nx, ny, nz, dtype);
    AFSI_REQUIRE(need >= 0, "too many elements or tiles for the deterministic spread");
    AFSI_REQUIRE(scratch_bytes >= need, "deterministic spread scratch too small (%lld of %lld bytes)",
                 static_cast<long long>(scratch_bytes), static_cast<long long>(need));
    const FusedDims g{nx, ny, nz, nodes, elements, nq};
    const DetTiles t = det_tiles(nx, ny, nz);
    const int64_t boxes = elements * 3, pairs = boxes * kDetKeys;
    const uint32_t none = uint32_t(t.first[3]);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* base = static_cast<unsigned char*>(scratch);
    AFSI_FUSED_DISPATCH(nodes_per_cell, pos_dtype, dtype, {
        const DetBoxLayout L = det_box_layout(elements, t, int64_t(sizeof(T)));
        T* slots = reinterpret_cast<T*>(base + L.slots);
        int32_t* meta = reinterpret_cast<int32_t*>(base + L.meta);
        uint32_t* keys_in = reinterpret_cast<uint32_t*>(base + L.keys_in);
        uint32_t* keys_out = reinterpret_cast<uint32_t*>(base + L.keys_out);
        int32_t* vals_in = reinterpret_cast<int32_t*>(base + L.vals_in);
        int32_t* vals_out = reinterpret_cast<int32_t*>(base + L.vals_out);
        int32_t* start = reinterpret_cast<int32_t*>(base + L.start);
        int32_t* end = reinterpret_cast<int32_t*>(base + L.end);
        int32_t* queue = reinterpret_cast<int32_t*>(base + L.queue);
        int32_t* queued = reinterpret_cast<int32_t*>(base + L.queued);
        if (cudaMemsetAsync(meta, 0, size_t(boxes) * kDetMeta * 4, s) != cudaSuccess ||
            cudaMemsetAsync(start, 0, size_t(t.first[3]) * 4, s) != cudaSuccess ||
            cudaMemsetAsync(end, 0, size_t(t.first[3]) * 4, s) != cudaSuccess ||
            cudaMemsetAsync(queued, 0, 4, s) != cudaSuccess)
            return fail(AFSI_ERR_CUDA, "deterministic spread: clearing the scratch failed");
        const Geo<TP> geo = make_geo<TP>(origin, spacing, limits);
        const size_t smem1 = sizeof(FStage<TP, T, NPC, kFBoxCap>) * kFWarps;
        const size_t smem2 = sizeof(FStage<TP, T, NPC, kDetBoxCap>) * kFWarps;
        static bool configured = false;  // once per instantiation, before any graph capture of it
        if (!configured) {
            cudaFuncSetAttribute(fused_spread_kernel<TP, T, NPC, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem1));
            cudaFuncSetAttribute(fused_spread_kernel<TP, T, NPC, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem2));
            configured = true;
        }
        fused_spread_kernel<TP, T, NPC, 1><<<fused_blocks(elements, kFWarps), kFWarps * 32, smem1, s>>>(
            static_cast<const TP*>(x), cells, static_cast<const TP*>(N_pos), static_cast<const T*>(N),
            static_cast<const T*>(W), static_cast<const T*>(value), geo, static_cast<T*>(u0), static_cast<T*>(u1),
            static_cast<T*>(u2), g, T(volume), status, slots, meta, queue, queued);
        if ((rc = launched("fe_det_spread boxes"))) return rc;
        // the boxes that did not fit the first pass's shared-memory box (none on most shells)
        fused_spread_kernel<TP, T, NPC, 2><<<unsigned(std::min<int64_t>(fused_blocks(elements, kFWarps), 148 * 4)),
                                             kFWarps * 32, smem2, s>>>(
            static_cast<const TP*>(x), cells, static_cast<const TP*>(N_pos), static_cast<const T*>(N),
            static_cast<const T*>(W), static_cast<const T*>(value), geo, static_cast<T*>(u0), static_cast<T*>(u1),
            static_cast<T*>(u2), g, T(volume), status, slots, meta, queue, queued);
        if ((rc = launched("fe_det_spread large boxes"))) return rc;
        det_box_keys_kernel<<<unsigned(std::min<int64_t>((boxes + 255) / 256, 148 * 32)), 256, 0, s>>>(
            meta, boxes, t, none, keys_in, vals_in, status);
        if ((rc = launched("fe_det_spread keys"))) return rc;
        size_t temp = size_t(L.temp_bytes);
        if (cub::DeviceRadixSort::SortPairs(base + L.temp, temp, keys_in, keys_out, vals_in, vals_out, int(pairs), 0,
                                            L.bits, s) != cudaSuccess)
            return fail(AFSI_ERR_CUDA, "deterministic spread: sort failed");
        det_box_ranges_kernel<<<unsigned(std::min<int64_t>((pairs + 255) / 256, 148 * 32)), 256, 0, s>>>(
            keys_out, pairs, none, start, end);
        if ((rc = launched("fe_det_spread ranges"))) return rc;
        det_box_reduce_kernel<T><<<unsigned(t.first[3]), kDetBatch * kDetParts, 0, s>>>(slots, meta, vals_out, start,
                                                                                        end, t, g,
                                                                      static_cast<T*>(u0), static_cast<T*>(u1),
                                                                      static_cast<T*>(u2));
        if ((rc = launched("fe_det_spread reduce"))) return rc;
    });
    return AFSI_OK;
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
        const size_t smem = sizeof(FGStage<TP, T, NPC>) * kGWarps;
        static bool configured = false;  // once per instantiation, before any graph capture of it
        if (!configured) {
            cudaFuncSetAttribute(fused_gather_kernel<TP, T, NPC, Local>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem));
            configured = true;
        }
        fused_gather_kernel<TP, T, NPC, Local><<<fused_blocks(elements, kGWarps), kGWarps * 32, smem, s>>>(
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
