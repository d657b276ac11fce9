// Deterministic, atomic-free spread over the shared IB tables.
//
// The atomic spreads (compact and P2) add each point's 64 links per component
// into the face arrays in whatever order the hardware schedules them, so
// results agree to rounding but not bitwise from run to run.  This mode fixes
// every summation order:
//   plan (once per stencil)  each point's component-c support origin gives its
//                            owning 8x8x8 face tile; the points are sorted by
//                            tile (stable radix sort: ties keep point order),
//                            with per-tile ranges;
//   chunks                   each tile's sorted rows in chunks of kChunkRows;
//                            one CTA per chunk: warp w takes the chunk's rows
//                            w, w+4, ... (kDetUnroll of them loaded together,
//                            added in order) into its own private 11x11x11
//                            box in shared memory (the tile plus the support
//                            overhang), the four boxes are summed in warp
//                            order and stored to the chunk's scratch slot;
//   halo reduction           every face adds the slots of the chunks of the
//                            (at most 8) tiles whose boxes cover it, in a
//                            fixed order, to its field value (plain stores).
// Each link contribution is computed exactly as in the atomic kernels
// ((phi_x phi_y) phi_z) f, so the result equals theirs to rounding and is
// bitwise reproducible.  Points whose support leaves the face array are
// skipped and flag AFSI_FLAG_INDEX, as there.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include "common.cuh"

namespace afsi {

constexpr int kTile = 8;                         // faces per tile edge
constexpr int kHalo = kTile + 3;                 // tile box edge with the support overhang
constexpr int kBox = kHalo * kHalo * kHalo;      // 1331 entries per tile box
constexpr int kDetWarps = 4;
constexpr int kChunkRows = 256;  // rows per CTA
constexpr int kDetUnroll = 4;    // rows per warp whose loads are issued together

struct DetGrid {
    int64_t nx, ny, nz, total;
};

__host__ __device__ __forceinline__ int64_t face_extent(const DetGrid& g, int c, int a) {
    return (a == 0 ? g.nx : a == 1 ? g.ny : g.nz) + (a == c);
}

__host__ __device__ __forceinline__ int64_t tiles_along(const DetGrid& g, int c, int a) {
    return (face_extent(g, c, a) + kTile - 1) / kTile;
}

__host__ __device__ __forceinline__ int64_t tile_count(const DetGrid& g, int c) {
    return tiles_along(g, c, 0) * tiles_along(g, c, 1) * tiles_along(g, c, 2);
}

// Row of axis a of component c in the shared (2,T,3) tables: lattice a != c.
__device__ __forceinline__ int64_t det_row(int64_t total, int64_t p, int c, int a) {
    return ((int64_t(a != c) * total) + p) * 3 + a;
}

__global__ void det_keys_kernel(const int64_t* __restrict__ base, DetGrid g, int c, uint32_t* __restrict__ keys,
                                int32_t* __restrict__ idx, int32_t* status) {
    const int64_t tiles = tile_count(g, c);
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < g.total;
         p += int64_t(gridDim.x) * blockDim.x) {
        int64_t o[3];
        bool inside = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            o[a] = base[det_row(g.total, p, c, a)];
            inside = inside && o[a] >= 0 && o[a] + 3 < face_extent(g, c, a);
        }
        if (!inside) flag(status, AFSI_FLAG_INDEX);
        keys[p] = uint32_t(inside ? (o[0] / kTile * tiles_along(g, c, 1) + o[1] / kTile) * tiles_along(g, c, 2) +
                                        o[2] / kTile
                                  : tiles);
        idx[p] = int32_t(p);
    }
}

// start[t] = first sorted position with key >= t, t = 0..tiles.
__global__ void det_starts_kernel(const uint32_t* __restrict__ sorted, int64_t n, int64_t tiles,
                                  int64_t* __restrict__ start) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t <= tiles; t += int64_t(gridDim.x) * blockDim.x) {
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (int64_t(sorted[mid]) < t)
                lo = mid + 1;
            else
                hi = mid;
        }
        start[t] = lo;
    }
}

// chunks[t] = number of kChunkRows chunks of tile t (tiles+1 entries, last 0).
__global__ void det_chunk_count_kernel(const int64_t* __restrict__ start, int64_t tiles, int64_t* __restrict__ chunks) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t <= tiles; t += int64_t(gridDim.x) * blockDim.x)
        chunks[t] = t < tiles ? (start[t + 1] - start[t] + kChunkRows - 1) / kChunkRows : 0;
}

// chunk_tile / chunk_lo of every chunk from the tile starts and chunk offsets.
__global__ void det_chunk_table_kernel(const int64_t* __restrict__ start, const int64_t* __restrict__ first,
                                       int64_t tiles, int32_t* __restrict__ chunk_tile,
                                       int64_t* __restrict__ chunk_lo) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < tiles; t += int64_t(gridDim.x) * blockDim.x)
        for (int64_t k = first[t]; k < first[t + 1]; ++k) {
            chunk_tile[k] = int32_t(t);
            chunk_lo[k] = start[t] + (k - first[t]) * kChunkRows;
        }
}

template <class T>
__global__ void __launch_bounds__(kDetWarps * 32) det_tile_kernel(const T* __restrict__ force,
                                                                  const int64_t* __restrict__ base,
                                                                  const T* __restrict__ phi, DetGrid g, int c,
                                                                  const int32_t* __restrict__ idx,
                                                                  const int64_t* __restrict__ start,
                                                                  const int32_t* __restrict__ chunk_tile,
                                                                  const int64_t* __restrict__ chunk_lo,
                                                                  const int64_t* __restrict__ first,
                                                                  T* __restrict__ scratch) {
    extern __shared__ __align__(16) unsigned char det_smem[];
    T* copies = reinterpret_cast<T*>(det_smem);  // [kDetWarps][kBox]
    int32_t* rows = reinterpret_cast<int32_t*>(copies + kDetWarps * kBox);  // [kChunkRows]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t chunk = blockIdx.x;
    if (chunk >= first[tile_count(g, c)]) return;  // the grid covers the bound on the chunk count
    const int64_t tile = chunk_tile[chunk];
    const int64_t lo = chunk_lo[chunk];
    const int n = int(min(int64_t(kChunkRows), start[tile + 1] - lo));
    for (int i = threadIdx.x; i < kDetWarps * kBox; i += blockDim.x) copies[i] = T(0);
    for (int i = threadIdx.x; i < n; i += blockDim.x) rows[i] = idx[lo + i];
    __syncthreads();
    const int64_t ty_n = tiles_along(g, c, 1), tz_n = tiles_along(g, c, 2);
    const int64_t t0[3] = {tile / (ty_n * tz_n) * kTile, (tile / tz_n) % ty_n * kTile, tile % tz_n * kTile};
    T* box = copies + warp * kBox;
    // lane: x offset li, y offset lj, z offsets kz, kz+1
    const int li = lane >> 3, lj = (lane >> 1) & 3, kz = (lane & 1) * 2;
    for (int j0 = warp; j0 < n; j0 += kDetWarps * kDetUnroll) {
        int off[kDetUnroll];
        T w[kDetUnroll], z0[kDetUnroll], z1[kDetUnroll], fq[kDetUnroll];
#pragma unroll
        for (int u = 0; u < kDetUnroll; ++u) {  // loads of kDetUnroll rows in flight
            const int j = j0 + u * kDetWarps;
            off[u] = -1;
            if (j < n) {
                const int64_t p = rows[j];
                const int64_t rx = det_row(g.total, p, c, 0), ry = det_row(g.total, p, c, 1),
                              rz = det_row(g.total, p, c, 2);
                const int lx = int(base[rx] - t0[0]) + li, ly = int(base[ry] - t0[1]) + lj,
                          lz = int(base[rz] - t0[2]) + kz;
                off[u] = (lx * kHalo + ly) * kHalo + lz;
                w[u] = phi[rx * 4 + li] * phi[ry * 4 + lj];
                z0[u] = phi[rz * 4 + kz];
                z1[u] = phi[rz * 4 + kz + 1];
                fq[u] = force[p * 3 + c];
            }
        }
#pragma unroll
        for (int u = 0; u < kDetUnroll; ++u) {  // added in row order
            if (off[u] >= 0) {
                box[off[u]] += (w[u] * z0[u]) * fq[u];
                box[off[u] + 1] += (w[u] * z1[u]) * fq[u];
            }
            __syncwarp();
        }
    }
    __syncthreads();
    T* out = scratch + chunk * kBox;
    for (int i = threadIdx.x; i < kBox; i += blockDim.x) {
        T s = copies[i];
#pragma unroll
        for (int w = 1; w < kDetWarps; ++w) s = s + copies[w * kBox + i];
        out[i] = s;
    }
}

// field[x,y,z] += sum of the chunk slots of the tiles covering it: tiles with
// (dx,dy,dz) in lexicographic order, each tile's chunks in order.
template <class T>
__global__ void det_reduce_kernel(const T* __restrict__ scratch, const int64_t* __restrict__ first, DetGrid g, int c,
                                  T* __restrict__ field) {
    const int64_t n0 = face_extent(g, c, 0), n1 = face_extent(g, c, 1), n2 = face_extent(g, c, 2);
    const int64_t ty_n = tiles_along(g, c, 1), tz_n = tiles_along(g, c, 2);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n0 * n1 * n2;
         i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t x = i / (n1 * n2), y = (i / n2) % n1, z = i % n2;
        const int64_t tx = x / kTile, ty = y / kTile, tz = z / kTile;
        const int lx = int(x % kTile), ly = int(y % kTile), lz = int(z % kTile);
        T s = T(0);
#pragma unroll
        for (int dx = 0; dx < 2; ++dx)
#pragma unroll
            for (int dy = 0; dy < 2; ++dy)
#pragma unroll
                for (int dz = 0; dz < 2; ++dz) {
                    const int bx = lx + dx * kTile, by = ly + dy * kTile, bz = lz + dz * kTile;
                    if (tx - dx < 0 || ty - dy < 0 || tz - dz < 0 || bx >= kHalo || by >= kHalo || bz >= kHalo)
                        continue;
                    const int64_t t = ((tx - dx) * ty_n + (ty - dy)) * tz_n + (tz - dz);
                    const int o = (bx * kHalo + by) * kHalo + bz;
                    for (int64_t k = first[t]; k < first[t + 1]; ++k) s = s + scratch[k * kBox + o];
                }
        field[i] = field[i] + s;
    }
}

// Point forces of one P2 group, F_q = (sum_a N[q,a] coef[cell_a]) W[e,q] / volume,
// in the order of the atomic P2 spread.
template <class T>
__global__ void p2_point_force_kernel(const T* __restrict__ value, const int64_t* __restrict__ cells,
                                      const T* __restrict__ N, const T* __restrict__ W, int64_t elements, int64_t nq,
                                      int64_t nodes, int64_t offset, T volume, T* __restrict__ force,
                                      int32_t* status) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < elements * nq;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t e = t / nq, q = t % nq;
        T F[3] = {T(0), T(0), T(0)};
        bool ok = true;
#pragma unroll
        for (int a = 0; a < 10; ++a) {
            const int64_t node = cells[e * 10 + a];
            if (node < 0 || node >= nodes) {
                ok = false;
                continue;
            }
            const T nv = N[q * 10 + a];
#pragma unroll
            for (int c = 0; c < 3; ++c) F[c] += nv * value[node * 3 + c];
        }
        if (!ok) flag(status, AFSI_FLAG_INDEX);
        const T w = W[e * nq + q];
#pragma unroll
        for (int c = 0; c < 3; ++c) force[(offset + t) * 3 + c] = ok ? (F[c] * w) / volume : T(0);
    }
}

}  // namespace afsi

using namespace afsi;

namespace {

struct DetLayout {
    int64_t idx, start[3], first[3], chunk_tile[3], chunk_lo[3], scratch, keys_in, keys_out, idx_in, temp,
        temp_bytes, bytes, max_chunks[3];
};

int64_t align256(int64_t v) { return (v + 255) & ~int64_t(255); }

DetLayout det_layout(const DetGrid& g, int32_t dtype) {
    DetLayout L;
    const int64_t esize = dtype == AFSI_F64 ? 8 : 4;
    int64_t off = 0;
    L.idx = off;
    off = align256(off + 3 * g.total * 4);
    int64_t most = 0;
    for (int c = 0; c < 3; ++c) {
        const int64_t tiles = tile_count(g, c);
        L.max_chunks[c] = g.total / kChunkRows + tiles;  // every tile may end in a partial chunk
        most = std::max(most, L.max_chunks[c]);
        L.start[c] = off;
        off = align256(off + (tiles + 1) * 8);
        L.first[c] = off;
        off = align256(off + (tiles + 1) * 8);
        L.chunk_tile[c] = off;
        off = align256(off + L.max_chunks[c] * 4);
        L.chunk_lo[c] = off;
        off = align256(off + L.max_chunks[c] * 8);
    }
    L.scratch = off;
    off = align256(off + most * kBox * esize);
    L.keys_in = off;
    off = align256(off + g.total * 4);
    int64_t tiles_all = 0;
    for (int c = 0; c < 3; ++c) tiles_all = std::max(tiles_all, tile_count(g, c));
    L.keys_out = off;  // also the chunk counts before their scan
    off = align256(off + std::max<int64_t>(g.total * 4, (tiles_all + 1) * 8));
    L.idx_in = off;
    off = align256(off + g.total * 4);
    size_t a = 0, b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, a, static_cast<const uint32_t*>(nullptr),
                                    static_cast<uint32_t*>(nullptr), static_cast<const int32_t*>(nullptr),
                                    static_cast<int32_t*>(nullptr), g.total > 0 ? g.total : 1);
    int64_t tiles_max = 0;
    for (int c = 0; c < 3; ++c) tiles_max = std::max(tiles_max, tile_count(g, c));
    cub::DeviceScan::ExclusiveSum(nullptr, b, static_cast<const int64_t*>(nullptr), static_cast<int64_t*>(nullptr),
                                  tiles_max + 1);
    L.temp = off;
    L.temp_bytes = int64_t(std::max(a, b));
    L.bytes = align256(off + L.temp_bytes);
    return L;
}

int32_t det_check(int64_t total, int64_t nx, int64_t ny, int64_t nz, int32_t dtype) {
    AFSI_REQUIRE(total > 0 && total < (int64_t(1) << 31), "deterministic spread needs 1..2^31-1 table rows");
    AFSI_REQUIRE(nx > 0 && ny > 0 && nz > 0 && (nx + 1) * (ny + 1) * (nz + 1) < (int64_t(1) << 31),
                 "invalid MAC grid for the deterministic spread");
    AFSI_REQUIRE(dtype == AFSI_F32 || dtype == AFSI_F64, "unsupported dtype code %d", int(dtype));
    return AFSI_OK;
}

int key_bits(int64_t limit) {
    int bits = 1;
    while (bits < 32 && (int64_t(1) << bits) <= limit) ++bits;
    return bits;
}

}  // namespace

extern "C" int64_t afsi_b200_det_plan_bytes(int64_t total, int64_t nx, int64_t ny, int64_t nz, int32_t dtype) {
    if (det_check(total, nx, ny, nz, dtype)) return -1;
    return det_layout(DetGrid{nx, ny, nz, total}, dtype).bytes;
}

extern "C" int32_t afsi_b200_det_plan(const int64_t* base, int64_t total, int64_t nx, int64_t ny, int64_t nz,
                                      void* plan, int64_t plan_bytes, int32_t* status, int32_t dtype,
                                      afsi_stream_t stream) {
    int32_t rc = det_check(total, nx, ny, nz, dtype);
    if (rc) return rc;
    AFSI_REQUIRE(base && plan, "null deterministic-spread argument");
    const DetGrid g{nx, ny, nz, total};
    const DetLayout L = det_layout(g, dtype);
    AFSI_REQUIRE(plan_bytes >= L.bytes, "deterministic-spread plan buffer too small");
    unsigned char* b = static_cast<unsigned char*>(plan);
    const unsigned blocks = unsigned(std::min<int64_t>((total + 255) / 256, 148 * 32));
    for (int c = 0; c < 3; ++c) {
        uint32_t* keys_in = reinterpret_cast<uint32_t*>(b + L.keys_in);
        uint32_t* keys_out = reinterpret_cast<uint32_t*>(b + L.keys_out);
        int32_t* idx_in = reinterpret_cast<int32_t*>(b + L.idx_in);
        int32_t* idx_out = reinterpret_cast<int32_t*>(b + L.idx) + c * total;
        int64_t* start = reinterpret_cast<int64_t*>(b + L.start[c]);
        const int64_t tiles = tile_count(g, c);
        det_keys_kernel<<<blocks, 256, 0, stream>>>(base, g, c, keys_in, idx_in, status);
        if ((rc = launched("det spread keys"))) return rc;
        size_t temp = size_t(L.temp_bytes);
        if (cub::DeviceRadixSort::SortPairs(b + L.temp, temp, keys_in, keys_out, idx_in, idx_out, total, 0,
                                            key_bits(tiles), stream) != cudaSuccess)
            return fail(AFSI_ERR_CUDA, "deterministic spread: sort failed");
        det_starts_kernel<<<unsigned((tiles + 256) / 256), 256, 0, stream>>>(keys_out, total, tiles, start);
        if ((rc = launched("det spread tile starts"))) return rc;
        // chunks per tile, their offsets, and the chunk table
        int64_t* counts = reinterpret_cast<int64_t*>(b + L.keys_out);  // the sorted keys are no longer needed
        int64_t* first = reinterpret_cast<int64_t*>(b + L.first[c]);
        det_chunk_count_kernel<<<unsigned((tiles + 256) / 256), 256, 0, stream>>>(start, tiles, counts);
        if ((rc = launched("det spread chunk counts"))) return rc;
        temp = size_t(L.temp_bytes);
        if (cub::DeviceScan::ExclusiveSum(b + L.temp, temp, counts, first, tiles + 1, stream) != cudaSuccess)
            return fail(AFSI_ERR_CUDA, "deterministic spread: scan failed");
        det_chunk_table_kernel<<<unsigned((tiles + 255) / 256), 256, 0, stream>>>(
            start, first, tiles, reinterpret_cast<int32_t*>(b + L.chunk_tile[c]),
            reinterpret_cast<int64_t*>(b + L.chunk_lo[c]));
        if ((rc = launched("det spread chunk table"))) return rc;
    }
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_det_spread(const void* force, const int64_t* base, const void* phi, int64_t total,
                                        int64_t nx, int64_t ny, int64_t nz, void* plan, int64_t plan_bytes,
                                        void* u0, void* u1, void* u2, int32_t dtype, afsi_stream_t stream) {
    int32_t rc = det_check(total, nx, ny, nz, dtype);
    if (rc) return rc;
    AFSI_REQUIRE(force && base && phi && plan && u0 && u1 && u2, "null deterministic-spread argument");
    const DetGrid g{nx, ny, nz, total};
    const DetLayout L = det_layout(g, dtype);
    AFSI_REQUIRE(plan_bytes >= L.bytes, "deterministic-spread plan buffer too small");
    unsigned char* b = static_cast<unsigned char*>(plan);
    void* fields[3] = {u0, u1, u2};
    AFSI_DISPATCH(dtype, {
        const size_t smem = size_t(kDetWarps) * kBox * sizeof(T) + kChunkRows * sizeof(int32_t);
        static bool configured = false;  // once per instantiation, before any graph capture of it
        if (!configured) {
            cudaFuncSetAttribute(det_tile_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            configured = true;
        }
        for (int c = 0; c < 3; ++c) {
            const int64_t tiles = tile_count(g, c);
            T* scratch = reinterpret_cast<T*>(b + L.scratch);
            (void)tiles;
            det_tile_kernel<T><<<unsigned(L.max_chunks[c]), kDetWarps * 32, smem, stream>>>(
                static_cast<const T*>(force), base, static_cast<const T*>(phi), g, c,
                reinterpret_cast<const int32_t*>(b + L.idx) + c * total,
                reinterpret_cast<const int64_t*>(b + L.start[c]), reinterpret_cast<const int32_t*>(b + L.chunk_tile[c]),
                reinterpret_cast<const int64_t*>(b + L.chunk_lo[c]), reinterpret_cast<const int64_t*>(b + L.first[c]),
                scratch);
            if ((rc = launched("det spread tiles"))) return rc;
            const int64_t faces = face_extent(g, c, 0) * face_extent(g, c, 1) * face_extent(g, c, 2);
            det_reduce_kernel<T><<<unsigned(std::min<int64_t>((faces + 255) / 256, 148 * 32)), 256, 0, stream>>>(
                scratch, reinterpret_cast<const int64_t*>(b + L.first[c]), g, c, static_cast<T*>(fields[c]));
            if ((rc = launched("det spread halo reduction"))) return rc;
        }
    });
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_p2_point_forces(const void* value, int64_t nodes, const int64_t* cells,
                                             int64_t elements, const void* N, int64_t nq, const void* W,
                                             int64_t total, int64_t offset, double volume, void* force,
                                             int32_t* status, int32_t dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(elements >= 0 && nq > 0 && offset >= 0 && elements * nq <= total - offset,
                 "P2 point forces exceed the table rows");
    AFSI_REQUIRE(isfinite(volume) && volume > 0, "invalid cell volume");
    if (elements == 0) return AFSI_OK;
    AFSI_REQUIRE(value && cells && N && W && force, "null device pointer");
    AFSI_DISPATCH(dtype, {
        p2_point_force_kernel<T><<<unsigned(std::min<int64_t>((elements * nq + 255) / 256, 148 * 32)), 256, 0,
                                   stream>>>(static_cast<const T*>(value), cells, static_cast<const T*>(N),
                                             static_cast<const T*>(W), elements, nq, nodes, offset, T(volume),
                                             static_cast<T*>(force), status);
    });
    return launched("p2 point forces");
}
