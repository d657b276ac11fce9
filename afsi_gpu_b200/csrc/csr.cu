// P1 CSR operators for the B200.
//
// For component c of a P1 interaction rule, B_c[node, face] = Σ over the
// cells holding the node, Σ over the cell's quadrature points of
// W·N[q,a]·φx·φy·φz, over the faces of the point's 4x4x4 support.  The
// reference (mac/csrc/ib.cu:22-116) visits every face ("site") of each cell's
// support box with one warp per site, its lanes over the cell's points, and
// adds the four nodal sums into a hash keyed node·nf + face.
//
// Here one warp owns one cell: the cell's points are staged in shared memory
// (relative bases, the three 4-weight rows, W and the four shape values), and
// the lanes walk the box sites, each lane accumulating its site's four nodal
// sums over the staged points in point order (no shuffles, no per-site binary
// search).  The hash table semantics are the reference's, so a table built
// here is interchangeable with one built there: SplitMix64 finaliser bucket
// (mac/csrc/ib.cu:14-19), linear probing over at most 128 slots, a key
// claimed with a 64-bit CAS on -1, the value added atomically, zero values
// skipped, and the flag set to 1 on a negative key or a failed probe.  The
// cached form only looks keys up and streams the misses out.
//
// hash -> CSR: empty slots become a sentinel just above the largest valid
// key, the whole table is radix-sorted (CUB) on the bits the keys use, the
// row boundaries come from one pass over the sorted keys, and the transpose
// is a second sort on column-major keys.  No host synchronisation: the
// number of entries and the validity flags land in a device info word.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <algorithm>
#include "common.cuh"

namespace afsi {

constexpr int kCellWarps = 4;        // warps per block in the contraction
constexpr int64_t kFar = 1 << 20;    // larger than any box extent: marks a point outside every site

__device__ __forceinline__ uint64_t hash_bucket(int64_t key, int64_t capacity) {
    uint64_t h = uint64_t(key);
    h = (h ^ (h >> 30)) * 0xbf58476d1ce4e5b9ull;
    h = (h ^ (h >> 27)) * 0x94d049bb133111ebull;
    return (h ^ (h >> 31)) & uint64_t(capacity - 1);
}

template <class T>
struct Table {
    int64_t* keys;
    T* values;
    int64_t capacity;
    int32_t* flag;
    // cached form: miss stream
    int64_t* mkeys;
    T* mvalues;
    unsigned long long* mcount;
    int64_t mcap;
};

template <class T, bool Cached>
__device__ void table_add(int64_t key, T value, const Table<T>& t) {
    if (value == T(0)) return;
    if (key < 0) {
        atomicExch(t.flag, 1);
        return;
    }
    uint64_t slot = hash_bucket(key, t.capacity);
    const uint64_t mask = uint64_t(t.capacity - 1);
    for (int probe = 0; probe < 128; ++probe, slot = (slot + 1) & mask) {
        int64_t previous;
        if (Cached)  // the key table is immutable during a cached launch
            previous = t.keys[slot];
        else
            previous = int64_t(atomicCAS(reinterpret_cast<unsigned long long*>(t.keys + slot), ~0ull,
                                         static_cast<unsigned long long>(key)));
        if (previous == key || (!Cached && previous == -1)) {
            atomicAdd(t.values + slot, value);
            return;
        }
        if (Cached && previous == -1) break;
    }
    if (Cached) {
        const unsigned long long i = atomicAdd(t.mcount, 1ull);
        if (i < static_cast<unsigned long long>(t.mcap)) {
            t.mkeys[i] = key;
            t.mvalues[i] = value;
        }
    } else {
        atomicExch(t.flag, 1);
    }
}

struct CellDims {
    int64_t total, offset, cells, nq, count, ny, nz, nf, nx;
    int c;
    bool shared;
};

template <class T>
struct CellStage {
    T phi[32][3][4];
    T w[32];
    T n[32][4];
    int d[32][3];
};

template <class T, bool Cached>
__global__ void __launch_bounds__(kCellWarps * 32) contract_kernel(const int64_t* __restrict__ base,
                                                                  const T* __restrict__ phi, const T* __restrict__ N,
                                                                  const T* __restrict__ W,
                                                                  const int64_t* __restrict__ cells,
                                                                  const int64_t* __restrict__ low,
                                                                  const int64_t* __restrict__ width,
                                                                  const int64_t* __restrict__ prefix, Table<T> t,
                                                                  CellDims g) {
    __shared__ CellStage<T> stage_all[kCellWarps];
    CellStage<T>& s = stage_all[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * kCellWarps;
    int lat[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) lat[a] = g.shared ? int(a != g.c) : g.c;
    for (int64_t e = int64_t(blockIdx.x) * kCellWarps + (threadIdx.x >> 5); e < g.cells; e += warps) {
        const int64_t first = prefix[e];
        if (first >= g.count) continue;
        const int64_t lx = low[e * 3], ly = low[e * 3 + 1], lz = low[e * 3 + 2];
        const int64_t wx = width[e * 3], wy = width[e * 3 + 1], wz = width[e * 3 + 2];
        const int64_t sites = prefix[e + 1] - first;
        if (wx <= 0 || wy <= 0 || wz <= 0 || wx > kFar || wy > kFar || wz > kFar || sites != wx * wy * wz) {
            if (lane == 0) atomicExch(t.flag, 1);  // malformed plan: nothing of this cell is added
            continue;
        }
        int64_t node[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) node[a] = cells[e * 4 + a];
        // site -> (sx, sy, sz), z fastest, advanced by mixed-radix addition of
        // 32 per batch (32-bit; the box extents are at most kFar)
        const int iwz = int(wz), iwy = int(wy);
        const int qz = 32 % iwz, qq = 32 / iwz, qy = qq % iwy, qx = qq / iwy;
        int sz = lane % iwz, sy = (lane / iwz) % iwy, sx = (lane / iwz) / iwy;
        for (int64_t t0 = 0; t0 < sites; t0 += 32) {
            const int64_t site = t0 + lane;
            T sums[4] = {T(0), T(0), T(0), T(0)};
            for (int64_t q0 = 0; q0 < g.nq; q0 += 32) {
                const int nj = int(g.nq - q0 < 32 ? g.nq - q0 : 32);
                if (t0 == 0 || g.nq > 32) {  // with one chunk, staged once for the first batch of sites
                    __syncwarp();
                    if (lane < nj) {
                        const int64_t row = g.offset + e * g.nq + q0 + lane;
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            const int64_t r = (int64_t(lat[a]) * g.total + row) * 3 + a;
                            const int64_t lo = a == 0 ? lx : a == 1 ? ly : lz;
                            const int64_t rel = base[r] - lo;
                            s.d[lane][a] = int(rel < 0 || rel > kFar ? kFar : rel);
#pragma unroll
                            for (int k = 0; k < 4; ++k) s.phi[lane][a][k] = phi[r * 4 + k];
                        }
                        s.w[lane] = W[e * g.nq + q0 + lane];
#pragma unroll
                        for (int a = 0; a < 4; ++a) s.n[lane][a] = N[(q0 + lane) * 4 + a];
                    }
                    __syncwarp();
                }
                for (int j = 0; j < nj; ++j) {
                    const unsigned dx = unsigned(sx - s.d[j][0]), dy = unsigned(sy - s.d[j][1]),
                                   dz = unsigned(sz - s.d[j][2]);
                    if (dx < 4u && dy < 4u && dz < 4u) {
                        const T k = ((s.phi[j][0][dx] * s.phi[j][1][dy]) * s.phi[j][2][dz]) * s.w[j];
#pragma unroll
                        for (int a = 0; a < 4; ++a) sums[a] += k * s.n[j][a];
                    }
                }
            }
            if (site < sites && first + site < g.count) {
                const int64_t gx = lx + sx, gy = ly + sy, gz = lz + sz;
                if (gx < 0 || gy < 0 || gz < 0 || gx >= g.nx || gy >= g.ny || gz >= g.nz) {
                    atomicExch(t.flag, 1);
                } else {
                    const int64_t face = (gx * g.ny + gy) * g.nz + gz;
#pragma unroll
                    for (int a = 0; a < 4; ++a) table_add<T, Cached>(node[a] * g.nf + face, sums[a], t);
                }
            }
            sz += qz;
            int carry = sz >= iwz ? 1 : 0;
            sz -= carry * iwz;
            sy += qy + carry;
            carry = sy >= iwy ? 1 : 0;
            sy -= carry * iwy;
            sx += qx + carry;
        }
    }
}

template <class T>
__global__ void accumulate_kernel(const int64_t* __restrict__ in_keys, const T* __restrict__ in_values, int64_t n,
                                  Table<T> t) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        table_add<T, false>(in_keys[i], in_values[i], t);
}

// low/width/size of every cell's support box for component c
// (mac/hash_transfer_assembly.py:122-138).
__global__ void plan_kernel(const int64_t* __restrict__ base, int64_t total, int64_t offset, int64_t cells,
                            int64_t nq, int c, bool shared, int64_t* __restrict__ low, int64_t* __restrict__ width,
                            int64_t* __restrict__ sizes) {
    const int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= cells) return;
    int64_t mn[3] = {INT64_MAX, INT64_MAX, INT64_MAX}, mx[3] = {INT64_MIN, INT64_MIN, INT64_MIN};
    for (int64_t q = 0; q < nq; ++q) {
        const int64_t row = offset + e * nq + q;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int lat = shared ? int(a != c) : c;
            const int64_t b = base[(int64_t(lat) * total + row) * 3 + a];
            mn[a] = b < mn[a] ? b : mn[a];
            mx[a] = b > mx[a] ? b : mx[a];
        }
    }
    int64_t size = 1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int64_t w = nq > 0 ? mx[a] - mn[a] + 4 : 0;
        low[e * 3 + a] = nq > 0 ? mn[a] : 0;
        width[e * 3 + a] = w;
        size *= w;
    }
    sizes[e] = size;
}

// Sort keys of the table: valid keys as they are, empty slots as the
// sentinel (the number of valid keys); counts entries and flags keys outside
// [0, sentinel) or nonfinite values (info[0] += entries, info[1] |= 1).
template <class T>
__global__ void table_keys_kernel(const int64_t* __restrict__ keys, const T* __restrict__ values, int64_t capacity,
                                  uint64_t sentinel, uint64_t* __restrict__ out, unsigned long long* info) {
    __shared__ unsigned long long block_count;
    if (threadIdx.x == 0) block_count = 0;
    __syncthreads();
    unsigned long long mine = 0;
    bool bad = false;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < capacity;
         i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t k = keys[i];
        if (k >= 0) {
            ++mine;
            bad = bad || uint64_t(k) >= sentinel || !isfinite(values[i]);
            out[i] = uint64_t(k);
        } else {
            out[i] = sentinel;
        }
    }
    atomicAdd(&block_count, mine);
    if (bad) atomicOr(info + 1, 1ull);
    __syncthreads();
    if (threadIdx.x == 0 && block_count) atomicAdd(info, block_count);
}

// Row pointers from sorted keys (row = key / divisor; sentinel and larger
// keys count as row `rows`): crow[r] = first index whose row >= r, i.e. the
// first key >= r * divisor, for r = 0..rows, one binary search per row (rows
// without entries cost no more than others, however long the run of them).
__global__ void row_pointers_kernel(const uint64_t* __restrict__ keys, int64_t n, uint64_t divisor, int64_t rows,
                                    int64_t* __restrict__ crow) {
    for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r <= rows;
         r += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t target = uint64_t(r) * divisor;
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            const int64_t mid = lo + ((hi - lo) >> 1);
            if (__ldg(keys + mid) < target)
                lo = mid + 1;
            else
                hi = mid;
        }
        crow[r] = lo;
    }
}

// minor[i] = key % divisor (the column) of every entry below the sentinel.
__global__ void minor_kernel(const uint64_t* __restrict__ keys, int64_t n, uint64_t sentinel, uint64_t divisor,
                             int64_t* __restrict__ minor) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t k = keys[i];
        if (k < sentinel) minor[i] = int64_t(k % divisor);
    }
}

// Column-major keys (col·rows + row) of the sorted B entries; sentinel past nnz.
__global__ void transpose_keys_kernel(const uint64_t* __restrict__ keys, int64_t n, uint64_t sentinel, uint64_t nf,
                                      uint64_t rows, uint64_t* __restrict__ out) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t k = keys[i];
        out[i] = k < sentinel ? (k % nf) * rows + k / nf : sentinel;
    }
}

// y[r·ys] = (Σ_j val[j]·x[col[j]·xs]) / divisor, L lanes per row.
template <class T, int L>
__global__ void csr_spmv_kernel(const int64_t* __restrict__ crow, const int64_t* __restrict__ col,
                                const T* __restrict__ val, int64_t rows, const T* __restrict__ x, int64_t xs,
                                T* __restrict__ y, int64_t ys, T divisor) {
    const int64_t groups = int64_t(gridDim.x) * blockDim.x / L;
    const int sub = threadIdx.x % L;
    for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / L; r < rows + (groups - rows % groups) % groups;
         r += groups) {
        T s = T(0);
        if (r < rows) {
            const int64_t a = crow[r], b = crow[r + 1];
            for (int64_t j = a + sub; j < b; j += L) s = fma(val[j], x[col[j] * xs], s);
        }
#pragma unroll
        for (int d = L / 2; d; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
        if (r < rows && sub == 0) y[r * ys] = s / divisor;
    }
}

inline int bit_length(uint64_t v) {
    int b = 0;
    while (v) {
        ++b;
        v >>= 1;
    }
    return b;
}

template <class T>
size_t sort_temp_bytes(int64_t capacity) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, static_cast<const uint64_t*>(nullptr),
                                    static_cast<uint64_t*>(nullptr), static_cast<const T*>(nullptr),
                                    static_cast<T*>(nullptr), int64_t(capacity));
    return bytes;
}

}  // namespace afsi

using namespace afsi;

namespace {

bool power_of_two(int64_t n) { return n > 0 && !(n & (n - 1)); }

template <class T>
Table<T> make_table(int64_t* keys, void* values, int64_t capacity, int32_t* flag) {
    Table<T> t;
    t.keys = keys;
    t.values = static_cast<T*>(values);
    t.capacity = capacity;
    t.flag = flag;
    t.mkeys = nullptr;
    t.mvalues = nullptr;
    t.mcount = nullptr;
    t.mcap = 0;
    return t;
}

int32_t contract(const int64_t* base, const void* phi, const void* N, const void* W, const int64_t* cells,
                 const int64_t* low, const int64_t* width, const int64_t* prefix, int64_t* keys, void* values,
                 int32_t* flag, int64_t capacity, int64_t* mkeys, void* mvalues, int64_t* mcount, int64_t mcap,
                 int64_t total, int64_t offset, int64_t elements, int64_t nq, int64_t count, int32_t component,
                 int64_t ny, int64_t nz, int64_t nf, int32_t shared, int32_t dtype, afsi_stream_t stream,
                 bool cached) {
    AFSI_REQUIRE(power_of_two(capacity), "power-of-two hash capacity required");
    AFSI_REQUIRE(elements >= 0 && nq > 0 && total >= 0, "invalid IB group sizes");
    AFSI_REQUIRE(offset >= 0 && offset <= total && elements * nq <= total - offset, "IB group offset is out of range");
    AFSI_REQUIRE(count >= 0 && (count == 0 || elements > 0) && component >= 0 && component < 3,
                 "invalid IB site count or component");
    AFSI_REQUIRE(ny > 0 && nz > 0 && nf > 0 && ny <= INT64_MAX / nz && nf % (ny * nz) == 0,
                 "invalid IB face dimensions");
    if (count == 0) return AFSI_OK;
    AFSI_REQUIRE(base && phi && N && W && cells && low && width && prefix && keys && values && flag,
                 "null device pointer");
    AFSI_REQUIRE(!cached || (mkeys && mvalues && mcount && mcap >= 0), "invalid IB missing stream");
    CellDims g;
    g.total = total;
    g.offset = offset;
    g.cells = elements;
    g.nq = nq;
    g.count = count;
    g.ny = ny;
    g.nz = nz;
    g.nf = nf;
    g.nx = nf / (ny * nz);
    g.c = component;
    g.shared = shared != 0;
    const int64_t want = (elements + kCellWarps - 1) / kCellWarps;
    const unsigned blocks = unsigned(want < 65535 * 8 ? want : 65535 * 8);
    AFSI_DISPATCH(dtype, {
        Table<T> t = make_table<T>(keys, values, capacity, flag);
        if (cached) {
            t.mkeys = mkeys;
            t.mvalues = static_cast<T*>(mvalues);
            t.mcount = reinterpret_cast<unsigned long long*>(mcount);
            t.mcap = mcap;
            contract_kernel<T, true><<<blocks, kCellWarps * 32, 0, stream>>>(
                base, static_cast<const T*>(phi), static_cast<const T*>(N), static_cast<const T*>(W), cells, low,
                width, prefix, t, g);
        } else {
            contract_kernel<T, false><<<blocks, kCellWarps * 32, 0, stream>>>(
                base, static_cast<const T*>(phi), static_cast<const T*>(N), static_cast<const T*>(W), cells, low,
                width, prefix, t, g);
        }
    });
    return launched(cached ? "cached_contract" : "hash_contract");
}

}  // namespace

extern "C" int32_t afsi_b200_hash_contract(const int64_t* base, const void* phi, const void* N, const void* W,
                                           const int64_t* cells, const int64_t* low, const int64_t* width,
                                           const int64_t* prefix, int64_t* keys, void* values, int32_t* flag,
                                           int64_t capacity, int64_t total, int64_t offset, int64_t elements,
                                           int64_t nq, int64_t count, int32_t component, int64_t ny, int64_t nz,
                                           int64_t nf, int32_t shared, int32_t dtype, afsi_stream_t stream) {
    return contract(base, phi, N, W, cells, low, width, prefix, keys, values, flag, capacity, nullptr, nullptr,
                    nullptr, 0, total, offset, elements, nq, count, component, ny, nz, nf, shared, dtype, stream,
                    false);
}

extern "C" int32_t afsi_b200_cached_contract(const int64_t* base, const void* phi, const void* N, const void* W,
                                             const int64_t* cells, const int64_t* low, const int64_t* width,
                                             const int64_t* prefix, const int64_t* keys, void* values,
                                             int32_t* flag, int64_t capacity, int64_t* missing_keys,
                                             void* missing_values, int64_t* missing_count, int64_t missing_capacity,
                                             int64_t total, int64_t offset, int64_t elements, int64_t nq,
                                             int64_t count, int32_t component, int64_t ny, int64_t nz, int64_t nf,
                                             int32_t shared, int32_t dtype, afsi_stream_t stream) {
    return contract(base, phi, N, W, cells, low, width, prefix, const_cast<int64_t*>(keys), values, flag, capacity,
                    missing_keys, missing_values, missing_count, missing_capacity, total, offset, elements, nq,
                    count, component, ny, nz, nf, shared, dtype, stream, true);
}

extern "C" int32_t afsi_b200_hash_accumulate(const int64_t* input_keys, const void* input_values, int64_t count,
                                             int64_t* keys, void* values, int32_t* flag, int64_t capacity,
                                             int32_t dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(power_of_two(capacity), "power-of-two hash capacity required");
    AFSI_REQUIRE(count >= 0, "negative entry count");
    if (count == 0) return AFSI_OK;
    AFSI_REQUIRE(input_keys && input_values && keys && values && flag, "null device pointer");
    const int64_t want = (count + 255) / 256;
    const unsigned blocks = unsigned(want < 65535 * 8 ? want : 65535 * 8);
    AFSI_DISPATCH(dtype, {
        accumulate_kernel<T><<<blocks, 256, 0, stream>>>(input_keys, static_cast<const T*>(input_values), count,
                                                         make_table<T>(keys, values, capacity, flag));
    });
    return launched("hash_accumulate");
}

extern "C" int64_t afsi_b200_p1_plan_scratch_bytes(int64_t elements) {
    size_t bytes = 0;
    cub::DeviceScan::InclusiveSum(nullptr, bytes, static_cast<const int64_t*>(nullptr),
                                  static_cast<int64_t*>(nullptr), elements > 0 ? elements : 1);
    return int64_t(bytes) + elements * 8 + 256;
}

extern "C" int32_t afsi_b200_p1_component_plan(const int64_t* base, int64_t total, int64_t offset,
                                               int64_t elements, int64_t nq, int32_t component, int32_t shared,
                                               int64_t* low, int64_t* width, int64_t* prefix, void* scratch,
                                               int64_t scratch_bytes, afsi_stream_t stream) {
    AFSI_REQUIRE(elements >= 0 && nq > 0 && component >= 0 && component < 3, "invalid IB plan arguments");
    AFSI_REQUIRE(offset >= 0 && offset <= total && elements * nq <= total - offset, "IB group offset is out of range");
    AFSI_REQUIRE(prefix, "null prefix");
    if (cudaMemsetAsync(prefix, 0, sizeof(int64_t), stream) != cudaSuccess)
        return fail(AFSI_ERR_CUDA, "prefix clear failed");
    if (elements == 0) return AFSI_OK;
    AFSI_REQUIRE(base && low && width && scratch, "null device pointer");
    AFSI_REQUIRE(scratch_bytes >= afsi_b200_p1_plan_scratch_bytes(elements), "plan scratch too small");
    int64_t* sizes = static_cast<int64_t*>(scratch);
    void* temp = static_cast<unsigned char*>(scratch) + ((elements * 8 + 255) / 256) * 256;
    size_t temp_bytes = size_t(scratch_bytes) - ((elements * 8 + 255) / 256) * 256;
    plan_kernel<<<blocks_for(elements, 256), 256, 0, stream>>>(base, total, offset, elements, nq, component,
                                                               shared != 0, low, width, sizes);
    int32_t rc = launched("p1_component_plan");
    if (rc) return rc;
    if (cub::DeviceScan::InclusiveSum(temp, temp_bytes, sizes, prefix + 1, elements, stream) != cudaSuccess)
        return fail(AFSI_ERR_CUDA, "box prefix scan failed");
    return launched("p1_component_plan scan");
}

// Blocks for one thread per row pointer (rows + 1 of them), at most 4096.
static unsigned rows_grid(int64_t rows) { return unsigned(rows / 256 + 1 < 4096 ? rows / 256 + 1 : 4096); }

extern "C" int64_t afsi_b200_hash_csr_scratch_bytes(int64_t capacity, int32_t dtype) {
    if (capacity <= 0) return 0;
    size_t temp = dtype == AFSI_F32 ? sort_temp_bytes<float>(capacity) : sort_temp_bytes<double>(capacity);
    return 2 * ((capacity * 8 + 255) / 256) * 256 + int64_t(temp) + 256;
}

extern "C" int32_t afsi_b200_hash_csr(const int64_t* keys, const void* values, int64_t capacity, int64_t rows,
                                      int64_t nf, int64_t* crow, int64_t* col, void* val, int64_t* t_crow,
                                      int64_t* t_col, void* t_val, int64_t* info, void* scratch,
                                      int64_t scratch_bytes, int32_t dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(power_of_two(capacity), "power-of-two hash capacity required");
    AFSI_REQUIRE(rows > 0 && nf > 0 && rows <= INT64_MAX / nf, "invalid CSR shape");
    AFSI_REQUIRE(keys && values && crow && col && val && t_crow && t_col && t_val && info && scratch,
                 "null device pointer");
    AFSI_REQUIRE(scratch_bytes >= afsi_b200_hash_csr_scratch_bytes(capacity, dtype), "CSR scratch too small");
    const uint64_t sentinel = uint64_t(rows) * uint64_t(nf);
    const int end_bit = bit_length(sentinel);
    const int64_t slab = ((capacity * 8 + 255) / 256) * 256;
    uint64_t* ka = static_cast<uint64_t*>(scratch);
    uint64_t* kb = reinterpret_cast<uint64_t*>(static_cast<unsigned char*>(scratch) + slab);
    void* temp = static_cast<unsigned char*>(scratch) + 2 * slab;
    size_t temp_bytes = size_t(scratch_bytes - 2 * slab);
    if (cudaMemsetAsync(info, 0, 2 * sizeof(int64_t), stream) != cudaSuccess)
        return fail(AFSI_ERR_CUDA, "info clear failed");
    const unsigned grid = unsigned(capacity / 256 + 1 < 4096 ? capacity / 256 + 1 : 4096);
    AFSI_DISPATCH(dtype, {
        table_keys_kernel<T><<<grid, 256, 0, stream>>>(keys, static_cast<const T*>(values), capacity, sentinel, ka,
                                                       reinterpret_cast<unsigned long long*>(info));
        int32_t rc = launched("hash_csr keys");
        if (rc) return rc;
        if (cub::DeviceRadixSort::SortPairs(temp, temp_bytes, ka, kb, static_cast<const T*>(values),
                                            static_cast<T*>(val), capacity, 0, end_bit, stream) != cudaSuccess)
            return fail(AFSI_ERR_CUDA, "CSR key sort failed");
        row_pointers_kernel<<<rows_grid(rows), 256, 0, stream>>>(kb, capacity, uint64_t(nf), rows, crow);
        minor_kernel<<<grid, 256, 0, stream>>>(kb, capacity, sentinel, uint64_t(nf), col);
        transpose_keys_kernel<<<grid, 256, 0, stream>>>(kb, capacity, sentinel, uint64_t(nf), uint64_t(rows), ka);
        if ((rc = launched("hash_csr rows"))) return rc;
        if (cub::DeviceRadixSort::SortPairs(temp, temp_bytes, ka, kb, static_cast<const T*>(val),
                                            static_cast<T*>(t_val), capacity, 0, end_bit, stream) != cudaSuccess)
            return fail(AFSI_ERR_CUDA, "CSR transpose sort failed");
        row_pointers_kernel<<<rows_grid(nf), 256, 0, stream>>>(kb, capacity, uint64_t(rows), nf, t_crow);
        minor_kernel<<<grid, 256, 0, stream>>>(kb, capacity, sentinel, uint64_t(rows), t_col);
    });
    return launched("hash_csr transpose");
}

extern "C" int32_t afsi_b200_csr_spmv(const int64_t* crow, const int64_t* col, const void* val, int64_t rows,
                                      int64_t nnz, const void* x, int64_t x_stride, void* y, int64_t y_stride,
                                      double divisor, int32_t dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(rows >= 0 && nnz >= 0 && x_stride > 0 && y_stride > 0 && divisor != 0.0, "invalid SpMV arguments");
    if (rows == 0) return AFSI_OK;
    AFSI_REQUIRE(crow && y && (nnz == 0 || (col && val && x)), "null device pointer");
    const int64_t avg = nnz / rows;
    AFSI_DISPATCH(dtype, {
        const T* v = static_cast<const T*>(val);
        const T* xv = static_cast<const T*>(x);
        T* yv = static_cast<T*>(y);
        if (avg >= 24) {
            const int64_t want = (rows * 32 + 255) / 256;
            const unsigned blocks = unsigned(want < 148 * 64 ? want : 148 * 64);
            csr_spmv_kernel<T, 32><<<blocks, 256, 0, stream>>>(crow, col, v, rows, xv, x_stride, yv, y_stride,
                                                               T(divisor));
        } else if (avg >= 6) {
            const int64_t want = (rows * 8 + 255) / 256;
            const unsigned blocks = unsigned(want < 148 * 64 ? want : 148 * 64);
            csr_spmv_kernel<T, 8><<<blocks, 256, 0, stream>>>(crow, col, v, rows, xv, x_stride, yv, y_stride,
                                                              T(divisor));
        } else {
            const int64_t want = (rows * 4 + 255) / 256;
            const unsigned blocks = unsigned(want < 148 * 64 ? want : 148 * 64);
            csr_spmv_kernel<T, 4><<<blocks, 256, 0, stream>>>(crow, col, v, rows, xv, x_stride, yv, y_stride,
                                                              T(divisor));
        }
    });
    return launched("csr_spmv");
}

// ------------------------------------------------------------ cached pattern
//
// finish_cached_component (mac/cached_transfer_assembly.py:97-175) on the
// device.  A cached P1 transfer keeps, per component, the table slots of its
// CSR entries in key order, the transpose order, and the row pointers of B and
// B^T.  When new quadrature contributions miss the cached keys they are
// inserted into the table and only the new keys are sorted and merged into
// both orders: every old and new entry gets one merge position from a binary
// search in the other (disjoint, individually sorted) array, as the reference
// does with searchsorted, and the row pointers grow by the prefix counts of
// the new rows and columns alone.  The first build is the same merge with no
// old pattern and the table's occupied keys (with their slots) as the new keys.
//
// Two launches sequences with one host read between them (the reference
// reads the number of new keys too):
//   afsi_b200_cache_new_keys  sorted unique missing keys absent from the
//                             pattern (or, with no pattern, the occupied table
//                             keys with their slots) and their count;
//   afsi_b200_cache_merge     the merged slots, transpose order, CSR indices,
//                             values and transpose values.

namespace afsi {

__device__ __forceinline__ int64_t lower_bound(const int64_t* a, int64_t n, int64_t v) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__device__ __forceinline__ int64_t upper_bound(const int64_t* a, int64_t n, int64_t v) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] <= v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void cache_gather_keys_kernel(const int64_t* __restrict__ table, const int64_t* __restrict__ slots,
                                         int64_t n, int64_t* __restrict__ out) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        out[i] = table[slots[i]];
}

// flags[j] = sorted[j] is the first of its run and not an old key.
__global__ void cache_flag_new_kernel(const int64_t* __restrict__ sorted, int64_t m, const int64_t* __restrict__ old,
                                      int64_t nnz, uint8_t* __restrict__ flags) {
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < m; j += int64_t(gridDim.x) * blockDim.x) {
        const int64_t k = sorted[j];
        const bool first = j == 0 || sorted[j - 1] != k;
        const int64_t at = lower_bound(old, nnz, k);
        flags[j] = first && !(at < nnz && old[at] == k);
    }
}

// Occupied table keys (others become `sentinel`, which sorts after every
// key) with their slot indices; *count += occupied slots (one atomic per warp).
__global__ void cache_occupied_kernel(const int64_t* __restrict__ table, int64_t capacity, int64_t sentinel,
                                      int64_t* __restrict__ keys, int64_t* __restrict__ index,
                                      unsigned long long* count) {
    for (int64_t i0 = int64_t(blockIdx.x) * blockDim.x; i0 < capacity; i0 += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = i0 + threadIdx.x;
        const bool occupied = i < capacity && table[i] >= 0;
        if (i < capacity) {
            keys[i] = occupied ? table[i] : sentinel;
            index[i] = i;
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, occupied);
        if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(count, (unsigned long long)__popc(ballot));
    }
}

// Merge positions of the old and new keys; the merged keys and slots (new
// slots from `new_slots`, or found in the table by linear probing).
__global__ void cache_merge_keys_kernel(const int64_t* __restrict__ old_keys, const int64_t* __restrict__ old_slots,
                                        int64_t nnz, const int64_t* __restrict__ new_keys,
                                        const int64_t* __restrict__ new_slots, int64_t k,
                                        const int64_t* __restrict__ table, int64_t capacity,
                                        int64_t* __restrict__ keys_out, int64_t* __restrict__ slots_out,
                                        int64_t* __restrict__ old_pos, int64_t* __restrict__ new_pos,
                                        int32_t* status) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < nnz + k;
         t += int64_t(gridDim.x) * blockDim.x) {
        if (t < nnz) {
            const int64_t p = t + upper_bound(new_keys, k, old_keys[t]);
            keys_out[p] = old_keys[t];
            slots_out[p] = old_slots[t];
            old_pos[t] = p;
        } else {
            const int64_t j = t - nnz, key = new_keys[j];
            const int64_t p = j + lower_bound(old_keys, nnz, key);
            int64_t slot = -1;
            if (new_slots) {
                slot = new_slots[j];
            } else {
                uint64_t s = hash_bucket(key, capacity);
                for (int attempt = 0; attempt < 128; ++attempt) {  // the insertion probe bound
                    if (table[s] == key) {
                        slot = int64_t(s);
                        break;
                    }
                    s = (s + 1) & uint64_t(capacity - 1);
                }
                if (slot < 0) {
                    flag(status, AFSI_FLAG_OVERFLOW);
                    slot = 0;
                }
            }
            keys_out[p] = key;
            slots_out[p] = slot;
            new_pos[j] = p;
        }
    }
}

// counts[key / nf] += 1 (rows) and tcounts[key % nf] += 1 (columns).
__global__ void cache_count_kernel(const int64_t* __restrict__ keys, int64_t k, int64_t nf, int64_t rows,
                                   unsigned long long* __restrict__ counts, unsigned long long* __restrict__ tcounts,
                                   int32_t* status) {
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < k; j += int64_t(gridDim.x) * blockDim.x) {
        const int64_t key = keys[j];
        if (key < 0 || key >= nf * rows) {
            flag(status, AFSI_FLAG_INDEX);
            continue;
        }
        atomicAdd(counts + key / nf, 1ull);
        atomicAdd(tcounts + key % nf, 1ull);
    }
}

// out[r] = base[r] + add[r] (base may be null).
__global__ void cache_pointers_kernel(const int64_t* __restrict__ base, const int64_t* __restrict__ add, int64_t n,
                                      int64_t* __restrict__ out) {
    for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x)
        out[r] = (base ? base[r] : 0) + add[r];
}

// Reverse (column-major) keys col * rows + row: of the old entries in
// transpose order, and of the new keys with their index.
__global__ void cache_reverse_kernel(const int64_t* __restrict__ old_keys, const int64_t* __restrict__ old_order,
                                     int64_t nnz, const int64_t* __restrict__ new_keys, int64_t k, int64_t nf,
                                     int64_t rows, int64_t* __restrict__ old_rk, int64_t* __restrict__ new_rk,
                                     int64_t* __restrict__ new_index) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < nnz + k;
         t += int64_t(gridDim.x) * blockDim.x) {
        if (t < nnz) {
            const int64_t key = old_keys[old_order[t]];
            old_rk[t] = (key % nf) * rows + key / nf;
        } else {
            const int64_t j = t - nnz, key = new_keys[j];
            new_rk[j] = (key % nf) * rows + key / nf;
            new_index[j] = j;
        }
    }
}

__global__ void cache_merge_transpose_kernel(const int64_t* __restrict__ old_rk, const int64_t* __restrict__ old_order,
                                             const int64_t* __restrict__ old_pos, int64_t nnz,
                                             const int64_t* __restrict__ new_rk, const int64_t* __restrict__ new_order,
                                             const int64_t* __restrict__ new_pos, int64_t k,
                                             int64_t* __restrict__ order_out) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < nnz + k;
         t += int64_t(gridDim.x) * blockDim.x) {
        if (t < nnz) {
            order_out[t + upper_bound(new_rk, k, old_rk[t])] = old_pos[old_order[t]];
        } else {
            const int64_t q = t - nnz;
            order_out[q + lower_bound(old_rk, nnz, new_rk[q])] = new_pos[new_order[q]];
        }
    }
}

template <class T>
__global__ void cache_finish_kernel(const int64_t* __restrict__ keys, const int64_t* __restrict__ slots,
                                    const int64_t* __restrict__ order, int64_t n, int64_t nf, int64_t rows,
                                    const T* __restrict__ table_values, int64_t* __restrict__ columns,
                                    int64_t* __restrict__ tcolumns, T* __restrict__ values, T* __restrict__ reverse,
                                    int32_t* status) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t key = keys[i];
        if (key < 0 || key >= nf * rows) flag(status, AFSI_FLAG_INDEX);
        columns[i] = key % nf;
        const T v = table_values[slots[i]];
        if (!isfinite(v)) flag(status, AFSI_FLAG_SUPPORT);
        values[i] = v;
        const int64_t o = order[i];
        tcolumns[i] = keys[o] / nf;
        reverse[i] = table_values[slots[o]];
    }
}

}  // namespace afsi

namespace {

unsigned cache_grid(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return unsigned(b < 1 ? 1 : (b < 148 * 32 ? b : 148 * 32));
}

int key_bits(int64_t limit) {
    int bits = 1;
    while (bits < 63 && (int64_t(1) << bits) <= limit) ++bits;
    return bits;
}

struct Carve {
    unsigned char* base;
    size_t used = 0, size;
    template <class T>
    T* take(int64_t n) {
        used = (used + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base + used);
        used += size_t(n > 0 ? n : 1) * sizeof(T);
        return p;
    }
};

size_t cub_bytes(int64_t n_sort, int64_t n_scan) {
    size_t a = 0, b = 0, c = 0, d = 0;
    const int64_t ns = n_sort > 0 ? n_sort : 1, nc = n_scan > 0 ? n_scan : 1;
    cub::DeviceRadixSort::SortPairs(nullptr, a, static_cast<const int64_t*>(nullptr), static_cast<int64_t*>(nullptr),
                                    static_cast<const int64_t*>(nullptr), static_cast<int64_t*>(nullptr), ns);
    cub::DeviceSelect::Flagged(nullptr, b, static_cast<const int64_t*>(nullptr), static_cast<const uint8_t*>(nullptr),
                               static_cast<int64_t*>(nullptr), static_cast<int64_t*>(nullptr), ns);
    cub::DeviceScan::ExclusiveSum(nullptr, c, static_cast<const unsigned long long*>(nullptr),
                                  static_cast<unsigned long long*>(nullptr), nc);
    cub::DeviceRadixSort::SortKeys(nullptr, d, static_cast<const int64_t*>(nullptr), static_cast<int64_t*>(nullptr),
                                   ns);
    return std::max(std::max(a, b), std::max(c, d));
}

}  // namespace

extern "C" int64_t afsi_b200_cache_scratch_bytes(int64_t capacity, int64_t nnz_old, int64_t missing, int64_t rows,
                                                 int64_t nf) {
    if (capacity < 0 || nnz_old < 0 || missing < 0 || rows < 1 || nf < 1) return -1;
    const int64_t k = std::max(missing, capacity);  // new keys: missing keys, or every occupied slot
    const int64_t words = 2 * nnz_old + 8 * k + nnz_old + k + 2 * (rows + 1) + 2 * (nf + 1) + 2 * (nnz_old + k);
    return words * 8 + k + 16 * 256 + int64_t(cub_bytes(k + nnz_old, std::max(rows, nf) + 1));
}

extern "C" int32_t afsi_b200_cache_new_keys(const int64_t* table_keys, int64_t capacity, const int64_t* old_slots,
                                            int64_t nnz_old, const int64_t* missing_keys, int64_t missing,
                                            int64_t limit, int64_t* new_keys, int64_t* new_slots, int64_t* count,
                                            void* scratch, int64_t scratch_bytes, afsi_stream_t stream) {
    AFSI_REQUIRE(table_keys && capacity > 0 && (capacity & (capacity - 1)) == 0 && new_keys && count && scratch,
                 "invalid cached-pattern arguments");
    AFSI_REQUIRE(nnz_old >= 0 && missing >= 0 && limit > 0, "invalid cached-pattern sizes");
    Carve c{static_cast<unsigned char*>(scratch), 0, size_t(scratch_bytes)};
    const int bits = key_bits(limit);
    if (cudaMemsetAsync(count, 0, 8, stream) != cudaSuccess) return fail(AFSI_ERR_CUDA, "cached pattern: memset");
    if (!old_slots) {
        // first build: the occupied keys in key order with their slots; the
        // first *count entries of new_keys / new_slots (capacity long) are them
        AFSI_REQUIRE(new_slots, "a first build returns the slots of its keys");
        int64_t* keys = c.take<int64_t>(capacity);
        int64_t* index = c.take<int64_t>(capacity);
        size_t temp_bytes = cub_bytes(capacity, 1);
        void* temp = c.take<unsigned char>(int64_t(temp_bytes));
        AFSI_REQUIRE(c.used <= c.size, "cached-pattern scratch too small");
        cache_occupied_kernel<<<cache_grid(capacity), 256, 0, stream>>>(
            table_keys, capacity, limit, keys, index, reinterpret_cast<unsigned long long*>(count));
        int32_t rc = launched("cache occupied keys");
        if (rc) return rc;
        if (cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, new_keys, index, new_slots, capacity, 0, bits,
                                            stream) != cudaSuccess)
            return fail(AFSI_ERR_CUDA, "cached pattern: sort failed");
        return launched("cache sort occupied keys");
    }
    AFSI_REQUIRE(missing_keys || missing == 0, "null missing keys");
    if (missing == 0) return AFSI_OK;
    int64_t* old_keys = c.take<int64_t>(nnz_old);
    int64_t* sorted = c.take<int64_t>(missing);
    uint8_t* flags = c.take<uint8_t>(missing);
    size_t temp_bytes = cub_bytes(missing, 1);
    void* temp = c.take<unsigned char>(int64_t(temp_bytes));
    AFSI_REQUIRE(c.used <= c.size, "cached-pattern scratch too small");
    if (nnz_old) cache_gather_keys_kernel<<<cache_grid(nnz_old), 256, 0, stream>>>(table_keys, old_slots, nnz_old, old_keys);
    if (cub::DeviceRadixSort::SortKeys(temp, temp_bytes, missing_keys, sorted, missing, 0, bits, stream) !=
        cudaSuccess)
        return fail(AFSI_ERR_CUDA, "cached pattern: sort failed");
    cache_flag_new_kernel<<<cache_grid(missing), 256, 0, stream>>>(sorted, missing, old_keys, nnz_old, flags);
    if (cub::DeviceSelect::Flagged(temp, temp_bytes, sorted, flags, new_keys, count, missing, stream) != cudaSuccess)
        return fail(AFSI_ERR_CUDA, "cached pattern: select failed");
    return launched("cache new keys");
}

extern "C" int32_t afsi_b200_cache_merge(const int64_t* table_keys, const void* table_values, int64_t capacity,
                                         const int64_t* old_slots, const int64_t* old_order, const int64_t* old_crow,
                                         const int64_t* old_tcrow, int64_t nnz_old, const int64_t* new_keys,
                                         const int64_t* new_slots, int64_t k, int64_t rows, int64_t nf,
                                         int64_t* slots, int64_t* order, int64_t* crow, int64_t* columns,
                                         int64_t* tcrow, int64_t* tcolumns, void* values, void* reverse,
                                         int32_t* status, void* scratch, int64_t scratch_bytes, int32_t dtype,
                                         afsi_stream_t stream) {
    AFSI_REQUIRE(table_keys && table_values && capacity > 0 && (capacity & (capacity - 1)) == 0,
                 "invalid cached-pattern table");
    AFSI_REQUIRE(nnz_old >= 0 && k >= 0 && rows > 0 && nf > 0 && (nnz_old == 0 || (old_slots && old_order && old_crow &&
                                                                                       old_tcrow)),
                 "invalid cached pattern");
    AFSI_REQUIRE(slots && order && crow && columns && tcrow && tcolumns && values && reverse && scratch &&
                     (k == 0 || new_keys),
                 "null cached-pattern output");
    const int64_t n = nnz_old + k;
    Carve c{static_cast<unsigned char*>(scratch), 0, size_t(scratch_bytes)};
    int64_t* old_keys = c.take<int64_t>(nnz_old);
    int64_t* old_rk = c.take<int64_t>(nnz_old);
    int64_t* old_pos = c.take<int64_t>(nnz_old);
    int64_t* new_pos = c.take<int64_t>(k);
    int64_t* new_rk = c.take<int64_t>(k);
    int64_t* new_rk_sorted = c.take<int64_t>(k);
    int64_t* new_index = c.take<int64_t>(k);
    int64_t* new_order = c.take<int64_t>(k);
    int64_t* keys = c.take<int64_t>(n);
    unsigned long long* counts = c.take<unsigned long long>(rows + 1);
    unsigned long long* tcounts = c.take<unsigned long long>(nf + 1);
    unsigned long long* scan = c.take<unsigned long long>(rows + 1);
    unsigned long long* tscan = c.take<unsigned long long>(nf + 1);
    size_t temp_bytes = cub_bytes(k, std::max(rows, nf) + 1);
    void* temp = c.take<unsigned char>(int64_t(temp_bytes));
    AFSI_REQUIRE(c.used <= c.size, "cached-pattern scratch too small");
    const int bits = key_bits(nf * rows);
    if (nnz_old)
        cache_gather_keys_kernel<<<cache_grid(nnz_old), 256, 0, stream>>>(table_keys, old_slots, nnz_old, old_keys);
    cache_merge_keys_kernel<<<cache_grid(n), 256, 0, stream>>>(old_keys, old_slots, nnz_old, new_keys, new_slots, k,
                                                               table_keys, capacity, keys, slots, old_pos, new_pos,
                                                               status);
    // row pointers grow by the prefix counts of the new keys' rows / columns
    if (cudaMemsetAsync(counts, 0, size_t(rows + 1) * 8, stream) != cudaSuccess ||
        cudaMemsetAsync(tcounts, 0, size_t(nf + 1) * 8, stream) != cudaSuccess)
        return fail(AFSI_ERR_CUDA, "cached pattern: memset");
    cache_count_kernel<<<cache_grid(k), 256, 0, stream>>>(new_keys, k, nf, rows, counts, tcounts, status);
    if (cub::DeviceScan::ExclusiveSum(temp, temp_bytes, counts, scan, rows + 1, stream) != cudaSuccess ||
        cub::DeviceScan::ExclusiveSum(temp, temp_bytes, tcounts, tscan, nf + 1, stream) != cudaSuccess)
        return fail(AFSI_ERR_CUDA, "cached pattern: scan failed");
    cache_pointers_kernel<<<cache_grid(rows + 1), 256, 0, stream>>>(old_crow, reinterpret_cast<const int64_t*>(scan),
                                                                     rows + 1, crow);
    cache_pointers_kernel<<<cache_grid(nf + 1), 256, 0, stream>>>(old_tcrow, reinterpret_cast<const int64_t*>(tscan),
                                                                   nf + 1, tcrow);
    // transpose order: merge of the old reverse keys and the sorted new ones
    cache_reverse_kernel<<<cache_grid(n), 256, 0, stream>>>(old_keys, old_order, nnz_old, new_keys, k, nf, rows,
                                                            old_rk, new_rk, new_index);
    if (k && cub::DeviceRadixSort::SortPairs(temp, temp_bytes, new_rk, new_rk_sorted, new_index, new_order, k, 0,
                                             bits, stream) != cudaSuccess)
        return fail(AFSI_ERR_CUDA, "cached pattern: sort failed");
    cache_merge_transpose_kernel<<<cache_grid(n), 256, 0, stream>>>(old_rk, old_order, old_pos, nnz_old,
                                                                    new_rk_sorted, new_order, new_pos, k, order);
    AFSI_DISPATCH(dtype, {
        cache_finish_kernel<T><<<cache_grid(n), 256, 0, stream>>>(keys, slots, order, n, nf, rows,
                                                                  static_cast<const T*>(table_values), columns,
                                                                  tcolumns, static_cast<T*>(values),
                                                                  static_cast<T*>(reverse), status);
    });
    return launched("cache merge");
}

namespace afsi {

template <class T>
__global__ void cache_values_kernel(const T* __restrict__ table_values, const int64_t* __restrict__ slots,
                                    const int64_t* __restrict__ order, int64_t n, T* __restrict__ values,
                                    T* __restrict__ reverse, int32_t* status) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const T v = table_values[slots[i]];
        if (!isfinite(v)) flag(status, AFSI_FLAG_SUPPORT);
        values[i] = v;
        reverse[i] = table_values[slots[order[i]]];
    }
}

}  // namespace afsi

extern "C" int32_t afsi_b200_cache_values(const void* table_values, const int64_t* slots, const int64_t* order,
                                          int64_t n, void* values, void* reverse, int32_t* status, int32_t dtype,
                                          afsi_stream_t stream) {
    AFSI_REQUIRE(n >= 0, "negative entry count");
    if (n == 0) return AFSI_OK;
    AFSI_REQUIRE(table_values && slots && order && values && reverse, "null cached-pattern argument");
    AFSI_DISPATCH(dtype, {
        cache_values_kernel<T><<<cache_grid(n), 256, 0, stream>>>(static_cast<const T*>(table_values), slots, order,
                                                                  n, static_cast<T*>(values),
                                                                  static_cast<T*>(reverse), status);
    });
    return launched("cache values");
}
