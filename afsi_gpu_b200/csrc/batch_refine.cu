// Batched FP64 iterative refinement around batched FP32 V-cycles: the
// batching form at the FP64 solve tolerance.
//
// No reference counterpart: the reference solves each 2D channel instance on
// its own in FP64 (ChannelMultigrid.solve, mac2d/multigrid.py:85-111).  Here
// every instance keeps an FP64 iterate p and right-hand side b; one
// refinement is
//     e = (FP32 V-cycles from zero on r32)      afsi_b200_mg_batch_vcycles
//     p = p + double(e)                          batch_refine_correct_kernel
//     r = b - A p  (FP64, the reference operator, mac2d/grid.py:61-71)
//     r32 = float(r), ||r|| per instance         batch_refine_residual_kernel
// for all instances at once, repeated until every instance meets its own
// tolerance max(atol, rtol ||b||) (the FP64 solver's, mac2d/multigrid.py:
// 94-99) or a refinement cap is reached.  The loop runs on the device: a
// CUDA graph holds the start (p = 0, r32 = float(b), the tolerances) and a
// WHILE conditional node whose body is one refinement.  Termination does not
// depend on any reduction finishing: the correction kernel of every body
// clears the loop condition, and only the residual kernel's last block sets
// it again, while the refinement count stays below the cap.
//
// Layout.  Instances are cut into 32 x 32 cell tiles (y fastest, 256
// threads, four cells per thread), listed instance by instance in a block
// map (entry << 21 | tile), so an instance's blocks are one contiguous range.
// Each block writes one partial sum of r^2; the last block to finish sums
// every instance's range in a fixed order (one warp per instance), so the
// norms do not depend on block scheduling.
#include <vector>
#include <cstring>
#include "mg_ops.cuh"

namespace afsi {
namespace {

constexpr int kRTileY = 32, kRTileX = 32;
constexpr int kRRowStep = kThreads / kRTileY;  // 8 rows apart
constexpr int kRRows = kRTileX / kRRowStep;    // 4 cells per thread
constexpr int kREntryBits = 11;
constexpr int kRLocalBits = 32 - kREntryBits;
constexpr int kRMaxInstances = 1 << kREntryBits;
constexpr int kRMaxRefinements = 64;

// State words (doubles) after the per-instance arrays.
enum { kLoopRefinements = 0, kLoopUnconverged = 1, kLoopNonfinite = 2, kLoopWorstRatio = 3, kLoopWords = 8 };

struct RefineEntry {
    Lv<double> L;
    double* p;
    const double* b;
    float* r32;
    const float* e32;
    int64_t first_block, blocks;
};

struct RefineLayout {
    int64_t blocks = 0;
    int64_t entries_off = 0, map_off = 0, partial_off = 0, state_off = 0, counter_off = 0, bytes = 0;
};

int64_t align16(int64_t v) { return (v + 15) & ~int64_t(15); }

int64_t tiles(int64_t nx, int64_t ny) { return ((ny + kRTileY - 1) / kRTileY) * ((nx + kRTileX - 1) / kRTileX); }

// Device views of the buffer.  State: norm[count], tol[count], rhs_norm[count],
// done_at[count] (refinements after which the instance first met its
// tolerance, -1 before), then kLoopWords loop words.
struct RefineView {
    const RefineEntry* entries;
    const uint32_t* map;
    double* partial;
    double* state;
    unsigned int* counter;
    int count;
};

int32_t layout_of(const afsi_refine_instance* inst, int32_t count, RefineLayout& lay) {
    AFSI_REQUIRE(inst && count >= 1 && count <= kRMaxInstances, "batched refinement needs 1..%d instances",
                 kRMaxInstances);
    lay = RefineLayout();
    for (int i = 0; i < count; ++i) {
        const afsi_refine_instance& a = inst[i];
        AFSI_REQUIRE(a.nx >= 4 && a.ny >= 4 && a.nx <= (1 << 20) && a.ny <= (1 << 20),
                     "instance %d: grid %lld x %lld out of range", i, (long long)a.nx, (long long)a.ny);
        AFSI_REQUIRE(a.p && a.b && a.r32 && a.e32, "instance %d: null buffer", i);
        AFSI_REQUIRE(a.h2[0] > 0 && a.h2[1] > 0, "instance %d: spacing must be positive", i);
        const int64_t t = tiles(a.nx, a.ny);
        AFSI_REQUIRE(t < (int64_t(1) << kRLocalBits), "instance %d: grid too large", i);
        lay.blocks += t;
    }
    AFSI_REQUIRE(lay.blocks < (int64_t(1) << 31), "batch too large for one launch");
    int64_t off = 0;
    lay.entries_off = off;
    off = align16(off + int64_t(count) * int64_t(sizeof(RefineEntry)));
    lay.map_off = off;
    off = align16(off + lay.blocks * 4);
    lay.partial_off = off;
    off = align16(off + lay.blocks * 8);
    lay.state_off = off;
    off = align16(off + (int64_t(count) * 4 + kLoopWords) * 8);
    lay.counter_off = off;
    off = align16(off + 16);
    lay.bytes = off;
    return AFSI_OK;
}

RefineView view_of(const RefineLayout& lay, void* buffer, int count) {
    unsigned char* b = static_cast<unsigned char*>(buffer);
    RefineView v;
    v.entries = reinterpret_cast<const RefineEntry*>(b + lay.entries_off);
    v.map = reinterpret_cast<const uint32_t*>(b + lay.map_off);
    v.partial = reinterpret_cast<double*>(b + lay.partial_off);
    v.state = reinterpret_cast<double*>(b + lay.state_off);
    v.counter = reinterpret_cast<unsigned int*>(b + lay.counter_off);
    v.count = count;
    return v;
}

__device__ __forceinline__ const RefineEntry& entry_of(const RefineView& v, int& x0, int& y) {
    const uint32_t w = v.map[blockIdx.x];
    const int ent = int(w >> kRLocalBits);
    const int tile = int(w & ((1u << kRLocalBits) - 1));
    const RefineEntry& e = v.entries[ent];
    const int gy = (e.L.ny + kRTileY - 1) / kRTileY;
    y = (tile % gy) * kRTileY + int(threadIdx.x) % kRTileY;
    x0 = (tile / gy) * kRTileX + int(threadIdx.x) / kRTileY;
    return e;
}

// p += double(e32) over the instance's cells; block 0 clears the loop
// condition first, so a body whose residual kernel does not set it ends the loop.
__global__ void __launch_bounds__(kThreads) batch_refine_correct_kernel(RefineView v,
                                                                        cudaGraphConditionalHandle handle,
                                                                        int has_handle) {
    pdl_enter();
    if (has_handle && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(handle, 0u);
    int x0, y;
    const RefineEntry& e = entry_of(v, x0, y);
    if (y >= e.L.ny) return;
#pragma unroll
    for (int m = 0; m < kRRows; ++m) {
        const int x = x0 + m * kRRowStep;
        if (x >= e.L.nx) break;
        const int64_t i = int64_t(x) * e.L.ny + y;
        e.p[i] = e.p[i] + double(e.e32[i]);
    }
}

// Start (start != 0): p = 0 and r = b.  Step: r = b - A p.  Both write
// r32 = float(r) and reduce ||r|| per instance; the last block updates the
// state and decides whether another refinement runs.
__global__ void __launch_bounds__(kThreads) batch_refine_residual_kernel(RefineView v, int start, double rtol,
                                                                         double atol, int max_refinements,
                                                                         cudaGraphConditionalHandle handle,
                                                                         int has_handle) {
    pdl_enter();
    int x0, y;
    const RefineEntry& e = entry_of(v, x0, y);
    double local = 0.0;
    if (y < e.L.ny) {
        double r[kRRows];
#pragma unroll
        for (int m = 0; m < kRRows; ++m) {
            const int x = x0 + m * kRRowStep;
            r[m] = 0.0;
            if (x >= e.L.nx) continue;
            const int64_t i = int64_t(x) * e.L.ny + y;
            if (start) {
                r[m] = e.b[i];
            } else {
                const double pc = e.p[i];
                r[m] = e.b[i] - neg_lap<AFSI_BC_CHANNEL, true>(e.p, i, x, y, 0, e.L, 0.0, pc);
            }
        }
#pragma unroll
        for (int m = 0; m < kRRows; ++m) {
            const int x = x0 + m * kRRowStep;
            if (x >= e.L.nx) break;
            const int64_t i = int64_t(x) * e.L.ny + y;
            if (start) e.p[i] = 0.0;
            e.r32[i] = float(r[m]);
            local += r[m] * r[m];
        }
    }
    __shared__ double sums[kThreads / 32];
    __shared__ bool last;
    local = block_sum(local, sums);
    if (threadIdx.x == 0) v.partial[blockIdx.x] = local;
    if (!grid_reduce_arrive(v.counter, &last)) return;
    // last block: per-instance norms in a fixed order, one warp per instance
    __shared__ int unconverged, nonfinite;
    __shared__ double worst;
    if (threadIdx.x == 0) {
        unconverged = 0;
        nonfinite = 0;
        worst = 0.0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* norm = v.state;
    double* tol = v.state + v.count;
    double* rhs_norm = v.state + 2 * v.count;
    double* done_at = v.state + 3 * v.count;
    double* loop = v.state + 4 * v.count;
    const double refinements = start ? 0.0 : loop[kLoopRefinements] + 1.0;
    for (int k = warp; k < v.count; k += kThreads / 32) {
        const RefineEntry& f = v.entries[k];
        double s = 0.0;
        for (int64_t j = lane; j < f.blocks; j += 32) s += __ldcg(v.partial + f.first_block + j);
        s = warp_sum(s);
        if (lane == 0) {
            const double n = sqrt(s);
            norm[k] = n;
            if (start) {
                rhs_norm[k] = n;
                tol[k] = fmax(atol, rtol * n);
                done_at[k] = -1.0;
            }
            const bool ok = isfinite(n);
            if (!ok) atomicOr(&nonfinite, 1);
            if (ok && n <= tol[k]) {
                if (done_at[k] < 0) done_at[k] = refinements;
            } else {
                atomicAdd(&unconverged, 1);
            }
            const double ratio = rhs_norm[k] > 0 ? n / rhs_norm[k] : 0.0;
            // max of non-negative doubles through their bit patterns
            atomicMax(reinterpret_cast<unsigned long long*>(&worst),
                      static_cast<unsigned long long>(__double_as_longlong(ok ? ratio : INFINITY)));
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        loop[kLoopRefinements] = refinements;
        loop[kLoopUnconverged] = double(unconverged);
        loop[kLoopNonfinite] = double(nonfinite);
        loop[kLoopWorstRatio] = worst;
        *v.counter = 0u;
        const bool again = unconverged > 0 && !nonfinite && refinements < double(max_refinements);
        if (has_handle) cudaGraphSetConditional(handle, again ? 1u : 0u);
    }
}

struct RefineGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t capture = nullptr;
};

void release(RefineGraph* g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->capture) cudaStreamDestroy(g->capture);
    delete g;
}

int32_t check_parameters(double rtol, double atol, int32_t max_refinements) {
    AFSI_REQUIRE(isfinite(rtol) && isfinite(atol) && rtol >= 0 && atol >= 0 && rtol + atol > 0,
                 "invalid refinement tolerances");
    AFSI_REQUIRE(max_refinements >= 1 && max_refinements <= kRMaxRefinements, "max_refinements must be 1..%d",
                 kRMaxRefinements);
    return AFSI_OK;
}

int32_t launch_residual(const RefineLayout& lay, const RefineView& v, int start, double rtol, double atol,
                        int max_refinements, cudaGraphConditionalHandle handle, int has_handle,
                        cudaStream_t stream) {
    return launch_pdl(start ? "batch refine start" : "batch refine residual", batch_refine_residual_kernel,
                      dim3(unsigned(lay.blocks)), dim3(kThreads), 0, stream, v, start, rtol, atol, max_refinements,
                      handle, has_handle);
}

int32_t launch_correct(const RefineLayout& lay, const RefineView& v, cudaGraphConditionalHandle handle,
                       int has_handle, cudaStream_t stream) {
    return launch_pdl("batch refine correct", batch_refine_correct_kernel, dim3(unsigned(lay.blocks)),
                      dim3(kThreads), 0, stream, v, handle, has_handle);
}

}  // namespace
}  // namespace afsi

using namespace afsi;

extern "C" int64_t afsi_b200_batch_refine_bytes(const afsi_refine_instance* instances, int32_t count) {
    RefineLayout lay;
    if (layout_of(instances, count, lay)) return -1;
    return lay.bytes;
}

extern "C" int64_t afsi_b200_batch_refine_state_offset(const afsi_refine_instance* instances, int32_t count) {
    RefineLayout lay;
    if (layout_of(instances, count, lay)) return -1;
    return lay.state_off;
}

extern "C" int32_t afsi_b200_batch_refine_setup(const afsi_refine_instance* instances, int32_t count,
                                                void* host_buffer, int64_t bytes) {
    RefineLayout lay;
    int32_t rc = layout_of(instances, count, lay);
    if (rc) return rc;
    AFSI_REQUIRE(host_buffer && bytes >= lay.bytes, "refinement buffer needs %lld bytes", (long long)lay.bytes);
    unsigned char* h = static_cast<unsigned char*>(host_buffer);
    std::memset(h, 0, size_t(lay.bytes));
    int64_t block = 0;
    uint32_t* map = reinterpret_cast<uint32_t*>(h + lay.map_off);
    for (int i = 0; i < count; ++i) {
        const afsi_refine_instance& a = instances[i];
        RefineEntry e;
        std::memset(&e, 0, sizeof(e));
        e.L.nx = int(a.nx);
        e.L.ny = int(a.ny);
        e.L.nz = 1;
        e.L.n = a.nx * a.ny;
        e.L.h2[0] = a.h2[0];
        e.L.h2[1] = a.h2[1];
        e.L.h2[2] = 1.0;
        e.L.ih2[0] = 1.0 / a.h2[0];
        e.L.ih2[1] = 1.0 / a.h2[1];
        e.L.ih2[2] = 1.0;
        e.p = a.p;
        e.b = a.b;
        e.r32 = a.r32;
        e.e32 = a.e32;
        e.first_block = block;
        e.blocks = tiles(a.nx, a.ny);
        std::memcpy(h + lay.entries_off + int64_t(i) * int64_t(sizeof(e)), &e, sizeof(e));
        for (int64_t t = 0; t < e.blocks; ++t) map[block++] = (uint32_t(i) << kRLocalBits) | uint32_t(t);
    }
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_batch_refine_start(const afsi_refine_instance* instances, int32_t count, void* buffer,
                                                double rtol, double atol, int32_t max_refinements,
                                                afsi_stream_t stream) {
    RefineLayout lay;
    int32_t rc = layout_of(instances, count, lay);
    if (rc || (rc = check_parameters(rtol, atol, max_refinements))) return rc;
    AFSI_REQUIRE(buffer && reinterpret_cast<uintptr_t>(buffer) % 16 == 0, "device buffer must be 16-byte aligned");
    return launch_residual(lay, view_of(lay, buffer, count), 1, rtol, atol, max_refinements, 0, 0,
                           static_cast<cudaStream_t>(stream));
}

extern "C" int32_t afsi_b200_batch_refine_step(const afsi_refine_instance* instances, int32_t count, void* buffer,
                                               double rtol, double atol, int32_t max_refinements,
                                               afsi_stream_t stream) {
    RefineLayout lay;
    int32_t rc = layout_of(instances, count, lay);
    if (rc || (rc = check_parameters(rtol, atol, max_refinements))) return rc;
    AFSI_REQUIRE(buffer && reinterpret_cast<uintptr_t>(buffer) % 16 == 0, "device buffer must be 16-byte aligned");
    const RefineView v = view_of(lay, buffer, count);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if ((rc = launch_correct(lay, v, 0, 0, s))) return rc;
    return launch_residual(lay, v, 0, rtol, atol, max_refinements, 0, 0, s);
}

extern "C" int32_t afsi_b200_batch_refine_graph_create(const afsi_refine_instance* instances, int32_t count,
                                                       void* buffer, const afsi_mg_plan* const* plans,
                                                       const void* vcycle_table, int32_t cycles, double rtol,
                                                       double atol, int32_t max_refinements, void** graph_out) {
    RefineLayout lay;
    int32_t rc = layout_of(instances, count, lay);
    if (rc || (rc = check_parameters(rtol, atol, max_refinements))) return rc;
    AFSI_REQUIRE(graph_out && plans && vcycle_table, "null refinement-graph argument");
    AFSI_REQUIRE(buffer && reinterpret_cast<uintptr_t>(buffer) % 16 == 0, "device buffer must be 16-byte aligned");
    AFSI_REQUIRE(cycles >= 1 && cycles <= 64, "1..64 V-cycles per refinement");
    for (int i = 0; i < count; ++i) {
        AFSI_REQUIRE(plans[i] && plans[i]->dtype == AFSI_F32 && plans[i]->bc == AFSI_BC_CHANNEL &&
                         plans[i]->level[0].shape[0] == instances[i].nx &&
                         plans[i]->level[0].shape[1] == instances[i].ny &&
                         plans[i]->level[0].rhs == instances[i].r32 && plans[i]->level[0].p == instances[i].e32,
                     "plan %d is not the FP32 channel plan of instance %d", i, i);
    }
    *graph_out = nullptr;
    const RefineView v = view_of(lay, buffer, count);
    RefineGraph* g = new RefineGraph;
    cudaGraphConditionalHandle handle;
    if (cudaStreamCreateWithFlags(&g->capture, cudaStreamNonBlocking) != cudaSuccess ||
        cudaGraphCreate(&g->graph, 0) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&handle, g->graph, 0, cudaGraphCondAssignDefault) != cudaSuccess) {
        release(g);
        return fail(AFSI_ERR_CUDA, "refinement graph setup failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    // the start kernel, captured into the top-level graph; it sets the condition
    if (cudaStreamBeginCaptureToGraph(g->capture, g->graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) !=
        cudaSuccess) {
        release(g);
        return fail(AFSI_ERR_CUDA, "refinement graph capture failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    rc = launch_residual(lay, v, 1, rtol, atol, max_refinements, handle, 1, g->capture);
    cudaGraph_t captured = nullptr;
    cudaError_t end = cudaStreamEndCapture(g->capture, &captured);
    if (rc || end != cudaSuccess) {
        release(g);
        return rc ? rc : fail(AFSI_ERR_CUDA, "refinement start capture: %s", cudaGetErrorString(end));
    }
    size_t nodes = 0;
    cudaGraphNode_t start_node = nullptr;
    if (cudaGraphGetNodes(g->graph, nullptr, &nodes) != cudaSuccess || nodes != 1 ||
        cudaGraphGetNodes(g->graph, &start_node, &nodes) != cudaSuccess) {
        release(g);
        return fail(AFSI_ERR_CUDA, "refinement graph: expected one start node");
    }
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t loop;
    if (cudaGraphAddNode(&loop, g->graph, &start_node, 1, &np) != cudaSuccess) {
        release(g);
        return fail(AFSI_ERR_CUDA, "refinement conditional node: %s", cudaGetErrorString(cudaGetLastError()));
    }
    cudaGraph_t body = np.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(g->capture, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) !=
        cudaSuccess) {
        release(g);
        return fail(AFSI_ERR_CUDA, "refinement body capture failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    rc = afsi_b200_mg_batch_vcycles(plans, count, vcycle_table, cycles, 1, g->capture);
    if (!rc) rc = launch_correct(lay, v, handle, 1, g->capture);
    if (!rc) rc = launch_residual(lay, v, 0, rtol, atol, max_refinements, handle, 1, g->capture);
    end = cudaStreamEndCapture(g->capture, &captured);
    if (rc) {
        release(g);
        return rc;
    }
    if (end != cudaSuccess || cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess) {
        release(g);
        return fail(AFSI_ERR_CUDA, "refinement graph instantiation failed: %s",
                    cudaGetErrorString(cudaGetLastError()));
    }
    *graph_out = g;
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_batch_refine_graph_launch(void* graph, afsi_stream_t stream) {
    AFSI_REQUIRE(graph, "null refinement graph");
    if (cudaGraphLaunch(static_cast<RefineGraph*>(graph)->exec, static_cast<cudaStream_t>(stream)) != cudaSuccess)
        return fail(AFSI_ERR_CUDA, "refinement graph launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    return AFSI_OK;
}

extern "C" int32_t afsi_b200_batch_refine_graph_destroy(void* graph) {
    release(static_cast<RefineGraph*>(graph));
    return AFSI_OK;
}
