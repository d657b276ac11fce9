// Crank-Nicolson Helmholtz Jacobi sweeps and blocked Stokes residual
// reductions on the 3D MAC grid (the kernels inside the Stokes FGMRES
// preconditioner and its convergence checks).
//
// Helmholtz (mac/_triton_helmholtz.py:6-77, CPU form mac/helmholtz.py:14-28):
//   initialize  rhs_c = b_c - s (p[i] - p[i-1])/h_c on interior component-
//               normal faces, 0 on the two walls; u_c = rhs_c / diag_c;
//   sweep       out_c = u + (r - u + alpha L_c u)/diag_c, 0 on the walls, with
//               L_c the face Laplacian whose missing neighbours are odd ghosts
//               (-u), summed x, y, z (mac/grid.py:96-105).
// All three face lattices in one launch (a flat index over the three arrays).
//
// Stokes reductions (mac/_triton_stokes.py:8-145): one partial per 256 cells,
// in the layouts the reference's reductions consume (mac/stokes_workspace.py):
//   start           [sum of u^2+v^2+w^2 over each cell's low faces, sum p, all p finite]
//   residual        momentum residual of the three low faces of each cell
//                   (u - alpha L u + scale G p - b, wall faces without L and G),
//                   divergence D u, residual = -inverse_scale D u, partials
//                   [sum m^2, sum div^2];
//   pressure input  [sum rhs, sum |rhs|, sum p, all rhs finite, all p finite];
//   pressure norm   [sum rhs^2, sum (rhs - A p)^2] with the Neumann operator.
// The library is built with --fmad=false, so every expression rounds as the
// reference's fusion-free kernels do; block sums are a fixed tree.
#include "common.cuh"

namespace afsi {

constexpr int kCells = 256;  // cells (threads) per block, one partial per block

struct Cells {
    int64_t nx, ny, nz;  // pressure cells
};

// Face array of component c: (nx+1, ny, nz), (nx, ny+1, nz), (nx, ny, nz+1).
__device__ __forceinline__ void face_dims(const Cells& g, int c, int64_t* n) {
    n[0] = g.nx + (c == 0);
    n[1] = g.ny + (c == 1);
    n[2] = g.nz + (c == 2);
}

template <class T>
struct Faces {
    T* f[3];
    // component pointer without dynamic indexing of the parameter array
    __device__ __forceinline__ T* at(int c) const { return c == 0 ? f[0] : (c == 1 ? f[1] : f[2]); }
};
template <class T>
struct ConstFaces {
    const T* f[3];
    __device__ __forceinline__ const T* at(int c) const { return c == 0 ? f[0] : (c == 1 ? f[1] : f[2]); }
};

// Flat index over the three face arrays back to back -> (component, local index).
__device__ __forceinline__ int split_faces(const Cells& g, int64_t t, int64_t* local) {
    const int64_t n0 = (g.nx + 1) * g.ny * g.nz, n1 = g.nx * (g.ny + 1) * g.nz;
    if (t < n0) {
        *local = t;
        return 0;
    }
    if (t < n0 + n1) {
        *local = t - n0;
        return 1;
    }
    *local = t - n0 - n1;
    return 2;
}

template <class T>
__global__ void __launch_bounds__(256) helmholtz_initialize_kernel(ConstFaces<T> b, const T* __restrict__ p,
                                                                   ConstFaces<T> diag, Faces<T> rhs, Faces<T> u,
                                                                   const T* __restrict__ param, Cells g,
                                                                   double hx, double hy, double hz, int64_t total) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= total) return;
    int64_t i;
    const int c = split_faces(g, t, &i);
    int64_t n[3];
    face_dims(g, c, n);
    const int64_t x = i / (n[1] * n[2]), y = (i / n[2]) % n[1], z = i % n[2];
    const int64_t coord = c == 0 ? x : (c == 1 ? y : z);
    const bool interior = coord > 0 && coord < n[c] - 1;
    T r = b.at(c)[i];
    if (p && interior) {
        // pressure cells on either side of the face
        const int64_t right = (x * g.ny + y) * g.nz + z;
        const int64_t stride = c == 0 ? g.ny * g.nz : (c == 1 ? g.nz : 1);
        const T h = T(c == 0 ? hx : (c == 1 ? hy : hz));
        r = r - param[1] * ((p[right] - p[right - stride]) / h);
    }
    if (!interior) r = T(0);
    rhs.at(c)[i] = r;
    u.at(c)[i] = r / diag.at(c)[i];
}

template <class T>
__global__ void __launch_bounds__(256) helmholtz_sweep_kernel(ConstFaces<T> u, ConstFaces<T> rhs, ConstFaces<T> diag,
                                                              Faces<T> out, const T* __restrict__ param, Cells g,
                                                              double hx2, double hy2, double hz2, int64_t total) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= total) return;
    int64_t i;
    const int c = split_faces(g, t, &i);
    int64_t n[3];
    face_dims(g, c, n);
    const int64_t x = i / (n[1] * n[2]), y = (i / n[2]) % n[1], z = i % n[2];
    const T* U = u.at(c);
    const T v = U[i];
    const int64_t sx = n[1] * n[2], sy = n[2];
    const T xm = x > 0 ? U[i - sx] : -v, xp = x + 1 < n[0] ? U[i + sx] : -v;
    const T ym = y > 0 ? U[i - sy] : -v, yp = y + 1 < n[1] ? U[i + sy] : -v;
    const T zm = z > 0 ? U[i - 1] : -v, zp = z + 1 < n[2] ? U[i + 1] : -v;
    T lap = (xm - T(2) * v + xp) / T(hx2);
    lap = lap + (ym - T(2) * v + yp) / T(hy2);
    lap = lap + (zm - T(2) * v + zp) / T(hz2);
    T value = v + (rhs.at(c)[i] - v + param[0] * lap) / diag.at(c)[i];
    const int64_t coord = c == 0 ? x : (c == 1 ? y : z);
    if (!(coord > 0 && coord < n[c] - 1)) value = T(0);
    out.at(c)[i] = value;
}

// Fixed-order block sums of K values per thread; thread 0 writes them.
template <int K>
__device__ __forceinline__ void block_partials(double (&v)[K], double* out) {
    __shared__ double sh[K][kCells / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) sh[k][warp] = v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = 0.0;
            for (int w = 0; w < kCells / 32; ++w) s += sh[k][w];
            out[k] = s;
        }
    }
}

// Minimum of a 0/1 flag over the block (1 only if every thread has 1).
__device__ __forceinline__ int block_all(int ok) { return __syncthreads_and(ok); }

template <class T>
__global__ void __launch_bounds__(kCells) stokes_start_kernel(ConstFaces<T> b, const T* __restrict__ p, Cells g,
                                                              T* __restrict__ out) {
    const int64_t n = g.nx * g.ny * g.nz;
    const int64_t cell = int64_t(blockIdx.x) * kCells + threadIdx.x;
    const bool active = cell < n;
    double v[2] = {0.0, 0.0};
    int finite = 1;
    if (active) {
        const int64_t i = cell / (g.ny * g.nz), j = (cell / g.nz) % g.ny, k = cell % g.nz;
        const T u = b.f[0][(i * g.ny + j) * g.nz + k];
        const T vv = b.f[1][(i * (g.ny + 1) + j) * g.nz + k];
        const T w = b.f[2][(i * g.ny + j) * (g.nz + 1) + k];
        const T pc = p[cell];
        v[0] = double(u * u + vv * vv + w * w);
        v[1] = double(pc);
        finite = isfinite(pc);
    }
    const int all = block_all(finite);
    double sums[2] = {v[0], v[1]};
    __shared__ double res[2];
    block_partials<2>(sums, res);
    if (threadIdx.x == 0) {
        out[blockIdx.x * 3] = T(res[0]);
        out[blockIdx.x * 3 + 1] = T(res[1]);
        out[blockIdx.x * 3 + 2] = T(all);
    }
}

// Momentum residual of component C's face with the cell's low index (i,j,k):
// center - alpha L center + scale G p - rhs; the wall face (coordinate 0) has
// no L and no G (mac/_triton_stokes.py:31-55).
template <class T, int C>
__device__ __forceinline__ T momentum(const T* __restrict__ U, const T* __restrict__ R, const T* __restrict__ P, T pc,
                                      T center, int64_t i, int64_t j, int64_t k, const Cells& g, const T* coef) {
    const int64_t n0 = g.nx + (C == 0), n1 = g.ny + (C == 1), n2 = g.nz + (C == 2);
    const int64_t coordinate = C == 0 ? i : (C == 1 ? j : k);
    const int64_t previous = C == 0 ? ((i - 1) * g.ny + j) * g.nz + k
                                    : (C == 1 ? (i * g.ny + j - 1) * g.nz + k : (i * g.ny + j) * g.nz + k - 1);
    const T inv_h = coef[3 + C];
    const int64_t index = (i * n1 + j) * n2 + k;
    T lap = T(0);
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const int64_t q = axis == 0 ? i : (axis == 1 ? j : k);
        const int64_t n = axis == 0 ? n0 : (axis == 1 ? n1 : n2);
        const int64_t stride = axis == 0 ? n1 * n2 : (axis == 1 ? n2 : 1);
        const T left = q > 0 ? U[index - stride] : -center;
        const T right = q + 1 < n ? U[index + stride] : -center;
        lap = lap + (left - T(2) * center + right) * coef[6 + axis];
    }
    if (coordinate == 0) lap = T(0);
    const T gp = coordinate > 0 ? (pc - P[previous]) * inv_h : T(0);
    return center - coef[0] * lap + coef[1] * gp - R[index];
}

template <class T>
__global__ void __launch_bounds__(kCells) stokes_residual_kernel(ConstFaces<T> u, const T* __restrict__ p,
                                                                 ConstFaces<T> b, T* __restrict__ residual,
                                                                 T* __restrict__ out, const T* __restrict__ coef,
                                                                 Cells g) {
    const int64_t n = g.nx * g.ny * g.nz;
    const int64_t cell = int64_t(blockIdx.x) * kCells + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (cell < n) {
        const int64_t i = cell / (g.ny * g.nz), j = (cell / g.nz) % g.ny, k = cell % g.nz;
        const int64_t iu = (i * g.ny + j) * g.nz + k;
        const int64_t iv = (i * (g.ny + 1) + j) * g.nz + k;
        const int64_t iw = (i * g.ny + j) * (g.nz + 1) + k;
        const T cu = u.f[0][iu], cv = u.f[1][iv], cw = u.f[2][iw];
        const T pc = p[cell];
        const T m0 = momentum<T, 0>(u.f[0], b.f[0], p, pc, cu, i, j, k, g, coef);
        const T m1 = momentum<T, 1>(u.f[1], b.f[1], p, pc, cv, i, j, k, g, coef);
        const T m2 = momentum<T, 2>(u.f[2], b.f[2], p, pc, cw, i, j, k, g, coef);
        const T r0 = u.f[0][iu + g.ny * g.nz], r1 = u.f[1][iv + g.nz], r2 = u.f[2][iw + 1];
        // directional sum order of the reference, no contraction
        const T div = ((r0 - cu) * coef[3] + (r1 - cv) * coef[4]) + (r2 - cw) * coef[5];
        residual[cell] = -coef[2] * div;
        v[0] = double((m0 * m0 + m1 * m1) + m2 * m2);
        v[1] = double(div * div);
    }
    __shared__ double res[2];
    block_partials<2>(v, res);
    if (threadIdx.x == 0) {
        out[blockIdx.x * 2] = T(res[0]);
        out[blockIdx.x * 2 + 1] = T(res[1]);
    }
}

template <class T>
__global__ void __launch_bounds__(kCells) pressure_input_kernel(const T* __restrict__ rhs, const T* __restrict__ p,
                                                                int64_t n, T* __restrict__ out) {
    const int64_t cell = int64_t(blockIdx.x) * kCells + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    int fr = 1, fp = 1;
    if (cell < n) {
        const T r = rhs[cell], pc = p[cell];
        v[0] = double(r);
        v[1] = double(fabs(r));
        v[2] = double(pc);
        fr = isfinite(r);
        fp = isfinite(pc);
    }
    const int all_r = block_all(fr);
    const int all_p = block_all(fp);
    __shared__ double res[3];
    block_partials<3>(v, res);
    if (threadIdx.x == 0) {
        T* o = out + blockIdx.x * 5;
        o[0] = T(res[0]);
        o[1] = T(res[1]);
        o[2] = T(res[2]);
        o[3] = T(all_r);
        o[4] = T(all_p);
    }
}

template <class T>
__global__ void __launch_bounds__(kCells) pressure_norm_kernel(const T* __restrict__ rhs, const T* __restrict__ p,
                                                               const T* __restrict__ h2, Cells g,
                                                               T* __restrict__ out) {
    const int64_t n = g.nx * g.ny * g.nz;
    const int64_t cell = int64_t(blockIdx.x) * kCells + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (cell < n) {
        const int64_t i = cell / (g.ny * g.nz), j = (cell / g.nz) % g.ny, k = cell % g.nz;
        const T pc = p[cell], r = rhs[cell];
        T lap = T(0);
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const int64_t q = axis == 0 ? i : (axis == 1 ? j : k);
            const int64_t nn = axis == 0 ? g.nx : (axis == 1 ? g.ny : g.nz);
            const int64_t stride = axis == 0 ? g.ny * g.nz : (axis == 1 ? g.nz : 1);
            const T hh = h2[axis];
            lap = lap - (q + 1 < nn ? (p[cell + stride] - pc) / hh : T(0));
            lap = lap + (q > 0 ? (pc - p[cell - stride]) / hh : T(0));
        }
        const T res = r - lap;
        v[0] = double(r * r);
        v[1] = double(res * res);
    }
    __shared__ double res[2];
    block_partials<2>(v, res);
    if (threadIdx.x == 0) {
        out[blockIdx.x * 2] = T(res[0]);
        out[blockIdx.x * 2 + 1] = T(res[1]);
    }
}

}  // namespace afsi

using namespace afsi;

namespace {

int32_t check_cells(const int64_t* shape, Cells* g) {
    AFSI_REQUIRE(shape && shape[0] > 0 && shape[1] > 0 && shape[2] > 0, "invalid MAC grid shape");
    AFSI_REQUIRE(shape[0] * shape[1] * shape[2] < (int64_t(1) << 40), "MAC grid too large");
    g->nx = shape[0];
    g->ny = shape[1];
    g->nz = shape[2];
    return AFSI_OK;
}

template <class T>
Faces<T> faces(void* const* f) {
    return Faces<T>{{static_cast<T*>(f[0]), static_cast<T*>(f[1]), static_cast<T*>(f[2])}};
}
template <class T>
ConstFaces<T> cfaces(const void* const* f) {
    return ConstFaces<T>{{static_cast<const T*>(f[0]), static_cast<const T*>(f[1]), static_cast<const T*>(f[2])}};
}

bool all3(const void* const* f) { return f && f[0] && f[1] && f[2]; }

int64_t face_total(const Cells& g) {
    return (g.nx + 1) * g.ny * g.nz + g.nx * (g.ny + 1) * g.nz + g.nx * g.ny * (g.nz + 1);
}

unsigned cell_blocks(const Cells& g) { return unsigned((g.nx * g.ny * g.nz + kCells - 1) / kCells); }

}  // namespace

extern "C" int64_t afsi_b200_stokes_partial_blocks(const int64_t* shape) {
    Cells g;
    if (check_cells(shape, &g)) return -1;
    return cell_blocks(g);
}

extern "C" int32_t afsi_b200_helmholtz_initialize(const void* const* b, const void* p, const void* const* diag,
                                                  void* const* rhs, void* const* u, const void* param,
                                                  const int64_t* shape, const double* spacing, int32_t dtype,
                                                  afsi_stream_t stream) {
    Cells g;
    int32_t rc = check_cells(shape, &g);
    if (rc) return rc;
    AFSI_REQUIRE(all3(b) && all3(diag) && all3(reinterpret_cast<const void* const*>(rhs)) &&
                     all3(reinterpret_cast<const void* const*>(u)) && param && spacing,
                 "null Helmholtz argument");
    const int64_t total = face_total(g);
    AFSI_DISPATCH(dtype, {
        helmholtz_initialize_kernel<T><<<blocks_for(total, 256), 256, 0, stream>>>(
            cfaces<T>(b), static_cast<const T*>(p), cfaces<T>(diag), faces<T>(rhs), faces<T>(u),
            static_cast<const T*>(param), g, spacing[0], spacing[1], spacing[2], total);
    });
    return launched("helmholtz initialize");
}

extern "C" int32_t afsi_b200_helmholtz_sweep(const void* const* u, const void* const* rhs, const void* const* diag,
                                             void* const* out, const void* param, const int64_t* shape,
                                             const double* spacing_squared, int32_t dtype, afsi_stream_t stream) {
    Cells g;
    int32_t rc = check_cells(shape, &g);
    if (rc) return rc;
    AFSI_REQUIRE(all3(u) && all3(rhs) && all3(diag) && all3(reinterpret_cast<const void* const*>(out)) && param &&
                     spacing_squared,
                 "null Helmholtz argument");
    const int64_t total = face_total(g);
    AFSI_DISPATCH(dtype, {
        helmholtz_sweep_kernel<T><<<blocks_for(total, 256), 256, 0, stream>>>(
            cfaces<T>(u), cfaces<T>(rhs), cfaces<T>(diag), faces<T>(out), static_cast<const T*>(param), g,
            spacing_squared[0], spacing_squared[1], spacing_squared[2], total);
    });
    return launched("helmholtz sweep");
}

extern "C" int32_t afsi_b200_stokes_start_partial(const void* const* b, const void* p, void* out,
                                                  const int64_t* shape, int32_t dtype, afsi_stream_t stream) {
    Cells g;
    int32_t rc = check_cells(shape, &g);
    if (rc) return rc;
    AFSI_REQUIRE(all3(b) && p && out, "null Stokes argument");
    AFSI_DISPATCH(dtype, {
        stokes_start_kernel<T><<<cell_blocks(g), kCells, 0, stream>>>(cfaces<T>(b), static_cast<const T*>(p), g,
                                                                       static_cast<T*>(out));
    });
    return launched("stokes start partial");
}

extern "C" int32_t afsi_b200_stokes_residual_partial(const void* const* u, const void* p, const void* const* b,
                                                     void* residual, void* out, const void* coefficients,
                                                     const int64_t* shape, int32_t dtype, afsi_stream_t stream) {
    Cells g;
    int32_t rc = check_cells(shape, &g);
    if (rc) return rc;
    AFSI_REQUIRE(all3(u) && all3(b) && p && residual && out && coefficients, "null Stokes argument");
    AFSI_DISPATCH(dtype, {
        stokes_residual_kernel<T><<<cell_blocks(g), kCells, 0, stream>>>(
            cfaces<T>(u), static_cast<const T*>(p), cfaces<T>(b), static_cast<T*>(residual), static_cast<T*>(out),
            static_cast<const T*>(coefficients), g);
    });
    return launched("stokes residual partial");
}

extern "C" int32_t afsi_b200_pressure_input_partial(const void* rhs, const void* p, int64_t n, void* out,
                                                    int32_t dtype, afsi_stream_t stream) {
    AFSI_REQUIRE(n > 0 && rhs && p && out, "invalid pressure input arguments");
    AFSI_DISPATCH(dtype, {
        pressure_input_kernel<T><<<unsigned((n + kCells - 1) / kCells), kCells, 0, stream>>>(
            static_cast<const T*>(rhs), static_cast<const T*>(p), n, static_cast<T*>(out));
    });
    return launched("pressure input partial");
}

extern "C" int32_t afsi_b200_pressure_norm_partial(const void* rhs, const void* p, void* out,
                                                   const void* spacing_squared, const int64_t* shape, int32_t dtype,
                                                   afsi_stream_t stream) {
    Cells g;
    int32_t rc = check_cells(shape, &g);
    if (rc) return rc;
    AFSI_REQUIRE(rhs && p && out && spacing_squared, "null pressure norm argument");
    AFSI_DISPATCH(dtype, {
        pressure_norm_kernel<T><<<cell_blocks(g), kCells, 0, stream>>>(
            static_cast<const T*>(rhs), static_cast<const T*>(p), static_cast<const T*>(spacing_squared), g,
            static_cast<T*>(out));
    });
    return launched("pressure norm partial");
}
