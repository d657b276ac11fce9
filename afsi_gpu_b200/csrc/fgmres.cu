// Kernels of the MG-preconditioned FGMRES solve of the CN saddle-point
// problem  H u + (dt/rho) G p = b,  D u = 0  on the 3D MAC grid
// (mac/stokes_fgmres.py:15-96).
//
// The Krylov vectors are packed [u0 | u1 | u2 | q]: the three face arrays,
// (nx+1,ny,nz), (nx,ny+1,nz), (nx,ny,nz+1), then the nx*ny*nz cell values,
// each row-major with z fastest (the reference's pack, stokes_fgmres.py:31-35).
//
// action (stokes_fgmres.py:36-43):
//     u'_c = (u_c - alpha L_c u) + h G_c q, zero on the two wall faces of
//            component c; L_c the face Laplacian with odd tangential ghosts
//            (-u), summed x, y, z (mac/grid.py:96-105); G_c the Neumann
//            gradient (mac/grid.py:74-83)
//     q'   = (-h) D u, D the divergence summed x, y, z (mac/grid.py:70-71)
// precondition (stokes_fgmres.py:46-63), around a Helmholtz solve of the
// velocity part and a multigrid pressure solve run by the caller:
//     rhs  = (-s)/h - D t           (t: the Helmholtz solution, s: q-part)
//     u    = t - G phi,  q = (phi + alpha rhs)/h
// with the means of rhs and q summed deterministically (per-block partials,
// the last block adds them in index order) for the caller to subtract.
//
// Each expression keeps the reference's operation order; the library is
// built with --fmad=false, so products and sums round as the reference's
// torch expressions do.
#include "common.cuh"

namespace afsi {
namespace {

constexpr int kT = 256;

struct Box {
    int64_t nx, ny, nz;
    double h[3];
    // face array sizes and the start of each part in the packed vector
    int64_t nf[3], off[4], total;
};

Box make_box(const int64_t* shape, const double* spacing) {
    Box b;
    b.nx = shape[0];
    b.ny = shape[1];
    b.nz = shape[2];
    for (int a = 0; a < 3; ++a) b.h[a] = spacing[a];
    b.nf[0] = (b.nx + 1) * b.ny * b.nz;
    b.nf[1] = b.nx * (b.ny + 1) * b.nz;
    b.nf[2] = b.nx * b.ny * (b.nz + 1);
    b.off[0] = 0;
    b.off[1] = b.nf[0];
    b.off[2] = b.nf[0] + b.nf[1];
    b.off[3] = b.off[2] + b.nf[2];
    b.total = b.off[3] + b.nx * b.ny * b.nz;
    return b;
}

__device__ __forceinline__ void dims_of(const Box& b, int c, int64_t* n) {
    n[0] = b.nx + (c == 0);
    n[1] = b.ny + (c == 1);
    n[2] = b.nz + (c == 2);
}

// Face (component c, local index i) of a flat face index t < off[3].
__device__ __forceinline__ int face_of(const Box& b, int64_t t, int64_t& i) {
    if (t < b.off[1]) {
        i = t;
        return 0;
    }
    if (t < b.off[2]) {
        i = t - b.off[1];
        return 1;
    }
    i = t - b.off[2];
    return 2;
}

template <class T>
__device__ __forceinline__ T h_of(const Box& b, int a) {
    return T(a == 0 ? b.h[0] : (a == 1 ? b.h[1] : b.h[2]));
}

// Divergence of the face fields U (u0, u1, u2 consecutive at U + off[c]) at cell (x,y,z).
template <class T>
__device__ __forceinline__ T divergence_at(const Box& b, const T* u0, const T* u1, const T* u2, int64_t x,
                                           int64_t y, int64_t z) {
    const int64_t i0 = (x * b.ny + y) * b.nz + z;
    const T d0 = (u0[i0 + b.ny * b.nz] - u0[i0]) / h_of<T>(b, 0);
    const int64_t i1 = (x * (b.ny + 1) + y) * b.nz + z;
    const T d1 = (u1[i1 + b.nz] - u1[i1]) / h_of<T>(b, 1);
    const int64_t i2 = (x * b.ny + y) * (b.nz + 1) + z;
    const T d2 = (u2[i2 + 1] - u2[i2]) / h_of<T>(b, 2);
    return (d0 + d1) + d2;
}

// G_c q at face (c; x, y, z) of its lattice: 0 on the two wall faces.
template <class T>
__device__ __forceinline__ T gradient_at(const Box& b, const T* q, int c, int64_t x, int64_t y, int64_t z,
                                         int64_t coord, int64_t n_c) {
    if (coord == 0 || coord == n_c - 1) return T(0);
    const int64_t right = (x * b.ny + y) * b.nz + z;  // the cell on the + side of the face
    const int64_t stride = c == 0 ? b.ny * b.nz : (c == 1 ? b.nz : 1);
    return (q[right] - q[right - stride]) / h_of<T>(b, c);
}

// Deterministic grid sum: per-block partial, last block adds them in order.
__device__ __forceinline__ void grid_sum(double v, double* partial, unsigned* counter, double* out) {
    __shared__ double sh[kT / 32];
    __shared__ bool last;
    v = block_sum(v, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
    if (!grid_reduce_arrive(counter, &last)) return;
    v = sum_partials(partial, gridDim.x, 1, 0, sh);
    if (threadIdx.x == 0) {
        *out = v;
        *counter = 0u;
    }
}

template <class T>
__global__ void __launch_bounds__(kT) action_kernel(const T* __restrict__ v, T* __restrict__ out, Box b, T alpha,
                                                    T hmin) {
    const int64_t t = int64_t(blockIdx.x) * kT + threadIdx.x;
    if (t >= b.total) return;
    const T* u0 = v;
    const T* u1 = v + b.off[1];
    const T* u2 = v + b.off[2];
    const T* q = v + b.off[3];
    if (t >= b.off[3]) {
        const int64_t i = t - b.off[3];
        const int64_t z = i % b.nz, y = (i / b.nz) % b.ny, x = i / (b.nz * b.ny);
        out[t] = (-hmin) * divergence_at(b, u0, u1, u2, x, y, z);
        return;
    }
    int64_t i;
    const int c = face_of(b, t, i);
    int64_t n[3];
    dims_of(b, c, n);
    const int64_t z = i % n[2], y = (i / n[2]) % n[1], x = i / (n[1] * n[2]);
    const int64_t coord = c == 0 ? x : (c == 1 ? y : z);
    const int64_t nc = c == 0 ? n[0] : (c == 1 ? n[1] : n[2]);
    if (coord == 0 || coord == nc - 1) {
        out[t] = T(0);
        return;
    }
    const T* U = c == 0 ? u0 : (c == 1 ? u1 : u2);
    const T val = U[i];
    const int64_t sx = n[1] * n[2], sy = n[2];
    const T xm = x > 0 ? U[i - sx] : -val, xp = x + 1 < n[0] ? U[i + sx] : -val;
    const T ym = y > 0 ? U[i - sy] : -val, yp = y + 1 < n[1] ? U[i + sy] : -val;
    const T zm = z > 0 ? U[i - 1] : -val, zp = z + 1 < n[2] ? U[i + 1] : -val;
    T lap = ((xm - T(2) * val) + xp) / T(b.h[0] * b.h[0]);
    lap = lap + ((ym - T(2) * val) + yp) / T(b.h[1] * b.h[1]);
    lap = lap + ((zm - T(2) * val) + zp) / T(b.h[2] * b.h[2]);
    const T g = gradient_at(b, q, c, x, y, z, coord, nc);
    out[t] = (val - alpha * lap) + hmin * g;
}

// rhs = (-s)/h - D t over the cells, with its sum.
template <class T>
__global__ void __launch_bounds__(kT) precondition_rhs_kernel(const T* __restrict__ t0, const T* __restrict__ t1,
                                                              const T* __restrict__ t2, const T* __restrict__ s,
                                                              T* __restrict__ rhs, Box b, T hmin, double* partial,
                                                              unsigned* counter, double* sum_out) {
    const int64_t i = int64_t(blockIdx.x) * kT + threadIdx.x;
    const int64_t cells = b.nx * b.ny * b.nz;
    double local = 0.0;
    if (i < cells) {
        const int64_t z = i % b.nz, y = (i / b.nz) % b.ny, x = i / (b.nz * b.ny);
        const T r = (-s[i]) / hmin - divergence_at(b, t0, t1, t2, x, y, z);
        rhs[i] = r;
        local = double(r);
    }
    grid_sum(local, partial, counter, sum_out);
}

// out = pack(t - G phi, (phi + alpha rhs)/h) with the sum of the q-part.
template <class T>
__global__ void __launch_bounds__(kT) precondition_result_kernel(const T* __restrict__ t0, const T* __restrict__ t1,
                                                                 const T* __restrict__ t2,
                                                                 const T* __restrict__ phi,
                                                                 const T* __restrict__ rhs, T* __restrict__ out,
                                                                 Box b, T alpha, T hmin, double* partial,
                                                                 unsigned* counter, double* sum_out) {
    const int64_t t = int64_t(blockIdx.x) * kT + threadIdx.x;
    double local = 0.0;
    if (t < b.off[3]) {
        int64_t i;
        const int c = face_of(b, t, i);
        int64_t n[3];
        dims_of(b, c, n);
        const int64_t z = i % n[2], y = (i / n[2]) % n[1], x = i / (n[1] * n[2]);
        const int64_t coord = c == 0 ? x : (c == 1 ? y : z);
        const int64_t nc = c == 0 ? n[0] : (c == 1 ? n[1] : n[2]);
        const T* tc = c == 0 ? t0 : (c == 1 ? t1 : t2);
        out[t] = tc[i] - gradient_at(b, phi, c, x, y, z, coord, nc);
    } else if (t < b.total) {
        const int64_t i = t - b.off[3];
        const T q = (phi[i] + alpha * rhs[i]) / hmin;
        out[t] = q;
        local = double(q);
    }
    grid_sum(local, partial, counter, sum_out);
}

int32_t check_box(const int64_t* shape, const double* spacing, Box& b) {
    AFSI_REQUIRE(shape && spacing, "null shape or spacing");
    for (int a = 0; a < 3; ++a) {
        AFSI_REQUIRE(shape[a] >= 2 && shape[a] <= (1 << 16), "cell count %lld out of range", (long long)shape[a]);
        AFSI_REQUIRE(spacing[a] > 0 && isfinite(spacing[a]), "spacing must be positive");
    }
    b = make_box(shape, spacing);
    AFSI_REQUIRE(b.total < (int64_t(1) << 40), "grid too large");
    return AFSI_OK;
}

struct Scratch {
    double* partial;
    unsigned* counter;
};

Scratch scratch_of(void* p, int64_t blocks) {
    unsigned char* c = static_cast<unsigned char*>(p);
    return Scratch{reinterpret_cast<double*>(c), reinterpret_cast<unsigned*>(c + blocks * 8)};
}

}  // namespace
}  // namespace afsi

using namespace afsi;

extern "C" int64_t afsi_b200_stokes_packed_size(const int64_t* shape) {
    if (!shape || shape[0] < 2 || shape[1] < 2 || shape[2] < 2) return -1;
    const double one[3] = {1, 1, 1};
    return make_box(shape, one).total;
}

extern "C" int64_t afsi_b200_stokes_precondition_scratch_bytes(const int64_t* shape) {
    const int64_t total = afsi_b200_stokes_packed_size(shape);
    if (total < 0) return -1;
    return (total + kT - 1) / kT * 8 + 16;
}

extern "C" int32_t afsi_b200_stokes_action(const void* v, void* out, const int64_t* shape, const double* spacing,
                                           double alpha, double h, int32_t dtype, afsi_stream_t stream) {
    Box b;
    int32_t rc = check_box(shape, spacing, b);
    if (rc) return rc;
    AFSI_REQUIRE(v && out && v != out, "action needs distinct input and output vectors");
    AFSI_DISPATCH(dtype, {
        action_kernel<T><<<blocks_for(b.total, kT), kT, 0, static_cast<cudaStream_t>(stream)>>>(
            static_cast<const T*>(v), static_cast<T*>(out), b, T(alpha), T(h));
    });
    return launched("stokes action");
}

extern "C" int32_t afsi_b200_stokes_precondition_rhs(const void* const* tentative, const void* s, void* rhs,
                                                     double* sum_out, void* scratch, const int64_t* shape,
                                                     const double* spacing, double h, int32_t dtype,
                                                     afsi_stream_t stream) {
    Box b;
    int32_t rc = check_box(shape, spacing, b);
    if (rc) return rc;
    AFSI_REQUIRE(tentative && tentative[0] && tentative[1] && tentative[2] && s && rhs && sum_out && scratch,
                 "null preconditioner argument");
    const int64_t cells = b.nx * b.ny * b.nz;
    const unsigned blocks = blocks_for(cells, kT);
    const Scratch sc = scratch_of(scratch, blocks_for(b.total, kT));
    AFSI_DISPATCH(dtype, {
        precondition_rhs_kernel<T><<<blocks, kT, 0, static_cast<cudaStream_t>(stream)>>>(
            static_cast<const T*>(tentative[0]), static_cast<const T*>(tentative[1]),
            static_cast<const T*>(tentative[2]), static_cast<const T*>(s), static_cast<T*>(rhs), b, T(h),
            sc.partial, sc.counter, sum_out);
    });
    return launched("stokes precondition rhs");
}

extern "C" int32_t afsi_b200_stokes_precondition_result(const void* const* tentative, const void* phi,
                                                        const void* rhs, void* out, double* sum_out, void* scratch,
                                                        const int64_t* shape, const double* spacing, double alpha,
                                                        double h, int32_t dtype, afsi_stream_t stream) {
    Box b;
    int32_t rc = check_box(shape, spacing, b);
    if (rc) return rc;
    AFSI_REQUIRE(tentative && tentative[0] && tentative[1] && tentative[2] && phi && rhs && out && sum_out &&
                     scratch,
                 "null preconditioner argument");
    const unsigned blocks = blocks_for(b.total, kT);
    const Scratch sc = scratch_of(scratch, blocks);
    AFSI_DISPATCH(dtype, {
        precondition_result_kernel<T><<<blocks, kT, 0, static_cast<cudaStream_t>(stream)>>>(
            static_cast<const T*>(tentative[0]), static_cast<const T*>(tentative[1]),
            static_cast<const T*>(tentative[2]), static_cast<const T*>(phi), static_cast<const T*>(rhs),
            static_cast<T*>(out), b, T(alpha), T(h), sc.partial, sc.counter, sum_out);
    });
    return launched("stokes precondition result");
}
