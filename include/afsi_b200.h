/*
 * afsi_b200.h — C-ABI of the B200 (sm_100a) IB-transfer and MAC-multigrid kernels.
 *
 * Every entry point takes raw device pointers, element counts, a dtype code
 * and a CUDA stream, launches asynchronously on that stream and returns a
 * host status (AFSI_OK or an AFSI_ERR_* code; afsi_b200_last_error() gives
 * the message of the calling thread's last failure).  Data-dependent faults
 * found on the device (support leaving the grid, a stencil index outside the
 * grid, a non-finite value) never trap: the kernel ORs an AFSI_FLAG_* bit
 * into the caller's device word `status` and skips the access.
 *
 * No entry point allocates, frees or synchronises, so every one may be
 * recorded into a CUDA graph.  Layouts are row-major, contiguous, z (or y in
 * 2D) fastest, exactly as the reference tensors.
 *
 * Reference interfaces replaced (paths inside afsi-torch 0.28.0,
 * src/afsi_torch/):
 *   indexed_gather / indexed_spread     mac/csrc/transfer.cpp:48-57
 *   compact_gather / compact_spread     mac/csrc/transfer.cpp:50-51
 *   p2_prepare_ / p2_spread_ /
 *   p2_gather_assemble_                 mac/csrc/p2_transfer.cpp:66-74
 *   compact prepare (_prepare)          mac/compact_transfer.py:21-26
 *   2D reflected prepare (_prepare)     mac2d/transfer.py:61-81
 *   MG kernel objects smooth / residual / restrict / residual_restrict /
 *   prolong_add                          mac/_triton_mg.py:121-151,
 *                                        mac2d/_triton_mg.py:78-100
 *   V-cycle block + residual norm       mac/mg_workspace.py:85-133,
 *                                        mac2d/mg_workspace.py:45-106
 */
#ifndef AFSI_B200_H
#define AFSI_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* afsi_stream_t; /* same object as cudaStream_t */

/* dtype codes */
#define AFSI_F32 0
#define AFSI_F64 1

/* host status */
#define AFSI_OK 0
#define AFSI_ERR_ARG 1     /* invalid argument (shape, size, null pointer, dtype) */
#define AFSI_ERR_CUDA 2    /* the CUDA runtime reported an error */

/* device status bits (OR-ed into *status; the caller zeroes it) */
#define AFSI_FLAG_SUPPORT 1  /* a point's 4-point support leaves the grid, or it is non-finite */
#define AFSI_FLAG_INDEX 2    /* a stencil table addressed outside the grid/node range */
#define AFSI_FLAG_OVERFLOW 4 /* a bounded table or buffer overflowed */
#define AFSI_FLAG_TIMEOUT 8  /* a bounded wait for an asynchronous copy gave up (the work it fed was skipped) */

/* Peskin weight forms: clamped two-branch kernel (ib.py:57-67, the torch
 * path) or the shared radical (mac/csrc/p2_transfer.cu:36-43). */
#define AFSI_PHI_CLAMPED 0
#define AFSI_PHI_RADICAL 1

const char* afsi_b200_last_error(void);
int32_t afsi_b200_version(void);
/* Kernels this process has launched through the library (graph replays excluded). */
int64_t afsi_b200_launch_count(void);

/* ------------------------------------------------------------------ prepare */

/* Binning + 1D weights on `lattices` staggered lattices
 * (mac/compact_transfer.py:21-26; shared face/centre tables of
 * mac/shared_stencil.py:8-19 when lattices==2).
 *   points (P,3); origins (lattices,3) and spacing (3) host arrays;
 *   base (lattices,P,3) int64; phi (lattices,P,3,4).
 * The support test of compact_transfer.py:94-96 (2 <= (x-grid_origin)/h <
 * shape-2, finite) is fused: a failing point sets AFSI_FLAG_SUPPORT. */
int32_t afsi_b200_compact_prepare(const void* points, int64_t count, int32_t lattices,
    const double* origins, const double* spacing, const double* grid_origin,
    const int64_t* shape, int32_t phi_form, int64_t* base, void* phi,
    int32_t* status, int32_t dtype, afsi_stream_t stream);

/* 2D reflected 4x4 stencils of both velocity components (mac2d/transfer.py:61-81).
 *   points (P,2); ids (2,P,16) int64; weights (2,P,16).
 * The support screen of mac2d/transfer.py:97-101 is fused (AFSI_FLAG_SUPPORT). */
int32_t afsi_b200_indexed_prepare2d(const void* points, int64_t count, int64_t nx, int64_t ny,
    double hx, double hy, double lx, double ly, int64_t* ids, void* weights,
    int32_t* status, int32_t dtype, afsi_stream_t stream);

/* P2 quadrature-point positions and shared face/centre tables for one
 * quadrature group (p2_prepare_, mac/csrc/p2_transfer.cpp:55-63 and
 * p2_transfer.cu:12-45).
 *   x (nodes,3); cells (elements,10) int64; N (nq,10);
 *   origin/spacing/limits host arrays (3); base (2,total,3); phi (2,total,3,4);
 *   rows offset..offset+elements*nq are written. */
int32_t afsi_b200_p2_prepare(const void* x, int64_t nodes, const int64_t* cells, int64_t elements,
    const void* N, int64_t nq, const double* origin, const double* spacing, const double* limits,
    int64_t* base, void* phi, int64_t total, int64_t offset, int32_t* status,
    int32_t dtype, afsi_stream_t stream);

/* Precision form of the P2 / P1 prepares (nodes_per_cell 10 or 4): positions,
 * bases and weights formed in FP64 from FP64 x and N exactly as
 * afsi_b200_p2_prepare / afsi_b200_p1_prepare do, the weights stored in
 * weight_dtype (AFSI_F32: the rounded FP64 weights), so the bases are the
 * FP64 bases.  No counterpart in the reference (its tables take the
 * positions' dtype). */
int32_t afsi_b200_fe_prepare_mixed(int32_t nodes_per_cell, const double* x, int64_t nodes, const int64_t* cells,
    int64_t elements, const double* N, int64_t nq, const double* origin, const double* spacing,
    const double* limits, int64_t* base, void* phi, int64_t total, int64_t offset, int32_t* status,
    int32_t weight_dtype, afsi_stream_t stream);

/* Deterministic, atomic-free spread over the shared (2,T,3)/(2,T,3,4)
 * tables (no counterpart in the reference, whose spreads add atomically).
 * afsi_b200_det_plan (once per stencil): each row's support is binned by
 *   its owning 8x8x8 face tile per component and the rows sorted by tile
 *   (stable); rows whose support leaves the face array flag AFSI_FLAG_INDEX
 *   and are left out.  plan: afsi_b200_det_plan_bytes() device bytes.
 * afsi_b200_det_spread: u_c += the spread of force[:, c] (force (T,3), one
 *   value per table row, already multiplied by W / volume): per tile, the
 *   rows in sorted order into per-warp shared-memory boxes summed in warp
 *   order, then every face adds the covering tiles' boxes in a fixed order.
 *   Bitwise reproducible; equal to the atomic spreads to rounding.
 * afsi_b200_p2_point_forces: force rows offset..offset+elements*nq of one
 *   P2 group, (sum_a N[q,a] value[cell_a]) * W[e,q] / volume as the P2
 *   spread forms them (p2_spread_, mac/csrc/p2_transfer.cu:98-188). */
int64_t afsi_b200_det_plan_bytes(int64_t total, int64_t nx, int64_t ny, int64_t nz, int32_t dtype);
int32_t afsi_b200_det_plan(const int64_t* base, int64_t total, int64_t nx, int64_t ny, int64_t nz, void* plan,
    int64_t plan_bytes, int32_t* status, int32_t dtype, afsi_stream_t stream);
int32_t afsi_b200_det_spread(const void* force, const int64_t* base, const void* phi, int64_t total, int64_t nx,
    int64_t ny, int64_t nz, void* plan, int64_t plan_bytes, void* u0, void* u1, void* u2, int32_t dtype,
    afsi_stream_t stream);
int32_t afsi_b200_p2_point_forces(const void* value, int64_t nodes, const int64_t* cells, int64_t elements,
    const void* N, int64_t nq, const void* W, int64_t total, int64_t offset, double volume, void* force,
    int32_t* status, int32_t dtype, afsi_stream_t stream);

/* Adaptive quadrature order per P2 element: ceil(density * D / dx), at least
 * min_order, D the diameter of the element's Bernstein control points
 * (_orders_p2, mac/adaptive_transfer.py:182-187, which the reference
 * compiles with torch.compile and follows with torch.equal against the last
 * rule's orders, :266-273).
 *   x (nodes,3); cells (elements,10) int64; orders (elements) int64 out;
 *   last_orders (elements) or NULL;
 *   summary int32[3+bins], cleared here: [0] elements whose order differs
 *   from last_orders (all when NULL), [1] largest order, [2] device flags
 *   (AFSI_FLAG_INDEX: node id out of range, AFSI_FLAG_SUPPORT: nonfinite
 *   position; such elements get order 0), [3+n] elements of order n < bins.
 *   bins in [1, 64].  The flags slot may be passed on as the status word of a
 *   following afsi_b200_p2_prepare so that one read covers both launches. */
int32_t afsi_b200_p2_orders(const void* x, int64_t nodes, const int64_t* cells, int64_t elements,
    double dx, double density, int64_t min_order, int64_t* orders, const int64_t* last_orders,
    int32_t* summary, int32_t bins, int32_t dtype, afsi_stream_t stream);

/* P1 counterparts of afsi_b200_p2_prepare / afsi_b200_p2_orders for 4-node
 * cells: positions sum N[q,a]*x[cell_a] over the four nodes
 * (mac/_triton_prepare.py:12-49); orders are ceil(density * longest edge /
 * dx), callers pass min_order 2 (_orders, mac/adaptive_transfer.py:167-170).
 * cells (elements,4); N (nq,4).  Same tables, status and summary contracts. */
int32_t afsi_b200_p1_prepare(const void* x, int64_t nodes, const int64_t* cells, int64_t elements,
    const void* N, int64_t nq, const double* origin, const double* spacing, const double* limits,
    int64_t* base, void* phi, int64_t total, int64_t offset, int32_t* status,
    int32_t dtype, afsi_stream_t stream);
int32_t afsi_b200_p1_orders(const void* x, int64_t nodes, const int64_t* cells, int64_t elements,
    double dx, double density, int64_t min_order, int64_t* orders, const int64_t* last_orders,
    int32_t* summary, int32_t bins, int32_t dtype, afsi_stream_t stream);

/* -------------------------------------------------------------- P1 CSR */

/* Support box of every cell of one quadrature group for component c
 * (component_plans, mac/hash_transfer_assembly.py:122-138): low (E,3) = min
 * base, width (E,3) = max - min + 4, prefix (E+1) = exclusive scan of the
 * box sizes (prefix[E] = the group's site count).  base is the (L,total,3)
 * table; shared != 0 for the (2,T,3) face/centre layout (axis a of
 * component c reads lattice a != c), else the (3,T,3) component layout.
 * scratch: afsi_b200_p1_plan_scratch_bytes(E) device bytes. */
int64_t afsi_b200_p1_plan_scratch_bytes(int64_t elements);
int32_t afsi_b200_p1_component_plan(const int64_t* base, int64_t total, int64_t offset, int64_t elements,
    int64_t nq, int32_t component, int32_t shared, int64_t* low, int64_t* width, int64_t* prefix,
    void* scratch, int64_t scratch_bytes, afsi_stream_t stream);

/* hash_contract_ (mac/csrc/ib.cpp:58-67, ib.cu:22-116): for each site of
 * each cell's box, the four nodal sums sum_q W*N[q,a]*phi_x*phi_y*phi_z are
 * added into the table (keys (capacity) int64, -1 = empty; values
 * (capacity)) under key node*nf + face.  capacity is a power of two; the
 * table's hashing and probing are the reference's (SplitMix64 bucket, linear
 * probe, at most 128 slots), and *flag is set to 1 on a failed probe, a
 * negative key, a site outside the face array or a malformed plan.  Only
 * sites < count are visited.  N (nq,4), W (elements,nq), cells (elements,4),
 * rows offset..offset+elements*nq of the tables. */
int32_t afsi_b200_hash_contract(const int64_t* base, const void* phi, const void* N, const void* W,
    const int64_t* cells, const int64_t* low, const int64_t* width, const int64_t* prefix,
    int64_t* keys, void* values, int32_t* flag, int64_t capacity, int64_t total, int64_t offset,
    int64_t elements, int64_t nq, int64_t count, int32_t component, int64_t ny, int64_t nz,
    int64_t nf, int32_t shared, int32_t dtype, afsi_stream_t stream);
/* cached_contract_ (mac/csrc/ib.cpp:69-81): keys are only looked up; a key
 * not in the table is appended to the missing stream (missing_count, int64,
 * counts every miss; entries past missing_capacity are not written). */
int32_t afsi_b200_cached_contract(const int64_t* base, const void* phi, const void* N, const void* W,
    const int64_t* cells, const int64_t* low, const int64_t* width, const int64_t* prefix,
    const int64_t* keys, void* values, int32_t* flag, int64_t capacity, int64_t* missing_keys,
    void* missing_values, int64_t* missing_count, int64_t missing_capacity, int64_t total,
    int64_t offset, int64_t elements, int64_t nq, int64_t count, int32_t component, int64_t ny,
    int64_t nz, int64_t nf, int32_t shared, int32_t dtype, afsi_stream_t stream);
/* hash_accumulate_ (mac/csrc/ib.cpp:83-92): insert count (key, value) pairs. */
int32_t afsi_b200_hash_accumulate(const int64_t* input_keys, const void* input_values, int64_t count,
    int64_t* keys, void* values, int32_t* flag, int64_t capacity, int32_t dtype, afsi_stream_t stream);

/* Table -> CSR of B (rows x nf, key = row*nf + col) and of its transpose
 * (finish_component, mac/hash_transfer_assembly.py:105-119): crow (rows+1),
 * col/val (capacity; the first nnz are B's entries, column-sorted rows),
 * t_crow (nf+1), t_col/t_val (capacity; Bᵀ).  info (device int64[2]):
 * [0] nnz, [1] 1 if a key lies outside [0, rows*nf) or a value is
 * nonfinite.  No host synchronisation.  scratch:
 * afsi_b200_hash_csr_scratch_bytes(capacity, dtype) device bytes. */
int64_t afsi_b200_hash_csr_scratch_bytes(int64_t capacity, int32_t dtype);
int32_t afsi_b200_hash_csr(const int64_t* keys, const void* values, int64_t capacity, int64_t rows, int64_t nf,
    int64_t* crow, int64_t* col, void* val, int64_t* t_crow, int64_t* t_col, void* t_val, int64_t* info,
    void* scratch, int64_t scratch_bytes, int32_t dtype, afsi_stream_t stream);

/* y[r*y_stride] = (sum_j val[j] * x[col[j]*x_stride]) / divisor for the rows
 * of a CSR matrix with nnz entries: the responses of the assembled P1
 * transfer (AssembledP1Transfer.spread/interpolate,
 * mac/assembled_transfer.py:195-212; torch.sparse.mm there).  Each row is
 * summed in a fixed order: deterministic. */
int32_t afsi_b200_csr_spmv(const int64_t* crow, const int64_t* col, const void* val, int64_t rows, int64_t nnz,
    const void* x, int64_t x_stride, void* y, int64_t y_stride, double divisor, int32_t dtype,
    afsi_stream_t stream);

/* ----------------------------------------------------------------- transfer */

/* out[p,c] = sum_k field[ids[p,k],c]*w[p,k]   (indexed_gather) */
int32_t afsi_b200_indexed_gather(const void* field, int64_t nodes, int64_t components,
    const int64_t* ids, const void* weights, int64_t points, int64_t neighbors,
    void* out, int32_t* status, int32_t dtype, afsi_stream_t stream);

/* out[ids[p,k],c] += (field[p,c]*w[p,k])/volume   (indexed_spread).
 * `out` (size,components) is accumulated into; zero it first for the
 * reference's fresh-output semantics. */
int32_t afsi_b200_indexed_spread(const void* field, int64_t points, int64_t components,
    const int64_t* ids, const void* weights, int64_t neighbors, int64_t size, double volume,
    void* out, int32_t* status, int32_t dtype, afsi_stream_t stream);

/* One component of the separable 3D transfer (compact_gather):
 * out[p] = sum_{ijk} field[(x*ny+y)*nz+z]*(phi_x[i]*phi_y[j])*phi_z[k].
 *   base (P,3) int64, phi (P,3,4); nx,ny,nz = this component's face shape. */
int32_t afsi_b200_compact_gather(const void* field, const int64_t* base, const void* phi,
    int64_t points, int64_t nx, int64_t ny, int64_t nz, void* out,
    int32_t* status, int32_t dtype, afsi_stream_t stream);

/* One component of compact_spread, accumulating (w*f)/volume into `out`. */
int32_t afsi_b200_compact_spread(const void* field, const int64_t* base, const void* phi,
    int64_t points, int64_t nx, int64_t ny, int64_t nz, double volume, void* out,
    int32_t* status, int32_t dtype, afsi_stream_t stream);

/* P2 fused spread of one quadrature group (p2_spread_): for element e and
 * point q, F = (sum_a N[q,a]*value[cells[e,a]])*W[e,q], spread with the shared
 * tables rows offset+e*nq+q into the three MAC face arrays (accumulated).
 * nx,ny,nz are cell counts. */
int32_t afsi_b200_p2_spread(const void* value, int64_t nodes, const int64_t* cells, int64_t elements,
    const void* N, int64_t nq, const void* W, const int64_t* base, const void* phi,
    int64_t total, int64_t offset, void* u0, void* u1, void* u2,
    int64_t nx, int64_t ny, int64_t nz, double volume, int32_t* status,
    int32_t dtype, afsi_stream_t stream);

/* P2 fused gather + FE assembly of one group (p2_gather_assemble_):
 * rhs[cells[e,a],c] += sum_q N[q,a]*W[e,q]*U_c(q), accumulated atomically. */
int32_t afsi_b200_p2_gather_assemble(const void* u0, const void* u1, const void* u2,
    const int64_t* cells, int64_t elements, const void* N, int64_t nq, const void* W,
    const int64_t* base, const void* phi, int64_t total, int64_t offset, void* rhs, int64_t nodes,
    int64_t nx, int64_t ny, int64_t nz, int32_t* status, int32_t dtype, afsi_stream_t stream);

/* Deterministic form of the assembly: element-local sums are written to
 * local (elements,10,3) in a fixed order (no atomics); afsi_b200_node_reduce
 * then sums them per node through a node->(element,slot) CSR. */
int32_t afsi_b200_p2_gather_local(const void* u0, const void* u1, const void* u2,
    const int64_t* cells, int64_t elements, const void* N, int64_t nq, const void* W,
    const int64_t* base, const void* phi, int64_t total, int64_t offset, void* local,
    int64_t nx, int64_t ny, int64_t nz, int32_t* status, int32_t dtype, afsi_stream_t stream);

/* rhs[n,:] (+)= sum_{k in crow[n]..crow[n+1]} local[slot[k],:] for 3 components,
 * slot = element*10+a; accumulate!=0 adds to rhs, else overwrites. */
int32_t afsi_b200_node_reduce(const void* local, int64_t slots, const int64_t* crow,
    const int64_t* slot, int64_t nodes, void* rhs, int32_t accumulate,
    int32_t* status, int32_t dtype, afsi_stream_t stream);

/* --------------------------------------------------------------- multigrid */

/* Boundary conditions of the pressure operator */
#define AFSI_BC_NEUMANN 0  /* closed box (mac/grid.py:86-93), singular, mean-zero gauge */
#define AFSI_BC_CHANNEL 1  /* 2D inlet/outlet channel (mac2d/grid.py:61-71), p=0 outlet */
#define AFSI_BC_PERIODIC 2 /* 2D periodic in x, Neumann walls in y, mean-zero gauge */
#define AFSI_BC_DIRICHLET 3 /* 3D open box, p = 0 on the physical faces (mac/open_boundary.py:14-52) */

/* Elementwise MG kernels on one level (the kernel-object interface of
 * mac/_triton_mg.py:121-151 and mac2d/_triton_mg.py:78-100).
 * shape = (nx,ny,nz) cells (nz=1 for 2D); h2 = h*h per axis;
 * inv_h2 = 1/h**2 per axis (the diagonal terms). */
int32_t afsi_b200_mg_smooth(const void* p, const void* rhs, void* out, const int64_t* shape,
    const double* h2, const double* inv_h2, int32_t dim, int32_t bc, int32_t dtype,
    afsi_stream_t stream);
int32_t afsi_b200_mg_residual(const void* p, const void* rhs, void* out, const int64_t* shape,
    const double* h2, int32_t dim, int32_t bc, int32_t dtype, afsi_stream_t stream);
/* coarse = mean of the 2^dim children of fine; shape = fine shape */
int32_t afsi_b200_mg_restrict(const void* fine, void* coarse, const int64_t* shape, int32_t dim,
    int32_t dtype, afsi_stream_t stream);
int32_t afsi_b200_mg_residual_restrict(const void* p, const void* rhs, void* coarse,
    const int64_t* shape, const double* h2, int32_t dim, int32_t bc, int32_t dtype,
    afsi_stream_t stream);
/* fine += prolong(coarse); shape = fine shape */
int32_t afsi_b200_mg_prolong_add(const void* coarse, void* fine, const int64_t* shape, int32_t dim,
    int32_t bc, int32_t dtype, afsi_stream_t stream);

#define AFSI_MG_MAX_LEVELS 12

typedef struct afsi_mg_level {
    int64_t shape[3];   /* cells per axis; shape[2]==1 in 2D */
    double h2[3];       /* h*h */
    double inv_h2[3];   /* 1/h**2 */
    void* p;            /* canonical iterate */
    void* ping;         /* Jacobi partner buffer */
    void* rhs;          /* right-hand side */
} afsi_mg_level;

typedef struct afsi_mg_plan {
    int32_t dim;           /* 2 or 3 */
    int32_t bc;            /* AFSI_BC_* */
    int32_t levels;        /* number of levels, finest first */
    int32_t smooth;        /* Jacobi sweeps before and after the correction */
    int32_t dtype;         /* dtype of p/ping/rhs */
    int32_t coarse_dtype;  /* dtype of coarse_inverse */
    afsi_mg_level level[AFSI_MG_MAX_LEVELS];
    const void* coarse_inverse;  /* (n,n), n = cells on the coarsest level */
    void* scratch;         /* reduction scratch, afsi_b200_mg_scratch_bytes() */
    int32_t smoother;      /* AFSI_MG_JACOBI (the reference's) or AFSI_MG_RED_BLACK */
} afsi_mg_plan;

/* Smoothers.  AFSI_MG_JACOBI is the reference's weighted Jacobi (omega 2/3,
 * mac/multigrid.py:107-110) with its mean gauge after every sweep.
 * AFSI_MG_RED_BLACK is a method change with no counterpart in the reference:
 * `smooth` red-black Gauss-Seidel sweeps (omega 1, in place) before and
 * after the coarse correction, coarse right-hand sides shifted to mean zero,
 * the finest iterate shifted to mean zero once per cycle (singular BCs); its
 * solves agree with the Jacobi solves at the solve tolerance, not per cycle.
 * The persistent entry point supports Jacobi only. */
#define AFSI_MG_JACOBI 0
#define AFSI_MG_RED_BLACK 1

/* Bytes of device scratch (zero-initialised once by the caller) a plan needs. */
int64_t afsi_b200_mg_scratch_bytes(const afsi_mg_plan* plan);

/* `cycles` V-cycles on level 0 (mac/mg_workspace.py:85-102,
 * mac2d/mg_workspace.py:53-62): weighted Jacobi (omega=2/3), residual
 * restriction, recursive correction, dense coarsest solve, prolongation.
 * p[0] and rhs[0] are read and p[0] is updated in place. */
int32_t afsi_b200_mg_vcycles(const afsi_mg_plan* plan, int32_t cycles, afsi_stream_t stream);

/* Persistent form of the above: all cycles in one cooperative launch (one
 * 1024-thread block per SM, grid barriers with a clock-bounded wait).
 * solve == 0: run `cycles` V-cycles.  solve != 0: run V-cycles until the
 * residual norm ||rhs[0] - A p[0]|| is <= tol, checked on the device after
 * every `check_every` cycles and after the last of at most `cycles`
 * (mac/multigrid.py:88-97); info (device double[3]) receives {cycles run,
 * last residual norm or -1 if unchecked, 0 or 1 if a barrier timed out}.
 * sync_scratch: afsi_b200_mg_sync_bytes() zero-initialised device bytes,
 * private to one stream at a time. */
/* The solve loop (mac/multigrid.py:88-97) as one CUDA graph: a WHILE
 * conditional node whose body runs check_every V-cycles, the residual norm
 * into `norm` (device double) and a decide kernel on `loop` (device
 * double[4]: [0] tol, written by the caller before each launch; [1] cycles
 * run, reset by the caller; [2] last residual norm; [3] 1 if it was
 * nonfinite).  The loop ends when the norm is <= tol, nonfinite, or another
 * block of check_every cycles would pass max_cycles (the caller runs any
 * remaining cycles itself).  Requires 1 <= check_every <= max_cycles.  The
 * graph is captured on a private stream and launched on the caller's. */
int32_t afsi_b200_mg_solve_graph_create(const afsi_mg_plan* plan, int32_t check_every, int32_t max_cycles,
    double* loop, double* norm, void** graph_out);
/* The same loop with the start of a solve in front of it, so that a solve is
 * one graph launch and one host read (mac/multigrid.py:125-172): the
 * statistics of the right-hand side and the initial iterate in level 0
 * (afsi_b200_vector_stats into `stats` [0:4] and [4:8]), for singular
 * operators their gauge shift (afsi_b200_subtract_mean) and the statistics
 * of the shifted right-hand side [8:12] (else a copy of [0:4]), the initial
 * residual norm, then a one-thread kernel that writes loop[0] =
 * max(atol, rtol sqrt(stats[10])), loop[1] = 0, loop[2] = the initial norm,
 * loop[3] = its nonfinite flag, and enters the loop only when that norm is
 * above the tolerance and the inputs are finite and (singular operators)
 * pass the compatibility screen |sum b|/n <= 1e-12 + rel |b|_1/n.
 * params: device double[4] = [rtol, atol, rel, n], written by the caller;
 * stat_scratch: the scratch of afsi_b200_vector_stats. */
int32_t afsi_b200_mg_solve_graph_create_started(const afsi_mg_plan* plan, int32_t check_every,
    int32_t max_cycles, double* loop, double* norm, double* stats, void* stat_scratch, const double* params,
    void** graph_out);
int32_t afsi_b200_mg_solve_graph_launch(void* graph, afsi_stream_t stream);
int32_t afsi_b200_mg_solve_graph_destroy(void* graph);

int64_t afsi_b200_mg_sync_bytes(void);
int32_t afsi_b200_mg_persistent(const afsi_mg_plan* plan, int32_t cycles, int32_t solve, int32_t check_every,
    double tol, double* info, void* sync_scratch, afsi_stream_t stream);

/* norm_out (device double) = || rhs[0] - A p[0] ||_2 (deterministic). */
int32_t afsi_b200_mg_residual_norm(const afsi_mg_plan* plan, double* norm_out, afsi_stream_t stream);

/* Same norm as afsi_b200_mg_residual_norm for one level (p, rhs of `shape`),
 * for callers that cannot allocate device memory.  No counterpart in the
 * reference (it always has PyTorch allocate).  Allocates nothing: its
 * reduction scratch is a 32 KB file-scope device array, so grids whose launch
 * needs more than 4096 reduction blocks are rejected with AFSI_ERR_ARG (2D
 * grids above about 2^20 cells; 3D grids whose y-z section exceeds about 2^20
 * cells).  The
 * first call on a device looks the array's address up (cudaGetSymbolAddress)
 * and caches it per device ordinal, which assumes the device's primary context
 * and no device reset afterwards.  Every call shares the array: calls that
 * overlap on the GPU race. */
int32_t afsi_b200_mg_residual_norm_noalloc(const void* p, const void* rhs, const int64_t* shape,
    const double* h2, int32_t dim, int32_t bc, double* norm_out, int32_t dtype, afsi_stream_t stream);

/* Batched V-cycles (the batching form; no counterpart in the reference, which
 * steps one ChannelMultigrid per instance, mac2d/multigrid.py:16-134): `count`
 * (1..2048) independent channel plans with the Jacobi smoother and the same
 * smooth count, dtype and coarse dtype advance together, each level operation
 * of all instances in one launch and the single-CTA coarse levels in one
 * launch with a CTA per instance.  Every plan's iterates are bitwise those of
 * afsi_b200_mg_vcycles on that plan alone.
 * afsi_b200_mg_batch_table_bytes: size of the batch table (-1: invalid plans).
 * afsi_b200_mg_batch_table: fills the table in HOST memory from the plans and,
 *   optionally (else NULL), one right-hand-side source per plan (a device array
 *   of the plan's finest shape and dtype); the caller copies it to a 16-byte
 *   aligned device buffer once.  The table holds the plans' buffer addresses.
 * afsi_b200_mg_batch_vcycles: `cycles` V-cycles of every plan; with start != 0
 *   first zeroes each plan's finest iterate and copies its source, if the
 *   table has sources, into its finest rhs.  `table` is the device copy, made
 *   from the same plans. */
int64_t afsi_b200_mg_batch_table_bytes(const afsi_mg_plan* const* plans, int32_t count);
int32_t afsi_b200_mg_batch_table(const afsi_mg_plan* const* plans, int32_t count,
    const void* const* rhs_sources, void* host_table, int64_t bytes);
int32_t afsi_b200_mg_batch_vcycles(const afsi_mg_plan* const* plans, int32_t count, const void* table,
    int32_t cycles, int32_t start, afsi_stream_t stream);
/* The same V-cycles in one cooperative launch (one 1024-thread CTA per SM,
 * grid barriers between the level operations, coarse jobs taken by the CTAs
 * in turn), bitwise equal to afsi_b200_mg_batch_vcycles.  sync_scratch:
 * afsi_b200_mg_sync_bytes() zero-initialised device bytes, one per concurrent
 * run; a barrier that waits longer than about a second sets the int32 error
 * word at byte offset 8 and the kernel returns; every call first clears the
 * counter, generation and error words (bytes 0-11). */
int32_t afsi_b200_mg_batch_persistent(const afsi_mg_plan* const* plans, int32_t count, const void* table,
    int32_t cycles, int32_t start, void* sync_scratch, afsi_stream_t stream);

/* Batched FP64 iterative refinement around the batched FP32 V-cycles (the
 * batching form at the FP64 solve tolerance; no counterpart in the reference,
 * which solves each channel instance alone in FP64 with ChannelMultigrid.solve,
 * mac2d/multigrid.py:85-111).  An instance is an FP64 iterate p and right-hand
 * side b on an nx x ny channel grid, and the finest right-hand side r32 and
 * iterate e32 of its FP32 channel plan.  One refinement: FP32 V-cycles from
 * zero on r32 give e32; p += double(e32); r = b - A p with the reference's
 * FP64 operator (mac2d/grid.py:61-71); r32 = float(r); ||r|| per instance.
 * Refinements repeat until every instance meets max(atol, rtol ||b||) (the
 * FP64 solver's tolerance, mac2d/multigrid.py:94-99) or max_refinements (1..64)
 * ran.  `buffer` is a device copy of the image afsi_b200_batch_refine_setup
 * fills in host memory (16-byte aligned, afsi_b200_batch_refine_bytes long);
 * after a run it holds, as doubles at afsi_b200_batch_refine_state_offset():
 * norm[count], tol[count], rhs_norm[count], done_at[count] (refinements after
 * which the instance first met its tolerance, -1 if never), then loop words
 * {refinements run, instances unconverged, nonfinite flag, largest ||r||/||b||}.
 * afsi_b200_batch_refine_start: p = 0, r32 = float(b), the norms and tolerances.
 * afsi_b200_batch_refine_step: the correction and residual of one refinement
 *   (the caller runs the V-cycles in between).
 * afsi_b200_batch_refine_graph_create: the whole solve as one CUDA graph (the
 *   start, then a WHILE node whose body is `cycles` batched V-cycles of `plans`
 *   over `vcycle_table` (a table made without right-hand-side sources), the
 *   correction and the residual); launched with .._graph_launch. */
typedef struct afsi_refine_instance {
    int64_t nx, ny;      /* cells */
    double h2[2];        /* hx^2, hy^2 */
    double* p;           /* FP64 iterate (written) */
    const double* b;     /* FP64 right-hand side */
    float* r32;          /* FP32 plan's finest right-hand side (written) */
    const float* e32;    /* FP32 plan's finest iterate (the correction) */
} afsi_refine_instance;

int64_t afsi_b200_batch_refine_bytes(const afsi_refine_instance* instances, int32_t count);
int64_t afsi_b200_batch_refine_state_offset(const afsi_refine_instance* instances, int32_t count);
int32_t afsi_b200_batch_refine_setup(const afsi_refine_instance* instances, int32_t count, void* host_buffer,
    int64_t bytes);
int32_t afsi_b200_batch_refine_start(const afsi_refine_instance* instances, int32_t count, void* buffer,
    double rtol, double atol, int32_t max_refinements, afsi_stream_t stream);
int32_t afsi_b200_batch_refine_step(const afsi_refine_instance* instances, int32_t count, void* buffer,
    double rtol, double atol, int32_t max_refinements, afsi_stream_t stream);
int32_t afsi_b200_batch_refine_graph_create(const afsi_refine_instance* instances, int32_t count, void* buffer,
    const afsi_mg_plan* const* plans, const void* vcycle_table, int32_t cycles, double rtol, double atol,
    int32_t max_refinements, void** graph_out);
int32_t afsi_b200_batch_refine_graph_launch(void* graph, afsi_stream_t stream);
int32_t afsi_b200_batch_refine_graph_destroy(void* graph);

/* Iterative refinement of an FP64 pressure solve by FP32 V-cycles (the
 * precision form; no counterpart in the reference, whose solver is FP64
 * throughout, mac/multigrid.py:125-172).
 * afsi_b200_mg_refine_residual: r32 = float(rhs - A p) with the residual
 * formed in FP64 by the reference's operator (mac/grid.py:86-93), and
 * norm_out (device double) = ||rhs - A p||_2 of the FP64 residual
 * (deterministic).  scratch: afsi_b200_mg_refine_scratch_bytes() device bytes,
 * 16-byte aligned, zero-initialised once (-1 for an invalid shape).
 * afsi_b200_mg_refine_correct: p += double(e) over n cells. */
int64_t afsi_b200_mg_refine_scratch_bytes(const int64_t* shape, int32_t dim, int32_t bc);
int32_t afsi_b200_mg_refine_residual(const double* p, const double* rhs, float* r32, const int64_t* shape,
    const double* h2, int32_t dim, int32_t bc, double* norm_out, void* scratch, afsi_stream_t stream);
int32_t afsi_b200_mg_refine_correct(double* p, const float* e, int64_t n, afsi_stream_t stream);

/* stats_out (device double[4]) = {sum(x), sum(|x|), sum(x^2), all finite ? 1 : 0}
 * over n values (deterministic order). */
int32_t afsi_b200_vector_stats(const void* x, int64_t n, double* stats_out, void* scratch,
    int32_t dtype, afsi_stream_t stream);
/* x -= mean, mean = stats[0]/n computed on the device. */
int32_t afsi_b200_subtract_mean(void* x, int64_t n, const double* stats, int32_t dtype,
    afsi_stream_t stream);

/* ---- cached CSR pattern maintenance ----------------------------------------
 * finish_cached_component / numeric_snapshot (mac/cached_transfer_assembly.py:
 * 97-175) on the device.  A pattern is its table slots in key order, its
 * transpose order and the row pointers of B (rows = nodes) and B^T (nf faces).
 * afsi_b200_cache_new_keys: with old_slots == NULL (a first build) the
 *   occupied table keys sorted with their slots into new_keys / new_slots
 *   (capacity long; the first *count are the keys); otherwise the sorted
 *   unique keys of missing_keys[0..missing) that the pattern's nnz_old keys
 *   lack, into new_keys (*count of them).  limit = nodes * nf bounds the keys.
 * afsi_b200_cache_merge: the pattern after adding the k sorted new keys
 *   (new_slots given, or looked up in the table by linear probing, at most
 *   128 slots; a failed lookup sets AFSI_FLAG_OVERFLOW): slots, transpose
 *   order, crow (nodes+1), columns, tcrow (nf+1), transpose columns, values
 *   and transpose values (nnz_old + k each); out-of-range keys set
 *   AFSI_FLAG_INDEX, nonfinite values AFSI_FLAG_SUPPORT.  Old pattern arrays
 *   may be NULL when nnz_old == 0.
 * afsi_b200_cache_values: values and transpose values of an unchanged pattern.
 * scratch: afsi_b200_cache_scratch_bytes(capacity, nnz_old, missing, nodes, nf). */
int64_t afsi_b200_cache_scratch_bytes(int64_t capacity, int64_t nnz_old, int64_t missing, int64_t rows, int64_t nf);
int32_t afsi_b200_cache_new_keys(const int64_t* table_keys, int64_t capacity, const int64_t* old_slots,
    int64_t nnz_old, const int64_t* missing_keys, int64_t missing, int64_t limit, int64_t* new_keys,
    int64_t* new_slots, int64_t* count, void* scratch, int64_t scratch_bytes, afsi_stream_t stream);
int32_t afsi_b200_cache_merge(const int64_t* table_keys, const void* table_values, int64_t capacity,
    const int64_t* old_slots, const int64_t* old_order, const int64_t* old_crow, const int64_t* old_tcrow,
    int64_t nnz_old, const int64_t* new_keys, const int64_t* new_slots, int64_t k, int64_t rows, int64_t nf,
    int64_t* slots, int64_t* order, int64_t* crow, int64_t* columns, int64_t* tcrow, int64_t* tcolumns,
    void* values, void* reverse, int32_t* status, void* scratch, int64_t scratch_bytes, int32_t dtype,
    afsi_stream_t stream);
int32_t afsi_b200_cache_values(const void* table_values, const int64_t* slots, const int64_t* order, int64_t n,
    void* values, void* reverse, int32_t* status, int32_t dtype, afsi_stream_t stream);

/* ---- CN Helmholtz sweeps and Stokes residual reductions --------------------
 * The kernels of the Stokes FGMRES preconditioner and its checks on the 3D MAC
 * grid of `shape` cells (nx, ny, nz).  Face arrays come as three pointers
 * (u (nx+1,ny,nz), v (nx,ny+1,nz), w (nx,ny,nz+1)), all in `dtype`.
 * afsi_b200_helmholtz_initialize (HelmholtzKernels.initialize,
 *   mac/_triton_helmholtz.py:6-31,64-70): rhs = b - param[1] G p on interior
 *   component-normal faces (p may be NULL: no pressure term), 0 on the walls;
 *   u = rhs / diag.  spacing: host double[3].
 * afsi_b200_helmholtz_sweep (HelmholtzKernels.sweep, :34-61,72-77): out = u +
 *   (rhs - u + param[0] L u)/diag with odd wall ghosts, 0 on the walls.
 *   spacing_squared: host double[3].
 * Stokes partials, one row per 256 cells (afsi_b200_stokes_partial_blocks):
 * afsi_b200_stokes_start_partial (start_partial, mac/_triton_stokes.py:16-27):
 *   out (blocks,3) = [sum b.b over the cells' low faces, sum p, all p finite];
 * afsi_b200_stokes_residual_partial (residual_partial, :58-84): residual
 *   (nx,ny,nz) = -coef[2] D u; out (blocks,2) = [sum |momentum residual|^2,
 *   sum (D u)^2]; coefficients (device, 9) = [alpha, dt/rho, rho/dt, 1/h (3),
 *   1/h^2 (3)] (mac/stokes_workspace.py:66-77);
 * afsi_b200_pressure_input_partial (:106-114): out (blocks,5) = [sum rhs,
 *   sum |rhs|, sum p, all rhs finite, all p finite] over n cells;
 * afsi_b200_pressure_norm_partial (:117-132): out (blocks,2) = [sum rhs^2,
 *   sum (rhs - A p)^2], A the Neumann operator; spacing_squared (device, 3). */
int64_t afsi_b200_stokes_partial_blocks(const int64_t* shape);
int32_t afsi_b200_helmholtz_initialize(const void* const* b, const void* p, const void* const* diag,
    void* const* rhs, void* const* u, const void* param, const int64_t* shape, const double* spacing,
    int32_t dtype, afsi_stream_t stream);
int32_t afsi_b200_helmholtz_sweep(const void* const* u, const void* const* rhs, const void* const* diag,
    void* const* out, const void* param, const int64_t* shape, const double* spacing_squared, int32_t dtype,
    afsi_stream_t stream);
int32_t afsi_b200_stokes_start_partial(const void* const* b, const void* p, void* out, const int64_t* shape,
    int32_t dtype, afsi_stream_t stream);
int32_t afsi_b200_stokes_residual_partial(const void* const* u, const void* p, const void* const* b,
    void* residual, void* out, const void* coefficients, const int64_t* shape, int32_t dtype,
    afsi_stream_t stream);
int32_t afsi_b200_pressure_input_partial(const void* rhs, const void* p, int64_t n, void* out, int32_t dtype,
    afsi_stream_t stream);
int32_t afsi_b200_pressure_norm_partial(const void* rhs, const void* p, void* out, const void* spacing_squared,
    const int64_t* shape, int32_t dtype, afsi_stream_t stream);

/* ---- table-free element transfers (P2 and matrix-free P1) --------------------
 * The P2 spread / gather-assemble (mac/csrc/p2_transfer.cu:98-188) and the
 * matrix-free P1 element transfer (mac/adaptive_cell.py:22-83,
 * mac/_triton_adaptive.py:25-128) without stencil tables: each point's
 * position x_q = sum_a N_pos[q,a] x[cell_a], its support check and its bases
 * and IB_4 weights on both lattices are formed inside the transfer kernel
 * with the arithmetic of afsi_b200_p2_prepare / afsi_b200_p1_prepare (bases
 * bit-exact with their tables), so no (2,P,3) / (2,P,3,4) arrays exist.
 * nodes_per_cell: 10 (P2) or 4 (P1).  x (nodes,3) and N_pos (nq,npc) in
 * pos_dtype; N (nq,npc), W (elements,nq), value (nodes,3), the face arrays and
 * rhs in dtype (FP64/FP64, FP64 positions with FP32 transfers, or FP32/FP32).
 * limits = shape - 2 per axis.  Spread accumulates into u0/u1/u2 (pre-zeroed
 * by the caller); gather adds into rhs (nodes,3), or writes per element
 * (elements,npc,3) in the _local form.  A point whose support leaves the grid
 * sets AFSI_FLAG_SUPPORT in *status and is skipped; an element with a node id
 * outside [0, nodes) sets AFSI_FLAG_INDEX and is skipped. */
int32_t afsi_b200_fe_fused_spread(int32_t nodes_per_cell, const void* x, int64_t nodes, const int64_t* cells,
    int64_t elements, const void* N_pos, const void* N, int64_t nq, const void* W, const void* value,
    const double* origin, const double* spacing, const double* limits, void* u0, void* u1, void* u2, int64_t nx,
    int64_t ny, int64_t nz, double volume, int32_t* status, int32_t pos_dtype, int32_t dtype, afsi_stream_t stream);
/* Deterministic table-free spread (no counterpart in the reference, whose
 * spreads add atomically): afsi_b200_fe_fused_spread's arithmetic up to the
 * element boxes (each accumulated in a fixed order), but a box is written to
 * its own scratch slot instead of being added to the face arrays with L2
 * reductions.  The boxes are then keyed by the 4x4x4 face tiles they overlap
 * and stably sorted by tile, and one CTA per tile adds, face by face, the
 * covering boxes' entries to u0/u1/u2 in an order fixed by the tile's sorted
 * box list (four partial sums over that list, added in turn).  No atomics: the
 * result is bitwise the same on every run and equals
 * afsi_b200_fe_fused_spread's to rounding.  scratch:
 * afsi_b200_fe_det_spread_bytes(elements, nx, ny, nz, dtype) device bytes
 * (one 512-entry slot per element and component, the tile keys and the sort
 * temporary), -1 when out of range (elements * 81 must stay below 2^31).  An
 * element whose box exceeds its slot (an extent above 8 faces on an axis, or
 * a padded shared-memory box above 640 entries) sets AFSI_FLAG_OVERFLOW and
 * contributes nothing; the other status bits as for
 * afsi_b200_fe_fused_spread.  Boxes of up to 288 padded entries take a first
 * pass at the atomic spread's occupancy, larger ones a second launch. */
int64_t afsi_b200_fe_det_spread_bytes(int64_t elements, int64_t nx, int64_t ny, int64_t nz, int32_t dtype);
int32_t afsi_b200_fe_det_spread(int32_t nodes_per_cell, const void* x, int64_t nodes, const int64_t* cells,
    int64_t elements, const void* N_pos, const void* N, int64_t nq, const void* W, const void* value,
    const double* origin, const double* spacing, const double* limits, void* u0, void* u1, void* u2, int64_t nx,
    int64_t ny, int64_t nz, double volume, void* scratch, int64_t scratch_bytes, int32_t* status,
    int32_t pos_dtype, int32_t dtype, afsi_stream_t stream);
int32_t afsi_b200_fe_fused_gather(int32_t nodes_per_cell, const void* x, int64_t nodes, const int64_t* cells,
    int64_t elements, const void* N_pos, const void* N, int64_t nq, const void* W, const void* u0, const void* u1,
    const void* u2, const double* origin, const double* spacing, const double* limits, void* rhs, int64_t nx,
    int64_t ny, int64_t nz, int32_t* status, int32_t pos_dtype, int32_t dtype, afsi_stream_t stream);
int32_t afsi_b200_fe_fused_gather_local(int32_t nodes_per_cell, const void* x, int64_t nodes, const int64_t* cells,
    int64_t elements, const void* N_pos, const void* N, int64_t nq, const void* W, const void* u0, const void* u1,
    const void* u2, const double* origin, const double* spacing, const double* limits, void* local, int64_t nx,
    int64_t ny, int64_t nz, int32_t* status, int32_t pos_dtype, int32_t dtype, afsi_stream_t stream);

/* ---- MG-preconditioned FGMRES for the CN saddle point -----------------------
 * mac/stokes_fgmres.py:15-96: H u + (dt/rho) G p = b, D u = 0.  Krylov vectors
 * are packed [u0 | u1 | u2 | q] (the three face arrays, then the cells; the
 * reference's pack, stokes_fgmres.py:31-35); afsi_b200_stokes_packed_size gives
 * the length (-1 for an invalid shape).
 * afsi_b200_stokes_action: out = [(u - alpha L u) + h G q on interior faces, 0 on
 *   each component's two wall faces; (-h) D u], the reference's action
 *   (stokes_fgmres.py:36-43) with its operation order.  v and out distinct.
 * afsi_b200_stokes_precondition_rhs: rhs = (-s)/h - D t for the Helmholtz
 *   solution t (three face arrays) and the q-part s; *sum_out = sum(rhs)
 *   (deterministic) for the caller's mean removal (stokes_fgmres.py:50-53).
 * afsi_b200_stokes_precondition_result: out = [t - G phi; (phi + alpha rhs)/h],
 *   *sum_out = sum of the q-part (stokes_fgmres.py:58-63).
 * scratch: afsi_b200_stokes_precondition_scratch_bytes(shape) device bytes,
 *   zero-initialised once, one stream at a time. */
int64_t afsi_b200_stokes_packed_size(const int64_t* shape);
int64_t afsi_b200_stokes_precondition_scratch_bytes(const int64_t* shape);
int32_t afsi_b200_stokes_action(const void* v, void* out, const int64_t* shape, const double* spacing,
    double alpha, double h, int32_t dtype, afsi_stream_t stream);
int32_t afsi_b200_stokes_precondition_rhs(const void* const* tentative, const void* s, void* rhs,
    double* sum_out, void* scratch, const int64_t* shape, const double* spacing, double h, int32_t dtype,
    afsi_stream_t stream);
int32_t afsi_b200_stokes_precondition_result(const void* const* tentative, const void* phi, const void* rhs,
    void* out, double* sum_out, void* scratch, const int64_t* shape, const double* spacing, double alpha,
    double h, int32_t dtype, afsi_stream_t stream);

/* ---- batched 2D transfers (the batching form) ------------------------------
 * Many independent 2D channel instances (TriangleTransfer, mac2d/transfer.py:
 * 61-127, one per instance in the reference) in one launch per operation.
 * Points of all instances are stored back to back, and the u (nx+1, ny) and
 * v (nx, ny+1) face arrays of all instances back to back; `instances` is a
 * DEVICE array of `count` (1..1024) entries ordered by point_offset.  Ids are
 * written batch-global (face offset of the instance included).  Positions,
 * bases and weights are formed in FP64 (points are FP64) and the weights
 * stored in weight_dtype; the spread divides by the instance's hx*hy and
 * accumulates into pre-zeroed u / v; the gather writes (total, 2). */
typedef struct afsi_batch2d_instance {
    int64_t nx, ny;              /* cells */
    double hx, hy, lx, ly;       /* spacing and lengths */
    int64_t point_offset;        /* first point of the instance in the batch */
    int64_t point_count;
    int64_t u_offset, v_offset;  /* first u / v face of the instance in the batch arrays */
} afsi_batch2d_instance;

int32_t afsi_b200_batch2d_prepare(const double* points, int64_t total, const afsi_batch2d_instance* instances,
    int32_t count, int64_t* ids, void* weights, int32_t* status, int32_t weight_dtype, afsi_stream_t stream);
int32_t afsi_b200_batch2d_spread(const void* force, const int64_t* ids, const void* weights, int64_t total,
    const afsi_batch2d_instance* instances, int32_t count, void* u, void* v, int64_t nu, int64_t nv,
    int32_t* status, int32_t dtype, afsi_stream_t stream);
int32_t afsi_b200_batch2d_gather(const void* u, const void* v, int64_t nu, int64_t nv, const int64_t* ids,
    const void* weights, int64_t total, void* out, int32_t* status, int32_t dtype, afsi_stream_t stream);

/* ---- consistent-mass Jacobi-PCG ------------------------------------------
 * Replaces MassSolver.solve / GraphMassSolver.solve (mac/mass_solver.py:39-103,
 * mac/mass_graph.py:129-225): M x = rhs for a (rows, cols) block, M a CSR
 * matrix, z = r/diag, one recurrence for all columns, the reference's
 * breakdown guard, restart, check schedule and true-residual acceptance.  The
 * checks run on the device; the caller reads `state` (device double
 * [AFSI_PCG_STATE_SLOTS]) once when the solve has stopped. */
#define AFSI_PCG_STATE_SLOTS 16
#define AFSI_PCG_RESIDUAL 4    /* ||r|| of the recurrence after the latest iteration */
#define AFSI_PCG_TOLERANCE 5   /* max(atol, rtol ||rhs||) */
#define AFSI_PCG_BROKEN 7      /* 1 once the breakdown guard fired */
#define AFSI_PCG_TRUE_NORM 9   /* ||rhs - M x|| of the latest true residual */
#define AFSI_PCG_ITERATIONS 10
#define AFSI_PCG_STATUS 11
#define AFSI_PCG_RHS_NORM 12

#define AFSI_PCG_RUNNING 0
#define AFSI_PCG_CONVERGED 1      /* true residual <= tolerance */
#define AFSI_PCG_BAD_INPUT 2      /* rhs or initial not finite */
#define AFSI_PCG_BREAKDOWN 3      /* guard fired, seen at a check */
#define AFSI_PCG_NONFINITE 4      /* nonfinite true residual */
#define AFSI_PCG_NOT_CONVERGED 5  /* max_iterations reached */

typedef struct afsi_pcg_plan {
    const int64_t* crow;  /* [rows+1] */
    const int64_t* col;   /* [nnz] int64 column indices, or NULL when col32 is given */
    const int32_t* col32; /* [nnz] int32 column indices (rows < 2^31), or NULL */
    const void* val;      /* [nnz] */
    const void* diagonal; /* Jacobi diagonal: [rows] when diagonal_per_row, else [rows*cols] */
    const void* rhs;      /* [rows*cols] */
    const void* initial;  /* [rows*cols] initial guess (zeros for none) */
    void* x;              /* [rows*cols] solution */
    void* r;              /* [rows*cols] workspace */
    void* d;
    void* Ad;
    double* state;        /* [AFSI_PCG_STATE_SLOTS] */
    void* scratch;        /* afsi_b200_pcg_scratch_bytes(), zero-initialised once */
    int64_t rows;
    int32_t cols;         /* 1, 2 or 3 */
    int32_t dtype;        /* AFSI_F32 or AFSI_F64, every array but crow/col/state */
    int32_t max_iterations;
    int32_t check_every;
    int32_t recompute_every;
    int32_t diagonal_per_row; /* 1: one diagonal value per row, shared by its columns */
    double rtol;
    double atol;
} afsi_pcg_plan;

int64_t afsi_b200_pcg_scratch_bytes(void);
/* x = initial, ||rhs||, tolerance, finiteness, then r = rhs - M x and the
 * first direction; stops (CONVERGED) when the initial guess already meets the
 * tolerance. */
int32_t afsi_b200_pcg_begin(const afsi_pcg_plan* plan, afsi_stream_t stream);
/* `count` iterations (each: Ad = M d and the step, then the check or the
 * direction update); no-ops once the status left RUNNING. */
int32_t afsi_b200_pcg_iterations(const afsi_pcg_plan* plan, int32_t count, afsi_stream_t stream);
/* The iteration loop as one CUDA graph (a WHILE node over one iteration);
 * launch it after afsi_b200_pcg_begin on the same stream. */
int32_t afsi_b200_pcg_graph_create(const afsi_pcg_plan* plan, void** graph_out);
int32_t afsi_b200_pcg_graph_launch(void* graph, afsi_stream_t stream);
int32_t afsi_b200_pcg_graph_destroy(void* graph);

#ifdef __cplusplus
}
#endif
#endif
