// Staged P2 element transfers (p2.cu), launched by the C-ABI in transfer.cu.
#pragma once
#include "common.cuh"

namespace afsi {

struct P2Dims {
    int64_t nx, ny, nz, total, offset, nq, nodes, elements;
};

template <class T>
int32_t launch_spread_staged(const T* value, const int64_t* cells, const T* N, const T* W, const int64_t* base,
                             const T* phi, T* u0, T* u1, T* u2, const P2Dims& g, T volume, int32_t* status,
                             int blocks, cudaStream_t stream);

template <class T, bool Local>
int32_t launch_gather_staged(const T* u0, const T* u1, const T* u2, const int64_t* cells, const T* N, const T* W,
                             const int64_t* base, const T* phi, T* out, const P2Dims& g, int32_t* status,
                             int blocks, cudaStream_t stream);

// Blocks of the staged kernels for `elements` elements (4 warps per block).
inline int staged_blocks(int64_t elements) { return int((elements + 3) / 4); }

}  // namespace afsi
