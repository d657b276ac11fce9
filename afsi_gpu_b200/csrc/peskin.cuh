// Peskin IB_4 one-dimensional weights shared by the prepare kernels.
#pragma once
#include "common.cuh"

namespace afsi {

// Clamped two-branch Peskin kernel, afsi_torch/ib.py:57-67.
template <class T>
__device__ __forceinline__ T peskin_clamped(T d) {
    const T r = fabs(d);
    const T a = r < T(1) ? r : T(1);
    const T b = r < T(1) ? T(1) : (r < T(2) ? r : T(2));
    const T inner = (T(3) - T(2) * a + sqrt(T(1) + T(4) * a - T(4) * (a * a))) / T(8);
    const T outer = (T(5) - T(2) * b - sqrt(T(-7) + T(12) * b - T(4) * (b * b))) / T(8);
    return r < T(1) ? inner : (r < T(2) ? outer : T(0));
}

// Shared-radical weights for f in [0,1), mac/csrc/p2_transfer.cu:36-43.
template <class T>
__device__ __forceinline__ void peskin_radical(T f, T w[4]) {
    const T rad = sqrt(T(1) + T(4) * f - T(4) * (f * f));
    w[0] = (T(3) - T(2) * f - rad) / T(8);
    w[1] = (T(3) - T(2) * f + rad) / T(8);
    w[2] = (T(1) + T(2) * f + rad) / T(8);
    w[3] = (T(1) + T(2) * f - rad) / T(8);
}

}  // namespace afsi
