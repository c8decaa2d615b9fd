// The per-row arithmetic shared by the single-problem and batched kernels.
#pragma once

#include "common.cuh"

namespace hb {

// Load schedules of the row kernels (see the configurations in kernels.cuh).
enum LoadSchedule : int { kPlain = 0, kStaged = 1 };

// One Gauss-Seidel row update, ComputeSYMGS_ref.cpp:72-80: sum = r_i - sum_j a_ij x_j
// (diagonal included, slot order), sum += x_i a_ii, x_i = sum / a_ii. FIRST: x
// enters as zero; the masked-out slots (and the diagonal) multiply a zero.
// Returns the new x_i.
// B: the matrix layout (rows per block of mat_index; 0 slot-major).
template <typename T, typename TR, bool FIRST, int SCHED, int B = (sizeof(T) == 4 ? kRowBlock32 : 0)>
__device__ __forceinline__ T gs_row(const T* __restrict__ val, const int* __restrict__ col, int64_t pitch,
                                    const TR* __restrict__ rhs, T* x, int q, uint32_t mask) {
  T sum = (T)rhs[q];
  T xd = (T)0;
  if (SCHED == kStaged) {
    T a[kSlots];
    int cl[kSlots];
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      if (mask & (1u << k)) {
        a[k] = __ldcs(val + mat_index<T, B>(k, q, pitch));
        cl[k] = __ldcs(col + mat_index<T, B>(k, q, pitch));
      }
    }
    T xv[kSlots];
#pragma unroll
    for (int k = 0; k < kSlots; ++k)
      if (mask & (1u << k)) xv[k] = __ldg(x + cl[k]);
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      if (mask & (1u << k)) {
        sum -= a[k] * xv[k];
        if (k == kDiagSlot) xd = xv[k];
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < kSlots; ++k) {
      if (mask & (1u << k)) {
        const T a = val[mat_index<T, B>(k, q, pitch)];
        const T xv = __ldg(x + col[mat_index<T, B>(k, q, pitch)]);
        sum -= a * xv;
        if (k == kDiagSlot) xd = xv;
      }
    }
  }
  const T d = val[mat_index<T, B>(kDiagSlot, q, pitch)];
  if (!FIRST) sum += xd * d;
  const T out = sum / d;
  x[q] = out;
  return out;
}

}  // namespace hb
