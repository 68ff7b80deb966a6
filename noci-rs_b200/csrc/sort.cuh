// Per-pair classification of the sorted evaluation pipeline (csrc/eval.cu), shared with the
// fused QMC spawn-and-classify kernel (csrc/qmc.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.cuh"
#include "wick_math.cuh"

namespace nw {

__device__ __forceinline__ DetRec load_det(const nw_det* dets, uint32_t i) {
  const ulonglong2* p = reinterpret_cast<const ulonglong2*>(dets + i);
  const ulonglong2 lo = __ldg(p);
  const ulonglong2 hi = __ldg(p + 1);
  return unpack_det(lo.x, lo.y, hi.x, hi.y);
}

__device__ __forceinline__ void store_hs(double* out, uint64_t i, double h, double s) {
  reinterpret_cast<double2*>(out)[i] = make_double2(h, s);
}

// Sort key of every pair (pair_sort_key) and its rank among the pairs with the same key, taken
// from the per-key counter with one global atomic per pair.  The class comes from the 16-bit
// determinant descriptors; the full records are read only for same-parent pairs, which need
// the excitation-distance rule.
__device__ __forceinline__ uint32_t classify_one(const EvalParams& P, uint2 ab, uint64_t i, double* __restrict__ out,
                                                 int out_stride, uint32_t* __restrict__ flag) {
  if (ab.x >= P.ndet || ab.y >= P.ndet) {
    atomicOr(flag, 1u);
    const double nan = __longlong_as_double(0x7FF8000000000000ll);
    if (out_stride == 2)
      store_hs(out, i, nan, nan);
    else
      out[i] = nan;
    return kSkipKey;
  }
  const uint32_t dx = __ldg(P.desc + ab.x), dw = __ldg(P.desc + ab.y);
  const int px = (int)(dx & 0xFF), pw = (int)(dw & 0xFF);
  if (px == pw && far_same_parent(load_det(P.dets, ab.x), load_det(P.dets, ab.y))) {
    if (out_stride == 2)
      store_hs(out, i, 0.0, 0.0);
    else
      out[i] = 0.0;
    return kSkipKey;
  }
  const int la = (int)((dx >> 8) & 15) + (int)((dw >> 8) & 15), lb = (int)(dx >> 12) + (int)(dw >> 12);
  const int ord = __ldg(P.order + px * P.nref + pw);
  if (ord < 0) return kSkipKey;  // reference pair outside the resident block: left unwritten
  return pair_sort_key(la, lb, ab.x, pw, ord, P.nfast, P.ndet, P.nbucket, P.shift);
}


}  // namespace nw
