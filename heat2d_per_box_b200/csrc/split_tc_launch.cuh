// Launch switches over the compiled variants of the split-precision kernels.
// Included by split_kernels.cu (floating slices) and split_fix.cu
// (fixed-point slices), each of which instantiates one kFix.
#pragma once
#include "split_tc.cuh"

namespace bfgt {
namespace splitk {

template <bool kFix>
void launch_form(int variant, int grid, size_t smem, cudaStream_t s, const FormTcLaunch &lp) {
  if (grid <= 0) return;
  const bool b = lp.descs != nullptr;
#define FORM_V(V, P, NT, YF, N)                                                    \
  case V:                                                                          \
    if (b) k_form_tc<true, P, NT, YF, N, kFix><<<grid, kThreads, smem, s>>>(lp);  \
    else k_form_tc<false, P, NT, YF, N, kFix><<<grid, kThreads, smem, s>>>(lp);   \
    break;
  if constexpr (kFix) {
    // Y is FP64 with fixed-point slices: no float2 variants
    switch (variant) {
      FORM_V(0, false, 1, false, 8) FORM_V(1, false, 2, false, 8) FORM_V(4, true, 1, false, 8)
      FORM_V(5, false, 1, false, 16) FORM_V(6, false, 2, false, 16) FORM_V(9, true, 1, false, 16)
    }
  } else {
    switch (variant) {
      FORM_V(0, false, 1, false, 8) FORM_V(1, false, 2, false, 8) FORM_V(2, false, 1, true, 8)
      FORM_V(3, false, 2, true, 8) FORM_V(4, true, 1, false, 8)
      FORM_V(5, false, 1, false, 16) FORM_V(6, false, 2, false, 16) FORM_V(7, false, 1, true, 16)
      FORM_V(8, false, 2, true, 16) FORM_V(9, true, 1, false, 16)
    }
  }
#undef FORM_V
}

template <bool kFix>
void launch_eval(int nnt, bool pack, bool n16, int grid, size_t smem, cudaStream_t s, const EvalTcLaunch &lp) {
  if (grid <= 0) return;
  const bool b = lp.descs != nullptr;
  switch (nnt) {
#define EVAL_K(X, B, P, N) k_eval_tc<X, B, P, N, kFix><<<grid, kEvalThreads, smem, s>>>(lp)
#define EVAL_NNT(X)                                                  \
  case X:                                                            \
    if (n16) {                                                       \
      if (pack) {                                                    \
        if (b) EVAL_K(X, true, true, 16);                            \
        else EVAL_K(X, false, true, 16);                             \
      } else {                                                       \
        if (b) EVAL_K(X, true, false, 16);                           \
        else EVAL_K(X, false, false, 16);                            \
      }                                                              \
    } else {                                                         \
      if (pack) {                                                    \
        if (b) EVAL_K(X, true, true, 8);                             \
        else EVAL_K(X, false, true, 8);                              \
      } else {                                                       \
        if (b) EVAL_K(X, true, false, 8);                            \
        else EVAL_K(X, false, false, 8);                             \
      }                                                              \
    }                                                                \
    break;
    EVAL_NNT(1) EVAL_NNT(2) EVAL_NNT(3) EVAL_NNT(4) EVAL_NNT(5) EVAL_NNT(6) EVAL_NNT(7) EVAL_NNT(8)
#undef EVAL_NNT
#undef EVAL_K
  }
}

template <bool kFix>
void set_smem_attrs() {
#define SMEM_ATTR(K) cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
#define SMEM_FORM2(P, NT, YF, N) \
  SMEM_ATTR((k_form_tc<false, P, NT, YF, N, kFix>)) SMEM_ATTR((k_form_tc<true, P, NT, YF, N, kFix>))
  SMEM_FORM2(false, 1, false, 8) SMEM_FORM2(false, 2, false, 8) SMEM_FORM2(true, 1, false, 8)
  SMEM_FORM2(false, 1, false, 16) SMEM_FORM2(false, 2, false, 16) SMEM_FORM2(true, 1, false, 16)
  if constexpr (!kFix) {
    SMEM_FORM2(false, 1, true, 8) SMEM_FORM2(false, 2, true, 8)
    SMEM_FORM2(false, 1, true, 16) SMEM_FORM2(false, 2, true, 16)
  }
#undef SMEM_FORM2
#define SMEM_EVAL(X, N)                                                                              \
  SMEM_ATTR((k_eval_tc<X, false, false, N, kFix>)) SMEM_ATTR((k_eval_tc<X, true, false, N, kFix>)) \
  SMEM_ATTR((k_eval_tc<X, false, true, N, kFix>)) SMEM_ATTR((k_eval_tc<X, true, true, N, kFix>))
#define SMEM_EVAL_N(N)                                                                                 \
  SMEM_EVAL(1, N) SMEM_EVAL(2, N) SMEM_EVAL(3, N) SMEM_EVAL(4, N) SMEM_EVAL(5, N) SMEM_EVAL(6, N) \
  SMEM_EVAL(7, N) SMEM_EVAL(8, N)
  SMEM_EVAL_N(8) SMEM_EVAL_N(16)
#undef SMEM_EVAL_N
#undef SMEM_EVAL
#undef SMEM_ATTR
}

}  // namespace splitk
}  // namespace bfgt
