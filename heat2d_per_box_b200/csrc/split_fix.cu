// The fixed-point (Ozaki) slice variants of the split-precision kernels
// (split_tc.cuh), compiled in their own translation unit.
#include "split_tc_launch.cuh"

namespace bfgt {
namespace splitk {

template void launch_form<true>(int, int, size_t, cudaStream_t, const FormTcLaunch &);
template void launch_eval<true>(int, bool, bool, int, size_t, cudaStream_t, const EvalTcLaunch &);
template void set_smem_attrs<true>();

}  // namespace splitk
}  // namespace bfgt
