// Pass kernels for the solve layout S = 9 rows per lane, WPL = 2 warp(s) per line.
#include "tgv_kernels.cuh"

namespace astr {
template cudaError_t launch_pass_t<9, 2>(int pass, const PassArgs& a, cudaStream_t st);
}  // namespace astr
