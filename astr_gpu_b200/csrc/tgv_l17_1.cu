// Pass kernels for the solve layout S = 17 rows per lane, WPL = 1 warp(s) per line.
#include "tgv_kernels.cuh"

namespace astr {
template cudaError_t launch_pass_t<17, 1>(int pass, const PassArgs& a, cudaStream_t st);
template cudaError_t launch_pass_batch_t<17, 1>(int pass, int dir, const PassArgs* dargs, const int* dcum,
                                                     int nbox, int nctas, int threads, size_t smem, cudaStream_t st);
}  // namespace astr
