// Adjoint line kernels for the solve layout S = 9 rows per lane, WPL = 1 warp(s) per line.
#include "adj_kernels.cuh"

namespace astr {
template cudaError_t launch_adj_lines_t<9, 1>(const AdjLineArgs& a, cudaStream_t st);
template cudaError_t launch_adj_grad_t<9, 1>(const PassArgs& a, cudaStream_t st);
}  // namespace astr
