// Adjoint line kernels for the solve layout S = 9 rows per lane, WPL = 4 warp(s) per line.
#include "adj_kernels.cuh"

namespace astr {
template cudaError_t launch_adj_lines_t<9, 4>(const AdjLineArgs& a, cudaStream_t st);
template cudaError_t launch_adj_grad_t<9, 4>(const PassArgs& a, cudaStream_t st);
}  // namespace astr
