// Device-side types of the discrete adjoint (see adj_kernels.cuh and adjoint.cu).
#pragma once
#include "tgv.cuh"

namespace astr {

constexpr int ADJ_BAND = 17;   // interior stencil of W = E^T B^T: rows node-8 .. node+8

// out(m) = sum_r W(m, r) y(r) of a transposed line operator, y indexed by node (= row - ext_lo).
struct AdjW {
  double wint[ADJ_BAND];   // interior nodes mlo..mhi: y(m + jlo + j), j = 0..nint-1
  int jlo, nint;
  int mlo, mhi;
  const int* sptr;          // other nodes, k = m (m < mlo) or mlo + m - mhi - 1: entries sptr[k]..sptr[k+1]-1
  const int* snode;         // node index of y
  const double* scoef;
};

struct AdjLineArgs {
  PassArgs p;               // geometry, TI/LP, dir; p.opd = the transposed system's lane tables
  AdjW w;
  const double* in;         // nf fields, field stride p.g.fs
  double* out;
  int nf;
  double alpha;
  int accumulate;
};

constexpr int ADJ_MAXF = 5;   // fields staged together by one CTA of the transposed line kernel

// Shared memory of the transposed line kernel staging nf fields at a time (nf <= ADJ_MAXF).
inline size_t adj_lines_smem(int TI, int LP, int WPL, int nf = ADJ_MAXF) {
  return ((size_t)nf * TI * LP + (size_t)TI * SCAN_PER_LINE * WPL) * sizeof(double);
}
inline size_t adj_grad_smem(int TI, int LP, int WPL) {
  return ((size_t)6 * TI * LP + (size_t)TI * SCAN_PER_LINE * WPL + (size_t)TI * 4 * 2 * NSP) * sizeof(double);
}

// ---- discrete adjoint (adjoint.cu)
struct AdjHostOp {
  HostOp tri;                    // A^T with its Thomas factors
  AdjW w;                        // W = E^T B^T (interior stencil; device list pointers unset)
  std::vector<int> sptr, snode;  // explicit columns of W near the line ends
  std::vector<double> scoef;
};
struct AdjDevOp {
  DevOp tri;
  AdjW w{};
  void* dmem = nullptr;
};
bool build_adjoint_op(const HostOp& fwd, AdjHostOp& out, std::string& err);
cudaError_t make_adj_devop(const AdjHostOp& h, Layout lay, AdjDevOp& out);
void free_adj_devop(AdjDevOp& d);
cudaError_t launch_adj_point1(const BoxGeo& g, const Thermo& th, const double* q, const double* G, const double* Y,
                              const double* lnew, double c1, double c2, double* lsave, double* lq, double* U,
                              double* lp, double* LG, cudaStream_t st);
cudaError_t launch_adj_point2(const BoxGeo& g, const Thermo& th, const double* q, const double* U, const double* lp,
                              double* lq, const double* lsum, cudaStream_t st);
cudaError_t launch_adj_objective(const BoxGeo& g, const double* q, double* lam, cudaStream_t st);
cudaError_t launch_kinetic_energy(const BoxGeo& g, const double* q, double* part, double* out, cudaStream_t st);

cudaError_t launch_adj_lines(const AdjLineArgs& a, int S, int WPL, cudaStream_t st);
cudaError_t launch_adj_grad(const PassArgs& a, int S, int WPL, cudaStream_t st);

}  // namespace astr
