// Output support: primitive variables at the plot points.
//
// The reference's ParaView writer (src/output.cpp:137-512, through
// solver::extrapolateUPpts, src/solver.cpp:630-670) converts the solution to
// primitive variables (rho, u, v, [w], p) at the solution points and
// interpolates them to the (P+3)^d plot points of each element (corners, flux
// points along the edges and the solution points) with opp_spts_to_ppts.  The
// kernel does both in one pass: a thread per (plot point, element), element
// fastest so the reads of one warp fall on consecutive elements of the
// [point][element][field] state.  Plot points that are solution points have a
// unit row in the operator, so those values are the state's own primitives.
#include <cuda_runtime.h>

#include "stage.hpp"

namespace frk {

template <int ND>
__global__ void __launch_bounds__(256) k_plot_primitives(const double *__restrict__ U,
                                                         const double *__restrict__ opp, double *__restrict__ Vp,
                                                         int nS, int nP, int E, double gamma) {
  constexpr int NF = ND + 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nP * E) return;
  const int e = (int)(t % E), p = (int)(t / E);
  const double *row = opp + (size_t)p * nS;
  double acc[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) acc[k] = 0.0;
  for (int s = 0; s < nS; s++) {
    const double w = row[s];
    const double *u = U + ((size_t)s * E + e) * NF;
    const double rho = u[0];
    double v[ND], v2 = 0.0;
#pragma unroll
    for (int d = 0; d < ND; d++) {
      v[d] = u[1 + d] / rho;
      v2 += v[d] * v[d];
    }
    acc[0] += w * rho;
#pragma unroll
    for (int d = 0; d < ND; d++) acc[1 + d] += w * v[d];
    acc[ND + 1] += w * ((gamma - 1) * (u[ND + 1] - 0.5 * rho * v2));
  }
  double *out = Vp + ((size_t)p * E + e) * NF;
#pragma unroll
  for (int k = 0; k < NF; k++) out[k] = acc[k];
}

void launch_plot_primitives(int nDims, const double *U, const double *opp, double *Vp, int nS, int nP, int E,
                            double gamma, cudaStream_t st) {
  const long long n = (long long)nP * E;
  const int threads = 256;
  const unsigned blocks = (unsigned)((n + threads - 1) / threads);
  if (blocks == 0) return;
  if (nDims == 2)
    k_plot_primitives<2><<<blocks, threads, 0, st>>>(U, opp, Vp, nS, nP, E, gamma);
  else
    k_plot_primitives<3><<<blocks, threads, 0, st>>>(U, opp, Vp, nS, nP, E, gamma);
}

}  // namespace frk
