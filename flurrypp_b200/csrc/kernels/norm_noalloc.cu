// Residual norm without any device allocation.
//
// fr_residual_norm works on a case and keeps its per-element partial norms
// in a buffer the case allocated.  Some callers cannot allocate device
// memory at all: a host application that owns every device byte through its
// own pool and forbids allocation calls from libraries, or a caller in a
// time-critical loop where the implicit synchronisation of cudaMalloc/cudaFree
// is not allowed.  fr_residual_norm_noalloc serves them: the caller passes the
// residual and the Jacobian determinants it already holds on the device, and
// the two-level reduction keeps its partial sums in one file-scope static
// device array of fixed size (declared below), which every GPU that loads the
// library holds until the process exits.
//
// Usage rules:
//   - The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current and keeps it for the
//     life of the process.  A cudaDeviceReset of that device reloads the
//     module and leaves the kept address stale, so the function must not be
//     called on a device after a cudaDeviceReset of it.
//   - No call may be made while its stream is being captured into a CUDA
//     graph: every call copies the weights from host memory and synchronises
//     the stream before it returns.
//   - Every call uses the same array.  Calls that overlap on the GPU (on
//     different streams, or from different host threads) race on it; issue
//     them one after another.
//   - Each call writes every partial it later reads, so nothing has to be
//     cleared between calls.
//   - divF and detJ must be FP64 arrays.  The precision form's working
//     arrays (which fr_device_ptr returns for a case created with
//     FR_PREC_MIXED) are FP32; the library knows every FP32 array it
//     allocated and refuses them with FR_ERR_ARG.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../../include/fr_b200.h"
#include "launch.cuh"

// true when p lies inside an FP32 device array allocated by a live case of
// this library (fr_case.cu)
bool fr_internal_is_fp32(const void *p);

namespace {

constexpr int kBlocks = 1024;  // partial sums per field
constexpr int kThreads = 256;
constexpr int kMaxFields = 5;
constexpr int kMaxSpts = FR_NOALLOC_MAX_SPTS;  // hexes up to order 5
// [kBlocks][kMaxFields] partials, [kMaxFields] result, [kMaxSpts] weights
constexpr int kScratch = kBlocks * kMaxFields + kMaxFields + kMaxSpts;
static __device__ __align__(256) double g_norm_scratch[kScratch];
static_assert(kScratch * sizeof(double) == FR_NOALLOC_SCRATCH_BYTES, "header and array disagree");

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_addr[kMaxDevices] = {nullptr};

// Per-element norm (ele::getNormResidual, reference src/ele.cpp:1922-1944),
// folded into per-block partials.
__global__ void __launch_bounds__(kThreads) k_norm_partial(const double *__restrict__ divF,
                                                           const double *__restrict__ detJ, int nS,
                                                           long long E, int nF, int resType,
                                                           double *__restrict__ scratch) {
  __shared__ double sh[kThreads][kMaxFields];
  const double *w = scratch + kBlocks * kMaxFields + kMaxFields;
  double acc[kMaxFields] = {0, 0, 0, 0, 0};
  for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < E; e += (long long)gridDim.x * kThreads) {
    for (int k = 0; k < nF; k++) {
      double r = 0;
      for (int s = 0; s < nS; s++) {
        const double d = divF[((long long)s * E + e) * nF + k];
        if (resType == 1)
          r += fabs(d) * w[s];
        else if (resType == 2)
          r += d * d / detJ[(long long)s * E + e] * w[s];
        else  // NaN-keeping maximum: a blown-up residual must reach the host check
          r = frk::nan_max(fabs(d) / detJ[(long long)s * E + e], r);
      }
      acc[k] = resType == 3 ? frk::nan_max(r, acc[k]) : acc[k] + r;
    }
  }
  for (int k = 0; k < nF; k++) sh[threadIdx.x][k] = acc[k];
  __syncthreads();
  for (int half = kThreads / 2; half > 0; half >>= 1) {
    if ((int)threadIdx.x < half)
      for (int k = 0; k < nF; k++)
        sh[threadIdx.x][k] = resType == 3 ? frk::nan_max(sh[threadIdx.x + half][k], sh[threadIdx.x][k])
                                          : sh[threadIdx.x][k] + sh[threadIdx.x + half][k];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < nF; k++) scratch[blockIdx.x * kMaxFields + k] = sh[0][k];
}

__global__ void k_norm_final(int nBlocks, int nF, int resType, double *__restrict__ scratch) {
  const int k = threadIdx.x;
  if (k >= nF) return;
  double r = 0;
  for (int b = 0; b < nBlocks; b++) {
    const double v = scratch[b * kMaxFields + k];
    r = resType == 3 ? frk::nan_max(v, r) : r + v;
  }
  scratch[kBlocks * kMaxFields + k] = resType == 2 ? sqrt(r) : r;
}

// Gauss-Legendre weights of n points by Newton iteration, on the stack.
void gauss_weights(int n, double *w) {
  const long double PI = 3.141592653589793238462643383279502884L;
  for (int i = 0; i < n; i++) {
    long double z = std::cos(PI * (i + 0.75L) / (n + 0.5L)), dp = 1.0L;
    for (int it = 0; it < 100; it++) {
      long double p0 = 1.0L, p1 = z;
      for (int k = 2; k <= n; k++) {
        long double pk = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      long double p = n == 1 ? z : p1;
      dp = n * (z * p1 - p0) / (z * z - 1.0L);
      if (n == 1) dp = 1.0L;
      long double dz = p / dp;
      z -= dz;
      if (std::fabs((double)dz) < 1e-19) break;
    }
    w[i] = (double)(2.0L / ((1.0L - z * z) * dp * dp));
  }
}

}  // namespace

extern "C" int fr_residual_norm_noalloc(const double *divF, const double *detJ, int nDims, int order, int nEles,
                                        int nFields, int resType, double *out, void *stream) {
  // sizes beyond the static array (order > 5, more than 5 fields) are refused
  if (!divF || !detJ || !out || (nDims != 2 && nDims != 3) || order < 0 || order > 5 || nFields != nDims + 2 ||
      resType < 1 || resType > 3 || nEles < 1 || nEles > FR_NOALLOC_MAX_ELES)
    return FR_ERR_ARG;
  // FP32 working arrays of a precision-form case would be read as doubles
  if (fr_internal_is_fp32(divF) || fr_internal_is_fp32(detJ)) return FR_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FR_ERR_CUDA;
  double *scratch;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, g_norm_scratch) != cudaSuccess || !p) return FR_ERR_CUDA;
      g_addr[dev] = static_cast<double *>(p);
    }
    scratch = g_addr[dev];
  }
  // solution-point quadrature weights (the reference's getQptWeights,
  // src/points.cpp:405-431), spt order x fastest
  const int n = order + 1, nS = nDims == 2 ? n * n : n * n * n;
  double w1[6], w[kMaxSpts];
  gauss_weights(n, w1);
  if (n == 1) w1[0] = 2.0;
  for (int s = 0; s < nS; s++) {
    const int i = s % n, j = (s / n) % n, k = s / (n * n);
    w[s] = nDims == 2 ? w1[j] * w1[i] : w1[k] * w1[j] * w1[i];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(scratch + kBlocks * kMaxFields + kMaxFields, w, nS * sizeof(double), cudaMemcpyHostToDevice,
                      st) != cudaSuccess)
    return FR_ERR_CUDA;
  long long want = ((long long)nEles + kThreads - 1) / kThreads;
  int blocks = (int)(want < kBlocks ? want : kBlocks);
  // launch results are taken from the launch calls themselves, so an error
  // the caller left pending before this call is neither reported as this
  // call's nor cleared
  const cudaError_t pending = cudaPeekAtLastError();
  long long nE = nEles;
  int nSl = nS, nFl = nFields, rt = resType;
  void *a1[] = {(void *)&divF, (void *)&detJ, &nSl, &nE, &nFl, &rt, &scratch};
  cudaError_t le = cudaLaunchKernel((const void *)k_norm_partial, dim3(blocks), dim3(kThreads), a1, 0, st);
  if (le == cudaSuccess) {
    void *a2[] = {&blocks, &nFl, &rt, &scratch};
    le = cudaLaunchKernel((const void *)k_norm_final, dim3(1), dim3(32), a2, 0, st);
  }
  if (le != cudaSuccess) {
    if (pending == cudaSuccess) cudaGetLastError();  // clear only this call's launch error
    return FR_ERR_CUDA;
  }
  if (cudaMemcpyAsync(out, scratch + kBlocks * kMaxFields, nFields * sizeof(double), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return FR_ERR_CUDA;
  for (int k = 0; k < nFields; k++)
    if (out[k] != out[k]) return FR_ERR_NONFINITE;
  return FR_OK;
}
