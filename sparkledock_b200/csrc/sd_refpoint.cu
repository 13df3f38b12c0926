// The ligand reference point on the GPU: Khachiyan's minimum-volume enclosing ellipsoid centre with
// tolerance 0.01, in the operation order of the reference's minimum_volume_ellipsoid
// (source/dock/src/prepare_gso_tasks.cc:106-267, one thread), the same order as the host version
// sd_reference_point (sd_synth.cc), so both give the reference's bits.
//
// One CTA runs the whole iteration.  What the reference sums sequentially stays sequential (its
// summation order is the result): the 16 entries of V = sum_i q_i (q_i u_i)^T are 16 threads each
// adding the atoms in ascending order, and the weight change's squared norm is one thread's sum;
// everything element-wise (the quadratic forms m_i, the weight update) is spread over the CTA, and
// the first atom of largest m_i comes from a reduction that breaks ties by the lower index.
#include <cuda_runtime.h>

#include <climits>
#include <string>

#include "sd_internal.h"
#include "sd_mvee.h"

namespace sd {
namespace {

constexpr int kMveeThreads = 256;

__device__ __forceinline__ double mvee_q(const double* p, int i, int a) { return a == 3 ? 1.0 : p[i * 3 + a]; }

// u, nu: device buffers of n weights; out: centre (3) and the iteration count (as a double)
__global__ void __launch_bounds__(kMveeThreads) mvee_kernel(const double* p, int n, double tol, double* u, double* nu,
                                                            double* out) {
  __shared__ double V[16], X[16];
  __shared__ double sh_m[kMveeThreads / 32], sh_step, sh_err;
  __shared__ int sh_j[kMveeThreads / 32], sh_best_j;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < n; i += blockDim.x) u[i] = 1.0 / n;
  double err = 1 + tol;
  int it = 0;
  while (err > tol && it < 100000) {
    ++it;
    __syncthreads();
    if (tid < 16) {
      const int a = tid >> 2, b = tid & 3;
      double sum = 0.0;
      for (int i = 0; i < n; ++i) sum += mvee_q(p, i, a) * (mvee_q(p, i, b) * u[i]);
      V[tid] = sum;
    }
    __syncthreads();
    if (tid == 0) sd_inverse4_lu(V, X);
    __syncthreads();
    // m_i = q_i^T (Ainv q_i) in the reference's order; each thread keeps its first strict maximum
    // above 0 (ascending i), then the CTA takes the largest, the lower index on ties
    double best = 0.0;
    int bj = INT_MAX;
    for (int i = tid; i < n; i += blockDim.x) {
      double t[4];
      for (int k = 0; k < 4; ++k) {
        double sum = 0.0;
        for (int m = 0; m < 4; ++m) sum += X[k * 4 + m] * mvee_q(p, i, m);
        t[k] = sum;
      }
      double m = 0.0;
      for (int k = 0; k < 4; ++k) m += mvee_q(p, i, k) * t[k];
      if (m > best) {
        best = m;
        bj = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oj = __shfl_xor_sync(0xffffffffu, bj, o);
      if (ob > best || (ob == best && oj < bj)) {
        best = ob;
        bj = oj;
      }
    }
    if (lane == 0) {
      sh_m[warp] = best;
      sh_j[warp] = bj;
    }
    __syncthreads();
    if (tid == 0) {
      double mx = sh_m[0];
      int j = sh_j[0];
      for (int w = 1; w < kMveeThreads / 32; ++w)
        if (sh_m[w] > mx || (sh_m[w] == mx && sh_j[w] < j)) {
          mx = sh_m[w];
          j = sh_j[w];
        }
      if (j == INT_MAX) {  // no m_i above 0: the reference keeps index 0 and maximum 0
        j = 0;
        mx = 0.0;
      }
      sh_best_j = j;
      sh_step = (mx - 3 - 1.0) / ((3 + 1.0) * (mx - 1.0));
    }
    __syncthreads();
    const double step = sh_step;
    for (int i = tid; i < n; i += blockDim.x) nu[i] = (1.0 - step) * u[i];
    __syncthreads();
    if (tid == 0) {
      nu[sh_best_j] += step;
      double e2 = 0.0;
      for (int i = 0; i < n; ++i) e2 += (nu[i] - u[i]) * (nu[i] - u[i]);
      sh_err = sqrt(e2);
    }
    __syncthreads();
    err = sh_err;
    double* tmp = u;
    u = nu;
    nu = tmp;
  }
  __syncthreads();
  if (tid < 3) {
    double c = 0.0;
    for (int i = 0; i < n; ++i) c += p[i * 3 + tid] * u[i];
    out[tid] = c;
  }
  if (tid == 3) out[3] = (double)it;
}

}  // namespace
}  // namespace sd

extern "C" int sd_reference_point_device(int device, const double* xyz, int n, double* center) {
  if (!xyz || n <= 0 || !center) return sd::fail(SD_ERR_ARG, "sd_reference_point_device: bad arguments");
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return sd::fail(SD_ERR_CUDA, "sd_reference_point_device: bad device");
  }
  double* d = nullptr;
  const size_t bytes = sizeof(double) * ((size_t)n * 5 + 4);
  if (cudaMalloc(&d, bytes) != cudaSuccess) {
    cudaGetLastError();
    return sd::fail(SD_ERR_OOM, "sd_reference_point_device: cudaMalloc failed");
  }
  double* p = d;
  double* u = d + (size_t)n * 3;
  double* nu = u + n;
  double* out = nu + n;
  cudaError_t e = cudaMemcpy(p, xyz, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    sd::mvee_kernel<<<1, sd::kMveeThreads>>>(p, n, 0.01, u, nu, out);
    e = cudaGetLastError();
  }
  double res[4] = {0, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpy(res, out, sizeof res, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return sd::fail(SD_ERR_CUDA, std::string("sd_reference_point_device: ") + cudaGetErrorString(e));
  for (int k = 0; k < 3; ++k) center[k] = res[k];
  return SD_OK;
}
