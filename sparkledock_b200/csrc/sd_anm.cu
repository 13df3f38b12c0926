// Normal modes of a structure (anisotropic network model), as the reference's setup computes
// them before docking: cal_anm (source/dock/src/cal_anm.cc:61-219) with build_hessian1D
// (:307-360), calModes (:403-514), norm (:516-540) and its GPU eigensolver eigh_gpu
// (source/dock/src/cuda/cal_anm.cu:28-91).
//
//  * coordinates re-centred on the mean of all atoms (norm; this also moves the structure);
//  * nodes: the CA atoms in file order (C4 when there is none);
//  * Hessian, 3N x 3N dense, cutoff 15 A, gamma 1: for every node pair within the cutoff the
//    off-diagonal block -g d d^T / |d|^2, and each diagonal block minus the sum of its row's
//    blocks, subtracted in increasing partner order as the reference's pair loop does (so the
//    matrix is bit-identical); built on the GPU, one thread per block element;
//  * eigenpairs: cusolverDnDsyevd on the lower triangle, the lowest n_modes + 6 kept, those
//    below 1e-6 dropped as zero modes;
//  * every atom of residue i takes node i's components (the reference assumes one CA per
//    residue, in order; a structure where that does not hold is refused);
//  * each mode normalised over all atoms, then scaled by sqrt(n_atoms) * rmsd / coef *
//    sqrt(1 / lambda), coef the mean over swarms x glowworms of sqrt(sum_m v_m^2 / lambda_m) with
//    v drawn from std::default_random_engine(324324) and std::normal_distribution(0, 1), as the
//    reference draws them (its OpenMP loop has no reduction clause: this is its one-thread result).
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "sd_internal.h"

namespace sd {
namespace {

// off-diagonal blocks of the node pairs within the cutoff (one thread per element of row a)
__global__ void hessian_offdiag_kernel(const double* xyz, int n, double cutoff2, double g, double* H) {
  const int dof = 3 * n;
  const long long total = (long long)dof * dof;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e / dof), c = (int)(e % dof);
    const int i = r / 3, k = r % 3, j = c / 3, l = c % 3;
    double v = 0.0;
    if (i != j) {
      const int a = i < j ? i : j, b = i < j ? j : i;  // the pair as the reference orders it
      const double d[3] = {xyz[b * 3] - xyz[a * 3], xyz[b * 3 + 1] - xyz[a * 3 + 1], xyz[b * 3 + 2] - xyz[a * 3 + 2]};
      double dist2 = 0.0;
      for (int m = 0; m < 3; ++m) dist2 += d[m] * d[m];
      if (!(dist2 > cutoff2)) v = d[k] * d[l] * (-g / dist2);
    }
    H[e] = v;
  }
}

// diagonal blocks: minus the pair blocks of each node, in increasing partner order
__global__ void hessian_diag_kernel(const double* xyz, int n, double cutoff2, double g, double* H) {
  const int dof = 3 * n;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * 9; e += gridDim.x * blockDim.x) {
    const int i = e / 9, k = (e % 9) / 3, l = e % 3;
    double v = 0.0;
    for (int p = 0; p < n; ++p) {
      if (p == i) continue;
      const int a = i < p ? i : p, b = i < p ? p : i;
      const double d[3] = {xyz[b * 3] - xyz[a * 3], xyz[b * 3 + 1] - xyz[a * 3 + 1], xyz[b * 3 + 2] - xyz[a * 3 + 2]};
      double dist2 = 0.0;
      for (int m = 0; m < 3; ++m) dist2 += d[m] * d[m];
      if (dist2 > cutoff2) continue;
      v -= d[k] * d[l] * (-g / dist2);
    }
    H[(size_t)(i * 3 + k) * dof + (i * 3 + l)] = v;
  }
}

}  // namespace
}  // namespace sd


extern "C" int sd_anm(const sd_structure* s, int n_modes, double rmsd, int n_swarms, int n_glowworms, int device,
                      double* modes_out, double* xyz_out, double* eigvals_out) {
  sd::NvtxRange nvtx_range("sd_anm");
  using namespace sd;
  if (!s || n_modes <= 0 || !(rmsd > 0) || n_swarms <= 0 || n_glowworms <= 0 || !modes_out)
    return fail(SD_ERR_ARG, "sd_anm: bad arguments");
  std::vector<double> xyz;
  std::vector<std::string> names;
  std::vector<int> rfirst;
  structure_atoms(s, xyz, names, rfirst);
  const int na = (int)names.size(), nres = (int)rfirst.size() - 1;
  // norm: re-centre on the mean of all atoms
  double m0 = 0, m1 = 0, m2 = 0;
  for (int i = 0; i < na; ++i) {
    m0 += xyz[i * 3];
    m1 += xyz[i * 3 + 1];
    m2 += xyz[i * 3 + 2];
  }
  m0 = m0 / na;
  m1 = m1 / na;
  m2 = m2 / na;
  for (int i = 0; i < na; ++i) {
    xyz[i * 3] -= m0;
    xyz[i * 3 + 1] -= m1;
    xyz[i * 3 + 2] -= m2;
  }
  // nodes
  std::vector<double> node;
  for (const char* nm : {"CA", "C4"}) {
    for (int i = 0; i < na; ++i)
      if (names[i] == nm)
        for (int k = 0; k < 3; ++k) node.push_back(xyz[i * 3 + k]);
    if (!node.empty()) break;
  }
  const int n = (int)node.size() / 3, dof = 3 * n;
  if (n == 0) return fail(SD_ERR_ARG, "sd_anm: no CA (or C4) atoms");
  if (n != nres) return fail(SD_ERR_NOTSUP, "sd_anm: the reference maps residue i to node i; needs one CA per residue");
  const int length = n_modes + 6;
  if (length > dof) return fail(SD_ERR_ARG, "sd_anm: more modes than degrees of freedom");

  if (cudaSetDevice(device) != cudaSuccess) return fail(SD_ERR_CUDA, "sd_anm: bad device");
  double *d_node = nullptr, *d_H = nullptr, *d_w = nullptr, *d_work = nullptr;
  int* d_info = nullptr;
  cusolverDnHandle_t h = nullptr;
  auto release = [&]() {
    cudaFree(d_node);
    cudaFree(d_H);
    cudaFree(d_w);
    cudaFree(d_work);
    cudaFree(d_info);
    if (h) cusolverDnDestroy(h);
  };
  auto cu = [&](cudaError_t e, const char* what) {
    if (e == cudaSuccess) return SD_OK;
    release();
    return fail(e == cudaErrorMemoryAllocation ? SD_ERR_OOM : SD_ERR_CUDA, std::string("sd_anm: ") + what + ": " +
                                                                              cudaGetErrorString(e));
  };
  int rc;
  if ((rc = cu(cudaMalloc(&d_node, sizeof(double) * node.size()), "cudaMalloc"))) return rc;
  if ((rc = cu(cudaMalloc(&d_H, sizeof(double) * (size_t)dof * dof), "cudaMalloc"))) return rc;
  if ((rc = cu(cudaMalloc(&d_w, sizeof(double) * dof), "cudaMalloc"))) return rc;
  if ((rc = cu(cudaMalloc(&d_info, sizeof(int)), "cudaMalloc"))) return rc;
  if ((rc = cu(cudaMemcpy(d_node, node.data(), sizeof(double) * node.size(), cudaMemcpyHostToDevice), "upload")))
    return rc;
  const double cutoff2 = 15.0 * 15.0, g = 1.0;
  hessian_offdiag_kernel<<<148 * 8, 256>>>(d_node, n, cutoff2, g, d_H);
  hessian_diag_kernel<<<(n * 9 + 255) / 256, 256>>>(d_node, n, cutoff2, g, d_H);
  if ((rc = cu(cudaGetLastError(), "Hessian kernels"))) return rc;
  if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) {
    release();
    return fail(SD_ERR_CUDA, "sd_anm: cusolverDnCreate");
  }
  int lwork = 0;
  if (cusolverDnDsyevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, dof, d_H, dof, d_w, &lwork) !=
      CUSOLVER_STATUS_SUCCESS) {
    release();
    return fail(SD_ERR_CUDA, "sd_anm: syevd buffer size");
  }
  lwork = static_cast<int>(lwork * 1.5);  // the workspace the reference gives it
  if ((rc = cu(cudaMalloc(&d_work, sizeof(double) * lwork), "cudaMalloc"))) return rc;
  if (cusolverDnDsyevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, dof, d_H, dof, d_w, d_work, lwork,
                       d_info) != CUSOLVER_STATUS_SUCCESS) {
    release();
    return fail(SD_ERR_CUDA, "sd_anm: syevd");
  }
  int info = 0;
  std::vector<double> w(length), vec((size_t)length * dof);
  if ((rc = cu(cudaMemcpy(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost), "download"))) return rc;
  if ((rc = cu(cudaMemcpy(w.data(), d_w, sizeof(double) * length, cudaMemcpyDeviceToHost), "download"))) return rc;
  // the lowest eigenvectors are the first columns of the column-major result
  if ((rc = cu(cudaMemcpy(vec.data(), d_H, sizeof(double) * (size_t)length * dof, cudaMemcpyDeviceToHost),
               "download")))
    return rc;
  release();
  if (info != 0) return fail(SD_ERR_NUMERIC, "sd_anm: eigensolver did not converge");

  int n_zeros = 0;
  for (int i = 0; i < length; ++i)
    if (w[i] < 1e-6) ++n_zeros;
  if (n_zeros + n_modes > length) return fail(SD_ERR_NUMERIC, "sd_anm: more zero modes than expected");
  std::vector<double> lam(w.begin() + n_zeros, w.begin() + n_zeros + n_modes);
  // extension to every atom: the atoms of residue i take node i's rows; then [atom*3+d][mode]
  std::vector<double> ev((size_t)na * 3 * n_modes);
  for (int r = 0; r < nres; ++r)
    for (int a = rfirst[r]; a < rfirst[r + 1]; ++a)
      for (int d = 0; d < 3; ++d)
        for (int m = 0; m < n_modes; ++m)
          ev[((size_t)a * 3 + d) * n_modes + m] = vec[(size_t)(m + n_zeros) * dof + r * 3 + d];
  for (int m = 0; m < n_modes; ++m) {
    double sum = 0;
    for (int i = 0; i < na * 3; ++i) sum += std::pow(ev[(size_t)i * n_modes + m], 2);
    sum = std::sqrt(sum);
    for (int i = 0; i < na * 3; ++i) ev[(size_t)i * n_modes + m] /= sum;
  }
  std::default_random_engine gen;
  std::normal_distribution<double> dist(0.0, 1.0);
  gen.seed(324324u);
  double coef = 0;
  for (long long i = 0; i < (long long)n_swarms * n_glowworms; ++i) {
    double sum = 0;
    for (int m = 0; m < n_modes; ++m) {
      const double v = dist(gen);
      const double var = 1.0 / lam[m];
      sum += v * v * var;
    }
    coef += std::sqrt(sum);
  }
  coef = coef / ((long long)n_swarms * n_glowworms);
  const double scale_item = std::sqrt((double)na) * rmsd / coef;
  for (int m = 0; m < n_modes; ++m) {
    const double sc = scale_item * std::sqrt(1.0 / lam[m]);
    for (int i = 0; i < na * 3; ++i) ev[(size_t)i * n_modes + m] *= sc;
  }
  for (int m = 0; m < n_modes; ++m)
    for (int i = 0; i < na * 3; ++i) modes_out[(size_t)m * na * 3 + i] = ev[(size_t)i * n_modes + m];
  if (xyz_out) std::copy(xyz.begin(), xyz.end(), xyz_out);
  if (eigvals_out) std::copy(lam.begin(), lam.end(), eigvals_out);
  return SD_OK;
}
