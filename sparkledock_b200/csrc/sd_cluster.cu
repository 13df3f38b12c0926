// Final-pose clustering of every swarm (BSAS), after the GSO steps.
//
// Semantics of the reference's GPU pipeline variant (source/dock/src/cuda/pipeline:2766-2960;
// kernels prepare_pair / BlockSortKernel, prepare_gso_task.cu:1139-1190):
//  * order the glowworms of a swarm by the key (int64)(score * 2^50) / 2^12 * 2^12 + index,
//    descending (scores equal to 2^-38 fall back to the larger index first);
//  * the first glowworm in that order starts cluster 0; then every glowworm in order, the first
//    one again included (so cluster 0 counts it twice, as in the reference), joins the first
//    cluster whose representative (its first member) lies within 4 A backbone RMSD, or starts a
//    new cluster;
//  * backbone RMSD: over the flagged receptor atoms then the flagged ligand atoms, each atom's
//    squared distance formed as ((0 + dx^2) + dy^2) + dz^2 and added in that order, divided by the
//    atom count, square root; no superposition.  Coordinates are the final poses through the
//    exact FP64 transforms (receptor ANM; ligand ANM, rotation, translation), as the reference
//    materialises them for its lightdock_<g>.pdb files.
// GPU work: one thread per (glowworm, backbone atom) materialises the coordinates; one CTA per
// swarm sorts and clusters, one thread per existing cluster computing that RMSD sequentially
// against the current glowworm staged in shared memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "sd_internal.h"
#include "sd_pose.cuh"

namespace sd {

namespace {

constexpr int kClusterThreads = 256;

// coordinates [ns][G][nbb][3] of the backbone atoms of swarms s0 .. s0+ns-1 (receptor first)
__global__ void materialise_backbone_kernel(const DevComplex* cplx, int ci, int s0, int ns, const int* rb_slot,
                                            int nbr, const int* lb_idx, int nbl, double* out) {
  const DevComplex& C = cplx[ci];
  const int nbb = nbr + nbl, G = C.G, nslots = nslots_of(C);
  const long long total = (long long)ns * G * nbb;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(i % nbb);
    const long long gg = i / nbb;  // glowworm within the chunk
    const double* pose = C.pos + ((size_t)s0 * G + (size_t)gg) * C.pl;
    double x, y, z;
    if (a < nbr) {
      receptor_exact(C, nslots, rb_slot[a], pose, x, y, z);
    } else {
      double q[4] = {pose[3], pose[4], pose[5], pose[6]}, qi[4];
      quat_inverse(q, qi);
      ligand_exact(C, lb_idx[a - nbr], pose, q, qi, x, y, z);
    }
    double* o = out + (size_t)i * 3;
    o[0] = x;
    o[1] = y;
    o[2] = z;
  }
}

__global__ void __launch_bounds__(kClusterThreads) bsas_kernel(const DevComplex* cplx, int ci, int s0,
                                                                const double* bb, int nbb, int* n_clusters,
                                                                int* rep, int* len, int* member) {
  extern __shared__ __align__(16) unsigned char smem[];
  const DevComplex& C = cplx[ci];
  const int G = C.G, s = s0 + blockIdx.x, tid = threadIdx.x;
  long long* key = reinterpret_cast<long long*>(smem);      // [G]
  int* order = reinterpret_cast<int*>(key + G);             // [G]
  int* crep = order + G;                                    // [G] representative of cluster c
  int* clen = crep + G;                                     // [G]
  double* cur = reinterpret_cast<double*>(clen + G + (G & 1));  // [nbb][3] current glowworm
  __shared__ int sh_ncl, sh_hit;
  const double* sbb = bb + (size_t)blockIdx.x * G * nbb * 3;
  for (int g = tid; g < G; g += blockDim.x) {
    double sc = C.scoring[(size_t)s * G + g] * 1125899906842624.0;  // x 2^50
    sc = fmin(fmax(sc, -9.2e18), 9.2e18);                            // keep the conversion defined
    key[g] = (long long)sc / 4096 * 4096 + g;
    clen[g] = 0;
  }
  __syncthreads();
  for (int g = tid; g < G; g += blockDim.x) {  // descending rank (keys are distinct)
    const long long k = key[g];
    int r = 0;
    for (int h = 0; h < G; ++h) r += key[h] > k ? 1 : 0;
    order[r] = g;
  }
  __syncthreads();
  if (tid == 0) {
    crep[0] = order[0];
    clen[0] = 1;
    sh_ncl = 1;
  }
  __syncthreads();
  for (int i = 0; i < G; ++i) {
    const int g = order[i];
    for (int a = tid; a < nbb * 3; a += blockDim.x) cur[a] = sbb[(size_t)g * nbb * 3 + a];
    if (tid == 0) sh_hit = 0x7fffffff;
    __syncthreads();
    const int ncl = sh_ncl;
    for (int c = tid; c < ncl; c += blockDim.x) {
      const double* r = sbb + (size_t)crep[c] * nbb * 3;
      double sum = 0.0;
      for (int a = 0; a < nbb; ++a) {
        const double dx = r[a * 3] - cur[a * 3], dy = r[a * 3 + 1] - cur[a * 3 + 1], dz = r[a * 3 + 2] - cur[a * 3 + 2];
        double t = 0.0;
        t += dx * dx;
        t += dy * dy;
        t += dz * dz;
        sum += t;
      }
      const double rmsd = sqrt(sum / nbb);
      if (rmsd <= 4.0) atomicMin(&sh_hit, c);
    }
    __syncthreads();
    if (tid == 0) {
      int c = sh_hit;
      if (c == 0x7fffffff) {
        c = sh_ncl++;
        crep[c] = g;
      }
      ++clen[c];
      member[(size_t)s * G + g] = c;
    }
    __syncthreads();
  }
  const int ncl = sh_ncl;
  for (int c = tid; c < G; c += blockDim.x) {
    rep[(size_t)s * G + c] = c < ncl ? crep[c] : -1;
    len[(size_t)s * G + c] = c < ncl ? clen[c] : 0;
  }
  if (tid == 0) n_clusters[s] = ncl;
}

// every atom of chosen glowworms (pose index swarm * G + glowworm): rec [n][nr][3] in the
// caller's atom order (rslot maps it to the tile slots), lig [n][nl][3]
__global__ void materialise_poses_kernel(const DevComplex* cplx, int ci, const int* poses, int n, const int* rslot,
                                         int nr, int nl, double* rec, double* lig) {
  const DevComplex& C = cplx[ci];
  const int na = nr + nl, nslots = nslots_of(C);
  const long long total = (long long)n * na;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / na), a = (int)(i % na);
    const double* pose = C.pos + (size_t)poses[k] * C.pl;
    double x, y, z, *o;
    if (a < nr) {
      receptor_exact(C, nslots, rslot[a], pose, x, y, z);
      o = rec + ((size_t)k * nr + a) * 3;
    } else {
      double q[4] = {pose[3], pose[4], pose[5], pose[6]}, qi[4];
      quat_inverse(q, qi);
      ligand_exact(C, a - nr, pose, q, qi, x, y, z);
      o = lig + ((size_t)k * nl + (a - nr)) * 3;
    }
    o[0] = x;
    o[1] = y;
    o[2] = z;
  }
}

}  // namespace

int materialise_launch(const DevComplex* d_cplx, int ci, const int* d_poses, int n, const int* d_rslot, int nr, int nl,
                       double* d_rec, double* d_lig, cudaStream_t st) {
  materialise_poses_kernel<<<148 * 8, 256, 0, st>>>(d_cplx, ci, d_poses, n, d_rslot, nr, nl, d_rec, d_lig);
  return cudaGetLastError() == cudaSuccess ? SD_OK : SD_ERR_CUDA;
}

size_t cluster_smem_bytes(int G, int nbb) {
  return (size_t)G * 8 + (size_t)G * 4 * 3 + ((G & 1) ? 4 : 0) + (size_t)nbb * 24;
}

int cluster_launch(const DevComplex* d_cplx, int ci, int s0, int ns, int G, const int* d_rb_slot, int nbr,
                   const int* d_lb_idx, int nbl, double* d_bb, int* d_ncl, int* d_rep, int* d_len, int* d_member,
                   cudaStream_t st) {
  const int nbb = nbr + nbl;
  materialise_backbone_kernel<<<148 * 8, 256, 0, st>>>(d_cplx, ci, s0, ns, d_rb_slot, nbr, d_lb_idx, nbl, d_bb);
  if (cudaGetLastError() != cudaSuccess) return SD_ERR_CUDA;
  const size_t sm = cluster_smem_bytes(G, nbb);
  if (cudaFuncSetAttribute(bsas_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
    return SD_ERR_CUDA;
  bsas_kernel<<<ns, kClusterThreads, sm, st>>>(d_cplx, ci, s0, d_bb, nbb, d_ncl, d_rep, d_len, d_member);
  return cudaGetLastError() == cudaSuccess ? SD_OK : SD_ERR_CUDA;
}

}  // namespace sd
