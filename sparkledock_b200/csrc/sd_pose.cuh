// Exact FP64 pose transforms shared by the scoring kernels.  Compiled with -fmad=false so each
// multiply and add rounds separately, in the order of the reference:
//   receptor  r = r0; for j: if mask: r += mode_j * ext_j        prepare_gso_tasks.cc:465-482
//   ligand    l = l0; for j: if mask: l += mode_j * ext_j        :487-504
//             l = q (0,l) conj(q)/|q|^2  (rotate)                :277-338
//             l += t                                             :518-526
#pragma once
#include "sd_internal.h"

namespace sd {

// quaternion inverse exactly as rotate() forms it (prepare_gso_tasks.cc:288-298)
__device__ __forceinline__ void quat_inverse(const double* q, double* qi) {
  double w = q[0], x = q[1], y = q[2], z = q[3];
  double n2 = w * w + x * x + y * y + z * z;
  qi[0] = q[0] / n2;
  qi[1] = -q[1] / n2;
  qi[2] = -q[2] / n2;
  qi[3] = -q[3] / n2;
}

// rotate one point (prepare_gso_tasks.cc:301-329), same expression order
__device__ __forceinline__ void quat_rotate(const double* q, const double* qi, double& px, double& py, double& pz) {
  double c0 = 0, c1 = px, c2 = py, c3 = pz;
  double d0 = (q[0] * c0 - q[1] * c1 - q[2] * c2 - q[3] * c3);
  double d1 = (q[0] * c1 + q[1] * c0 + q[2] * c3 - q[3] * c2);
  double d2 = (q[0] * c2 - q[1] * c3 + q[2] * c0 + q[3] * c1);
  double d3 = (q[0] * c3 + q[1] * c2 - q[2] * c1 + q[3] * c0);
  px = (d0 * qi[1] + d1 * qi[0] + d2 * qi[3] - d3 * qi[2]);
  py = (d0 * qi[2] - d1 * qi[3] + d2 * qi[0] + d3 * qi[1]);
  pz = (d0 * qi[3] + d1 * qi[2] - d2 * qi[1] + d3 * qi[0]);
}

// receptor atom in tile slot `slot`, extents e_rec = pose + 7
__device__ __forceinline__ void receptor_exact(const DevComplex& C, int nslots, int slot, const double* pose,
                                               double& x, double& y, double& z) {
  x = C.r_xyz[slot * 3];
  y = C.r_xyz[slot * 3 + 1];
  z = C.r_xyz[slot * 3 + 2];
  const int mk = C.r_mask[slot];
  for (int m = 0; m < C.nmr; ++m) {
    const double e = pose[7 + m];
    const double* M = C.r_modes + ((size_t)m * nslots + slot) * 3;
    if (mk == 1) {
      x += M[0] * e;
      y += M[1] * e;
      z += M[2] * e;
    }
  }
}

// ligand atom j (original order)
__device__ __forceinline__ void ligand_exact(const DevComplex& C, int j, const double* pose, const double* q,
                                             const double* qi, double& x, double& y, double& z) {
  x = C.l_xyz[j * 3];
  y = C.l_xyz[j * 3 + 1];
  z = C.l_xyz[j * 3 + 2];
  const int mk = C.l_mask[j];
  for (int m = 0; m < C.nml; ++m) {
    const double e = pose[7 + C.nmr + m];
    const double* M = C.l_modes + ((size_t)m * C.nl + j) * 3;
    if (mk == 1) {
      x += M[0] * e;
      y += M[1] * e;
      z += M[2] * e;
    }
  }
  quat_rotate(q, qi, x, y, z);
  x += pose[0];
  y += pose[1];
  z += pose[2];
}

// ligand atom in chunk slot s (chunk-ordered copies, same arithmetic as ligand_exact)
__device__ __forceinline__ void ligand_exact_chunk(const DevComplex& C, int s, const double* pose, const double* q,
                                                   const double* qi, double& x, double& y, double& z) {
  const int nls = C.nlchunks * SD_TILE;
  x = C.lc_xyz[s * 3];
  y = C.lc_xyz[s * 3 + 1];
  z = C.lc_xyz[s * 3 + 2];
  const int mk = C.lc_mask[s];
  for (int m = 0; m < C.nml; ++m) {
    const double e = pose[7 + C.nmr + m];
    const double* M = C.lc_modes + ((size_t)m * nls + s) * 3;
    if (mk == 1) {
      x += M[0] * e;
      y += M[1] * e;
      z += M[2] * e;
    }
  }
  quat_rotate(q, qi, x, y, z);
  x += pose[0];
  y += pose[1];
  z += pose[2];
}

__device__ __forceinline__ int nslots_of(const DevComplex& C) { return C.ntiles * SD_TILE; }

}  // namespace sd
