// pyDock-style electrostatics + Lennard-Jones energy and its adjoint (project-defined; the
// reference has no such scoring function).  Specification, also restated by the oracle
// (oracle/sd_oracle.c, or_pydock_*):
//   x = |r_i - l_j|^2
//   elec_ij = 332.0636/4 * q_i q_j / (x + 1)           distance-dependent dielectric 4r, soft core
//   lj_ij   = 4 eps_ij (s^6 - s^3),  s = sig_ij^2 / (x + 0.5 sig_ij^2)
//             eps_ij = sqrt(eps_a eps_b), sig_ij = (sig_a + sig_b)/2 (20-type table)
//   S(x; on, off) = CHARMM switch (off - x)^2 (off + 2x - 3 on) / (off - on)^3 on on < x < off
//   E = sum_{x < 225} elec S(x;196,225) + 0.1 sum_{x < 64} lj S(x;49,64);   score = -E
// Gradient with respect to the pose: translation (3), left tangent rotation w with
// q <- exp(w/2) q (3), receptor and ligand ANM extents:
//   dE/dt = sum_j F_j, dE/dw = sum_j (l_j - t) x F_j, dE/de_lig_m = sum_j mask_j (R M_mj).F_j,
//   dE/de_rec_m = sum_i mask_i M_mi.G_i, with F_j = dE/dl_j, G_i = dE/dr_i (pair forces).
//
// Kernel: one CTA (8 warps) per pose at a time, persistent over a work list; receptor tiles of
// 32 (one lane per atom) culled against the ligand sphere and against spatial ligand chunks;
// per candidate ligand atom every lane evaluates its pair.  GRAD adds per-lane receptor force
// accumulators (projected onto the receptor modes at the end of each tile) and per-ligand-atom
// force accumulators in shared memory (one warp reduction + one shared atomic per component
// and ligand atom), projected onto t, w and the ligand modes at the end of the pose.
#include <cuda_runtime.h>

#include "sd_internal.h"
#include "sd_pose.cuh"

namespace sd {

namespace {

constexpr int kPdWarps = 8;
constexpr double kKe = 332.0636 / 4.0;

// a ligand atom in shared memory (position relative to t, charge): one 16-byte load in FP32
template <class T>
struct alignas(16) LigAtom {
  T x, y, z, q;
};
// the LJ pair parameters of two types, read together
template <class T>
struct alignas(2 * sizeof(T)) LjPair {
  T eps, sig2;
};

// the switch with its constant 1 / (off2 - on2)^3 passed in (both widths are fixed)
template <class T>
__device__ __forceinline__ void pd_switch(T x, T on2, T off2, T rden, T& s, T& ds) {
  if (x <= on2) {
    s = T(1);
    ds = T(0);
    return;
  }
  if (x >= off2) {
    s = T(0);
    ds = T(0);
    return;
  }
  const T a = off2 - x;
  s = a * a * (off2 + T(2) * x - T(3) * on2) * rden;
  ds = T(6) * a * (on2 - x) * rden;
}

// pair energy and dE/dx for x < 225; two divisions per pair (1 / (x + 1) and, inside 8 A,
// 1 / (x + sig2 / 2)), every other quotient a product with them
template <class T>
__device__ __forceinline__ T pd_pair(T x, T qq, T eps, T sig2, T& dedx) {
  T s, ds;
  const T inv = T(1) / (x + T(1));
  const T el = qq * inv;
  pd_switch<T>(x, T(196), T(225), T(1) / T(24389), s, ds);  // (225 - 196)^3
  T e = el * s;
  T de = -el * inv * s + el * ds;
  if (x < T(64)) {
    const T rden = T(1) / (x + T(0.5) * sig2);
    const T sv = sig2 * rden;
    const T s2 = sv * sv, s3 = s2 * sv, s6 = s3 * s3;
    const T lj = T(4) * eps * (s6 - s3);
    const T dsv = -sv * rden;
    const T dlj = T(4) * eps * (T(6) * s3 * s2 - T(3) * s2) * dsv;  // d(s^6 - s^3)/ds = 6 s^5 - 3 s^2
    pd_switch<T>(x, T(49), T(64), T(1) / T(3375), s, ds);  // (64 - 49)^3
    e += T(0.1) * (lj * s);
    de += T(0.1) * (dlj * s + lj * ds);
  }
  dedx = de;
  return e;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace

// out_grad: nullable [n][6 + nmr + nml] (GRAD), energies go to C.scoring as score (-E) and to
// L.energy_out (E) when set.  kSpill: the per-pose arrays live in this CTA's slice of the global
// scratch L.spill instead of shared memory (ligands too large for it).
template <class T, bool GRAD, bool kSpill>
__global__ void __launch_bounds__(kPdWarps * 32) pydock_kernel(ScoreLaunch L, double* out_grad) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  unsigned char* const smem = kSpill ? L.spill + (size_t)blockIdx.x * L.spill_stride : smem_dyn;
  __shared__ double sh_pose[7 + 2 * SD_MAX_MODES];
  __shared__ double sh_q[4], sh_qi[4];
  __shared__ LjPair<T> sh_lj[SD_LJ_TYPES * SD_LJ_TYPES];
  __shared__ double sh_red[kPdWarps][32];
  __shared__ float sh_rot[9];
  __shared__ float sh_bound[2];
  __shared__ int sh_item, sh_ntile, sh_next;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int k = tid; k < SD_LJ_TYPES * SD_LJ_TYPES; k += blockDim.x) {
    const int a = k / SD_LJ_TYPES, b = k % SD_LJ_TYPES;
    sh_lj[k].eps = (T)sqrt(L.lj_eps[a] * L.lj_eps[b]);
    const double sg = 0.5 * (L.lj_sigma[a] + L.lj_sigma[b]);
    sh_lj[k].sig2 = (T)(sg * sg);
  }
  StepCtl* ctl = L.ctl;
  const int parity = ctl->parity;
  const int count = ctl->count[parity];
  const int* work = L.work[parity];
  unsigned long long n_done = 0;

  for (;;) {
    __syncthreads();
    if (tid == 0) sh_item = atomicAdd(&ctl->grab[parity], 1);
    __syncthreads();
    const int item = sh_item;
    if (item >= count) break;
    const int w = work[item];
    const int ci = wi_complex(w), p = wi_local(w);
    const DevComplex& C = L.cplx[ci];
    const int nslots = nslots_of(C), pl = C.pl, nlc = C.nlchunks, nls = nlc * SD_TILE;
    const double* pose_g = C.pos + (size_t)p * pl;
    if (tid < pl) sh_pose[tid] = pose_g[tid];
    __syncthreads();
    if (tid == 0) {
      for (int k = 0; k < 4; ++k) sh_q[k] = sh_pose[3 + k];
      quat_inverse(sh_q, sh_qi);
      float dR = 0.f, dL = 0.f;
      for (int m = 0; m < C.nmr; ++m) dR += fabsf((float)sh_pose[7 + m]) * C.mnorm_r[m];
      for (int m = 0; m < C.nml; ++m) dL += fabsf((float)sh_pose[7 + C.nmr + m]) * C.mnorm_l[m];
      sh_bound[0] = dR * 1.0001f + 1e-4f;
      sh_bound[1] = dL * 1.0001f + 1e-4f;
      const double n = sqrt(sh_q[0] * sh_q[0] + sh_q[1] * sh_q[1] + sh_q[2] * sh_q[2] + sh_q[3] * sh_q[3]);
      const float w0 = (float)(sh_q[0] / n), x = (float)(sh_q[1] / n), y = (float)(sh_q[2] / n),
                  z = (float)(sh_q[3] / n);
      sh_rot[0] = 1 - 2 * (y * y + z * z);
      sh_rot[1] = 2 * (x * y - w0 * z);
      sh_rot[2] = 2 * (x * z + w0 * y);
      sh_rot[3] = 2 * (x * y + w0 * z);
      sh_rot[4] = 1 - 2 * (x * x + z * z);
      sh_rot[5] = 2 * (y * z - w0 * x);
      sh_rot[6] = 2 * (x * z - w0 * y);
      sh_rot[7] = 2 * (y * z + w0 * x);
      sh_rot[8] = 1 - 2 * (x * x + y * y);
      sh_ntile = 0;
      sh_next = 0;
      double rx = C.lig_ref[0], ry = C.lig_ref[1], rz = C.lig_ref[2];
      quat_rotate(sh_q, sh_qi, rx, ry, rz);
      double* ref = C.ref + (size_t)p * 3;
      ref[0] = rx + sh_pose[0];
      ref[1] = ry + sh_pose[1];
      ref[2] = rz + sh_pose[2];
    }
    __syncthreads();
    const double tx = sh_pose[0], ty = sh_pose[1], tz = sh_pose[2];
    const float dR = sh_bound[0], dL = sh_bound[1];
    // shared layout: ligand atoms [nls] (LigAtom<T>), llj [nls] (int), chunk spheres [nlc] (float4),
    // tile list [ntiles] (int), GRAD: fx, fy, fz [nls] (T)
    LigAtom<T>* la = reinterpret_cast<LigAtom<T>*>(smem);
    T* fx = reinterpret_cast<T*>(la + nls);  // GRAD only
    T* fy = fx + (GRAD ? nls : 0);
    T* fz = fy + (GRAD ? nls : 0);
    float4* chS = reinterpret_cast<float4*>(fz + (GRAD ? nls : 0));
    int* llj = reinterpret_cast<int*>(chS + nlc);
    int* lorig = llj + nls;
    int* tlist = lorig + nls;
    for (int s = tid; s < nls; s += blockDim.x) {
      const int j = C.l_perm[s];
      lorig[s] = j;
      if (j >= 0) {
        double x, y, z;
        ligand_exact(C, j, sh_pose, sh_q, sh_qi, x, y, z);
        la[s] = LigAtom<T>{(T)(x - tx), (T)(y - ty), (T)(z - tz), (T)(kKe * (double)C.l_q[j])};
        llj[s] = C.l_lj[j] * SD_LJ_TYPES;
      } else {
        la[s] = LigAtom<T>{(T)1e18, (T)1e18, (T)1e18, T(0)};
        llj[s] = 0;
      }
      if (GRAD) fx[s] = fy[s] = fz[s] = T(0);
    }
    for (int c = tid; c < nlc; c += blockDim.x) {
      const float4 cc = C.l_chunk[c];
      const float X = sh_rot[0] * cc.x + sh_rot[1] * cc.y + sh_rot[2] * cc.z;
      const float Y = sh_rot[3] * cc.x + sh_rot[4] * cc.y + sh_rot[5] * cc.z;
      const float Z = sh_rot[6] * cc.x + sh_rot[7] * cc.y + sh_rot[8] * cc.z;
      chS[c] = make_float4(X, Y, Z, cc.w + dL);
    }
    const float lig_reach = C.lig_radius + dL;
    for (int k = tid; k < C.ntiles; k += blockDim.x) {
      const float4 tile = C.r_tile[k];
      const float cx = (float)((double)tile.x - tx), cy = (float)((double)tile.y - ty),
                  cz = (float)((double)tile.z - tz);
      const float reach = 15.0f + dR + SD_CULL_MARGIN + tile.w + lig_reach;
      if (cx * cx + cy * cy + cz * cz <= reach * reach) tlist[atomicAdd(&sh_ntile, 1)] = k;
    }
    __syncthreads();
    const int ntile = sh_ntile;
    double es = 0.0;  // energy: FP64 per-lane sum of the pair terms
    T grec[SD_MAX_MODES];
    for (int m = 0; m < SD_MAX_MODES; ++m) grec[m] = T(0);

    for (;;) {
      int ti = 0;
      if (lane == 0) ti = atomicAdd(&sh_next, 1);
      ti = __shfl_sync(0xffffffffu, ti, 0);
      if (ti >= ntile) break;
      const int k = tlist[ti];
      const float4 tile = C.r_tile[k];
      const float cx = (float)((double)tile.x - tx), cy = (float)((double)tile.y - ty),
                  cz = (float)((double)tile.z - tz);
      const float reach = 15.0f + dR + SD_CULL_MARGIN + tile.w;
      const float reach2 = reach * reach;
      const int slot = k * SD_TILE + lane;
      const bool active = C.r_orig[slot] >= 0;
      T rx = (T)1e18, ry = (T)1e18, rz = (T)1e18, rq = T(0);
      int rlj = 0;
      if (active) {
        double x, y, z;
        receptor_exact(C, nslots, slot, sh_pose, x, y, z);
        rx = (T)(x - tx);
        ry = (T)(y - ty);
        rz = (T)(z - tz);
        rq = (T)C.r_q[slot];
        rlj = C.r_lj[slot];
      }
      T gx = T(0), gy = T(0), gz = T(0);  // dE/dr_i
      for (int cb = 0; cb < nlc; cb += 32) {
        const int c = cb + lane;
        bool cnear = false;
        if (c < nlc) {
          const float4 ch = chS[c];
          const float ex = ch.x - cx, ey = ch.y - cy, ez = ch.z - cz, r = reach + ch.w;
          cnear = ex * ex + ey * ey + ez * ez <= r * r;
        }
        unsigned cm = __ballot_sync(0xffffffffu, cnear);
        while (cm) {
          const int cc = cb + __ffs(cm) - 1;
          cm &= cm - 1;
          const int sb = cc * SD_TILE;
          const LigAtom<T> ca = la[sb + lane];
          const float ax = (float)ca.x - cx, ay = (float)ca.y - cy, az = (float)ca.z - cz;
          unsigned am = __ballot_sync(0xffffffffu, ax * ax + ay * ay + az * az <= reach2);
          // this lane's pair with candidate slot s: energy, dE/dr_i into (gx, gy, gz), and the
          // force on the ligand atom into f
          auto pair = [&](int s, T f[3]) {
            const LigAtom<T> a = la[s];
            const T dx = rx - a.x, dy = ry - a.y, dz = rz - a.z;
            const T x = dx * dx + dy * dy + dz * dz;
            if (x < T(225)) {
              T dedx;
              // the table is symmetric (products and sums of the two types' parameters), so it is
              // read as [ligand type][receptor type]: the lanes of one candidate read consecutive
              // entries instead of entries 20 apart that meet in a few banks
              const LjPair<T> lj = sh_lj[llj[s] + rlj];
              const T e = pd_pair<T>(x, rq * a.q, lj.eps, lj.sig2, dedx);
              es += (double)e;
              if (GRAD) {
                const T g2 = T(2) * dedx;
                gx += g2 * dx;
                gy += g2 * dy;
                gz += g2 * dz;
                f[0] = -g2 * dx;
                f[1] = -g2 * dy;
                f[2] = -g2 * dz;
              }
            }
          };
          if (!GRAD) {
            while (am) {
              const int b = __ffs(am) - 1;
              am &= am - 1;
              T f[3];
              pair(sb + b, f);
            }
          } else {
            // candidates several at a time share one warp reduction of their ligand forces
            const bool h16 = (lane & 16) != 0, h8 = (lane & 8) != 0;
            if constexpr (sizeof(T) == 8) {
              // FP64 (registers to spare), four: an exchange across the half-warps and one across
              // the quarter-warps leave candidate A's partial forces in lanes 0-7, B's in 8-15,
              // C's in 16-23 and D's in 24-31; three more levels finish all four
              while (am) {
                int b[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                  b[q] = am ? __ffs(am) - 1 : -1;
                  if (am) am &= am - 1;
                }
                T f[4][3];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                  f[q][0] = f[q][1] = f[q][2] = T(0);
                  if (b[q] >= 0) pair(sb + b[q], f[q]);
                }
                T r[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                  T k0 = h16 ? f[2][k] : f[0][k], k1 = h16 ? f[3][k] : f[1][k];
                  k0 += __shfl_xor_sync(0xffffffffu, h16 ? f[0][k] : f[2][k], 16);
                  k1 += __shfl_xor_sync(0xffffffffu, h16 ? f[1][k] : f[3][k], 16);
                  T v = (h8 ? k1 : k0) + __shfl_xor_sync(0xffffffffu, h8 ? k0 : k1, 8);
                  for (int o = 4; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                  r[k] = v;
                }
                const int bq = b[(h16 ? 2 : 0) + (h8 ? 1 : 0)];
                if ((lane & 7) == 0 && bq >= 0) {
                  atomicAdd(&fx[sb + bq], r[0]);
                  atomicAdd(&fy[sb + bq], r[1]);
                  atomicAdd(&fz[sb + bq], r[2]);
                }
              }
            } else {
              // FP32, two: one exchange across the half-warps leaves candidate A's partial forces
              // in lanes 0-15 and B's in 16-31; four more levels finish both
              while (am) {
                const int b0 = __ffs(am) - 1;
                am &= am - 1;
                int b1 = -1;
                if (am) {
                  b1 = __ffs(am) - 1;
                  am &= am - 1;
                }
                T fa[3] = {T(0), T(0), T(0)}, fb[3] = {T(0), T(0), T(0)};
                pair(sb + b0, fa);
                if (b1 >= 0) pair(sb + b1, fb);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                  T v = (h16 ? fb[k] : fa[k]) + __shfl_xor_sync(0xffffffffu, h16 ? fa[k] : fb[k], 16);
                  for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                  fa[k] = v;
                }
                const int s = sb + (h16 ? b1 : b0);
                if ((lane & 15) == 0 && (!h16 || b1 >= 0)) {
                  atomicAdd(&fx[s], fa[0]);
                  atomicAdd(&fy[s], fa[1]);
                  atomicAdd(&fz[s], fa[2]);
                }
              }
            }
          }
        }
      }
      if (GRAD && active && C.r_mask[slot] == 1) {
        for (int m = 0; m < C.nmr; ++m) {
          const double* M = C.r_modes + ((size_t)m * nslots + slot) * 3;
          grec[m] += (T)M[0] * gx + (T)M[1] * gy + (T)M[2] * gz;
        }
      }
    }
    __syncthreads();
    // pose results: energy (and gradient) reduced in FP64 over the block
    double acc[1 + 6 + 2 * SD_MAX_MODES];
    const int ng = GRAD ? 6 + C.nmr + C.nml : 0;
    acc[0] = es;
    if (GRAD) {
      for (int k = 1; k <= ng; ++k) acc[k] = 0.0;
      for (int m = 0; m < C.nmr; ++m) acc[1 + 6 + m] = (double)grec[m];
      // ligand side: F_j projected on t, w, ligand modes
      double Rm[9];
      {
        // rotation of rotate() for the (possibly non-unit) quaternion, in FP64
        const double* q = sh_q;
        const double n2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
        const double w0 = q[0], x = q[1], y = q[2], z = q[3];
        Rm[0] = (w0 * w0 + x * x - y * y - z * z) / n2;
        Rm[1] = 2 * (x * y - w0 * z) / n2;
        Rm[2] = 2 * (x * z + w0 * y) / n2;
        Rm[3] = 2 * (x * y + w0 * z) / n2;
        Rm[4] = (w0 * w0 - x * x + y * y - z * z) / n2;
        Rm[5] = 2 * (y * z - w0 * x) / n2;
        Rm[6] = 2 * (x * z - w0 * y) / n2;
        Rm[7] = 2 * (y * z + w0 * x) / n2;
        Rm[8] = (w0 * w0 - x * x - y * y + z * z) / n2;
      }
      for (int s = tid; s < nls; s += blockDim.x) {
        const int j = lorig[s];
        if (j < 0) continue;
        const double Fx = (double)fx[s], Fy = (double)fy[s], Fz = (double)fz[s];
        const double px = (double)la[s].x, py = (double)la[s].y, pz = (double)la[s].z;  // l_j - t
        acc[1] += Fx;
        acc[2] += Fy;
        acc[3] += Fz;
        acc[4] += py * Fz - pz * Fy;
        acc[5] += pz * Fx - px * Fz;
        acc[6] += px * Fy - py * Fx;
        if (C.l_mask[j] == 1)
          for (int m = 0; m < C.nml; ++m) {
            const double* M = C.l_modes + ((size_t)m * C.nl + j) * 3;
            const double RMx = Rm[0] * M[0] + Rm[1] * M[1] + Rm[2] * M[2];
            const double RMy = Rm[3] * M[0] + Rm[4] * M[1] + Rm[5] * M[2];
            const double RMz = Rm[6] * M[0] + Rm[7] * M[1] + Rm[8] * M[2];
            acc[1 + 6 + C.nmr + m] += RMx * Fx + RMy * Fy + RMz * Fz;
          }
      }
    }
    for (int k = 0; k <= ng; ++k) {
      const double v = warp_sum<double>(acc[k]);
      if (lane == 0) sh_red[warp][k] = v;
    }
    __syncthreads();
    if (tid <= ng) {
      double v = 0.0;
      for (int i = 0; i < kPdWarps; ++i) v += sh_red[i][tid];
      if (tid == 0) {
        C.scoring[p] = -v;
        if (L.energy_out) L.energy_out[p] = v;
        ++n_done;
      } else if (GRAD && out_grad) {
        out_grad[(size_t)p * ng + (tid - 1)] = v;
      }
    }
  }
  if (tid == 0 && n_done) atomicAdd(&ctl->stats[ST_SCORED], n_done);
}

size_t pydock_smem_bytes(int precision, bool grad, int max_nl, int max_nr) {
  const size_t nlc = (size_t)(max_nl + SD_TILE - 1) / SD_TILE, nls = nlc * SD_TILE;
  const size_t ts = precision == SD_PREC_MIXED ? 4 : 8;
  return ts * nls * (4 + (grad ? 3 : 0)) + 16 * nlc + 4 * nls * 2 + 4 * ((max_nr + SD_TILE - 1) / SD_TILE) + 16;
}

const void* pydock_kernel_ptr(int precision, bool grad, bool spill) {
  if (precision == SD_PREC_MIXED) {
    if (spill) return grad ? (const void*)pydock_kernel<float, true, true> : (const void*)pydock_kernel<float, false, true>;
    return grad ? (const void*)pydock_kernel<float, true, false> : (const void*)pydock_kernel<float, false, false>;
  }
  if (spill) return grad ? (const void*)pydock_kernel<double, true, true> : (const void*)pydock_kernel<double, false, true>;
  return grad ? (const void*)pydock_kernel<double, true, false> : (const void*)pydock_kernel<double, false, false>;
}

int pydock_launch(const ScoreLaunch& L, int precision, bool grad, double* out_grad, int grid, size_t smem,
                  cudaStream_t st, bool spill) {
  ScoreLaunch l = L;
  void* args[] = {(void*)&l, (void*)&out_grad};
  if (cudaLaunchKernel(pydock_kernel_ptr(precision, grad, spill), dim3(grid), dim3(kPdWarps * 32), args,
                       spill ? 0 : smem, st) != cudaSuccess)
    return SD_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? SD_OK : SD_ERR_CUDA;
}

int pydock_threads() { return kPdWarps * 32; }

}  // namespace sd
