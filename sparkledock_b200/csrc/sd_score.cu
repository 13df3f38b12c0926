// DFIRE pair scoring of glowworm poses on sm_100a.
//
// Replaces the reference's pose kernels + DFIRE tile kernel + energy reduce
// (prepare_gso_task.cu:268-494, :1820-2286, :2377-2433) and follows the CPU semantics of
// cdfire_calculate_dfire (prepare_gso_tasks.cc:1522-1615):
//   E = sum_i ( sum_j [d2_ij <= 225] table[tR_i][tL_j][dist_to_bins[(int)(2 sqrt(d2)-1)]-1] )
//   score = -(0.0157 E - 4.7)
//
// Design (one persistent kernel, one CTA per pose at a time, dynamic work grabbing):
//  * the ligand of the pose is transformed once into shared memory (exact FP64 transform);
//  * receptor atoms are pre-sorted into spatial tiles of 32 (one warp lane per atom); a warp
//    takes a tile, skips it when its bounding sphere (inflated by the pose's ANM displacement
//    bound) is beyond 15 A of the ligand's sphere, and otherwise builds ballot masks of the
//    ligand atoms that can reach the tile, 32 at a time, visiting them in ascending j;
//  * FP64 modes: each lane's partial v_i sums its pairs in ascending j exactly as the
//    reference, and the pose energy adds the v_i in ascending original i (zeros skipped:
//    adding +0.0 never changes a sum), so energies are bit-identical to the reference
//    order with or without culling;
//  * MIXED (sd_score_mixed.cuh): distances from FP32 coordinates centred on the pose
//    translation, an exact per-pair bin unless d2 lies within a proven error bound B of a bin
//    or cutoff edge, in which case the pair is recomputed in FP64 exactly (counted); FP64 sums
//    of the FP64 table values.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "sd_internal.h"
#include "sd_pose.cuh"

namespace sd {

__constant__ double c_T[32];   // exact FP64 key thresholds: key(d2) = #{m>=1 : T[m] <= d2}
__constant__ float c_Tf[32];   // same as float, with c_Tf[30] = 225 (cutoff)

void set_key_thresholds(const double* t) {
  double T[32];
  float Tf[32];
  for (int m = 0; m < 32; ++m) {
    T[m] = m < 30 ? t[m] : 1e300;
    Tf[m] = m < 30 ? (float)t[m] : (m == 30 ? 225.0f : 3.0e38f);
  }
  Tf[0] = 0.0f;
  cudaMemcpyToSymbol(c_T, T, sizeof T);
  cudaMemcpyToSymbol(c_Tf, Tf, sizeof Tf);
}

// dist_to_bins[key] - 1 (interface.h:30-35) for key 0..29; key 29 (d2 == 225) gives 20, which
// with the flat index reads the next ligand type's bin 0 exactly as the reference does.
__constant__ int c_binlut[32] = {0,  0,  0,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13,
                                 13, 14, 14, 15, 15, 16, 16, 17, 17, 18, 18, 19, 19, 20, 20, 20};

struct LigD {
  double x, y, z;
  int col;
  int pad;
};

__device__ __forceinline__ int exact_key(double d2, const double* T) {
  float f = sqrtf((float)d2) * 2.0f - 1.0f;
  int k = (int)f;
  k = k < 0 ? 0 : (k > 29 ? 29 : k);
  if (k < 29 && d2 >= T[k + 1]) ++k;
  else if (k > 0 && d2 < T[k]) --k;
  return k;
}

// PREC: SD_PREC_FP64_REF (no culling) or SD_PREC_FP64 (culled); the mixed-precision kernel is
// in sd_score_mixed.cuh.  16 warps per CTA: the per-pose shared memory (receptor accumulators,
// ligand atoms) allows two CTAs per SM, so the warps per CTA set the SM's residency.
// kSpill: the per-pose arrays live in this CTA's slice of the global scratch L.spill instead
// (complexes too large for shared memory); the arithmetic is the same.
constexpr int kFp64Threads = 512;

template <int PREC, bool kSpill>
__global__ void __launch_bounds__(kFp64Threads) dfire_score_kernel(ScoreLaunch L) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  unsigned char* const smem = kSpill ? L.spill + (size_t)blockIdx.x * L.spill_stride : smem_dyn;
  __shared__ double sh_pose[7 + 2 * SD_MAX_MODES];
  __shared__ double sh_q[4], sh_qi[4];
  __shared__ double sh_T[32];
  __shared__ float sh_Tf[32];
  __shared__ int sh_lut[32];
  __shared__ int sh_item;
  __shared__ int sh_ntile, sh_next;
  __shared__ float sh_bound[4];  // dR, dL
  __shared__ unsigned long long sh_fallback, sh_z, sh_cut, sh_pairs, sh_evals;

  constexpr bool kCull = PREC != SD_PREC_FP64_REF;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid < 32) {
    sh_T[tid] = c_T[tid];
    sh_Tf[tid] = c_Tf[tid];
    sh_lut[tid] = c_binlut[tid];
  }
  if (tid == 0) {
    sh_fallback = 0;
    sh_z = 0;
    sh_cut = 0;
    sh_pairs = 0;
    sh_evals = 0;
  }
  unsigned long long n_pairs = 0, n_evals = 0;  // per thread
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
    const int nl = C.nl, nr = C.nr, nslots = nslots_of(C), pl = C.pl;
    const double* pose_g = C.pos + (size_t)p * pl;
    if (tid < pl) sh_pose[tid] = pose_g[tid];
    __syncthreads();
    if (tid == 0) {
      sh_q[0] = sh_pose[3];
      sh_q[1] = sh_pose[4];
      sh_q[2] = sh_pose[5];
      sh_q[3] = sh_pose[6];
      quat_inverse(sh_q, sh_qi);
      float dR = 0.f, dL = 0.f;
      for (int m = 0; m < C.nmr; ++m) dR += fabsf((float)sh_pose[7 + m]) * C.mnorm_r[m];
      for (int m = 0; m < C.nml; ++m) dL += fabsf((float)sh_pose[7 + C.nmr + m]) * C.mnorm_l[m];
      dR = dR * 1.0001f + 1e-4f;
      dL = dL * 1.0001f + 1e-4f;
      sh_bound[0] = dR;
      sh_bound[1] = dL;
    }
    __syncthreads();
    // ---- ligand of this pose into shared memory ----
    const double tx = sh_pose[0], ty = sh_pose[1], tz = sh_pose[2];
    float4* ligF = reinterpret_cast<float4*>(smem);  // centred FP32 (x,y,z, col bits)
    LigD* ligD = reinterpret_cast<LigD*>(smem + (size_t)16 * ((nl + 1) & ~1));
    double* vacc = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(ligD) + (size_t)32 * nl);
    int* tlist = reinterpret_cast<int*>(vacc + nr);  // tiles within reach of the ligand
    int* tord = tlist + C.ntiles;                    // the same, closest to t first
    float* tdist = reinterpret_cast<float*>(tord + C.ntiles);
    if (tid == 0) {
      sh_ntile = 0;
      sh_next = 0;
    }
    for (int j = tid; j < nl; j += blockDim.x) {
      double x, y, z;
      ligand_exact(C, j, sh_pose, sh_q, sh_qi, x, y, z);
      const int col = C.l_col[j];
      ligF[j] = make_float4((float)(x - tx), (float)(y - ty), (float)(z - tz), __int_as_float(col));
      ligD[j] = LigD{x, y, z, col, 0};
    }
    for (int i = tid; i < nr; i += blockDim.x) vacc[i] = 0.0;
    if (tid == 0) {
      // ligand reference point (prepare_gso_tasks.cc:460, :513, :524-526)
      double x = C.lig_ref[0], y = C.lig_ref[1], z = C.lig_ref[2];
      quat_rotate(sh_q, sh_qi, x, y, z);
      double* ref = C.ref + (size_t)p * 3;
      ref[0] = x + tx;
      ref[1] = y + ty;
      ref[2] = z + tz;
    }
    __syncthreads();
    const float dR = sh_bound[0], dL = sh_bound[1];
    const float tile_reach_base = 15.0f + dR + SD_CULL_MARGIN;
    const float lig_reach = C.lig_radius + dL;
    for (int k = tid; k < C.ntiles; k += blockDim.x) {
      bool keep = true;
      if (kCull) {
        const float4 tile = C.r_tile[k];
        const float cx = (float)((double)tile.x - tx), cy = (float)((double)tile.y - ty),
                    cz = (float)((double)tile.z - tz);
        const float reach = tile_reach_base + tile.w + lig_reach;
        keep = cx * cx + cy * cy + cz * cz <= reach * reach;
        if (keep) {
          const int at = atomicAdd(&sh_ntile, 1);
          tlist[at] = k;
          // a NaN distance (non-finite pose) ranks last: the ranking below must stay a strict total
          // order, or tord would not be a permutation of the kept tiles
          const float dd = cx * cx + cy * cy + cz * cz;
          tdist[at] = dd == dd ? dd : 3.0e38f;
        }
      } else {
        tlist[atomicAdd(&sh_ntile, 1)] = k;
      }
    }
    __syncthreads();
    const int ntile = sh_ntile;
    // culled: the tiles closest to the ligand centre (t) have the most pairs; taking them first
    // lets the warps finish a pose together (the tile order does not touch the summation order)
    const bool sorted = kCull && ntile <= 512;
    if (sorted) {
      for (int t = tid; t < ntile; t += blockDim.x) {
        const float d = tdist[t];
        int rank = 0;
        for (int u = 0; u < ntile; ++u) {
          const float e = tdist[u];
          rank += (e < d || (e == d && u < t)) ? 1 : 0;
        }
        tord[rank] = tlist[t];
      }
      __syncthreads();
    }
    const int* tl = sorted ? tord : tlist;

    for (;;) {
      int ti = 0;
      if (lane == 0) ti = atomicAdd(&sh_next, 1);
      ti = __shfl_sync(0xffffffffu, ti, 0);
      if (ti >= ntile) break;
      const int k = tl[ti];
      const float4 tile = C.r_tile[k];
      const float cx = (float)((double)tile.x - tx), cy = (float)((double)tile.y - ty),
                  cz = (float)((double)tile.z - tz);
      const float reach = tile_reach_base + tile.w;
      const float reach2 = reach * reach;
      const int slot = k * SD_TILE + lane;
      const int orig = C.r_orig[slot];
      const bool active = orig >= 0;
      double rx = 0, ry = 0, rz = 0;
      int row = 0;
      if (active) {
        receptor_exact(C, nslots, slot, sh_pose, rx, ry, rz);
        row = C.r_row[slot];
      }
      double v = 0.0;  // FP64 partial of receptor atom `orig`
      for (int base = 0; base < nl; base += 32) {
        const int j = base + lane;
        bool cand = j < nl;
        if (kCull && cand) {
          const float4 lj = ligF[j];
          const float ex = lj.x - cx, ey = lj.y - cy, ez = lj.z - cz;
          cand = ex * ex + ey * ey + ez * ez <= reach2;
        }
        unsigned mask = __ballot_sync(0xffffffffu, cand);
        while (mask) {
          const int b = __ffs(mask) - 1;
          mask &= mask - 1;
          const int jj = base + b;
          n_evals += active;
          {
            const LigD l = ligD[jj];
            const double ddx = rx - l.x, ddy = ry - l.y, ddz = rz - l.z;
            const double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
            if (active && d2 <= SD_CUTOFF2) {
              int key;
              if (d2 == 0.0) {
                key = 0;
                atomicAdd(&sh_z, 1ull);
              } else {
                key = exact_key(d2, sh_T);
                if (key == 29) atomicAdd(&sh_cut, 1ull);
              }
              v += L.table64[row + l.col + sh_lut[key]];
              ++n_pairs;
            }
          }
        }
      }
      if (active) vacc[orig] = v;
    }
    __syncthreads();
    double E;
    {
      // reference order: E += v_i for i ascending (zero partials skipped)
      E = 0.0;
      if (warp == 0) {
        for (int base = 0; base < nr; base += 32) {
          const double vv = base + lane < nr ? vacc[base + lane] : 0.0;
          unsigned m = __ballot_sync(0xffffffffu, vv != 0.0);
          while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            E += __shfl_sync(0xffffffffu, vv, b);
          }
        }
      }
    }
    if (tid == 0) {
      const double score = ((E)*0.0157 - 4.7) * -1;
      C.scoring[p] = score;
      if (L.energy_out) L.energy_out[p] = E;
      ++n_done;
    }
  }
  if (n_pairs) atomicAdd(&sh_pairs, n_pairs);
  if (n_evals) atomicAdd(&sh_evals, n_evals);
  __syncthreads();
  if (tid == 0) {
    if (sh_pairs) atomicAdd(&ctl->stats[ST_PAIRS], sh_pairs);
    if (sh_evals) atomicAdd(&ctl->stats[ST_EVALS], sh_evals);
    if (n_done) atomicAdd(&ctl->stats[ST_SCORED], n_done);
    if (sh_fallback) atomicAdd(&ctl->stats[ST_FALLBACK], sh_fallback);
    if (sh_z) atomicAdd(&ctl->stats[ST_D2ZERO], sh_z);
    if (sh_cut) atomicAdd(&ctl->stats[ST_D2CUT], sh_cut);
  }
}

}  // namespace sd

#include "sd_score_mixed.cuh"

namespace sd {

// compiled variants of the mixed DFIRE kernel (kernel, warps per CTA, minimum resident CTAs per
// SM); the host autotuner times them on the context's own poses and keeps the fastest
struct MixedVariant {
  const void* fn;
  int warps;
  int min_blocks;
};
#define SD_MIXED(W, B) { (const void*)dfire_score_mixed_kernel<W, B, false>, W, B }
// variant 0 (the default before the autotuner has run) is the fastest measured on the
// 3002 / 1274-atom workload.  The variants give bit-identical energies (same per-tile work and
// summation order), so the tuner's choice never changes a result.
static const MixedVariant kMixedVariants[] = {
    SD_MIXED(8, 3), SD_MIXED(4, 5), SD_MIXED(4, 4), SD_MIXED(8, 2),
};
// the spill instantiation of the mixed kernel: variant 0's shape (the per-tile work, and so every
// energy, is the same in every variant)
static const MixedVariant kMixedSpill = {(const void*)dfire_score_mixed_kernel<8, 3, true>, 8, 3};

constexpr int kNumMixedVariants = sizeof(kMixedVariants) / sizeof(kMixedVariants[0]);
static_assert(kNumMixedVariants <= SD_MAX_VARIANTS, "variant table");

static const MixedVariant& mixed_variant(int v) { return kMixedVariants[v < 0 || v >= kNumMixedVariants ? 0 : v]; }

size_t score_smem_bytes(int precision, int scoring, int max_nr, int max_nl, int variant) {
  if (scoring == SD_SCORING_PYDOCK) return pydock_smem_bytes(precision, false, max_nl, max_nr);
  if (precision == SD_PREC_MIXED) {
    const size_t nlc = (size_t)(max_nl + SD_TILE - 1) / SD_TILE;
    const size_t ntiles = (size_t)(max_nr + SD_TILE - 1) / SD_TILE;
    (void)variant;  // every variant uses the same dynamic layout
    return (size_t)8 * ((ntiles + 1) & ~(size_t)1) + (size_t)16 * (nlc * SD_TILE + nlc) + 4 * (3 * ntiles + nlc);
  }
  return (size_t)16 * ((max_nl + 1) & ~1) + (size_t)32 * max_nl + (size_t)8 * max_nr +
         (size_t)12 * ((max_nr + SD_TILE - 1) / SD_TILE);
}

int mixed_variant_count() { return kNumMixedVariants; }
int mixed_variant_warps(int v) { return mixed_variant(v).warps; }
int mixed_variant_min_blocks(int v) { return mixed_variant(v).min_blocks; }

int score_threads_of(int precision, int scoring, int variant) {
  if (scoring == SD_SCORING_PYDOCK) return pydock_threads();
  return precision == SD_PREC_MIXED ? mixed_variant_warps(variant) * 32 : kFp64Threads;
}

int score_threads_spill(int precision, int scoring) {
  if (scoring == SD_SCORING_PYDOCK) return pydock_threads();
  return precision == SD_PREC_MIXED ? kMixedSpill.warps * 32 : kFp64Threads;
}

const void* score_kernel_ptr(int precision, int scoring, int variant, bool spill) {
  if (scoring == SD_SCORING_PYDOCK) return pydock_kernel_ptr(precision, false, spill);
  switch (precision) {
    case SD_PREC_FP64_REF:
      return spill ? (const void*)dfire_score_kernel<SD_PREC_FP64_REF, true>
                   : (const void*)dfire_score_kernel<SD_PREC_FP64_REF, false>;
    case SD_PREC_FP64:
      return spill ? (const void*)dfire_score_kernel<SD_PREC_FP64, true>
                   : (const void*)dfire_score_kernel<SD_PREC_FP64, false>;
    default: return spill ? kMixedSpill.fn : mixed_variant(variant).fn;
  }
}

int score_launch(const ScoreLaunch& L, int precision, int scoring, int grid, int threads, size_t smem,
                 cudaStream_t st, int variant, bool spill) {
  if (scoring == SD_SCORING_PYDOCK) return pydock_launch(L, precision, false, nullptr, grid, smem, st, spill);
  const void* fn = score_kernel_ptr(precision, scoring, variant, spill);
  const int nthreads = precision == SD_PREC_MIXED ? (spill ? kMixedSpill.warps : mixed_variant(variant).warps) * 32
                                                  : threads;
  ScoreLaunch l = L;
  void* args[] = {(void*)&l};
  if (cudaLaunchKernel(fn, dim3(grid), dim3(nthreads), args, spill ? 0 : smem, st) != cudaSuccess) return SD_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? SD_OK : SD_ERR_CUDA;
}

// ---- per-pair bins of one pose (parity/debug): thread per pair ----
__global__ void dfire_bins_kernel(const DevComplex* cplx, int ci, const double* pose, int precision, int* bins,
                                  int* fallback) {
  const DevComplex& C = cplx[ci];
  const int nl = C.nl, nslots = nslots_of(C);
  const long long total = (long long)nslots * nl;
  double q[4] = {pose[3], pose[4], pose[5], pose[6]}, qi[4];
  quat_inverse(q, qi);
  const double tx = pose[0], ty = pose[1], tz = pose[2];
  float dL = 0.f;
  for (int m = 0; m < C.nml; ++m) dL += fabsf((float)pose[7 + C.nmr + m]) * C.mnorm_l[m];
  dL = dL * 1.0001f + 1e-4f;
  const float RL = C.lig_radius + dL;
  const float u32 = 5.9604645e-8f;
  const float B = 2.0f * (2.02f * u32 * (26.2f * (2.0f * RL + 15.1f) + 228.0f) + 3.0f * u32 * 228.0f) + 1e-6f;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int slot = (int)(idx / nl), j = (int)(idx % nl);
    const int orig = C.r_orig[slot];
    if (orig < 0) continue;
    double rx, ry, rz, lx, ly, lz;
    receptor_exact(C, nslots, slot, pose, rx, ry, rz);
    ligand_exact(C, j, pose, q, qi, lx, ly, lz);
    int bin = -1;
    if (precision != SD_PREC_MIXED) {
      const double ddx = rx - lx, ddy = ry - ly, ddz = rz - lz;
      const double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
      if (d2 <= SD_CUTOFF2) bin = c_binlut[d2 == 0.0 ? 0 : exact_key(d2, c_T)];
    } else {
      const float ex = (float)(rx - tx) - (float)(lx - tx), ey = (float)(ry - ty) - (float)(ly - ty),
                  ez = (float)(rz - tz) - (float)(lz - tz);
      const float d2 = fmaf(ez, ez, fmaf(ey, ey, ex * ex));
      if (d2 <= 225.0f + B) {
        float f = sqrtf(d2) * 2.0f - 1.0f;
        int key = (int)f;
        key = key < 0 ? 0 : (key > 29 ? 29 : key);
        const bool near = (d2 - c_Tf[key] <= B) || (c_Tf[key + 1] - d2 <= B);
        if (near) {
          atomicAdd(fallback, 1);
          const double ddx = rx - lx, ddy = ry - ly, ddz = rz - lz;
          const double e2 = ddx * ddx + ddy * ddy + ddz * ddz;
          if (e2 <= SD_CUTOFF2) bin = c_binlut[e2 == 0.0 ? 0 : exact_key(e2, c_T)];
        } else {
          bin = c_binlut[key];
        }
      }
    }
    bins[(size_t)orig * nl + j] = bin;
  }
}

int bins_launch(const DevComplex* cplx, int c, const double* d_pose, int precision, int* d_bins, int nr, int nl,
                int* d_fallback, cudaStream_t st) {
  (void)nr;
  (void)nl;
  dfire_bins_kernel<<<148 * 8, 256, 0, st>>>(cplx, c, d_pose, precision, d_bins, d_fallback);
  return cudaGetLastError() == cudaSuccess ? SD_OK : SD_ERR_CUDA;
}

}  // namespace sd
