// Mixed-precision DFIRE scoring (FP32 distances, exact bins, compensated FP32 sums).
//
// Same contract as the FP64 kernels in sd_score.cu (energy of cdfire_calculate_dfire,
// prepare_gso_tasks.cc:1522-1615, with every bin identical to the FP64 reference bin), but the
// summation order is free, which this kernel uses three ways:
//  * the ligand is kept in spatial chunks of 32 atoms (k-d order, ligand frame), so a receptor
//    tile first rejects whole ligand chunks by bounding spheres, then single atoms by ballot;
//  * stage 1 (one lane per receptor atom, one ligand atom broadcast per iteration) only tests
//    d^2 and appends the in-cutoff pairs {d^2, table row+column, pair id} to a per-warp ring
//    in shared memory (warp-aggregated compaction);
//  * stage 2 drains the ring 64 pairs at a time, two independent pairs per lane: key from a
//    fast reciprocal square root, the exact-bin guard against the proven FP32 error bound B,
//    two table gathers in flight, Kahan accumulation.  Pairs within B of a bin edge or of the
//    cutoff are recomputed from the exact FP64 pose transform (counted as fallbacks).
// Included by sd_score.cu (shares its constant-memory key thresholds and bin table).
#pragma once

namespace sd {
namespace {

constexpr int kWarps = 4;
constexpr int kRing = 128;  // entries per warp ring (power of two)

struct Ring {
  float d2[kWarps][kRing];
  int base[kWarps][kRing];
  int pid[kWarps][kRing];
};

__device__ __forceinline__ int exact_key_m(double d2, const double* T) {
  float f = sqrtf((float)d2) * 2.0f - 1.0f;
  int k = (int)f;
  k = k < 0 ? 0 : (k > 29 ? 29 : k);
  if (k < 29 && d2 >= T[k + 1]) ++k;
  else if (k > 0 && d2 < T[k]) --k;
  return k;
}

struct PoseCtx {
  const DevComplex* C;
  int nslots;
  const double* pose;
  const double* q;
  const double* qi;
  const double* T;
  const float* Tf;
  const int* lut;
  const float* table;
  float B;
};

// value of one in-cutoff candidate pair; returns false when the exact FP64 distance shows the
// pair is outside the cutoff
__device__ __forceinline__ bool pair_value(const PoseCtx& P, float d2, int base, int pid, float& val,
                                           unsigned long long& nfb, unsigned long long& nz, unsigned long long& ncut) {
  // key estimate; d2 == 0 gives NaN -> 0 and is caught by the edge guard below
  const float r = d2 * rsqrtf(d2);
  int key = (int)fmaf(r, 2.0f, -1.0f);
  key = key < 0 ? 0 : (key > 29 ? 29 : key);
  const bool near = (d2 - P.Tf[key] <= P.B) || (P.Tf[key + 1] - d2 <= P.B);
  if (near) {
    ++nfb;
    const int slot = pid >> 13, lslot = pid & 8191;
    const int j = P.C->l_perm[lslot];
    double rx, ry, rz, lx, ly, lz;
    receptor_exact(*P.C, P.nslots, slot, P.pose, rx, ry, rz);
    ligand_exact(*P.C, j, P.pose, P.q, P.qi, lx, ly, lz);
    const double dx = rx - lx, dy = ry - ly, dz = rz - lz;
    const double e2 = dx * dx + dy * dy + dz * dz;
    if (!(e2 <= SD_CUTOFF2)) return false;
    if (e2 == 0.0) {
      key = 0;
      ++nz;
    } else {
      key = exact_key_m(e2, P.T);
      if (key == 29) ++ncut;
    }
  }
  val = P.table[base + P.lut[key]];
  return true;
}

}  // namespace

__global__ void __launch_bounds__(kWarps * 32, 5) dfire_score_mixed_kernel(ScoreLaunch L) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ Ring ring;
  __shared__ double sh_pose[7 + 2 * SD_MAX_MODES];
  __shared__ double sh_q[4], sh_qi[4];
  __shared__ double sh_T[32];
  __shared__ float sh_Tf[32];
  __shared__ int sh_lut[32];
  __shared__ double sh_red[32];
  __shared__ int sh_item;
  __shared__ int sh_ntile, sh_next;
  __shared__ float sh_bound[4];
  __shared__ float sh_rot[9];
  __shared__ unsigned long long sh_fallback, sh_z, sh_cut, sh_pairs, sh_evals;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid < 32) {
    sh_T[tid] = c_T[tid];
    sh_Tf[tid] = c_Tf[tid];
    sh_lut[tid] = c_binlut[tid];
  }
  if (tid == 0) sh_fallback = sh_z = sh_cut = sh_pairs = sh_evals = 0;
  StepCtl* ctl = L.ctl;
  const int parity = ctl->parity;
  const int count = ctl->count[parity];
  const int* work = L.work[parity];
  unsigned long long n_done = 0, nfb = 0, nz = 0, ncut = 0, npairs = 0, nevals = 0;
  const unsigned lt_mask = (1u << lane) - 1u;

  for (;;) {
    __syncthreads();
    if (tid == 0) sh_item = atomicAdd(&ctl->grab[parity], 1);
    __syncthreads();
    const int item = sh_item;
    if (item >= count) break;
    const int w = work[item];
    const int ci = wi_complex(w), p = wi_local(w);
    const DevComplex& C = L.cplx[ci];
    const int nslots = nslots_of(C), pl = C.pl, nlc = C.nlchunks;
    const double* pose_g = C.pos + (size_t)p * pl;
    if (tid < pl) sh_pose[tid] = pose_g[tid];
    __syncthreads();
    if (tid == 0) {
      for (int k = 0; k < 4; ++k) sh_q[k] = sh_pose[3 + k];
      quat_inverse(sh_q, sh_qi);
      float dR = 0.f, dL = 0.f;
      for (int m = 0; m < C.nmr; ++m) dR += fabsf((float)sh_pose[7 + m]) * C.mnorm_r[m];
      for (int m = 0; m < C.nml; ++m) dL += fabsf((float)sh_pose[7 + C.nmr + m]) * C.mnorm_l[m];
      dR = dR * 1.0001f + 1e-4f;
      dL = dL * 1.0001f + 1e-4f;
      sh_bound[0] = dR;
      sh_bound[1] = dL;
      const float RL = C.lig_radius + dL;
      const float u32 = 5.9604645e-8f;
      sh_bound[2] = 2.0f * (2.02f * u32 * (26.2f * (2.0f * RL + 15.1f) + 228.0f) + 3.0f * u32 * 228.0f) + 1e-6f;
      // rotation matrix of the unit quaternion (chunk centres only; culling margin covers it)
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
    float4* ligS = reinterpret_cast<float4*>(smem);               // [nlc*32] centred, col bits
    float4* chS = ligS + (size_t)nlc * SD_TILE;                   // [nlc] centre + radius
    int* tlist = reinterpret_cast<int*>(chS + nlc);               // [ntiles] tiles within reach
    if (tid == 0) {
      sh_ntile = 0;
      sh_next = 0;
    }
    for (int s = tid; s < nlc * SD_TILE; s += blockDim.x) {
      const int j = C.l_perm[s];
      if (j >= 0) {
        double x, y, z;
        ligand_exact(C, j, sh_pose, sh_q, sh_qi, x, y, z);
        ligS[s] = make_float4((float)(x - tx), (float)(y - ty), (float)(z - tz), __int_as_float(C.l_col[j]));
      } else {
        ligS[s] = make_float4(1e18f, 1e18f, 1e18f, __int_as_float(0));
      }
    }
    for (int c = tid; c < nlc; c += blockDim.x) {
      const float4 cc = C.l_chunk[c];
      const float X = sh_rot[0] * cc.x + sh_rot[1] * cc.y + sh_rot[2] * cc.z;
      const float Y = sh_rot[3] * cc.x + sh_rot[4] * cc.y + sh_rot[5] * cc.z;
      const float Z = sh_rot[6] * cc.x + sh_rot[7] * cc.y + sh_rot[8] * cc.z;
      chS[c] = make_float4(X, Y, Z, cc.w + dL);
    }
    __syncthreads();
    const float lig_reach = C.lig_radius + dL;
    // tiles whose sphere can reach the ligand sphere (order is free: sums are order-free here)
    for (int k = tid; k < C.ntiles; k += blockDim.x) {
      const float4 tile = C.r_tile[k];
      const float cx = (float)((double)tile.x - tx), cy = (float)((double)tile.y - ty),
                  cz = (float)((double)tile.z - tz);
      const float reach = 15.0f + dR + SD_CULL_MARGIN + tile.w + lig_reach;
      if (cx * cx + cy * cy + cz * cz <= reach * reach) tlist[atomicAdd(&sh_ntile, 1)] = k;
    }
    __syncthreads();
    const int ntile = sh_ntile;
    PoseCtx P{&C, nslots, sh_pose, sh_q, sh_qi, sh_T, sh_Tf, sh_lut, L.table32, sh_bound[2]};
    float ks = 0.f, kc = 0.f;
    int head = 0, tail = 0;  // warp-uniform ring cursors
    float* rd2 = ring.d2[warp];
    int* rbase = ring.base[warp];
    int* rpid = ring.pid[warp];

    auto kahan = [&](float v) {
      const float y = v - kc;
      const float t = ks + y;
      kc = (t - ks) - y;
      ks = t;
    };
    // stage 2: consume n (<= 64) ring entries, two per lane
    auto drain = [&](int n) {
      const int i0 = tail + lane, i1 = tail + 32 + lane;
      const bool v0 = lane < n, v1 = lane + 32 < n;
      float a0 = 0.f, a1 = 0.f;
      bool k0 = false, k1 = false;
      if (v0) k0 = pair_value(P, rd2[i0 & (kRing - 1)], rbase[i0 & (kRing - 1)], rpid[i0 & (kRing - 1)], a0, nfb, nz, ncut);
      if (v1) k1 = pair_value(P, rd2[i1 & (kRing - 1)], rbase[i1 & (kRing - 1)], rpid[i1 & (kRing - 1)], a1, nfb, nz, ncut);
      if (k0) {
        kahan(a0);
        ++npairs;
      }
      if (k1) {
        kahan(a1);
        ++npairs;
      }
      tail += n;
      __syncwarp();
    };

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
      const int orig = C.r_orig[slot];
      const bool active = orig >= 0;
      float fx = 1e18f, fy = 1e18f, fz = 1e18f;
      int row = 0;
      if (active) {
        double rx, ry, rz;
        receptor_exact(C, nslots, slot, sh_pose, rx, ry, rz);
        fx = (float)(rx - tx);
        fy = (float)(ry - ty);
        fz = (float)(rz - tz);
        row = C.r_row[slot];
      }
      const float cut2 = 225.0f + P.B;
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
          const int sbase = cc * SD_TILE;
          const float4 la = ligS[sbase + lane];
          const float ax = la.x - cx, ay = la.y - cy, az = la.z - cz;
          unsigned am = __ballot_sync(0xffffffffu, ax * ax + ay * ay + az * az <= reach2);
          while (am) {
            const int b = __ffs(am) - 1;
            am &= am - 1;
            const int ls = sbase + b;
            const float4 l = ligS[ls];
            const float ex = fx - l.x, ey = fy - l.y, ez = fz - l.z;
            const float d2 = fmaf(ez, ez, fmaf(ey, ey, ex * ex));
            const bool in = d2 <= cut2;  // inactive lanes sit at 1e18
            nevals += active;
            const unsigned bm = __ballot_sync(0xffffffffu, in);
            if (in) {
              const int pos = (head + __popc(bm & lt_mask)) & (kRing - 1);
              rd2[pos] = d2;
              rbase[pos] = row + __float_as_int(l.w);
              rpid[pos] = (slot << 13) | ls;
            }
            head += __popc(bm);
            __syncwarp();
            if (head - tail >= 64) drain(64);
          }
        }
      }
    }
    while (head - tail > 0) drain(min(64, head - tail));
    // FP64 block reduction of the compensated per-thread sums
    double v = (double)ks - (double)kc;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh_red[warp] = v;
    __syncthreads();
    if (tid == 0) {
      double E = 0.0;
      for (int i = 0; i < kWarps; ++i) E += sh_red[i];
      const double score = ((E)*0.0157 - 4.7) * -1;
      C.scoring[p] = score;
      if (L.energy_out) L.energy_out[p] = E;
      ++n_done;
    }
  }
  if (nfb) atomicAdd(&sh_fallback, nfb);
  if (nz) atomicAdd(&sh_z, nz);
  if (ncut) atomicAdd(&sh_cut, ncut);
  if (npairs) atomicAdd(&sh_pairs, npairs);
  if (nevals) atomicAdd(&sh_evals, nevals);
  __syncthreads();
  if (tid == 0) {
    if (n_done) atomicAdd(&ctl->stats[ST_SCORED], n_done);
    if (sh_fallback) atomicAdd(&ctl->stats[ST_FALLBACK], sh_fallback);
    if (sh_z) atomicAdd(&ctl->stats[ST_D2ZERO], sh_z);
    if (sh_cut) atomicAdd(&ctl->stats[ST_D2CUT], sh_cut);
    if (sh_pairs) atomicAdd(&ctl->stats[ST_PAIRS], sh_pairs);
    if (sh_evals) atomicAdd(&ctl->stats[ST_EVALS], sh_evals);
  }
}

}  // namespace sd
