// Mixed-precision DFIRE scoring (FP16/FP32 distances, exact bins, FP64 sums of table values).
// Included by sd_score.cu (shares its constant-memory key thresholds and bin table).
//
// Same contract as the FP64 kernels in sd_score.cu (energy of cdfire_calculate_dfire,
// prepare_gso_tasks.cc:1522-1615, with every bin identical to the FP64 reference bin), but the
// summation order is free, which this kernel uses:
//  * the ligand is kept in spatial chunks of 32 atoms (k-d order, ligand frame); a receptor
//    tile (one warp, one lane per receptor atom) rejects whole ligand chunks by bounding
//    spheres, then single atoms by ballot, and collects the surviving ligand atoms as
//    candidates;
//  * stage 1 takes candidates 32 at a time: their coordinates are staged once in a per-warp
//    buffer, every lane tests its receptor atom against all 32 (fully unrolled, broadcast
//    reads) and keeps a 32-bit in-cutoff mask; one warp scan per batch then appends the
//    in-cutoff pairs (ligand slot, lane) to a per-warp ring;
//  * stage 2 drains the ring 64 pairs at a time, two per lane: recompute d^2 (same FP32
//    expression, so the same value), key from a fast reciprocal square root, the exact-bin
//    guard against the proven FP32 error bound B, two table gathers in flight, and each lane
//    adds the FP64 table value of its pairs with one FP64 add.  The FP64 pipe is otherwise
//    idle here; compensated FP32 (Kahan) sums were measured to leave ~2e-5 absolute error at
//    60k pairs per pose, because every compensation step rounds the incoming value, and they
//    cost five FP32 adds per pair.
//    Pairs within B of a bin edge or of the cutoff are recomputed from the exact FP64 pose
//    transform (counted as fallbacks).
#pragma once

namespace sd {
namespace {

constexpr int kRing = 1024;  // per-warp ring of in-cutoff pairs (a batch adds at most 32*32)

struct __align__(16) WarpBufs {
  float4 cand_xyz[32];   // staged candidate ligand atoms (centred FP32, col bits)
  __half cand_h[16][8];  // FP16 pre-filter: per candidate pair {x0,x1,y0,y1,z0,z1,-,-}, tile-centred
  int cand_slot[64];     // pending candidate ligand slots
  float rx[32], ry[32], rz[32];  // this tile's receptor atoms (centred FP32); SoA: one bank per lane
  int rrow[32];
  int ring[kRing];       // packed (ligand slot << 5 | lane)
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
  const float4* key4;  // per key: {lower threshold, upper threshold, bin bits, 0}
  const double* table;  // FP64 DFIRE table: one 8-byte gather per pair
  float B;
};

// exact FP64 key of one pair near a bin edge or the cutoff (rare: kept out of line so that its
// registers do not weigh on the hot loop); returns -1 when the pair is outside the cutoff and
// sets *edge to 1 for d^2 == 0, 2 for d^2 == 225
__device__ __noinline__ int exact_pair_key(const DevComplex* C, int nslots, const double* pose, const double* q,
                                           const double* qi, const double* T, int slot, int j, int* edge) {
  double rx, ry, rz, lx, ly, lz;
  receptor_exact(*C, nslots, slot, pose, rx, ry, rz);
  ligand_exact(*C, j, pose, q, qi, lx, ly, lz);
  const double dx = rx - lx, dy = ry - ly, dz = rz - lz;
  const double e2 = dx * dx + dy * dy + dz * dz;
  *edge = 0;
  if (!(e2 <= SD_CUTOFF2)) return -1;
  if (e2 == 0.0) {
    *edge = 1;
    return 0;
  }
  const int key = exact_key_m(e2, T);
  if (key == 29) *edge = 2;
  return key;
}

// value of one in-cutoff candidate pair (slot = receptor slot, ls = ligand chunk slot);
// returns false when the exact FP64 distance shows the pair is outside the cutoff
__device__ __forceinline__ bool pair_value(const PoseCtx& P, float d2, int base, int slot, int ls, double& val,
                                           unsigned long long& nfb, unsigned long long& nz, unsigned long long& ncut) {
  // key estimate; d2 == 0 gives NaN -> 0 and is caught by the edge guard below
  const float r = d2 * rsqrtf(d2);
  int key = (int)fmaf(r, 2.0f, -1.0f);
  key = key < 0 ? 0 : (key > 29 ? 29 : key);
  const float4 kk = P.key4[key];
  int bin = __float_as_int(kk.z);
  const bool near = (d2 - kk.x <= P.B) || (kk.y - d2 <= P.B);
  if (near) {
    ++nfb;
    int edge;
    key = exact_pair_key(P.C, P.nslots, P.pose, P.q, P.qi, P.T, slot, P.C->l_perm[ls], &edge);
    if (key < 0) return false;
    nz += edge == 1;
    ncut += edge == 2;
    bin = __float_as_int(P.key4[key].z);
  }
  val = P.table[base + bin];
  return true;
}

}  // namespace

// kH16: stage 1 tests candidate pairs two at a time in packed FP16 on tile-centred coordinates
// against 229 A^2, a superset of the FP32 test (FP16 error on d^2 <= 1.75 A^2 for pairs within
// the cutoff: |coordinates| <= 22.5 A after centring, 2^-11 rounding per conversion and
// subtraction, half an ulp of 256 per multiply-add); stage 2 recomputes d^2 in FP32 and keeps
// only d^2 <= 225 + B, so the result is identical to the FP32 pre-filter.
template <int kWarps, int kMinBlocks, bool kH16>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) dfire_score_mixed_kernel(ScoreLaunch L) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ WarpBufs wb[kWarps];
  __shared__ double sh_pose[7 + 2 * SD_MAX_MODES];
  __shared__ double sh_q[4], sh_qi[4];
  __shared__ double sh_T[32];
  __shared__ float4 sh_key4[32];
  __shared__ double sh_red[32];
  __shared__ int sh_item;
  __shared__ int sh_ntile, sh_next;
  __shared__ float sh_bound[4];
  __shared__ float sh_rot[9];
  __shared__ unsigned long long sh_fallback, sh_z, sh_cut, sh_pairs, sh_evals;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid < 32) {
    sh_T[tid] = c_T[tid];
    const int k = tid < 30 ? tid : 29;
    sh_key4[tid] = make_float4(c_Tf[k], c_Tf[k + 1], __int_as_float(c_binlut[k]), 0.f);
  }
  if (tid == 0) sh_fallback = sh_z = sh_cut = sh_pairs = sh_evals = 0;
  StepCtl* ctl = L.ctl;
  const int parity = ctl->parity;
  const int count = ctl->count[parity];
  const int* work = L.work[parity];
  unsigned long long n_done = 0, nfb = 0, nz = 0, ncut = 0, npairs = 0, nevals = 0, nguard = 0;
  const unsigned lt_mask = (1u << lane) - 1u;
  WarpBufs& W = wb[warp];

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
      dR = dR * 1.0001f + 1e-4f;
      dL = dL * 1.0001f + 1e-4f;
      sh_bound[0] = dR;
      sh_bound[1] = dL;
      // bound of |FP32 d2 - FP64 d2| for pairs within 15.1 A (coordinates centred on t)
      const float RL = C.lig_radius + dL;
      const float u32 = 5.9604645e-8f;
      sh_bound[2] = 2.0f * (2.02f * u32 * (26.2f * (2.0f * RL + 15.1f) + 228.0f) + 3.0f * u32 * 228.0f) + 1e-6f;
      // rotation matrix of the unit quaternion (chunk centres only; the culling margin covers it)
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
      // ligand reference point (prepare_gso_tasks.cc:460, :513, :524-526)
      double rx = C.lig_ref[0], ry = C.lig_ref[1], rz = C.lig_ref[2];
      quat_rotate(sh_q, sh_qi, rx, ry, rz);
      double* ref = C.ref + (size_t)p * 3;
      ref[0] = rx + sh_pose[0];
      ref[1] = ry + sh_pose[1];
      ref[2] = rz + sh_pose[2];
      sh_ntile = 0;
      sh_next = 0;
    }
    __syncthreads();
    const double tx = sh_pose[0], ty = sh_pose[1], tz = sh_pose[2];
    const float dR = sh_bound[0], dL = sh_bound[1];
    float4* ligS = reinterpret_cast<float4*>(smem);  // [nlc*32] centred, col bits
    float4* chS = ligS + (size_t)nlc * SD_TILE;      // [nlc] centre + radius
    int* tlist = reinterpret_cast<int*>(chS + nlc);  // [ntiles] tiles within reach
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
    PoseCtx P{&C, nslots, sh_pose, sh_q, sh_qi, sh_T, sh_key4, L.table64, sh_bound[2]};
    const float cut2 = 225.0f + P.B;
    double acc = 0.0;  // per-thread FP64 sum of the table values of its pairs

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
      W.rx[lane] = fx;
      W.ry[lane] = fy;
      W.rz[lane] = fz;
      W.rrow[lane] = row;
      const int nact = __popc(__ballot_sync(0xffffffffu, active));
      int ncand = 0, head = 0, tail = 0;  // warp-uniform

      // stage 2: consume n (<= 64) ring entries, two per lane
      auto drain = [&](int n) {
        const int i0 = tail + lane, i1 = tail + 32 + lane;
        const bool v0 = lane < n, v1 = lane + 32 < n;
        double a0 = 0.0, a1 = 0.0;
        bool k0 = false, k1 = false;
        if (v0) {
          const int e = W.ring[i0 & (kRing - 1)];
          const int ls = e >> 5, rl = e & 31;
          if ((unsigned)ls >= (unsigned)nls) {  // guard: never taken unless the ring is corrupt
            ++nguard;
          } else {
          const float4 Lg = ligS[ls];
          const float ex = W.rx[rl] - Lg.x, ey = W.ry[rl] - Lg.y, ez = W.rz[rl] - Lg.z;
          const float d2 = fmaf(ez, ez, fmaf(ey, ey, ex * ex));
          if (d2 <= cut2)
            k0 = pair_value(P, d2, W.rrow[rl] + __float_as_int(Lg.w), k * SD_TILE + rl, ls, a0, nfb, nz, ncut);
          }
        }
        if (v1) {
          const int e = W.ring[i1 & (kRing - 1)];
          const int ls = e >> 5, rl = e & 31;
          if ((unsigned)ls >= (unsigned)nls) {  // guard: never taken unless the ring is corrupt
            ++nguard;
          } else {
          const float4 Lg = ligS[ls];
          const float ex = W.rx[rl] - Lg.x, ey = W.ry[rl] - Lg.y, ez = W.rz[rl] - Lg.z;
          const float d2 = fmaf(ez, ez, fmaf(ey, ey, ex * ex));
          if (d2 <= cut2)
            k1 = pair_value(P, d2, W.rrow[rl] + __float_as_int(Lg.w), k * SD_TILE + rl, ls, a1, nfb, nz, ncut);
          }
        }
        if (k0) {
          acc += a0;
          ++npairs;
        }
        if (k1) {
          acc += a1;
          ++npairs;
        }
        tail += n;
      };
      // stage 1: test the first 32 pending candidates against every lane's receptor atom
      auto batch = [&](int nb) {
        __syncwarp();
        unsigned m = 0;
        if (!kH16) {
          // unused candidate places sit at -1e18, inactive receptor lanes at +1e18: never in range
          if (lane < nb) W.cand_xyz[lane] = ligS[W.cand_slot[lane]];
          else W.cand_xyz[lane] = make_float4(-1e18f, -1e18f, -1e18f, 0.f);
          __syncwarp();
#pragma unroll
          for (int b = 0; b < 32; ++b) {
            const float4 l = W.cand_xyz[b];
            const float ex = fx - l.x, ey = fy - l.y, ez = fz - l.z;
            const float d2 = fmaf(ez, ez, fmaf(ey, ey, ex * ex));
            m |= (d2 <= cut2 ? 1u : 0u) << b;
          }
          // only real candidates and real receptor atoms may produce pairs
          m &= active ? (nb >= 32 ? 0xffffffffu : ((1u << nb) - 1u)) : 0u;
        } else {
          // candidate 2i in the low half, 2i+1 in the high half of pair slot i; unused places
          // at -1000 and inactive receptor lanes at +inf (1e18 overflows): never in range
          __half hx = __float2half_rn(-1000.f), hy = hx, hz = hx;
          if (lane < nb) {
            const float4 l = ligS[W.cand_slot[lane]];
            hx = __float2half_rn(l.x - cx);
            hy = __float2half_rn(l.y - cy);
            hz = __float2half_rn(l.z - cz);
          }
          __half* q = W.cand_h[lane >> 1];
          q[0 + (lane & 1)] = hx;
          q[2 + (lane & 1)] = hy;
          q[4 + (lane & 1)] = hz;
          __syncwarp();
          const __half2 rx2 = __half2half2(__float2half_rn(fx - cx));
          const __half2 ry2 = __half2half2(__float2half_rn(fy - cy));
          const __half2 rz2 = __half2half2(__float2half_rn(fz - cz));
          const __half2 th2 = __float2half2_rn(229.0f);
          unsigned M = 0;
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const uint4 qq = *reinterpret_cast<const uint4*>(W.cand_h[i]);
            const __half2 dx = __hsub2(rx2, *reinterpret_cast<const __half2*>(&qq.x));
            const __half2 dy = __hsub2(ry2, *reinterpret_cast<const __half2*>(&qq.y));
            const __half2 dz = __hsub2(rz2, *reinterpret_cast<const __half2*>(&qq.z));
            const __half2 d2 = __hfma2(dz, dz, __hfma2(dy, dy, __hmul2(dx, dx)));
            M |= __hle2_mask(d2, th2) & (0x00010001u << i);
          }
          // back to candidate order: bit i -> 2i, bit 16+i -> 2i+1
          unsigned lo = M & 0xffffu, hi = M >> 16;
          lo = (lo | (lo << 8)) & 0x00ff00ffu;
          lo = (lo | (lo << 4)) & 0x0f0f0f0fu;
          lo = (lo | (lo << 2)) & 0x33333333u;
          lo = (lo | (lo << 1)) & 0x55555555u;
          hi = (hi | (hi << 8)) & 0x00ff00ffu;
          hi = (hi | (hi << 4)) & 0x0f0f0f0fu;
          hi = (hi | (hi << 2)) & 0x33333333u;
          hi = (hi | (hi << 1)) & 0x55555555u;
          m = lo | (hi << 1);
          m &= active ? (nb >= 32 ? 0xffffffffu : ((1u << nb) - 1u)) : 0u;
        }
        nevals += (unsigned long long)(lane == 0 ? nb * nact : 0);
        // exclusive scan of the per-lane pair counts
        const int cnt = __popc(m);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        if (head - tail + total > kRing)  // only for very dense batches: empty the ring first
          while (head - tail > 0) drain(min(64, head - tail));
        int pos = head + incl - cnt;
        while (m) {
          const int b = __ffs(m) - 1;
          m &= m - 1;
          W.ring[pos & (kRing - 1)] = (W.cand_slot[b] << 5) | lane;
          ++pos;
        }
        head += total;
        __syncwarp();
        // keep the candidates beyond the first 32
        const int rest = ncand - nb;
        int carry = 0;
        if (lane < rest) carry = W.cand_slot[32 + lane];
        __syncwarp();
        if (lane < rest) W.cand_slot[lane] = carry;
        ncand = rest;
        __syncwarp();
        while (head - tail >= 64) drain(64);
      };

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
          const float4 la = ligS[sb + lane];
          const float ax = la.x - cx, ay = la.y - cy, az = la.z - cz;
          const bool cand = ax * ax + ay * ay + az * az <= reach2;
          const unsigned am = __ballot_sync(0xffffffffu, cand);
          if (cand) W.cand_slot[ncand + __popc(am & lt_mask)] = sb + lane;
          ncand += __popc(am);
          if (ncand >= 32) batch(32);
        }
      }
      if (ncand > 0) batch(ncand);
      while (head - tail > 0) drain(min(64, head - tail));
      __syncwarp();
    }
    // FP64 block reduction of the per-thread sums
    double v = acc;
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
  if (nguard) atomicAdd(&ctl->stats[ST_GUARD], nguard);
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
