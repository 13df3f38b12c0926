// Mixed-precision DFIRE scoring (included by sd_score.cu: shares its constant-memory key
// thresholds and exact_key).
//
// Same contract as the FP64 kernels: the energy of cdfire_calculate_dfire
// (prepare_gso_tasks.cc:1522-1615) with every bin identical to the FP64 reference bin, FP64 sums
// of FP64 table values, but in a free order, which the kernel uses:
//  * persistent CTAs grab poses from the device work list; per pose the ligand is transformed
//    (exact FP64, rounded to FP32 centred on the pose translation t) only for the spatial chunks
//    of 32 atoms that some receptor tile within reach can reach, and the near receptor tiles are
//    ordered largest-first (closest to the ligand centroid) so warps finish a pose together;
//  * a warp takes a receptor tile (one lane per atom, FP64 ANM transform rounded to FP32),
//    rejects ligand chunks by bounding spheres and ligand atoms by ballot, and stages the
//    surviving candidates 32 at a time into one of two per-warp batch buffers, in the bit order
//    of the stage-1 mask (candidate 2i at position i, 2i+1 at position 16+i);
//  * stage 1 tests a pair with the dot-product form of the distance in packed FP16, three
//    HFMA2 per two candidates: s = r.l - |l|^2/2 >= (|r|^2 - thr)/2, on coordinates centred on
//    the tile centre.  thr is set per tile from a proven bound on the FP16 error (below), so
//    every pair whose FP32 d^2 is within the cutoff passes; tiles or poses whose magnitudes
//    would make the bound loose pass every candidate, and stage 2 filters exactly;
//  * in-cutoff pairs are appended to a per-warp ring of 16-bit entries (buffer, position,
//    receptor lane) by a warp scan; stage 2 drains it 64 entries per round (two per lane), reads
//    the candidate and the receptor atom from 4-byte arrays and a float4 (mostly broadcast
//    reads), recomputes the FP32 d^2 and takes the key from a fast reciprocal square root.  The
//    key's edges ((k+1)/2)^2 and ((k+2)/2)^2 (the upper one stopped at the cutoff) are
//    compared with d^2 - edge computed with one rounding against the FP32 error bound B, so a
//    pair that is not near an edge has its FP64 bin proven; near pairs are recomputed from the
//    exact FP64 transform (counted as fallbacks);
//  * the table is gathered from a key-indexed copy [168][168][32] (entry k is the value the
//    reference reads for key k, including the d^2 == 225 read of the next ligand type's bin 0),
//    so no bin lookup is needed; a rejected or padding pair gathers a zero past the table instead
//    of branching, and each round's gathers (through L2 only) are added by the next round, so
//    they are in flight while the next round is evaluated.  Each lane sums its values in FP64
//    (Kahan sums of an FP32-rounded table were measured to miss 1e-5 at 60k pairs per pose).
//  * Fixed summation order: a tile's lane sums are reduced by warp shuffles when the tile is
//    done and stored in a per-pose shared slot of that tile; at the pose end warp 0 adds the
//    slots in a fixed order.  What happens inside a tile depends only on the pose and the tile,
//    never on which warp took it or when, and no compiled variant changes it, so a pose's energy
//    is the same bits in every run, every variant and every entry point.
//
// FP16 bound (u = 2^-11, R >= |r - c| for the tile's atoms, Lb >= |l - c| for its candidates,
// w = |l - c|^2 / 2):  |s_fp16 - (r.l - w)| <= u (2.001 R Lb + w) + 3u (1.002 R Lb + 1.001 w)
// <= u (5.1 R Lb + 2.1 Lb^2) = Es, and the right-hand side rounds by at most u (R^2 + thr)/2 = Ea,
// so thr = 225 + B + 2 Es + 2 Ea + 0.01 keeps every pair with FP32 d^2 <= 225 + B.
#pragma once

namespace sd {
namespace {

constexpr int kRingCap = 1088;  // < 64 left over + at most 32 x 32 from one batch
constexpr int kZeroIdxKey = SD_TABLE_KEYS;   // a zero past the key-indexed table

// exact FP64 key of one pair near a bin edge or the cutoff; -1 when the pair is outside the
// cutoff; *edge = 1 for d^2 == 0, 2 for d^2 == 225 (inlined: measured fewer spills than a call)
__device__ __forceinline__ int exact_pair_key(const DevComplex* C, int nslots, const double* pose,
                                                     const double* q, const double* qi, const double* T, int slot,
                                                     int j, int* edge) {
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
  const int key = exact_key(e2, T);
  if (key == 29) *edge = 2;
  return key;
}

struct __align__(16) RingBufs {
  float candf[4][64];        // x, y, z, col bits of [buffer][position]: ligand atom centred on t
  __half candh[16][8];       // position pair i: {x(2i), x(2i+1), y.., y.., z.., z.., -w.., -w..}
  float4 rec[32];            // receptor atom of each lane centred on t, row bits
  unsigned short cslot[64];  // [buffer][position]: ligand chunk slot (exact fallback only)
  unsigned short pend[64];   // pending candidate ligand slots (below SD_MAX_LIG)
  unsigned short ring[kRingCap];  // (buffer << 10) | (position << 5) | lane
};

}  // namespace

// Variants differ only in warps per CTA and resident CTAs per SM: a tile is always processed by
// one warp in the same way, so they give identical energies.  kSpill: the per-pose arrays (tile
// sums, transformed ligand, chunk spheres, tile lists) live in this CTA's slice of the global
// scratch L.spill, for complexes too large for shared memory; the arithmetic is the same.
template <int kWarps, int kMinBlocks, bool kSpill>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) dfire_score_mixed_kernel(ScoreLaunch L) {
  constexpr int kG = 64;  // entries per stage-2 round, two per lane
  constexpr int kSortMax = 512;        // near tiles ordered largest-first up to this many
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  unsigned char* const smem = kSpill ? L.spill + (size_t)blockIdx.x * L.spill_stride : smem_dyn;
  __shared__ RingBufs wb[kWarps];
  __shared__ double sh_pose[7 + 2 * SD_MAX_MODES];
  __shared__ double sh_q[4], sh_qi[4];
  __shared__ double sh_T[32];
  __shared__ float sh_gc[3];      // ligand centroid, rotated (centred on t)
  __shared__ double sh_red[1];
  __shared__ int sh_item, sh_ntile, sh_next;
  __shared__ float sh_bound[4];
  __shared__ float sh_rot[9];
  __shared__ unsigned long long sh_cnt[5];  // fallback, d2 == 0, d2 == 225, pairs, evaluations

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid < 32) sh_T[tid] = c_T[tid];
  if (tid < 5) sh_cnt[tid] = 0;
  StepCtl* ctl = L.ctl;
  const int parity = ctl->parity;
  const int count = ctl->count[parity];
  const int* work = L.work[parity];
  unsigned n_done = 0;
  const unsigned lt_mask = (1u << lane) - 1u;
  RingBufs& W = wb[warp];

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
    if (warp == 0) {
      // pose prologue spread over warp 0: quaternion inverse (one division per lane, bit-identical
      // to quat_inverse), FP32 rotation for culling, ANM displacement bounds, reference point
      if (lane < 4) {
        const double w0 = sh_pose[3], x = sh_pose[4], y = sh_pose[5], z = sh_pose[6];
        const double n2 = w0 * w0 + x * x + y * y + z * z;
        const double qv = sh_pose[3 + lane];
        sh_q[lane] = qv;
        sh_qi[lane] = (lane == 0 ? qv : -qv) / n2;
      }
      {
        const float qw = (float)sh_pose[3], qx = (float)sh_pose[4], qy = (float)sh_pose[5], qz = (float)sh_pose[6];
        const float in = rsqrtf(qw * qw + qx * qx + qy * qy + qz * qz);
        const float w0 = qw * in, x = qx * in, y = qy * in, z = qz * in;
        float rv = 0.f;
        switch (lane) {
          case 0: rv = 1 - 2 * (y * y + z * z); break;
          case 1: rv = 2 * (x * y - w0 * z); break;
          case 2: rv = 2 * (x * z + w0 * y); break;
          case 3: rv = 2 * (x * y + w0 * z); break;
          case 4: rv = 1 - 2 * (x * x + z * z); break;
          case 5: rv = 2 * (y * z - w0 * x); break;
          case 6: rv = 2 * (x * z - w0 * y); break;
          case 7: rv = 2 * (y * z + w0 * x); break;
          case 8: rv = 1 - 2 * (x * x + y * y); break;
          default: break;
        }
        if (lane < 9) sh_rot[lane] = rv;
      }
      float tR = lane < C.nmr ? fabsf((float)sh_pose[7 + lane]) * C.mnorm_r[lane] : 0.f;
      float tL = lane < C.nml ? fabsf((float)sh_pose[7 + C.nmr + lane]) * C.mnorm_l[lane] : 0.f;
      for (int o = 16; o > 0; o >>= 1) {
        tR += __shfl_xor_sync(0xffffffffu, tR, o);
        tL += __shfl_xor_sync(0xffffffffu, tL, o);
      }
      __syncwarp();
      if (lane < 3)
        sh_gc[lane] = sh_rot[3 * lane] * C.lig_ctr[0] + sh_rot[3 * lane + 1] * C.lig_ctr[1] +
                      sh_rot[3 * lane + 2] * C.lig_ctr[2];
      if (lane == 0) {
        const float dR = tR * 1.0001f + 1e-4f, dL = tL * 1.0001f + 1e-4f;
        sh_bound[0] = dR;
        sh_bound[1] = dL;
        // bound of |FP32 d2 - FP64 d2| for pairs within 15.1 A (coordinates centred on t)
        const float RL = C.lig_radius + dL;
        const float u32 = 5.9604645e-8f;
        sh_bound[2] = 2.0f * (2.02f * u32 * (26.2f * (2.0f * RL + 15.1f) + 228.0f) + 3.0f * u32 * 228.0f) + 1e-6f;
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
    }
    __syncthreads();
    const double tx = sh_pose[0], ty = sh_pose[1], tz = sh_pose[2];
    const float dR = sh_bound[0], dL = sh_bound[1], B = sh_bound[2];
    const int nls = nlc * SD_TILE, ntiles = C.ntiles;
    double* tsum = reinterpret_cast<double*>(smem);  // [ntiles] FP64 energy of each tile of the pose
    float4* ligS = reinterpret_cast<float4*>(tsum + ((ntiles + 1) & ~1));  // [nls] centred on t, col bits
    float4* chS = ligS + nls;                        // [nlc] centre + radius
    int* tlist = reinterpret_cast<int*>(chS + nlc);  // [ntiles] tiles within reach
    int* tord = tlist + ntiles;                      // [ntiles] the same, largest first
    float* tdist = reinterpret_cast<float*>(tord + ntiles);  // [ntiles]
    int* cneed = reinterpret_cast<int*>(tdist + ntiles);     // [nlc] chunk within reach of a near tile
    for (int c = tid; c < nlc; c += blockDim.x) {
      const float4 cc = C.l_chunk[c];
      const float X = sh_rot[0] * cc.x + sh_rot[1] * cc.y + sh_rot[2] * cc.z;
      const float Y = sh_rot[3] * cc.x + sh_rot[4] * cc.y + sh_rot[5] * cc.z;
      const float Z = sh_rot[6] * cc.x + sh_rot[7] * cc.y + sh_rot[8] * cc.z;
      chS[c] = make_float4(X, Y, Z, cc.w + dL);
      cneed[c] = 0;
    }
    for (int k = tid; k < ntiles; k += blockDim.x) tsum[k] = 0.0;
    const float lig_reach = C.lig_radius + dL;
    for (int k = tid; k < ntiles; k += blockDim.x) {
      const float4 tile = C.r_tile[k];
      const float cx = (float)((double)tile.x - tx), cy = (float)((double)tile.y - ty),
                  cz = (float)((double)tile.z - tz);
      const float reach = 15.0f + dR + SD_CULL_MARGIN + tile.w + lig_reach;
      if (cx * cx + cy * cy + cz * cz <= reach * reach) {
        // distance from the ligand centroid: the closest tiles have the most pairs
        const int at = atomicAdd(&sh_ntile, 1);
        const float ex = cx - sh_gc[0], ey = cy - sh_gc[1], ez = cz - sh_gc[2];
        tlist[at] = k;
        // a NaN distance (non-finite quaternion) ranks last: the ranking below must stay a strict
        // total order, or tord would not be a permutation of the near tiles
        const float dd = ex * ex + ey * ey + ez * ez;
        tdist[at] = dd == dd ? dd : 3.0e38f;
      }
    }
    __syncthreads();
    const int ntile = sh_ntile;
    const bool sorted = ntile <= kSortMax;
    // which ligand chunks any near tile can reach (the same test as the per-tile one below, with
    // 0.01 A to spare, so a chunk that is not needed is never read)
    for (int t = warp; t < ntile; t += kWarps) {
      const float4 tile = C.r_tile[tlist[t]];
      const float cx = (float)((double)tile.x - tx), cy = (float)((double)tile.y - ty),
                  cz = (float)((double)tile.z - tz);
      const float rt = 15.0f + dR + SD_CULL_MARGIN + tile.w;
      for (int c = lane; c < nlc; c += 32) {
        const float4 ch = chS[c];
        const float ex = ch.x - cx, ey = ch.y - cy, ez = ch.z - cz, r = rt + ch.w + 0.01f;
        if (ex * ex + ey * ey + ez * ez <= r * r) cneed[c] = 1;
      }
    }
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
    }
    __syncthreads();
    auto lig_atom = [&](int s) {
      if (s >= nls || !cneed[s >> 5]) return;
      if (C.l_perm[s] >= 0) {
        double x, y, z;
        ligand_exact_chunk(C, s, sh_pose, sh_q, sh_qi, x, y, z);
        ligS[s] = make_float4((float)(x - tx), (float)(y - ty), (float)(z - tz), __int_as_float(C.lc_colk[s]));
      } else {
        ligS[s] = make_float4(1e18f, 1e18f, 1e18f, __int_as_float(0));
      }
    };
    for (int s = tid; s < nls; s += 2 * kWarps * 32) {
      lig_atom(s);
      lig_atom(s + kWarps * 32);
    }
    __syncthreads();
    const int* tl = sorted ? tord : tlist;
    const float cut2 = 225.0f + B;
    double acc = 0.0;               // per-lane FP64 sum of table values
    double pv0 = 0.0, pv1 = 0.0;    // values gathered by the previous round, added by the next
    const double* table = L.tablek;
    unsigned npairs = 0, nevals = 0;

    for (;;) {
      int ti = 0;
      if (lane == 0) ti = atomicAdd(&sh_next, 1);
      ti = __shfl_sync(0xffffffffu, ti, 0);
      if (ti >= ntile) break;
      const int k = tl[ti];
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
        row = C.r_rowk[slot];
      }
      W.rec[lane] = make_float4(fx, fy, fz, __int_as_float(row));
      const unsigned act_mask = __ballot_sync(0xffffffffu, active);
      const int nact = __popc(act_mask);
      // stage-1 constants of this lane
      __half2 rx2, ry2, rz2, a2;
      const float R = tile.w + dR + SD_CULL_MARGIN, Lb = reach + 0.01f;
      const bool tight = R <= 40.0f && Lb <= 80.0f;  // warp-uniform
      {
        const float u16 = 4.8828125e-4f;
        const float Es = u16 * (5.1f * R * Lb + 2.1f * Lb * Lb);
        const float thr0 = 225.0f + B + 1e-3f + 2.0f * Es;
        const float thr = thr0 + u16 * (R * R + thr0 + 10.0f) + 2e-4f + 0.01f;
        const float ux = fx - cx, uy = fy - cy, uz = fz - cz;
        const float a = 0.5f * (ux * ux + uy * uy + uz * uz) - 0.5f * thr;
        const bool use = active && tight;
        rx2 = __float2half2_rn(use ? ux : 0.f);
        ry2 = __float2half2_rn(use ? uy : 0.f);
        rz2 = __float2half2_rn(use ? uz : 0.f);
        // loose tile: every candidate passes (s = 0 > -65504); inactive lane: none does
        a2 = __float2half2_rn(!active ? 65504.f : (tight ? a : -65504.f));
      }
      int ncand = 0, head = 0, par = 0, oldL = 0;  // ring holds entries [0, head)
      int cb = 0;
      unsigned cm = 0;

      for (;;) {
        // collect candidates until a batch is full or the ligand is exhausted
        while (ncand < 32) {
          if (cm == 0) {
            if (cb >= nlc) break;
            const int c = cb + lane;
            bool cnear = false;
            if (c < nlc) {
              const float4 ch = chS[c];
              const float ex = ch.x - cx, ey = ch.y - cy, ez = ch.z - cz, r = reach + ch.w;
              cnear = ex * ex + ey * ey + ez * ez <= r * r;  // same expression as the cneed test
            }
            cm = __ballot_sync(0xffffffffu, cnear);
            cb += 32;
            continue;
          }
          const int sb = (cb - 32 + __ffs(cm) - 1) * SD_TILE;
          cm &= cm - 1;
          const float4 la = ligS[sb + lane];
          const float ax = la.x - cx, ay = la.y - cy, az = la.z - cz;
          const bool cand = fmaf(az, az, fmaf(ay, ay, ax * ax)) <= reach2;
          const unsigned am = __ballot_sync(0xffffffffu, cand);
          if (cand) W.pend[ncand + __popc(am & lt_mask)] = (unsigned short)(sb + lane);
          ncand += __popc(am);
        }
        const bool exhausted = cm == 0 && cb >= nlc;
        if (ncand == 0 && head == 0) break;
        const int nb = min(ncand, 32);
        const bool final_batch = exhausted && ncand <= 32;
        if (nb > 0) {
          // stage the batch into buffer par, in mask bit order
          __syncwarp();
          const int pos = (lane >> 1) | ((lane & 1) << 4);
          float4 l4 = make_float4(-1e18f, -1e18f, -1e18f, 0.f);
          int s = 0;
          if (lane < nb) {
            s = W.pend[lane];
            l4 = ligS[s];
          }
          W.candf[0][par * 32 + pos] = l4.x;
          W.candf[1][par * 32 + pos] = l4.y;
          W.candf[2][par * 32 + pos] = l4.z;
          W.candf[3][par * 32 + pos] = l4.w;
          W.cslot[par * 32 + pos] = (unsigned short)s;
          {
            // unused place: s = -60000, never in range; loose tile: every place passes
            float lx = 0.f, ly = 0.f, lz = 0.f, nw = tight ? -60000.f : 0.f;
            if (lane < nb && tight) {
              lx = l4.x - cx;
              ly = l4.y - cy;
              lz = l4.z - cz;
              nw = fmaxf(-0.5f * (lx * lx + ly * ly + lz * lz), -60000.f);
            }
            // lanes 2i and 2i+1 fill candh[i] with one 8-byte store each: the even lane the x and y
            // pairs, the odd lane the z and w pairs (conflict-free, where 16-bit stores collide)
            const __half2 xy = __floats2half2_rn(lx, ly), zw = __floats2half2_rn(lz, nw);
            const bool odd = lane & 1;
            const __half2 other = __shfl_xor_sync(0xffffffffu, odd ? xy : zw, 1);
            const __half2 mine = odd ? zw : xy;
            const __half2 lo = odd ? other : mine, hi = odd ? mine : other;  // even lane's, odd lane's
            const __half2 o0 = __lows2half2(lo, hi), o1 = __highs2half2(lo, hi);
            uint2 u;
            u.x = reinterpret_cast<const unsigned&>(o0);
            u.y = reinterpret_cast<const unsigned&>(o1);
            *reinterpret_cast<uint2*>(reinterpret_cast<unsigned char*>(W.candh[lane >> 1]) + 8 * (lane & 1)) = u;
          }
          __syncwarp();
          // stage 1: bit b of m <=> (this lane's receptor atom, candidate at position b) in range
          unsigned M = 0;
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const uint4 qq = *reinterpret_cast<const uint4*>(W.candh[i]);
            __half2 sv = __hfma2(rx2, *reinterpret_cast<const __half2*>(&qq.x), *reinterpret_cast<const __half2*>(&qq.w));
            sv = __hfma2(ry2, *reinterpret_cast<const __half2*>(&qq.y), sv);
            sv = __hfma2(rz2, *reinterpret_cast<const __half2*>(&qq.z), sv);
            M |= __hge2_mask(sv, a2) & (0x00010001u << i);
          }
          const unsigned lo = (1u << ((nb + 1) >> 1)) - 1u, hi = (1u << (nb >> 1)) - 1u;
          unsigned m = M & (lo | (hi << 16)) & (active ? 0xffffffffu : 0u);
          nevals += lane == 0 ? (unsigned)(nb * nact) : 0u;
          // append this lane's pairs to the ring
          const int cnt = __popc(m);
          int incl = cnt;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
          }
          const int total = __shfl_sync(0xffffffffu, incl, 31);
          int at = head + incl - cnt;
          const unsigned tag = ((unsigned)par << 10) | (unsigned)lane;
          // two entries per iteration: the highest and the lowest bit left
          while (m) {
            const int b = 31 - __clz(m);
            const unsigned low = m & (0u - m);
            const int b2 = 31 - __clz(low);
            m &= ~((1u << b) | low);
            W.ring[at] = (unsigned short)(tag | ((unsigned)b << 5));
            if (b2 != b) W.ring[at + 1] = (unsigned short)(tag | ((unsigned)b2 << 5));
            at += b2 != b ? 2 : 1;
          }
          head += total;
          // keep the candidates beyond the first 32
          const int rest = ncand - nb;
          int carry = 0;
          if (lane < rest) carry = W.pend[32 + lane];
          __syncwarp();
          if (lane < rest) W.pend[lane] = (unsigned short)carry;
          ncand = rest;
          par ^= 1;
        }
        __syncwarp();
        // stage 2: drain whole rounds of kG; everything at the end of the tile, or when entries
        // of the previous batch would otherwise outlive its buffer
        const int upto = (final_batch || (oldL > 0 && head < kG)) ? head : (head & ~(kG - 1));
        auto pair = [&](int t0, int h, int n) -> int {
          const unsigned e = W.ring[t0 + h * 32 + lane];
          const int cix = (int)(e >> 5) & 63, rl = (int)e & 31;
          const float4 rr = W.rec[rl];
          const float ex = rr.x - W.candf[0][cix], ey = rr.y - W.candf[1][cix], ez = rr.z - W.candf[2][cix];
          const int col = __float_as_int(W.candf[3][cix]);
          const float d2 = fmaf(ez, ez, fmaf(ey, ey, ex * ex));
          bool ok = (h * 32 + lane < n) && d2 <= cut2;
          // key estimate; d2 == 0 gives NaN -> 0 and lies within B of edge 0 (exact path)
          const float r = d2 * rsqrtf(d2);
          const int key = (int)fmaf(r, 2.0f, -1.0f) & 31;
          // key edges ((key+1)/2)^2 and ((key+2)/2)^2, differences with one rounding; the upper
          // edge stops at the cutoff 15^2, so key 29 (d^2 == 225 only) always takes the exact
          // path: the FP32 cut2 = 225 + B may round above 225 + B
          int idx = __float_as_int(rr.w) + col + key;
          const float hk = fmaf((float)key, 0.5f, 0.5f), hk1 = fminf(hk + 0.5f, 15.0f);
          const bool near = fmaf(-hk, hk, d2) <= B || fmaf(hk1, hk1, -d2) <= B;
          if (ok && near) {
            atomicAdd(&sh_cnt[0], 1ull);
            int edge;
            const int kx = exact_pair_key(&C, nslots, sh_pose, sh_q, sh_qi, sh_T, k * SD_TILE + rl,
                                          C.l_perm[W.cslot[cix]], &edge);
            if (kx < 0) {
              ok = false;
            } else {
              idx = __float_as_int(rr.w) + col + kx;
              if (edge) atomicAdd(&sh_cnt[edge], 1ull);
            }
          }
          npairs += ok ? 1u : 0u;
          return ok ? idx : kZeroIdxKey;
        };
        // the gathers go through L2 only (ld.global.cg): each is used once, and cached in L1 they
        // would evict the receptor / ligand atom and mode lines that the next tiles read again
        for (int t0 = 0; t0 < upto; t0 += kG) {
          const int n = min(kG, upto - t0);
          acc += pv0;
          pv0 = __ldcg(table + pair(t0, 0, n));
          acc += pv1;
          pv1 = __ldcg(table + pair(t0, 1, n));
        }
        // move the leftover (< kG) entries to the front
        const int left = head - upto;
        unsigned short e0 = 0, e1 = 0;
        if (lane < left) e0 = W.ring[upto + lane];
        if (lane + 32 < left) e1 = W.ring[upto + 32 + lane];
        __syncwarp();
        if (lane < left) W.ring[lane] = e0;
        if (lane + 32 < left) W.ring[lane + 32] = e1;
        head = left;
        oldL = left;
        if (final_batch) break;
      }
      __syncwarp();
      // the tile's energy: the last round's gathers, then the lane sums in a fixed shuffle order,
      // into the tile's slot
      acc += pv0;
      acc += pv1;
      pv0 = 0.0;
      pv1 = 0.0;
      double v = acc;
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) tsum[k] = v;
      acc = 0.0;
    }
    // counters, then the pose energy: warp 0 adds the tile slots in a fixed order
    const unsigned wp = __reduce_add_sync(0xffffffffu, npairs);
    if (lane == 0) {
      if (wp) atomicAdd(&sh_cnt[3], (unsigned long long)wp);
      if (nevals) atomicAdd(&sh_cnt[4], (unsigned long long)nevals);
    }
    __syncthreads();
    if (warp == 0) {
      double v = 0.0;
      for (int k = lane; k < ntiles; k += 32) v += tsum[k];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) sh_red[0] = v;
    }
    __syncthreads();
    if (tid == 0) {
      const double E = sh_red[0];
      const double score = ((E)*0.0157 - 4.7) * -1;
      C.scoring[p] = score;
      if (L.energy_out) L.energy_out[p] = E;
      ++n_done;
    }
  }
  __syncthreads();
  if (tid == 0) {
    if (n_done) atomicAdd(&ctl->stats[ST_SCORED], (unsigned long long)n_done);
    if (sh_cnt[0]) atomicAdd(&ctl->stats[ST_FALLBACK], sh_cnt[0]);
    if (sh_cnt[1]) atomicAdd(&ctl->stats[ST_D2ZERO], sh_cnt[1]);
    if (sh_cnt[2]) atomicAdd(&ctl->stats[ST_D2CUT], sh_cnt[2]);
    if (sh_cnt[3]) atomicAdd(&ctl->stats[ST_PAIRS], sh_cnt[3]);
    if (sh_cnt[4]) atomicAdd(&ctl->stats[ST_EVALS], sh_cnt[4]);
  }
}

}  // namespace sd
