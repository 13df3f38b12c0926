// GSO update of all swarms: luciferin, neighbours, probabilistic selection, movement and
// vision range.  One CTA per swarm, one thread per glowworm, FP64 with no contraction.
//
// Semantics: cal_gso_tasks_cpu passes 1-3 after scoring (prepare_gso_tasks.cc:558-559,
// :600-707, :716-814) with compute_probability_moving_from_neighbors (:1463-1488),
// select_random_neighbor (:1424-1459), slerp (:1370-1421) and move_extent (:1352-1368).
// Replaces the reference GPU kernels generate_energy_v2 / cal_move_neighbors /
// move_position_v2 (prepare_gso_task.cu:2377-2433, :791-897, :1059-1136).
//
// The update is synchronous (every glowworm selects from pre-move state): luciferin and
// reference points of the swarm are staged in shared memory, and a barrier separates the
// reads of the chosen neighbours' positions from the writes of the moved positions.  The
// neighbour list is never stored: its length, probability total and the cumulative choice
// are recomputed in two ordered scans over the swarm, which gives the same floating-point
// sums as the reference's list.  Moved glowworms are appended to the next work list; the
// last CTA to finish advances the step (parity, draw cursors, counters) so that the whole
// step can be replayed from a CUDA graph.
#include <cuda_runtime.h>

#include <string>

#include "sd_crmath.h"
#include "sd_internal.h"

namespace sd {

__device__ __forceinline__ void move_extent_dev(double* self, const double* other, int n_ext, double step) {
  double delta[SD_MAX_MODES];
  double n = 0;
  for (int i = 0; i < n_ext; ++i) {
    delta[i] = other[i] - self[i];
    n += delta[i] * delta[i];
  }
  n = sqrt(n);
  if (n >= 1e-8) {
    for (int i = 0; i < n_ext; ++i) {
      delta[i] *= step / n;
      self[i] += delta[i];
    }
  }
}

__device__ __forceinline__ void slerp_dev(double* self, double* other, double step) {
  double sn = 0, on = 0;
  for (int i = 0; i < 4; ++i) {
    sn += (self[i] * self[i]);
    on += (other[i] * other[i]);
  }
  sn = sqrt(sn);
  on = sqrt(on);
  for (int i = 0; i < 4; ++i) {
    self[i] /= sn;
    other[i] /= on;
  }
  double q_dot = 0;
  for (int i = 0; i < 4; ++i) q_dot += self[i] * other[i];
  if (q_dot < 0) {
    q_dot = q_dot * -1;
    for (int i = 0; i < 4; ++i) self[i] = -self[i];
  }
  if (q_dot > 0.9995) {
    for (int i = 0; i < 4; ++i) self[i] = self[i] + step * (other[i] - self[i]);
    double rn = 0;
    for (int i = 0; i < 4; ++i) rn += (self[i] * self[i]);
    rn = sqrt(rn);
    for (int i = 0; i < 4; ++i) self[i] /= rn;
  } else {
    q_dot = (q_dot < 1) ? q_dot : 1;
    q_dot = (q_dot > -1) ? q_dot : -1;
    const double omega = sd_acos_cr(q_dot);
    const double so = sd_sin_cr(omega);
    const double tmp0 = (sd_sin_cr((1.0 - step) * omega) / so);
    const double tmp1 = (sd_sin_cr(step * omega) / so);
    for (int i = 0; i < 4; ++i) self[i] = tmp0 * self[i] + tmp1 * other[i];
  }
}

// Neighbours of glowworm g (luciferin shL[G] and reference points shR[G][3] of its swarm in shared
// memory; vision range vr) in ascending n (prepare_gso_tasks.cc:615-640), their probability total
// (:1476-1484) and the first whose cumulative probability reaches the draw *u (:1441-1450).
// Returns the choice (g itself without neighbours) and the count in nn; counts the draws <= 0 with
// neighbours (the reference reads neighbors[-1]; the first is taken) and the cumulative shortfalls
// (the last is taken).
__device__ __forceinline__ int choose_neighbour(const double* shL, const double* shR, int G, int g, double Lg,
                                                double vr, const double* u_ptr, int& nn,
                                                unsigned long long* uzero, unsigned long long* shortfall) {
  const double cx = shR[g * 3], cy = shR[g * 3 + 1], cz = shR[g * 3 + 2];
  const double sq = vr * vr;
  double total = 0;
  nn = 0;
  for (int n = 0; n < G; ++n) {
    const double Ln = shL[n];
    if (n != g && Lg < Ln) {
      const double dx = cx - shR[n * 3], dy = cy - shR[n * 3 + 1], dz = cz - shR[n * 3 + 2];
      double distance = 0;
      distance += dx * dx;
      distance += dy * dy;
      distance += dz * dz;
      if (distance < sq) {
        ++nn;
        total += Ln - Lg;
      }
    }
  }
  if (nn == 0) return g;
  const double u = *u_ptr;
  double sum = 0.0;
  int picked = -1, last = -1;
  if (!(sum < u)) atomicAdd(uzero, 1ull);
  for (int n = 0; n < G && picked < 0; ++n) {
    const double Ln = shL[n];
    if (n != g && Lg < Ln) {
      const double dx = cx - shR[n * 3], dy = cy - shR[n * 3 + 1], dz = cz - shR[n * 3 + 2];
      double distance = 0;
      distance += dx * dx;
      distance += dy * dy;
      distance += dz * dz;
      if (distance < sq) {
        last = n;
        if (!(sum < u)) {
          picked = n;  // only reached when u <= 0
        } else {
          sum += (Ln - Lg) / total;
          if (!(sum < u)) picked = n;
        }
      }
    }
  }
  if (picked < 0) {
    picked = last;
    atomicAdd(shortfall, 1ull);
  }
  return picked;
}

// Movement of one glowworm towards the chosen neighbour's pose mv (prepare_gso_tasks.cc:772-794):
// translation by step_t along the direction, slerp of the quaternion, receptor and ligand extents.
__device__ __forceinline__ void move_towards(double* cur, double* mv, int nmr, int nml, const GsoParamsDev& P) {
  double delta[3], n = 0;
  for (int d = 0; d < 3; ++d) {
    delta[d] = mv[d] - cur[d];
    n += (delta[d] * delta[d]);
  }
  n = sqrt(n);
  if (n >= 1e-8) {
    for (int d = 0; d < 3; ++d) {
      delta[d] *= (P.step_t / n);
      cur[d] += delta[d];
    }
  }
  slerp_dev(cur + 3, mv + 3, P.step_r);
  move_extent_dev(cur + 7, mv + 7, nmr, P.step_nm);
  move_extent_dev(cur + 7 + nmr, mv + 7 + nmr, nml, P.step_nm);
}

__global__ void __launch_bounds__(SD_MAX_G) gso_kernel(GsoLaunch L) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int sh_base, sh_last;
  __shared__ unsigned long long sh_uzero, sh_short;
  const int sw_packed = L.swarm_map[blockIdx.x];
  const int ci = wi_complex(sw_packed), s = wi_local(sw_packed);
  DevComplex& C = L.cplx[ci];
  const int G = C.G, pl = C.pl, g = threadIdx.x;
  const bool live = g < G;
  double* shL = reinterpret_cast<double*>(smem);  // [G]
  double* shR = shL + G;                          // [G][3]
  StepCtl* ctl = L.ctl;
  const int parity = ctl->parity;
  const GsoParamsDev P = L.p;
  if (g == 0) {
    sh_uzero = 0;
    sh_short = 0;
  }
  const size_t k = (size_t)s * G + g;
  // luciferin (prepare_gso_tasks.cc:558)
  double Lg = 0.0;
  if (live) {
    Lg = (1.0 - P.rho) * C.luciferin[k] + P.gamma * C.scoring[k];
    C.luciferin[k] = Lg;
    C.step[k] += 1;
    shL[g] = Lg;
    shR[g * 3] = C.ref[k * 3];
    shR[g * 3 + 1] = C.ref[k * 3 + 1];
    shR[g * 3 + 2] = C.ref[k * 3 + 2];
  }
  __syncthreads();
  int sel = g, nn = 0;
  if (live)
    sel = choose_neighbour(shL, shR, G, g, Lg, C.vision[k],
                           C.draws + (size_t)s * C.draw_steps * G + (size_t)C.draw_cursor * G + g, nn, &sh_uzero,
                           &sh_short);
  // copy of the chosen neighbour's pre-move position (:689-693)
  double mv[7 + 2 * SD_MAX_MODES], cur[7 + 2 * SD_MAX_MODES];
  if (live) {
    const double* src = C.pos + ((size_t)s * G + sel) * pl;
    const double* own = C.pos + k * pl;
    for (int i = 0; i < pl; ++i) {
      mv[i] = src[i];
      cur[i] = own[i];
    }
  }
  __syncthreads();  // all reads of pre-move positions are done
  bool moved = false;
  if (live) {
    moved = sel != g;
    C.moved[k] = moved ? 1 : 0;
    C.nnei[k] = nn;
    C.select[k] = sel;
    if (moved) {
      move_towards(cur, mv, C.nmr, C.nml, P);
      double* own = C.pos + k * pl;
      for (int i = 0; i < pl; ++i) own[i] = cur[i];
    }
    // vision range (:806-808)
    double vr = C.vision[k] + P.beta * (P.max_neighbors - nn);
    if (vr < 0.0) vr = 0;
    if (vr > P.max_vision) vr = P.max_vision;
    C.vision[k] = vr;
  }
  // next work list: moved glowworms, in glowworm order within the swarm
  const unsigned bal = __ballot_sync(0xffffffffu, moved);
  __shared__ int sh_wcount[SD_MAX_G / 32], sh_woff[SD_MAX_G / 32];
  const int lane = g & 31, wid = g >> 5, nw = blockDim.x >> 5;
  if (lane == 0) sh_wcount[wid] = __popc(bal);
  __syncthreads();
  if (g == 0) {
    int acc = 0;
    for (int w = 0; w < nw; ++w) {
      sh_woff[w] = acc;
      acc += sh_wcount[w];
    }
    sh_base = acc ? atomicAdd(&ctl->count[parity ^ 1], acc) : 0;
  }
  __syncthreads();
  if (moved) {
    const int pos_in = sh_base + sh_woff[wid] + __popc(bal & ((1u << lane) - 1u));
    L.work[parity ^ 1][pos_in] = wi_pack(ci, (int)k);
  }
  // last block advances the step
  __syncthreads();
  if (g == 0) {
    if (sh_uzero) atomicAdd(&ctl->stats[ST_UZERO], sh_uzero);
    if (sh_short) atomicAdd(&ctl->stats[ST_SHORT], sh_short);
    __threadfence();
    const int done = atomicAdd(&ctl->done_blocks, 1);
    sh_last = done == L.nswarms_total - 1;
  }
  __syncthreads();
  if (sh_last && g == 0) {
    __threadfence();
    ctl->count[parity] = 0;
    ctl->grab[parity] = 0;
    ctl->grab[parity ^ 1] = 0;
    ctl->parity = parity ^ 1;
    ctl->done_blocks = 0;
    ctl->step += 1;
    ctl->stats[ST_STEPS] += 1;
    __threadfence();
  }
  if (sh_last && g < L.ncplx) {
    // draws of the next step: one column further for every complex
    __threadfence();
    L.cplx[g].draw_cursor += 1;
  }
}

// Swarms of more than SD_MAX_G glowworms (more than one CTA's threads): the same update with each
// thread taking glowworms tid, tid + blockDim.x, ...  A thread can no longer hold the chosen
// neighbours' pre-move poses of all its glowworms across a barrier, so every pose is first copied to
// L.pos_prev (one row of SD_POSE_LEN(10, 10) doubles per glowworm of the context) and the moves read
// the copies.  Moved glowworms are appended to the next work list one CTA-wide chunk at a time.
__global__ void __launch_bounds__(SD_MAX_G) gso_kernel_large(GsoLaunch L) {
  constexpr int kRow = SD_POSE_LEN(SD_MAX_MODES, SD_MAX_MODES);
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int sh_base, sh_last;
  __shared__ unsigned long long sh_uzero, sh_short;
  __shared__ int sh_wcount[SD_MAX_G / 32], sh_woff[SD_MAX_G / 32];
  const int sw_packed = L.swarm_map[blockIdx.x];
  const int ci = wi_complex(sw_packed), s = wi_local(sw_packed);
  DevComplex& C = L.cplx[ci];
  const int G = C.G, pl = C.pl, tid = threadIdx.x, B = blockDim.x;
  double* shL = reinterpret_cast<double*>(smem);  // [G]
  double* shR = shL + G;                          // [G][3]
  StepCtl* ctl = L.ctl;
  const int parity = ctl->parity;
  const GsoParamsDev P = L.p;
  double* prev = L.pos_prev + ((size_t)C.gbase + (size_t)s * G) * kRow;
  if (tid == 0) {
    sh_uzero = 0;
    sh_short = 0;
  }
  // luciferin (prepare_gso_tasks.cc:558), staging, pre-move copies
  for (int g = tid; g < G; g += B) {
    const size_t k = (size_t)s * G + g;
    const double Lg = (1.0 - P.rho) * C.luciferin[k] + P.gamma * C.scoring[k];
    C.luciferin[k] = Lg;
    C.step[k] += 1;
    shL[g] = Lg;
    shR[g * 3] = C.ref[k * 3];
    shR[g * 3 + 1] = C.ref[k * 3 + 1];
    shR[g * 3 + 2] = C.ref[k * 3 + 2];
    for (int i = 0; i < pl; ++i) prev[(size_t)g * kRow + i] = C.pos[k * pl + i];
  }
  __syncthreads();
  unsigned moved_bits = 0;  // bit c: glowworm c * B + tid moved
  for (int g = tid, c = 0; g < G; g += B, ++c) {
    const size_t k = (size_t)s * G + g;
    int nn = 0;
    const int sel = choose_neighbour(shL, shR, G, g, shL[g], C.vision[k],
                                     C.draws + (size_t)s * C.draw_steps * G + (size_t)C.draw_cursor * G + g, nn,
                                     &sh_uzero, &sh_short);
    const bool moved = sel != g;
    C.moved[k] = moved ? 1 : 0;
    C.nnei[k] = nn;
    C.select[k] = sel;
    if (moved) {
      double mv[kRow], cur[kRow];
      for (int i = 0; i < pl; ++i) {
        mv[i] = prev[(size_t)sel * kRow + i];
        cur[i] = prev[(size_t)g * kRow + i];
      }
      move_towards(cur, mv, C.nmr, C.nml, P);
      for (int i = 0; i < pl; ++i) C.pos[k * pl + i] = cur[i];
      moved_bits |= 1u << c;
    }
    // vision range (:806-808)
    double vr = C.vision[k] + P.beta * (P.max_neighbors - nn);
    if (vr < 0.0) vr = 0;
    if (vr > P.max_vision) vr = P.max_vision;
    C.vision[k] = vr;
  }
  // next work list, chunk by chunk, in glowworm order within a chunk
  const int lane = tid & 31, wid = tid >> 5, nw = B >> 5;
  for (int c = 0; c * B < G; ++c) {
    const bool moved = (moved_bits >> c) & 1u;
    const unsigned bal = __ballot_sync(0xffffffffu, moved);
    if (lane == 0) sh_wcount[wid] = __popc(bal);
    __syncthreads();
    if (tid == 0) {
      int acc = 0;
      for (int w = 0; w < nw; ++w) {
        sh_woff[w] = acc;
        acc += sh_wcount[w];
      }
      sh_base = acc ? atomicAdd(&ctl->count[parity ^ 1], acc) : 0;
    }
    __syncthreads();
    if (moved) {
      const int pos_in = sh_base + sh_woff[wid] + __popc(bal & ((1u << lane) - 1u));
      L.work[parity ^ 1][pos_in] = wi_pack(ci, s * G + c * B + tid);
    }
    __syncthreads();
  }
  // last block advances the step
  if (tid == 0) {
    if (sh_uzero) atomicAdd(&ctl->stats[ST_UZERO], sh_uzero);
    if (sh_short) atomicAdd(&ctl->stats[ST_SHORT], sh_short);
    __threadfence();
    const int done = atomicAdd(&ctl->done_blocks, 1);
    sh_last = done == L.nswarms_total - 1;
  }
  __syncthreads();
  if (sh_last && tid == 0) {
    __threadfence();
    ctl->count[parity] = 0;
    ctl->grab[parity] = 0;
    ctl->grab[parity ^ 1] = 0;
    ctl->parity = parity ^ 1;
    ctl->done_blocks = 0;
    ctl->step += 1;
    ctl->stats[ST_STEPS] += 1;
    __threadfence();
  }
  if (sh_last && tid < L.ncplx) {
    __threadfence();
    L.cplx[tid].draw_cursor += 1;
  }
}

int gso_launch(const GsoLaunch& L, int threads, cudaStream_t st) {
  // shared: luciferin + reference points of the swarm's glowworms
  const size_t smem = (size_t)SD_MAX_G * 4 * sizeof(double);
  gso_kernel<<<L.nswarms_total, threads, smem, st>>>(L);
  return cudaGetLastError() == cudaSuccess ? SD_OK : SD_ERR_CUDA;
}

// once per context that has such swarms, before any capture: the large kernel's shared memory
int gso_prepare_large() {
  return cudaFuncSetAttribute((const void*)gso_kernel_large, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)((size_t)SD_MAX_GLOWWORMS * 4 * sizeof(double))) == cudaSuccess
             ? SD_OK
             : SD_ERR_CUDA;
}

int gso_launch_large(const GsoLaunch& L, int max_g, cudaStream_t st) {
  // shared: luciferin + reference points of the swarm's glowworms
  const size_t smem = (size_t)max_g * 4 * sizeof(double);
  gso_kernel_large<<<L.nswarms_total, SD_MAX_G, smem, st>>>(L);
  return cudaGetLastError() == cudaSuccess ? SD_OK : SD_ERR_CUDA;
}

// the slerp's correctly rounded functions evaluated on the device (parity checking): fn 0 acos,
// fn 1 sin
__global__ void crmath_eval_kernel(int fn, const double* x, long long n, double* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = fn == 0 ? sd_acos_cr(x[i]) : sd_sin_cr(x[i]);
}

}  // namespace sd

extern "C" int sd_crmath_eval(int device, int fn, const double* x, long long n, double* out) {
  if ((fn != 0 && fn != 1) || n < 0 || (n > 0 && (!x || !out))) return sd::fail(SD_ERR_ARG, "sd_crmath_eval: bad arguments");
  if (n == 0) return SD_OK;
  if (cudaSetDevice(device) != cudaSuccess) return sd::fail(SD_ERR_CUDA, "sd_crmath_eval: bad device");
  double* d = nullptr;
  if (cudaMalloc(&d, (size_t)n * 2 * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return sd::fail(SD_ERR_OOM, "sd_crmath_eval: cudaMalloc failed");
  }
  cudaError_t e = cudaMemcpy(d, x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    sd::crmath_eval_kernel<<<148 * 8, 256>>>(fn, d, n, d + n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d + n, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? SD_OK : sd::fail(SD_ERR_CUDA, std::string("sd_crmath_eval: ") + cudaGetErrorString(e));
}
