// Host runtime behind the C ABI (include/sparkle_b200.h): context, device layout, state,
// draws, the CUDA-graph step driver and stateless scoring.
//
// Replaces the memory management and step loop of cal_gso_tasks_gpu
// (reference source/dock/src/cuda/prepare_gso_task.cu:2479-2972): instead of per-call
// allocation, per-swarm-chunk uploads and a host synchronisation after every step, a context
// keeps everything resident in HBM for its lifetime, and each step is two kernels replayed
// from one captured CUDA graph (score moved poses -> GSO update), with the moved-pose work
// list built on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "sd_internal.h"

namespace sd {

static thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define SD_CUDA(call)                                                                                  \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess)                                                                             \
      return fail(e_ == cudaErrorMemoryAllocation ? SD_ERR_OOM : SD_ERR_CUDA,                           \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                                 \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

struct ComplexHost {
  DevComplex d;          // host copy of the device descriptor
  int nslots = 0;
  int draws_steps = 0;   // columns uploaded
  int draws_used = 0;    // host mirror of draw_cursor
  bool state_set = false;
  std::vector<void*> owned;
};

void key_thresholds_host(double* t) {
  t[0] = 4.9406564584124654e-324;
  for (int m = 1; m < 30; ++m) {
    double lo = 0.0, hi = 226.0;
    for (;;) {
      double mid = 0.5 * (lo + hi);
      if (mid == lo || mid == hi) break;
      if ((int)(std::sqrt(mid) * 2.0 - 1.0) >= m) hi = mid; else lo = mid;
    }
    while ((int)(std::sqrt(std::nextafter(hi, 0.0)) * 2.0 - 1.0) >= m) hi = std::nextafter(hi, 0.0);
    while ((int)(std::sqrt(hi) * 2.0 - 1.0) < m) hi = std::nextafter(hi, 1e300);
    t[m] = hi;
  }
}

// Spatial tiles of 32 receptor atoms: recursive bisection along the widest axis at a multiple
// of 32, so that every tile except possibly the last is full and compact.
void build_tiles(const double* xyz, int n, std::vector<int>& slots) {
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::vector<std::pair<int, int>> stack = {{0, n}};
  std::vector<std::pair<int, int>> leaves;
  while (!stack.empty()) {
    auto [a, b] = stack.back();
    stack.pop_back();
    const int m = b - a;
    if (m <= SD_TILE) {
      leaves.push_back({a, b});
      continue;
    }
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int k = a; k < b; ++k)
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::min(lo[d], xyz[idx[k] * 3 + d]);
        hi[d] = std::max(hi[d], xyz[idx[k] * 3 + d]);
      }
    int ax = 0;
    for (int d = 1; d < 3; ++d)
      if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
    const int ntile = (m + SD_TILE - 1) / SD_TILE;
    const int split = a + SD_TILE * ((ntile + 1) / 2);
    std::nth_element(idx.begin() + a, idx.begin() + split, idx.begin() + b,
                     [&](int u, int v) { return xyz[u * 3 + ax] < xyz[v * 3 + ax]; });
    stack.push_back({split, b});
    stack.push_back({a, split});
  }
  std::sort(leaves.begin(), leaves.end());
  slots.assign((size_t)leaves.size() * SD_TILE, -1);
  for (size_t t = 0; t < leaves.size(); ++t)
    for (int k = leaves[t].first; k < leaves[t].second; ++k) slots[t * SD_TILE + (k - leaves[t].first)] = idx[k];
}

}  // namespace sd

using namespace sd;

struct sd_ctx {
  int device = 0;
  int nsm = 148;
  cudaStream_t stream = nullptr;
  int ncplx = 0;
  int scoring = SD_SCORING_DFIRE;
  int precision = SD_PREC_MIXED;
  sd_gso_params params{};
  std::vector<ComplexHost> cx;
  DevComplex* d_cplx = nullptr;
  DevComplex* d_cplx_scratch = nullptr;
  double* d_table64 = nullptr;
  double* d_tablek = nullptr;   // key-indexed copy [168][168][32] + 32 zeros
  double* d_lj_eps = nullptr;
  double* d_lj_sigma = nullptr;
  StepCtl* d_ctl = nullptr;
  StepCtl* d_ctl_scratch = nullptr;
  int* d_work[2] = {nullptr, nullptr};
  int* d_swarm_map = nullptr;
  double* d_pos_prev = nullptr;  // swarms over SD_MAX_G glowworms: pre-move pose copies
  int total_glowworms = 0;
  int total_swarms = 0;
  int max_nr = 0, max_nl = 0, max_G = 0;
  // stateless scratch
  DevBuf s_pose, s_score, s_ref, s_energy, s_work, s_grad, s_bins;
  // per-CTA global scratch of the spill instantiations (complexes too large for shared memory)
  DevBuf s_spill;
  int smem_optin = 0;      // shared memory a CTA may use on this device (opt-in maximum)
  // step graph
  cudaGraphExec_t graph = nullptr;
  int graph_precision = -1;
  int score_threads = 256;
  int score_grid = 0;
  size_t score_smem = 0;
  bool score_spill = false;  // the last configured scorer launch uses the spill instantiation
  size_t spill_stride = 0;
  // autotuner state (mixed-precision DFIRE kernel variants)
  int mixed_variant = 0;
  bool tuned = false;
  double tune_ms[SD_MAX_VARIANTS] = {};
};

namespace {

int ensure(sd_ctx* c, DevBuf& b, size_t bytes) {
  if (b.bytes >= bytes) return SD_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  SD_CUDA(cudaMalloc(&b.p, bytes));
  b.bytes = bytes;
  (void)c;
  return SD_OK;
}

template <class T>
int upload(sd_ctx* c, ComplexHost& h, const T* src, size_t n, const T** dst) {
  T* p = nullptr;
  SD_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  h.owned.push_back(p);
  if (n) SD_CUDA(cudaMemcpyAsync(p, src, n * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  *dst = p;
  return SD_OK;
}

template <class T>
int alloc_dev(ComplexHost& h, size_t n, T** dst) {
  T* p = nullptr;
  SD_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  h.owned.push_back(p);
  *dst = p;
  return SD_OK;
}

int check_desc(const sd_complex_desc& d, int scoring) {
  if (d.n_rec <= 0 || d.n_lig <= 0) return fail(SD_ERR_ARG, "complex: empty receptor or ligand");
  if (d.n_rec > SD_MAX_REC) return fail(SD_ERR_ARG, "complex: receptor has more than 4,194,304 atoms");
  if (d.n_lig > SD_MAX_LIG) return fail(SD_ERR_ARG, "complex: ligand has more than 65,504 atoms");
  if (d.n_swarms <= 0 || d.n_glowworms <= 0 || d.n_glowworms > SD_MAX_GLOWWORMS)
    return fail(SD_ERR_ARG, "complex: swarms must be > 0 and glowworms in 1..6144");
  if ((long long)d.n_swarms * d.n_glowworms >= (1 << 24))
    return fail(SD_ERR_ARG, "complex: more than 2^24 glowworms");
  if (d.n_modes_rec < 0 || d.n_modes_rec > SD_MAX_MODES || d.n_modes_lig < 0 || d.n_modes_lig > SD_MAX_MODES)
    return fail(SD_ERR_ARG, "complex: ANM modes must be in 0..10");
  if (!d.rec_xyz || !d.lig_xyz || !d.rec_mask || !d.lig_mask || !d.rec_dfire_type || !d.lig_dfire_type)
    return fail(SD_ERR_ARG, "complex: NULL coordinate, mask or type array");
  if ((d.n_modes_rec && !d.rec_modes) || (d.n_modes_lig && !d.lig_modes))
    return fail(SD_ERR_ARG, "complex: NULL mode array");
  for (int i = 0; i < d.n_rec; ++i)
    if (d.rec_dfire_type[i] < 0 || d.rec_dfire_type[i] >= SD_DFIRE_TYPES)
      return fail(SD_ERR_ARG, "complex: receptor DFIRE type out of 0..167");
  for (int i = 0; i < d.n_lig; ++i)
    if (d.lig_dfire_type[i] < 0 || d.lig_dfire_type[i] >= SD_DFIRE_TYPES)
      return fail(SD_ERR_ARG, "complex: ligand DFIRE type out of 0..167");
  for (int i = 0; i < 3 * d.n_rec; ++i)
    if (!std::isfinite(d.rec_xyz[i])) return fail(SD_ERR_NUMERIC, "complex: non-finite receptor coordinate");
  for (int i = 0; i < 3 * d.n_lig; ++i)
    if (!std::isfinite(d.lig_xyz[i])) return fail(SD_ERR_NUMERIC, "complex: non-finite ligand coordinate");
  if (scoring == SD_SCORING_PYDOCK) {
    if (!d.rec_charge || !d.lig_charge || !d.rec_lj_type || !d.lig_lj_type)
      return fail(SD_ERR_ARG, "complex: pyDock scoring needs charges and LJ types");
    for (int i = 0; i < d.n_rec; ++i)
      if (d.rec_lj_type[i] < 0 || d.rec_lj_type[i] >= SD_LJ_TYPES) return fail(SD_ERR_ARG, "complex: LJ type out of 0..19");
    for (int i = 0; i < d.n_lig; ++i)
      if (d.lig_lj_type[i] < 0 || d.lig_lj_type[i] >= SD_LJ_TYPES) return fail(SD_ERR_ARG, "complex: LJ type out of 0..19");
  }
  return SD_OK;
}

float round_up_f(double v) {
  float f = (float)v;
  if ((double)f < v) f = std::nextafter(f, 3.0e38f);
  return f;
}

int setup_complex(sd_ctx* c, const sd_complex_desc& d, ComplexHost& h, int gbase, int sbase) {
  DevComplex& D = h.d;
  memset(&D, 0, sizeof D);
  D.nr = d.n_rec;
  D.nl = d.n_lig;
  D.nmr = d.n_modes_rec;
  D.nml = d.n_modes_lig;
  D.S = d.n_swarms;
  D.G = d.n_glowworms;
  D.pl = SD_POSE_LEN(d.n_modes_rec, d.n_modes_lig);
  D.gbase = gbase;
  D.sbase = sbase;
  for (int k = 0; k < 3; ++k) D.lig_ref[k] = d.lig_ref_point[k];

  // receptor tiles
  std::vector<int> slots;
  build_tiles(d.rec_xyz, d.n_rec, slots);
  const int nslots = (int)slots.size();
  D.ntiles = nslots / SD_TILE;
  h.nslots = nslots;
  std::vector<double> rxyz((size_t)nslots * 3, 0.0), rmodes((size_t)std::max(1, D.nmr) * nslots * 3, 0.0);
  std::vector<int> rmask(nslots, 0), rrow(nslots, 0), rrowk(nslots, 0), rlj(nslots, 0);
  std::vector<float> rq(nslots, 0.f);
  std::vector<float4> tiles(D.ntiles);
  for (int s = 0; s < nslots; ++s) {
    const int i = slots[s];
    if (i < 0) continue;
    for (int k = 0; k < 3; ++k) rxyz[(size_t)s * 3 + k] = d.rec_xyz[(size_t)i * 3 + k];
    for (int m = 0; m < D.nmr; ++m)
      for (int k = 0; k < 3; ++k)
        rmodes[((size_t)m * nslots + s) * 3 + k] = d.rec_modes[((size_t)m * d.n_rec + i) * 3 + k];
    rmask[s] = d.rec_mask[i];
    rrow[s] = d.rec_dfire_type[i] * SD_ROW;
    rrowk[s] = d.rec_dfire_type[i] * SD_ROWK;
    if (d.rec_charge) rq[s] = (float)d.rec_charge[i];
    if (d.rec_lj_type) rlj[s] = d.rec_lj_type[i];
  }
  for (int t = 0; t < D.ntiles; ++t) {
    double ctr[3] = {0, 0, 0};
    int cnt = 0;
    for (int l = 0; l < SD_TILE; ++l) {
      const int i = slots[t * SD_TILE + l];
      if (i < 0) continue;
      for (int k = 0; k < 3; ++k) ctr[k] += d.rec_xyz[(size_t)i * 3 + k];
      ++cnt;
    }
    float cf[3];
    for (int k = 0; k < 3; ++k) cf[k] = (float)(ctr[k] / std::max(cnt, 1));
    double rad = 0;
    for (int l = 0; l < SD_TILE; ++l) {
      const int i = slots[t * SD_TILE + l];
      if (i < 0) continue;
      double s2 = 0;
      for (int k = 0; k < 3; ++k) {
        const double dd = d.rec_xyz[(size_t)i * 3 + k] - (double)cf[k];
        s2 += dd * dd;
      }
      rad = std::max(rad, std::sqrt(s2));
    }
    tiles[t] = make_float4(cf[0], cf[1], cf[2], round_up_f(rad * (1 + 1e-6) + 1e-4));
  }
  // per-mode maximal atom displacement per unit extent (masked atoms only)
  for (int m = 0; m < D.nmr; ++m) {
    double mx = 0;
    for (int i = 0; i < d.n_rec; ++i) {
      if (d.rec_mask[i] != 1) continue;
      const double* M = d.rec_modes + ((size_t)m * d.n_rec + i) * 3;
      mx = std::max(mx, std::sqrt(M[0] * M[0] + M[1] * M[1] + M[2] * M[2]));
    }
    D.mnorm_r[m] = round_up_f(mx * (1 + 1e-6) + 1e-7);
  }
  for (int m = 0; m < D.nml; ++m) {
    double mx = 0;
    for (int i = 0; i < d.n_lig; ++i) {
      if (d.lig_mask[i] != 1) continue;
      const double* M = d.lig_modes + ((size_t)m * d.n_lig + i) * 3;
      mx = std::max(mx, std::sqrt(M[0] * M[0] + M[1] * M[1] + M[2] * M[2]));
    }
    D.mnorm_l[m] = round_up_f(mx * (1 + 1e-6) + 1e-7);
  }
  double lr = 0;
  for (int i = 0; i < d.n_lig; ++i) {
    const double* p = d.lig_xyz + (size_t)i * 3;
    lr = std::max(lr, std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]));
  }
  D.lig_radius = round_up_f(lr * (1 + 1e-6) + 1e-4);

  int rc;
  if ((rc = upload(c, h, slots.data(), slots.size(), &D.r_orig))) return rc;
  if ((rc = upload(c, h, rxyz.data(), rxyz.size(), &D.r_xyz))) return rc;
  if ((rc = upload(c, h, rmodes.data(), rmodes.size(), &D.r_modes))) return rc;
  if ((rc = upload(c, h, rmask.data(), rmask.size(), &D.r_mask))) return rc;
  if ((rc = upload(c, h, rrow.data(), rrow.size(), &D.r_row))) return rc;
  if ((rc = upload(c, h, rrowk.data(), rrowk.size(), &D.r_rowk))) return rc;
  if ((rc = upload(c, h, tiles.data(), tiles.size(), &D.r_tile))) return rc;
  if ((rc = upload(c, h, rq.data(), rq.size(), &D.r_q))) return rc;
  if ((rc = upload(c, h, rlj.data(), rlj.size(), &D.r_lj))) return rc;

  // ligand chunks (spatial order) for the mixed-precision kernel
  {
    std::vector<int> lslots;
    build_tiles(d.lig_xyz, d.n_lig, lslots);
    D.nlchunks = (int)lslots.size() / SD_TILE;
    std::vector<float4> lch(D.nlchunks);
    for (int t = 0; t < D.nlchunks; ++t) {
      double ctr[3] = {0, 0, 0};
      int cnt = 0;
      for (int l = 0; l < SD_TILE; ++l) {
        const int j = lslots[t * SD_TILE + l];
        if (j < 0) continue;
        for (int k = 0; k < 3; ++k) ctr[k] += d.lig_xyz[(size_t)j * 3 + k];
        ++cnt;
      }
      float cf[3];
      for (int k = 0; k < 3; ++k) cf[k] = (float)(ctr[k] / std::max(cnt, 1));
      double rad = 0;
      for (int l = 0; l < SD_TILE; ++l) {
        const int j = lslots[t * SD_TILE + l];
        if (j < 0) continue;
        double s2 = 0;
        for (int k = 0; k < 3; ++k) {
          const double dd = d.lig_xyz[(size_t)j * 3 + k] - (double)cf[k];
          s2 += dd * dd;
        }
        rad = std::max(rad, std::sqrt(s2));
      }
      lch[t] = make_float4(cf[0], cf[1], cf[2], round_up_f(rad * (1 + 1e-6) + 1e-4));
    }
    const size_t nls = lslots.size();
    std::vector<double> cxyz(nls * 3, 0.0), cmodes((size_t)std::max(1, D.nml) * nls * 3, 0.0);
    std::vector<int> cmask(nls, 0), ccolk(nls, 0);
    for (size_t s = 0; s < nls; ++s) {
      const int j = lslots[s];
      if (j < 0) continue;
      for (int k = 0; k < 3; ++k) cxyz[s * 3 + k] = d.lig_xyz[(size_t)j * 3 + k];
      for (int m = 0; m < D.nml; ++m)
        for (int k = 0; k < 3; ++k) cmodes[((size_t)m * nls + s) * 3 + k] = d.lig_modes[((size_t)m * d.n_lig + j) * 3 + k];
      cmask[s] = d.lig_mask[j];
      ccolk[s] = d.lig_dfire_type[j] * SD_KEYS;
    }
    double lc[3] = {0, 0, 0};
    for (int j = 0; j < d.n_lig; ++j)
      for (int k = 0; k < 3; ++k) lc[k] += d.lig_xyz[(size_t)j * 3 + k];
    for (int k = 0; k < 3; ++k) D.lig_ctr[k] = (float)(lc[k] / std::max(1, d.n_lig));
    int rc2;
    if ((rc2 = upload(c, h, lslots.data(), lslots.size(), &D.l_perm))) return rc2;
    if ((rc2 = upload(c, h, lch.data(), lch.size(), &D.l_chunk))) return rc2;
    if ((rc2 = upload(c, h, cxyz.data(), cxyz.size(), &D.lc_xyz))) return rc2;
    if ((rc2 = upload(c, h, cmodes.data(), cmodes.size(), &D.lc_modes))) return rc2;
    if ((rc2 = upload(c, h, cmask.data(), cmask.size(), &D.lc_mask))) return rc2;
    if ((rc2 = upload(c, h, ccolk.data(), ccolk.size(), &D.lc_colk))) return rc2;
  }
  std::vector<int> lcol(d.n_lig), llj(d.n_lig, 0);
  std::vector<float> lq(d.n_lig, 0.f);
  for (int j = 0; j < d.n_lig; ++j) {
    lcol[j] = d.lig_dfire_type[j] * SD_DFIRE_BINS;
    if (d.lig_charge) lq[j] = (float)d.lig_charge[j];
    if (d.lig_lj_type) llj[j] = d.lig_lj_type[j];
  }
  if ((rc = upload(c, h, d.lig_xyz, (size_t)d.n_lig * 3, &D.l_xyz))) return rc;
  if ((rc = upload(c, h, d.lig_modes, (size_t)D.nml * d.n_lig * 3, &D.l_modes))) return rc;
  if ((rc = upload(c, h, d.lig_mask, (size_t)d.n_lig, &D.l_mask))) return rc;
  if ((rc = upload(c, h, lcol.data(), lcol.size(), &D.l_col))) return rc;
  if ((rc = upload(c, h, lq.data(), lq.size(), &D.l_q))) return rc;
  if ((rc = upload(c, h, llj.data(), llj.size(), &D.l_lj))) return rc;

  const size_t n = (size_t)D.S * D.G;
  if ((rc = alloc_dev(h, n * D.pl, &D.pos))) return rc;
  if ((rc = alloc_dev(h, n, &D.scoring))) return rc;
  if ((rc = alloc_dev(h, n, &D.luciferin))) return rc;
  if ((rc = alloc_dev(h, n, &D.vision))) return rc;
  if ((rc = alloc_dev(h, n, &D.step))) return rc;
  if ((rc = alloc_dev(h, n, &D.moved))) return rc;
  if ((rc = alloc_dev(h, n, &D.nnei))) return rc;
  if ((rc = alloc_dev(h, n, &D.select))) return rc;
  if ((rc = alloc_dev(h, n * 3, &D.ref))) return rc;
  SD_CUDA(cudaMemsetAsync(D.scoring, 0, n * sizeof(double), c->stream));
  SD_CUDA(cudaMemsetAsync(D.ref, 0, n * 3 * sizeof(double), c->stream));
  D.draws = nullptr;
  D.draw_steps = 0;
  D.draw_cursor = 0;
  return SD_OK;
}

int push_descriptors(sd_ctx* c) {
  std::vector<DevComplex> v(c->ncplx);
  for (int i = 0; i < c->ncplx; ++i) v[i] = c->cx[i].d;
  SD_CUDA(cudaMemcpyAsync(c->d_cplx, v.data(), sizeof(DevComplex) * c->ncplx, cudaMemcpyHostToDevice, c->stream));
  return SD_OK;
}

// rebuild the first work list from moved/step of every complex
int rebuild_worklist(sd_ctx* c) {
  std::vector<int> work;
  work.reserve(c->total_glowworms);
  for (int ci = 0; ci < c->ncplx; ++ci) {
    const DevComplex& D = c->cx[ci].d;
    const size_t n = (size_t)D.S * D.G;
    std::vector<int> moved(n), step(n);
    SD_CUDA(cudaMemcpyAsync(moved.data(), D.moved, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    SD_CUDA(cudaMemcpyAsync(step.data(), D.step, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    SD_CUDA(cudaStreamSynchronize(c->stream));
    for (size_t k = 0; k < n; ++k)
      if (moved[k] || step[k] == 0) work.push_back(wi_pack(ci, (int)k));
  }
  StepCtl ctl;
  SD_CUDA(cudaMemcpy(&ctl, c->d_ctl, sizeof ctl, cudaMemcpyDeviceToHost));
  ctl.count[0] = (int)work.size();
  ctl.count[1] = 0;
  ctl.grab[0] = ctl.grab[1] = 0;
  ctl.parity = 0;
  ctl.done_blocks = 0;
  if (!work.empty())
    SD_CUDA(cudaMemcpyAsync(c->d_work[0], work.data(), work.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(c->d_ctl, &ctl, sizeof ctl, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaStreamSynchronize(c->stream));
  return SD_OK;
}

// The spill scratch, grown to at least bytes.  The step graph holds the scratch's address, so a new
// scratch means a new capture at the next step.
int grow_spill(sd_ctx* c, size_t bytes) {
  if (c->s_spill.bytes >= bytes) return SD_OK;
  if (c->graph) {
    cudaStreamSynchronize(c->stream);
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  return ensure(c, c->s_spill, bytes);
}

// Launch shape of the scorer on this context: persistent grid (resident CTAs x SMs), dynamic shared
// memory, threads.  When the per-pose arrays of the largest complex do not fit in the shared memory
// a CTA may use, the spill instantiation is chosen (no dynamic shared memory) and the context's
// spill scratch is sized to grid x per-CTA bytes; alloc = false refuses that instead of allocating.
int configure_score_v(sd_ctx* c, int precision, int variant, int* grid, size_t* smem, bool alloc = true) {
  const size_t need = score_smem_bytes(precision, c->scoring, c->max_nr, c->max_nl, variant);
  const void* k = score_kernel_ptr(precision, c->scoring, variant, false);
  cudaFuncAttributes fa;
  SD_CUDA(cudaFuncGetAttributes(&fa, k));
  const bool spill = need + fa.sharedSizeBytes > (size_t)c->smem_optin;
  size_t sm = need;
  int threads = score_threads_of(precision, c->scoring, variant);
  if (spill) {
    k = score_kernel_ptr(precision, c->scoring, variant, true);
    sm = 0;
    threads = score_threads_spill(precision, c->scoring);
  }
  SD_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(sm, 1)));
  int per_sm = 0;
  SD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, sm));
  if (per_sm < 1) return fail(SD_ERR_ARG, "scoring kernel does not fit on an SM (shared memory)");
  *grid = per_sm * c->nsm;
  *smem = sm;
  c->score_threads = threads;
  c->score_spill = spill;
  if (spill) {
    const size_t stride = (need + 255) & ~(size_t)255;
    if (c->s_spill.bytes < stride * (size_t)*grid) {
      if (!alloc) return fail(SD_ERR_NOTSUP, "complex too large for shared memory: its scorer needs the context's "
                                             "global scratch, which this call may not allocate");
      int rc = grow_spill(c, stride * (size_t)*grid);
      if (rc) return rc;
    }
    c->spill_stride = stride;
  }
  return SD_OK;
}

int configure_score(sd_ctx* c, int precision, int* grid, size_t* smem, bool alloc = true) {
  return configure_score_v(c, precision, c->mixed_variant, grid, smem, alloc);
}

// the spill scratch of the last configured launch (null pointers when it uses shared memory)
void set_spill(const sd_ctx* c, ScoreLaunch& L) {
  L.spill = c->score_spill ? (unsigned char*)c->s_spill.p : nullptr;
  L.spill_stride = c->score_spill ? c->spill_stride : 0;
}

// Autotuner: times every compiled variant of the mixed DFIRE kernel (warps per CTA x resident
// CTAs per SM) on up to 16384 of the context's current poses, three times each, keeps the fastest
// for this context.  Results are cached per (device, largest receptor, largest ligand).
// SPARKLE_TUNE=0 keeps the default variant; SPARKLE_MIXED_VARIANT=k forces variant k.
int autotune_mixed(sd_ctx* c) {
  c->tuned = true;
  const int nv = mixed_variant_count();
  if (const char* f = getenv("SPARKLE_MIXED_VARIANT")) {
    const int v = atoi(f);
    if (v >= 0 && v < nv) c->mixed_variant = v;
    return SD_OK;
  }
  if (const char* t = getenv("SPARKLE_TUNE"))
    if (atoi(t) == 0) return SD_OK;
  struct Key {
    int dev, nr, nl;
  };
  static std::vector<std::pair<Key, int>> cache;
  for (auto& e : cache)
    if (e.first.dev == c->device && e.first.nr == c->max_nr && e.first.nl == c->max_nl) {
      c->mixed_variant = e.second;
      return SD_OK;
    }
  // sample poses of every complex into the stateless scratch
  const int per = std::max(1, 16384 / c->ncplx);
  std::vector<int> counts(c->ncplx), offs(c->ncplx);
  int total = 0;
  size_t pos_bytes = 0;
  for (int ci = 0; ci < c->ncplx; ++ci) {
    const DevComplex& D = c->cx[ci].d;
    counts[ci] = std::min(per, D.S * D.G);
    offs[ci] = total;
    total += counts[ci];
    pos_bytes = std::max(pos_bytes, (size_t)D.pl * 8);
  }
  int rc;
  if ((rc = ensure(c, c->s_pose, (size_t)total * pos_bytes))) return rc;
  if ((rc = ensure(c, c->s_score, (size_t)total * 8))) return rc;
  if ((rc = ensure(c, c->s_energy, (size_t)total * 8))) return rc;
  if ((rc = ensure(c, c->s_ref, (size_t)total * 24))) return rc;
  if ((rc = ensure(c, c->s_work, (size_t)total * 4))) return rc;
  std::vector<int> work(total);
  std::vector<DevComplex> scratch(c->ncplx);
  for (int ci = 0; ci < c->ncplx; ++ci) {
    const DevComplex& D = c->cx[ci].d;
    DevComplex S = D;
    S.pos = (double*)((char*)c->s_pose.p + (size_t)offs[ci] * pos_bytes);
    S.scoring = (double*)c->s_score.p + offs[ci];
    S.ref = (double*)c->s_ref.p + 3 * (size_t)offs[ci];
    scratch[ci] = S;
    SD_CUDA(cudaMemcpyAsync(S.pos, D.pos, (size_t)counts[ci] * D.pl * 8, cudaMemcpyDeviceToDevice, c->stream));
    for (int i = 0; i < counts[ci]; ++i) work[offs[ci] + i] = wi_pack(ci, i);
  }
  SD_CUDA(cudaMemcpyAsync(c->d_cplx_scratch, scratch.data(), sizeof(DevComplex) * c->ncplx, cudaMemcpyHostToDevice,
                          c->stream));
  SD_CUDA(cudaMemcpyAsync(c->s_work.p, work.data(), (size_t)total * 4, cudaMemcpyHostToDevice, c->stream));
  StepCtl ctl;
  SD_CUDA(cudaStreamSynchronize(c->stream));
  SD_CUDA(cudaMemcpy(&ctl, c->d_ctl_scratch, sizeof ctl, cudaMemcpyDeviceToHost));
  ctl.count[0] = total;
  ctl.count[1] = 0;
  ctl.parity = 0;
  ScoreLaunch L{};
  L.cplx = c->d_cplx_scratch;
  L.ctl = c->d_ctl_scratch;
  L.work[0] = L.work[1] = (const int*)c->s_work.p;
  L.table64 = c->d_table64;
  L.tablek = c->d_tablek;
  L.lj_eps = c->d_lj_eps;
  L.lj_sigma = c->d_lj_sigma;
  cudaEvent_t e0, e1;
  SD_CUDA(cudaEventCreate(&e0));
  SD_CUDA(cudaEventCreate(&e1));
  int best = 0;
  double best_ms = 1e300;
  for (int v = 0; v < nv && v < SD_MAX_VARIANTS; ++v) {
    int grid;
    size_t sm;
    if (configure_score_v(c, SD_PREC_MIXED, v, &grid, &sm) != SD_OK) {
      c->tune_ms[v] = -1;
      continue;
    }
    if (c->score_spill) {
      // too large for shared memory: one spill instantiation, nothing to choose
      c->tune_ms[v] = -1;
      break;
    }
    double vbest = 1e300;
    for (int rep = 0; rep < 3; ++rep) {
      ctl.grab[0] = ctl.grab[1] = 0;
      SD_CUDA(cudaMemcpyAsync(c->d_ctl_scratch, &ctl, sizeof ctl, cudaMemcpyHostToDevice, c->stream));
      SD_CUDA(cudaEventRecord(e0, c->stream));
      if ((rc = score_launch(L, SD_PREC_MIXED, c->scoring, grid, c->score_threads, sm, c->stream, v, false)))
        return fail(rc, std::string("autotune launch: ") + cudaGetErrorString(cudaGetLastError()));
      SD_CUDA(cudaEventRecord(e1, c->stream));
      SD_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      SD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      vbest = std::min(vbest, (double)ms);
    }
    c->tune_ms[v] = vbest;
    if (vbest < best_ms) {
      best_ms = vbest;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->mixed_variant = best;
  cache.push_back({Key{c->device, c->max_nr, c->max_nl}, best});
  return SD_OK;
}

int enqueue_step(sd_ctx* c, int precision, int grid, size_t sm) {
  int rc;
  ScoreLaunch L{};
  L.cplx = c->d_cplx;
  L.ctl = c->d_ctl;
  L.work[0] = c->d_work[0];
  L.work[1] = c->d_work[1];
  L.table64 = c->d_table64;
  L.tablek = c->d_tablek;
  L.lj_eps = c->d_lj_eps;
  L.lj_sigma = c->d_lj_sigma;
  L.energy_out = nullptr;
  set_spill(c, L);
  if ((rc = score_launch(L, precision, c->scoring, grid, c->score_threads, sm, c->stream, c->mixed_variant,
                         c->score_spill)))
    return fail(rc, std::string("score kernel launch: ") + cudaGetErrorString(cudaGetLastError()));
  GsoLaunch G{};
  G.cplx = c->d_cplx;
  G.ctl = c->d_ctl;
  G.work[0] = c->d_work[0];
  G.work[1] = c->d_work[1];
  G.swarm_map = c->d_swarm_map;
  G.nswarms_total = c->total_swarms;
  G.ncplx = c->ncplx;
  G.p.rho = c->params.rho;
  G.p.gamma = c->params.gamma;
  G.p.beta = c->params.beta;
  G.p.max_vision = c->params.max_vision_range;
  G.p.step_t = c->params.translation_step;
  G.p.step_r = c->params.rotation_step;
  G.p.step_nm = c->params.nmodes_step;
  G.p.max_neighbors = c->params.max_neighbors;
  G.pos_prev = c->d_pos_prev;
  const int threads = (c->max_G + 31) / 32 * 32;
  if ((rc = c->max_G > SD_MAX_G ? gso_launch_large(G, c->max_G, c->stream) : gso_launch(G, threads, c->stream)))
    return fail(rc, std::string("GSO kernel launch: ") + cudaGetErrorString(cudaGetLastError()));
  return SD_OK;
}

}  // namespace

namespace sd {
// Read-only view of a context for sd_score_poses_noalloc (sd_noalloc.cu): the device
// descriptor of one complex, table pointers and the launch shape of the scoring kernel.
// Makes the context's device current; allocates nothing.
int ctx_noalloc_view(sd_ctx* c, int ci, int precision, DevComplex* desc, ScoreLaunch* L, int* grid, size_t* smem,
                     int* device, cudaStream_t* stream, int* scoring, int* variant) {
  if (!c || ci < 0 || ci >= c->ncplx) return fail(SD_ERR_ARG, "sd_score_poses_noalloc: bad context or complex");
  if (precision < SD_PREC_FP64_REF || precision > SD_PREC_MIXED)
    return fail(SD_ERR_ARG, "sd_score_poses_noalloc: unknown precision");
  SD_CUDA(cudaSetDevice(c->device));
  // a complex too large for shared memory uses the context's spill scratch, allocated by an
  // earlier allocating call; this call only uses it when it is already large enough
  int rc = configure_score(c, precision, grid, smem, false);
  if (rc) return rc;
  *desc = c->cx[ci].d;
  memset(L, 0, sizeof *L);
  set_spill(c, *L);
  L->table64 = c->d_table64;
  L->tablek = c->d_tablek;
  L->lj_eps = c->d_lj_eps;
  L->lj_sigma = c->d_lj_sigma;
  *device = c->device;
  *stream = c->stream;
  *scoring = c->scoring;
  *variant = c->mixed_variant;
  return SD_OK;
}
}  // namespace sd

extern "C" {

const char* sd_last_error(void) { return g_err.c_str(); }
const char* sd_version(void) { return "sparkle_b200 0.1 (sm_100a)"; }

int sd_device_count(int* n) {
  if (!n) return fail(SD_ERR_ARG, "sd_device_count: NULL");
  int k = 0;
  if (cudaGetDeviceCount(&k) != cudaSuccess) k = 0;
  cudaGetLastError();
  *n = k;
  return SD_OK;
}

int sd_ctx_create(const sd_complex_desc* complexes, int n_complexes, const sd_tables* tables,
                  const sd_gso_params* params, int scoring, int precision, int device, sd_ctx** out) {
  sd::NvtxRange nvtx_range("sd_ctx_create");
  if (!out) return fail(SD_ERR_ARG, "sd_ctx_create: out is NULL");
  *out = nullptr;
  if (!complexes || n_complexes <= 0 || n_complexes > SD_MAX_COMPLEX)
    return fail(SD_ERR_ARG, "sd_ctx_create: need 1..32 complexes");
  if (!tables || !tables->dfire_energy) return fail(SD_ERR_ARG, "sd_ctx_create: DFIRE table required");
  if (scoring != SD_SCORING_DFIRE && scoring != SD_SCORING_PYDOCK)
    return fail(SD_ERR_ARG, "sd_ctx_create: unknown scoring function");
  if (scoring == SD_SCORING_PYDOCK && (!tables->lj_eps || !tables->lj_sigma))
    return fail(SD_ERR_ARG, "sd_ctx_create: pyDock scoring needs LJ tables");
  if (precision < SD_PREC_FP64_REF || precision > SD_PREC_MIXED)
    return fail(SD_ERR_ARG, "sd_ctx_create: unknown precision");
  for (int i = 0; i < n_complexes; ++i) {
    int rc = check_desc(complexes[i], scoring);
    if (rc) return rc;
  }
  // device memory the context will hold (tables, per-complex data, state, work lists), checked
  // against SPARKLE_DEVICE_BUDGET_MB when set (a forced budget, e.g. to test the OOM path)
  {
    size_t bytes = (size_t)(SD_TABLE_SIZE + 32) * 12 + (size_t)(SD_TABLE_KEYS + 32) * 8 + 4096;
    for (int i = 0; i < n_complexes; ++i) {
      const sd_complex_desc& d = complexes[i];
      const size_t nr = (size_t)((d.n_rec + SD_TILE - 1) / SD_TILE) * SD_TILE, nl = (size_t)d.n_lig;
      const size_t n = (size_t)d.n_swarms * d.n_glowworms, pl = SD_POSE_LEN(d.n_modes_rec, d.n_modes_lig);
      bytes += nr * (24 + 24 * d.n_modes_rec + 20) + nl * (24 + 24 * d.n_modes_lig + 20) * 2;
      bytes += n * (8 * pl + 8 * 3 + 4 * 4 + 24 + 8);
    }
    if (const char* b = getenv("SPARKLE_DEVICE_BUDGET_MB")) {
      const double budget = atof(b) * 1048576.0;
      if ((double)bytes > budget)
        return fail(SD_ERR_OOM, "sd_ctx_create: needs about " + std::to_string(bytes >> 20) +
                                    " MiB of device memory, over SPARKLE_DEVICE_BUDGET_MB=" + b);
    }
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(SD_ERR_CUDA, "sd_ctx_create: no CUDA device");
  }
  if (device < 0 || device >= ndev) return fail(SD_ERR_ARG, "sd_ctx_create: bad device index");
  SD_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  SD_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) return fail(SD_ERR_NOTSUP, "sd_ctx_create: needs a Blackwell (sm_100) GPU");

  sd_ctx* c = new sd_ctx();
  c->device = device;
  c->nsm = prop.multiProcessorCount;
  c->smem_optin = (int)prop.sharedMemPerBlockOptin;
  c->ncplx = n_complexes;
  c->scoring = scoring;
  c->precision = precision;
  if (params) c->params = *params; else sd_gso_params_default(&c->params);
  auto bail = [&](int rc) {
    sd_ctx_destroy(c);
    return rc;
  };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(SD_ERR_CUDA, "cudaStreamCreate failed"));
  double T[30];
  key_thresholds_host(T);
  set_key_thresholds(T);
  c->cx.resize(n_complexes);
  int gbase = 0, sbase = 0;
  for (int i = 0; i < n_complexes; ++i) {
    int rc = setup_complex(c, complexes[i], c->cx[i], gbase, sbase);
    if (rc) return bail(rc);
    gbase += complexes[i].n_swarms * complexes[i].n_glowworms;
    sbase += complexes[i].n_swarms;
    c->max_nr = std::max(c->max_nr, complexes[i].n_rec);
    c->max_nl = std::max(c->max_nl, complexes[i].n_lig);
    c->max_G = std::max(c->max_G, complexes[i].n_glowworms);
  }
  c->total_glowworms = gbase;
  c->total_swarms = sbase;
  auto cu = [&](cudaError_t e, const char* what) {
    if (e == cudaSuccess) return SD_OK;
    return fail(e == cudaErrorMemoryAllocation ? SD_ERR_OOM : SD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  int rc;
  if ((rc = cu(cudaMalloc(&c->d_cplx, sizeof(DevComplex) * n_complexes), "cudaMalloc"))) return bail(rc);
  if ((rc = cu(cudaMalloc(&c->d_cplx_scratch, sizeof(DevComplex) * n_complexes), "cudaMalloc"))) return bail(rc);
  if ((rc = cu(cudaMalloc(&c->d_table64, sizeof(double) * (SD_TABLE_SIZE + 32)), "cudaMalloc"))) return bail(rc);
  if ((rc = cu(cudaMalloc(&c->d_tablek, sizeof(double) * (SD_TABLE_KEYS + 32)), "cudaMalloc"))) return bail(rc);
  if ((rc = cu(cudaMalloc(&c->d_lj_eps, sizeof(double) * SD_LJ_TYPES), "cudaMalloc"))) return bail(rc);
  if ((rc = cu(cudaMalloc(&c->d_lj_sigma, sizeof(double) * SD_LJ_TYPES), "cudaMalloc"))) return bail(rc);
  if ((rc = cu(cudaMalloc(&c->d_ctl, sizeof(StepCtl)), "cudaMalloc"))) return bail(rc);
  if ((rc = cu(cudaMalloc(&c->d_ctl_scratch, sizeof(StepCtl)), "cudaMalloc"))) return bail(rc);
  for (int p = 0; p < 2; ++p)
    if ((rc = cu(cudaMalloc(&c->d_work[p], sizeof(int) * std::max(1, c->total_glowworms)), "cudaMalloc"))) return bail(rc);
  if ((rc = cu(cudaMalloc(&c->d_swarm_map, sizeof(int) * c->total_swarms), "cudaMalloc"))) return bail(rc);
  if (c->max_G > SD_MAX_G) {
    if ((rc = cu(cudaMalloc(&c->d_pos_prev, sizeof(double) * SD_POSE_LEN(SD_MAX_MODES, SD_MAX_MODES) *
                                               (size_t)c->total_glowworms), "cudaMalloc")))
      return bail(rc);
    if ((rc = gso_prepare_large())) return bail(fail(rc, "large-swarm GSO kernel: shared memory attribute"));
  }
  {
    std::vector<double> t64(SD_TABLE_SIZE + 32, 0.0);
    for (int i = 0; i < SD_TABLE_SIZE; ++i) {
      if (!std::isfinite(tables->dfire_energy[i])) return bail(fail(SD_ERR_NUMERIC, "non-finite DFIRE table entry"));
      t64[i] = tables->dfire_energy[i];
    }
    // key-indexed copy: entry [tR][tL][k] is what the reference reads for key k, the flat index
    // tR*3360 + tL*20 + dist_to_bins[k]-1 (key 29, d^2 == 225, reads bin 20: the next ligand
    // type's bin 0, or the zero padding after the last type pair)
    static const int kBin[30] = {0, 0, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 13, 14, 14, 15, 15, 16, 16, 17, 17, 18, 18, 19, 19, 20};
    std::vector<double> tk((size_t)SD_TABLE_KEYS + 32, 0.0);
    for (int a = 0; a < SD_DFIRE_TYPES; ++a)
      for (int b = 0; b < SD_DFIRE_TYPES; ++b)
        for (int k = 0; k < 30; ++k)
          tk[(size_t)a * SD_ROWK + b * SD_KEYS + k] = t64[(size_t)a * SD_ROW + b * SD_DFIRE_BINS + kBin[k]];
    std::vector<double> eps(SD_LJ_TYPES, 0.0), sig(SD_LJ_TYPES, 0.0);
    if (tables->lj_eps && tables->lj_sigma)
      for (int i = 0; i < SD_LJ_TYPES; ++i) {
        eps[i] = tables->lj_eps[i];
        sig[i] = tables->lj_sigma[i];
      }
    std::vector<int> smap(c->total_swarms);
    for (int ci = 0, s0 = 0; ci < n_complexes; ++ci)
      for (int s = 0; s < complexes[ci].n_swarms; ++s) smap[s0++] = wi_pack(ci, s);
    StepCtl ctl;
    memset(&ctl, 0, sizeof ctl);
    if ((rc = cu(cudaMemcpy(c->d_table64, t64.data(), t64.size() * 8, cudaMemcpyHostToDevice), "upload"))) return bail(rc);
    if ((rc = cu(cudaMemcpy(c->d_tablek, tk.data(), tk.size() * 8, cudaMemcpyHostToDevice), "upload"))) return bail(rc);
    if ((rc = cu(cudaMemcpy(c->d_lj_eps, eps.data(), eps.size() * 8, cudaMemcpyHostToDevice), "upload"))) return bail(rc);
    if ((rc = cu(cudaMemcpy(c->d_lj_sigma, sig.data(), sig.size() * 8, cudaMemcpyHostToDevice), "upload"))) return bail(rc);
    if ((rc = cu(cudaMemcpy(c->d_swarm_map, smap.data(), smap.size() * 4, cudaMemcpyHostToDevice), "upload"))) return bail(rc);
    if ((rc = cu(cudaMemcpy(c->d_ctl, &ctl, sizeof ctl, cudaMemcpyHostToDevice), "upload"))) return bail(rc);
  }
  if ((rc = push_descriptors(c))) return bail(rc);
  if ((rc = cu(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize"))) return bail(rc);
  *out = c;
  return SD_OK;
}

int sd_ctx_destroy(sd_ctx* c) {
  if (!c) return SD_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->graph) cudaGraphExecDestroy(c->graph);
  for (auto& h : c->cx)
    for (void* p : h.owned) cudaFree(p);
  void* ps[] = {c->d_cplx, c->d_cplx_scratch, c->d_table64, c->d_tablek, c->d_lj_eps, c->d_lj_sigma, c->d_ctl,
                c->d_ctl_scratch, c->d_work[0], c->d_work[1], c->d_swarm_map, c->d_pos_prev, c->s_pose.p, c->s_score.p,
                c->s_ref.p, c->s_energy.p, c->s_work.p, c->s_grad.p, c->s_bins.p, c->s_spill.p};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return SD_OK;
}

int sd_ctx_stream(sd_ctx* c, void** s) {
  if (!c || !s) return fail(SD_ERR_ARG, "sd_ctx_stream: NULL");
  *s = (void*)c->stream;
  return SD_OK;
}

int sd_pose_len(const sd_ctx* c, int ci, int* pl) {
  if (!c || !pl || ci < 0 || ci >= c->ncplx) return fail(SD_ERR_ARG, "sd_pose_len: bad arguments");
  *pl = c->cx[ci].d.pl;
  return SD_OK;
}

int sd_init_state(sd_ctx* c, int ci, const double* pos) {
  if (!c || !pos || ci < 0 || ci >= c->ncplx) return fail(SD_ERR_ARG, "sd_init_state: bad arguments");
  SD_CUDA(cudaSetDevice(c->device));
  const DevComplex& D = c->cx[ci].d;
  const size_t n = (size_t)D.S * D.G;
  for (size_t i = 0; i < n * D.pl; ++i)
    if (!std::isfinite(pos[i])) return fail(SD_ERR_NUMERIC, "sd_init_state: non-finite pose");
  std::vector<double> luc(n, c->params.initial_luciferin), vis(n, c->params.initial_vision_range), zero(n, 0.0);
  std::vector<int> izero(n, 0), sel(n);
  for (size_t k = 0; k < n; ++k) sel[k] = (int)(k % D.G);
  SD_CUDA(cudaMemcpyAsync(D.pos, pos, n * D.pl * 8, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.luciferin, luc.data(), n * 8, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.vision, vis.data(), n * 8, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.scoring, zero.data(), n * 8, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemsetAsync(D.ref, 0, n * 3 * 8, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.step, izero.data(), n * 4, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.moved, izero.data(), n * 4, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.nnei, izero.data(), n * 4, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.select, sel.data(), n * 4, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaStreamSynchronize(c->stream));
  c->cx[ci].state_set = true;
  return rebuild_worklist(c);
}

int sd_set_state(sd_ctx* c, int ci, const sd_swarm_state* st) {
  if (!c || !st || ci < 0 || ci >= c->ncplx) return fail(SD_ERR_ARG, "sd_set_state: bad arguments");
  if (!st->pos || !st->scoring || !st->luciferin || !st->vision_range || !st->step || !st->moved || !st->nnei_len ||
      !st->select || !st->ligand_reference_pose)
    return fail(SD_ERR_ARG, "sd_set_state: every state field is required");
  SD_CUDA(cudaSetDevice(c->device));
  const DevComplex& D = c->cx[ci].d;
  const size_t n = (size_t)D.S * D.G;
  for (size_t k = 0; k < n; ++k)
    if (st->select[k] < 0 || st->select[k] >= D.G) return fail(SD_ERR_ARG, "sd_set_state: select out of range");
  SD_CUDA(cudaMemcpyAsync(D.pos, st->pos, n * D.pl * 8, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.scoring, st->scoring, n * 8, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.luciferin, st->luciferin, n * 8, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.vision, st->vision_range, n * 8, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.step, st->step, n * 4, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.moved, st->moved, n * 4, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.nnei, st->nnei_len, n * 4, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.select, st->select, n * 4, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(D.ref, st->ligand_reference_pose, n * 3 * 8, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaStreamSynchronize(c->stream));
  c->cx[ci].state_set = true;
  return rebuild_worklist(c);
}

int sd_get_state(sd_ctx* c, int ci, sd_swarm_state* st) {
  if (!c || !st || ci < 0 || ci >= c->ncplx) return fail(SD_ERR_ARG, "sd_get_state: bad arguments");
  SD_CUDA(cudaSetDevice(c->device));
  const DevComplex& D = c->cx[ci].d;
  const size_t n = (size_t)D.S * D.G;
  auto cp = [&](void* dst, const void* src, size_t bytes) -> int {
    if (!dst) return SD_OK;
    SD_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    return SD_OK;
  };
  int rc;
  if ((rc = cp(st->pos, D.pos, n * D.pl * 8))) return rc;
  if ((rc = cp(st->scoring, D.scoring, n * 8))) return rc;
  if ((rc = cp(st->luciferin, D.luciferin, n * 8))) return rc;
  if ((rc = cp(st->vision_range, D.vision, n * 8))) return rc;
  if ((rc = cp(st->step, D.step, n * 4))) return rc;
  if ((rc = cp(st->moved, D.moved, n * 4))) return rc;
  if ((rc = cp(st->nnei_len, D.nnei, n * 4))) return rc;
  if ((rc = cp(st->select, D.select, n * 4))) return rc;
  if ((rc = cp(st->ligand_reference_pose, D.ref, n * 3 * 8))) return rc;
  SD_CUDA(cudaStreamSynchronize(c->stream));
  return SD_OK;
}

int sd_set_draws(sd_ctx* c, int ci, const double* u, int n_steps) {
  if (!c || !u || n_steps <= 0 || ci < 0 || ci >= c->ncplx) return fail(SD_ERR_ARG, "sd_set_draws: bad arguments");
  SD_CUDA(cudaSetDevice(c->device));
  ComplexHost& h = c->cx[ci];
  DevComplex& D = h.d;
  const size_t n = (size_t)D.S * n_steps * D.G;
  if (h.draws_steps < n_steps) {
    if (D.draws) {
      SD_CUDA(cudaStreamSynchronize(c->stream));
      auto it = std::find(h.owned.begin(), h.owned.end(), (void*)D.draws);
      if (it != h.owned.end()) h.owned.erase(it);
      cudaFree((void*)D.draws);
      D.draws = nullptr;
    }
    double* p = nullptr;
    SD_CUDA(cudaMalloc(&p, n * 8));
    h.owned.push_back(p);
    D.draws = p;
    h.draws_steps = n_steps;
  }
  SD_CUDA(cudaMemcpyAsync((void*)D.draws, u, n * 8, cudaMemcpyHostToDevice, c->stream));
  D.draw_steps = n_steps;
  D.draw_cursor = 0;
  h.draws_used = 0;
  h.draws_steps = std::max(h.draws_steps, n_steps);
  // only this complex's descriptor changes; the others keep their device cursors
  SD_CUDA(cudaMemcpyAsync(&c->d_cplx[ci], &D, sizeof(DevComplex), cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaStreamSynchronize(c->stream));
  h.draws_steps = n_steps;
  return SD_OK;
}

int sd_step(sd_ctx* c, int n_steps, int sync) {
  sd::NvtxRange nvtx_range("sd_step");
  if (!c || n_steps < 0) return fail(SD_ERR_ARG, "sd_step: bad arguments");
  SD_CUDA(cudaSetDevice(c->device));
  for (auto& h : c->cx) {
    if (!h.state_set) return fail(SD_ERR_STATE, "sd_step: state not set for every complex");
    if (h.draws_used + n_steps > h.d.draw_steps)
      return fail(SD_ERR_STATE, "sd_step: not enough random draws set (sd_set_draws)");
  }
  if (!c->tuned && c->precision == SD_PREC_MIXED && c->scoring == SD_SCORING_DFIRE) {
    int rc = autotune_mixed(c);
    if (rc) return rc;
  }
  if (!c->graph || c->graph_precision != c->precision) {
    if (c->graph) {
      cudaGraphExecDestroy(c->graph);
      c->graph = nullptr;
    }
    int grid;
    size_t sm;
    int rc = configure_score(c, c->precision, &grid, &sm);
    if (rc) return rc;
    cudaGraph_t g;
    SD_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    rc = enqueue_step(c, c->precision, grid, sm);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (rc) {
      if (e == cudaSuccess) cudaGraphDestroy(g);
      return rc;
    }
    SD_CUDA(e);
    cudaError_t ie = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    SD_CUDA(ie);
    c->graph_precision = c->precision;
  }
  for (int s = 0; s < n_steps; ++s) SD_CUDA(cudaGraphLaunch(c->graph, c->stream));
  for (auto& h : c->cx) h.draws_used += n_steps;
  if (sync) SD_CUDA(cudaStreamSynchronize(c->stream));
  return SD_OK;
}

int sd_get_stats(sd_ctx* c, sd_stats* out) {
  if (!c || !out) return fail(SD_ERR_ARG, "sd_get_stats: NULL");
  SD_CUDA(cudaSetDevice(c->device));
  SD_CUDA(cudaStreamSynchronize(c->stream));
  StepCtl a, b;
  SD_CUDA(cudaMemcpy(&a, c->d_ctl, sizeof a, cudaMemcpyDeviceToHost));
  SD_CUDA(cudaMemcpy(&b, c->d_ctl_scratch, sizeof b, cudaMemcpyDeviceToHost));
  out->scored_poses = (long long)a.stats[ST_SCORED];
  out->steps = (long long)a.stats[ST_STEPS];
  out->pairs_fallback = (long long)(a.stats[ST_FALLBACK] + b.stats[ST_FALLBACK]);
  out->edge_d2_zero = (long long)(a.stats[ST_D2ZERO] + b.stats[ST_D2ZERO]);
  out->edge_d2_cutoff = (long long)(a.stats[ST_D2CUT] + b.stats[ST_D2CUT]);
  out->edge_u_zero = (long long)a.stats[ST_UZERO];
  out->edge_shortfall = (long long)a.stats[ST_SHORT];
  out->timeouts = (long long)(a.stats[ST_TIMEOUT] + b.stats[ST_TIMEOUT]);
  out->pairs_in_cutoff = (long long)a.stats[ST_PAIRS];
  out->pairs_evaluated = (long long)a.stats[ST_EVALS];
  return SD_OK;
}

int sd_get_tuning(sd_ctx* c, int* variant, int* warps, int* min_blocks, double* ms, int n_ms) {
  if (!c) return fail(SD_ERR_ARG, "sd_get_tuning: NULL context");
  if (variant) *variant = c->mixed_variant;
  if (warps) *warps = mixed_variant_warps(c->mixed_variant);
  if (min_blocks) *min_blocks = mixed_variant_min_blocks(c->mixed_variant);
  if (ms)
    for (int v = 0; v < n_ms; ++v) ms[v] = v < mixed_variant_count() && c->tuned ? c->tune_ms[v] : 0.0;
  return SD_OK;
}

int sd_mixed_variant_count(void) { return mixed_variant_count(); }

int sd_set_precision(sd_ctx* c, int precision) {
  if (!c || precision < SD_PREC_FP64_REF || precision > SD_PREC_MIXED)
    return fail(SD_ERR_ARG, "sd_set_precision: bad arguments");
  c->precision = precision;
  return SD_OK;
}

int sd_score_poses(sd_ctx* c, int ci, const double* poses, int n, int precision, double* score_out,
                   double* energy_out) {
  sd::NvtxRange nvtx_range("sd_score_poses");
  if (!c || !poses || !score_out || n < 0 || ci < 0 || ci >= c->ncplx)
    return fail(SD_ERR_ARG, "sd_score_poses: bad arguments");
  if (precision < SD_PREC_FP64_REF || precision > SD_PREC_MIXED)
    return fail(SD_ERR_ARG, "sd_score_poses: unknown precision");
  if (n == 0) return SD_OK;
  if (n >= (1 << 24)) return fail(SD_ERR_ARG, "sd_score_poses: more than 2^24 poses");
  SD_CUDA(cudaSetDevice(c->device));
  const DevComplex& D = c->cx[ci].d;
  for (size_t i = 0; i < (size_t)n * D.pl; ++i)
    if (!std::isfinite(poses[i])) return fail(SD_ERR_NUMERIC, "sd_score_poses: non-finite pose");
  int rc;
  if ((rc = ensure(c, c->s_pose, (size_t)n * D.pl * 8))) return rc;
  if ((rc = ensure(c, c->s_score, (size_t)n * 8))) return rc;
  if ((rc = ensure(c, c->s_energy, (size_t)n * 8))) return rc;
  if ((rc = ensure(c, c->s_ref, (size_t)n * 3 * 8))) return rc;
  if ((rc = ensure(c, c->s_work, (size_t)n * 4))) return rc;
  std::vector<int> work(n);
  for (int i = 0; i < n; ++i) work[i] = wi_pack(ci, i);
  DevComplex S = D;
  S.pos = (double*)c->s_pose.p;
  S.scoring = (double*)c->s_score.p;
  S.ref = (double*)c->s_ref.p;
  StepCtl ctl;
  SD_CUDA(cudaMemcpy(&ctl, c->d_ctl_scratch, sizeof ctl, cudaMemcpyDeviceToHost));
  ctl.count[0] = n;
  ctl.count[1] = 0;
  ctl.grab[0] = ctl.grab[1] = 0;
  ctl.parity = 0;
  SD_CUDA(cudaMemcpyAsync(c->s_pose.p, poses, (size_t)n * D.pl * 8, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(c->s_work.p, work.data(), (size_t)n * 4, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(&c->d_cplx_scratch[ci], &S, sizeof S, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(c->d_ctl_scratch, &ctl, sizeof ctl, cudaMemcpyHostToDevice, c->stream));
  int grid;
  size_t sm;
  if ((rc = configure_score(c, precision, &grid, &sm))) return rc;
  ScoreLaunch L{};
  L.cplx = c->d_cplx_scratch;
  L.ctl = c->d_ctl_scratch;
  L.work[0] = (const int*)c->s_work.p;
  L.work[1] = (const int*)c->s_work.p;
  L.table64 = c->d_table64;
  L.tablek = c->d_tablek;
  L.lj_eps = c->d_lj_eps;
  L.lj_sigma = c->d_lj_sigma;
  L.energy_out = (double*)c->s_energy.p;
  set_spill(c, L);
  if ((rc = score_launch(L, precision, c->scoring, grid, c->score_threads, sm, c->stream, c->mixed_variant,
                         c->score_spill)))
    return fail(rc, std::string("score kernel: ") + cudaGetErrorString(cudaGetLastError()));
  SD_CUDA(cudaMemcpyAsync(score_out, c->s_score.p, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
  if (energy_out)
    SD_CUDA(cudaMemcpyAsync(energy_out, c->s_energy.p, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
  SD_CUDA(cudaStreamSynchronize(c->stream));
  return SD_OK;
}

int sd_dfire_bins(sd_ctx* c, int ci, const double* pose, int precision, int* bins_out) {
  sd::NvtxRange nvtx_range("sd_dfire_bins");
  if (!c || !pose || !bins_out || ci < 0 || ci >= c->ncplx) return fail(SD_ERR_ARG, "sd_dfire_bins: bad arguments");
  SD_CUDA(cudaSetDevice(c->device));
  const DevComplex& D = c->cx[ci].d;
  const size_t nb = (size_t)D.nr * D.nl;
  int rc;
  if ((rc = ensure(c, c->s_bins, nb * 4 + 64))) return rc;
  if ((rc = ensure(c, c->s_pose, (size_t)D.pl * 8))) return rc;
  SD_CUDA(cudaMemcpyAsync(c->s_pose.p, pose, (size_t)D.pl * 8, cudaMemcpyHostToDevice, c->stream));
  int* d_bins = (int*)c->s_bins.p;
  int* d_fb = (int*)((char*)c->s_bins.p + nb * 4);
  SD_CUDA(cudaMemsetAsync(d_fb, 0, 4, c->stream));
  if ((rc = bins_launch(c->d_cplx, ci, (const double*)c->s_pose.p, precision, d_bins, D.nr, D.nl, d_fb, c->stream)))
    return fail(rc, "bins kernel launch failed");
  SD_CUDA(cudaMemcpyAsync(bins_out, d_bins, nb * 4, cudaMemcpyDeviceToHost, c->stream));
  SD_CUDA(cudaStreamSynchronize(c->stream));
  return SD_OK;
}

int sd_pydock_grad(sd_ctx* c, int ci, const double* poses, int n, int precision, double* energy_out,
                   double* grad_out) {
  sd::NvtxRange nvtx_range("sd_pydock_grad");
  if (!c || !poses || !grad_out || n < 0 || ci < 0 || ci >= c->ncplx)
    return fail(SD_ERR_ARG, "sd_pydock_grad: bad arguments");
  if (c->scoring != SD_SCORING_PYDOCK) return fail(SD_ERR_ARG, "sd_pydock_grad: context scoring is not pyDock");
  if (precision < SD_PREC_FP64_REF || precision > SD_PREC_MIXED)
    return fail(SD_ERR_ARG, "sd_pydock_grad: unknown precision");
  if (n == 0) return SD_OK;
  if (n >= (1 << 24)) return fail(SD_ERR_ARG, "sd_pydock_grad: more than 2^24 poses");
  SD_CUDA(cudaSetDevice(c->device));
  const DevComplex& D = c->cx[ci].d;
  const int ng = 6 + D.nmr + D.nml;
  for (size_t i = 0; i < (size_t)n * D.pl; ++i)
    if (!std::isfinite(poses[i])) return fail(SD_ERR_NUMERIC, "sd_pydock_grad: non-finite pose");
  int rc;
  if ((rc = ensure(c, c->s_pose, (size_t)n * D.pl * 8))) return rc;
  if ((rc = ensure(c, c->s_score, (size_t)n * 8))) return rc;
  if ((rc = ensure(c, c->s_energy, (size_t)n * 8))) return rc;
  if ((rc = ensure(c, c->s_ref, (size_t)n * 3 * 8))) return rc;
  if ((rc = ensure(c, c->s_work, (size_t)n * 4))) return rc;
  if ((rc = ensure(c, c->s_grad, (size_t)n * ng * 8))) return rc;
  std::vector<int> work(n);
  for (int i = 0; i < n; ++i) work[i] = wi_pack(ci, i);
  DevComplex S = D;
  S.pos = (double*)c->s_pose.p;
  S.scoring = (double*)c->s_score.p;
  S.ref = (double*)c->s_ref.p;
  StepCtl ctl;
  SD_CUDA(cudaMemcpy(&ctl, c->d_ctl_scratch, sizeof ctl, cudaMemcpyDeviceToHost));
  ctl.count[0] = n;
  ctl.count[1] = 0;
  ctl.grab[0] = ctl.grab[1] = 0;
  ctl.parity = 0;
  SD_CUDA(cudaMemcpyAsync(c->s_pose.p, poses, (size_t)n * D.pl * 8, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(c->s_work.p, work.data(), (size_t)n * 4, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(&c->d_cplx_scratch[ci], &S, sizeof S, cudaMemcpyHostToDevice, c->stream));
  SD_CUDA(cudaMemcpyAsync(c->d_ctl_scratch, &ctl, sizeof ctl, cudaMemcpyHostToDevice, c->stream));
  const size_t need = pydock_smem_bytes(precision, true, c->max_nl, c->max_nr);
  const void* k = pydock_kernel_ptr(precision, true, false);
  cudaFuncAttributes fa;
  SD_CUDA(cudaFuncGetAttributes(&fa, k));
  // a ligand too large for shared memory: the spill instantiation, per-CTA arrays in global scratch
  const bool spill = need + fa.sharedSizeBytes > (size_t)c->smem_optin;
  const size_t sm = spill ? 0 : need;
  if (spill) k = pydock_kernel_ptr(precision, true, true);
  SD_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(sm, 1)));
  int per_sm = 0;
  SD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, pydock_threads(), sm));
  if (per_sm < 1) return fail(SD_ERR_ARG, "pyDock gradient kernel does not fit on an SM");
  const size_t stride = (need + 255) & ~(size_t)255;
  if (spill && (rc = grow_spill(c, stride * (size_t)per_sm * c->nsm))) return rc;
  ScoreLaunch L{};
  L.spill = spill ? (unsigned char*)c->s_spill.p : nullptr;
  L.spill_stride = spill ? stride : 0;
  L.cplx = c->d_cplx_scratch;
  L.ctl = c->d_ctl_scratch;
  L.work[0] = (const int*)c->s_work.p;
  L.work[1] = (const int*)c->s_work.p;
  L.table64 = c->d_table64;
  L.tablek = c->d_tablek;
  L.lj_eps = c->d_lj_eps;
  L.lj_sigma = c->d_lj_sigma;
  L.energy_out = (double*)c->s_energy.p;
  if ((rc = pydock_launch(L, precision, true, (double*)c->s_grad.p, per_sm * c->nsm, sm, c->stream, spill)))
    return fail(rc, std::string("pyDock gradient kernel: ") + cudaGetErrorString(cudaGetLastError()));
  if (energy_out)
    SD_CUDA(cudaMemcpyAsync(energy_out, c->s_energy.p, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
  SD_CUDA(cudaMemcpyAsync(grad_out, c->s_grad.p, (size_t)n * ng * 8, cudaMemcpyDeviceToHost, c->stream));
  SD_CUDA(cudaStreamSynchronize(c->stream));
  return SD_OK;
}

int sd_refine_poses(sd_ctx* c, int ci, double* poses, int n, int iters, double step, int precision,
                    double* energy_before, double* energy_after) {
  sd::NvtxRange nvtx_range("sd_refine_poses");
  if (!c || !poses || n < 0 || iters < 0 || !(step > 0) || ci < 0 || ci >= c->ncplx)
    return fail(SD_ERR_ARG, "sd_refine_poses: bad arguments");
  if (c->scoring != SD_SCORING_PYDOCK) return fail(SD_ERR_ARG, "sd_refine_poses: context scoring is not pyDock");
  if (n == 0) return SD_OK;
  const DevComplex& D = c->cx[ci].d;
  const int pl = D.pl, ng = 6 + D.nmr + D.nml;
  const double RL = std::max(1.0, (double)D.lig_radius);
  std::vector<double> sc(n), E(n), Ec(n), g((size_t)n * ng), cand((size_t)n * pl), alpha(n, step);
  int rc;
  if ((rc = sd_score_poses(c, ci, poses, n, SD_PREC_FP64, sc.data(), E.data()))) return rc;
  if (energy_before) std::copy(E.begin(), E.end(), energy_before);
  for (int it = 0; it < iters; ++it) {
    if ((rc = sd_pydock_grad(c, ci, poses, n, precision, nullptr, g.data()))) return rc;
    for (int i = 0; i < n; ++i) {
      const double* gi = g.data() + (size_t)i * ng;
      const double* p0 = poses + (size_t)i * pl;
      double* p1 = cand.data() + (size_t)i * pl;
      std::copy(p0, p0 + pl, p1);
      double nrm = 0;
      for (int k = 0; k < ng; ++k) {
        const double v = (k >= 3 && k < 6) ? gi[k] / RL : gi[k];
        nrm += v * v;
      }
      nrm = std::sqrt(nrm);
      if (!(nrm > 0) || !std::isfinite(nrm)) continue;
      const double a = alpha[i] / nrm;
      for (int k = 0; k < 3; ++k) p1[k] -= a * gi[k];
      // rotation by the angle vector -a * g_w / RL^2 (arc length a * |g_w| / RL at radius RL)
      const double w[3] = {-a * gi[3] / (RL * RL), -a * gi[4] / (RL * RL), -a * gi[5] / (RL * RL)};
      const double th = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
      if (th > 0) {
        const double s2 = std::sin(0.5 * th) / th, c2 = std::cos(0.5 * th);
        const double dq[4] = {c2, s2 * w[0], s2 * w[1], s2 * w[2]};
        const double q[4] = {p1[3], p1[4], p1[5], p1[6]};
        p1[3] = dq[0] * q[0] - dq[1] * q[1] - dq[2] * q[2] - dq[3] * q[3];
        p1[4] = dq[0] * q[1] + dq[1] * q[0] + dq[2] * q[3] - dq[3] * q[2];
        p1[5] = dq[0] * q[2] - dq[1] * q[3] + dq[2] * q[0] + dq[3] * q[1];
        p1[6] = dq[0] * q[3] + dq[1] * q[2] - dq[2] * q[1] + dq[3] * q[0];
      }
      for (int k = 6; k < ng; ++k) p1[7 + (k - 6)] -= a * gi[k];
    }
    if ((rc = sd_score_poses(c, ci, cand.data(), n, SD_PREC_FP64, sc.data(), Ec.data()))) return rc;
    for (int i = 0; i < n; ++i) {
      if (Ec[i] < E[i]) {
        std::copy(cand.data() + (size_t)i * pl, cand.data() + (size_t)(i + 1) * pl, poses + (size_t)i * pl);
        E[i] = Ec[i];
        alpha[i] *= 1.5;
      } else {
        alpha[i] *= 0.5;
      }
    }
  }
  if (energy_after) std::copy(E.begin(), E.end(), energy_after);
  return SD_OK;
}

int sd_materialise_poses(sd_ctx* c, int ci, const int* poses, int n, double* rec_xyz_out, double* lig_xyz_out) {
  sd::NvtxRange nvtx_range("sd_materialise_poses");
  if (!c || ci < 0 || ci >= c->ncplx || !poses || n <= 0 || (!rec_xyz_out && !lig_xyz_out))
    return fail(SD_ERR_ARG, "sd_materialise_poses: bad arguments");
  if (!c->cx[ci].state_set) return fail(SD_ERR_STATE, "sd_materialise_poses: no state");
  SD_CUDA(cudaSetDevice(c->device));
  const DevComplex& D = c->cx[ci].d;
  const long long SG = (long long)D.S * D.G;
  for (int k = 0; k < n; ++k)
    if (poses[k] < 0 || poses[k] >= SG) return fail(SD_ERR_ARG, "sd_materialise_poses: pose index out of range");
  const int nr = D.nr, nl = D.nl, nslots = D.ntiles * SD_TILE;
  std::vector<int> orig(nslots), slot_of(nr, 0);
  SD_CUDA(cudaMemcpy(orig.data(), D.r_orig, sizeof(int) * nslots, cudaMemcpyDeviceToHost));
  for (int sl = 0; sl < nslots; ++sl)
    if (orig[sl] >= 0) slot_of[orig[sl]] = sl;
  // poses per launch: coordinates of at most 256 MiB on the device
  const size_t per_pose = (size_t)(nr + nl) * 3 * sizeof(double);
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)n, ((size_t)256 << 20) / per_pose));
  int *d_poses = nullptr, *d_slot = nullptr;
  double* d_xyz = nullptr;
  auto release = [&]() {
    cudaFree(d_poses);
    cudaFree(d_slot);
    cudaFree(d_xyz);
  };
  auto cu = [&](cudaError_t e) {
    if (e == cudaSuccess) return SD_OK;
    release();
    return fail(e == cudaErrorMemoryAllocation ? SD_ERR_OOM : SD_ERR_CUDA,
                std::string("sd_materialise_poses: ") + cudaGetErrorString(e));
  };
  int rc;
  if ((rc = cu(cudaMalloc(&d_poses, sizeof(int) * chunk)))) return rc;
  if ((rc = cu(cudaMalloc(&d_slot, sizeof(int) * std::max(1, nr))))) return rc;
  if ((rc = cu(cudaMalloc(&d_xyz, per_pose * chunk)))) return rc;
  if ((rc = cu(cudaMemcpy(d_slot, slot_of.data(), sizeof(int) * nr, cudaMemcpyHostToDevice)))) return rc;
  for (int k0 = 0; k0 < n; k0 += chunk) {
    const int m = std::min(chunk, n - k0);
    double* d_rec = d_xyz;
    double* d_lig = d_xyz + (size_t)m * nr * 3;
    if ((rc = cu(cudaMemcpyAsync(d_poses, poses + k0, sizeof(int) * m, cudaMemcpyHostToDevice, c->stream))))
      return rc;
    if ((rc = materialise_launch(c->d_cplx, ci, d_poses, m, d_slot, nr, nl, d_rec, d_lig, c->stream))) {
      release();
      return fail(rc, "sd_materialise_poses: launch failed");
    }
    if (rec_xyz_out && (rc = cu(cudaMemcpyAsync(rec_xyz_out + (size_t)k0 * nr * 3, d_rec, sizeof(double) * m * nr * 3,
                                                cudaMemcpyDeviceToHost, c->stream))))
      return rc;
    if (lig_xyz_out && (rc = cu(cudaMemcpyAsync(lig_xyz_out + (size_t)k0 * nl * 3, d_lig, sizeof(double) * m * nl * 3,
                                                cudaMemcpyDeviceToHost, c->stream))))
      return rc;
    if ((rc = cu(cudaStreamSynchronize(c->stream)))) return rc;
  }
  release();
  return SD_OK;
}

int sd_cluster(sd_ctx* c, int ci, const int* rec_backbone, const int* lig_backbone, int* n_clusters,
               int* cluster_rep, int* cluster_len, int* member_of) {
  sd::NvtxRange nvtx_range("sd_cluster");
  if (!c || ci < 0 || ci >= c->ncplx || !rec_backbone || !lig_backbone || !n_clusters || !cluster_rep ||
      !cluster_len || !member_of)
    return fail(SD_ERR_ARG, "sd_cluster: bad arguments");
  if (!c->cx[ci].state_set) return fail(SD_ERR_STATE, "sd_cluster: no state");
  SD_CUDA(cudaSetDevice(c->device));
  const DevComplex& D = c->cx[ci].d;
  const int S = D.S, G = D.G, nslots = D.ntiles * SD_TILE;
  // receptor slot of each flagged atom (atoms are stored in spatial tile order)
  std::vector<int> orig(nslots), slot_of(D.nr, -1), rb, lb;
  SD_CUDA(cudaMemcpy(orig.data(), D.r_orig, sizeof(int) * nslots, cudaMemcpyDeviceToHost));
  for (int sl = 0; sl < nslots; ++sl)
    if (orig[sl] >= 0) slot_of[orig[sl]] = sl;
  for (int i = 0; i < D.nr; ++i)
    if (rec_backbone[i]) rb.push_back(slot_of[i]);
  for (int j = 0; j < D.nl; ++j)
    if (lig_backbone[j]) lb.push_back(j);
  const int nbr = (int)rb.size(), nbl = (int)lb.size(), nbb = nbr + nbl;
  if (nbb == 0) return fail(SD_ERR_ARG, "sd_cluster: no backbone atoms flagged");
  if (cluster_smem_bytes(G, nbb) > 227 * 1024) return fail(SD_ERR_NOTSUP, "sd_cluster: too many backbone atoms");
  // swarms per launch: coordinates of at most ~1 GiB on the device
  const size_t per_swarm = (size_t)G * nbb * 3 * sizeof(double);
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)S, ((size_t)1 << 30) / per_swarm));
  int* d_rb = nullptr;
  int* d_lb = nullptr;
  int* d_out = nullptr;
  double* d_bb = nullptr;
  auto release = [&]() {
    cudaFree(d_rb);
    cudaFree(d_lb);
    cudaFree(d_out);
    cudaFree(d_bb);
  };
  auto cu = [&](cudaError_t e) {
    if (e == cudaSuccess) return SD_OK;
    release();
    return fail(e == cudaErrorMemoryAllocation ? SD_ERR_OOM : SD_ERR_CUDA, std::string("sd_cluster: ") + cudaGetErrorString(e));
  };
  int rc;
  if ((rc = cu(cudaMalloc(&d_rb, sizeof(int) * std::max(1, nbr))))) return rc;
  if ((rc = cu(cudaMalloc(&d_lb, sizeof(int) * std::max(1, nbl))))) return rc;
  if ((rc = cu(cudaMalloc(&d_out, sizeof(int) * ((size_t)S + 3 * (size_t)S * G))))) return rc;
  if ((rc = cu(cudaMalloc(&d_bb, per_swarm * chunk)))) return rc;
  if (nbr && (rc = cu(cudaMemcpy(d_rb, rb.data(), sizeof(int) * nbr, cudaMemcpyHostToDevice)))) return rc;
  if (nbl && (rc = cu(cudaMemcpy(d_lb, lb.data(), sizeof(int) * nbl, cudaMemcpyHostToDevice)))) return rc;
  int* d_ncl = d_out;
  int* d_rep = d_out + S;
  int* d_len = d_rep + (size_t)S * G;
  int* d_mem = d_len + (size_t)S * G;
  for (int s0 = 0; s0 < S; s0 += chunk) {
    const int ns = std::min(chunk, S - s0);
    if ((rc = cluster_launch(c->d_cplx, ci, s0, ns, G, d_rb, nbr, d_lb, nbl, d_bb, d_ncl, d_rep, d_len, d_mem,
                             c->stream))) {
      release();
      return fail(rc, "sd_cluster: launch failed");
    }
  }
  if ((rc = cu(cudaStreamSynchronize(c->stream)))) return rc;
  if ((rc = cu(cudaMemcpy(n_clusters, d_ncl, sizeof(int) * S, cudaMemcpyDeviceToHost)))) return rc;
  if ((rc = cu(cudaMemcpy(cluster_rep, d_rep, sizeof(int) * S * G, cudaMemcpyDeviceToHost)))) return rc;
  if ((rc = cu(cudaMemcpy(cluster_len, d_len, sizeof(int) * S * G, cudaMemcpyDeviceToHost)))) return rc;
  if ((rc = cu(cudaMemcpy(member_of, d_mem, sizeof(int) * S * G, cudaMemcpyDeviceToHost)))) return rc;
  release();
  return SD_OK;
}

}  // extern "C"
