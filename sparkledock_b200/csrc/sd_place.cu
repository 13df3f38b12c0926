// Swarm centres and starting poses, as the reference's setup places them before docking:
// calculate_start_pos (source/dock/src/cal_anm.cc:775-990) with calculate_surface_point
// (:541-774), select_surface (:991-1018), points_on_sphere (:1101-1113) and the k-means of
// source/dock/src/kmeans.cc:126-241 (kmeans_init_centers3, run_kmeans3).
//
// On the receptor and ligand as read (before centring):
//  1. surface points: every atom of a residue whose name is in the surface list;
//  2. surface distance: 10 A, or a quarter of the ligand's largest interatomic distance when
//     that is 20 A or more;
//  3. k-means++ seeding (mt19937(324324)) and 100 Lloyd iterations of the surface points into
//     n_swarms centroids;
//  4. 100 points on a Fibonacci sphere of radius surface distance around every centroid; a point
//     is dropped when it lies within the surface distance of another centroid that is within
//     20 A of its own, or within 3 A of any receptor atom;
//  5. k-means++ seeding (a fresh mt19937(324324)) and 500 Lloyd iterations of the kept points
//     into n_swarms centres, moved into the centred frame (+ the receptor translation);
//  6. per swarm and glowworm, in order: a uniform point in the swarm_radius ball around the
//     centre (rejection from the cube, mt19937(seed + rank) uniform doubles), a uniform unit
//     quaternion from three more draws, and with ANM the extents from
//     std::default_random_engine(anm_seed) normal(0, 1) draws, receptor modes then ligand.
//
// Every comparison the reference makes is made here on the same FP64 values (a distance is the
// square root of ((dx^2 + dy^2) + dz^2), formed without contraction), so the result is the
// reference's to the bit:
//  * k-means++ seeding keeps each point's distance to its nearest chosen centre incrementally
//    (the reference recomputes the minimum over all chosen centres every round; the minimum is
//    the same value), one CTA; the two sequential FP64 chains of a round (the sum of those
//    distances, then the running subtraction that picks the next centre) run on one thread in
//    point order, as the reference's loops do;
//  * Lloyd assignment: one thread per point over the centres in order, the first strict minimum
//    of the square-rooted distance; a centre whose squared distance is not below the best one's
//    is skipped without the square root (its distance cannot be strictly smaller);
//  * Lloyd update: one warp per centre sums its members in point order (a ballot over the
//    assignment), then divides by the count;
//  * an iteration whose assignment equals the previous one reproduces the previous centres, so
//    the remaining iterations are skipped (a fixed point).
// Where the reference's result is undefined the call fails: too few surface points or kept
// points for the swarm count (the reference aborts or reads uninitialised centres), or an empty
// k-means cluster (its centre is 0/0, and in the first stage its sample points later make the
// reference index a cluster -1).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "sd_internal.h"

namespace sd {
namespace {

constexpr int kSpheresPerCentroid = 100;  // DEFAULT_SPHERES_PER_CENTROID
constexpr double kSurfaceCutoff = 3.0;    // SWARM_DISTANCE_TO_SURFACE_CUTOFF
constexpr double kNeighbourCentroid = 20.0;
constexpr double kDefaultSwarmRadius = 10.0;  // DEFAULT_SWARM_RADIUS
constexpr unsigned kKmeansSeed = 324324;
constexpr int kSurfaceIters = 100, kFinalIters = 500;
constexpr int kSeedThreads = 1024;
constexpr int kSeedSmemPoints = 25600;  // nearest-distance array kept in shared memory up to this
constexpr int kPollEvery = 8;           // Lloyd iterations between host checks of the fixed point

const char* const kSurfaceResidues[26] = {"ARG", "ASN", "ASP", "ASX", "CSO", "GLN", "GLU", "GLX", "GLY",
                                          "HID", "HIE", "HIP", "IS",  "HSD", "HSE", "HSP", "LYS", "PHD",
                                          "PRO", "PTR", "SEP", "SER", "THR", "TPO", "TYR", "HIS"};

__device__ __forceinline__ double dist2(double ax, double ay, double az, double bx, double by, double bz) {
  const double dx = __dsub_rn(ax, bx), dy = __dsub_rn(ay, by), dz = __dsub_rn(az, bz);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__device__ __forceinline__ double dist(double ax, double ay, double az, double bx, double by, double bz) {
  return __dsqrt_rn(dist2(ax, ay, az, bx, by, bz));
}

// largest squared interatomic distance (as an ordered bit pattern: squares are >= 0)
__global__ void max_pair_d2_kernel(const double* xyz, int n, unsigned long long* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = xyz[i * 3], y = xyz[i * 3 + 1], z = xyz[i * 3 + 2];
    double m = 0.0;
    for (int j = i + 1; j < n; ++j) m = fmax(m, dist2(x, y, z, xyz[j * 3], xyz[j * 3 + 1], xyz[j * 3 + 2]));
    atomicMax(out, (unsigned long long)__double_as_longlong(m));
  }
}

// k-means++ seeding (kmeans_init_centers3), one CTA.  prob[k-1] is round k's uniform draw.
// kShared: the nearest-distance array lives in shared memory (n <= kSeedSmemPoints), else in
// mind_global.  The two chains of a round stay strictly sequential; their loads are issued in
// blocks of kChainBlock ahead of the dependent adds.
constexpr int kChainBlock = 16;

template <bool kShared>
__global__ void __launch_bounds__(kSeedThreads) kpp_seed_kernel(const double* pts, int n, int K, int first,
                                                                  const double* prob, double* mind_global,
                                                                  double* centers) {
  extern __shared__ double mind_shared[];
  double* mind = kShared ? mind_shared : mind_global;
  __shared__ int sel;
  const int tid = threadIdx.x;
  for (int k = tid; k < K; k += blockDim.x)
    for (int d = 0; d < 3; ++d) centers[k * 3 + d] = pts[first * 3 + d];
  for (int p = tid; p < n; p += blockDim.x) mind[p] = DBL_MAX;
  __syncthreads();
  for (int k = 1; k < K; ++k) {
    const double cx = centers[(k - 1) * 3], cy = centers[(k - 1) * 3 + 1], cz = centers[(k - 1) * 3 + 2];
    for (int p = tid; p < n; p += blockDim.x) {
      const double d = dist(pts[p * 3], pts[p * 3 + 1], pts[p * 3 + 2], cx, cy, cz);
      if (d < mind[p]) mind[p] = d;
    }
    __syncthreads();
    if (tid == 0) {
      // the sum of the distances, in point order
      double sum = 0.0;
      int p = 0;
      for (; p + kChainBlock <= n; p += kChainBlock) {
        double v[kChainBlock];
#pragma unroll
        for (int j = 0; j < kChainBlock; ++j) v[j] = mind[p + j];
#pragma unroll
        for (int j = 0; j < kChainBlock; ++j) sum = __dadd_rn(sum, v[j]);
      }
      for (; p < n; ++p) sum = __dadd_rn(sum, mind[p]);
      sum = __dmul_rn(sum, prob[k - 1]);
      // the running subtraction: the first point at which it is no longer positive
      int s = -1;
      for (p = 0; p + kChainBlock <= n && s < 0; p += kChainBlock) {
        double v[kChainBlock];
#pragma unroll
        for (int j = 0; j < kChainBlock; ++j) v[j] = mind[p + j];
#pragma unroll
        for (int j = 0; j < kChainBlock; ++j) {
          sum = __dsub_rn(sum, v[j]);
          if (s < 0 && !(sum > 0)) s = p + j;
        }
      }
      for (; p < n && s < 0; ++p) {
        sum = __dsub_rn(sum, mind[p]);
        if (!(sum > 0)) s = p;
      }
      sel = s;
    }
    __syncthreads();
    if (sel >= 0 && tid < 3) centers[k * 3 + tid] = pts[sel * 3 + tid];
    __syncthreads();
  }
}

// Lloyd assignment (run_kmeans3's first loop); marks changed[it] when any point moves
__global__ void lloyd_assign_kernel(const double* pts, int n, const double* centers, int K, int* group,
                                    int* changed, int it, const int* done) {
  if (*done) return;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const double px = pts[p * 3], py = pts[p * 3 + 1], pz = pts[p * 3 + 2];
    double best = (double)FLT_MAX, best2 = INFINITY;
    int kid = -1;
    for (int k = 0; k < K; ++k) {
      const double d2 = dist2(centers[k * 3], centers[k * 3 + 1], centers[k * 3 + 2], px, py, pz);
      if (!(d2 < best2)) continue;  // sqrt(d2) >= best (or NaN): not a strict minimum
      const double d = __dsqrt_rn(d2);
      if (d < best) {
        best = d;
        best2 = d2;
        kid = k;
      }
    }
    if (group[p] != kid) changed[it] = 1;
    group[p] = kid;
  }
}

// Lloyd update (run_kmeans3's second loop): one warp per centre, members summed in point order
__global__ void lloyd_update_kernel(const double* pts, int n, const int* group, int K, double* centers,
                                    const int* changed, int it, int* done) {
  if (*done) return;
  if (!changed[it]) {  // same assignment as the previous iteration: the centres stay
    if (blockIdx.x == 0 && threadIdx.x == 0) *done = 1;
    return;
  }
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * (blockDim.x >> 5);
  for (int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < K; k += nwarps) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    int cnt = 0;
    for (int base = 0; base < n; base += 32) {
      const int p = base + lane;
      const bool mine = p < n && group[p] == k;
      unsigned b = __ballot_sync(0xffffffffu, mine);
      double x = 0.0, y = 0.0, z = 0.0;
      if (mine) {
        x = pts[p * 3];
        y = pts[p * 3 + 1];
        z = pts[p * 3 + 2];
      }
      while (b) {
        const int l = __ffs(b) - 1;
        b &= b - 1;
        sx = __dadd_rn(sx, __shfl_sync(0xffffffffu, x, l));
        sy = __dadd_rn(sy, __shfl_sync(0xffffffffu, y, l));
        sz = __dadd_rn(sz, __shfl_sync(0xffffffffu, z, l));
        ++cnt;
      }
    }
    if (lane == 0) {
      const double c = 1.0 * cnt;
      centers[k * 3] = __ddiv_rn(sx, c);
      centers[k * 3 + 1] = __ddiv_rn(sy, c);
      centers[k * 3 + 2] = __ddiv_rn(sz, c);
    }
  }
}

// sphere points around every centroid, then the two filters (keep[i * 100 + p])
__global__ void sample_filter_kernel(const double* cent, int K, const double* unit, double sdist,
                                     const double* rec, int nrec, double* samp, int* keep) {
  const int total = K * kSpheresPerCentroid;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int i = e / kSpheresPerCentroid, p = e % kSpheresPerCentroid;
    const double cx = cent[i * 3], cy = cent[i * 3 + 1], cz = cent[i * 3 + 2];
    const double sx = __dadd_rn(__dmul_rn(unit[p * 3], sdist), cx);
    const double sy = __dadd_rn(__dmul_rn(unit[p * 3 + 1], sdist), cy);
    const double sz = __dadd_rn(__dmul_rn(unit[p * 3 + 2], sdist), cz);
    samp[e * 3] = sx;
    samp[e * 3 + 1] = sy;
    samp[e * 3 + 2] = sz;
    bool ok = true;
    for (int j = 0; j < K && ok; ++j) {
      if (j == i) continue;
      const double jx = cent[j * 3], jy = cent[j * 3 + 1], jz = cent[j * 3 + 2];
      if (dist(cx, cy, cz, jx, jy, jz) <= kNeighbourCentroid && dist(sx, sy, sz, jx, jy, jz) <= sdist) ok = false;
    }
    for (int a = 0; a < nrec && ok; ++a) {
      const double d2 = dist2(sx, sy, sz, rec[a * 3], rec[a * 3 + 1], rec[a * 3 + 2]);
      if (d2 < 9.5 && __dsqrt_rn(d2) <= kSurfaceCutoff) ok = false;
    }
    keep[e] = ok ? 1 : 0;
  }
}

struct DevBuf {
  std::vector<void*> ptrs;
  ~DevBuf() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <class T>
  cudaError_t alloc(T** p, size_t count) {
    void* v = nullptr;
    const cudaError_t e = cudaMalloc(&v, sizeof(T) * (count ? count : 1));
    if (e == cudaSuccess) ptrs.push_back(v);
    *p = static_cast<T*>(v);
    return e;
  }
};

int cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? SD_ERR_OOM : SD_ERR_CUDA,
              std::string("sd_place_swarms: ") + what + ": " + cudaGetErrorString(e));
}

// kmeans_init_centers3 + run_kmeans3 of n points into K centres; centres_out [K][3] on the host
int kmeans(const double* d_pts, int n, int K, int iters, std::vector<double>& centres_out) {
  std::mt19937 gen(kKmeansSeed);
  std::uniform_int_distribution<int> pick(0, n - 1);
  const int first = pick(gen);
  std::vector<double> prob(K > 1 ? K - 1 : 1);
  for (int k = 1; k < K; ++k) {
    std::uniform_real_distribution<float> u(0.0, 1.0);
    prob[k - 1] = u(gen);
  }
  DevBuf b;
  double *d_prob, *d_mind, *d_cent;
  int *d_group, *d_changed, *d_done;
  cudaError_t e;
  if ((e = b.alloc(&d_prob, prob.size())) || (e = b.alloc(&d_mind, n)) || (e = b.alloc(&d_cent, (size_t)K * 3)) ||
      (e = b.alloc(&d_group, n)) || (e = b.alloc(&d_changed, iters)) || (e = b.alloc(&d_done, 1)))
    return cuda_fail(e, "cudaMalloc");
  if ((e = cudaMemcpy(d_prob, prob.data(), sizeof(double) * prob.size(), cudaMemcpyHostToDevice)) ||
      (e = cudaMemset(d_group, 0xff, sizeof(int) * n)) || (e = cudaMemset(d_changed, 0, sizeof(int) * iters)) ||
      (e = cudaMemset(d_done, 0, sizeof(int))))
    return cuda_fail(e, "upload");
  if (n <= kSeedSmemPoints) {
    const size_t smem = sizeof(double) * n;
    if ((e = cudaFuncSetAttribute(kpp_seed_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
      return cuda_fail(e, "k-means++ shared memory");
    kpp_seed_kernel<true><<<1, kSeedThreads, smem>>>(d_pts, n, K, first, d_prob, d_mind, d_cent);
  } else {
    kpp_seed_kernel<false><<<1, kSeedThreads, 0>>>(d_pts, n, K, first, d_prob, d_mind, d_cent);
  }
  if ((e = cudaGetLastError())) return cuda_fail(e, "k-means++ launch");
  const int ablocks = std::min((n + 255) / 256, 148 * 8), ublocks = std::min((K + 7) / 8, 148 * 8);
  for (int it = 0; it < iters; ++it) {
    if (it > 0 && it % kPollEvery == 0) {
      int done = 0;
      if ((e = cudaMemcpy(&done, d_done, sizeof(int), cudaMemcpyDeviceToHost))) return cuda_fail(e, "Lloyd poll");
      if (done) break;
    }
    lloyd_assign_kernel<<<ablocks, 256>>>(d_pts, n, d_cent, K, d_group, d_changed, it, d_done);
    lloyd_update_kernel<<<ublocks, 256>>>(d_pts, n, d_group, K, d_cent, d_changed, it, d_done);
  }
  if ((e = cudaGetLastError())) return cuda_fail(e, "Lloyd launch");
  centres_out.resize((size_t)K * 3);
  if ((e = cudaMemcpy(centres_out.data(), d_cent, sizeof(double) * K * 3, cudaMemcpyDeviceToHost)))
    return cuda_fail(e, "download");
  for (double v : centres_out)
    if (!std::isfinite(v))
      return fail(SD_ERR_NUMERIC, "sd_place_swarms: a k-means cluster ended empty (the reference's result is "
                                  "undefined there)");
  return SD_OK;
}

}  // namespace

// the reference's per-glowworm sampling around the centres (calculate_start_pos :825-888)
void sample_start_poses(const double* centres, int S, int G, int nmr, int nml, bool use_anm, int seed, int anm_seed,
                        double swarm_radius, int rank, double* poses) {
  const double PI = 3.14159265358979323846;
  std::mt19937 gen(seed + rank);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  std::default_random_engine nm_gen(anm_seed);
  std::normal_distribution<double> nrm(0.0, 1.0);
  const int pl = 7 + nmr + nml;
  const double r2 = swarm_radius * swarm_radius;
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < G; ++j) {
      double* p = poses + ((size_t)i * G + j) * pl;
      double g[3];
      while (true) {
        const double a = u(gen), b = u(gen), c = u(gen);
        const double x = (2 * a - 1) * swarm_radius, y = (2 * b - 1) * swarm_radius, z = (2 * c - 1) * swarm_radius;
        if (x * x + y * y + z * z <= r2) {
          g[0] = x;
          g[1] = y;
          g[2] = z;
          break;
        }
      }
      for (int d = 0; d < 3; ++d) p[d] = centres[i * 3 + d] + g[d];
      const double u1 = u(gen), u2 = u(gen), u3 = u(gen);
      p[3] = std::sqrt(1 - u1) * std::sin(2 * PI * u2);
      p[4] = std::sqrt(1 - u1) * std::cos(2 * PI * u2);
      p[5] = std::sqrt(u1) * std::sin(2 * PI * u3);
      p[6] = std::sqrt(u1) * std::cos(2 * PI * u3);
      for (int m = 0; m < nmr + nml; ++m) p[7 + m] = use_anm ? nrm(nm_gen) : 0.0;
    }
}

}  // namespace sd

extern "C" int sd_place_swarms(const sd_structure* receptor, const sd_structure* ligand, int n_swarms, int n_glowworms,
                               int n_modes_rec, int n_modes_lig, int use_anm, int starting_points_seed, int anm_seed,
                               double swarm_radius, int rank, int device, double* centers_out, double* poses_out) {
  sd::NvtxRange nvtx_range("sd_place_swarms");
  using namespace sd;
  if (!receptor || !ligand || n_swarms <= 0 || n_glowworms <= 0 || n_modes_rec < 0 || n_modes_lig < 0 || rank < 0 ||
      !(swarm_radius > 0) || (!centers_out && !poses_out))
    return fail(SD_ERR_ARG, "sd_place_swarms: bad arguments");
  const std::vector<double>& rec = structure_raw_xyz(receptor);
  const std::vector<double>& lig = structure_raw_xyz(ligand);
  const std::vector<std::string>& rname = structure_residue_names(receptor);
  const std::vector<int>& rfirst = structure_residue_first(receptor);
  const int nrec = (int)rec.size() / 3, nlig = (int)lig.size() / 3;
  // surface points (select_surface)
  std::vector<double> surf;
  for (size_t r = 0; r + 1 < rfirst.size(); ++r) {
    bool is_surface = false;
    for (const char* s : kSurfaceResidues) is_surface = is_surface || rname[r] == s;
    if (is_surface) surf.insert(surf.end(), rec.begin() + (size_t)rfirst[r] * 3, rec.begin() + (size_t)rfirst[r + 1] * 3);
  }
  const int nsurf = (int)surf.size() / 3;
  if (nsurf <= n_swarms)
    return fail(SD_ERR_ARG, "sd_place_swarms: " + std::to_string(nsurf) + " surface atoms for " +
                                std::to_string(n_swarms) + " swarms (the reference needs more points than swarms)");
  if (cudaSetDevice(device) != cudaSuccess) return fail(SD_ERR_CUDA, "sd_place_swarms: bad device");
  DevBuf b;
  double *d_rec, *d_lig, *d_surf, *d_cent, *d_unit, *d_samp, *d_kept;
  int* d_keep;
  unsigned long long* d_max;
  const int nsamp = n_swarms * kSpheresPerCentroid;
  cudaError_t e;
  if ((e = b.alloc(&d_rec, rec.size())) || (e = b.alloc(&d_lig, lig.size())) || (e = b.alloc(&d_surf, surf.size())) ||
      (e = b.alloc(&d_cent, (size_t)n_swarms * 3)) || (e = b.alloc(&d_unit, kSpheresPerCentroid * 3)) ||
      (e = b.alloc(&d_samp, (size_t)nsamp * 3)) || (e = b.alloc(&d_keep, nsamp)) || (e = b.alloc(&d_max, 1)))
    return cuda_fail(e, "cudaMalloc");
  if ((e = cudaMemcpy(d_rec, rec.data(), sizeof(double) * rec.size(), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(d_lig, lig.data(), sizeof(double) * lig.size(), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(d_surf, surf.data(), sizeof(double) * surf.size(), cudaMemcpyHostToDevice)) ||
      (e = cudaMemset(d_max, 0, sizeof(unsigned long long))))
    return cuda_fail(e, "upload");
  // surface distance from the ligand's diameter
  max_pair_d2_kernel<<<std::max(1, std::min((nlig + 127) / 128, 148 * 4)), 128>>>(d_lig, nlig, d_max);
  unsigned long long maxbits = 0;
  if ((e = cudaGetLastError()) || (e = cudaMemcpy(&maxbits, d_max, sizeof(maxbits), cudaMemcpyDeviceToHost)))
    return cuda_fail(e, "ligand diameter");
  double m2;
  std::memcpy(&m2, &maxbits, sizeof(m2));
  const double lig_diameter = std::sqrt(m2);
  const double sdist = lig_diameter < kDefaultSwarmRadius * 2 ? kDefaultSwarmRadius : lig_diameter / 4.0;
  // surface k-means
  std::vector<double> cent;
  int rc = kmeans(d_surf, nsurf, n_swarms, kSurfaceIters, cent);
  if (rc) return rc;
  // sphere points (points_on_sphere, the same unit points around every centroid) and filters
  std::vector<double> unit(kSpheresPerCentroid * 3);
  {
    const double PI = 3.14159265358979323846;
    const double increment = PI * (3.0 - std::sqrt(5.0)), offset = 2.0 / kSpheresPerCentroid;
    for (int i = 0; i < kSpheresPerCentroid; ++i) {
      const double y = i * offset - 1.0 + (offset / 2.0), r = std::sqrt(1 - y * y), phi = i * increment;
      unit[i * 3] = std::cos(phi) * r;
      unit[i * 3 + 1] = y;
      unit[i * 3 + 2] = std::sin(phi) * r;
    }
  }
  if ((e = cudaMemcpy(d_cent, cent.data(), sizeof(double) * cent.size(), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(d_unit, unit.data(), sizeof(double) * unit.size(), cudaMemcpyHostToDevice)))
    return cuda_fail(e, "upload");
  sample_filter_kernel<<<std::max(1, std::min((nsamp + 127) / 128, 148 * 8)), 128>>>(d_cent, n_swarms, d_unit, sdist,
                                                                                      d_rec, nrec, d_samp, d_keep);
  std::vector<double> samp((size_t)nsamp * 3);
  std::vector<int> keep(nsamp);
  if ((e = cudaGetLastError()) ||
      (e = cudaMemcpy(samp.data(), d_samp, sizeof(double) * samp.size(), cudaMemcpyDeviceToHost)) ||
      (e = cudaMemcpy(keep.data(), d_keep, sizeof(int) * nsamp, cudaMemcpyDeviceToHost)))
    return cuda_fail(e, "sphere points");
  std::vector<double> kept;
  for (int i = 0; i < nsamp; ++i)
    if (keep[i]) kept.insert(kept.end(), samp.begin() + (size_t)i * 3, samp.begin() + (size_t)i * 3 + 3);
  const int nkept = (int)kept.size() / 3;
  if (nkept <= n_swarms)
    return fail(SD_ERR_ARG, "sd_place_swarms: " + std::to_string(nkept) + " sphere points kept for " +
                                std::to_string(n_swarms) + " swarms (the reference leaves the centres undefined)");
  if ((e = b.alloc(&d_kept, kept.size())) ||
      (e = cudaMemcpy(d_kept, kept.data(), sizeof(double) * kept.size(), cudaMemcpyHostToDevice)))
    return cuda_fail(e, "upload");
  rc = kmeans(d_kept, nkept, n_swarms, kFinalIters, cent);
  if (rc) return rc;
  const double* t = structure_translation(receptor);
  for (int i = 0; i < n_swarms; ++i)
    for (int d = 0; d < 3; ++d) cent[i * 3 + d] += t[d];
  if (centers_out) std::copy(cent.begin(), cent.end(), centers_out);
  if (poses_out)
    sample_start_poses(cent.data(), n_swarms, n_glowworms, n_modes_rec, n_modes_lig, use_anm != 0,
                       starting_points_seed, anm_seed, swarm_radius, rank, poses_out);
  return SD_OK;
}
