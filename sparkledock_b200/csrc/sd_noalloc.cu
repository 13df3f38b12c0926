// sd_score_poses_noalloc: stateless pose scoring that allocates no memory during the call.
//
// Who needs it: callers that must not allocate device memory while they score, for example
// code that records its GPU work into a CUDA graph (stream capture) or a host framework
// whose memory manager owns all device memory in its steady state and forbids the CUDA
// allocator there.  They pass their own device buffers for poses and results; the few
// words of bookkeeping the scoring kernel needs besides its inputs and outputs (its work
// list, its grab counters and a per-call copy of the complex descriptor) live in the
// file-scope array below instead of in memory allocated per call.
//
// The array is statically sized (SD_NOALLOC_SCRATCH_BYTES, 288 KiB) and is part of every
// GPU that loads this library, until the process exits.  All calls on a device share it and
// it keeps the last call's contents; each call rewrites what it reads (descriptor, counters,
// work list) before the scoring kernel runs.  Two calls whose GPU work overlaps in time
// (different streams, or different contexts on one device) therefore race on it: callers
// must order such calls.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "sd_internal.h"

namespace sd {
// defined in sd_api.cu: the parts of a context this call reads (no allocation)
int ctx_noalloc_view(sd_ctx* c, int ci, int precision, DevComplex* desc, ScoreLaunch* L, int* grid, size_t* smem,
                     int* device, cudaStream_t* stream, int* scoring, int* variant);
}  // namespace sd

using namespace sd;

namespace {

constexpr int kMaxPoses = SD_NOALLOC_MAX_POSES;
constexpr size_t kCtlBytes = 256;
constexpr size_t kDescBytes = ((sizeof(DevComplex) * SD_MAX_COMPLEX + 255) / 256) * 256;
constexpr size_t kWorkBytes = sizeof(int) * (size_t)kMaxPoses;
constexpr size_t kScratchBytes = kCtlBytes + kDescBytes + kWorkBytes;
static_assert(sizeof(StepCtl) <= kCtlBytes, "StepCtl outgrew its scratch slot");
static_assert(kScratchBytes <= SD_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the stated size");

// the scratch: [StepCtl | DevComplex x SD_MAX_COMPLEX | work list x kMaxPoses]
static __device__ __align__(256) unsigned char g_noalloc_scratch[SD_NOALLOC_SCRATCH_BYTES];

// device address of g_noalloc_scratch per device (host code cannot use the symbol itself)
std::mutex g_mu;
void* g_addr[64] = {};

__global__ void noalloc_prepare_kernel(unsigned char* scratch, DevComplex desc, int ci, int n) {
  StepCtl* ctl = reinterpret_cast<StepCtl*>(scratch);
  DevComplex* cplx = reinterpret_cast<DevComplex*>(scratch + kCtlBytes);
  int* work = reinterpret_cast<int*>(scratch + kCtlBytes + kDescBytes);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid == 0) {
    StepCtl z;
    memset(&z, 0, sizeof z);
    z.count[0] = n;
    *ctl = z;
    cplx[ci] = desc;
  }
  for (int i = tid; i < n; i += gridDim.x * blockDim.x) work[i] = wi_pack(ci, i);
}

}  // namespace

extern "C" int sd_score_poses_noalloc(sd_ctx* ctx, int complex_idx, const double* d_poses, int n, int precision,
                                      double* d_score, double* d_energy, double* d_ref, int sync) {
  if (!ctx || !d_poses || !d_score || !d_ref || n < 0)
    return fail(SD_ERR_ARG, "sd_score_poses_noalloc: NULL argument or negative count");
  if (n > kMaxPoses)
    return fail(SD_ERR_ARG, "sd_score_poses_noalloc: " + std::to_string(n) + " poses exceed the maximum of " +
                                std::to_string(kMaxPoses) + " per call");
  DevComplex desc;
  ScoreLaunch L{};
  int grid = 0, device = 0, scoring = SD_SCORING_DFIRE, variant = 0;
  size_t smem = 0;
  cudaStream_t stream = nullptr;
  int rc = ctx_noalloc_view(ctx, complex_idx, precision, &desc, &L, &grid, &smem, &device, &stream, &scoring, &variant);
  if (rc) return rc;
  if (n == 0) return SD_OK;
  if (device < 0 || device >= 64) return fail(SD_ERR_ARG, "sd_score_poses_noalloc: device index above 63");
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[device]) {
      // once per device, with that device current (ctx_noalloc_view made it current)
      cudaError_t e = cudaGetSymbolAddress(&g_addr[device], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_addr[device] = nullptr;
        return fail(SD_ERR_CUDA, std::string("sd_score_poses_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      }
    }
    base = g_addr[device];
  }
  unsigned char* scratch = static_cast<unsigned char*>(base);
  desc.pos = const_cast<double*>(d_poses);
  desc.scoring = d_score;
  desc.ref = d_ref;
  noalloc_prepare_kernel<<<(n + 255) / 256, 256, 0, stream>>>(scratch, desc, complex_idx, n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SD_ERR_CUDA, std::string("sd_score_poses_noalloc: ") + cudaGetErrorString(e));
  L.cplx = reinterpret_cast<const DevComplex*>(scratch + kCtlBytes);
  L.ctl = reinterpret_cast<StepCtl*>(scratch);
  L.work[0] = reinterpret_cast<const int*>(scratch + kCtlBytes + kDescBytes);
  L.work[1] = L.work[0];
  L.energy_out = d_energy;
  if ((rc = score_launch(L, precision, scoring, grid, score_threads_of(precision, scoring, variant), smem, stream,
                         variant)))
    return fail(rc, std::string("sd_score_poses_noalloc: scoring kernel: ") + cudaGetErrorString(cudaGetLastError()));
  if (sync) {
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(SD_ERR_CUDA, std::string("sd_score_poses_noalloc: ") + cudaGetErrorString(e));
  }
  return SD_OK;
}
