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
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <algorithm>
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

// StepCtl.stats slot the prepare kernel uses to count non-finite pose values of the call
constexpr int kNonFiniteSlot = 10;
static_assert(kNonFiniteSlot > ST_EVALS && kNonFiniteSlot < 12, "free StepCtl.stats slot");

// device address of g_noalloc_scratch per device (host code cannot use the symbol itself), with
// the id of the CUDA context it was looked up in: a cudaDeviceReset in the process ends that
// context and unloads the module, so a new context id means the address must be looked up again
std::mutex g_mu;
void* g_addr[64] = {};
unsigned long long g_ctx_id[64] = {};

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// id of the current CUDA context (0 when the driver cannot say; the address is then looked up
// on every call, which is correct but slower)
unsigned long long current_ctx_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
    resolved = true;
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

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

// counts the non-finite values of the poses into the call's StepCtl (after the prepare kernel)
__global__ void noalloc_check_kernel(unsigned char* scratch, const double* poses, long long nvals) {
  StepCtl* ctl = reinterpret_cast<StepCtl*>(scratch);
  unsigned long long bad = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvals; i += (long long)gridDim.x * blockDim.x)
    bad += isfinite(poses[i]) ? 0ull : 1ull;
  for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, o);
  if ((threadIdx.x & 31) == 0 && bad) atomicAdd(&ctl->stats[kNonFiniteSlot], bad);
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
  if (sync) {
    // synchronising the stream would invalidate a capture the caller has open on it
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      cudaGetLastError();
      return fail(SD_ERR_ARG, "sd_score_poses_noalloc: sync must be 0 while the context stream is being captured");
    }
  }
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    const unsigned long long ctx_id = current_ctx_id();
    if (!g_addr[device] || ctx_id == 0 || ctx_id != g_ctx_id[device]) {
      // once per device (per CUDA context), with that device current (ctx_noalloc_view made it
      // current)
      void* a = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&a, g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_addr[device] = nullptr;
        return fail(SD_ERR_CUDA, std::string("sd_score_poses_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      }
      g_addr[device] = a;
      g_ctx_id[device] = ctx_id;
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
  if (sync) {
    const long long nvals = (long long)n * desc.pl;
    noalloc_check_kernel<<<(int)std::min<long long>((nvals + 255) / 256, 1184), 256, 0, stream>>>(scratch, d_poses,
                                                                                                  nvals);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(SD_ERR_CUDA, std::string("sd_score_poses_noalloc: ") + cudaGetErrorString(e));
  }
  L.cplx = reinterpret_cast<const DevComplex*>(scratch + kCtlBytes);
  L.ctl = reinterpret_cast<StepCtl*>(scratch);
  L.work[0] = reinterpret_cast<const int*>(scratch + kCtlBytes + kDescBytes);
  L.work[1] = L.work[0];
  L.energy_out = d_energy;
  const bool spill = L.spill != nullptr;
  if ((rc = score_launch(L, precision, scoring, grid,
                         spill ? score_threads_spill(precision, scoring) : score_threads_of(precision, scoring, variant),
                         smem, stream, variant, spill)))
    return fail(rc, std::string("sd_score_poses_noalloc: scoring kernel: ") + cudaGetErrorString(cudaGetLastError()));
  if (sync) {
    unsigned long long bad = 0;
    e = cudaMemcpyAsync(&bad, &reinterpret_cast<StepCtl*>(scratch)->stats[kNonFiniteSlot], sizeof bad,
                        cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(SD_ERR_CUDA, std::string("sd_score_poses_noalloc: ") + cudaGetErrorString(e));
    if (bad) return fail(SD_ERR_NUMERIC, "sd_score_poses_noalloc: " + std::to_string(bad) + " non-finite pose values");
  }
  return SD_OK;
}
