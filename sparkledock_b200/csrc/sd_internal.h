// Internal declarations shared by the host runtime and the kernels.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/sparkle_b200.h"

#if defined(__CUDACC__)
#include <cuda_runtime.h>
#endif

#define SD_TABLE_SIZE (SD_DFIRE_TYPES * SD_DFIRE_TYPES * SD_DFIRE_BINS)
#define SD_ROW (SD_DFIRE_TYPES * SD_DFIRE_BINS)  /* 3360 */
#define SD_KEYS 32              /* bin keys per type pair in the key-indexed table (30 used) */
#define SD_ROWK (SD_DFIRE_TYPES * SD_KEYS)        /* 5376 */
#define SD_TABLE_KEYS (SD_DFIRE_TYPES * SD_ROWK)  /* key-indexed table entries, followed by 32 zeros */
#define SD_CUTOFF2 225.0
#define SD_MAX_COMPLEX 32
#define SD_TILE 32              /* receptor atoms per tile (one warp lane each) */
#define SD_MAX_LIG 65504        /* ligand atoms: the mixed scorer's 16-bit ligand slot indices */
#define SD_MAX_REC (1 << 22)    /* receptor atoms */
#define SD_MAX_G 1024           /* glowworms per swarm with one thread each (one CTA per swarm) */
#define SD_MAX_GLOWWORMS 6144   /* glowworms per swarm: luciferin + reference points in shared memory */
#define SD_CULL_MARGIN 0.05f    /* A, covers FP32 rounding of the conservative culling tests */
#define SD_MAX_VARIANTS 16      /* compiled variants of the mixed DFIRE kernel (autotuner) */
#define SD_NOALLOC_MAX_POSES 65536           /* poses per sd_score_poses_noalloc call */
#define SD_NOALLOC_SCRATCH_BYTES (288 * 1024) /* its file-scope device scratch array */

namespace sd {

// a named NVTX range over a scope: the entry points show up by name on a profiler's timeline
// (no cost when no profiler is attached)
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// thread-local error message; returns code
int fail(int code, const std::string& msg);
void mvee_center(const double* p, int n, double tol, double* center);

// accessors of sd_structure (sd_structure.cc)
int structure_atoms(const sd_structure* s, std::vector<double>& xyz, std::vector<std::string>& names,
                    std::vector<int>& residue_first);
const std::vector<double>& structure_raw_xyz(const sd_structure* s);
const std::vector<std::string>& structure_residue_names(const sd_structure* s);
const std::vector<int>& structure_residue_first(const sd_structure* s);
const double* structure_translation(const sd_structure* s);

}  // namespace sd

#if defined(__CUDACC__)
namespace sd {

// ---- device-side view of one complex (lives in device memory, read by every kernel) ----
struct DevComplex {
  int nr, nl, nmr, nml, S, G, pl;
  int ntiles;           // receptor tiles of SD_TILE slots
  int gbase, sbase;     // first global glowworm / swarm index of this complex
  // receptor in tile order (slot = tile*32 + lane); padded slots have orig = -1
  const int* r_orig;
  const double* r_xyz;     // [nslots][3]
  const double* r_modes;   // [nmr][nslots][3]
  const int* r_mask;       // [nslots]
  const int* r_row;        // [nslots] DFIRE row base tR*3360
  const int* r_rowk;       // [nslots] key-indexed row base tR*5376
  const float4* r_tile;    // [ntiles] centre (rest frame) + radius
  const float* r_q;        // [nslots] charge (pyDock)
  const int* r_lj;         // [nslots] LJ type (pyDock)
  // ligand in original order
  const double* l_xyz;     // [nl][3]
  const double* l_modes;   // [nml][nl][3]
  const int* l_mask;
  const int* l_col;        // [nl] tL*20
  const float* l_q;
  const int* l_lj;
  // ligand in spatial chunks of 32 (mixed precision only; order-free sums)
  int nlchunks;
  const int* l_perm;       // [nlchunks*32] chunk slot -> original ligand index, or -1
  const float4* l_chunk;   // [nlchunks] centre (ligand frame) + radius
  // the ligand again in chunk-slot order (coalesced reads in the mixed kernels; padding slots 0)
  const double* lc_xyz;    // [nlchunks*32][3]
  const double* lc_modes;  // [nml][nlchunks*32][3]
  const int* lc_mask;      // [nlchunks*32]
  const int* lc_colk;      // [nlchunks*32] key-indexed column base tL*32
  float lig_ctr[3];        // ligand centroid (ligand frame)
  float mnorm_r[SD_MAX_MODES], mnorm_l[SD_MAX_MODES];  // max per-atom mode norm (rounded up)
  float lig_radius;        // max |l0_j| (rounded up)
  double lig_ref[3];
  // GSO state [S][G]
  double* pos;
  double* scoring;
  double* luciferin;
  double* vision;
  int* step;
  int* moved;
  int* nnei;
  int* select;
  double* ref;             // [S][G][3]
  const double* draws;     // [S][draw_steps][G]
  int draw_steps;
  int draw_cursor;         // advanced by the GSO kernel (device copy authoritative)
};

struct StepCtl {
  int count[2];            // items in work list [parity]
  int grab[2];             // next item to grab in list [parity]
  int parity;
  int done_blocks;         // GSO blocks finished in this step
  int step;
  int pad;
  unsigned long long stats[12];  // mirrors sd_stats order
};

enum { ST_SCORED = 0, ST_STEPS, ST_FALLBACK, ST_D2ZERO, ST_D2CUT, ST_UZERO, ST_SHORT, ST_TIMEOUT, ST_PAIRS, ST_EVALS };

struct GsoParamsDev {
  double rho, gamma, beta, max_vision, step_t, step_r, step_nm;
  int max_neighbors;
};

// work item: complex index in the top 8 bits, local glowworm index below
__host__ __device__ inline int wi_pack(int c, int local) { return (c << 24) | local; }
__host__ __device__ inline int wi_complex(int w) { return (int)((unsigned)w >> 24); }
__host__ __device__ inline int wi_local(int w) { return w & 0xFFFFFF; }

struct ScoreLaunch {
  const DevComplex* cplx;
  StepCtl* ctl;
  const int* work[2];
  const double* table64;   // [SD_TABLE_SIZE + 32] zero padded
  const double* tablek;    // [SD_TABLE_KEYS + 32] key-indexed: [tR][tL][key] = table64[tR*3360 + tL*20 + bin(key)]
  const double* lj_eps;    // [20] pyDock
  const double* lj_sigma;
  double* energy_out;      // nullable [local glowworm] raw energies (stateless scoring)
  // per-CTA global scratch that replaces the dynamic shared memory of the spill instantiations
  // (complexes whose per-pose arrays do not fit in shared memory); null otherwise
  unsigned char* spill;
  size_t spill_stride;     // bytes per CTA
};

struct GsoLaunch {
  DevComplex* cplx;
  StepCtl* ctl;
  int* work[2];
  const int* swarm_map;    // [total swarms] packed (complex, local swarm)
  int nswarms_total;
  int ncplx;               // <= 32 (the last CTA's first warp advances their draw cursors)
  GsoParamsDev p;
  double* pos_prev;        // swarms over SD_MAX_G glowworms: pre-move pose copies [glowworms][27]
};

// kernel launchers (sd_score.cu, sd_gso.cu)
// spill: the instantiation that keeps its per-pose arrays in L.spill instead of shared memory
int score_launch(const ScoreLaunch& L, int precision, int scoring, int grid, int threads, size_t smem,
                 cudaStream_t st, int variant, bool spill);
size_t score_smem_bytes(int precision, int scoring, int max_nr, int max_nl, int variant);
int score_threads_of(int precision, int scoring, int variant);
int score_threads_spill(int precision, int scoring);
const void* score_kernel_ptr(int precision, int scoring, int variant, bool spill);
int mixed_variant_count();
int mixed_variant_warps(int v);
int mixed_variant_min_blocks(int v);
int gso_launch(const GsoLaunch& L, int threads, cudaStream_t st);
int gso_launch_large(const GsoLaunch& L, int max_g, cudaStream_t st);
int gso_prepare_large();
int bins_launch(const DevComplex* cplx, int c, const double* d_pose, int precision, int* d_bins, int nr, int nl,
                int* d_fallback, cudaStream_t st);
size_t pydock_smem_bytes(int precision, bool grad, int max_nl, int max_nr);
const void* pydock_kernel_ptr(int precision, bool grad, bool spill);
int pydock_launch(const ScoreLaunch& L, int precision, bool grad, double* out_grad, int grid, size_t smem,
                  cudaStream_t st, bool spill);
int pydock_threads();
void set_key_thresholds(const double* t64);
size_t cluster_smem_bytes(int G, int nbb);
int materialise_launch(const DevComplex* d_cplx, int ci, const int* d_poses, int n, const int* d_rslot, int nr, int nl,
                       double* d_rec, double* d_lig, cudaStream_t st);
int cluster_launch(const DevComplex* d_cplx, int ci, int s0, int ns, int G, const int* d_rb_slot, int nbr,
                   const int* d_lb_idx, int nbl, double* d_bb, int* d_ncl, int* d_rep, int* d_len, int* d_member,
                   cudaStream_t st);

}  // namespace sd
#endif  // __CUDACC__
