// cal_gso_tasks_b200.cc -- the reference-side binding of the GSO hot path.
//
// A maintainer compiles this file in place of the reference's GPU translation unit
// (source/dock/src/cuda/prepare_gso_task.cu) and links libsparkle_b200.so; nothing above it
// changes.  It defines cal_gso_tasks_gpu with the reference's own signature
// (source/dock/include/prepare_gso_tasks.h:18-21), the function prepare_gso_tasks
// (source/dock/src/prepare_gso_tasks.cc:1151-1256) calls when USE_CUDA is set, and runs the whole
// GSO loop through the C ABI of include/sparkle_b200.h: one context for the rank's swarms, the
// reference's draws, STEPS GSO steps, the positions written back into centers.pos and the
// swarm_<i>/gso_<STEPS>.out files the reference writes (prepare_gso_task.cu:2838-2905).
//
// Environment: SPARKLE_STEPS (the reference's compile-time STEPS, default 100) and
// SPARKLE_PRECISION (mixed | fp64 | fp64_ref, default mixed).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "prepare_gso_tasks.h"  // reference header: Complex, SwarmCenters, FastDifire
#include "sparkle_b200.h"

namespace {

int precision_from_env() {
  const char* p = getenv("SPARKLE_PRECISION");
  if (!p || !strcmp(p, "mixed")) return SD_PREC_MIXED;
  if (!strcmp(p, "fp64")) return SD_PREC_FP64;
  if (!strcmp(p, "fp64_ref")) return SD_PREC_FP64_REF;
  fprintf(stderr, "sparkle_b200: SPARKLE_PRECISION must be mixed, fp64 or fp64_ref; using mixed\n");
  return SD_PREC_MIXED;
}

bool ok(int rc, const char* what) {
  if (rc == SD_OK) return true;
  fprintf(stderr, "sparkle_b200: %s: %s\n", what, sd_last_error());
  return false;
}

}  // namespace

void cal_gso_tasks_gpu(SwarmCenters& centers, Complex& receptor, Complex& lignad, FastDifire& fastdifire, int seed,
                       double step_translation, double step_rotation, bool use_anm, double nmodes_step, int anm_rec,
                       int anm_lig, bool local_minimization, int swarms, int num_glowworms,
                       double* receptor_reference_points, double* receptor_poles, double* ligand_reference_points,
                       double* ligand_poles, int* dfire_objects_rec, int* dfire_objects_lig, int object_size_rec,
                       int object_size_lig, int rank, int size) {
  (void)seed, (void)step_translation, (void)step_rotation, (void)use_anm, (void)nmodes_step;
  (void)local_minimization, (void)swarms, (void)receptor_reference_points, (void)receptor_poles;
  (void)ligand_poles, (void)object_size_rec, (void)object_size_lig, (void)size;
  const int steps = getenv("SPARKLE_STEPS") ? atoi(getenv("SPARKLE_STEPS")) : 100;  // the STEPS macro
  sd_complex_desc d;
  memset(&d, 0, sizeof d);
  d.n_rec = receptor.num_atoms;
  d.n_lig = lignad.num_atoms;
  d.rec_xyz = receptor.atom_coordinates;
  d.lig_xyz = lignad.atom_coordinates;
  d.rec_mask = receptor.mask;
  d.lig_mask = lignad.mask;
  d.n_modes_rec = anm_rec;
  d.n_modes_lig = anm_lig;
  d.rec_modes = receptor.modes;
  d.lig_modes = lignad.modes;
  d.rec_dfire_type = dfire_objects_rec;
  d.lig_dfire_type = dfire_objects_lig;
  for (int k = 0; k < 3; ++k) d.lig_ref_point[k] = ligand_reference_points[k];
  d.n_swarms = centers.swarm_chunk;
  d.n_glowworms = num_glowworms;
  sd_tables t = {fastdifire.difire_energy, nullptr, nullptr};
  sd_gso_params p;
  sd_gso_params_default(&p);  // the reference's defaults; its movement steps are the literal 0.5
  int ndev = 0;
  sd_device_count(&ndev);
  const int device = ndev ? rank % ndev : 0;  // the reference's rank -> GPU mapping
  sd_ctx* ctx = nullptr;
  if (!ok(sd_ctx_create(&d, 1, &t, &p, SD_SCORING_DFIRE, precision_from_env(), device, &ctx), "sd_ctx_create"))
    return;
  const int pl = SD_POSE_LEN(anm_rec, anm_lig);
  double* pos = centers.pos + (size_t)centers.swarm_start * centers.pos_len;
  const size_t n = (size_t)d.n_swarms * num_glowworms;
  std::vector<double> u((size_t)d.n_swarms * steps * num_glowworms);
  std::vector<double> luc(n), vis(n), sc(n);
  std::vector<int> nnei(n);
  sd_swarm_state st = {pos, sc.data(), luc.data(), vis.data(), nullptr, nullptr, nnei.data(), nullptr, nullptr};
  // the CPU path's draws: mt19937(0) over the rank's swarms (prepare_gso_tasks.cc:411-427)
  if (ok(sd_gso_draws(0, d.n_swarms, steps, num_glowworms, u.data()), "sd_gso_draws") &&
      ok(sd_init_state(ctx, 0, pos), "sd_init_state") && ok(sd_set_draws(ctx, 0, u.data(), steps), "sd_set_draws") &&
      ok(sd_step(ctx, steps, 1), "sd_step") && ok(sd_get_state(ctx, 0, &st), "sd_get_state"))
    ok(sd_write_gso_output(".", centers.swarm_start, d.n_swarms, num_glowworms, pl, steps, pos, luc.data(),
                           nnei.data(), vis.data(), sc.data()),
       "sd_write_gso_output");
  sd_ctx_destroy(ctx);
}
