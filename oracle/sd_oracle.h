/*
 * ORACLE — test infrastructure only.  A plain-C restatement of the reference's CPU GSO
 * docking path (menggerSherry/SparkleDock source/dock/src/prepare_gso_tasks.cc), used by
 * tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the checker.  The product
 * (sparkledock_b200/) never links, imports or calls anything here.
 *
 * Pins: the restatement is validated against the reference's own compiled functions
 * (oracle/_ref, built from the reference sources by oracle/Makefile) and against the
 * committed golden vectors in tests/golden/ that were produced from them.
 */
#ifndef SD_ORACLE_H
#define SD_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

#define OR_TYPES 168
#define OR_BINS 20
#define OR_MAX_MODES 10

typedef struct {
  int nr, nl, nmr, nml, S, G;
  const double* rec_xyz;   /* [nr][3] */
  const double* lig_xyz;   /* [nl][3] */
  const int* rec_mask;
  const int* lig_mask;
  const double* rec_modes; /* [nmr][nr][3] */
  const double* lig_modes; /* [nml][nl][3] */
  const int* rec_type;     /* DFIRE objects 0..167 */
  const int* lig_type;
  const double* table;     /* [168*168*20] */
  double lig_ref[3];
  /* pyDock-style terms (project-defined scoring; NULL for DFIRE) */
  const double* rec_charge;
  const double* lig_charge;
  const int* rec_lj;
  const int* lig_lj;
  const double* lj_eps;    /* [20] */
  const double* lj_sigma;  /* [20] */
  /* GSO parameters */
  double rho, gamma, beta, max_vision;
  int max_neighbors;
  double step_t, step_r, step_nm;
  int scoring;             /* 0 DFIRE, 1 pyDock */
  int cr_math;             /* 1: correctly rounded acos/sin in slerp, 0: platform libm (reference) */
} or_system;

typedef struct {
  double* pos;       /* [S][G][7+nmr+nml] */
  double* scoring;   /* [S][G] */
  double* luciferin; /* [S][G] */
  double* vision;    /* [S][G] */
  int* step;
  int* moved;
  int* nnei;
  int* select;
  double* ref;       /* [S][G][3] */
} or_state;

typedef struct {
  long long scored, d2_zero, d2_cutoff, u_zero, shortfall;
} or_counts;

/* std::mt19937(seed) + uniform_real_distribution<double>(0,1), swarm->step->glowworm */
void or_gso_draws(unsigned int seed, int S, int steps, int G, double* out);

/* pose transforms (exact reference operation order) */
void or_receptor_pose(const or_system* sys, const double* pose, double* rec_out);
void or_ligand_pose(const or_system* sys, const double* pose, double* lig_out, double* ref_out);

/* DFIRE: returns the raw table sum E; score = ((E*0.0157) - 4.7) * -1 */
double or_dfire_energy(const or_system* sys, const double* rec, const double* lig,
                       int* bins /* nullable [nr][nl] */, or_counts* c);
double or_score_pose(const or_system* sys, const double* pose, double* energy_out,
                     double* ref_out, int* bins, or_counts* c);
void or_score_poses(const or_system* sys, const double* poses, int n, double* scores,
                    double* energies, int nthreads);

/* pyDock-style elec + LJ energy (project-defined) and its gradient (FP64). */
double or_pydock_energy(const or_system* sys, const double* pose);
void or_pydock_grad(const or_system* sys, const double* pose, double* grad /* 6+nmr+nml */);

/* one GSO step; score_override (nullable [S][G]) replaces the oracle's own scores for the
 * glowworms rescored this step (step-locked checking). */
void or_gso_step(const or_system* sys, or_state* st, const double* u_step /* [S][G] */,
                 const double* score_override, or_counts* c, int nthreads);
void or_init_state(const or_system* sys, or_state* st, const double* pos0,
                   double luciferin0, double vision0);

/* Final-pose clustering of every swarm (BSAS of the reference's GPU pipeline variant,
 * source/dock/src/cuda/pipeline:2766-2960, keys as prepare_pair, prepare_gso_task.cu:1170-1187):
 * pos [S][G][pose_len], scores [S][G], backbone flags per receptor / ligand atom; outputs
 * n_clusters [S], rep / size [S][G] (first n_clusters[s] used), member [S][G]. */
void or_cluster(const or_system* sys, const double* pos, const double* scores, const int* rec_bb,
                const int* lig_bb, int* n_clusters, int* rep, int* size, int* member);
double or_sin_cr(double x);
double or_acos_cr(double x);
/* out[i] = or_acos_cr(x[i]) (fn 0) or or_sin_cr(x[i]) (fn 1) */
void or_crmath_eval(int fn, const double* x, long long n, double* out);
/* slerp of the reference (prepare_gso_tasks.cc:1370-1421) with cr or libm math */
void or_slerp(double* self, double* other, double step, int cr_math);

/* Seeded synthetic complexes and tables, restating the product's generator (or_synth.c):
 * caller-allocated arrays of the given sizes. */
typedef struct {
  double* rec_xyz;     /* [nr][3] */
  double* lig_xyz;     /* [nl][3] */
  double* rec_modes;   /* [nmr][nr][3] */
  double* lig_modes;   /* [nml][nl][3] */
  double* rec_charge;  /* [nr] */
  double* lig_charge;  /* [nl] */
  double* poses;       /* [S][G][7+nmr+nml] */
  int* rec_mask;
  int* lig_mask;
  int* rec_type;
  int* lig_type;
  int* rec_lj;
  int* lig_lj;
  double lig_ref[3];   /* Khachiyan centre of the ligand, tolerance 0.01 */
} or_synth_out;
void or_synth_generate(int nr, int nl, int S, int G, int nmr, int nml, unsigned long long seed, or_synth_out* o);
void or_synth_tables(unsigned long long seed, double* dfire, double* eps, double* sigma);
void or_mvee_center(const double* p, int n, double tol, double* center);

/* Exact key thresholds: smallest double x with (int)(sqrt(x)*2.0-1.0) >= m, m = 1..29 */
void or_key_thresholds(double* t30);

#ifdef __cplusplus
}
#endif
#endif
