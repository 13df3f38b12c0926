/*
 * sparkle_b200.h — C ABI of the B200 GSO docking path.
 *
 * This boundary replaces the reference's hot-path entry points:
 *
 *   prepare_gso_tasks(SwarmCenters&, Complex& rec, Complex& lig, FastDifire&, int seed,
 *                     double step_t, double step_r, bool use_anm, double step_nm,
 *                     int anm_rec, int anm_lig, bool local_min, int swarms, int G,
 *                     int rank, int size)
 *       source/dock/include/prepare_gso_tasks.h:8-11, body source/dock/src/prepare_gso_tasks.cc:1151-1256
 *   cal_gso_tasks_gpu(...) / cal_gso_tasks_cpu(...)
 *       source/dock/include/prepare_gso_tasks.h:18-26
 *   cdfire_calculate_dfire(double* E, ..., int* rec_objects, int* lig_objects, FastDifire&,
 *                          double* rec_xyz, double* lig_xyz, int Nr, int Nl, int g, int s)
 *       source/dock/include/prepare_gso_tasks.h:36-40 (the scoring "plugin")
 *
 * Plain pointers and sizes only.  All pointers passed in are HOST pointers unless the
 * argument name says otherwise; the context copies what it needs and owns its device
 * memory for its lifetime.  Every call returns an int status (SD_OK == 0); a failing
 * call leaves a message for sd_last_error().  Nothing here calls exit().
 *
 * Threading: one context is used by one host thread at a time; distinct contexts may be
 * used concurrently.  Each context owns one CUDA stream on its device.
 *
 * Devices: every call that touches a GPU makes its device (the context's, or the device
 * argument) current on the calling thread, as cudaSetDevice does, and leaves it current on
 * return.  A caller that drives several GPUs from one thread selects its own device again
 * after a call.
 */
#ifndef SPARKLE_B200_H
#define SPARKLE_B200_H

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---- status codes ---- */
#define SD_OK 0
#define SD_ERR_ARG 1      /* bad argument (sizes, NULL, out-of-range type, ...) */
#define SD_ERR_OOM 2      /* device or pinned allocation failed */
#define SD_ERR_CUDA 3     /* a CUDA runtime call failed */
#define SD_ERR_TIMEOUT 4  /* a bounded device wait gave up */
#define SD_ERR_NUMERIC 5  /* NaN/Inf met in a pose or energy */
#define SD_ERR_STATE 6    /* call out of order (no state set, draws exhausted, ...) */
#define SD_ERR_NOTSUP 7   /* valid request this build does not support */

/* ---- fixed model constants (reference source/dock/include/fastdfire.h:91-93, interface.h:30-35) ---- */
#define SD_DFIRE_TYPES 168
#define SD_DFIRE_BINS 20
#define SD_MAX_MODES 10     /* DEFAULT_NMODES_REC / _LIG, prepare_gso_tasks.cc:23-24 */
#define SD_LJ_TYPES 20
#define SD_POSE_LEN(nm_rec, nm_lig) (7 + (nm_rec) + (nm_lig))

/* scoring functions selectable by setup.json "scoring" */
#define SD_SCORING_DFIRE 0   /* reference DFIRE (prepare_gso_tasks.cc:1522-1615) */
#define SD_SCORING_PYDOCK 1  /* project-defined elec + LJ (no reference counterpart) */

/* precision / algorithm of the pair stage */
#define SD_PREC_FP64_REF 0   /* FP64, all Nr*Nl pairs, reference pair order: bit-exact energies */
#define SD_PREC_FP64 1       /* FP64 with the cutoff cell culling; same order -> bit-exact */
#define SD_PREC_MIXED 2      /* FP16/FP32 distances, exact bins (FP64 near-edge fallback), FP64 sums */

/* One receptor/ligand complex and its swarms.  Mirrors the fields of the reference's
 * Complex (source/prep/include/complex.h:10-104: atom_coordinates, mask, modes, num_atoms)
 * and the per-atom DFIRE objects made by get_docking_model (prepare_gso_tasks.cc:31-69). */
typedef struct {
  int n_rec, n_lig;
  const double* rec_xyz;        /* [n_rec][3], receptor frame */
  const double* lig_xyz;        /* [n_lig][3], ligand frame (rotation centre at origin) */
  const int* rec_mask;          /* [n_rec], 0/1 ANM mask (get_nm_mask) */
  const int* lig_mask;          /* [n_lig] */
  int n_modes_rec, n_modes_lig; /* 0..SD_MAX_MODES */
  const double* rec_modes;      /* [n_modes_rec][n_rec][3] */
  const double* lig_modes;      /* [n_modes_lig][n_lig][3] */
  const int* rec_dfire_type;    /* [n_rec], 0..167 */
  const int* lig_dfire_type;    /* [n_lig], 0..167 */
  const double* rec_charge;     /* [n_rec] partial charges (pyDock scoring; may be NULL for DFIRE) */
  const double* lig_charge;     /* [n_lig] */
  const int* rec_lj_type;       /* [n_rec], 0..19 (pyDock scoring; may be NULL for DFIRE) */
  const int* lig_lj_type;       /* [n_lig] */
  double lig_ref_point[3];      /* ligand reference point, ligand frame (minimum_volume_ellipsoid centre) */
  int n_swarms, n_glowworms;
} sd_complex_desc;

/* Scoring tables shared by all complexes of a context. */
typedef struct {
  const double* dfire_energy;   /* [168*168*20], FastDifire.difire_energy layout [tR][tL][bin] */
  const double* lj_eps;         /* [20] well depths (kcal/mol), pyDock scoring */
  const double* lj_sigma;       /* [20] radii (A), pyDock scoring */
} sd_tables;

/* GSO parameters.  Defaults are the reference's Glowworm defaults (interface.h:9-26) and the
 * literal 0.5 movement steps (prepare_gso_tasks.cc:783, :791-794). */
typedef struct {
  double rho, gamma, beta;
  double initial_luciferin, initial_vision_range, max_vision_range;
  int max_neighbors;
  double translation_step, rotation_step, nmodes_step;
} sd_gso_params;

/* Per-glowworm state of one complex, structure-of-arrays, [S][G] row-major (swarm-major),
 * the reference's SoA (prepare_gso_tasks.cc:370-409).  In sd_get_state any pointer may be
 * NULL to skip that field; in sd_set_state all pointers are required. */
typedef struct {
  double* pos;                  /* [S][G][pose_len]: tx,ty,tz, qw,qx,qy,qz, ext_rec[], ext_lig[] */
  double* scoring;              /* [S][G] last score of each glowworm */
  double* luciferin;            /* [S][G] */
  double* vision_range;         /* [S][G] */
  int* step;                    /* [S][G] steps taken */
  int* moved;                   /* [S][G] moved in the last step (rescored next step) */
  int* nnei_len;                /* [S][G] neighbour count of the last step */
  int* select;                  /* [S][G] neighbour chosen in the last step (self if none) */
  double* ligand_reference_pose;/* [S][G][3] ligand reference point in the receptor frame */
} sd_swarm_state;

/* Counters of the rare paths, cumulative since context creation. */
typedef struct {
  long long scored_poses;       /* poses rescored (moved or first step) */
  long long steps;              /* GSO steps taken */
  long long pairs_fallback;     /* MIXED: pairs re-evaluated in FP64 near a bin or cutoff edge */
  long long edge_d2_zero;       /* pairs at distance 0 (reference reads dist_to_bins[-1]) */
  long long edge_d2_cutoff;     /* pairs at d^2 == 225 exactly (reference reads bin 20) */
  long long edge_u_zero;        /* draws u <= 0 with neighbours (reference reads neighbors[-1]) */
  long long edge_shortfall;     /* cumulative probability < u after all neighbours */
  long long timeouts;           /* bounded device waits that gave up */
  long long pairs_in_cutoff;    /* receptor-ligand pairs with d^2 <= 225 met while rescoring (GSO steps) */
  long long pairs_evaluated;    /* pair distances computed after culling (GSO steps) */
} sd_stats;

typedef struct sd_ctx sd_ctx;

/* ---- library ---- */
const char* sd_last_error(void);          /* thread-local message of the last failing call */
const char* sd_version(void);
int sd_device_count(int* n);              /* visible CUDA devices (0 without a GPU) */
void sd_gso_params_default(sd_gso_params* p);

/* Reference random draws: u[s][t][g] ~ uniform_real_distribution<double>(0,1) over
 * std::mt19937(seed) in swarm -> step -> glowworm order (prepare_gso_tasks.cc:411-427). */
int sd_gso_draws(unsigned int seed, int n_swarms, int n_steps, int n_glowworms, double* u_out);

/* ---- context ---- */
int sd_ctx_create(const sd_complex_desc* complexes, int n_complexes, const sd_tables* tables,
                  const sd_gso_params* params, int scoring, int precision, int device,
                  sd_ctx** out);
int sd_ctx_destroy(sd_ctx* ctx);
int sd_ctx_stream(sd_ctx* ctx, void** cuda_stream_out);  /* the context's cudaStream_t */
int sd_pose_len(const sd_ctx* ctx, int complex_idx, int* pose_len);

/* Starting state: pos as given, luciferin/vision range from params, step = moved = 0
 * (the reference's SoA initialisation, prepare_gso_tasks.cc:386-400). */
int sd_init_state(sd_ctx* ctx, int complex_idx, const double* pos);
int sd_set_state(sd_ctx* ctx, int complex_idx, const sd_swarm_state* st);
int sd_get_state(sd_ctx* ctx, int complex_idx, sd_swarm_state* st);

/* Random draws for the next n_steps of one complex, layout [S][n_steps][G]; replaces any
 * draws not yet used. */
int sd_set_draws(sd_ctx* ctx, int complex_idx, const double* u, int n_steps);

/* n_steps GSO steps of every complex (pose -> score -> luciferin -> select -> move;
 * reference step driver prepare_gso_task.cu:2745-2822, semantics of
 * prepare_gso_tasks.cc:429-819).  Asynchronous on the context stream unless sync != 0. */
int sd_step(sd_ctx* ctx, int n_steps, int sync);

int sd_get_stats(sd_ctx* ctx, sd_stats* out);
/* Autotuner result for the mixed-precision DFIRE kernel: the chosen compiled variant, its warps
 * per CTA and minimum resident CTAs per SM, and (if ms != NULL) the measured time of each
 * variant on the context's poses (0 before the first mixed sd_step).  The tuner runs once per
 * context before its first mixed step; SPARKLE_TUNE=0 disables it, SPARKLE_MIXED_VARIANT=k
 * forces a variant. */
int sd_get_tuning(sd_ctx* ctx, int* variant, int* warps, int* min_blocks, double* ms, int n_ms);
/* ---- Structures from PDB files (the setup stage in front of the GSO path) ----
 * Reads the first structure of a PDB file as the reference's setup does (read_input_structure,
 * source/prep/src/read_input_structure.cc:60-307; generate_complex, source/prep/src/complex.cc;
 * init_center_translate + translate, source/prep/src/initialization.cc:3-29; get_nm_mask,
 * complex.cc:143-209; get_docking_model, source/dock/src/prepare_gso_tasks.cc:31-69): atoms of
 * the first MODEL, coordinates through float, centred on the mean of the non-hydrogen atoms, the
 * normal-mode mask (protein and nucleic residues), the DFIRE atom type of every atom and a
 * backbone flag (CA or P).  Errors: unreadable file, no atoms, unrecognised element, atom without
 * a DFIRE type. */
typedef struct sd_structure sd_structure;
#define SD_PDB_NOXT 1 /* ignore OXT atoms (setup.json "noxt") */
#define SD_PDB_NOH 2  /* ignore hydrogens ("noh") */
#define SD_PDB_NOW 4  /* ignore waters, HOH ("now") */
int sd_structure_load(const char* pdb_path, int flags, sd_structure** out);
int sd_structure_info(const sd_structure* s, int* n_atoms, int* n_residues);
/* Any output may be NULL: xyz [n][3] (centred), nm_mask [n], dfire_type [n], backbone [n],
 * translation [3] (the vector added to the file's coordinates). */
int sd_structure_arrays(const sd_structure* s, double* xyz, int* nm_mask, int* dfire_type, int* backbone,
                        double* translation);
int sd_structure_free(sd_structure* s);

/* One pose written as the reference writes its lightdock_<g>.pdb files (write_pdb,
 * source/dock/src/prepare_gso_tasks.cc:1279-1345; the pipeline variant's final writer,
 * source/dock/src/cuda/pipeline:2599-2750): the receptor's atoms then the ligand's, each numbered
 * from 1, every record with the fields as read (record name, atom name, alternate location,
 * residue name and number, chain, insertion code, occupancy, B-factor, element) and the given
 * coordinates [n_atoms][3] (e.g. from sd_materialise_poses), %.3f / %.2f in the PDB columns.
 * ligand and lig_xyz may both be NULL.  Fails where the reference's column padding would be
 * negative (it throws there): more than 99,999 atoms, a residue name over 3 characters, a residue
 * number over 4, or a coordinate that needs more than 8 columns. */
int sd_write_pose_pdb(const char* path, const sd_structure* receptor, const double* rec_xyz,
                      const sd_structure* ligand, const double* lig_xyz);

/* Normal modes of a structure (ANM), as the reference's setup computes them: cal_anm
 * (source/dock/src/cal_anm.cc:61-219) with its GPU eigensolver (source/dock/src/cuda/cal_anm.cu:
 * 28-91).  Coordinates re-centred on the mean of all atoms; CA atoms (else C4) as nodes; Hessian
 * with cutoff 15 A, gamma 1 (built on `device`); the lowest n_modes + 6 eigenpairs from
 * cuSOLVER syevd, those below 1e-6 dropped; every atom of residue i takes node i's components
 * (one CA per residue required); modes normalised, then scaled to `rmsd` with the reference's
 * draws over n_swarms x n_glowworms extents.  modes_out [n_modes][n_atoms][3] (the layout of
 * sd_complex_desc.rec_modes / lig_modes); xyz_out [n_atoms][3], the re-centred coordinates the
 * modes belong to (may be NULL); eigvals_out [n_modes] (may be NULL). */
int sd_anm(const sd_structure* s, int n_modes, double rmsd, int n_swarms, int n_glowworms, int device,
           double* modes_out, double* xyz_out, double* eigvals_out);
/* Khachiyan minimum-volume enclosing ellipsoid centre of n points (tolerance 0.01), the ligand
 * reference point of minimum_volume_ellipsoid (source/dock/src/prepare_gso_tasks.cc:106-267):
 * its operation order, including that of the Eigen 4x4 inverse it calls, so the centre is
 * bit-identical to the reference's (single-threaded) result; O(n) per iteration. */
int sd_reference_point(const double* xyz, int n, double* center);
/* The same centre computed on `device` (one CTA; the reference's summation orders kept), bit-identical
 * to sd_reference_point. */
int sd_reference_point_device(int device, const double* xyz, int n, double* center);
/* Seeded starting poses [n_swarms][n_glowworms][pose_len] around a receptor centred at the
 * origin, for synthetic complexes (no residues to place swarms on): swarm centres at uniform
 * directions on a shell 10 A outside its bounding sphere, each glowworm at its centre plus
 * N(0, 2 A) per axis, a uniform random unit quaternion and N(0, 1) ANM extents.  Structures read
 * from PDB files are placed by sd_place_swarms. */
int sd_starting_poses(const double* rec_xyz, int n_rec, int n_swarms, int n_glowworms, int n_modes_rec,
                      int n_modes_lig, unsigned long long seed, double* poses);

/* Swarm centres and starting poses as the reference's setup places them: calculate_start_pos
 * (source/dock/src/cal_anm.cc:775-990) with calculate_surface_point (:541-774) and the k-means
 * of source/dock/src/kmeans.cc:126-241, on the structures as read (before centring).  Surface
 * atoms clustered into n_swarms centroids (k-means++ from mt19937(324324), 100 Lloyd
 * iterations); 100 sphere points around each at the surface distance (10 A, or a quarter of the
 * ligand's diameter when that is >= 20 A), those near another centroid or within 3 A of the
 * receptor dropped; the rest clustered into the swarm centres (500 iterations), moved into the
 * centred frame.  Poses: per swarm and glowworm a point in the swarm_radius ball (lightdock's
 * default 10), a uniform quaternion (mt19937(starting_points_seed + rank) doubles) and, with
 * use_anm, N(0, 1) extents from std::default_random_engine(anm_seed), receptor modes first
 * (without use_anm the extents are 0).  The k-means and filters run on `device`, bit-identical
 * to the reference.  centers_out [n_swarms][3] (may be NULL); poses_out
 * [n_swarms][n_glowworms][7 + n_modes_rec + n_modes_lig] (may be NULL).  Fails where the
 * reference is undefined: no more surface atoms or kept points than swarms, or an empty cluster. */
int sd_place_swarms(const sd_structure* receptor, const sd_structure* ligand, int n_swarms, int n_glowworms,
                    int n_modes_rec, int n_modes_lig, int use_anm, int starting_points_seed, int anm_seed,
                    double swarm_radius, int rank, int device, double* centers_out, double* poses_out);

/* Every atom of chosen glowworms of complex complex_idx at their current (final) poses, through
 * the exact FP64 transforms the scorer uses (receptor ANM; ligand ANM, rotation, translation), as
 * the reference materialises the final poses for its lightdock_<g>.pdb files (prepare_receptor /
 * prepare_ligand after the last step, source/dock/src/cuda/pipeline:2492-2500).  poses[k] =
 * swarm * n_glowworms + glowworm; rec_xyz_out [n][n_rec][3] and lig_xyz_out [n][n_lig][3] in the
 * atom order of sd_complex_desc (either may be NULL). */
int sd_materialise_poses(sd_ctx* ctx, int complex_idx, const int* poses, int n, double* rec_xyz_out,
                         double* lig_xyz_out);

/* Final-pose clustering of every swarm of complex ci (BSAS, as the reference's GPU pipeline
 * variant clusters before writing cluster.repr, source/dock/src/cuda/pipeline:2766-2960):
 * glowworms ordered by score (descending; key (int64)(score * 2^50) / 2^12 * 2^12 + index), each
 * joins the first cluster whose representative (first member) is within 4 A backbone RMSD, else
 * starts a new cluster.  Backbone RMSD over the flagged atoms (rec_backbone [n_rec],
 * lig_backbone [n_lig], e.g. sd_structure_arrays' CA / P flags) of the final poses, receptor
 * then ligand, no superposition.  As in the reference, the first glowworm in score order is
 * compared with its own cluster again, so cluster 0's size counts it twice.  Outputs:
 * n_clusters [S]; cluster_rep, cluster_len [S][G] (first n_clusters[s] entries of each swarm are
 * used); member_of [S][G] (cluster of each glowworm). */
int sd_cluster(sd_ctx* ctx, int ci, const int* rec_backbone, const int* lig_backbone, int* n_clusters,
               int* cluster_rep, int* cluster_len, int* member_of);
/* <dir>/swarm_<offset+s>/cluster.repr for n_swarms swarms from sd_cluster's outputs and the
 * swarms' scores [S][G] ("<c>:<size>:<score>:<rep>:lightdock_<rep>.pdb" per cluster). */
int sd_write_cluster_repr(const char* dir, int swarm_offset, int n_swarms, int n_glowworms, const int* n_clusters,
                          const int* cluster_rep, const int* cluster_len, const double* scoring);

/* Number of compiled variants of the mixed-precision DFIRE kernel (valid SPARKLE_MIXED_VARIANT
 * values are 0 .. count-1; sd_get_tuning reports one time per variant). */
int sd_mixed_variant_count(void);
int sd_set_precision(sd_ctx* ctx, int precision);

/* Score n arbitrary poses of one complex ([n][pose_len], host): score (reference sign
 * convention, higher is better) and, if not NULL, raw energy and the ligand reference pose.
 * DFIRE: energy = sum of table values, score = -(0.0157*energy - 4.7).
 * PYDOCK: energy = E_elec + w_vdw*E_lj, score = -energy. */
int sd_score_poses(sd_ctx* ctx, int complex_idx, const double* poses, int n, int precision,
                   double* score_out, double* energy_out);

/* sd_score_poses without any allocation during the call, for callers that must not allocate
 * device memory while they score (work recorded into a CUDA graph by stream capture, or a
 * host framework whose memory manager owns all device memory in its steady state).  No
 * counterpart in the reference.  Inputs and outputs are the caller's DEVICE buffers on the
 * context's device: d_poses [n][pose_len], d_score [n], d_energy [n] (may be NULL), d_ref [n][3]
 * (ligand reference points).  n <= 65536 per call, else SD_ERR_ARG.  The scoring kernel's
 * bookkeeping (work list, counters, descriptor copy) lives in a 288 KiB file-scope device
 * array that every GPU loading this library holds until exit; all calls on a device share it
 * and each call rewrites it first, so calls whose GPU work overlaps (other streams or contexts
 * on the same device) race and must be ordered by the caller.  Runs on the context stream,
 * asynchronously unless sync != 0.  sync must be 0 while the stream is being captured (a
 * synchronisation would invalidate the capture; SD_ERR_ARG).  Poses must be finite: with
 * sync != 0 the call also counts non-finite pose values on the device and returns
 * SD_ERR_NUMERIC if there are any (the outputs of such a call are not meaningful); with sync == 0
 * nothing is checked.  These calls do not add to the counters of sd_get_stats.  The first call on
 * a device (and the first after a cudaDeviceReset) looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture. */
int sd_score_poses_noalloc(sd_ctx* ctx, int complex_idx, const double* d_poses, int n, int precision,
                           double* d_score, double* d_energy, double* d_ref, int sync);

/* Per-pair DFIRE bins of one pose (debug / parity): bins_out[i*n_lig + j] = table bin 0..19,
 * -1 when d^2 > 225.  Receptor order i and ligand order j are the caller's. */
int sd_dfire_bins(sd_ctx* ctx, int complex_idx, const double* pose, int precision, int* bins_out);

/* PYDOCK only: energy and its gradient with respect to the 6 rigid coordinates and the ANM
 * extents, grad_out[n][6 + n_modes_rec + n_modes_lig] =
 *   dE/dt (3), dE/dw (3; left tangent rotation q <- exp(w/2) q), dE/de_rec, dE/de_lig.
 * Project-defined (no reference counterpart). */
int sd_pydock_grad(sd_ctx* ctx, int complex_idx, const double* poses, int n, int precision,
                   double* energy_out, double* grad_out);

/* Result files of the reference GPU path (prepare_gso_task.cu:2838-2905): writes
 * <dir>/swarm_<swarm_offset+s>/gso_<steps>.out for s in [0, n_swarms) from host state arrays
 * ([S][G][pose_len] positions, [S][G] luciferin, neighbour counts, vision ranges, scores).
 * Host only; creates the swarm directories. */
int sd_write_gso_output(const char* dir, int swarm_offset, int n_swarms, int n_glowworms, int pose_len,
                        int steps, const double* pos, const double* luciferin, const int* nnei_len,
                        const double* vision_range, const double* scoring);

/* Checkpoints of one complex's GSO state, so that a long run can stop and resume (no counterpart
 * in the reference, which writes only its final files).  A versioned binary file of the sizes, the
 * number of GSO steps taken and the number the run was started with (the caller's counts; the
 * reference's draws [S][STEPS][G] depend on the latter), every field of sd_swarm_state, and a
 * 64-bit FNV-1a hash; it is written under a temporary name and renamed when complete.  Resume:
 * sd_read_checkpoint, sd_set_state, then sd_set_draws with the draws of the remaining steps
 * (u[s][t][g] for t >= steps_done of the same run's sd_gso_draws): the trajectory continues as if
 * uninterrupted.  sd_read_checkpoint fails on other sizes, a truncated or a corrupted file. Host
 * only; every field pointer of st is required; steps_done / steps_total outputs may be NULL. */
int sd_write_checkpoint(const char* path, int n_swarms, int n_glowworms, int pose_len, long long steps_done,
                        long long steps_total, const sd_swarm_state* st);
int sd_read_checkpoint(const char* path, int n_swarms, int n_glowworms, int pose_len, long long* steps_done,
                       long long* steps_total, sd_swarm_state* st);
int sd_checkpoint_info(const char* path, int* n_swarms, int* n_glowworms, int* pose_len, long long* steps_done,
                       long long* steps_total);

/* Optional post-GSO local refinement (pyDock-scoring contexts; project-defined, no reference
 * counterpart): `iters` steepest-descent steps on the smooth elec + LJ energy using the GPU
 * adjoint at `precision`, along the normalised gradient in (t, R_L*w, e_rec, e_lig) coordinates
 * (R_L the ligand radius, so every component moves in Angstrom-like units), starting at `step`
 * A.  A step is kept only when the plain FP64 energy of the moved pose is lower (then the
 * pose's step grows by 1.5x, else it halves), so the FP64 energy never increases.
 * poses [n][pose_len] in/out (host); energy_before / energy_after [n] FP64 energies (nullable). */
int sd_refine_poses(sd_ctx* ctx, int complex_idx, double* poses, int n, int iters, double step, int precision,
                    double* energy_before, double* energy_after);

/* Diagnostics: the correctly rounded acos (fn 0) and sin (fn 1) that the GSO update's slerp
 * (prepare_gso_tasks.cc:1370-1421) uses, evaluated by a device kernel on n host values x into
 * out (parity checking of the device arithmetic against a host restatement). */
int sd_crmath_eval(int device, int fn, const double* x, long long n, double* out);

/* ---- synthetic complexes (seeded), for tests and benchmarks ---- */
typedef struct {
  int n_rec, n_lig, n_swarms, n_glowworms, n_modes_rec, n_modes_lig;
  unsigned long long seed;
} sd_synth_spec;

/* Sizes a caller must allocate for sd_synth_generate: all arrays of sd_complex_desc plus
 * the starting poses [S][G][pose_len].  Returns the bytes of one contiguous buffer. */
int sd_synth_buffer_size(const sd_synth_spec* spec, long long* bytes);
/* Fills buf (sd_synth_buffer_size bytes) and points the fields of *desc into it; writes the
 * starting poses to *poses_out (inside buf). */
int sd_synth_generate(const sd_synth_spec* spec, void* buf, sd_complex_desc* desc,
                      double** poses_out);
/* Seeded synthetic DFIRE table N(0,1) [168*168*20] and LJ table [20] x2. */
int sd_synth_tables(unsigned long long seed, double* dfire_energy, double* lj_eps,
                    double* lj_sigma);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* SPARKLE_B200_H */
