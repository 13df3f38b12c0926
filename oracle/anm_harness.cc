// ORACLE test infrastructure only: drives the reference's own ANM code (cal_anm,
// source/dock/src/cal_anm.cc:61-219, with its GPU eigensolver source/dock/src/cuda/cal_anm.cu),
// compiled unmodified from the reference tree by oracle/Makefile, on a structure set up by the
// reference's own reader (read_input_structure, init_center_translate, translate, get_nm_mask).
// The reference's eigensolver ends with cudaDeviceReset(), so callers run this in a separate
// process.
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "anm.h"
#include "cal_anm.h"
#include "complex.h"
#include "freesasa.h"
#include "initialization.h"
#include "mpi.h"
#include "read_input_structure.h"
#include "swarm_centers.h"
#include "translate.h"

int MPI_Abort(MPI_Comm, int code) {
  std::fprintf(stderr, "MPI_Abort(%d) reached in the ANM harness\n", code);
  std::abort();
}
freesasa_structure* freesasa_structure_new(void) { std::abort(); }
freesasa_structure* freesasa_structure_from_pdb(FILE*, const void*, int) { std::abort(); }
int freesasa_structure_n(const freesasa_structure*) { std::abort(); }
freesasa_result* freesasa_calc_structure(const freesasa_structure*, const void*) { std::abort(); }

extern "C" {

// The reference's setup of one structure followed by cal_anm; copies out the modes
// [n_modes][n_atoms*3] and the coordinates after cal_anm's re-centring.  Returns the atom count
// (or -1 when over cap).
int ref_cal_anm(const char* path, int noxt, int noh, int now, int n_modes, double rmsd, int swarms, int glowworms,
                double* modes, double* xyz, int cap) {
  Complex c;
  read_input_structure(c, path, noxt != 0, noh != 0, now != 0, false, (int)strlen(path));
  init_center_translate(c.translation, c.atom_coordinates, c.elements, c.structure_size, c.num_atoms,
                        c.num_structures);
  translate(c.atom_coordinates, c.translation, c.structure_size, c.num_atoms, c.num_structures);
  get_nm_mask(c.mask, c.residue_name, c.STANDARD_TYPES, c.MODIFIED_TYPES, c.DNA_STANDARD_TYPES,
              c.RNA_STANDARD_TYPES, c.residue_atom_number, c.residue_size);
  ANM anm;
  cal_anm(c, anm, n_modes, rmsd, 324324, swarms, glowworms, 0, 1);
  const int n = c.num_atoms;
  if (n > cap) return -1;
  std::memcpy(modes, c.modes, sizeof(double) * (size_t)c.n_modes * n * 3);
  std::memcpy(xyz, c.atom_coordinates, sizeof(double) * (size_t)n * 3);
  return n;
}

// The reference's swarm placement (calculate_start_pos, source/dock/src/cal_anm.cc:775-990) on
// two structures set up as run_simulation does before it (read, centring translation computed but
// not applied): swarm centres [swarms][3] and poses [swarms][glowworms][7 + anm_rec + anm_lig].
// swarms > 0 (the SASA-derived count is not driven), no membrane, no dense sampling.
int ref_start_positions(const char* rec_path, const char* lig_path, int noxt, int noh, int now, int swarms,
                        int glowworms, int seed, int anm_seed, int anm_rec, int anm_lig, int use_anm,
                        double swarm_radius, double* centers, double* poses) {
  Complex rec, lig;
  read_input_structure(rec, rec_path, noxt != 0, noh != 0, now != 0, false, (int)strlen(rec_path));
  read_input_structure(lig, lig_path, noxt != 0, noh != 0, now != 0, false, (int)strlen(lig_path));
  init_center_translate(rec.translation, rec.atom_coordinates, rec.elements, rec.structure_size, rec.num_atoms,
                        rec.num_structures);
  init_center_translate(lig.translation, lig.atom_coordinates, lig.elements, lig.structure_size, lig.num_atoms,
                        lig.num_structures);
  SwarmCenters c;
  calculate_start_pos(c, rec, lig, swarms, glowworms, seed, rec.translation, lig.translation, 50.0, use_anm != 0,
                      anm_seed, anm_rec, anm_lig, false, false, false, swarm_radius, false, 0.0, 0, false, rec_path, 0,
                      1);
  std::memcpy(centers, c.s, sizeof(double) * 3 * c.swarms);
  const int pl = 7 + anm_rec + anm_lig;
  for (size_t i = 0; i < (size_t)c.swarms * glowworms; ++i)
    for (int k = 0; k < pl; ++k) poses[i * pl + k] = (k < 7 || use_anm) ? c.pos[i * pl + k] : 0.0;
  const int n = c.swarms;
  free_swarmcenters(c);
  return n;
}

// The reference's Hessian (build_hessian1D, cutoff 15, gamma 1) of n nodes [n][3] into H [3n][3n]; CPU.
void ref_build_hessian(const double* nodes, int n, double* H) {
  std::vector<double> coords(nodes, nodes + (size_t)n * 3), kirchhoff((size_t)n * n, 0.0);
  std::memset(H, 0, sizeof(double) * (size_t)9 * n * n);
  build_hessian1D(H, kirchhoff.data(), 15.0, 1.0, n, coords.data());
}

// The reference's norm (re-centring on the mean of all atoms) of xyz [n][3], in place; CPU.
void ref_norm(double* xyz, int n) { norm(xyz, n); }

// The extent normalisation cal_anm computes (its lines 166-182, one thread): the mean over n_draws
// of sqrt(sum_m v_m^2 / lambda_m), v from std::default_random_engine(324324) and
// std::normal_distribution(0, 1) of this C++ library.
double harness_extent_coef(const double* lam, int n_modes, long long n_draws) {
  std::default_random_engine generator;
  std::normal_distribution<double> distribution(0.0, 1.0);
  generator.seed(324324u);
  double coef = 0;
  for (long long i = 0; i < n_draws; ++i) {
    double sum = 0;
    for (int j = 0; j < n_modes; ++j) {
      const double v = distribution(generator);
      sum += v * v * (1.0 / lam[j]);
    }
    coef += std::sqrt(sum);
  }
  return coef / n_draws;
}

}  // extern "C"
