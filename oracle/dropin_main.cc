// Test infrastructure: a main-shaped driver of the reference's own hot-path entry point, for the
// drop-in test.  It follows the reference's main (source/simulation/run_simulation.cc:48-114) for
// one rank without MPI: read_input_structure, init_center_translate, translate and get_nm_mask on
// both structures (the reference's own code, compiled from its sources), then
// prepare_gso_tasks (source/dock/src/prepare_gso_tasks.cc:1151-1256, compiled unmodified), which
// loads ./data/DCparams, types the atoms, computes the ellipsoid reference points and, with
// USE_CUDA set, calls cal_gso_tasks_gpu -- here the binding linked in its place
// (sparkledock_b200/bindings/cal_gso_tasks_b200.cc) over libsparkle_b200.so.
//
// The swarm placement and the normal modes, which the reference's main computes before the call
// (calculate_start_pos, cal_anm), are read from files instead, so that the test fixes them:
//   dropin_run receptor.pdb ligand.pdb poses.bin swarms glowworms n_modes_rec n_modes_lig
//              [rec_modes.bin lig_modes.bin]
// poses.bin: doubles [swarms][glowworms][7 + n_modes_rec + n_modes_lig]; *_modes.bin: doubles
// [n_modes][atoms][3].
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "complex.h"
#include "fastdfire.h"
#include "initialization.h"
#include "prepare_gso_tasks.h"
#include "read_input_structure.h"
#include "swarm_centers.h"
#include "translate.h"

static double* read_doubles(const char* path, size_t n) {
  FILE* f = fopen(path, "rb");
  if (!f) return nullptr;
  double* p = new double[n];
  const size_t got = fread(p, sizeof(double), n, f);
  fclose(f);
  if (got != n) {
    delete[] p;
    return nullptr;
  }
  return p;
}

static void setup(Complex& c, const char* path) {
  read_input_structure(c, path, false, false, false, false, (int)strlen(path));
  init_center_translate(c.translation, c.atom_coordinates, c.elements, c.structure_size, c.num_atoms,
                        c.num_structures);
  translate(c.atom_coordinates, c.translation, c.structure_size, c.num_atoms, c.num_structures);
  get_nm_mask(c.mask, c.residue_name, c.STANDARD_TYPES, c.MODIFIED_TYPES, c.DNA_STANDARD_TYPES,
              c.RNA_STANDARD_TYPES, c.residue_atom_number, c.residue_size);
  c.n_modes = 0;
  c.modes = nullptr;
}

int main(int argc, char** argv) {
  if (argc != 8 && argc != 10) {
    fprintf(stderr, "usage: dropin_run rec.pdb lig.pdb poses.bin swarms glowworms nm_rec nm_lig [rec_modes lig_modes]\n");
    return 2;
  }
  const int S = atoi(argv[4]), G = atoi(argv[5]), nmr = atoi(argv[6]), nml = atoi(argv[7]);
  const int pl = 7 + nmr + nml;
  Complex receptor, ligand;
  setup(receptor, argv[1]);
  setup(ligand, argv[2]);
  if (argc == 10) {
    receptor.n_modes = nmr;
    ligand.n_modes = nml;
    receptor.modes = read_doubles(argv[8], (size_t)nmr * receptor.num_atoms * 3);
    ligand.modes = read_doubles(argv[9], (size_t)nml * ligand.num_atoms * 3);
    if (!receptor.modes || !ligand.modes) {
      fprintf(stderr, "dropin_run: cannot read the mode files\n");
      return 2;
    }
  }
  SwarmCenters centers;
  memset(&centers, 0, sizeof centers);
  centers.swarms = S;
  centers.swarm_start = 0;
  centers.swarm_chunk = S;
  centers.pos_len = G * pl;
  centers.anm_rec = nmr;
  centers.anm_lig = nml;
  centers.pos = read_doubles(argv[3], (size_t)S * G * pl);
  if (!centers.pos) {
    fprintf(stderr, "dropin_run: cannot read the poses\n");
    return 2;
  }
  FastDifire score;
  // run_simulation.cc:106-109: anm_seed, translation and rotation steps, use_anm, nmodes_step, the
  // mode counts, local minimisation, swarms, glowworms, rank, size
  prepare_gso_tasks(centers, receptor, ligand, score, 324324, 0.5, 0.5, argc == 10, 0.5, nmr, nml, false, S, G, 0, 1);
  printf("dropin_run: done, %d swarms x %d glowworms\n", S, G);
  return 0;
}
