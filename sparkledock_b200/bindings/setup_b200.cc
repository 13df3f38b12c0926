// setup_b200.cc -- the reference-side binding of the setup stages in front of the GSO path.
//
// Replaces calculate_start_pos (source/dock/src/cal_anm.cc:775-990) and cal_anm
// (source/dock/src/cal_anm.cc:61-219) in the reference's main (source/simulation/run_simulation.cc),
// called after get_nm_mask.  sd_place_swarms reads the structures as the reference does and returns
// the swarm centres in the centred frame, as calculate_start_pos leaves them; sd_anm re-centres
// each structure as cal_anm does and writes the coordinates back.  Returns false (with a message)
// where the reference would abort or is undefined.
#include <cstdio>

#include "complex.h"  // reference headers
#include "config_args.h"
#include "swarm_centers.h"
#include "sparkle_b200.h"

bool setup_b200(const ConfigArgs& args, SwarmCenters& centers, Complex& receptor, Complex& ligand, int rank,
                int size) {
  const int flags = (args.noxt ? SD_PDB_NOXT : 0) | (args.noh ? SD_PDB_NOH : 0) | (args.now ? SD_PDB_NOW : 0);
  sd_structure* r = nullptr;
  sd_structure* l = nullptr;
  int ndev = 0;
  sd_device_count(&ndev);
  const int device = ndev ? rank % ndev : 0;
  const int nmr = args.use_anm ? args.anm_rec : 0, nml = args.use_anm ? args.anm_lig : 0;
  const int pl = 7 + args.anm_rec + args.anm_lig;
  bool ok = sd_structure_load(args.receptor_pdb.c_str(), flags, &r) == SD_OK &&
            sd_structure_load(args.ligand_pdb.c_str(), flags, &l) == SD_OK;
  if (ok) {
    centers.swarms = args.swarms;
    centers.anm_rec = args.anm_rec;
    centers.anm_lig = args.anm_lig;
    centers.pos_len = args.glowworms * pl;
    centers.s = new double[(size_t)args.swarms * 3];
    centers.pos = new double[(size_t)args.swarms * args.glowworms * pl];
    // the reference's static swarm partition over ranks (cal_anm.cc:621-626)
    const int base = args.swarms / size, extra = args.swarms % size;
    centers.swarm_chunk = rank < extra ? base + 1 : base;
    centers.swarm_start = rank < extra ? rank * (base + 1) : extra * (base + 1) + (rank - extra) * base;
    ok = sd_place_swarms(r, l, args.swarms, args.glowworms, args.anm_rec, args.anm_lig, args.use_anm ? 1 : 0,
                         args.starting_points_seed, args.anm_seed, args.swarm_radius, rank, device, centers.s,
                         centers.pos) == SD_OK;
  }
  if (ok && nmr > 0) {
    receptor.n_modes = nmr;
    receptor.modes = new double[(size_t)nmr * receptor.num_atoms * 3];
    ok = sd_anm(r, nmr, args.anm_rec_rmsd, args.swarms, args.glowworms, device, receptor.modes,
                receptor.atom_coordinates, nullptr) == SD_OK;
  }
  if (ok && nml > 0) {
    ligand.n_modes = nml;
    ligand.modes = new double[(size_t)nml * ligand.num_atoms * 3];
    ok = sd_anm(l, nml, args.anm_lig_rmsd, args.swarms, args.glowworms, device, ligand.modes,
                ligand.atom_coordinates, nullptr) == SD_OK;
  }
  if (!ok) fprintf(stderr, "sparkle_b200: %s\n", sd_last_error());
  sd_structure_free(r);
  sd_structure_free(l);
  return ok;
}
