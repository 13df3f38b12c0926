// ORACLE — test infrastructure only.  Drives the reference's own compiled CPU functions
// (source/dock/src/prepare_gso_tasks.cc, compiled unmodified from the reference tree by
// oracle/Makefile into oracle/_ref/) so that the C restatement in sd_oracle.c can be checked
// against them, and so that the reference's CPU scoring path can be timed as a baseline.
//
// Called functions of the reference:  cdfire_calculate_dfire (:1522), rotate (:277),
// slerp (:1370), move_extent (:1352), compute_probability_moving_from_neighbors (:1463),
// select_random_neighbor (:1424), minimum_volume_ellipsoid (:106), cal_gso_tasks_cpu (:359).
// The ANM loops and the three-pass step driver live inline in cal_gso_tasks_cpu
// (:429-819); ref_gso_step restates them statement for statement, with the number of steps
// as a parameter, and calls the functions above for everything else.
#include <omp.h>
#include <sys/wait.h>
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <string>
#include <vector>

#include "complex.h"
#include "fastdfire.h"
#include "initialization.h"
#include "read_input_structure.h"
#include "translate.h"
#include "prepare_gso_tasks.h"
#include "swarm_centers.h"

extern "C" {
#include "sd_oracle.h"
}

void minimum_volume_ellipsoid(double* center, double* poles, double* atom_coordinates, double precision,
                              int num_atoms);

// The reference translation unit calls the GPU path when USE_CUDA is set; the harness never
// sets it.  The symbol must still resolve for the shared library to load.
void cal_gso_tasks_gpu(SwarmCenters&, Complex&, Complex&, FastDifire&, int, double, double, bool, double, int,
                       int, bool, int, int, double*, double*, double*, double*, int*, int*, int, int, int, int) {
  fprintf(stderr, "ref harness: GPU path not available\n");
  abort();
}

namespace {

// pose of one glowworm with the reference's inline ANM loops and its rotate()
void ref_pose(const or_system* s, const double* pose, double* rec, double* lig, double* ref) {
  memcpy(rec, s->rec_xyz, sizeof(double) * 3 * s->nr);
  memcpy(lig, s->lig_xyz, sizeof(double) * 3 * s->nl);
  ref[0] = s->lig_ref[0];
  ref[1] = s->lig_ref[1];
  ref[2] = s->lig_ref[2];
  for (int j = 0; j < s->nmr; j++) {
    const double* rep_modes = &s->rec_modes[(size_t)j * s->nr * 3];
    double rec_instant = pose[7 + j];
    for (int p = 0; p < s->nr; p++) {
      if (s->rec_mask[p] == 1) {
        rec[p * 3] += rep_modes[p * 3] * rec_instant;
        rec[p * 3 + 1] += rep_modes[p * 3 + 1] * rec_instant;
        rec[p * 3 + 2] += rep_modes[p * 3 + 2] * rec_instant;
      }
    }
  }
  for (int j = 0; j < s->nml; j++) {
    const double* rep_modes = &s->lig_modes[(size_t)j * s->nl * 3];
    double rec_instant = pose[7 + s->nmr + j];
    for (int p = 0; p < s->nl; p++) {
      if (s->lig_mask[p] == 1) {
        lig[p * 3] += rep_modes[p * 3] * rec_instant;
        lig[p * 3 + 1] += rep_modes[p * 3 + 1] * rec_instant;
        lig[p * 3 + 2] += rep_modes[p * 3 + 2] * rec_instant;
      }
    }
  }
  double q[4] = {pose[3], pose[4], pose[5], pose[6]};
  rotate(lig, q, s->nl);
  rotate(ref, q, 1);
  for (int ii = 0; ii < s->nl; ii++) {
    lig[ii * 3] += pose[0];
    lig[ii * 3 + 1] += pose[1];
    lig[ii * 3 + 2] += pose[2];
  }
  ref[0] += pose[0];
  ref[1] += pose[1];
  ref[2] += pose[2];
}

double ref_dfire(const or_system* s, FastDifire& fd, double* rec, double* lig) {
  double energy = 0.0;
  int idx_len = 0;
  cdfire_calculate_dfire(&energy, idx_len, nullptr, nullptr, const_cast<int*>(s->rec_type),
                         const_cast<int*>(s->lig_type), fd, rec, lig, s->nr, s->nl, -1, -1);
  return energy;
}

}  // namespace

extern "C" {

// score one pose with the reference's transform + scorer; returns the score
double ref_score_pose(const or_system* s, const double* pose, double* ref_out, double* rec_out, double* lig_out) {
  FastDifire fd;
  fd.difire_energy = const_cast<double*>(s->table);
  double* rec = new double[3 * s->nr];
  double* lig = new double[3 * s->nl];
  double ref[3];
  ref_pose(s, pose, rec, lig, ref);
  double e = ref_dfire(s, fd, rec, lig);
  if (ref_out) memcpy(ref_out, ref, sizeof ref);
  if (rec_out) memcpy(rec_out, rec, sizeof(double) * 3 * s->nr);
  if (lig_out) memcpy(lig_out, lig, sizeof(double) * 3 * s->nl);
  delete[] rec;
  delete[] lig;
  return e;  // already the score: cdfire_calculate_dfire applies -(0.0157 E - 4.7)
}

void ref_slerp(double* self, double* other, double step) { slerp(self, other, step); }

// The reference's draws: std::mt19937(seed) and std::uniform_real_distribution<double>(0,1)
// in the order of prepare_gso_tasks.cc:411-427.
void ref_gso_draws(unsigned int seed, int S, int steps, int G, double* out) {
  std::uniform_real_distribution<double> distribution(0.0, 1.0);
  std::mt19937 gen(seed);
  for (int i = 0; i < S; i++)
    for (int s = 0; s < steps; s++)
      for (int j = 0; j < G; j++) out[(size_t)i * steps * G + (size_t)s * G + j] = distribution(gen);
}

// One GSO step, restating cal_gso_tasks_cpu's three passes (prepare_gso_tasks.cc:429-819)
// over the reference's helper functions.  nthreads parallelises pass 1 over swarms as the
// reference does (:432).  Returns the number of poses rescored.
long long ref_gso_step(const or_system* s, or_state* st, const double* u_step, int nthreads) {
  const int S = s->S, G = s->G, pl = 7 + s->nmr + s->nml;
  FastDifire fd;
  fd.difire_energy = const_cast<double*>(s->table);
  long long scored = 0;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic) reduction(+ : scored)
  for (int i = 0; i < S; i++) {
    double* rec = new double[3 * s->nr];
    double* lig = new double[3 * s->nl];
    for (int g = 0; g < G; g++) {
      int k = i * G + g;
      double* pos = &st->pos[(size_t)k * pl];
      if (st->moved[k] || st->step[k] == 0) {
        ref_pose(s, pos, rec, lig, &st->ref[(size_t)k * 3]);
        st->scoring[k] = ref_dfire(s, fd, rec, lig);
        scored++;
      }
      st->luciferin[k] = (1.0 - s->rho) * st->luciferin[k] + s->gamma * st->scoring[k];
      st->step[k] += 1;
    }
    delete[] rec;
    delete[] lig;
  }
  double* sel_pos = new double[(size_t)S * G * pl];
  int* neighbors = new int[G];
  for (int i = 0; i < S; i++) {
    for (int g = 0; g < G; g++) {
      int k = i * G + g;
      double* cur = &st->ref[(size_t)k * 3];
      memset(neighbors, 0, sizeof(int) * G);
      double sq = st->vision[k] * st->vision[k];
      int nn = 0;
      for (int n = 0; n < G; n++) {
        if (n != g && st->luciferin[k] < st->luciferin[i * G + n]) {
          double* nr = &st->ref[((size_t)i * G + n) * 3];
          double distance = 0;
          for (int d = 0; d < 3; d++) distance += ((cur[d] - nr[d]) * (cur[d] - nr[d]));
          if (distance < sq) neighbors[nn++] = n;
        }
      }
      st->nnei[k] = nn;
      double* probabilities = new double[nn + 1];
      compute_probability_moving_from_neighbors(probabilities, neighbors, &st->luciferin[(size_t)i * G], nn,
                                                st->luciferin[k]);
      int select_local[1];
      // select_random_neighbor writes select[n]; give it a one-slot array at index 0
      int* sel_arr = new int[G];
      select_random_neighbor(sel_arr, u_step[k], neighbors, probabilities, 0, g, nn, -1);
      st->select[k] = sel_arr[g];
      (void)select_local;
      delete[] sel_arr;
      delete[] probabilities;
      memcpy(&sel_pos[(size_t)k * pl], &st->pos[((size_t)i * G + st->select[k]) * pl], sizeof(double) * pl);
    }
  }
  delete[] neighbors;
  for (int i = 0; i < S; i++) {
    for (int g = 0; g < G; g++) {
      int k = i * G + g;
      int nei = st->select[k];
      double* cur = &st->pos[(size_t)k * pl];
      double* mv = &sel_pos[(size_t)k * pl];
      st->moved[k] = g != nei;
      if (g != nei) {
        double delta[3], n = 0;
        for (int d = 0; d < 3; d++) {
          delta[d] = mv[d] - cur[d];
          n += (delta[d] * delta[d]);
        }
        n = sqrt(n);
        if (n >= 1e-8) {
          for (int d = 0; d < 3; d++) {
            delta[d] *= (s->step_t / n);
            cur[d] += delta[d];
          }
        }
        slerp(&cur[3], &mv[3], s->step_r);
        move_extent(&cur[7], &mv[7], s->nmr, s->step_nm);
        move_extent(&cur[7 + s->nmr], &mv[7 + s->nmr], s->nml, s->step_nm);
      }
      st->vision[k] = st->vision[k] + s->beta * (s->max_neighbors - st->nnei[k]);
      if (st->vision[k] < 0.0) st->vision[k] = 0;
      if (st->vision[k] > s->max_vision) st->vision[k] = s->max_vision;
    }
  }
  delete[] sel_pos;
  return scored;
}

// Ligand reference point with the reference's Khachiyan ellipsoid (:106-267, precision 0.01
// as at :1196).
void ref_min_volume_ellipsoid(const double* xyz, int n, double* center, double* poles) {
  minimum_volume_ellipsoid(center, poles, const_cast<double*>(xyz), 0.01, n);
}

// Runs the unmodified cal_gso_tasks_cpu (STEPS = 3 compiled in, ends with exit(0)) in a
// forked child with USE_CUDA unset and returns its stdout (the reference's printf probes)
// in buf.  The starting poses are pos0 [S][G][pl].  Returns the child's exit status or -1.
int ref_run_cal_gso_tasks_cpu(const or_system* s, const double* pos0, int nthreads, char* buf, int buflen) {
  int fds[2];
  if (pipe(fds) != 0) return -1;
  fflush(stdout);
  pid_t pid = fork();
  if (pid < 0) return -1;
  if (pid == 0) {
    close(fds[0]);
    dup2(fds[1], 1);
    unsetenv("USE_CUDA");
    Complex rec, lig;
    rec.num_atoms = s->nr;
    lig.num_atoms = s->nl;
    rec.atom_coordinates = const_cast<double*>(s->rec_xyz);
    lig.atom_coordinates = const_cast<double*>(s->lig_xyz);
    rec.mask = const_cast<int*>(s->rec_mask);
    lig.mask = const_cast<int*>(s->lig_mask);
    rec.modes = const_cast<double*>(s->rec_modes);
    lig.modes = const_cast<double*>(s->lig_modes);
    FastDifire fd;
    fd.difire_energy = const_cast<double*>(s->table);
    SwarmCenters c;
    int pl = 7 + s->nmr + s->nml;
    c.pos = new double[(size_t)s->S * s->G * pl];
    memcpy(c.pos, pos0, sizeof(double) * (size_t)s->S * s->G * pl);
    c.pos_len = s->G * pl;
    c.anm_rec = s->nmr;
    c.anm_lig = s->nml;
    c.swarms = s->S;
    c.swarm_start = 0;
    c.swarm_chunk = s->S;
    double rref[3] = {0, 0, 0}, rpoles[18] = {0}, lref[3] = {s->lig_ref[0], s->lig_ref[1], s->lig_ref[2]},
           lpoles[18] = {0};
    char nt[16];
    snprintf(nt, sizeof nt, "%d", nthreads);
    setenv("NUM_THREADS", nt, 1);
    cal_gso_tasks_cpu(c, rec, lig, fd, 0, 0.5, 0.5, true, 0.5, s->nmr, s->nml, false, s->S, s->G, rref, rpoles, lref,
                      lpoles, const_cast<int*>(s->rec_type), const_cast<int*>(s->lig_type));
    _exit(3);  // not reached: the reference ends with exit(0)
  }
  close(fds[1]);
  int off = 0;
  while (off < buflen - 1) {
    ssize_t r = read(fds[0], buf + off, buflen - 1 - off);
    if (r <= 0) break;
    off += (int)r;
  }
  buf[off] = 0;
  // drain anything left so the child never blocks on a full pipe
  char sink[4096];
  while (read(fds[0], sink, sizeof sink) > 0) {
  }
  close(fds[0]);
  int status = 0;
  waitpid(pid, &status, 0);
  return WIFEXITED(status) ? WEXITSTATUS(status) : -1;
}

// The reference's own setup chain for one structure, as run_simulation.cc:53-79 and
// prepare_gso_tasks.cc:1177-1188 run it: read_input_structure, init_center_translate, translate,
// get_nm_mask, get_docking_model.  Copies out up to cap atoms; returns the atom count (or -1).
int ref_load_structure(const char* path, int noxt, int noh, int now, double* xyz, int* mask, int* dfire,
                       double* translation, int cap) {
  Complex c;
  read_input_structure(c, path, noxt != 0, noh != 0, now != 0, false, (int)strlen(path));
  init_center_translate(c.translation, c.atom_coordinates, c.elements, c.structure_size, c.num_atoms,
                        c.num_structures);
  translate(c.atom_coordinates, c.translation, c.structure_size, c.num_atoms, c.num_structures);
  get_nm_mask(c.mask, c.residue_name, c.STANDARD_TYPES, c.MODIFIED_TYPES, c.DNA_STANDARD_TYPES,
              c.RNA_STANDARD_TYPES, c.residue_atom_number, c.residue_size);
  FastDifire fd;
  const int nobj = (int)c.chain.size() * c.residue_atom_number[c.num_res_type];
  int* objs = new int[nobj > 0 ? nobj : 1];
  get_docking_model(objs, c, fd);
  const int n = c.num_atoms;
  if (n > cap) {
    delete[] objs;
    return -1;
  }
  memcpy(xyz, c.atom_coordinates, sizeof(double) * 3 * n);
  memcpy(mask, c.mask, sizeof(int) * n);
  memcpy(dfire, objs, sizeof(int) * n);
  memcpy(translation, c.translation, sizeof(double) * 3);
  delete[] objs;
  return n;
}

// The reference's pose file writer (write_pdb, prepare_gso_tasks.cc:1279-1345, the format of the
// pipeline's lightdock_<g>.pdb files) for a receptor and a ligand read by read_input_structure,
// with the given coordinates [n][3] of each, into out_path (receptor atoms, then ligand atoms).
// Returns 0, or -1 when the file cannot be opened.
int ref_write_pose_pdb(const char* rec_path, const char* lig_path, int noxt, int noh, int now,
                       const double* rec_xyz, const double* lig_xyz, const char* out_path) {
  Complex r, l;
  read_input_structure(r, rec_path, noxt != 0, noh != 0, now != 0, false, (int)strlen(rec_path));
  read_input_structure(l, lig_path, noxt != 0, noh != 0, now != 0, false, (int)strlen(lig_path));
  std::ofstream f(out_path);
  if (!f.is_open()) return -1;
  std::vector<double> rc(rec_xyz, rec_xyz + (size_t)3 * r.num_atoms), lc(lig_xyz, lig_xyz + (size_t)3 * l.num_atoms);
  write_pdb(r, f, rc.data());
  write_pdb(l, f, lc.data());
  return 0;
}

}  // extern "C"
