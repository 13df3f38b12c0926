// Seeded synthetic docking systems: compact globular "proteins", DFIRE/LJ tables, ANM modes,
// swarm centres and starting poses.  Stands in for the reference's PDB parsing + ANM + surface
// sampling setup (source/dock/src/cal_anm.cc:61-219, :541-900), which the hot path only
// consumes through Complex fields and SwarmCenters.pos.
//
// Globule: N points uniform in a sphere of radius 2.2*N^(1/3) A by rejection sampling with a
// 3.0 A minimum separation (cell grid), centred on their centroid (as init_center_translate +
// translate do, prepare: run_simulation.cc:58-59, :77-78).  Starting poses follow
// calculate_start_pos (cal_anm.cc:833-896): Shoemake quaternion in the reference's component
// order, N(0,1) ANM extents; the translation is the swarm centre plus N(0, 2 A) per axis.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include "sd_internal.h"
#include "sd_mvee.h"

namespace sd {

namespace {

struct Rng {
  std::mt19937_64 g;
  explicit Rng(uint64_t s) : g(s) {}
  double uniform() { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
  double normal() {  // Box-Muller
    double u1 = 1.0 - uniform();  // (0,1]
    double u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
  int below(int n) { return (int)(uniform() * n); }
};

void globule(Rng& r, int n, double* xyz) {
  const double R = 2.2 * std::cbrt((double)n);
  const double dmin = 3.0, dmin2 = dmin * dmin;
  const int nc = (int)std::ceil(2.0 * R / dmin) + 1;
  std::vector<std::vector<int>> cells((size_t)nc * nc * nc);
  auto cell_of = [&](double v) { return std::min(nc - 1, std::max(0, (int)((v + R) / dmin))); };
  int placed = 0;
  long long attempts = 0;
  while (placed < n) {
    double x = (2 * r.uniform() - 1) * R, y = (2 * r.uniform() - 1) * R, z = (2 * r.uniform() - 1) * R;
    ++attempts;
    if (x * x + y * y + z * z > R * R) continue;
    int cx = cell_of(x), cy = cell_of(y), cz = cell_of(z);
    bool ok = true;
    for (int a = std::max(0, cx - 1); a <= std::min(nc - 1, cx + 1) && ok; ++a)
      for (int b = std::max(0, cy - 1); b <= std::min(nc - 1, cy + 1) && ok; ++b)
        for (int c = std::max(0, cz - 1); c <= std::min(nc - 1, cz + 1) && ok; ++c)
          for (int k : cells[((size_t)a * nc + b) * nc + c]) {
            double dx = xyz[k * 3] - x, dy = xyz[k * 3 + 1] - y, dz = xyz[k * 3 + 2] - z;
            if (dx * dx + dy * dy + dz * dz < dmin2) {
              ok = false;
              break;
            }
          }
    if (!ok) continue;
    xyz[placed * 3] = x;
    xyz[placed * 3 + 1] = y;
    xyz[placed * 3 + 2] = z;
    cells[((size_t)cx * nc + cy) * nc + cz].push_back(placed);
    ++placed;
  }
  double c[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) c[d] += xyz[i * 3 + d];
  for (int d = 0; d < 3; ++d) c[d] /= n;
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) xyz[i * 3 + d] -= c[d];
}

// nm orthonormal 3N-vectors by modified Gram-Schmidt on Gaussian vectors
void modes(Rng& r, int n, int nm, double* m) {
  const size_t len = (size_t)n * 3;
  for (int k = 0; k < nm; ++k) {
    double* v = m + k * len;
    for (size_t i = 0; i < len; ++i) v[i] = r.normal();
    for (int p = 0; p < k; ++p) {
      const double* u = m + p * len;
      double dot = 0;
      for (size_t i = 0; i < len; ++i) dot += u[i] * v[i];
      for (size_t i = 0; i < len; ++i) v[i] -= dot * u[i];
    }
    double nrm = 0;
    for (size_t i = 0; i < len; ++i) nrm += v[i] * v[i];
    nrm = std::sqrt(nrm);
    for (size_t i = 0; i < len; ++i) v[i] /= nrm;
  }
}

void atoms(Rng& r, int n, int* type, double* charge, int* lj, int* mask) {
  for (int i = 0; i < n; ++i) type[i] = r.below(SD_DFIRE_TYPES);
  for (int i = 0; i < n; ++i) {
    double u = r.uniform();
    charge[i] = u < 0.05 ? -1.0 : u < 0.20 ? -0.5 : u < 0.80 ? 0.0 : u < 0.95 ? 0.5 : 1.0;
  }
  for (int i = 0; i < n; ++i) lj[i] = r.below(SD_LJ_TYPES);
  // ANM mask: 1 for standard residues in the reference (get_nm_mask); a few 0s here
  for (int i = 0; i < n; ++i) mask[i] = r.uniform() < 0.03 ? 0 : 1;
}

}  // namespace

// Starting poses: swarm centres at independent uniform directions on a shell 10 A outside the
// receptor's bounding sphere (receptor centred at the origin), each glowworm at its centre plus
// N(0, 2 A) per axis, a uniform random unit quaternion (Shoemake) and N(0, 1) ANM extents.
void starting_poses(Rng& rs, const double* rec_xyz, int n_rec, int S, int G, int nmr, int nml, double* poses) {
  double rmax = 0;
  for (int i = 0; i < n_rec; ++i)
    rmax = std::max(rmax, std::sqrt(rec_xyz[i * 3] * rec_xyz[i * 3] + rec_xyz[i * 3 + 1] * rec_xyz[i * 3 + 1] +
                                    rec_xyz[i * 3 + 2] * rec_xyz[i * 3 + 2]));
  const double shell = rmax + 10.0;
  const int pl = SD_POSE_LEN(nmr, nml);
  const double PI = 3.14159265358979323846;
  for (int sw = 0; sw < S; ++sw) {
    double v[3], n2 = 0;
    do {
      n2 = 0;
      for (int k = 0; k < 3; ++k) {
        v[k] = rs.normal();
        n2 += v[k] * v[k];
      }
    } while (n2 < 1e-12);
    double nrm = std::sqrt(n2);
    double c[3] = {v[0] / nrm * shell, v[1] / nrm * shell, v[2] / nrm * shell};
    for (int g = 0; g < G; ++g) {
      double* p = poses + ((size_t)sw * G + g) * pl;
      for (int k = 0; k < 3; ++k) p[k] = c[k] + 2.0 * rs.normal();
      double u1 = rs.uniform(), u2 = rs.uniform(), u3 = rs.uniform();
      p[3] = std::sqrt(1 - u1) * std::sin(2 * PI * u2);
      p[4] = std::sqrt(1 - u1) * std::cos(2 * PI * u2);
      p[5] = std::sqrt(u1) * std::sin(2 * PI * u3);
      p[6] = std::sqrt(u1) * std::cos(2 * PI * u3);
      for (int k = 0; k < nmr + nml; ++k) p[7 + k] = rs.normal();
    }
  }
}



// Khachiyan's minimum-volume enclosing ellipsoid centre with tolerance tol, in the operation
// order of the reference's minimum_volume_ellipsoid (prepare_gso_tasks.cc:106-267, with its
// helpers multiplyDiagonalMatrix / multiplyMatrices / transpose, :71-104, one thread), so the
// centre is bit-identical to the reference's:
//   q_i = (x_i, y_i, z_i, 1), u_i = 1/N;  V[a][b] = sum_i q_i[a] * (q_i[b] * u_i) (ascending i);
//   A = the 4x4 matrix whose column-major data is V, inverted as above;
//   m_i = sum_k q_i[k] * (sum_m Ainv(m, k) * q_i[m]);  j = first index of the largest m_i (> 0);
//   step = ((m_j - 3) - 1) / (4 (m_j - 1));  u <- (1 - step) u, u_j += step;
//   error = sqrt(sum_i (u_new - u_old)^2);  repeat while error > tol;
//   centre[d] = sum_i p_i[d] * u_i.
// Only the diagonal m_i of the reference's N x N product is formed (each entry is computed the
// same way whether or not the rest of the matrix is), O(N) per iteration.
void mvee_center(const double* p, int n, double tol, double* center) {
  std::vector<double> u(n, 1.0 / n), nu(n), w((size_t)4 * n);
  double err = 1 + tol;
  int it = 0;
  auto q = [&](int i, int a) { return a == 3 ? 1.0 : p[(size_t)i * 3 + a]; };
  while (err > tol && it < 100000) {
    ++it;
    double V[16];
    for (int a = 0; a < 4; ++a)
      for (int i = 0; i < n; ++i) w[(size_t)a * n + i] = q(i, a) * u[i];
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        double sum = 0.0;
        for (int i = 0; i < n; ++i) sum += q(i, a) * w[(size_t)b * n + i];
        V[a * 4 + b] = sum;
      }
    double X[16];
    sd_inverse4_lu(V, X);
    double mx = 0.0;
    int j = 0;
    for (int i = 0; i < n; ++i) {
      double t[4];
      for (int k = 0; k < 4; ++k) {
        double sum = 0.0;
        for (int m = 0; m < 4; ++m) sum += X[k * 4 + m] * q(i, m);
        t[k] = sum;
      }
      double m = 0.0;
      for (int k = 0; k < 4; ++k) m += q(i, k) * t[k];
      if (m > mx) {
        mx = m;
        j = i;
      }
    }
    const double step = (mx - 3 - 1.0) / ((3 + 1.0) * (mx - 1.0));
    for (int i = 0; i < n; ++i) nu[i] = (1.0 - step) * u[i];
    nu[j] += step;
    double e2 = 0.0;
    for (int i = 0; i < n; ++i) e2 += (nu[i] - u[i]) * (nu[i] - u[i]);
    err = std::sqrt(e2);
    u.swap(nu);
  }
  for (int d = 0; d < 3; ++d) {
    double c = 0.0;
    for (int i = 0; i < n; ++i) c += p[(size_t)i * 3 + d] * u[i];
    center[d] = c;
  }
}

}  // namespace sd

namespace {
struct Layout {
  size_t rec_xyz, lig_xyz, rec_modes, lig_modes, rec_charge, lig_charge, poses;
  size_t rec_mask, lig_mask, rec_type, lig_type, rec_lj, lig_lj, total;
};
Layout layout_of(const sd_synth_spec* s) {
  Layout L;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~(size_t)255;
    return o;
  };
  const size_t nr = s->n_rec, nl = s->n_lig, pl = SD_POSE_LEN(s->n_modes_rec, s->n_modes_lig);
  L.rec_xyz = take(nr * 3 * 8);
  L.lig_xyz = take(nl * 3 * 8);
  L.rec_modes = take((size_t)s->n_modes_rec * nr * 3 * 8);
  L.lig_modes = take((size_t)s->n_modes_lig * nl * 3 * 8);
  L.rec_charge = take(nr * 8);
  L.lig_charge = take(nl * 8);
  L.poses = take((size_t)s->n_swarms * s->n_glowworms * pl * 8);
  L.rec_mask = take(nr * 4);
  L.lig_mask = take(nl * 4);
  L.rec_type = take(nr * 4);
  L.lig_type = take(nl * 4);
  L.rec_lj = take(nr * 4);
  L.lig_lj = take(nl * 4);
  L.total = off;
  return L;
}
bool spec_ok(const sd_synth_spec* s) {
  return s && s->n_rec > 0 && s->n_lig > 0 && s->n_swarms > 0 && s->n_glowworms > 0 && s->n_modes_rec >= 0 &&
         s->n_modes_rec <= SD_MAX_MODES && s->n_modes_lig >= 0 && s->n_modes_lig <= SD_MAX_MODES &&
         s->n_rec <= 200000 && s->n_lig <= 200000;
}
}  // namespace

extern "C" int sd_synth_buffer_size(const sd_synth_spec* spec, long long* bytes) {
  if (!spec_ok(spec) || !bytes) return sd::fail(SD_ERR_ARG, "sd_synth_buffer_size: bad spec");
  *bytes = (long long)layout_of(spec).total;
  return SD_OK;
}

extern "C" int sd_synth_generate(const sd_synth_spec* s, void* buf, sd_complex_desc* d, double** poses_out) {
  if (!spec_ok(s) || !buf || !d) return sd::fail(SD_ERR_ARG, "sd_synth_generate: bad arguments");
  Layout L = layout_of(s);
  char* b = (char*)buf;
  double* rec_xyz = (double*)(b + L.rec_xyz);
  double* lig_xyz = (double*)(b + L.lig_xyz);
  double* rec_modes = (double*)(b + L.rec_modes);
  double* lig_modes = (double*)(b + L.lig_modes);
  double* rec_charge = (double*)(b + L.rec_charge);
  double* lig_charge = (double*)(b + L.lig_charge);
  double* poses = (double*)(b + L.poses);
  int* rec_mask = (int*)(b + L.rec_mask);
  int* lig_mask = (int*)(b + L.lig_mask);
  int* rec_type = (int*)(b + L.rec_type);
  int* lig_type = (int*)(b + L.lig_type);
  int* rec_lj = (int*)(b + L.rec_lj);
  int* lig_lj = (int*)(b + L.lig_lj);

  sd::Rng rr(s->seed * 4 + 1), rl(s->seed * 4 + 2), rs(s->seed * 4 + 3);
  sd::globule(rr, s->n_rec, rec_xyz);
  sd::atoms(rr, s->n_rec, rec_type, rec_charge, rec_lj, rec_mask);
  sd::modes(rr, s->n_rec, s->n_modes_rec, rec_modes);
  sd::globule(rl, s->n_lig, lig_xyz);
  sd::atoms(rl, s->n_lig, lig_type, lig_charge, lig_lj, lig_mask);
  sd::modes(rl, s->n_lig, s->n_modes_lig, lig_modes);

  memset(d, 0, sizeof *d);
  d->n_rec = s->n_rec;
  d->n_lig = s->n_lig;
  d->rec_xyz = rec_xyz;
  d->lig_xyz = lig_xyz;
  d->rec_mask = rec_mask;
  d->lig_mask = lig_mask;
  d->n_modes_rec = s->n_modes_rec;
  d->n_modes_lig = s->n_modes_lig;
  d->rec_modes = rec_modes;
  d->lig_modes = lig_modes;
  d->rec_dfire_type = rec_type;
  d->lig_dfire_type = lig_type;
  d->rec_charge = rec_charge;
  d->lig_charge = lig_charge;
  d->rec_lj_type = rec_lj;
  d->lig_lj_type = lig_lj;
  sd::mvee_center(lig_xyz, s->n_lig, 0.01, d->lig_ref_point);
  d->n_swarms = s->n_swarms;
  d->n_glowworms = s->n_glowworms;

  sd::starting_poses(rs, rec_xyz, s->n_rec, s->n_swarms, s->n_glowworms, s->n_modes_rec, s->n_modes_lig, poses);
  if (poses_out) *poses_out = poses;
  return SD_OK;
}

extern "C" int sd_starting_poses(const double* rec_xyz, int n_rec, int n_swarms, int n_glowworms, int n_modes_rec,
                                 int n_modes_lig, unsigned long long seed, double* poses) {
  if (!rec_xyz || !poses || n_rec <= 0 || n_swarms <= 0 || n_glowworms <= 0 || n_modes_rec < 0 ||
      n_modes_rec > SD_MAX_MODES || n_modes_lig < 0 || n_modes_lig > SD_MAX_MODES)
    return sd::fail(SD_ERR_ARG, "sd_starting_poses: bad arguments");
  sd::Rng rs(seed * 4 + 3);
  sd::starting_poses(rs, rec_xyz, n_rec, n_swarms, n_glowworms, n_modes_rec, n_modes_lig, poses);
  return SD_OK;
}

extern "C" int sd_reference_point(const double* xyz, int n, double* center) {
  if (!xyz || n <= 0 || !center) return sd::fail(SD_ERR_ARG, "sd_reference_point: bad arguments");
  sd::mvee_center(xyz, n, 0.01, center);
  return SD_OK;
}

extern "C" int sd_synth_tables(unsigned long long seed, double* dfire, double* eps, double* sigma) {
  sd::Rng r(seed * 4 + 0);
  if (dfire)
    for (size_t i = 0; i < (size_t)SD_DFIRE_TYPES * SD_DFIRE_TYPES * SD_DFIRE_BINS; ++i) dfire[i] = r.normal();
  sd::Rng r2(seed * 4 + 7);
  for (int i = 0; i < SD_LJ_TYPES; ++i) {
    double e = 0.05 + 0.25 * r2.uniform();
    double s = 2.8 + 1.4 * r2.uniform();
    if (eps) eps[i] = e;
    if (sigma) sigma[i] = s;
  }
  return SD_OK;
}

extern "C" int sd_gso_draws(unsigned int seed, int S, int steps, int G, double* out) {
  if (S <= 0 || steps <= 0 || G <= 0 || !out) return sd::fail(SD_ERR_ARG, "sd_gso_draws: bad arguments");
  // prepare_gso_tasks.cc:411-427: one engine, swarm -> step -> glowworm
  std::uniform_real_distribution<double> distribution(0.0, 1.0);
  std::mt19937 gen(seed);
  for (int i = 0; i < S; i++)
    for (int s = 0; s < steps; s++)
      for (int j = 0; j < G; j++) out[(size_t)i * steps * G + (size_t)s * G + j] = distribution(gen);
  return SD_OK;
}

extern "C" void sd_gso_params_default(sd_gso_params* p) {
  if (!p) return;
  p->rho = 0.4;
  p->gamma = 0.6;
  p->beta = 0.08;
  p->initial_luciferin = 5.0;
  p->initial_vision_range = 0.2;
  p->max_vision_range = 5.0;
  p->max_neighbors = 5;
  p->translation_step = 0.5;
  p->rotation_step = 0.5;
  p->nmodes_step = 0.5;
}
