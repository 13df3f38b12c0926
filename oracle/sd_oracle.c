/*
 * ORACLE — test infrastructure only (see sd_oracle.h).  Plain-C restatement of the
 * reference's CPU GSO docking path; every function cites the reference lines it follows
 * (paths relative to the menggerSherry/SparkleDock tree).  Compiled with
 * -ffp-contract=off so that every operation rounds like the reference's own build.
 */
#include "sd_oracle.h"
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------------------------
 * std::mt19937 and std::uniform_real_distribution<double>(0,1) as used by the reference
 * (prepare_gso_tasks.cc:411-427).  MT19937 is the published Matsumoto-Nishimura generator;
 * the double draw is the C++ standard's generate_canonical<double,53> over a 32-bit engine:
 * two draws, (g1 + g2 * 2^32) / 2^64, clamped below 1.
 * ------------------------------------------------------------------------------------- */
typedef struct { uint32_t mt[624]; int idx; } or_mt;

static void mt_seed(or_mt* m, uint32_t seed) {
  m->mt[0] = seed;
  for (int i = 1; i < 624; ++i)
    m->mt[i] = 1812433253u * (m->mt[i - 1] ^ (m->mt[i - 1] >> 30)) + (uint32_t)i;
  m->idx = 624;
}

static uint32_t mt_next(or_mt* m) {
  if (m->idx >= 624) {
    for (int i = 0; i < 624; ++i) {
      uint32_t y = (m->mt[i] & 0x80000000u) | (m->mt[(i + 1) % 624] & 0x7fffffffu);
      uint32_t v = m->mt[(i + 397) % 624] ^ (y >> 1);
      if (y & 1u) v ^= 0x9908b0dfu;
      m->mt[i] = v;
    }
    m->idx = 0;
  }
  uint32_t y = m->mt[m->idx++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

static double mt_canonical(or_mt* m) {
  double sum = 0.0, tmp = 1.0;
  for (int k = 0; k < 2; ++k) {
    sum += (double)mt_next(m) * tmp;
    tmp *= 4294967296.0;
  }
  double r = sum / tmp;
  if (r >= 1.0) r = nextafter(1.0, 0.0);
  return r * (1.0 - 0.0) + 0.0;
}

void or_gso_draws(unsigned int seed, int S, int steps, int G, double* out) {
  or_mt m;
  mt_seed(&m, seed);
  for (int i = 0; i < S; ++i)
    for (int s = 0; s < steps; ++s)
      for (int j = 0; j < G; ++j) out[(size_t)i * steps * G + (size_t)s * G + j] = mt_canonical(&m);
}

/* ---------------------------------------------------------------------------------------
 * Correctly rounded sin/acos (double-double evaluation, one rounding) for the slerp.
 * Independent C restatement of the method named in the product's header: Taylor series in
 * double-double for sin/cos on |x| <= 2, Newton on cos(y) = x for acos.
 * ------------------------------------------------------------------------------------- */
typedef struct { double hi, lo; } dd_t;
static dd_t dd_two_sum(double a, double b) {
  double s = a + b, bb = s - a;
  dd_t r = {s, (a - (s - bb)) + (b - bb)};
  return r;
}
static dd_t dd_fast(double a, double b) {
  double s = a + b;
  dd_t r = {s, b - (s - a)};
  return r;
}
static dd_t dd_prod(double a, double b) {
  double p = a * b;
  dd_t r = {p, fma(a, b, -p)};
  return r;
}
static dd_t dd_mul(dd_t a, dd_t b) {
  dd_t p = dd_prod(a.hi, b.hi);
  p.lo = fma(a.hi, b.lo, p.lo);
  p.lo = fma(a.lo, b.hi, p.lo);
  return dd_fast(p.hi, p.lo);
}
static dd_t dd_divd(dd_t a, double d) {
  double q1 = a.hi / d;
  dd_t p = dd_prod(q1, d);
  double r = ((a.hi - p.hi) - p.lo) + a.lo;
  return dd_fast(q1, r / d);
}
static dd_t dd_one_minus(dd_t a) {
  dd_t s = dd_two_sum(1.0, -a.hi);
  s.lo -= a.lo;
  return dd_fast(s.hi, s.lo);
}
static dd_t dd_sin(dd_t x) {
  dd_t x2 = dd_mul(x, x), p = {1.0, 0.0};
  for (int k = 17; k >= 1; --k) p = dd_one_minus(dd_divd(dd_mul(x2, p), (double)(2 * k) * (double)(2 * k + 1)));
  return dd_mul(x, p);
}
static dd_t dd_cos(dd_t x) {
  dd_t x2 = dd_mul(x, x), p = {1.0, 0.0};
  for (int k = 17; k >= 1; --k) p = dd_one_minus(dd_divd(dd_mul(x2, p), (double)(2 * k - 1) * (double)(2 * k)));
  return p;
}
double or_sin_cr(double x) {
  dd_t x0 = {x, 0.0};
  dd_t r = dd_sin(x0);
  return r.hi + r.lo;
}
double or_acos_cr(double x) {
  double y0 = acos(x);
  if (!(x > -1.0 && x < 1.0)) return y0;
  int neg = x < 0.0;
  double ax = neg ? -x : x;
  double y = neg ? acos(ax) : y0;
  if (y < 1e-8) return neg ? 3.141592653589793 - y : y;
  dd_t yy = {y, 0.0};
  dd_t c = dd_cos(yy), s = dd_sin(yy);
  double delta = ((c.hi - ax) + c.lo) / s.hi;
  dd_t y1 = dd_two_sum(y, delta);
  if (!neg) return y1.hi + y1.lo;
  dd_t pi = {3.141592653589793116e+00, 1.224646799147353207e-16};
  dd_t a = dd_two_sum(pi.hi, -y1.hi);
  a.lo += pi.lo - y1.lo;
  a = dd_fast(a.hi, a.lo);
  return a.hi + a.lo;
}

void or_crmath_eval(int fn, const double* x, long long n, double* out) {
  for (long long i = 0; i < n; ++i) out[i] = fn == 0 ? or_acos_cr(x[i]) : or_sin_cr(x[i]);
}

/* ---------------------------------------------------------------------------------------
 * Pose transforms.
 * receptor: r = r0 + sum_j mask * mode_j * ext_j  (prepare_gso_tasks.cc:458, :465-482)
 * ligand:   l = rotate(l0 + sum_j mask * mode_j * ext_j, q) + t  (:459-460, :487-526)
 * rotate:   q * (0,p) * conj(q)/|q|^2 in the reference's exact expression order (:277-338)
 * ------------------------------------------------------------------------------------- */
void or_receptor_pose(const or_system* sys, const double* pose, double* r) {
  memcpy(r, sys->rec_xyz, sizeof(double) * 3 * (size_t)sys->nr);
  for (int j = 0; j < sys->nmr; ++j) {
    const double* m = sys->rec_modes + (size_t)j * sys->nr * 3;
    double e = pose[7 + j];
    for (int p = 0; p < sys->nr; ++p) {
      if (sys->rec_mask[p] == 1) {
        r[p * 3] += m[p * 3] * e;
        r[p * 3 + 1] += m[p * 3 + 1] * e;
        r[p * 3 + 2] += m[p * 3 + 2] * e;
      }
    }
  }
}

static void or_rotate(double* coord, const double* q, int n) {
  double w = q[0], x = q[1], y = q[2], z = q[3];
  double n2 = w * w + x * x + y * y + z * z;
  double qi[4];
  qi[0] = q[0] / n2;
  qi[1] = -q[1] / n2;
  qi[2] = -q[2] / n2;
  qi[3] = -q[3] / n2;
  for (int i = 0; i < n; ++i) {
    double c[4], c2[4];
    c[0] = 0;
    c[1] = coord[i * 3];
    c[2] = coord[i * 3 + 1];
    c[3] = coord[i * 3 + 2];
    c2[0] = (q[0] * c[0] - q[1] * c[1] - q[2] * c[2] - q[3] * c[3]);
    c2[1] = (q[0] * c[1] + q[1] * c[0] + q[2] * c[3] - q[3] * c[2]);
    c2[2] = (q[0] * c[2] - q[1] * c[3] + q[2] * c[0] + q[3] * c[1]);
    c2[3] = (q[0] * c[3] + q[1] * c[2] - q[2] * c[1] + q[3] * c[0]);
    c[1] = (c2[0] * qi[1] + c2[1] * qi[0] + c2[2] * qi[3] - c2[3] * qi[2]);
    c[2] = (c2[0] * qi[2] - c2[1] * qi[3] + c2[2] * qi[0] + c2[3] * qi[1]);
    c[3] = (c2[0] * qi[3] + c2[1] * qi[2] - c2[2] * qi[1] + c2[3] * qi[0]);
    coord[i * 3] = c[1];
    coord[i * 3 + 1] = c[2];
    coord[i * 3 + 2] = c[3];
  }
}

void or_ligand_pose(const or_system* sys, const double* pose, double* l, double* ref) {
  memcpy(l, sys->lig_xyz, sizeof(double) * 3 * (size_t)sys->nl);
  for (int j = 0; j < sys->nml; ++j) {
    const double* m = sys->lig_modes + (size_t)j * sys->nl * 3;
    double e = pose[7 + sys->nmr + j];
    for (int p = 0; p < sys->nl; ++p) {
      if (sys->lig_mask[p] == 1) {
        l[p * 3] += m[p * 3] * e;
        l[p * 3 + 1] += m[p * 3 + 1] * e;
        l[p * 3 + 2] += m[p * 3 + 2] * e;
      }
    }
  }
  or_rotate(l, pose + 3, sys->nl);
  for (int i = 0; i < sys->nl; ++i) {
    l[i * 3] += pose[0];
    l[i * 3 + 1] += pose[1];
    l[i * 3 + 2] += pose[2];
  }
  if (ref) {
    ref[0] = sys->lig_ref[0];
    ref[1] = sys->lig_ref[1];
    ref[2] = sys->lig_ref[2];
    or_rotate(ref, pose + 3, 1);
    ref[0] += pose[0];
    ref[1] += pose[1];
    ref[2] += pose[2];
  }
}

/* ---------------------------------------------------------------------------------------
 * DFIRE (prepare_gso_tasks.cc:1522-1615, bins interface.h:30-35).
 * For each receptor atom i (outer) a partial v over ligand atoms j (inner) is added to E.
 * Edges the reference leaves undefined: d2 == 0 gives index -1 (here: bin 0, counted);
 * d2 == 225 gives dist_to_bins[29] - 1 = 20, i.e. flat index +20 = next type's bin 0,
 * which the reference reads and which is kept here, except past the table end (0.0).
 * ------------------------------------------------------------------------------------- */
static const unsigned int or_dist_to_bins[50] = {
    1,  1,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 14, 15, 15, 16, 16, 17, 17, 18, 18,
    19, 19, 20, 20, 21, 21, 22, 22, 23, 23, 24, 24, 25, 25, 26, 26, 27, 27, 28, 28, 29, 29, 30, 30, 31};

double or_dfire_energy(const or_system* sys, const double* rec, const double* lig, int* bins,
                       or_counts* c) {
  double energy = 0.0;
  const size_t tsize = (size_t)OR_TYPES * OR_TYPES * OR_BINS;
  for (int i = 0; i < sys->nr; ++i) {
    double v = 0;
    for (int j = 0; j < sys->nl; ++j) {
      double dist = (rec[i * 3 + 0] - lig[j * 3 + 0]) * (rec[i * 3 + 0] - lig[j * 3 + 0]) +
                    (rec[i * 3 + 1] - lig[j * 3 + 1]) * (rec[i * 3 + 1] - lig[j * 3 + 1]) +
                    (rec[i * 3 + 2] - lig[j * 3 + 2]) * (rec[i * 3 + 2] - lig[j * 3 + 2]);
      int bin = -1;
      if (dist <= 225.) {
        int d = (int)(sqrt(dist) * 2.0 - 1.0);
        if (d < 0) {
          d = 0;
          if (c) c->d2_zero++;
        }
        if (d == 29 && c) c->d2_cutoff++;
        bin = (int)or_dist_to_bins[d] - 1;
        size_t idx = (size_t)sys->rec_type[i] * 168 * 20 + (size_t)sys->lig_type[j] * 20 + (size_t)bin;
        double value = idx < tsize ? sys->table[idx] : 0.0;
        v += value;
      }
      if (bins) bins[(size_t)i * sys->nl + j] = bin;
    }
    energy += v;
  }
  return energy;
}

/* ---------------------------------------------------------------------------------------
 * pyDock-style electrostatics + Lennard-Jones (project-defined; no reference code).
 *   elec: 332.0636/4 * qi*qj / (r^2 + 1)          (eps(r) = 4r, soft core 1 A^2), r < 15 A
 *   LJ  : 4*eps_ij*(s^6 - s^3), s = sig_ij^2/(r^2 + 0.5*sig_ij^2), r < 8 A
 *         eps_ij = sqrt(eps_i*eps_j), sig_ij = (sig_i + sig_j)/2
 *   both multiplied by the CHARMM switch S(r^2) over the last 1 A of their cutoff
 *   E = E_elec + 0.1 * E_lj ; score = -E
 * ------------------------------------------------------------------------------------- */
#define PD_KE (332.0636 / 4.0)
#define PD_SOFT_E 1.0
#define PD_SOFT_LJ 0.5
#define PD_WVDW 0.1
#define PD_EL_ON2 196.0
#define PD_EL_OFF2 225.0
#define PD_LJ_ON2 49.0
#define PD_LJ_OFF2 64.0

static void pd_switch(double x, double on2, double off2, double* s, double* ds) {
  if (x <= on2) { *s = 1.0; *ds = 0.0; return; }
  if (x >= off2) { *s = 0.0; *ds = 0.0; return; }
  double den = (off2 - on2) * (off2 - on2) * (off2 - on2);
  *s = (off2 - x) * (off2 - x) * (off2 + 2.0 * x - 3.0 * on2) / den;
  *ds = 6.0 * (off2 - x) * (on2 - x) / den;
}

/* pair energy and d(energy)/d(r^2) */
static double pd_pair(const or_system* sys, int i, int j, double x, double* dedx) {
  double e = 0.0, de = 0.0, s, ds;
  if (x < PD_EL_OFF2) {
    double qq = PD_KE * sys->rec_charge[i] * sys->lig_charge[j];
    double inv = 1.0 / (x + PD_SOFT_E);
    pd_switch(x, PD_EL_ON2, PD_EL_OFF2, &s, &ds);
    double el = qq * inv;
    e += el * s;
    de += -el * inv * s + el * ds;
  }
  if (x < PD_LJ_OFF2) {
    int a = sys->rec_lj[i], b = sys->lig_lj[j];
    double eps = sqrt(sys->lj_eps[a] * sys->lj_eps[b]);
    double sig = 0.5 * (sys->lj_sigma[a] + sys->lj_sigma[b]);
    double sig2 = sig * sig;
    double den = x + PD_SOFT_LJ * sig2;
    double sv = sig2 / den;
    double s3 = sv * sv * sv, s6 = s3 * s3;
    double lj = 4.0 * eps * (s6 - s3);
    double dsv = -sv / den;
    double dlj = 4.0 * eps * (6.0 * s6 / sv - 3.0 * s3 / sv) * dsv;
    pd_switch(x, PD_LJ_ON2, PD_LJ_OFF2, &s, &ds);
    e += PD_WVDW * lj * s;
    de += PD_WVDW * (dlj * s + lj * ds);
  }
  *dedx = de;
  return e;
}

double or_pydock_energy(const or_system* sys, const double* pose) {
  double* rec = (double*)malloc(sizeof(double) * 3 * (size_t)sys->nr);
  double* lig = (double*)malloc(sizeof(double) * 3 * (size_t)sys->nl);
  or_receptor_pose(sys, pose, rec);
  or_ligand_pose(sys, pose, lig, NULL);
  double E = 0.0;
  for (int i = 0; i < sys->nr; ++i) {
    double v = 0.0;
    for (int j = 0; j < sys->nl; ++j) {
      double dx = rec[i * 3] - lig[j * 3], dy = rec[i * 3 + 1] - lig[j * 3 + 1], dz = rec[i * 3 + 2] - lig[j * 3 + 2];
      double x = dx * dx + dy * dy + dz * dz, de;
      if (x < PD_EL_OFF2) v += pd_pair(sys, i, j, x, &de);
    }
    E += v;
  }
  free(rec);
  free(lig);
  return E;
}

/* rotation matrix of the reference's rotate() for quaternion q (any norm) */
static void quat_matrix(const double* q, double R[3][3]) {
  double e[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int c = 0; c < 3; ++c) {
    double v[3] = {e[c][0], e[c][1], e[c][2]};
    or_rotate(v, q, 1);
    for (int r = 0; r < 3; ++r) R[r][c] = v[r];
  }
}

void or_pydock_grad(const or_system* sys, const double* pose, double* grad) {
  int nr = sys->nr, nl = sys->nl;
  double* rec = (double*)malloc(sizeof(double) * 3 * (size_t)nr);
  double* lig = (double*)malloc(sizeof(double) * 3 * (size_t)nl);
  double* fr = (double*)calloc(3 * (size_t)nr, sizeof(double));
  double* fl = (double*)calloc(3 * (size_t)nl, sizeof(double));
  or_receptor_pose(sys, pose, rec);
  or_ligand_pose(sys, pose, lig, NULL);
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nl; ++j) {
      double dx = rec[i * 3] - lig[j * 3], dy = rec[i * 3 + 1] - lig[j * 3 + 1], dz = rec[i * 3 + 2] - lig[j * 3 + 2];
      double x = dx * dx + dy * dy + dz * dz, de;
      if (x >= PD_EL_OFF2) continue;
      pd_pair(sys, i, j, x, &de);
      double g[3] = {2.0 * de * dx, 2.0 * de * dy, 2.0 * de * dz};  /* dE/dr_i */
      for (int k = 0; k < 3; ++k) {
        fr[i * 3 + k] += g[k];
        fl[j * 3 + k] -= g[k];
      }
    }
  int nmr = sys->nmr, nml = sys->nml;
  for (int k = 0; k < 6 + nmr + nml; ++k) grad[k] = 0.0;
  double R[3][3];
  quat_matrix(pose + 3, R);
  for (int j = 0; j < nl; ++j) {
    const double* g = fl + j * 3;
    double p[3] = {lig[j * 3] - pose[0], lig[j * 3 + 1] - pose[1], lig[j * 3 + 2] - pose[2]};
    grad[0] += g[0];
    grad[1] += g[1];
    grad[2] += g[2];
    grad[3] += p[1] * g[2] - p[2] * g[1];
    grad[4] += p[2] * g[0] - p[0] * g[2];
    grad[5] += p[0] * g[1] - p[1] * g[0];
    if (sys->lig_mask[j] == 1)
      for (int m = 0; m < nml; ++m) {
        const double* M = sys->lig_modes + ((size_t)m * nl + j) * 3;
        double RM[3];
        for (int r = 0; r < 3; ++r) RM[r] = R[r][0] * M[0] + R[r][1] * M[1] + R[r][2] * M[2];
        grad[6 + nmr + m] += RM[0] * g[0] + RM[1] * g[1] + RM[2] * g[2];
      }
  }
  for (int i = 0; i < nr; ++i) {
    if (sys->rec_mask[i] != 1) continue;
    const double* g = fr + i * 3;
    for (int m = 0; m < nmr; ++m) {
      const double* M = sys->rec_modes + ((size_t)m * nr + i) * 3;
      grad[6 + m] += M[0] * g[0] + M[1] * g[1] + M[2] * g[2];
    }
  }
  free(rec);
  free(lig);
  free(fr);
  free(fl);
}

double or_score_pose(const or_system* sys, const double* pose, double* energy_out, double* ref_out,
                     int* bins, or_counts* c) {
  double* rec = (double*)malloc(sizeof(double) * 3 * (size_t)sys->nr);
  double* lig = (double*)malloc(sizeof(double) * 3 * (size_t)sys->nl);
  double ref[3];
  or_receptor_pose(sys, pose, rec);
  or_ligand_pose(sys, pose, lig, ref);
  double energy, score;
  if (sys->scoring == 1) {
    free(rec);
    free(lig);
    energy = or_pydock_energy(sys, pose);
    score = -energy;
  } else {
    energy = or_dfire_energy(sys, rec, lig, bins, c);
    score = ((energy)*0.0157 - 4.7) * -1;
    free(rec);
    free(lig);
  }
  if (energy_out) *energy_out = energy;
  if (ref_out) memcpy(ref_out, ref, sizeof ref);
  return score;
}

void or_score_poses(const or_system* sys, const double* poses, int n, double* scores,
                    double* energies, int nthreads) {
  int pl = 7 + sys->nmr + sys->nml;
#pragma omp parallel for schedule(dynamic) num_threads(nthreads > 0 ? nthreads : 1)
  for (int p = 0; p < n; ++p) {
    double e;
    scores[p] = or_score_pose(sys, poses + (size_t)p * pl, &e, NULL, NULL, NULL);
    if (energies) energies[p] = e;
  }
}

/* ---------------------------------------------------------------------------------------
 * GSO helpers: move_extent (:1352-1368), slerp (:1370-1421).
 * ------------------------------------------------------------------------------------- */
static void or_move_extent(double* self, const double* other, int n_ext, double step) {
  double delta[OR_MAX_MODES];
  double n = 0;
  for (int i = 0; i < n_ext; ++i) {
    delta[i] = other[i] - self[i];
    n += delta[i] * delta[i];
  }
  n = sqrt(n);
  if (n >= 1e-8) {
    for (int i = 0; i < n_ext; ++i) {
      delta[i] *= step / n;
      self[i] += delta[i];
    }
  }
}

void or_slerp(double* self, double* other, double step, int cr) {
  double sn = 0, on = 0;
  for (int i = 0; i < 4; ++i) {
    sn += (self[i] * self[i]);
    on += (other[i] * other[i]);
  }
  sn = sqrt(sn);
  on = sqrt(on);
  for (int i = 0; i < 4; ++i) {
    self[i] /= sn;
    other[i] /= on;
  }
  double q_dot = 0;
  for (int i = 0; i < 4; ++i) q_dot += self[i] * other[i];
  if (q_dot < 0) {
    q_dot = q_dot * -1;
    for (int i = 0; i < 4; ++i) self[i] = -self[i];
  }
  if (q_dot > 0.9995) {
    for (int i = 0; i < 4; ++i) self[i] = self[i] + step * (other[i] - self[i]);
    double rn = 0;
    for (int i = 0; i < 4; ++i) rn += (self[i] * self[i]);
    rn = sqrt(rn);
    for (int i = 0; i < 4; ++i) self[i] /= rn;
  } else {
    q_dot = (q_dot < 1) ? q_dot : 1;
    q_dot = (q_dot > -1) ? q_dot : -1;
    double omega = cr ? or_acos_cr(q_dot) : acos(q_dot);
    double so = cr ? or_sin_cr(omega) : sin(omega);
    double a = (1.0 - step) * omega, b = step * omega;
    double tmp0 = ((cr ? or_sin_cr(a) : sin(a)) / so);
    double tmp1 = ((cr ? or_sin_cr(b) : sin(b)) / so);
    for (int i = 0; i < 4; ++i) self[i] = tmp0 * self[i] + tmp1 * other[i];
  }
}

void or_init_state(const or_system* sys, or_state* st, const double* pos0, double luciferin0,
                   double vision0) {
  int n = sys->S * sys->G, pl = 7 + sys->nmr + sys->nml;
  memcpy(st->pos, pos0, sizeof(double) * (size_t)n * pl);
  for (int k = 0; k < n; ++k) {
    st->scoring[k] = 0;
    st->luciferin[k] = luciferin0;
    st->vision[k] = vision0;
    st->step[k] = 0;
    st->moved[k] = 0;
    st->nnei[k] = 0;
    st->select[k] = k % sys->G;
    st->ref[k * 3] = st->ref[k * 3 + 1] = st->ref[k * 3 + 2] = 0.0;
  }
}

/* ---------------------------------------------------------------------------------------
 * One GSO step: the three passes of cal_gso_tasks_cpu (prepare_gso_tasks.cc:429-819).
 *   pass 1 (:432-570)  rescore moved (or first-step) glowworms; luciferin for all
 *   pass 2 (:584-708)  neighbours (ascending n), probabilities (:1463-1488), selection
 *                      (:1424-1459), copy of the chosen neighbour's pre-move position
 *   pass 3 (:716-814)  move toward the copy; vision range update and clamp
 * The update is synchronous: passes 2 and 3 read only state of the earlier passes.
 * ------------------------------------------------------------------------------------- */
void or_gso_step(const or_system* sys, or_state* st, const double* u_step, const double* score_override,
                 or_counts* cnt, int nthreads) {
  const int S = sys->S, G = sys->G, pl = 7 + sys->nmr + sys->nml;
  if (nthreads <= 0) nthreads = 1;
  or_counts local = {0, 0, 0, 0, 0};

  /* pass 1 */
  long long scored = 0, z = 0, cut = 0;
#pragma omp parallel for schedule(dynamic) num_threads(nthreads) reduction(+ : scored, z, cut)
  for (int i = 0; i < S; ++i) {
    for (int g = 0; g < G; ++g) {
      int k = i * G + g;
      if (st->moved[k] || st->step[k] == 0) {
        double* pose = st->pos + (size_t)k * pl;
        or_counts c1 = {0, 0, 0, 0, 0};
        double e;
        double sc = or_score_pose(sys, pose, &e, st->ref + (size_t)k * 3, NULL, &c1);
        st->scoring[k] = score_override ? score_override[k] : sc;
        scored++;
        z += c1.d2_zero;
        cut += c1.d2_cutoff;
      }
      st->luciferin[k] = (1.0 - sys->rho) * st->luciferin[k] + sys->gamma * st->scoring[k];
      st->step[k] += 1;
    }
  }
  local.scored = scored;
  local.d2_zero = z;
  local.d2_cutoff = cut;

  /* pass 2 */
  double* sel_pos = (double*)malloc(sizeof(double) * (size_t)S * G * pl);
  int* neighbors = (int*)malloc(sizeof(int) * (size_t)G);
  double* prob = (double*)malloc(sizeof(double) * (size_t)G);
  for (int i = 0; i < S; ++i) {
    const double* L = st->luciferin + (size_t)i * G;
    for (int g = 0; g < G; ++g) {
      int k = i * G + g;
      const double* cur = st->ref + (size_t)k * 3;
      double sq = st->vision[k] * st->vision[k];
      int nn = 0;
      for (int n = 0; n < G; ++n) {
        if (n != g && L[g] < L[n]) {
          const double* nr = st->ref + ((size_t)i * G + n) * 3;
          double distance = 0;
          for (int d = 0; d < 3; ++d) distance += ((cur[d] - nr[d]) * (cur[d] - nr[d]));
          if (distance < sq) neighbors[nn++] = n;
        }
      }
      st->nnei[k] = nn;
      double total = 0;
      for (int a = 0; a < nn; ++a) {
        double diff = L[neighbors[a]] - L[g];
        prob[a] = diff;
        total += diff;
      }
      for (int a = 0; a < nn; ++a) prob[a] /= total;
      double u = u_step[k];
      int sel;
      if (nn == 0) {
        sel = g;
      } else {
        double sum = 0.0;
        int ii = 0;
        while (sum < u && ii < nn) {
          sum += prob[ii];
          ii += 1;
        }
        if (ii == 0) {
          ii = 1; /* u <= 0: the reference reads neighbors[-1] */
          local.u_zero++;
        } else if (sum < u) {
          local.shortfall++; /* reference reads past the list; take the last neighbour */
        }
        sel = neighbors[ii - 1];
      }
      st->select[k] = sel;
      memcpy(sel_pos + (size_t)k * pl, st->pos + ((size_t)i * G + sel) * pl, sizeof(double) * pl);
    }
  }
  free(neighbors);
  free(prob);

  /* pass 3 */
  for (int i = 0; i < S; ++i) {
    for (int g = 0; g < G; ++g) {
      int k = i * G + g;
      int sel = st->select[k];
      double* cur = st->pos + (size_t)k * pl;
      double* mv = sel_pos + (size_t)k * pl;
      st->moved[k] = g != sel;
      if (g != sel) {
        double delta[3], n = 0;
        for (int d = 0; d < 3; ++d) {
          delta[d] = mv[d] - cur[d];
          n += (delta[d] * delta[d]);
        }
        n = sqrt(n);
        if (n >= 1e-8) {
          for (int d = 0; d < 3; ++d) {
            delta[d] *= (sys->step_t / n);
            cur[d] += delta[d];
          }
        }
        or_slerp(cur + 3, mv + 3, sys->step_r, sys->cr_math);
        or_move_extent(cur + 7, mv + 7, sys->nmr, sys->step_nm);
        or_move_extent(cur + 7 + sys->nmr, mv + 7 + sys->nmr, sys->nml, sys->step_nm);
      }
      st->vision[k] = st->vision[k] + sys->beta * (sys->max_neighbors - st->nnei[k]);
      if (st->vision[k] < 0.0) st->vision[k] = 0;
      if (st->vision[k] > sys->max_vision) st->vision[k] = sys->max_vision;
    }
  }
  free(sel_pos);
  if (cnt) {
    cnt->scored += local.scored;
    cnt->d2_zero += local.d2_zero;
    cnt->d2_cutoff += local.d2_cutoff;
    cnt->u_zero += local.u_zero;
    cnt->shortfall += local.shortfall;
  }
}

void or_key_thresholds(double* t) {
  /* t[m] = smallest double x > 0 with (int)(sqrt(x)*2.0 - 1.0) >= m; t[0] = smallest x with key 0 */
  t[0] = 4.9406564584124654e-324;
  for (int m = 1; m < 30; ++m) {
    double lo = 0.0, hi = 226.0; /* key(lo) < m <= key(hi) */
    while (1) {
      double mid = 0.5 * (lo + hi);
      if (mid == lo || mid == hi) break;
      if ((int)(sqrt(mid) * 2.0 - 1.0) >= m) hi = mid; else lo = mid;
    }
    /* hi is within one ulp; walk to the exact boundary */
    while ((int)(sqrt(nextafter(hi, 0.0)) * 2.0 - 1.0) >= m) hi = nextafter(hi, 0.0);
    while ((int)(sqrt(hi) * 2.0 - 1.0) < m) hi = nextafter(hi, 1e300);
    t[m] = hi;
  }
}

/* ---------------------------------------------------------------------------------------
 * Final-pose clustering (pipeline:2766-2960).  Key: (int64)(score * 2^50) / 2^12 * 2^12 + g,
 * sorted descending; cluster 0 starts with the first glowworm, then every glowworm in order
 * (the first again) joins the first cluster whose representative is within 4 A RMSD over the
 * flagged atoms (per atom ((0 + dx^2) + dy^2) + dz^2 added in order, receptor then ligand,
 * divided by the count, square root), else starts a new cluster.
 * ------------------------------------------------------------------------------------- */
void or_cluster(const or_system* sys, const double* pos, const double* scores, const int* rec_bb,
                const int* lig_bb, int* n_clusters, int* rep, int* size, int* member) {
  const int S = sys->S, G = sys->G, nr = sys->nr, nl = sys->nl, pl = 7 + sys->nmr + sys->nml;
  int nbb = 0;
  for (int i = 0; i < nr; ++i) nbb += rec_bb[i] != 0;
  for (int j = 0; j < nl; ++j) nbb += lig_bb[j] != 0;
  double* rec = (double*)malloc(sizeof(double) * 3 * nr);
  double* lig = (double*)malloc(sizeof(double) * 3 * nl);
  double* bb = (double*)malloc(sizeof(double) * 3 * (size_t)nbb * G);
  long long* key = (long long*)malloc(sizeof(long long) * G);
  int* order = (int*)malloc(sizeof(int) * G);
  for (int s = 0; s < S; ++s) {
    for (int g = 0; g < G; ++g) {
      const double* p = pos + ((size_t)s * G + g) * pl;
      double refp[3];
      or_receptor_pose(sys, p, rec);
      or_ligand_pose(sys, p, lig, refp);
      double* o = bb + (size_t)g * nbb * 3;
      int k = 0;
      for (int i = 0; i < nr; ++i)
        if (rec_bb[i]) { o[k * 3] = rec[i * 3]; o[k * 3 + 1] = rec[i * 3 + 1]; o[k * 3 + 2] = rec[i * 3 + 2]; ++k; }
      for (int j = 0; j < nl; ++j)
        if (lig_bb[j]) { o[k * 3] = lig[j * 3]; o[k * 3 + 1] = lig[j * 3 + 1]; o[k * 3 + 2] = lig[j * 3 + 2]; ++k; }
      double sc = scores[(size_t)s * G + g] * 1125899906842624.0;
      if (sc > 9.2e18) sc = 9.2e18;
      if (sc < -9.2e18) sc = -9.2e18;
      key[g] = (long long)sc / 4096 * 4096 + g;
    }
    for (int g = 0; g < G; ++g) {
      int r = 0;
      for (int h = 0; h < G; ++h) r += key[h] > key[g];
      order[r] = g;
    }
    int* crep = rep + (size_t)s * G;
    int* clen = size + (size_t)s * G;
    for (int c = 0; c < G; ++c) { crep[c] = -1; clen[c] = 0; }
    int ncl = 1;
    crep[0] = order[0];
    clen[0] = 1;
    for (int i = 0; i < G; ++i) {
      const int g = order[i];
      const double* cur = bb + (size_t)g * nbb * 3;
      int hit = -1;
      for (int c = 0; c < ncl && hit < 0; ++c) {
        const double* r = bb + (size_t)crep[c] * nbb * 3;
        double sum = 0.0;
        for (int a = 0; a < nbb; ++a) {
          const double dx = r[a * 3] - cur[a * 3], dy = r[a * 3 + 1] - cur[a * 3 + 1], dz = r[a * 3 + 2] - cur[a * 3 + 2];
          double t = 0.0;
          t += dx * dx;
          t += dy * dy;
          t += dz * dz;
          sum += t;
        }
        if (sqrt(sum / nbb) <= 4.0) hit = c;
      }
      if (hit < 0) { hit = ncl++; crep[hit] = g; }
      ++clen[hit];
      member[(size_t)s * G + g] = hit;
    }
    n_clusters[s] = ncl;
  }
  free(rec); free(lig); free(bb); free(key); free(order);
}
