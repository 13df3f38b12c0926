/*
 * ORACLE — test infrastructure only.  Plain-C restatement of the seeded synthetic docking
 * systems that the product generates (sd_synth_generate / sd_synth_tables): compact globules,
 * DFIRE / LJ tables, orthonormal ANM modes, the Khachiyan ligand reference point and the
 * starting poses.  It exists so that the benchmark's reference arm and the CPU tests can build
 * exactly the same inputs without loading the product library; tests/test_oracle_cpu.py checks
 * that every array it writes is bit-identical to the product's.
 *
 * Engine: std::mt19937_64 restated from its published definition (Matsumoto & Nishimura 2000,
 * 64-bit parameters of ISO C++ [rand.predef]); uniform doubles from the top 53 bits; normals by
 * Box-Muller with the platform libm (log, cos, sqrt), the same calls the product makes.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "sd_oracle.h"

#define MT64_N 312
#define MT64_M 156

typedef struct {
  uint64_t x[MT64_N];
  int i;
} or_mt64;

static void mt64_seed(or_mt64* m, uint64_t s) {
  m->x[0] = s;
  for (int i = 1; i < MT64_N; ++i) m->x[i] = 6364136223846793005ULL * (m->x[i - 1] ^ (m->x[i - 1] >> 62)) + (uint64_t)i;
  m->i = MT64_N;
}

static uint64_t mt64_next(or_mt64* m) {
  if (m->i >= MT64_N) {
    for (int k = 0; k < MT64_N; ++k) {
      const uint64_t y = (m->x[k] & 0xFFFFFFFF80000000ULL) | (m->x[(k + 1) % MT64_N] & 0x7FFFFFFFULL);
      uint64_t v = m->x[(k + MT64_M) % MT64_N] ^ (y >> 1);
      if (y & 1ULL) v ^= 0xB5026F5AA96619E9ULL;
      m->x[k] = v;
    }
    m->i = 0;
  }
  uint64_t z = m->x[m->i++];
  z ^= (z >> 29) & 0x5555555555555555ULL;
  z ^= (z << 17) & 0x71D67FFFEDA60000ULL;
  z ^= (z << 37) & 0xFFF7EEE000000000ULL;
  z ^= z >> 43;
  return z;
}

static double u01(or_mt64* m) { return (double)(mt64_next(m) >> 11) * (1.0 / 9007199254740992.0); }

static double nrm(or_mt64* m) {
  const double u1 = 1.0 - u01(m);
  const double u2 = u01(m);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

static int below(or_mt64* m, int n) { return (int)(u01(m) * n); }

typedef struct {
  int* idx;
  int n, cap;
} cell_t;

static void globule(or_mt64* r, int n, double* xyz) {
  const double R = 2.2 * cbrt((double)n);
  const double dmin = 3.0, dmin2 = dmin * dmin;
  const int nc = (int)ceil(2.0 * R / dmin) + 1;
  cell_t* cells = (cell_t*)calloc((size_t)nc * nc * nc, sizeof(cell_t));
  int placed = 0;
  while (placed < n) {
    const double x = (2 * u01(r) - 1) * R, y = (2 * u01(r) - 1) * R, z = (2 * u01(r) - 1) * R;
    if (x * x + y * y + z * z > R * R) continue;
    int c3[3];
    const double v3[3] = {x, y, z};
    for (int d = 0; d < 3; ++d) {
      int c = (int)((v3[d] + R) / dmin);
      c = c < 0 ? 0 : c;
      c3[d] = c > nc - 1 ? nc - 1 : c;
    }
    int ok = 1;
    for (int a = c3[0] > 0 ? c3[0] - 1 : 0; a <= (c3[0] + 1 < nc - 1 ? c3[0] + 1 : nc - 1) && ok; ++a)
      for (int b = c3[1] > 0 ? c3[1] - 1 : 0; b <= (c3[1] + 1 < nc - 1 ? c3[1] + 1 : nc - 1) && ok; ++b)
        for (int c = c3[2] > 0 ? c3[2] - 1 : 0; c <= (c3[2] + 1 < nc - 1 ? c3[2] + 1 : nc - 1) && ok; ++c) {
          const cell_t* ce = &cells[((size_t)a * nc + b) * nc + c];
          for (int q = 0; q < ce->n; ++q) {
            const int k = ce->idx[q];
            const double dx = xyz[k * 3] - x, dy = xyz[k * 3 + 1] - y, dz = xyz[k * 3 + 2] - z;
            if (dx * dx + dy * dy + dz * dz < dmin2) {
              ok = 0;
              break;
            }
          }
        }
    if (!ok) continue;
    xyz[placed * 3] = x;
    xyz[placed * 3 + 1] = y;
    xyz[placed * 3 + 2] = z;
    cell_t* ce = &cells[((size_t)c3[0] * nc + c3[1]) * nc + c3[2]];
    if (ce->n == ce->cap) {
      ce->cap = ce->cap ? 2 * ce->cap : 8;
      ce->idx = (int*)realloc(ce->idx, sizeof(int) * ce->cap);
    }
    ce->idx[ce->n++] = placed;
    ++placed;
  }
  for (size_t k = 0; k < (size_t)nc * nc * nc; ++k) free(cells[k].idx);
  free(cells);
  double c[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) c[d] += xyz[i * 3 + d];
  for (int d = 0; d < 3; ++d) c[d] /= n;
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) xyz[i * 3 + d] -= c[d];
}

/* nm orthonormal 3N-vectors: modified Gram-Schmidt on Gaussian vectors */
static void modes(or_mt64* r, int n, int nm, double* m) {
  const size_t len = (size_t)n * 3;
  for (int k = 0; k < nm; ++k) {
    double* v = m + k * len;
    for (size_t i = 0; i < len; ++i) v[i] = nrm(r);
    for (int p = 0; p < k; ++p) {
      const double* u = m + p * len;
      double dot = 0;
      for (size_t i = 0; i < len; ++i) dot += u[i] * v[i];
      for (size_t i = 0; i < len; ++i) v[i] -= dot * u[i];
    }
    double s = 0;
    for (size_t i = 0; i < len; ++i) s += v[i] * v[i];
    s = sqrt(s);
    for (size_t i = 0; i < len; ++i) v[i] /= s;
  }
}

static void atoms(or_mt64* r, int n, int* type, double* charge, int* lj, int* mask) {
  for (int i = 0; i < n; ++i) type[i] = below(r, OR_TYPES);
  for (int i = 0; i < n; ++i) {
    const double u = u01(r);
    charge[i] = u < 0.05 ? -1.0 : u < 0.20 ? -0.5 : u < 0.80 ? 0.0 : u < 0.95 ? 0.5 : 1.0;
  }
  for (int i = 0; i < n; ++i) lj[i] = below(r, 20);
  for (int i = 0; i < n; ++i) mask[i] = u01(r) < 0.03 ? 0 : 1;
}

/* 4x4 inverse, column-major in and out, in the operation order of the reference's Eigen build of
 * MatrixXd::inverse() (Eigen 3.4 vendored with the reference: PartialPivLU, unblocked for this
 * size, then triangular solves of P I): see or_mvee_center. */
static void lu_inverse4(const double* in, double* out) {
  double m[4][4]; /* m[c][r] */
  int t[4];
  memcpy(m, in, sizeof m);
  for (int k = 0; k < 4; ++k) {
    int p = k;
    for (int r = k + 1; r < 4; ++r)
      if (fabs(m[k][r]) > fabs(m[k][p])) p = r;
    t[k] = p;
    if (fabs(m[k][p]) != 0.0) {
      if (p != k)
        for (int c = 0; c < 4; ++c) {
          const double v = m[c][k];
          m[c][k] = m[c][p];
          m[c][p] = v;
        }
      for (int r = k + 1; r < 4; ++r) m[k][r] = m[k][r] / m[k][k];
    }
    for (int c = k + 1; c < 4; ++c)
      for (int r = k + 1; r < 4; ++r) m[c][r] = m[c][r] - m[k][r] * m[c][k];
  }
  double x[4][4]; /* x[c][r] */
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) x[c][r] = c == r ? 1.0 : 0.0;
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 4; ++c) {
      const double v = x[c][k];
      x[c][k] = x[c][t[k]];
      x[c][t[k]] = v;
    }
  /* unit lower, forward */
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 4; ++c)
      for (int r = k + 1; r < 4; ++r) x[c][r] = x[c][r] - x[c][k] * m[k][r];
  /* upper, backward: multiply by the reciprocal of the diagonal */
  for (int k = 3; k >= 0; --k) {
    const double rd = 1.0 / m[k][k];
    for (int c = 0; c < 4; ++c) {
      x[c][k] = x[c][k] * rd;
      for (int r = 0; r < k; ++r) x[c][r] = x[c][r] - x[c][k] * m[k][r];
    }
  }
  memcpy(out, x, sizeof x);
}

/* Khachiyan minimum-volume enclosing ellipsoid centre, tolerance tol, restating the reference's
 * minimum_volume_ellipsoid (source/dock/src/prepare_gso_tasks.cc:106-267, with its matrix helpers
 * at :71-104, run on one thread) operation for operation: weights u = 1/N; per iteration
 * V[a][b] = sum_i q_i[a] (q_i[b] u_i) over ascending atoms (q = [p, 1]); the inverse of the
 * column-major matrix with data V (lu_inverse4); m_i = sum_k q_i[k] (sum_c Ainv(c,k) q_i[c]);
 * the first atom of largest m_i > 0 gains weight step = ((m - 3) - 1) / (4 (m - 1)) while the
 * others shrink by (1 - step); the weight change's 2-norm ends the loop below tol; the centre is
 * sum_i p_i u_i. */
void or_mvee_center(const double* p, int n, double tol, double* center) {
  double* u = (double*)malloc(sizeof(double) * n);
  double* un = (double*)malloc(sizeof(double) * n);
  for (int i = 0; i < n; ++i) u[i] = 1.0 / n;
  double err = 1 + tol;
  for (int it = 0; err > tol && it < 100000; ++it) {
    double V[16];
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        double acc = 0.0;
        for (int i = 0; i < n; ++i) {
          const double qa = a < 3 ? p[i * 3 + a] : 1.0, qb = b < 3 ? p[i * 3 + b] : 1.0;
          acc += qa * (qb * u[i]);
        }
        V[a * 4 + b] = acc;
      }
    double inv[16];
    lu_inverse4(V, inv);
    int best = 0;
    double top = 0.0;
    for (int i = 0; i < n; ++i) {
      const double q[4] = {p[i * 3], p[i * 3 + 1], p[i * 3 + 2], 1.0};
      double m = 0.0;
      for (int k = 0; k < 4; ++k) {
        double y = 0.0;
        for (int c = 0; c < 4; ++c) y += inv[k * 4 + c] * q[c];
        m += q[k] * y;
      }
      if (m > top) {
        top = m;
        best = i;
      }
    }
    const double step = (top - 3 - 1.0) / ((3 + 1.0) * (top - 1.0));
    for (int i = 0; i < n; ++i) un[i] = (1.0 - step) * u[i];
    un[best] += step;
    double e2 = 0.0;
    for (int i = 0; i < n; ++i) e2 += (un[i] - u[i]) * (un[i] - u[i]);
    err = sqrt(e2);
    for (int i = 0; i < n; ++i) u[i] = un[i];
  }
  for (int d = 0; d < 3; ++d) {
    double c = 0.0;
    for (int i = 0; i < n; ++i) c += p[i * 3 + d] * u[i];
    center[d] = c;
  }
  free(u);
  free(un);
}

static void starting_poses(or_mt64* rs, const double* rec, int nr, int S, int G, int nmr, int nml, double* poses) {
  double rmax = 0;
  for (int i = 0; i < nr; ++i) {
    const double v = sqrt(rec[i * 3] * rec[i * 3] + rec[i * 3 + 1] * rec[i * 3 + 1] + rec[i * 3 + 2] * rec[i * 3 + 2]);
    rmax = v > rmax ? v : rmax;
  }
  const double shell = rmax + 10.0;
  const int pl = 7 + nmr + nml;
  const double PI = 3.14159265358979323846;
  for (int sw = 0; sw < S; ++sw) {
    double v[3], n2 = 0;
    do {
      n2 = 0;
      for (int k = 0; k < 3; ++k) {
        v[k] = nrm(rs);
        n2 += v[k] * v[k];
      }
    } while (n2 < 1e-12);
    const double nn = sqrt(n2);
    const double c[3] = {v[0] / nn * shell, v[1] / nn * shell, v[2] / nn * shell};
    for (int g = 0; g < G; ++g) {
      double* p = poses + ((size_t)sw * G + g) * pl;
      for (int k = 0; k < 3; ++k) p[k] = c[k] + 2.0 * nrm(rs);
      const double u1 = u01(rs), u2 = u01(rs), u3 = u01(rs);
      p[3] = sqrt(1 - u1) * sin(2 * PI * u2);
      p[4] = sqrt(1 - u1) * cos(2 * PI * u2);
      p[5] = sqrt(u1) * sin(2 * PI * u3);
      p[6] = sqrt(u1) * cos(2 * PI * u3);
      for (int k = 0; k < nmr + nml; ++k) p[7 + k] = nrm(rs);
    }
  }
}

void or_synth_generate(int nr, int nl, int S, int G, int nmr, int nml, unsigned long long seed, or_synth_out* o) {
  or_mt64* rr = (or_mt64*)malloc(sizeof(or_mt64));
  or_mt64* rl = (or_mt64*)malloc(sizeof(or_mt64));
  or_mt64* rs = (or_mt64*)malloc(sizeof(or_mt64));
  mt64_seed(rr, seed * 4 + 1);
  mt64_seed(rl, seed * 4 + 2);
  mt64_seed(rs, seed * 4 + 3);
  globule(rr, nr, o->rec_xyz);
  atoms(rr, nr, o->rec_type, o->rec_charge, o->rec_lj, o->rec_mask);
  modes(rr, nr, nmr, o->rec_modes);
  globule(rl, nl, o->lig_xyz);
  atoms(rl, nl, o->lig_type, o->lig_charge, o->lig_lj, o->lig_mask);
  modes(rl, nl, nml, o->lig_modes);
  or_mvee_center(o->lig_xyz, nl, 0.01, o->lig_ref);
  starting_poses(rs, o->rec_xyz, nr, S, G, nmr, nml, o->poses);
  free(rr);
  free(rl);
  free(rs);
}

void or_synth_tables(unsigned long long seed, double* dfire, double* eps, double* sigma) {
  or_mt64* r = (or_mt64*)malloc(sizeof(or_mt64));
  mt64_seed(r, seed * 4 + 0);
  if (dfire)
    for (size_t i = 0; i < (size_t)OR_TYPES * OR_TYPES * OR_BINS; ++i) dfire[i] = nrm(r);
  mt64_seed(r, seed * 4 + 7);
  for (int i = 0; i < 20; ++i) {
    const double e = 0.05 + 0.25 * u01(r);
    const double s = 2.8 + 1.4 * u01(r);
    if (eps) eps[i] = e;
    if (sigma) sigma[i] = s;
  }
  free(r);
}
