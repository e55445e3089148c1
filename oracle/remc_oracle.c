/* FP64 CPU oracle for the REMC docking hot path (TEST INFRASTRUCTURE ONLY:
 * imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg to check the engine's results; the product never links it). See remc_oracle.h for the
 * reference files each function follows.
 *
 * Build: cc -O2 -fPIC -shared (default x86-64 target: no FMA contraction, so
 * the FP32/FP64 move arithmetic rounds exactly like the reference's). */
#include "remc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- Philox */
/* Philox4x32-10, Salmon et al., "Parallel random numbers: as easy as 1, 2, 3",
 * SC'11: multipliers 0xD2511F53, 0xCD9E8D57, Weyl key increments 0x9E3779B9,
 * 0xBB67AE85, ten rounds. */
void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

static double u32_to_unit(uint32_t x) { return (double)x * (1.0 / 4294967296.0); }

void oracle_step_uniforms(uint64_t seed, uint32_t step, uint32_t slot, uint32_t system,
                          double u[6]) {
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t ctr[4] = {step, slot, system, 0u};
  uint32_t x[4];
  oracle_philox4x32_10(ctr, key, x);
  u[0] = u32_to_unit(x[0]);
  u[1] = u32_to_unit(x[1]);
  u[2] = u32_to_unit(x[2]);
  u[3] = u32_to_unit(x[3]);
  ctr[3] = 1u;
  oracle_philox4x32_10(ctr, key, x);
  u[4] = u32_to_unit(x[0]);
  u[5] = u32_to_unit(x[1]);
}

double oracle_exchange_uniform(uint64_t seed, uint32_t round, uint32_t pair, uint32_t system) {
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t ctr[4] = {round, pair, system, 2u};
  uint32_t x[4];
  oracle_philox4x32_10(ctr, key, x);
  return u32_to_unit(x[0]);
}

/* ---------------------------------------------------------------- energy */
static int bead_mol(const oracle_system* s, int b) {
  /* binary search in mol_start */
  int lo = 0, hi = s->n_mol - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) / 2;
    if (s->mol_start[mid] <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

/* Minimum-image distance (Replica.cpp:589-600: d - L*round(d/L) per axis). */
static double min_image_r(const float* pa, const float* pb, double L, double d[3]) {
  double r2 = 0.0;
  for (int k = 0; k < 3; ++k) {
    double x = (double)pa[k] - (double)pb[k];
    x = x - L * round(x / L);
    d[k] = x;
    r2 += x * x;
  }
  return sqrt(r2);
}

/* Pair energy pieces: lj (in LJ accumulator units, crowder terms included)
 * and dh (q q exp(-r/xi)/r), following Replica.cpp:637-724. */
static void pair_terms(const oracle_system* s, const oracle_params* p, int ta, int tb,
                       int crowder_pair, double r, double* lj, double* dh) {
  *lj = 0.0;
  *dh = 0.0;
  if (crowder_pair) {
    double cut = (double)p->crowder_cutoff;
    if (cut > 0.0 && !(r < cut)) return;
    if (p->crowder_mode == 0) {
      double t = 6.0 / r;
      double t3 = t * t * t;
      *lj = t3 * t3;
    } else {
      double sig = (double)s->type_rho[ta] + (double)s->type_rho[tb];
      double t = sig / r;
      double t3 = t * t * t;
      double t6 = t3 * t3;
      *lj = (double)p->crowder_eps * t6 * t6;
    }
    return;
  }
  double eps = (double)s->eps_table[ta * 32 + tb];
  double sigma = 0.5 * ((double)s->type_vdw[ta] + (double)s->type_vdw[tb]);
  double t = sigma / r;
  double t3 = t * t * t;
  double s6 = t3 * t3;
  double LJ = -4.0 * eps * s6 * (s6 - 1.0);
  if (eps > 0.0 && r < sigma * 1.122462048309372981433533049679) LJ = -LJ + 2.0 * eps;
  *lj = LJ;
  *dh = (double)s->type_q[ta] * (double)s->type_q[tb] * exp(-r / (double)p->debye_length) / r;
}

static double combine(const oracle_params* p, double lj, double dh) {
  return (lj * (double)p->lj_cf + dh * (double)p->dh_const) * (double)p->kbt_cf;
}

double oracle_pair_energy(const oracle_system* s, const oracle_params* p, int a, int b,
                          const float* pos) {
  int ma = bead_mol(s, a), mb = bead_mol(s, b);
  if (ma == mb) return 0.0;
  double d[3];
  double r = min_image_r(pos + 3 * a, pos + 3 * b, (double)s->box, d);
  int crowd = (s->mol_role[ma] == -1) || (s->mol_role[mb] == -1);
  double lj, dh;
  pair_terms(s, p, s->bead_type[a], s->bead_type[b], crowd, r, &lj, &dh);
  return combine(p, lj, dh);
}

double oracle_energy_full(const oracle_system* s, const oracle_params* p, const float* pos) {
  double lj_acc = 0.0, dh_acc = 0.0;
  for (int mi = 0; mi < s->n_mol; ++mi) {
    for (int mj = mi + 1; mj < s->n_mol; ++mj) {
      int crowd = (s->mol_role[mi] == -1) || (s->mol_role[mj] == -1);
      for (int a = s->mol_start[mi]; a < s->mol_start[mi + 1]; ++a) {
        for (int b = s->mol_start[mj]; b < s->mol_start[mj + 1]; ++b) {
          double d[3];
          double r = min_image_r(pos + 3 * a, pos + 3 * b, (double)s->box, d);
          double lj, dh;
          pair_terms(s, p, s->bead_type[a], s->bead_type[b], crowd, r, &lj, &dh);
          lj_acc += lj;
          dh_acc += dh;
        }
      }
    }
  }
  return combine(p, lj_acc, dh_acc);
}

double oracle_energy_molecule(const oracle_system* s, const oracle_params* p, const float* pos,
                              int m, const float* mpos) {
  double lj_acc = 0.0, dh_acc = 0.0;
  int m0 = s->mol_start[m], m1 = s->mol_start[m + 1];
  for (int mj = 0; mj < s->n_mol; ++mj) {
    if (mj == m) continue;
    int crowd = (s->mol_role[m] == -1) || (s->mol_role[mj] == -1);
    for (int a = m0; a < m1; ++a) {
      for (int b = s->mol_start[mj]; b < s->mol_start[mj + 1]; ++b) {
        double d[3];
        double r = min_image_r(mpos + 3 * (a - m0), pos + 3 * b, (double)s->box, d);
        double lj, dh;
        pair_terms(s, p, s->bead_type[a], s->bead_type[b], crowd, r, &lj, &dh);
        lj_acc += lj;
        dh_acc += dh;
      }
    }
  }
  return combine(p, lj_acc, dh_acc);
}

/* Sum of the magnitudes of the pair terms of molecule m at positions mpos
 * against every other molecule: the scale of the cancellation in a move's
 * dE (the sum of these terms at the new and at the old position). */
double oracle_energy_molecule_abs(const oracle_system* s, const oracle_params* p,
                                  const float* pos, int m, const float* mpos) {
  double acc = 0.0;
  int m0 = s->mol_start[m], m1 = s->mol_start[m + 1];
  for (int mj = 0; mj < s->n_mol; ++mj) {
    if (mj == m) continue;
    int crowd = (s->mol_role[m] == -1) || (s->mol_role[mj] == -1);
    for (int a = m0; a < m1; ++a) {
      for (int b = s->mol_start[mj]; b < s->mol_start[mj + 1]; ++b) {
        double d[3];
        double r = min_image_r(mpos + 3 * (a - m0), pos + 3 * b, (double)s->box, d);
        double lj, dh;
        pair_terms(s, p, s->bead_type[a], s->bead_type[b], crowd, r, &lj, &dh);
        acc += fabs(combine(p, lj, dh));
      }
    }
  }
  return acc;
}

double oracle_noncrowder_pair_energy(const oracle_system* s, const oracle_params* p,
                                     const float* pos) {
  double total = 0.0;
  for (int mi = 0; mi < s->n_mol; ++mi) {
    if (s->mol_role[mi] == -1) continue;
    for (int mj = mi + 1; mj < s->n_mol; ++mj) {
      if (s->mol_role[mj] == -1) continue;
      double lj_acc = 0.0, dh_acc = 0.0;
      for (int a = s->mol_start[mi]; a < s->mol_start[mi + 1]; ++a)
        for (int b = s->mol_start[mj]; b < s->mol_start[mj + 1]; ++b) {
          double d[3];
          double r = min_image_r(pos + 3 * a, pos + 3 * b, (double)s->box, d);
          double lj, dh;
          pair_terms(s, p, s->bead_type[a], s->bead_type[b], 0, r, &lj, &dh);
          lj_acc += lj;
          dh_acc += dh;
        }
      total += combine(p, lj_acc, dh_acc);
    }
  }
  return total;
}

/* ----------------------------------------------------------------- moves */
/* Replica::translate (Replica.cpp:333-364) and Molecule::setPosition
 * (Molecule.cpp:247-260), and Molecule::rotateQ (Molecule.cpp:288-333) with
 * Quaternion::rotateVector (Quaternion.cpp:84-101): same operations in the same
 * precisions and order. */
int oracle_propose(const oracle_system* s, const oracle_replica* r, int m, const double u[6],
                   float* new_pos, float* new_rel, float* new_centre, double* new_quat) {
  int m0 = s->mol_start[m], n = s->mol_start[m + 1] - m0;
  int rotate = (u[1] < 0.5);
  if (r->translate_only_crowders && s->mol_role[m] == -1) rotate = 0;
  const float* c = r->centre + 3 * m;
  const double* q0 = r->quat + 4 * m;
  if (!rotate) {
    float vx = (float)(u[2] - 0.5), vy = (float)(0.5 - u[3]), vz = (float)(u[4] - 0.5);
    float mag = sqrtf(vx * vx + vy * vy + vz * vz);
    if (mag != 0.0f) {
      vx = vx / mag;
      vy = vy / mag;
      vz = vz / mag;
    }
    float step = r->translate_step;
    float tx = vx * step, ty = vy * step, tz = vz * step;
    float L = s->box;
    float nx = c[0] + tx, ny = c[1] + ty, nz = c[2] + tz;
    nx = fmodf(nx + L, L);
    ny = fmodf(ny + L, L);
    nz = fmodf(nz + L, L);
    new_centre[0] = nx;
    new_centre[1] = ny;
    new_centre[2] = nz;
    memcpy(new_quat, q0, 4 * sizeof(double));
    for (int k = 0; k < n; ++k) {
      const float* rl = r->rel + 3 * (m0 + k);
      new_rel[3 * k] = rl[0];
      new_rel[3 * k + 1] = rl[1];
      new_rel[3 * k + 2] = rl[2];
      new_pos[3 * k] = rl[0] + nx;
      new_pos[3 * k + 1] = rl[1] + ny;
      new_pos[3 * k + 2] = rl[2] + nz;
    }
    return 0;
  }
  /* random axis (Replica.cpp:311-318) */
  double ax = u[2] - 0.5, ay = 0.5 - u[3], az = u[4] - 0.5;
  double am = sqrt(ax * ax + ay * ay + az * az);
  ax /= am;
  ay /= am;
  az /= am;
  /* q = (cos(a/2), sin(a/2) axis), normalised; rotation = q * rotation */
  double sina = r->rotate_sin_half, cosa = r->rotate_cos_half;
  double qw = cosa, qx = sina * ax, qy = sina * ay, qz = sina * az;
  double qm = sqrt(qw * qw + qx * qx + qy * qy + qz * qz);
  qw /= qm;
  qx /= qm;
  qy /= qm;
  qz /= qm;
  new_quat[0] = qw * q0[0] - qx * q0[1] - qy * q0[2] - qz * q0[3];
  new_quat[1] = qw * q0[1] + qx * q0[0] + qy * q0[3] - qz * q0[2];
  new_quat[2] = qw * q0[2] - qx * q0[3] + qy * q0[0] + qz * q0[1];
  new_quat[3] = qw * q0[3] + qx * q0[2] - qy * q0[1] + qz * q0[0];
  new_centre[0] = c[0];
  new_centre[1] = c[1];
  new_centre[2] = c[2];
  double w2 = qw * qw, x2 = qx * qx, y2 = qy * qy, z2 = qz * qz;
  double wx = qw * qx, wy = qw * qy, wz = qw * qz;
  double xy = qx * qy, xz = qx * qz, yz = qy * qz;
  for (int k = 0; k < n; ++k) {
    const float* rl = r->rel + 3 * (m0 + k);
    double vx = rl[0], vy = rl[1], vz = rl[2];
    float rx = (float)(vx * (w2 + x2 - y2 - z2) + (vy * (xy - wz) + vz * (wy + xz)) * 2.0);
    float ry = (float)((vx * (wz + xy) + vz * (yz - wx)) * 2.0 + vy * (w2 - x2 + y2 - z2));
    float rz = (float)((vx * (xz - wy) + vy * (yz + wx)) * 2.0 + vz * (w2 - x2 - y2 + z2));
    new_rel[3 * k] = rx;
    new_rel[3 * k + 1] = ry;
    new_rel[3 * k + 2] = rz;
    new_pos[3 * k] = rx + c[0];
    new_pos[3 * k + 1] = ry + c[1];
    new_pos[3 * k + 2] = rz + c[2];
  }
  return 1;
}

/* Metropolis test (Replica.cpp:438-459) with an FP64 energy change:
 * accept if dE < 0, else if u < exp(-dE * 4184 / (R * T)). */
static int metropolis(double dE, double u, float temperature) {
  if (dE < 0.0) return 1;
  double beta = 4184.0 / ((double)8.314472f * (double)temperature);
  return (u < exp(-dE * beta)) ? 2 : 0;
}

void oracle_mc_run(const oracle_system* s, const oracle_params* p, oracle_replica* r,
                   uint64_t seed, uint32_t step0, uint32_t slot, uint32_t system, int n_steps,
                   int energy_mode, int* flags, int* mol, double* dE_out) {
  int maxlen = 0;
  for (int m = 0; m < s->n_mol; ++m) {
    int n = s->mol_start[m + 1] - s->mol_start[m];
    if (n > maxlen) maxlen = n;
  }
  float* np = (float*)malloc(sizeof(float) * 3 * (size_t)maxlen);
  float* nr = (float*)malloc(sizeof(float) * 3 * (size_t)maxlen);
  float* trial = NULL;
  if (energy_mode == 1) trial = (float*)malloc(sizeof(float) * 3 * (size_t)s->n_beads);
  for (int st = 0; st < n_steps; ++st) {
    double u[6];
    oracle_step_uniforms(seed, step0 + (uint32_t)st, slot, system, u);
    int m = (int)(u[0] * (double)s->n_mol);
    float nc[3];
    double nq[4];
    oracle_propose(s, r, m, u, np, nr, nc, nq);
    int m0 = s->mol_start[m], n = s->mol_start[m + 1] - m0;
    double dE;
    if (energy_mode == 0) {
      double e_new = oracle_energy_molecule(s, p, r->pos, m, np);
      double e_old = oracle_energy_molecule(s, p, r->pos, m, r->pos + 3 * m0);
      dE = e_new - e_old;
    } else {
      memcpy(trial, r->pos, sizeof(float) * 3 * (size_t)s->n_beads);
      memcpy(trial + 3 * m0, np, sizeof(float) * 3 * (size_t)n);
      dE = oracle_energy_full(s, p, trial) - r->energy;
    }
    int f = metropolis(dE, u[5], r->temperature);
    if (f) {
      memcpy(r->pos + 3 * m0, np, sizeof(float) * 3 * (size_t)n);
      memcpy(r->rel + 3 * m0, nr, sizeof(float) * 3 * (size_t)n);
      memcpy(r->centre + 3 * m, nc, sizeof(nc));
      memcpy(r->quat + 4 * m, nq, sizeof(nq));
      r->energy = (energy_mode == 0) ? r->energy + dE : r->energy + dE;
      if (f == 1)
        r->accept++;
      else
        r->acceptA++;
    } else {
      r->reject++;
    }
    if (flags) flags[st] = f;
    if (mol) mol[st] = m;
    if (dE_out) dE_out[st] = dE;
  }
  free(np);
  free(nr);
  free(trial);
}

/* ------------------------------------------------------------- exchange */
/* main.cpp:1427-1453: delta = (1/T_i - 1/T_j)(E_i - E_j) 4184/R,
 * accept if u < min(1, exp(delta)); Replica::exchangeReplicas swaps the
 * temperature (and label/statistics), never coordinates or step sizes. */
int oracle_exchange_round(int R, int offset, const float* ladder, const double* energies,
                          int* temp_of_slot, int* slot_of_temp, uint64_t seed, uint32_t round,
                          uint32_t system, int* accepted) {
  int count = 0, pair = 0;
  for (int t = offset; t < R - 1; t += 2, ++pair) {
    int a = slot_of_temp[t], b = slot_of_temp[t + 1];
    double Ti = (double)ladder[t], Tj = (double)ladder[t + 1];
    double delta = (1.0 / Ti - 1.0 / Tj) * (energies[a] - energies[b]) *
                   (double)(4184.0f / 8.314472f);
    double u = oracle_exchange_uniform(seed, round, (uint32_t)pair, system);
    double pacc = exp(delta);
    if (pacc > 1.0) pacc = 1.0;
    int acc = (u < pacc);
    if (acc) {
      slot_of_temp[t] = b;
      slot_of_temp[t + 1] = a;
      temp_of_slot[a] = t + 1;
      temp_of_slot[b] = t;
      count++;
    }
    if (accepted) accepted[pair] = acc;
  }
  return count;
}

/* -------------------------------------------------------------- adjoint */
void oracle_energy_adjoint(const oracle_system* s, const oracle_params* p, const float* pos,
                           const float* raw_table, double* forces, double* dE_dlambda,
                           double* dE_dxi, double* dE_deps) {
  double lj_scale = (double)p->lj_cf * (double)p->kbt_cf;
  double dh_scale = (double)p->dh_const * (double)p->kbt_cf;
  double xi = (double)p->debye_length;
  memset(forces, 0, sizeof(double) * 3 * (size_t)s->n_beads);
  memset(dE_deps, 0, sizeof(double) * 32 * 32);
  double dl = 0.0, dx = 0.0;
  for (int mi = 0; mi < s->n_mol; ++mi) {
    for (int mj = mi + 1; mj < s->n_mol; ++mj) {
      int crowd = (s->mol_role[mi] == -1) || (s->mol_role[mj] == -1);
      for (int a = s->mol_start[mi]; a < s->mol_start[mi + 1]; ++a) {
        for (int b = s->mol_start[mj]; b < s->mol_start[mj + 1]; ++b) {
          double d[3];
          double r = min_image_r(pos + 3 * a, pos + 3 * b, (double)s->box, d);
          int ta = s->bead_type[a], tb = s->bead_type[b];
          double dedr = 0.0; /* d e / d r, kcal/mol/A */
          if (crowd) {
            double cut = (double)p->crowder_cutoff;
            if (!(cut > 0.0 && !(r < cut))) {
              if (p->crowder_mode == 0) {
                double t = 6.0 / r, t3 = t * t * t;
                dedr = -6.0 * t3 * t3 / r * lj_scale;
              } else {
                double sig = (double)s->type_rho[ta] + (double)s->type_rho[tb];
                double t = sig / r, t3 = t * t * t, t6 = t3 * t3;
                dedr = -12.0 * (double)p->crowder_eps * t6 * t6 / r * lj_scale;
              }
            }
          } else {
            double eps = (double)s->eps_table[ta * 32 + tb];
            double sigma = 0.5 * ((double)s->type_vdw[ta] + (double)s->type_vdw[tb]);
            double t = sigma / r, t3 = t * t * t, s6 = t3 * t3;
            double g = -4.0 * s6 * (s6 - 1.0);           /* dLJ/deps */
            double dg = 24.0 * s6 * (2.0 * s6 - 1.0) / r; /* d g / d r */
            if (eps > 0.0 && r < sigma * 1.122462048309372981433533049679) {
              g = -g + 2.0;
              dg = -dg;
            }
            double de_deps = g * lj_scale;
            dE_deps[ta * 32 + tb] += de_deps;
            if (ta != tb) dE_deps[tb * 32 + ta] += de_deps;
            dl += de_deps * ((double)raw_table[ta * 20 + tb] - (double)p->e0);
            double qq = (double)s->type_q[ta] * (double)s->type_q[tb];
            double ex = exp(-r / xi);
            dx += qq * ex / (xi * xi) * dh_scale;
            dedr = eps * dg * lj_scale + qq * ex * (-1.0 / (xi * r) - 1.0 / (r * r)) * dh_scale;
          }
          for (int k = 0; k < 3; ++k) {
            double f = dedr * d[k] / r;
            forces[3 * a + k] -= f;
            forces[3 * b + k] += f;
          }
        }
      }
    }
  }
  *dE_dlambda = dl;
  *dE_dxi = dx;
}

/* ----------------------------------------------------------- post-processing */
static void post_normalize(double q[4]) {
  double m = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  q[0] /= m;
  q[1] /= m;
  q[2] /= m;
  q[3] /= m;
}

/* Quaternion::rotateVector (Quaternion.cpp:84-101), FP64, result rounded to FP32. */
static void post_rotate(const double q[4], const float* v, float* out) {
  double w = q[0], x = q[1], y = q[2], z = q[3];
  double w2 = w * w, x2 = x * x, y2 = y * y, z2 = z * z;
  double wx = w * x, wy = w * y, wz = w * z, xy = x * y, xz = x * z, yz = y * z;
  double vx = v[0], vy = v[1], vz = v[2];
  out[0] = (float)(vx * (w2 + x2 - y2 - z2) + (vy * (xy - wz) + vz * (wy + xz)) * 2.0);
  out[1] = (float)((vx * (wz + xy) + vz * (yz - wx)) * 2.0 + vy * (w2 - x2 + y2 - z2));
  out[2] = (float)((vx * (xz - wy) + vy * (yz + wx)) * 2.0 + vz * (w2 - x2 - y2 + z2));
}

/* positioni -= boundary * round(v / boundary), v = positioni - molecule 0's
 * position, per axis in FP32 (pdbgen.cpp:196-203) */
static void post_image(float* c, const float* p, float box) {
  for (int k = 0; k < 3; ++k) {
    float v = c[k] - p[k];
    c[k] -= box * roundf(v / box);
  }
}

void oracle_post_rebuild(const float* rel0, const int* mol_start, int n_mol, const int* shift,
                         const float* centre0, float box, const double* quat,
                         const float* centre, float* pos) {
  float p0[3] = {centre[0], centre[1], centre[2]};
  if (shift[0]) post_image(p0, centre0, box);
  for (int m = 0; m < n_mol; ++m) {
    double q[4] = {quat[4 * m], quat[4 * m + 1], quat[4 * m + 2], quat[4 * m + 3]};
    post_normalize(q); /* pdbgen.cpp:191 */
    post_normalize(q); /* Molecule::setRotation (Molecule.cpp:335-346) */
    float c[3] = {centre[3 * m], centre[3 * m + 1], centre[3 * m + 2]};
    if (m == 0) {
      c[0] = p0[0];
      c[1] = p0[1];
      c[2] = p0[2];
    } else if (shift[m]) {
      post_image(c, p0, box);
    }
    for (int b = mol_start[m]; b < mol_start[m + 1]; ++b) {
      float r[3];
      post_rotate(q, rel0 + 3 * b, r);
      pos[3 * b] = r[0] + c[0];
      pos[3 * b + 1] = r[1] + c[1];
      pos[3 * b + 2] = r[2] + c[2];
    }
  }
}

/* Vector3f::magnitude of a - b (post processor/pdbgensrc/vector3f.h:35). */
static float post_dist(const float* a, const float* b) {
  float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return sqrtf(dx * dx + dy * dy + dz * dz);
}

double oracle_post_drms(const float* sim, const float* ref, const int* mol_start, int n_mol,
                        int reverse, float native_cut, float recovered_cut, long long* counts) {
  double drms = 0.0, N = 0.0;
  long long nat = 0, rec = 0, bind = 0;
  for (int I = 0; I < n_mol; ++I)
    for (int J = I + 1; J < n_mol; ++J)
      for (int i = mol_start[I]; i < mol_start[I + 1]; ++i)
        for (int j = mol_start[J]; j < mol_start[J + 1]; ++j) {
          N += 1.0;
          float ds = post_dist(sim + 3 * i, sim + 3 * j);
          float de = post_dist(ref + 3 * i, ref + 3 * j);
          drms += fabsf(ds - de);
          if (de < native_cut) {
            ++nat;
            if (ds < recovered_cut) ++rec;
          }
          if (ds < native_cut) ++bind;
        }
  drms /= N;
  if (reverse) {
    double drms2 = 0.0;
    for (int I = 0; I < n_mol; ++I)
      for (int J = I + 1; J < n_mol; ++J)
        for (int i = mol_start[I]; i < mol_start[I + 1]; ++i)
          for (int j = mol_start[J]; j < mol_start[J + 1]; ++j) {
            int li = i - mol_start[I], lj = j - mol_start[J];
            float ds = post_dist(sim + 3 * i, sim + 3 * j);
            float dr = post_dist(ref + 3 * (mol_start[J] + li), ref + 3 * (mol_start[I] + lj));
            drms2 += fabsf(ds - dr);
          }
    drms2 /= N;
    if (drms2 < drms) drms = drms2;
  }
  if (counts) {
    counts[0] = nat;
    counts[1] = rec;
    counts[2] = bind;
  }
  return drms;
}
