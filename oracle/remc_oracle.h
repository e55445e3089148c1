/* FP64 CPU oracle for the REMC docking hot path (TEST INFRASTRUCTURE).
 *
 * A plain-C restatement of the reference algorithm, used only by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg, to check the engine's results.
 * The product library never links it.
 *
 * Reference files followed (paths inside iantunbridge/RemcDockingSimulator):
 *   energy ............ simulation engine/src/Replica.cpp:533-600, 603-745
 *   molecule pair E ... simulation engine/src/Replica.cpp:793-828
 *   moves ............. simulation engine/src/Replica.cpp:303-364,
 *                       Molecule.cpp:88-102, 146-171, 247-333, Quaternion.cpp:84-101
 *   Metropolis ........ simulation engine/src/Replica.cpp:438-459
 *   exchange .......... simulation engine/src/main.cpp:1427-1453, Replica.cpp:145-159
 *   constants ......... simulation engine/src/definitions.h:11-35, 84-93
 *
 * Pair terms and accumulations are FP64 (the reference evaluates most pair
 * terms in FP32 with FP64 accumulators); the move arithmetic keeps the
 * reference's own precisions (FP32 positions, FP64 quaternions) so that a
 * trajectory can be followed bit for bit.
 */
#ifndef REMC_ORACLE_H
#define REMC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Energy model parameters (mirrors remc_params in include/remc_b200.h). */
typedef struct {
  float lambda_;        /* contact-energy scale (definitions.h:35: 0.159) */
  float e0;             /* contact-energy offset (definitions.h:34: -2.27) */
  float debye_length;   /* Xi, Angstrom (definitions.h:22: 10) */
  float dh_const;       /* 1.602176487^2 * 0.948 (Replica.cpp:624) */
  float lj_cf;          /* LJ_CONVERSION_FACTOR (definitions.h:23) */
  float kbt_cf;         /* KBTConversionFactor (definitions.h:18) */
  int crowder_mode;     /* 0: (6/r)^6 (Replica.cpp:584-587); 1: ((rho_i+rho_j)/r)^12 */
  float crowder_cutoff; /* 15 A in mode 0 (definitions.h:89); <=0: no cutoff */
  float crowder_eps;    /* prefactor of the r^-12 term (mode 1) */
} oracle_params;

/* One system (one replica's coordinates). Arrays are caller-owned.
 * Per bead: type (0..19 amino acid, 20+k crowder species), molecule index.
 * Per type (32 entries): vdw radius, charge, crowder radius rho.
 * eps_table[32*32]: eps_ab = float(lambda*(M_ab - e0)) for a,b < 20. */
typedef struct {
  int n_beads;
  int n_mol;
  const int* mol_start;  /* n_mol+1 */
  const int* mol_role;   /* n_mol: 0 chain, -1 crowder */
  const int* bead_type;  /* n_beads */
  const float* type_vdw; /* 32 */
  const float* type_q;   /* 32 */
  const float* type_rho; /* 32 */
  const float* eps_table;/* 32*32 */
  float box;
} oracle_system;

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11). */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* The six uniforms of MC step `step` of (system, slot):
 * u[0] molecule, u[1] move type, u[2..4] direction, u[5] Metropolis. */
void oracle_step_uniforms(uint64_t seed, uint32_t step, uint32_t slot, uint32_t system,
                          double u[6]);
/* Uniform for the exchange test of temperature pair `pair` in round `round`. */
double oracle_exchange_uniform(uint64_t seed, uint32_t round, uint32_t pair, uint32_t system);

/* Pair energy of beads a, b (different molecules) at squared min-image
 * distance, in kcal/mol; FP64. */
double oracle_pair_energy(const oracle_system* s, const oracle_params* p, int a, int b,
                          const float* pos);

/* Full-system energy (Replica::E), FP64 accumulation, kcal/mol. */
double oracle_energy_full(const oracle_system* s, const oracle_params* p, const float* pos);

/* Energy of molecule m against every other bead at positions pos, with the
 * beads of m taken from mpos (n_m*3 floats) instead. */
double oracle_energy_molecule(const oracle_system* s, const oracle_params* p, const float* pos,
                              int m, const float* mpos);

/* Non-crowder pair energy sum used by Replica::sample (Replica.cpp:1723-1743):
 * sum over chain pairs i<j of E(mol_i, mol_j) with the KH+DH model and no
 * crowder rule (Replica.cpp:793-828). */
/* Sum of |pair term| of molecule m at mpos against all other molecules. */
double oracle_energy_molecule_abs(const oracle_system* s, const oracle_params* p,
                                  const float* pos, int m, const float* mpos);
double oracle_noncrowder_pair_energy(const oracle_system* s, const oracle_params* p,
                                     const float* pos);

/* Mutable per-replica state. pos/rel: 3*n_beads floats; centre: 3*n_mol;
 * quat: 4*n_mol doubles (w,x,y,z). */
typedef struct {
  float* pos;
  float* rel;
  float* centre;
  double* quat;
  double energy;
  float temperature;
  float translate_step;
  double rotate_cos_half; /* cos(rotate_step/2) */
  double rotate_sin_half; /* sin(rotate_step/2) */
  int translate_only_crowders; /* 1: crowders are always translated */
  int accept;  /* dE < 0 */
  int acceptA; /* Boltzmann */
  int reject;
} oracle_replica;

/* Apply the move of uniforms u to molecule m of r (no energy). Writes the
 * proposed bead positions/relative positions into new_pos/new_rel (3*n_m each)
 * and the proposed centre/quaternion into new_centre/new_quat; returns 1 for a
 * rotation, 0 for a translation. */
int oracle_propose(const oracle_system* s, const oracle_replica* r, int m, const double u[6],
                   float* new_pos, float* new_rel, float* new_centre, double* new_quat);

/* Run n_steps MC steps. Per step writes flags (0 reject, 1 accept dE<0,
 * 2 accept Boltzmann), the moved molecule and dE (new - old, FP64).
 * `energy_mode` 0: accumulate E += dE (what the GPU engine does);
 * 1: recompute the full energy each step (what the reference does). */
void oracle_mc_run(const oracle_system* s, const oracle_params* p, oracle_replica* r,
                   uint64_t seed, uint32_t step0, uint32_t slot, uint32_t system, int n_steps,
                   int energy_mode, int* flags, int* mol, double* dE);

/* One replica-exchange round over R replica slots of one system.
 * temp_of_slot[R]: temperature index held by each slot; slot_of_temp[R]: its
 * inverse; ladder[R]: temperature of each index (increasing); energies[R] per
 * slot. Pairs (t, t+1) for t = offset, offset+2, ... Swaps the mapping on
 * acceptance. Returns the number of exchanges; writes the accepted flags per
 * pair into accepted[] (length (R - offset) / 2). */
int oracle_exchange_round(int R, int offset, const float* ladder, const double* energies,
                          int* temp_of_slot, int* slot_of_temp, uint64_t seed, uint32_t round,
                          uint32_t system, int* accepted);

/* Adjoint: per-bead forces F = -dE/dr (3*n_beads), dE/dlambda, dE/dxi and
 * dE/deps[32*32] (upper+lower symmetric entries both accumulated). FP64. */
void oracle_energy_adjoint(const oracle_system* s, const oracle_params* p, const float* pos,
                           const float* raw_table, double* forces, double* dE_dlambda,
                           double* dE_dxi, double* dE_deps);

/* Post-processing.
 * oracle_post_rebuild: pdbgen's pose reconstruction
 * (post processor/pdbgensrc/pdbgen.cpp:166-215): quaternion normalised twice
 * (pdbgen, Molecule::setRotation, Quaternion.cpp:18-27), rel0 rotated by
 * Quaternion::rotateVector, shifted centres moved to the image nearest
 * molecule 0 (molecule 0 against centre0), bead = rel + centre (FP32).
 * oracle_post_drms: DRMS(Replica*, Replica*, bool)
 * (post processor/pdbgensrc/drms.cpp:7-57) in its loop order, and the contact
 * counts of DRMS(Replica*, Replica*) (simulation engine/src/main.cpp:789-836)
 * with the thresholds as arguments. One frame per call. */
void oracle_post_rebuild(const float* rel0, const int* mol_start, int n_mol, const int* shift,
                         const float* centre0, float box, const double* quat,
                         const float* centre, float* pos);
double oracle_post_drms(const float* sim, const float* ref, const int* mol_start, int n_mol,
                        int reverse, float native_cut, float recovered_cut, long long* counts);

#ifdef __cplusplus
}
#endif
#endif
