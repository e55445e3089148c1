/* remc_b200.h - C ABI of the B200 replica-exchange Monte Carlo docking engine.
 *
 * One handle holds many independent REMC systems (rigid residue-level chains
 * and crowders in a periodic box), each with its own replicas, resident on one
 * GPU. Every entry point returns an int status (REMC_OK = 0, negative on
 * error; remc_last_error_string() gives the message). No entry point exits or
 * aborts the process. A handle is not thread-safe: use one handle per host
 * thread. All work is stream-ordered on a handle-owned CUDA stream.
 *
 * Counterparts in the reference (iantunbridge/RemcDockingSimulator, paths
 * inside the project):
 *   remc_energy_full ....... Replica::EonDevice / CUDA_EonDevice
 *                            (simulation engine/src/Replica.cpp:1601-1616,
 *                             CudaFunctions.cu:304-385) and Replica::E()
 *                            (Replica.cpp:603-745)
 *   remc_sweep ............. Replica::MCSearch (Replica.cpp:368-478), run for
 *                            all replicas of all systems at once
 *   remc_exchange .......... the exchange loop of REMCSimulation
 *                            (main.cpp:1427-1453) + Replica::exchangeReplicas
 *                            (Replica.cpp:145-159)
 *   remc_upload_state ...... Replica::ReplicaDataToDevice (Replica.cpp:1308-1417)
 *   remc_download_state .... Replica::ReplicaDataToHost (Replica.cpp:1433-1480)
 *   remc_set_type_tables ... copyLJPotentialDataToDevice + bindLJTexture
 *                            (CudaFunctions.cu:20-33, 112-131)
 *   remc_set_params ........ the compile-time constants of definitions.h:11-35
 *                            and CUDA_setBoxDimension (CudaFunctions.cu:169-174)
 *   remc_delta_energy ...... no reference counterpart (the reference always
 *                            recomputes the full energy); ΔE of one rigid move
 */
#ifndef REMC_B200_H
#define REMC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define REMC_OK 0
#define REMC_ERR_INVALID (-1)   /* bad argument */
#define REMC_ERR_CUDA (-2)      /* CUDA runtime error */
#define REMC_ERR_NOMEM (-3)     /* device or host allocation failed */
#define REMC_ERR_STATE (-4)     /* call out of order (e.g. no state uploaded) */
#define REMC_ERR_NUMERIC (-5)   /* non-finite input coordinates */
#define REMC_ERR_TIMEOUT (-6)   /* a bounded device-side wait gave up */

#define REMC_NUM_AMINO 20       /* residue types 0..19 */
#define REMC_MAX_TYPES 24       /* 20 residue types + up to 4 crowder species */

typedef struct remc_handle remc_handle;

/* Energy model. Defaults (remc_default_params) are the reference's
 * compile-time values (definitions.h:11-35, 89; Replica.cpp:624). */
typedef struct {
  float lambda_;        /* contact-energy scale lambda (0.159) */
  float e0;             /* contact-energy offset e0 (-2.27) */
  float debye_length;   /* Debye length Xi in Angstrom (10) */
  float dh_const;       /* 0.948 * 1.602176487^2 */
  float lj_cf;          /* LJ_CONVERSION_FACTOR 0.3507221006079 */
  float kbt_cf;         /* KBTConversionFactor 1/(294 R/4184) */
  int crowder_mode;     /* 0: (6/r)^6 (reference); 1: eps_c ((rho_i+rho_j)/r)^12 */
  float crowder_cutoff; /* crowder pair cutoff in Angstrom (15); <= 0: none */
  float crowder_eps;    /* eps_c, prefactor of the r^-12 crowder term */
} remc_params;

/* One system: topology shared by all of its replicas. Bead types 0..19 are
 * residue types; types 20..23 are crowder species. A molecule is a crowder
 * iff mol_role = -1; all beads of a crowder molecule must have crowder types,
 * all beads of a chain residue types. */
typedef struct {
  int n_beads;
  int n_mol;
  int n_replicas;
  const int* mol_start;   /* [n_mol + 1], mol_start[0] = 0, increasing */
  const int* mol_role;    /* [n_mol]: 0 chain, -1 crowder */
  const int* bead_type;   /* [n_beads] */
  float box;              /* periodic box edge, Angstrom */
  int translate_only_crowders; /* 1: crowders are never rotated */
} remc_system_desc;

void remc_default_params(remc_params* p);

int remc_create(const remc_system_desc* systems, int n_systems, const remc_params* params,
                remc_handle** out);
int remc_destroy(remc_handle* h);
int remc_set_params(remc_handle* h, const remc_params* params);

/* Per-type tables (REMC_MAX_TYPES entries each): vdW radius (sigma_ij is the
 * mean of the two radii), charge, crowder radius rho; raw pair table
 * M[20*20] (eps_ab = lambda (M_ab - e0) evaluated in FP32, as the reference
 * does at CudaFunctions.cu:581-594). */
int remc_set_type_tables(remc_handle* h, const float* vdw, const float* charge, const float* rho,
                         const float* pair_table_20x20);

/* Instance layout: replica-instances are numbered system by system, slot by
 * slot: inst = sum_{s' < s} R_s' + slot. Bead arrays are 3 floats per bead per
 * instance in the same order; molecule arrays 3 floats (centre) or 4 doubles
 * (quaternion w,x,y,z) per molecule per instance. */
int remc_upload_state(remc_handle* h, const float* pos, const float* rel, const float* centre,
                      const double* quat);
int remc_download_state(remc_handle* h, float* pos, float* rel, float* centre, double* quat);

/* Temperature ladder per system (R floats per system, increasing, the
 * instance order above), translate step (float) and rotate step (radians,
 * double) per instance. Resets every slot to hold temperature index = slot. */
int remc_set_replica_params(remc_handle* h, const float* ladder, const float* translate_step,
                            const double* rotate_step);

/* Full-system energy of every instance (kcal/mol), written to out[n_inst]
 * (host) when out != NULL; also becomes each instance's running energy. */
int remc_energy_full(remc_handle* h, double* out);
int remc_get_energies(remc_handle* h, double* out);

/* Advance every replica of every system by n_steps Metropolis steps (one
 * persistent launch per sweep). Random numbers: Philox4x32-10 with key =
 * seed, counter = (step0 + s, slot, system, purpose). */
int remc_sweep(remc_handle* h, int n_steps, uint64_t seed, uint32_t step0);
/* Same trajectory as remc_sweep, one kernel launch per replica per step
 * (the per-replica launch pattern of the reference). */
int remc_sweep_plain(remc_handle* h, int n_steps, uint64_t seed, uint32_t step0);

/* One exchange round in every system: temperature pairs (t, t+1) for
 * t = offset, offset + 2, ...; counter = (round, pair, system, 2). */
int remc_exchange(remc_handle* h, uint64_t seed, uint32_t round, int offset);

/* temp_of_slot[n_inst]: temperature index held by each instance's slot. */
int remc_get_temperature_map(remc_handle* h, int* temp_of_slot);
/* Checkpoint restore (no reference counterpart; the reference's resume path,
 * main.cpp:119-160, re-derives conformations from rounded text): set the
 * temperature index held by every slot (a permutation of 0..R-1 within each
 * system), and the running energy and chain-chain energy of every instance
 * (noncrowder may be NULL), so that a restored run continues bit for bit. */
int remc_set_temperature_map(remc_handle* h, const int* temp_of_slot);
int remc_set_energies(remc_handle* h, const double* energy, const double* noncrowder);
/* Per-instance move counters since the last reset: accepted with dE < 0,
 * accepted by the Boltzmann test, rejected; exchange counters per system. */
int remc_get_counters(remc_handle* h, int* accept, int* acceptA, int* reject);
int remc_reset_counters(remc_handle* h);

/* Pair evaluations made by the sweeps since the last counter reset, summed
 * over instances: residue-residue pairs (Kim-Hummer + Debye-Hueckel) and
 * pairs involving a crowder. A dE pair counts twice (old and new position). */
int remc_get_pair_evaluations(remc_handle* h, uint64_t* residue_pairs, uint64_t* crowder_pairs);

/* Sampling (Replica::sample, Replica.cpp:1717-1780, driven as in
 * MCthreadableFunction, main.cpp:975-989): inside every sweep, after each
 * chunk of `sample_every` steps, a replica is sampled if the chunk's label
 * (sweep start step + chunk start) is >= sample_after. It counts as bound if
 * its potential, plus the chain-chain pair energy when crowders are present
 * (the reference's sum), is below bound_threshold (-1.1844 kcal/mol in the
 * reference, definitions.h:84). Bound samples append a record and one pose per
 * molecule to device buffers of max_records / max_poses entries (0: count
 * only); records that do not fit are counted as dropped. sample_every = 0
 * turns sampling off. Chains must precede crowders in every system. */
typedef struct {
  int inst;
  uint32_t label;
  double e_noncrowder;  /* the value compared with the threshold */
  double e_total;       /* potential */
  float temperature;
  int n_mol;
  int pose_offset;      /* first pose of this record in the pose array */
} remc_sample;
typedef struct {
  double q[4];          /* rotation quaternion w, x, y, z */
  float centre[3];
} remc_sample_pose;
int remc_set_sampling(remc_handle* h, int sample_every, uint32_t sample_after,
                      double bound_threshold, int max_records, int max_poses);
/* Per-instance samples taken and bound samples since the last counter reset. */
int remc_get_sample_counters(remc_handle* h, int* samples, int* bound);
/* Copy out the records and poses written since the last call and clear the
 * buffers. n_dropped receives the records that did not fit. */
int remc_read_samples(remc_handle* h, remc_sample* records, int max_records,
                      remc_sample_pose* poses, int max_poses, int* n_records, int* n_poses,
                      int* n_dropped);
/* Chain-chain part of each instance's energy (sum of E(Molecule*,Molecule*)
 * over chain pairs, Replica.cpp:793-828), tracked with the running energy. */
int remc_get_noncrowder_energies(remc_handle* h, double* out);

/* Adjoint of the full energy of every instance (no reference counterpart:
 * the reference has no gradients). Outputs (host, any may be NULL):
 *   forces[3 per bead per instance]      F = -dE/dr (FP32, kcal/mol/A)
 *   mol_force_torque[6 per molecule]     sum F and torque sum rel x F about
 *                                        the centre (FP64)
 *   dE_dlambda[n_inst], dE_dxi[n_inst]   kcal/mol per unit lambda / per A
 *   dE_deps[400 per instance]            derivative with respect to the
 *                                        symmetric contact energy eps_ab
 *                                        (entries ab and ba both hold it)
 *   energy[n_inst]                       the energy the adjoint saw
 * Forces are summed with FP32 atomics (order-dependent in the last bits). */
int remc_energy_adjoint(remc_handle* h, float* forces, double* mol_force_torque,
                        double* dE_dlambda, double* dE_dxi, double* dE_deps, double* energy);

/* The handle's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events after the engine's. */
int remc_get_stream(remc_handle* h, void** stream);

/* dE of moving molecule `mol` of instance `inst` to new_pos (3 floats per
 * bead, host), FP32 pairs with FP64 sum; the state is not changed. */
int remc_delta_energy(remc_handle* h, int inst, int mol, const float* new_pos, double* dE);

/* Run n_blocks of (sweep of steps_per_block steps, exchange round), the step
 * and round counters advancing on the device, as one CUDA graph per block
 * (captured on first use, replayed afterwards). */
int remc_run(remc_handle* h, int n_blocks, int steps_per_block, uint64_t seed, uint32_t step0,
             uint32_t round0);

/* Autotuner: times a probe sweep of probe_steps steps for each candidate
 * schedule (threads per replica 128 or 256; molecule centres in shared or
 * global memory; CTAs per replica 1, 2, 4, 8 where replicas are few) on the
 * handle's own systems, restores the state after every probe, and keeps the
 * fastest. Outputs (may be NULL): the chosen
 * threads, layout and probe time in ms. No reference counterpart (the
 * reference fixes its block size by system size, main.cpp:1746-1747). */
int remc_autotune(remc_handle* h, int probe_steps, uint64_t seed, int* threads,
                  int* mol_in_smem, float* best_ms);
/* Set the sweep schedule directly (threads 32, 64, 128 or 256). */
int remc_set_schedule(remc_handle* h, int threads, int mol_in_smem);
/* CTAs per replica: 1, or a thread-block cluster of 2, 4 or 8 CTAs that share
 * each replica's pair loops (for batches with fewer replicas than SMs). The
 * autotuner also tries clusters when n_inst * size <= 2 * SMs. No reference
 * counterpart. */
int remc_set_cluster(remc_handle* h, int cluster);
int remc_get_schedule(remc_handle* h, int* threads, int* mol_in_smem, int* cluster);
/* Where the sweep keeps each replica's beads: 1 = resident in shared memory
 * (the default whenever the largest system fits), 0 = in place in global
 * memory, with the chain's trial buffers in global scratch. Systems too large
 * for shared memory (about 13,000 beads, or chains of thousands of residues)
 * get 0 at remc_create; the reference's GPU path has no size limit either
 * (CudaFunctions.cu:304-385 tiles over global memory). Results are identical
 * either way. No reference counterpart. */
int remc_set_bead_storage(remc_handle* h, int in_shared_memory);
/* Per system, 1 when the sweep folds the minimum image (min(|d|, L - |d|) per
 * axis instead of d - L rint(d/L)): set at every remc_upload_state when, on
 * every axis, [min(p_min, -R), max(p_max, L + R)] is shorter than 1.5 L (with
 * a margin), p the uploaded bead positions and R the largest bead distance
 * from its centre, so that no bead pair the sweep can reach is 1.5 box
 * lengths apart (moved molecules keep their centre in [0, L)). Results
 * equal the unfolded ones except for pairs half a box apart to within a
 * rounding. No reference counterpart. */
int remc_get_fold_flags(remc_handle* h, int* per_system);
int remc_get_bead_storage(remc_handle* h, int* in_shared_memory);
/* Work order of the persistent sweep (single CTAs per replica). 1 (the
 * default): before each launch, a kernel sums what every replica's proposals
 * for the block cost (the pair evaluations of each step's moved molecule plus
 * a per-step allowance) and a second ranks the replicas, so the work queue
 * hands out the most expensive blocks first and the slots finish together.
 * 0: the static order fixed at remc_create (by each system's expected cost
 * per step). Results are identical either way: every replica's trajectory is
 * independent of when it runs. launches_per_sweep (may be NULL): kernels per
 * sweep launch, 4 with the cost order (proposals, cost, rank, sweep), else 2.
 * No reference counterpart. */
int remc_set_work_order(remc_handle* h, int by_cost);
int remc_get_work_order(remc_handle* h, int* by_cost, int* launches_per_sweep);

int remc_sync(remc_handle* h);
/* Failure-path check: runs one warp whose bounded device-side wait (the one
 * the energy kernel uses for its tile copies) waits for something that never
 * happens, gives up after `polls` polls (1 .. 2^20) and sets the handle's
 * error word. Returns REMC_ERR_TIMEOUT, as a call whose tile copy never
 * landed would; the handle stays usable. No reference counterpart (the
 * reference aborts through cutil on device errors). */
int remc_check_wait_timeout(remc_handle* h, int polls);
int remc_num_instances(const remc_handle* h);
const char* remc_last_error_string(void);

#ifdef __cplusplus
}
#endif
#endif
