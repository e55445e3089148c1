// Test-oracle harness around the reference CPU engine (TEST INFRASTRUCTURE).
//
// This file is compiled together with the UNMODIFIED reference sources
// (simulation engine/src/{Replica,Molecule,AminoAcids,AminoAcid,vector3f,
// Quaternion,Residue,TorsionalLookupMatrix,Link}.cpp) by oracle/build.py into
// oracle/_ref/libremcref.so. Only tests, smoke() and bench.py's CPU baseline
// load it, to check the engine's results. The product never links it.
//
// It exposes a plain C ABI so the Python tests can:
//   * build a reference `Replica` from flat arrays (same state the GPU engine
//     holds: absolute bead positions, relative positions, centres, rotation
//     quaternions), bypassing the PDB loader;
//   * evaluate the reference's own `Replica::E()` (Replica.cpp:603-745) and
//     `Replica::E(Molecule*,Molecule*)` (Replica.cpp:793-828);
//   * run the reference's own `Replica::MCSearch` (Replica.cpp:368-478) one step
//     at a time, with its GSL generators fed from a caller-supplied uniform
//     stream (the shared Philox stream), and report every accept/reject.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#define private public  // Replica::translate/rotate are private; the harness probes them
#include "Replica.h"
#undef private

namespace {

struct Harness {
  AminoAcids aa;
  Replica rep;
  int ok;
  // argument evaluation order of the reference's random-vector constructors,
  // measured at start-up: order[k] = which component the k-th draw lands in.
  int vec_order_f[3];
  int vec_order_d[3];
};

void fill_amino_acids(AminoAcids& aa, const float* vdw, const float* charge,
                      const float* table) {
  for (int i = 0; i < 20; ++i) {
    aa.data[i].vanderWaalRadius = vdw[i];
    aa.data[i].electrostaticCharge = charge[i];
    aa.data[i].index = i;
    aa.data[i].shortSymbol = (char)('a' + i);
    std::snprintf(aa.data[i].sname, 4, "T%02d", i);
    std::snprintf(aa.data[i].name, 20, "type%02d", i);
    for (int j = 0; j < 20; ++j) aa.LJpotentials[i][j] = table[i * 20 + j];
  }
  aa.clean = true;
}

int probe_component(const Vector3f& v) {
  if (v.x != 0.0f) return 0;
  if (v.y != 0.0f) return 1;
  return 2;
}
int probe_component_d(const Vector3double& v) {
  if (v.x != 0.0) return 0;
  if (v.y != 0.0) return 1;
  return 2;
}

// Determine in which vector component the k-th uniform draw of
// createNormalisedRandomVector{,d} (Replica.cpp:303-318) ends up: C++ leaves the
// evaluation order of constructor arguments unspecified.
void probe_vector_order(Harness* h) {
  gsl_rng* r = gsl_rng_alloc(gsl_rng_mt19937);
  for (int k = 0; k < 3; ++k) {
    remc_stub_feed_clear(r);
    for (int t = 0; t < 3; ++t) remc_stub_feed(r, t == k ? 0.9 : 0.5);
    h->vec_order_f[k] = probe_component(h->rep.createNormalisedRandomVector(r));
    remc_stub_feed_clear(r);
    for (int t = 0; t < 3; ++t) remc_stub_feed(r, t == k ? 0.9 : 0.5);
    h->vec_order_d[k] = probe_component_d(h->rep.createNormalisedRandomVectord(r));
  }
  gsl_rng_free(r);
}

}  // namespace

extern "C" {

// Build a reference Replica.
//   vdw[20], charge[20], table[400]: the amino-acid table and the raw pair table
//     M_ab (the reference evaluates eps_ab = lambda*(M_ab - e0), definitions.h:33-35)
//   mol_start[n_mol+1], mol_role[n_mol] (0 = chain, -1 = crowder)
//   bead_type[N] (0..19), pos/rel [3N] float, centre [3*n_mol] float, quat [4*n_mol] (w,x,y,z)
void* ref_replica_create(const float* vdw, const float* charge, const float* table, int n_mol,
                         const int* mol_start, const int* mol_role, const int* bead_type,
                         const float* pos, const float* rel, const float* centre,
                         const double* quat, float box, float temperature) {
  Harness* h = new Harness();
  fill_amino_acids(h->aa, vdw, charge, table);
  Replica& r = h->rep;
  r.setAminoAcidData(h->aa);
  r.setBoundingValue(box);
  r.initTimers();
  r.reserveConiguousMoleculeArray(n_mol);
  r.moleculeCount = n_mol;
  r.residueCount = mol_start[n_mol];
  r.maxMoleculeSize = 0;
  r.nonCrowderCount = 0;
  for (int m = 0; m < n_mol; ++m) {
    Molecule& M = r.molecules[m];
    int n = mol_start[m + 1] - mol_start[m];
    M.AminoAcidsData = h->aa;
    M.index = m;
    M.Residues = new Residue[n];
    M.residueCount = n;
    for (int k = 0; k < n; ++k) {
      int b = mol_start[m] + k;
      Residue& R = M.Residues[k];
      R.aminoAcidIndex = bead_type[b];
      R.electrostaticCharge = h->aa.data[bead_type[b]].electrostaticCharge;
      R.vanderWaalRadius = h->aa.data[bead_type[b]].vanderWaalRadius;
      R.position = Vector3f(pos[3 * b], pos[3 * b + 1], pos[3 * b + 2]);
      R.relativePosition = Vector3f(rel[3 * b], rel[3 * b + 1], rel[3 * b + 2]);
      R.chainId = 'A';
      R.resSeq = k + 1;
      R.moleculeID = m;
    }
    M.center = Vector3f(centre[3 * m], centre[3 * m + 1], centre[3 * m + 2]);
    M.position = M.center;
    M.rotation = Quaternion(quat[4 * m], quat[4 * m + 1], quat[4 * m + 2], quat[4 * m + 3]);
    M.moleculeRoleIdentifier = 0.0f;
    if (mol_role[m] == -1)
      M.setMoleculeRoleIdentifier(CROWDER_IDENTIFIER);  // Molecule.cpp:120-142
    else
      r.nonCrowderCount++;
    if (n > r.maxMoleculeSize) r.maxMoleculeSize = n;
  }
  r.setTemperature(temperature);
  r.potential = r.E();
  // generators used by MCSearch, switched to fed mode
  r.rng_moleculeSelection = gsl_rng_alloc(gsl_rng_mt19937);
  r.rng_rotate = gsl_rng_alloc(gsl_rng_mt19937);
  r.rng_rotateAmount = gsl_rng_alloc(gsl_rng_mt19937);
  r.rng_translate = gsl_rng_alloc(gsl_rng_mt19937);
  r.rng_translateAmount = gsl_rng_alloc(gsl_rng_mt19937);
  r.MCRng = gsl_rng_alloc(gsl_rng_mt19937);
  r.MCKbRng = gsl_rng_alloc(gsl_rng_mt19937);
  probe_vector_order(h);
  h->ok = 1;
  return h;
}

void ref_replica_destroy(void* hp) {
  Harness* h = (Harness*)hp;
  if (!h) return;
  h->rep.freeRNGs();
  for (int m = 0; m < h->rep.moleculeCount; ++m) delete[] h->rep.molecules[m].Residues;
  delete h;
}

double ref_replica_E(void* hp) { return ((Harness*)hp)->rep.E(); }

float ref_replica_E_pair(void* hp, int a, int b) {
  Harness* h = (Harness*)hp;
  return h->rep.E(&h->rep.molecules[a], &h->rep.molecules[b]);
}

double ref_replica_potential(void* hp) { return ((Harness*)hp)->rep.potential; }

void ref_replica_set_steps(void* hp, float translate_step, double rotate_step) {
  Harness* h = (Harness*)hp;
  h->rep.setTranslateStep(translate_step);
  h->rep.setRotateStep(rotate_step);
}

void ref_replica_get_state(void* hp, float* pos, float* rel, float* centre, double* quat) {
  Replica& r = ((Harness*)hp)->rep;
  int b = 0;
  for (int m = 0; m < r.moleculeCount; ++m) {
    Molecule& M = r.molecules[m];
    for (int k = 0; k < M.residueCount; ++k, ++b) {
      pos[3 * b] = M.Residues[k].position.x;
      pos[3 * b + 1] = M.Residues[k].position.y;
      pos[3 * b + 2] = M.Residues[k].position.z;
      rel[3 * b] = M.Residues[k].relativePosition.x;
      rel[3 * b + 1] = M.Residues[k].relativePosition.y;
      rel[3 * b + 2] = M.Residues[k].relativePosition.z;
    }
    centre[3 * m] = M.center.x;
    centre[3 * m + 1] = M.center.y;
    centre[3 * m + 2] = M.center.z;
    quat[4 * m] = M.rotation.w;
    quat[4 * m + 1] = M.rotation.x;
    quat[4 * m + 2] = M.rotation.y;
    quat[4 * m + 3] = M.rotation.z;
  }
}

// Run `n_steps` steps of the reference's own Replica::MCSearch, feeding its
// generators from u[6*n_steps]: per step (molecule, move type, three vector
// draws in component order x,y,z, Metropolis). Writes per step:
//   flags[s] = 0 reject, 1 accept with dE < 0, 2 accept by Boltzmann test
//   mol[s] = molecule moved, energies[s] = potential after the step.
// Returns the number of fed-queue underflows (0 when the stream lined up).
int ref_replica_mcsearch(void* hp, int n_steps, const double* u, int* flags, int* mol,
                         double* energies) {
  Harness* h = (Harness*)hp;
  Replica& r = h->rep;
  int underflow = 0;
  for (int s = 0; s < n_steps; ++s) {
    const double* us = u + 6 * s;
    gsl_rng* all[7] = {r.rng_moleculeSelection, r.MCRng, r.rng_rotate, r.rng_translate,
                       r.MCKbRng, r.rng_rotateAmount, r.rng_translateAmount};
    for (int k = 0; k < 7; ++k) remc_stub_feed_clear(all[k]);
    remc_stub_feed(r.rng_moleculeSelection, us[0]);
    // gsl_ran_bernoulli returns 1 (= rotate, Replica.cpp:320-321) when u < 0.5
    remc_stub_feed(r.MCRng, us[1]);
    // the k-th draw lands in component vec_order[k]; feed so component c gets us[2+c]
    for (int k = 0; k < 3; ++k) {
      remc_stub_feed(r.rng_rotate, us[2 + h->vec_order_d[k]]);
      remc_stub_feed(r.rng_translate, us[2 + h->vec_order_f[k]]);
    }
    remc_stub_feed(r.MCKbRng, us[5]);
    int a0 = r.accept, a1 = r.acceptA;
    // which molecule will move: same arithmetic as gsl_rng_uniform_int
    mol[s] = (int)(us[0] * (double)r.moleculeCount);
    r.MCSearch(1);
    flags[s] = (r.accept != a0) ? 1 : ((r.acceptA != a1) ? 2 : 0);
    energies[s] = r.potential;
    for (int k = 0; k < 7; ++k) {
      underflow += all[k]->feed_underflow;
      all[k]->feed_underflow = 0;
    }
  }
  return underflow;
}

// Evaluate the reference random-vector helpers on one fed triple (checks the
// vector mapping the GPU engine reproduces).
void ref_random_vectors(void* hp, const double* u3, float* vf, double* vd) {
  Harness* h = (Harness*)hp;
  gsl_rng* r = gsl_rng_alloc(gsl_rng_mt19937);
  remc_stub_feed_clear(r);
  for (int k = 0; k < 3; ++k) remc_stub_feed(r, u3[h->vec_order_f[k]]);
  Vector3f a = h->rep.createNormalisedRandomVector(r);
  remc_stub_feed_clear(r);
  for (int k = 0; k < 3; ++k) remc_stub_feed(r, u3[h->vec_order_d[k]]);
  Vector3double b = h->rep.createNormalisedRandomVectord(r);
  gsl_rng_free(r);
  vf[0] = a.x; vf[1] = a.y; vf[2] = a.z;
  vd[0] = b.x; vd[1] = b.y; vd[2] = b.z;
}

// Timing driver for the CPU baseline (ref_time_mcsearch below): the
// reference's own Replica::MCSearch (Replica.cpp:368-478, full Replica::E()
// every step, MT19937 draws) on replicas spread over host threads, after
// seeding each. (The reference executable itself cannot load more than 30
// molecules: Replica::loadMolecule grows its array with a shallow memcpy and
// the deleted originals free the file names the copies still hold.)
// Leave fed mode and seed the replica's seven MT19937 generators (from
// `seed`), as Replica::initRNGs does from the clock (Replica.cpp:265-300).
void ref_replica_seed(void* hp, unsigned seed) {
  Replica& r = ((Harness*)hp)->rep;
  gsl_rng* all[7] = {r.rng_moleculeSelection, r.MCRng, r.rng_rotate, r.rng_translate,
                     r.MCKbRng, r.rng_rotateAmount, r.rng_translateAmount};
  for (int k = 0; k < 7; ++k) {
    all[k]->fed = 0;
    gsl_rng_set(all[k], 7u * seed + (unsigned)k + 1u);
  }
}

// accept, acceptA, reject of the replica (Replica.h:120-122).
void ref_replica_counters(void* hp, int* out) {
  Replica& r = ((Harness*)hp)->rep;
  out[0] = r.accept;
  out[1] = r.acceptA;
  out[2] = r.reject;
}

// The reference's own Replica::MCSearch(n_steps) on `n` replicas over
// `n_threads` host threads, replicas assigned in contiguous slices as
// MCthreadableFunction does (main.cpp:879-883), with their own generators
// (not fed). Returns wall seconds.
double ref_run_mcsearch(void** handles, int n, int n_threads, int n_steps) {
  if (n_threads < 1) n_threads = 1;
  if (n_threads > n) n_threads = n;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> pool;
  const int per = (n + n_threads - 1) / n_threads;
  for (int t = 0; t < n_threads; ++t) {
    pool.emplace_back([=]() {
      for (int i = t * per; i < n && i < (t + 1) * per; ++i)
        ((Harness*)handles[i])->rep.MCSearch(n_steps);
    });
  }
  for (auto& th : pool) th.join();
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

double ref_time_mcsearch(void** handles, int n, int n_threads, int n_steps) {
  for (int i = 0; i < n; ++i) ref_replica_seed(handles[i], 1000u + (unsigned)i);
  return ref_run_mcsearch(handles, n, n_threads, n_steps);
}

}  // extern "C"
