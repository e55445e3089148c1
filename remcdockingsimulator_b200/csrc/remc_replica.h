// remc_replica.h - C++ facade of the B200 REMC engine under the reference's
// class and method names (namespace remc).
//
// The reference's host API (simulation engine/src/Replica.h:29-302,
// Molecule.h:24-126, AminoAcids.h:6-27) is mapped onto the batched C ABI of
// remc_b200.h:
//   AminoAcids::loadAminoAcidData / loadLJPotentialData .. AminoAcids.cpp:25-139
//   Molecule::initFromPDB (CA beads) ....................... Molecule.cpp:430-830
//   Molecule::translate / setPosition / rotateQ / setRotation,
//     saveBeforeStateChange / undoStateChange .............. Molecule.cpp:88-102,
//                                                            146-171, 247-346
//   Replica::loadMolecule ................................. Replica.cpp:230-263
//   Replica::E / EonDevice ........ remc_energy_full (the energy always runs on
//                                   the GPU; Replica.cpp:603-745, 1601-1616)
//   Replica::MCSearch ............. remc_sweep on a one-replica handle
//                                   (Replica.cpp:368-478)
//   Replica::exchangeReplicas ..... swap of label, temperature and statistics
//                                   (Replica.cpp:145-159)
//   Replica::ReplicaDataToDevice / ReplicaDataToHost / MoleculeDataToDevice /
//     FreeDevice .................. remc_create + remc_upload_state /
//                                   remc_download_state / remc_destroy
//   ReplicaExchange ............... the replica loop of REMCSimulation
//                                   (main.cpp:1106-1567) as remc_run: all
//                                   replicas of one system in one handle, MC
//                                   blocks and exchange rounds replayed as a
//                                   CUDA graph
//
// Error behaviour: the reference aborts the process on a CUDA failure; the
// facade throws remc::Error with the engine's message instead. Random numbers
// are the engine's counter-based Philox stream keyed by each Replica's seed
// (the reference seeds GSL generators from the clock, Replica.cpp:265-300).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/remc_b200.h"

namespace remc {

constexpr float CROWDER_IDENTIFIER = -1.0f;      // definitions.h:92
constexpr float BOUND_ENERGY_VALUE = -1.1844f;   // definitions.h:84
constexpr float INITIAL_TRANSLATIONAL_STEP = 0.5f;  // definitions.h:78
constexpr float INITIAL_ROTATIONAL_STEP = 0.2f;     // definitions.h:81
constexpr float BOUNDING_VALUE = 150.0f;            // definitions.h:63

class Error : public std::runtime_error {
 public:
  using std::runtime_error::runtime_error;
};

struct Vector3f {
  float x = 0.0f, y = 0.0f, z = 0.0f;
  Vector3f() = default;
  Vector3f(float x_, float y_, float z_) : x(x_), y(y_), z(z_) {}
};

struct Vector3double {
  double x = 0.0, y = 0.0, z = 0.0;
  Vector3double() = default;
  Vector3double(double x_, double y_, double z_) : x(x_), y(y_), z(z_) {}
  void normalizeInPlace();  // vector3f.cpp:36-43
};

struct Quaternion {
  double w = 1.0, x = 0.0, y = 0.0, z = 0.0;
  Quaternion() = default;
  Quaternion(double w_, double x_, double y_, double z_) : w(w_), x(x_), y(y_), z(z_) {}
  void normalize();                                  // Quaternion.cpp:18-27
  Quaternion operator*(const Quaternion& q2) const;  // Quaternion.cpp:36-48
  Vector3f rotateVector(const Vector3f& v) const;    // Quaternion.cpp:84-101
};

struct AminoAcid {
  std::string name, sname;
  char symbol = 0;
  float vdwRadius = 0.0f;
  float electrostaticCharge = 0.0f;
};

class AminoAcids {
 public:
  AminoAcid data[REMC_NUM_AMINO];
  float LJpotentials[REMC_NUM_AMINO][REMC_NUM_AMINO] = {};
  bool loadAminoAcidData(const char* path);
  bool loadLJPotentialData(const char* path);
  int getAminoAcidIndex(const char* name) const;
  AminoAcid get(int i) const { return data[i]; }
  float getLJp(int a, int b) const { return LJpotentials[a][b]; }
};

struct Residue {
  Vector3f position;
  Vector3f relativePosition;
  int aminoAcidIndex = 0;
  float electrostaticCharge = 0.0f;
  float vdwRadius = 0.0f;
};

class Molecule {
 public:
  std::vector<Residue> Residues;
  int residueCount = 0;
  Vector3f center;
  Vector3f position;
  Quaternion rotation;
  float moleculeRoleIdentifier = 0.0f;
  int index = 0;
  std::string filename;
  AminoAcids AminoAcidsData;

  bool initFromPDB(const char* pdbfilename);
  bool translate(const Vector3f& v);
  void setPosition(const Vector3f& v);
  bool rotateQ(const Vector3double& axis, double angle);
  void setRotation(Quaternion q);
  void saveBeforeStateChange(const Molecule* m);
  void undoStateChange(const Molecule* m);
  void setMoleculeRoleIdentifier(float r) { moleculeRoleIdentifier = r; }
  float getMoleculeRoleIdentifier() const { return moleculeRoleIdentifier; }
  int getLength() const { return residueCount; }
  int getIndex() const { return index; }
  Vector3f getPosition() const { return position; }
  Quaternion getRotation() const { return rotation; }
  bool isCrowder() const { return moleculeRoleIdentifier == CROWDER_IDENTIFIER; }
};

class ReplicaExchange;

class Replica {
 public:
  Replica();
  ~Replica();
  Replica(const Replica& r);
  Replica& operator=(const Replica& r);
  void copy(const Replica& r);  // Replica.cpp:63-105: molecules, tables, settings

  void setAminoAcidData(const AminoAcids& a) { aminoAcids = a; }
  int loadMolecule(const char* pdbfilename);
  int loadMolecule(const char* pdbfilename, Vector3f position, Vector3double rotationAxis,
                   double rotationAmount);

  double E();          // full energy of this replica, computed on the GPU
  double EonDevice();  // the same (the reference's CUDA path)
  void MCSearch(int steps);
  void exchangeReplicas(Replica& r);

  void ReplicaDataToDevice();
  void ReplicaDataToHost();
  void MoleculeDataToDevice(int moleculeId);
  void FreeDevice();

  // Kept for interface compatibility: the engine picks its own schedule.
  void setBlockSize(int b) { blockSize = b; }
  int getBlockSize() const { return blockSize; }
  // Replace the 20x20 raw contact table M_ab (host memory, row-major).
  void setLJpotentials(const float* ljp);

  void setBoundingValue(float value) { boundingValue = value; }
  float getBoundingValue() const { return boundingValue; }
  void setTranslateStep(float t) { translateStep = t; }
  void setRotateStep(double r) { rotateStep = r; }
  void setTemperature(float t) { temperature = t; }
  void setLabel(short l) { label = l; }

  // Engine settings with no reference counterpart.
  void setSeed(uint64_t seed) { seed_ = seed; }
  uint64_t getSeed() const { return seed_; }
  void setParams(const remc_params& p);
  const remc_params& getParams() const { return params_; }
  void setCrowderRadius(float r) { crowderRadius_ = r; }
  void setTranslateOnlyCrowders(bool v) { translateOnlyCrowders_ = v; }

  AminoAcids aminoAcids;
  std::vector<Molecule> molecules;
  int moleculeCount = 0;
  int residueCount = 0;
  int maxMoleculeSize = 0;
  int nonCrowderCount = 0;
  float boundingValue = BOUNDING_VALUE;
  float temperature = 300.0f;
  short label = -1;
  double potential = 0.0;
  float translateStep = INITIAL_TRANSLATIONAL_STEP;
  double rotateStep = INITIAL_ROTATIONAL_STEP;
  int blockSize = 32;
  int accept = 0, acceptA = 0, reject = 0;
  int totalAcceptReject = 0, totalAccept = 0;
  int boundSamples = 0, samplesSinceLastExchange = 0;
  int totalBoundSamples = 0, totalSamples = 0;
  bool replicaIsOnDevice = false;

 private:
  friend class ReplicaExchange;
  // engine layout of this replica's topology and state
  void topology(std::vector<int>& mol_start, std::vector<int>& role,
                std::vector<int>& type) const;
  void packState(float* pos, float* rel, float* centre, double* quat) const;
  void unpackState(const float* pos, const float* rel, const float* centre, const double* quat);
  void typeTables(float* vdw, float* charge, float* rho) const;
  bool sameTopology(const Replica& r) const;
  void ensureHandle();

  remc_handle* h_ = nullptr;
  std::vector<int> devMolStart_;  // topology the handle was created for
  float devBox_ = 0.0f;
  uint64_t seed_;
  uint32_t step_ = 0;  // Philox step counter of this replica's stream
  remc_params params_;
  bool paramsSet_ = false;
  bool ljOverride_ = false;
  float lj_[REMC_NUM_AMINO * REMC_NUM_AMINO] = {};
  float crowderRadius_ = 0.0f;
  bool translateOnlyCrowders_ = false;
};

// All replicas of one system advanced together: per block, steps_per_block
// Metropolis steps for every replica, then one neighbour exchange round
// (main.cpp:1378-1487), replayed as a CUDA graph. The replicas must share the
// topology and box and have strictly increasing temperatures in the order
// given; conformations stay with their Replica objects, and exchanges move
// temperature and label between them as Replica::exchangeReplicas does.
class ReplicaExchange {
 public:
  ReplicaExchange(std::vector<Replica*> replicas, uint64_t seed);
  ~ReplicaExchange();
  ReplicaExchange(const ReplicaExchange&) = delete;
  ReplicaExchange& operator=(const ReplicaExchange&) = delete;
  void run(int n_blocks, int steps_per_block);
  // exchange rounds run so far
  int rounds() const { return round_; }
  // Pick threads per replica, shared-memory layout and CTAs per replica by
  // probe sweeps on these replicas (remc_autotune; the state is restored);
  // or set the CTAs per replica directly (1, 2, 4 or 8).
  void autotune(int probe_steps = 256);
  void setCluster(int ctas_per_replica);

 private:
  void upload();
  void download();
  std::vector<Replica*> reps_;
  std::vector<float> ladder_;
  std::vector<short> labelOfTemp_;
  remc_handle* h_ = nullptr;
  uint64_t seed_;
  uint32_t step_ = 0, round_ = 0;
};

}  // namespace remc
