// remc_replica_check - command-line driver of the C++ facade, used by the
// tests to compare the facade with the Python engine and the oracle.
//
//   remc_replica_check moves  <AminoAcids> <pairs> <pdb>
//   remc_replica_check energy <AminoAcids> <pairs> <box> <pdb|c:pdb>...
//   remc_replica_check mc     <AminoAcids> <pairs> <box> <T> <steps> <seed> <out> <pdb|c:pdb>...
//   remc_replica_check remc   <AminoAcids> <pairs> <box> <R> <Tmin> <Tmax> <blocks> <steps>
//                             <seed> <out> <pdb|c:pdb>...
//
// A "c:" prefix loads the PDB as a crowder. Results go to stdout (one value per
// line, %.9g for floats, %.17g for doubles) and state to <out> as text.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "remc_replica.h"

using namespace remc;

namespace {

void load_tables(AminoAcids& aa, const char* amino, const char* pairs) {
  if (!aa.loadAminoAcidData(amino)) throw Error(std::string("cannot read ") + amino);
  if (!aa.loadLJPotentialData(pairs)) throw Error(std::string("cannot read ") + pairs);
}

void load_molecules(Replica& r, int argc, char** argv, int first) {
  for (int i = first; i < argc; ++i) {
    const bool crowder = std::strncmp(argv[i], "c:", 2) == 0;
    const int m = r.loadMolecule(crowder ? argv[i] + 2 : argv[i]);
    if (crowder) r.molecules[m].setMoleculeRoleIdentifier(CROWDER_IDENTIFIER);
  }
}

void print_molecule(const Molecule& m) {
  std::printf("centre %.9g %.9g %.9g\n", m.center.x, m.center.y, m.center.z);
  std::printf("quat %.17g %.17g %.17g %.17g\n", m.rotation.w, m.rotation.x, m.rotation.y,
              m.rotation.z);
  for (const Residue& r : m.Residues)
    std::printf("bead %d %.9g %.9g %.9g %.9g %.9g %.9g\n", r.aminoAcidIndex, r.position.x,
                r.position.y, r.position.z, r.relativePosition.x, r.relativePosition.y,
                r.relativePosition.z);
}

void write_state(const char* path, const std::vector<Replica*>& reps) {
  FILE* f = std::fopen(path, "w");
  if (!f) throw Error(std::string("cannot write ") + path);
  for (const Replica* r : reps) {
    std::fprintf(f, "replica %d %.9g %.17g %d %d %d\n", (int)r->label, r->temperature,
                 r->potential, r->accept, r->acceptA, r->reject);
    for (const Molecule& m : r->molecules) {
      std::fprintf(f, "mol %.9g %.9g %.9g %.17g %.17g %.17g %.17g\n", m.center.x, m.center.y,
                   m.center.z, m.rotation.w, m.rotation.x, m.rotation.y, m.rotation.z);
      for (const Residue& b : m.Residues)
        std::fprintf(f, "bead %.9g %.9g %.9g\n", b.position.x, b.position.y, b.position.z);
    }
  }
  std::fclose(f);
}

int moves(int argc, char** argv) {
  if (argc < 5) return 2;
  AminoAcids aa;
  load_tables(aa, argv[2], argv[3]);
  Molecule m;
  m.AminoAcidsData = aa;
  if (!m.initFromPDB(argv[4])) throw Error("cannot read pdb");
  print_molecule(m);
  Molecule saved;
  saved.saveBeforeStateChange(&m);
  m.translate(Vector3f(1.25f, -0.5f, 3.0f));
  print_molecule(m);
  m.setPosition(Vector3f(10.0f, 20.0f, 30.0f));
  print_molecule(m);
  Vector3double ax(0.3, -0.4, 0.5);
  ax.normalizeInPlace();
  m.rotateQ(ax, 0.7);
  print_molecule(m);
  m.undoStateChange(&saved);
  print_molecule(m);
  return 0;
}

int energy(int argc, char** argv) {
  if (argc < 6) return 2;
  Replica r;
  load_tables(r.aminoAcids, argv[2], argv[3]);
  r.setBoundingValue(std::strtof(argv[4], nullptr));
  load_molecules(r, argc, argv, 5);
  std::printf("%.17g\n", r.E());
  std::printf("%.17g\n", r.EonDevice());
  return 0;
}

int mc(int argc, char** argv) {
  if (argc < 10) return 2;
  Replica r;
  load_tables(r.aminoAcids, argv[2], argv[3]);
  r.setBoundingValue(std::strtof(argv[4], nullptr));
  r.setTemperature(std::strtof(argv[5], nullptr));
  const int steps = std::atoi(argv[6]);
  r.setSeed(std::strtoull(argv[7], nullptr, 10));
  load_molecules(r, argc, argv, 9);
  r.potential = r.E();
  std::printf("%.17g\n", r.potential);
  // two calls continue one stream: steps/2 + (steps - steps/2)
  r.MCSearch(steps / 2);
  r.MCSearch(steps - steps / 2);
  std::printf("%.17g\n%d %d %d\n", r.potential, r.accept, r.acceptA, r.reject);
  write_state(argv[8], {&r});
  return 0;
}

int remc_cmd(int argc, char** argv) {
  if (argc < 13) return 2;
  const int R = std::atoi(argv[5]);
  const float tmin = std::strtof(argv[6], nullptr), tmax = std::strtof(argv[7], nullptr);
  const int blocks = std::atoi(argv[8]), steps = std::atoi(argv[9]);
  const uint64_t seed = std::strtoull(argv[10], nullptr, 10);
  std::vector<Replica> reps(R);
  // geometric ladder of REMCSimulation (main.cpp:1161-1169)
  const double g = R > 1 ? std::pow(double(tmax / tmin), 1.0 / double(R - 1)) : 1.0;
  for (int k = 0; k < R; ++k) {
    load_tables(reps[k].aminoAcids, argv[2], argv[3]);
    reps[k].setBoundingValue(std::strtof(argv[4], nullptr));
    load_molecules(reps[k], argc, argv, 12);
    reps[k].setTemperature(float(double(tmin) * std::pow(g, k)));
    reps[k].setLabel((short)k);
  }
  std::vector<Replica*> ptr;
  for (Replica& r : reps) ptr.push_back(&r);
  ReplicaExchange ex(ptr, seed);
  // REMC_CHECK_CLUSTER=c runs the replicas on clusters of c CTAs
  if (const char* c = std::getenv("REMC_CHECK_CLUSTER")) ex.setCluster(std::atoi(c));
  ex.run(blocks, steps);
  for (Replica* r : ptr) std::printf("%d %.9g %.17g\n", (int)r->label, r->temperature, r->potential);
  write_state(argv[11], ptr);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: remc_replica_check moves|energy|mc|remc ...\n");
    return 2;
  }
  try {
    const std::string cmd = argv[1];
    if (cmd == "moves") return moves(argc, argv);
    if (cmd == "energy") return energy(argc, argv);
    if (cmd == "mc") return mc(argc, argv);
    if (cmd == "remc") return remc_cmd(argc, argv);
  } catch (const Error& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 2;
}
