// The reference's -c check (simulation engine/src/main.cpp:1652-1707) around
// its own Replica code, built with -DEnableCUDA against libremc_b200.so by
// oracle/build.py (TEST INFRASTRUCTURE).
//
// For the ten docked structures data/conf{1..10}/1{a,b}.pdb in the check's
// 118.4 A box it prints the reference's own Replica::E() on the CPU and
// Replica::EonDevice() (Replica.cpp:1601-1616: ReplicaDataToDevice, then
// CUDA_EonDevice, here the B200 kernel) as "CPU,GPU,err", as the check does.
// One step differs from main.cpp's check: each Replica reserves its molecule
// array (Replica::reserveConiguousMoleculeArray) before loading, as the
// start-up path does (main.cpp:1716). The check's stack Replicas leave the
// array pointer uninitialised (the constructor, Replica.cpp:9-40, never sets
// it), and Replica::loadMolecule deletes it (Replica.cpp:229-245), so the
// reference's own -c run crashes there.
#include <cmath>
#include <cstdio>

#include "Replica.h"

int main() {
  AminoAcids aa;
  aa.loadAminoAcidData(AMINOACIDDATASOURCE);
  aa.loadLJPotentialData(LJPDSOURCE);
  cuInit(0);
  float* ljp = nullptr;
  if (cudaMalloc((void**)&ljp, LJArraySize) != cudaSuccess) {
    printf("cudaMalloc failed\n");
    return 1;
  }
  copyLJPotentialDataToDevice(ljp, &aa);
  const float box = 118.4f;
  CUDA_setBoxDimension(box);
  bindLJTexture(ljp);
  char name[64];
  for (int i = 1; i <= 10; i++) {
    Replica r;
    r.aminoAcids = aa;
    r.label = i;
    r.setBoundingValue(box);
    r.reserveConiguousMoleculeArray(2);
    snprintf(name, sizeof(name), "data/conf%d/1a.pdb", i);
    r.loadMolecule(name);
    snprintf(name, sizeof(name), "data/conf%d/1b.pdb", i);
    r.loadMolecule(name);
    r.initTimers();
    r.E();
    r.setDeviceLJPotentials(ljp);
    r.setBlockSize(TILE_DIM);
    r.ReplicaDataToDevice();
    const double gpu = r.EonDevice();
    const double cpu = r.E();
    printf("CPU,GPU,err: %24.20f %24.20f %24.20f\n", cpu, gpu, std::fabs(cpu - gpu));
    r.FreeDevice();
  }
  unbindLJTexture();
  cudaFree(ljp);
  return remc_reference_abi_status() == 0 ? 0 : 2;
}
