/* remc_reference_abi.h - drop-in replacements for the reference's CUDA C ABI.
 *
 * The reference (iantunbridge/RemcDockingSimulator) calls its GPU energy
 * through the extern "C" functions of simulation engine/src/cudaExterns.h.
 * This header declares the same entry points, implemented by B200 kernels in
 * libremc_b200.so, so the reference's Replica::EonDevice / EonDeviceAsync /
 * ReplicaDataToDevice path can link against this library unchanged apart from
 * one type: copyLJPotentialDataToDevice and LJPotentialDataToDevice take the
 * 20x20 contact table as a plain float array (the memory of
 * AminoAcids::LJpotentials) instead of an AminoAcids*.
 *
 * Data layout (the reference's own, Replica.cpp:1308-1417):
 *   residuePositions[i] = (x, y, z, molecule index as float); padding beads
 *                         have w = -2 (PADDER_IDENTIFIER)
 *   residueMeta[i]      = (residue type as float, charge, vdW radius,
 *                          molecule role: -1 crowder, 0 otherwise)
 *   LJPotentials        = device pointer to the raw 20x20 table M_ab
 *                         (eps_ab = lambda (M_ab - e0), definitions.h:33-35)
 *   datasetSize         = bead count padded to a multiple of blockSize
 * Energies are kcal/mol, computed as Replica::E() (Replica.cpp:603-745) with
 * FP32 pair terms and FP64 sums. The reference's void signatures are kept;
 * remc_reference_abi_status() returns the last call's status (REMC_OK or a
 * negative REMC_ERR_* code) and remc_last_error_string() its message.
 */
#ifndef REMC_REFERENCE_ABI_H
#define REMC_REFERENCE_ABI_H

#include <cuda_runtime.h>

#include "remc_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* cudaExterns.h:13 - returns a new device copy of the 20x20 table. */
float* LJPotentialDataToDevice(const float* lj_table_20x20);
/* cudaExterns.h:14 - copies the table into caller-allocated device memory. */
void copyLJPotentialDataToDevice(float* dev_LJPotentialData, const float* lj_table_20x20);

/* cudaExterns.h:16 - the reference's body only prints; kept as a no-op. */
void MCSearchOnDevice(void);

/* cudaExterns.h:19-20 - rigid moves of one molecule in device memory:
 * rotation by axis (x,y,z) and angle w about *d_center, translation by
 * (x,y,z) also moving *d_center (CudaFunctions.cu:798-862). */
void CUDA_rotateMolecule(float4* d_residuePositions, int* d_startPosition, int* d_moleculeLength,
                         int moleculeLength, float4* d_rotationVector, float4* d_center,
                         cudaStream_t stream);
void CUDA_translateMolecule(float4* d_residuePositions, int* d_startPosition,
                            int* d_moleculeLength, int moleculeLength, float4* d_translation,
                            float4* d_center, cudaStream_t stream);

/* cudaExterns.h:23 - full-system energy into *result (host), synchronous.
 * residueCount, moleculePositions, moleculeCount, blockSize and
 * sharedMemSize are accepted for compatibility; datasetSize beads are read.
 * Runs on the legacy default stream. Safe to call from several host threads
 * at once: the calls take turns on their shared partial-sum buffer. */
void CUDA_EonDevice(float4* residuePositions, float4* residueMeta, int* residueCount,
                    int* moleculePositions, int* moleculeCount, float* LJPotentials,
                    double* result, int blockSize, int datasetSize, int sharedMemSize);

/* cudaExterns.h:27-30 - host <-> device copies; return 0 or a CUDA error. */
int CUDA_memcpy_to_device(void* destination, void* source, int mem_size);
int CUDA_memcpy_to_host(void* destination, void* source, int mem_size);
int CUDA_memcpy_to_device_async(void* destination, void* source, int mem_size,
                                cudaStream_t stream);
int CUDA_memcpy_to_host_async(void* destination, void* source, int mem_size,
                              cudaStream_t stream);

/* cudaExterns.h:35 - energy on `stream`. The reference leaves one float per
 * block in device_result (resultSize x resultSize) for the host to sum and
 * scale by KBTConversionFactor (Replica::SumGridResults, Replica.cpp:1195-1216);
 * here device_result[0] holds the whole sum in those units and the other
 * entries are zero, so the same host summation gives the energy.
 * Each (device, stream) has its own partial-sum buffer, kept until exit and
 * grown only after the stream's queued work has finished: energies queued on
 * different streams (the reference gives every replica thread its own,
 * main.cpp:924-954) may run concurrently, from any host threads. */
void CUDA_EonDevice_async(float4* residuePositions, float4* residueMeta, int* residueCount,
                          int* moleculePositions, int* moleculeCount, float* LJPotentials,
                          float* device_result, int resultSize, int blockSize, int datasetSize,
                          int sharedMemSize, cudaStream_t stream);
/* cudaExterns.h:36 - a no-op in the reference; kept as one. */
void CUDA_Esum_async(float* result, float* d_resultMatrix, int resultSize, int datasetSize,
                     cudaStream_t stream);

/* cudaExterns.h:38 - prints the CUDA error string of `code`. */
void printCudaError(int code);
/* cudaExterns.h:21 - prints the visible devices. */
void cudaInfo(void);

/* cudaExterns.h:40-41 - periodic box edge used by the energy calls. */
void CUDA_setBoxDimension(float value);
void CUDA_freeBoxDimension(void);

/* cudaExterns.h:44-45 - the reference binds the table to a texture; here the
 * pointer is recorded and used when a call passes LJPotentials = NULL. */
void bindLJTexture(float* ljp);
void unbindLJTexture(void);

/* Allocation-free variant of CUDA_EonDevice. No counterpart in the reference:
 * the reference's CUDA_EonDevice allocates and frees its partial sums on every
 * call. This entry point allocates nothing, for callers that cannot call
 * cudaMalloc: hosts whose device memory is owned by another allocator (a
 * framework's caching arena that has reserved the GPU), and loops that cannot
 * afford cudaMalloc/cudaFree's implicit device synchronisation on every Monte
 * Carlo step. The caller passes device inputs (same layout as CUDA_EonDevice)
 * and a device pointer for the result (one double, kcal/mol); the work is
 * ordered on `stream` and the call does not wait for it. The partial sums live
 * in one fixed device array of REMC_NOALLOC_MAX_ITEMS doubles (256 KiB) that
 * every GPU loading this library holds until the process exits, so
 * datasetSize is limited to REMC_NOALLOC_MAX_BEADS beads; larger sizes return
 * REMC_ERR_INVALID with a message. The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress) and should come before any
 * stream capture on that device. All calls share the array and each call
 * overwrites every partial it reads, so nothing needs clearing between calls;
 * calls that overlap on the GPU (different streams, or different host threads
 * on one device) race on it. Returns REMC_OK or a negative REMC_ERR_* code. */
#define REMC_NOALLOC_MAX_ITEMS 32768
#define REMC_NOALLOC_MAX_BEADS 32640
int CUDA_EonDevice_noalloc(const float4* residuePositions, const float4* residueMeta,
                           const float* LJPotentials, int datasetSize, double* d_result,
                           cudaStream_t stream);

/* The device buffers and addresses the calls above keep per device are not
 * renewed after cudaDeviceReset: do not reset a device while this library
 * uses it. */

/* Energy-model constants used by the calls above (default: the reference's
 * compile-time values, remc_default_params). No reference counterpart. */
int remc_reference_abi_set_params(const remc_params* params);
/* Status of the last call above (REMC_OK or REMC_ERR_*). No reference
 * counterpart: the reference's functions return void and abort on error. */
int remc_reference_abi_status(void);

#ifdef __cplusplus
}
#endif
#endif
