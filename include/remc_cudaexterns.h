/* remc_cudaexterns.h - builds the reference's own GPU code against this
 * library without editing it.
 *
 * The reference's host code (simulation engine/src/Replica.{h,cpp}, main.cpp)
 * declares its GPU entry points in cudaExterns.h and implements them in
 * CudaFunctions.cu, which CUDA 12 no longer compiles (texture references,
 * string-named symbols, cutil). Force-include this header when compiling the
 * reference's sources with -DEnableCUDA:
 *
 *     g++ -DEnableCUDA -include remc_cudaexterns.h -I<this include dir> ...
 *
 * It takes cudaExterns.h's include guard, so the reference's own
 * `#include "cudaExterns.h"` (Replica.h:25, main.cpp:20,29) adds nothing, and
 * it declares the same entry points from remc_reference_abi.h, implemented in
 * libremc_b200.so. The reference passes its AminoAcids object to the two
 * table calls (main.cpp:916,1661,1763, Replica.cpp:1100); the C++ overloads
 * below pass that object's 20x20 table, which is what the library reads, so
 * those call sites compile unchanged. Link with -lremc_b200 -lcudart in place
 * of CudaFunctions.o and -lcutil.
 */
#ifndef CUDAEXTERNS_H_
#define CUDAEXTERNS_H_

#include "remc_reference_abi.h"

#ifdef __cplusplus
#include "AminoAcids.h" /* the reference's class (AminoAcids.h:13: LJpotentials[20][20]) */

inline float* LJPotentialDataToDevice(AminoAcids* a) {
  return LJPotentialDataToDevice(&a->LJpotentials[0][0]);
}
inline void copyLJPotentialDataToDevice(float* dev_LJPotentialData, AminoAcids* a) {
  copyLJPotentialDataToDevice(dev_LJPotentialData, &a->LJpotentials[0][0]);
}
#endif

#endif /* CUDAEXTERNS_H_ */
