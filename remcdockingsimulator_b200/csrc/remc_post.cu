// Batched post-processing (include/remc_post.h): pose reconstruction of bound
// conformations and DRMS against a reference conformation, one CTA per frame.
//
// Reconstruction follows pdbgen (post processor/pdbgensrc/pdbgen.cpp:166-215)
// in the reference's precisions: the pose quaternion is normalised twice in
// FP64 (pdbgen, then Molecule::setRotation), relative positions are rotated
// by Quaternion::rotateVector (FP64, rounded to FP32), the centre of a shifted
// molecule moves by box * round(v / box) with v its FP32 offset from molecule
// 0's position, and bead = rel + centre in FP32. All with explicit rounding
// intrinsics, so the result is bit-identical to the host arithmetic.
//
// DRMS follows drms.cpp:7-57 (FP32 Vector3f::magnitude of the FP32 difference,
// |d_sim - d_ref| in FP32, summed in FP64); each thread sums the pairs of its
// i beads and the CTA adds the per-thread sums in a fixed order.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "../../include/remc_b200.h"
#include "../../include/remc_post.h"
#include "remc_device.cuh"
#include "remc_internal.h"

using namespace remc;

namespace {

int fail(int code, const char* msg) {
  record_error(msg);
  return code;
}

// Quaternion::normalize (Quaternion.cpp:18-27) in FP64, exact rounding.
__device__ __forceinline__ void normalize_q(double q[4]) {
  const double m = __dsqrt_rn(__dadd_rn(
      __dadd_rn(__dadd_rn(__dmul_rn(q[0], q[0]), __dmul_rn(q[1], q[1])), __dmul_rn(q[2], q[2])),
      __dmul_rn(q[3], q[3])));
  q[0] = __ddiv_rn(q[0], m);
  q[1] = __ddiv_rn(q[1], m);
  q[2] = __ddiv_rn(q[2], m);
  q[3] = __ddiv_rn(q[3], m);
}

// The image of c nearest p: c - box * round((c - p) / box), per axis in FP32
// (pdbgen.cpp:196-203, round half away from zero).
__device__ __forceinline__ float3 nearest_image(float3 c, float3 p, float box) {
  const float vx = __fsub_rn(c.x, p.x), vy = __fsub_rn(c.y, p.y), vz = __fsub_rn(c.z, p.z);
  return make_float3(__fsub_rn(c.x, __fmul_rn(box, roundf(__fdiv_rn(vx, box)))),
                     __fsub_rn(c.y, __fmul_rn(box, roundf(__fdiv_rn(vy, box)))),
                     __fsub_rn(c.z, __fmul_rn(box, roundf(__fdiv_rn(vz, box)))));
}

__global__ void rebuild_kernel(const float* __restrict__ rel0, const int* __restrict__ ms,
                               int n_mol, const int* __restrict__ shift, float3 centre0,
                               float box, const double* __restrict__ quat,
                               const float* __restrict__ centre, int n_beads,
                               float* __restrict__ pos, float* __restrict__ centre_out) {
  const int f = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const float* cf = centre + (size_t)f * n_mol * 3;
  const double* qf = quat + (size_t)f * n_mol * 4;
  // molecule 0's position after its own shift (every warp derives it)
  float3 p0 = make_float3(cf[0], cf[1], cf[2]);
  if (shift[0]) p0 = nearest_image(p0, centre0, box);
  for (int m = warp; m < n_mol; m += nw) {
    double q[4] = {qf[4 * m], qf[4 * m + 1], qf[4 * m + 2], qf[4 * m + 3]};
    normalize_q(q);  // pdbgen.cpp:191
    normalize_q(q);  // Molecule::setRotation
    const QuatProducts qp = quat_products(q[0], q[1], q[2], q[3]);
    float3 c = make_float3(cf[3 * m], cf[3 * m + 1], cf[3 * m + 2]);
    if (m == 0)
      c = p0;
    else if (shift[m])
      c = nearest_image(c, p0, box);
    if (centre_out && lane == 0) {
      float* o = centre_out + ((size_t)f * n_mol + m) * 3;
      o[0] = c.x;
      o[1] = c.y;
      o[2] = c.z;
    }
    for (int b = ms[m] + lane; b < ms[m + 1]; b += 32) {
      const float3 r = rotate_rel(qp, rel0[3 * b], rel0[3 * b + 1], rel0[3 * b + 2]);
      float* o = pos + ((size_t)f * n_beads + b) * 3;
      o[0] = __fadd_rn(r.x, c.x);
      o[1] = __fadd_rn(r.y, c.y);
      o[2] = __fadd_rn(r.z, c.z);
    }
  }
}

// |a - b| as Vector3f::magnitude computes it: FP32 squares summed left to
// right, FP32 square root.
__device__ __forceinline__ float dist3(const float* a, const float* b) {
  const float dx = __fsub_rn(a[0], b[0]), dy = __fsub_rn(a[1], b[1]), dz = __fsub_rn(a[2], b[2]);
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
}

constexpr int kDrmsThreads = 256;

__global__ void __launch_bounds__(kDrmsThreads) drms_kernel(
    const float* __restrict__ frames, const float* __restrict__ ref, const int* __restrict__ ms,
    const int* __restrict__ mol_of, int n_mol, int n_beads, int reverse, float native_cut,
    float recovered_cut, double* __restrict__ drms, double* __restrict__ drms_rev,
    unsigned long long* __restrict__ counts) {
  __shared__ double s_a[kDrmsThreads], s_b[kDrmsThreads];
  __shared__ unsigned long long s_c[3][kDrmsThreads];
  const int f = blockIdx.x, tid = threadIdx.x;
  const float* x = frames + (size_t)f * n_beads * 3;
  double sa = 0.0, sb = 0.0;
  unsigned long long cn = 0, cr = 0, cb = 0;
  for (int i = tid; i < n_beads; i += kDrmsThreads) {
    const int I = mol_of[i], li = i - ms[I];
    for (int j = ms[I + 1]; j < n_beads; ++j) {  // beads of molecules J > I
      const float ds = dist3(x + 3 * i, x + 3 * j);
      const float de = dist3(ref + 3 * i, ref + 3 * j);
      sa += (double)fabsf(__fsub_rn(ds, de));
      cn += de < native_cut ? 1ull : 0ull;
      cr += (de < native_cut && ds < recovered_cut) ? 1ull : 0ull;
      cb += ds < native_cut ? 1ull : 0ull;
      if (reverse) {
        // drms.cpp:45-46: the reference's molecules I and J swapped
        const int J = mol_of[j], lj = j - ms[J];
        const float dr = dist3(ref + 3 * (ms[J] + li), ref + 3 * (ms[I] + lj));
        sb += (double)fabsf(__fsub_rn(ds, dr));
      }
    }
  }
  s_a[tid] = sa;
  s_b[tid] = sb;
  s_c[0][tid] = cn;
  s_c[1][tid] = cr;
  s_c[2][tid] = cb;
  __syncthreads();
  if (tid == 0) {
    double a = 0.0, b = 0.0;
    unsigned long long c[3] = {0, 0, 0};
    for (int t = 0; t < kDrmsThreads; ++t) {
      a += s_a[t];
      b += s_b[t];
      for (int k = 0; k < 3; ++k) c[k] += s_c[k][t];
    }
    drms[f] = a;
    drms_rev[f] = b;
    for (int k = 0; k < 3; ++k) counts[3 * f + k] = c[k];
  }
}

template <class T>
int to_device(T** d, const T* h, size_t n) {
  if (cudaMalloc((void**)d, sizeof(T) * (n ? n : 1)) != cudaSuccess)
    return fail(REMC_ERR_NOMEM, "post: device allocation failed");
  if (n && cudaMemcpy(*d, h, sizeof(T) * n, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(REMC_ERR_CUDA, "post: host to device copy failed");
  return REMC_OK;
}

struct DevBufs {
  std::vector<void*> p;
  ~DevBufs() {
    for (void* q : p) cudaFree(q);
  }
  template <class T>
  int up(T** d, const T* h, size_t n) {
    *d = nullptr;
    int rc = to_device(d, h, n);
    if (*d) p.push_back(*d);
    return rc;
  }
  template <class T>
  int alloc(T** d, size_t n) {
    *d = nullptr;
    if (cudaMalloc((void**)d, sizeof(T) * (n ? n : 1)) != cudaSuccess)
      return fail(REMC_ERR_NOMEM, "post: device allocation failed");
    p.push_back(*d);
    return REMC_OK;
  }
};

int check_starts(const int* mol_start, int n_mol) {
  if (!mol_start || n_mol <= 0 || mol_start[0] != 0)
    return fail(REMC_ERR_INVALID, "post: mol_start must start at 0");
  for (int m = 0; m < n_mol; ++m)
    if (mol_start[m + 1] <= mol_start[m])
      return fail(REMC_ERR_INVALID, "post: every molecule needs at least one bead");
  return REMC_OK;
}

}  // namespace

extern "C" {

int remc_post_rebuild(const float* rel0, const int* mol_start, int n_mol, const int* shift,
                      const float* centre0, float box, const double* quat, const float* centre,
                      int n_frames, float* pos, float* centre_out) {
  int rc = check_starts(mol_start, n_mol);
  if (rc) return rc;
  if (!rel0 || !shift || !centre0 || !quat || !centre || !pos || n_frames < 0)
    return fail(REMC_ERR_INVALID, "post_rebuild: null argument");
  if (!(box > 0.0f) || !std::isfinite(box)) return fail(REMC_ERR_INVALID, "post_rebuild: bad box");
  if (n_frames == 0) return REMC_OK;
  const int nb = mol_start[n_mol];
  DevBufs B;
  float *d_rel, *d_cen, *d_pos, *d_cout = nullptr;
  int *d_ms, *d_shift;
  double* d_q;
  if ((rc = B.up(&d_rel, rel0, 3 * (size_t)nb)) || (rc = B.up(&d_ms, mol_start, n_mol + 1)) ||
      (rc = B.up(&d_shift, shift, n_mol)) || (rc = B.up(&d_q, quat, 4 * (size_t)n_mol * n_frames)) ||
      (rc = B.up(&d_cen, centre, 3 * (size_t)n_mol * n_frames)) ||
      (rc = B.alloc(&d_pos, 3 * (size_t)nb * n_frames)))
    return rc;
  if (centre_out && (rc = B.alloc(&d_cout, 3 * (size_t)n_mol * n_frames))) return rc;
  rebuild_kernel<<<n_frames, 256>>>(d_rel, d_ms, n_mol, d_shift,
                                    make_float3(centre0[0], centre0[1], centre0[2]), box, d_q,
                                    d_cen, nb, d_pos, d_cout);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpy(pos, d_pos, sizeof(float) * 3 * (size_t)nb * n_frames, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && centre_out)
    e = cudaMemcpy(centre_out, d_cout, sizeof(float) * 3 * (size_t)n_mol * n_frames,
                   cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    char msg[256];
    snprintf(msg, sizeof(msg), "post_rebuild: %s", cudaGetErrorString(e));
    return fail(REMC_ERR_CUDA, msg);
  }
  return REMC_OK;
}

int remc_post_drms(const float* frames, int n_frames, const float* ref, const int* mol_start,
                   int n_mol, int reverse, float native_cut, float recovered_cut, double* drms,
                   long long* native, long long* recovered, long long* binding) {
  int rc = check_starts(mol_start, n_mol);
  if (rc) return rc;
  if (!frames || !ref || !drms || n_frames < 0) return fail(REMC_ERR_INVALID, "post_drms: null argument");
  if (n_mol < 2) return fail(REMC_ERR_INVALID, "post_drms: needs at least two molecules");
  if (reverse)
    for (int m = 1; m < n_mol; ++m)
      if (mol_start[m + 1] - mol_start[m] != mol_start[1] - mol_start[0])
        return fail(REMC_ERR_INVALID, "post_drms: reverse order needs molecules of equal length");
  if (n_frames == 0) return REMC_OK;
  const int nb = mol_start[n_mol];
  std::vector<int> mol_of(nb);
  double n_pairs = 0.0;
  for (int m = 0; m < n_mol; ++m) {
    for (int b = mol_start[m]; b < mol_start[m + 1]; ++b) mol_of[b] = m;
    n_pairs += (double)(mol_start[m + 1] - mol_start[m]) * (double)(nb - mol_start[m + 1]);
  }
  DevBufs B;
  float *d_x, *d_ref;
  int *d_ms, *d_mol;
  double *d_a, *d_b;
  unsigned long long* d_c;
  if ((rc = B.up(&d_x, frames, 3 * (size_t)nb * n_frames)) || (rc = B.up(&d_ref, ref, 3 * (size_t)nb)) ||
      (rc = B.up(&d_ms, mol_start, n_mol + 1)) || (rc = B.up(&d_mol, mol_of.data(), (size_t)nb)) ||
      (rc = B.alloc(&d_a, n_frames)) || (rc = B.alloc(&d_b, n_frames)) ||
      (rc = B.alloc(&d_c, 3 * (size_t)n_frames)))
    return rc;
  drms_kernel<<<n_frames, kDrmsThreads>>>(d_x, d_ref, d_ms, d_mol, n_mol, nb, reverse ? 1 : 0,
                                          native_cut, recovered_cut, d_a, d_b, d_c);
  std::vector<double> a(n_frames), b(n_frames);
  std::vector<unsigned long long> c(3 * (size_t)n_frames);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(a.data(), d_a, sizeof(double) * n_frames, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(b.data(), d_b, sizeof(double) * n_frames, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemcpy(c.data(), d_c, sizeof(unsigned long long) * c.size(), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    char msg[256];
    snprintf(msg, sizeof(msg), "post_drms: %s", cudaGetErrorString(e));
    return fail(REMC_ERR_CUDA, msg);
  }
  for (int f = 0; f < n_frames; ++f) {
    // drms.cpp:32 and :52: drms /= N; reverse: min(drms, drms2 / N)
    double d = a[f] / n_pairs;
    if (reverse) d = std::min(d, b[f] / n_pairs);
    drms[f] = d;
    if (native) native[f] = (long long)c[3 * f];
    if (recovered) recovered[f] = (long long)c[3 * f + 1];
    if (binding) binding[f] = (long long)c[3 * f + 2];
  }
  return REMC_OK;
}

}  // extern "C"
