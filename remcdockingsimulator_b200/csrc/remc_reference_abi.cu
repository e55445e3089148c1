// Drop-in replacements for the reference's CUDA C ABI (include/remc_reference_abi.h),
// in the reference's own device data layout.
//
// Energy: tiled upper-triangle pair sum. A persistent grid walks the
// (i-tile, j-tile >= i-tile) items of 128 beads; each CTA stages the j-tile
// (positions + metadata) in shared memory, each thread keeps one i bead in
// registers, pair terms are FP32 (MUFU rsqrt/ex2) and each item's sum goes to
// a per-item FP64 partial; a second kernel adds the partials in a fixed order
// (deterministic result). Follows Replica::E (Replica.cpp:603-745) and the
// reference kernel's masking rules (CudaFunctions.cu:483-548): padding beads
// have position w < 0, beads of the same molecule share w, a pair involving a
// crowder (metadata w = -1) is (6/r)^6 inside 15 A.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>

#include "../../include/remc_reference_abi.h"
#include "remc_device.cuh"
#include "remc_internal.h"

using namespace remc;

namespace {

constexpr int kRefTile = 128;
constexpr int kMaxDevices = 64;

struct RefConsts {
  float lambda_, e0, c_xi;
  float lj_scale, dh_scale;  // LJ_CF * KBT_CF, DH constant * KBT_CF
  float box, invbox;
  float cutoff2;             // crowder cutoff squared (inf: none)
};

thread_local int g_status = REMC_OK;
std::mutex g_mutex;
float g_box = 150.0f;  // BOUNDING_VALUE until CUDA_setBoxDimension (definitions.h:68)
float* g_bound_table = nullptr;
bool g_params_set = false;
remc_params g_params;

// Scratch for the per-item partials of the allocating energy calls, one
// buffer per (device, stream). A call holds its buffer's lock from the
// lookup until its last launch (and, on the synchronous path, its result
// copy) is enqueued, so calls on one stream take their turns in stream order,
// and calls on different streams or host threads never share partials.
struct ScratchSlot {
  std::mutex mu;
  double* ptr = nullptr;
  size_t cap = 0;
};
std::mutex g_slots_mutex;
std::map<std::pair<int, cudaStream_t>, std::unique_ptr<ScratchSlot>> g_slots;

void set_status(int code, const char* what, cudaError_t e = cudaSuccess) {
  g_status = code;
  if (code != REMC_OK) {
    char buf[256];
    snprintf(buf, sizeof(buf), "%s%s%s", what, e != cudaSuccess ? ": " : "",
             e != cudaSuccess ? cudaGetErrorString(e) : "");
    record_error(buf);
  }
}

RefConsts make_consts(float* unscale = nullptr) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_params_set) {
    remc_default_params(&g_params);
    g_params_set = true;
  }
  if (unscale) *unscale = 1.0f / (float)((double)g_params.kbt_cf);
  RefConsts C;
  C.lambda_ = g_params.lambda_;
  C.e0 = g_params.e0;
  C.c_xi = (float)(-1.4426950408889634 / (double)g_params.debye_length);
  C.lj_scale = (float)((double)g_params.lj_cf * (double)g_params.kbt_cf);
  C.dh_scale = (float)((double)g_params.dh_const * (double)g_params.kbt_cf);
  C.box = g_box;
  C.invbox = 1.0f / g_box;
  C.cutoff2 = g_params.crowder_cutoff > 0.0f ? g_params.crowder_cutoff * g_params.crowder_cutoff
                                             : INFINITY;
  return C;
}

// Triangle index of item (ti, tj), tj >= ti, of T tiles.
__host__ __device__ __forceinline__ int tri_index(int ti, int tj, int T) {
  return ti * T - (ti * (ti - 1)) / 2 + (tj - ti);
}

__global__ void __launch_bounds__(kRefTile) ref_energy_tiles(
    const float4* __restrict__ pos, const float4* __restrict__ meta,
    const float* __restrict__ lj_table, int P, int T, double* __restrict__ partials, RefConsts C) {
  __shared__ float s_M[400];
  __shared__ float4 s_jp[kRefTile];
  __shared__ float4 s_jm[kRefTile];
  __shared__ double s_red[kRefTile / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < 400; i += kRefTile) s_M[i] = lj_table[i];
  const float two_third = 1.2599210498948732f;  // 2^(1/3)
  for (int item = blockIdx.x; item < T * T; item += gridDim.x) {
    const int ti = item / T, tj = item % T;
    if (tj < ti) continue;
    __syncthreads();  // the previous item is done with the j-tile
    const int j0 = tj * kRefTile;
    const int jn = min(kRefTile, P - j0);
    if (tid < jn) {
      s_jp[tid] = pos[j0 + tid];
      s_jm[tid] = meta[j0 + tid];
    }
    __syncthreads();
    const int i = ti * kRefTile + tid;
    float lj = 0.0f, dh = 0.0f;
    if (i < P) {
      const float4 pi = pos[i], mi = meta[i];
      if (pi.w > -2.0f) {  // not a padding bead
        const bool icrowd = mi.w == -1.0f;
        const int jstart = (ti == tj) ? tid + 1 : 0;
        for (int jj = jstart; jj < jn; ++jj) {
          const float4 pj = s_jp[jj];
          if (pj.w < 0.0f || pj.w == pi.w) continue;  // padding or same molecule
          const float4 mj = s_jm[jj];
          const float r2 = pair_r2(pi, pj, C.box, C.invbox);
          const float rinv = fast_rsqrt(r2);
          const float rinv2 = rinv * rinv;
          if (icrowd || mj.w == -1.0f) {
            const float i6 = rinv2 * rinv2 * rinv2;
            if (r2 < C.cutoff2) lj += 46656.0f * i6;  // (6/r)^6
          } else {
            int idx = __float2int_rn(20.0f * mi.x + mj.x);
            idx = min(max(idx, 0), 399);
            const float eps = C.lambda_ * (s_M[idx] - C.e0);
            const float sig = (mi.z + mj.z) * 0.5f;
            const float sig2 = sig * sig;
            const float s2 = sig2 * rinv2;
            const float s6 = s2 * s2 * s2;
            float L = 4.0f * eps * fmaf(-s6, s6, s6);
            if (eps > 0.0f && r2 < sig2 * two_third) L = 2.0f * eps - L;
            lj += L;
            const float r = r2 * rinv;
            dh += mi.y * mj.y * fast_ex2(r * C.c_xi) * rinv;
          }
        }
      }
    }
    double v = (double)lj * (double)C.lj_scale + (double)dh * (double)C.dh_scale;
    v = warp_sum(v);
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < kRefTile / 32; ++w) t += s_red[w];
      partials[tri_index(ti, tj, T)] = t;
    }
  }
}

// Fixed-order sum of n partials into *out (one CTA).
__global__ void ref_energy_sum(const double* __restrict__ partials, int n, double* __restrict__ out,
                               float* __restrict__ grid_out, int grid_n, float unscale) {
  __shared__ double s[256];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += partials[i];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0 && out) *out = s[0];
  if (grid_out) {
    // the reference's per-block layout: the host sums it and scales by KBT_CF
    for (int i = threadIdx.x; i < grid_n; i += blockDim.x)
      grid_out[i] = (i == 0) ? (float)(s[0] * (double)unscale) : 0.0f;
  }
}

__global__ void rotate_molecule_kernel(float4* pos, const int* start, const int* length,
                                       const float4* rv, const float4* center) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= *length) return;
  const float4 r = *rv;
  const float4 c = *center;
  // unit quaternion of the axis-angle (CudaFunctions.cu:798-840)
  float qw = cosf(r.w * 0.5f), sh = sinf(r.w * 0.5f);
  float qx = r.x * sh, qy = r.y * sh, qz = r.z * sh;
  const float inv = rsqrtf(qx * qx + qy * qy + qz * qz + qw * qw);
  qw *= inv;
  qx *= inv;
  qy *= inv;
  qz *= inv;
  float4& p = pos[*start + k];
  const float vx = p.x - c.x, vy = p.y - c.y, vz = p.z - c.z;
  p.x = vx * (qw * qw + qx * qx - qy * qy - qz * qz) + vy * (qx * qy - qw * qz) * 2.0f +
        vz * (qw * qy + qx * qz) * 2.0f + c.x;
  p.y = vx * (qw * qz + qx * qy) * 2.0f + vy * (qw * qw - qx * qx + qy * qy - qz * qz) +
        vz * (qy * qz - qw * qx) * 2.0f + c.y;
  p.z = vx * (qx * qz - qw * qy) * 2.0f + vy * (qy * qz + qw * qx) * 2.0f +
        vz * (qw * qw - qx * qx - qy * qy + qz * qz) + c.z;
}

__global__ void translate_molecule_kernel(float4* pos, const int* start, const int* length,
                                          const float4* t) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= *length) return;
  const float4 v = *t;
  float4& p = pos[*start + k];
  p.x += v.x;
  p.y += v.y;
  p.z += v.z;
}

// Runs after translate_molecule_kernel in stream order: the centre moves once.
__global__ void translate_center_kernel(float4* center, const float4* t) {
  const float4 v = *t;
  center->x += v.x;
  center->y += v.y;
  center->z += v.z;
}

// The scratch buffer of (current device, stream), locked by `lock`, holding
// at least n doubles. Growing it first waits for the work already queued on
// the stream (the only work that can still read the old buffer) and frees it.
// Returns null on failure.
double* stream_scratch(cudaStream_t stream, size_t n, std::unique_lock<std::mutex>& lock) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return nullptr;
  ScratchSlot* slot;
  {
    std::lock_guard<std::mutex> g(g_slots_mutex);
    std::unique_ptr<ScratchSlot>& p = g_slots[std::make_pair(dev, stream)];
    if (!p) p.reset(new ScratchSlot());
    slot = p.get();
  }
  lock = std::unique_lock<std::mutex>(slot->mu);
  if (slot->cap < n) {
    if (slot->ptr) {
      if (cudaStreamSynchronize(stream) != cudaSuccess) return nullptr;
      cudaFree(slot->ptr);
      slot->ptr = nullptr;
      slot->cap = 0;
    }
    const size_t cap = std::max<size_t>(n, 4096);
    if (cudaMalloc(&slot->ptr, cap * sizeof(double)) != cudaSuccess) {
      slot->ptr = nullptr;
      return nullptr;
    }
    slot->cap = cap;
  }
  return slot->ptr;
}

// ---- allocation-free energy (CUDA_EonDevice_noalloc)
// Fixed scratch for the per-item partials: a file-scope device array, so the
// entry point never allocates. Every GPU that loads this library holds it
// (256 KiB) until the process exits. REMC_NOALLOC_MAX_ITEMS items of 128 x 128
// beads cover up to 255 tiles, i.e. 32640 beads.
constexpr int kNoAllocMaxItems = REMC_NOALLOC_MAX_ITEMS;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxItems];

// Device address of g_noalloc_scratch, looked up once per device (the host
// name of a __device__ array is only a host-side stand-in).
double* g_noalloc_ptr[kMaxDevices] = {nullptr};

bool energy_args_ok(const float4* pos, const float4* meta, const float* table, int P) {
  if (!pos || !meta) {
    set_status(REMC_ERR_INVALID, "null position or metadata pointer");
    return false;
  }
  if (!table) {
    set_status(REMC_ERR_STATE, "no contact table: pass LJPotentials or call bindLJTexture");
    return false;
  }
  if (P <= 0) {
    set_status(REMC_ERR_INVALID, "datasetSize must be positive");
    return false;
  }
  return true;
}

// Enqueue the energy of P beads on `stream`: partials in scratch[0..n),
// total in scratch[n]; optionally the reference's per-block grid.
int enqueue_energy(const float4* pos, const float4* meta, const float* table, int P,
                   double* scratch, float* grid_out, int grid_n, cudaStream_t stream) {
  const int T = (P + kRefTile - 1) / kRefTile;
  const int n = T * (T + 1) / 2;
  float unscale = 1.0f;
  const RefConsts C = make_consts(&unscale);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::min(T * T, sms * 8);
  ref_energy_tiles<<<grid, kRefTile, 0, stream>>>(pos, meta, table, P, T, scratch, C);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_status(REMC_ERR_CUDA, "energy kernel launch", e);
    return REMC_ERR_CUDA;
  }
  ref_energy_sum<<<1, 256, 0, stream>>>(scratch, n, scratch + n, grid_out, grid_n, unscale);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_status(REMC_ERR_CUDA, "energy sum launch", e);
    return REMC_ERR_CUDA;
  }
  return REMC_OK;
}

}  // namespace

extern "C" {

int remc_reference_abi_status(void) { return g_status; }

int remc_reference_abi_set_params(const remc_params* p) {
  if (!p || !(p->debye_length > 0.0f)) {
    set_status(REMC_ERR_INVALID, "bad parameters");
    return REMC_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  g_params = *p;
  g_params_set = true;
  g_status = REMC_OK;
  return REMC_OK;
}

float* LJPotentialDataToDevice(const float* table) {
  float* d = nullptr;
  if (!table) {
    set_status(REMC_ERR_INVALID, "null table");
    return nullptr;
  }
  cudaError_t e = cudaMalloc(&d, 400 * sizeof(float));
  if (e != cudaSuccess) {
    set_status(REMC_ERR_NOMEM, "cudaMalloc", e);
    return nullptr;
  }
  e = cudaMemcpy(d, table, 400 * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d);
    set_status(REMC_ERR_CUDA, "cudaMemcpy", e);
    return nullptr;
  }
  set_status(REMC_OK, "");
  return d;
}

void copyLJPotentialDataToDevice(float* dev, const float* table) {
  if (!dev || !table) {
    set_status(REMC_ERR_INVALID, "null pointer");
    return;
  }
  cudaError_t e = cudaMemcpy(dev, table, 400 * sizeof(float), cudaMemcpyHostToDevice);
  set_status(e == cudaSuccess ? REMC_OK : REMC_ERR_CUDA, "cudaMemcpy", e);
}

void MCSearchOnDevice(void) { set_status(REMC_OK, ""); }

void CUDA_rotateMolecule(float4* d_pos, int* d_start, int* d_len, int moleculeLength,
                         float4* d_rot, float4* d_center, cudaStream_t stream) {
  if (!d_pos || !d_start || !d_len || !d_rot || !d_center || moleculeLength < 0) {
    set_status(REMC_ERR_INVALID, "bad argument");
    return;
  }
  if (moleculeLength == 0) return;
  rotate_molecule_kernel<<<(moleculeLength + 255) / 256, 256, 0, stream>>>(d_pos, d_start, d_len,
                                                                           d_rot, d_center);
  cudaError_t e = cudaGetLastError();
  set_status(e == cudaSuccess ? REMC_OK : REMC_ERR_CUDA, "rotate launch", e);
}

void CUDA_translateMolecule(float4* d_pos, int* d_start, int* d_len, int moleculeLength,
                            float4* d_t, float4* d_center, cudaStream_t stream) {
  if (!d_pos || !d_start || !d_len || !d_t || !d_center || moleculeLength < 0) {
    set_status(REMC_ERR_INVALID, "bad argument");
    return;
  }
  if (moleculeLength > 0)
    translate_molecule_kernel<<<(moleculeLength + 255) / 256, 256, 0, stream>>>(d_pos, d_start,
                                                                              d_len, d_t);
  translate_center_kernel<<<1, 1, 0, stream>>>(d_center, d_t);
  cudaError_t e = cudaGetLastError();
  set_status(e == cudaSuccess ? REMC_OK : REMC_ERR_CUDA, "translate launch", e);
}

void CUDA_EonDevice(float4* pos, float4* meta, int* residueCount, int* moleculePositions,
                    int* moleculeCount, float* LJPotentials, double* result, int blockSize,
                    int datasetSize, int sharedMemSize) {
  (void)residueCount;
  (void)moleculePositions;
  (void)moleculeCount;
  (void)blockSize;
  (void)sharedMemSize;
  const float* table = LJPotentials ? LJPotentials : g_bound_table;
  if (!result) {
    set_status(REMC_ERR_INVALID, "null result pointer");
    return;
  }
  if (!energy_args_ok(pos, meta, table, datasetSize)) return;
  const int T = (datasetSize + kRefTile - 1) / kRefTile;
  const size_t n = (size_t)T * (T + 1) / 2;
  // the reference's synchronous path runs on the legacy default stream; the
  // result copy is made under the scratch lock, before another host thread
  // can queue its energy on the same buffer
  std::unique_lock<std::mutex> lock;
  double* scratch = stream_scratch(0, n + 1, lock);
  if (!scratch) {
    set_status(REMC_ERR_NOMEM, "scratch allocation failed");
    return;
  }
  if (enqueue_energy(pos, meta, table, datasetSize, scratch, nullptr, 0, 0) != REMC_OK) return;
  cudaError_t e = cudaMemcpy(result, scratch + n, sizeof(double), cudaMemcpyDeviceToHost);
  set_status(e == cudaSuccess ? REMC_OK : REMC_ERR_CUDA, "result copy", e);
}

void CUDA_EonDevice_async(float4* pos, float4* meta, int* residueCount, int* moleculePositions,
                          int* moleculeCount, float* LJPotentials, float* device_result,
                          int resultSize, int blockSize, int datasetSize, int sharedMemSize,
                          cudaStream_t stream) {
  (void)residueCount;
  (void)moleculePositions;
  (void)moleculeCount;
  (void)blockSize;
  (void)sharedMemSize;
  const float* table = LJPotentials ? LJPotentials : g_bound_table;
  if (!device_result || resultSize <= 0) {
    set_status(REMC_ERR_INVALID, "bad result buffer");
    return;
  }
  if (!energy_args_ok(pos, meta, table, datasetSize)) return;
  const int T = (datasetSize + kRefTile - 1) / kRefTile;
  const size_t n = (size_t)T * (T + 1) / 2;
  // the stream's own scratch: energies queued on other streams run
  // concurrently on other buffers, and the next call on this stream reuses
  // this one only after this call's kernels, in stream order
  std::unique_lock<std::mutex> lock;
  double* scratch = stream_scratch(stream, n + 1, lock);
  if (!scratch) {
    set_status(REMC_ERR_NOMEM, "scratch allocation failed");
    return;
  }
  if (enqueue_energy(pos, meta, table, datasetSize, scratch, device_result,
                     resultSize * resultSize, stream) != REMC_OK)
    return;
  set_status(REMC_OK, "");
}

void CUDA_Esum_async(float*, float*, int, int, cudaStream_t) { set_status(REMC_OK, ""); }

int CUDA_memcpy_to_device(void* dst, void* src, int n) {
  return (int)cudaMemcpy(dst, src, (size_t)n, cudaMemcpyHostToDevice);
}
int CUDA_memcpy_to_host(void* dst, void* src, int n) {
  return (int)cudaMemcpy(dst, src, (size_t)n, cudaMemcpyDeviceToHost);
}
int CUDA_memcpy_to_device_async(void* dst, void* src, int n, cudaStream_t s) {
  return (int)cudaMemcpyAsync(dst, src, (size_t)n, cudaMemcpyHostToDevice, s);
}
int CUDA_memcpy_to_host_async(void* dst, void* src, int n, cudaStream_t s) {
  return (int)cudaMemcpyAsync(dst, src, (size_t)n, cudaMemcpyDeviceToHost, s);
}

void printCudaError(int code) { printf("CUDA error: %s\n", cudaGetErrorString((cudaError_t)code)); }

void cudaInfo(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    printf("ERROR: no devices supporting CUDA.\n");
    set_status(REMC_ERR_CUDA, "no CUDA device");
    return;
  }
  for (int i = 0; i < n; ++i) {
    cudaDeviceProp p;
    cudaGetDeviceProperties(&p, i);
    printf("CUDA Device %d: %s, %zu MB, %d SMs, sm_%d%d\n", i, p.name, p.totalGlobalMem >> 20,
           p.multiProcessorCount, p.major, p.minor);
  }
  set_status(REMC_OK, "");
}

void CUDA_setBoxDimension(float value) {
  if (!(value > 0.0f) || !std::isfinite(value)) {
    set_status(REMC_ERR_INVALID, "box edge must be positive");
    return;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  g_box = value;
  g_status = REMC_OK;
}

void CUDA_freeBoxDimension(void) { set_status(REMC_OK, ""); }

void bindLJTexture(float* ljp) {
  std::lock_guard<std::mutex> lock(g_mutex);
  g_bound_table = ljp;
  g_status = REMC_OK;
}

void unbindLJTexture(void) {
  std::lock_guard<std::mutex> lock(g_mutex);
  g_bound_table = nullptr;
  g_status = REMC_OK;
}

int CUDA_EonDevice_noalloc(const float4* pos, const float4* meta, const float* LJPotentials,
                           int datasetSize, double* d_result, cudaStream_t stream) {
  const float* table = LJPotentials ? LJPotentials : g_bound_table;
  if (!d_result) {
    set_status(REMC_ERR_INVALID, "null result pointer");
    return REMC_ERR_INVALID;
  }
  if (!energy_args_ok(pos, meta, table, datasetSize)) return g_status;
  const int T = (datasetSize + kRefTile - 1) / kRefTile;
  const long long n = (long long)T * (T + 1) / 2;
  if (n > kNoAllocMaxItems) {
    char buf[160];
    snprintf(buf, sizeof(buf),
             "datasetSize %d exceeds the allocation-free limit of %d beads (%d tile pairs)",
             datasetSize, REMC_NOALLOC_MAX_BEADS, kNoAllocMaxItems);
    set_status(REMC_ERR_INVALID, buf);
    return REMC_ERR_INVALID;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_status(REMC_ERR_CUDA, "cudaGetDevice", e);
    return REMC_ERR_CUDA;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_noalloc_ptr[dev]) {
      // once per device, with that device current
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        set_status(REMC_ERR_CUDA, "cudaGetSymbolAddress(scratch)", e);
        return REMC_ERR_CUDA;
      }
      g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    scratch = g_noalloc_ptr[dev];
  }
  // every item writes its partial before the sum reads it: no clearing needed
  const RefConsts C = make_consts();
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::min(T * T, sms * 8);
  ref_energy_tiles<<<grid, kRefTile, 0, stream>>>(pos, meta, table, datasetSize, T, scratch, C);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_status(REMC_ERR_CUDA, "energy kernel launch", e);
    return REMC_ERR_CUDA;
  }
  ref_energy_sum<<<1, 256, 0, stream>>>(scratch, (int)n, d_result, nullptr, 0, 1.0f);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_status(REMC_ERR_CUDA, "energy sum launch", e);
    return REMC_ERR_CUDA;
  }
  set_status(REMC_OK, "");
  return REMC_OK;
}

}  // extern "C"
