// B200 replica-exchange Monte Carlo engine: kernels and the C ABI of
// include/remc_b200.h.
//
// Data layout in HBM (all replica-instances of all systems of one handle):
//   pos    float4[inst beads]  x, y, z, bits(mol << 8 | type)   (SoA per bead)
//   rel    float4[inst beads]  position relative to the molecule centre
//   centre float4[inst mols]   molecule centre (Molecule::center)
//   quat   double[4*inst mols] accumulated rotation (Molecule::rotation)
//   energy double[inst]        running total energy (Replica::potential)
// Instance g of system s, slot k: beads at bead_base(s) + k*N_s, molecules at
// mol_base(s) + k*M_s.
//
// Kernels:
//   sweep_kernel       one CTA per replica-instance, persistent over a whole
//                      sweep of n_steps Metropolis steps; the instance's beads
//                      and molecule centres stay resident in shared memory, each
//                      step is proposal -> trial positions -> FP32 pair dE with
//                      FP64 reduction -> Metropolis (Replica::MCSearch,
//                      Replica.cpp:368-478, with dE in place of the full E).
//   energy_tile_kernel persistent grid over (instance, i-tile, j-tile) work
//                      items of the upper triangle; per-item FP64 partials in a
//                      scratch array, reduced per instance in fixed order by
//                      energy_reduce_kernel (Replica::E / E_TiledKernel,
//                      CudaFunctions.cu:455-685).
//   exchange_kernel    one warp per system, disjoint temperature pairs in
//                      parallel lanes (main.cpp:1427-1453).
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "remc_device.cuh"
#include "remc_internal.h"

using namespace remc;

namespace {

thread_local std::string g_last_error;

}  // namespace

void remc::record_error(const char* message) { g_last_error = message ? message : ""; }

namespace {

int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define REMC_CUDA_TRY(expr)                                                              \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess)                                                               \
      return set_error(REMC_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(_e));   \
  } while (0)

struct SysDev {
  int n_beads, n_mol, n_rep, lmax;
  int inst0, bead_base, mol_base, mstart_off;
  float box, invbox;
  int translate_only_crowders;
  int n_chain_beads;  // beads of residue type; the rest are crowders
  int crowd_type;     // the one bead type of every crowder, or -1 (none or mixed)
  // 1: every bead pair is within 1.5 box lengths on each axis, for the state
  // uploaded last and every state the sweep can reach from it (set on the
  // device by fold_flag_kernel at each upload; the sweep then folds the
  // minimum image)
  int fold_mi;
};

// Per-step proposal record: everything about step s of one replica that does
// not depend on the replica's state (Philox draws, chosen molecule, move type,
// translation vector, step quaternion). Written by proposal_kernel for a
// whole sweep, streamed through shared memory by sweep_kernel.
struct StepRec {
  double q[4];      // step quaternion (rotation)
  double thr;       // Metropolis threshold -log(u)/beta: accept iff dE < thr
  float t[3];       // translation vector
  int m;            // molecule
  int m0;           // its first bead
  int info;         // bits 0-29: its bead count; bit 30: rotation; bit 31: crowder
};
constexpr int kRecRotate = 1 << 30;
constexpr int kRecCrowd = (int)(1u << 31);
constexpr int kRecCount = kRecRotate - 1;
static_assert(sizeof(StepRec) == 64, "StepRec layout");

struct ProposalArgs {
  const SysDev* sys;
  const int* inst_sys;
  const int* mol_start;
  const int* mol_role;
  const int* mrole_off;  // per system: offset of its roles in mol_role
  const float* tstep;
  const double* rot_cs;
  const float* ladder;
  const int* temp_idx;
  StepRec* recs;         // [n_inst][rec_stride]
  const uint32_t* ctrl;
  uint32_t step0;
  uint32_t seed_lo, seed_hi;
  int n_inst, n_steps, rec_stride;
};

// One thread per (instance, step): Replica::MCSearch's choices for that step
// (Replica.cpp:384-402) from the counter-based stream.
__global__ void __launch_bounds__(256) proposal_kernel(ProposalArgs P) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)P.n_inst * P.n_steps) return;
  const int inst = (int)(idx / P.n_steps), s = (int)(idx % P.n_steps);
  const int sysid = P.inst_sys[inst];
  const SysDev S = P.sys[sysid];
  const int slot = inst - S.inst0;
  const uint32_t step = (P.ctrl ? P.ctrl[0] : P.step0) + (uint32_t)s;
  uint4 c = make_uint4(step, (uint32_t)slot, (uint32_t)sysid, 0u);
  const uint2 k = make_uint2(P.seed_lo, P.seed_hi);
  const uint4 x = philox4x32_10(c, k);
  c.w = 1u;
  const uint4 y = philox4x32_10(c, k);
  const double u0 = u32_unit(x.x), u1 = u32_unit(x.y), u2 = u32_unit(x.z), u3 = u32_unit(x.w);
  const double u4 = u32_unit(y.x), u5 = u32_unit(y.y);
  StepRec r;
  r.m = (int)__dmul_rn(u0, (double)S.n_mol);
  const bool crowd = P.mol_role[P.mrole_off[sysid] + r.m] == -1;
  const bool rotate = (u1 < 0.5) && !(S.translate_only_crowders && crowd);
  r.m0 = P.mol_start[S.mstart_off + r.m];
  r.info = (P.mol_start[S.mstart_off + r.m + 1] - r.m0) | (rotate ? kRecRotate : 0) |
           (crowd ? kRecCrowd : 0);
  // u < exp(-beta dE)  <=>  dE < -log(u)/beta  (Replica.cpp:451); u = 0 never
  // passes the reference's test, so its threshold is -inf
  const float T = P.ladder[S.inst0 + P.temp_idx[inst]];
  const double beta = 4184.0 / ((double)8.314472f * (double)T);
  r.thr = u5 > 0.0 ? -log(u5) / beta : -INFINITY;
  if (rotate) {
    step_quaternion(u2, u3, u4, P.rot_cs[2 * inst], P.rot_cs[2 * inst + 1], r.q);
    r.t[0] = r.t[1] = r.t[2] = 0.0f;
  } else {
    const float3 t = translate_vector(u2, u3, u4, P.tstep[inst]);
    r.t[0] = t.x;
    r.t[1] = t.y;
    r.t[2] = t.z;
    r.q[0] = 1.0;
    r.q[1] = r.q[2] = r.q[3] = 0.0;
  }
  P.recs[(size_t)inst * P.rec_stride + s] = r;
}

// Work order of the persistent sweep. Its makespan is set by the replicas that
// take longest, and a replica's block of steps costs what its proposals ask
// for: which molecules move (a chain of n beads against the other N - n
// beads, or one bead) is drawn before the sweep. block_cost_kernel sums, per
// instance, the pair evaluations of its n_steps records plus `step_cost` per
// step for the step's fixed work (record, reduction, barrier, decision); a
// one-bead rotation has no pairs. Integer sums, so the result does not depend
// on the order of the additions. One CTA per instance.
__global__ void __launch_bounds__(256) block_cost_kernel(const SysDev* __restrict__ sys,
                                                         const int* __restrict__ inst_sys,
                                                         const StepRec* __restrict__ recs,
                                                         int rec_stride, int n_steps,
                                                         long long step_cost,
                                                         long long* __restrict__ cost) {
  const int inst = blockIdx.x;
  const int N = sys[inst_sys[inst]].n_beads;
  const StepRec* r = recs + (size_t)inst * rec_stride;
  long long c = 0;
  for (int s = threadIdx.x; s < n_steps; s += blockDim.x) {
    const int info = r[s].info;
    const long long n = info & kRecCount;
    const bool still = (info & kRecRotate) && n == 1;  // a one-bead rotation moves nothing
    c += (still ? 0 : n * (N - n)) + step_cost;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  __shared__ unsigned long long s_sum;
  if (threadIdx.x == 0) s_sum = 0ull;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) atomicAdd(&s_sum, (unsigned long long)c);
  __syncthreads();
  if (threadIdx.x == 0) cost[inst] = (long long)s_sum;
}

// order[k] = the instance of rank k by decreasing cost, ties by instance
// index: a strict total order, so the ranks are a permutation. One warp per
// instance; its lanes split the n comparisons (n up to kMaxRankedInst).
constexpr int kMaxRankedInst = 65536;
__global__ void __launch_bounds__(256) rank_kernel(const long long* __restrict__ cost, int n,
                                                   int* __restrict__ order) {
  const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n) return;  // whole warps
  const long long ci = cost[i];
  unsigned rank = 0;
  for (int j = lane; j < n; j += 32) {
    const long long cj = cost[j];
    rank += (cj > ci) || (cj == ci && j < i);
  }
  rank = __reduce_add_sync(0xffffffffu, rank);
  if (lane == 0) order[rank] = i;
}

// A bound conformation recorded by Replica::sample (Replica.cpp:1717-1780):
// header + one pose (rotation quaternion, centre) per molecule.
struct SampleHeader {
  int inst;
  uint32_t label;     // step label (start of the sampling chunk, main.cpp:983-987)
  double e_nc;        // potential + chain-chain pair energy (the sample() sum)
  double e;           // potential
  float temperature;
  int n_mol;
  uint32_t pose_offset;
  int pad;
};
struct SamplePose {
  double q[4];
  float c[3];
  float pad;
};

struct SweepArgs {
  const SysDev* sys;
  const int* inst_sys;
  const int* inst_list;  // instances, largest expected cost first
  int* queue;            // work counter (persistent grid), or null: CTA b runs inst_list[b]
  int n_list;
  float4* pos;
  float4* rel;
  float4* centre;
  double* quat;
  const int* mol_start;
  const float4* tab;
  const StepRec* recs;   // [n_inst][rec_stride]
  double* energy;
  double* ecc;           // chain-chain part of the energy (sample() sum)
  const int* temp_idx;
  const float* ladder;
  // sampling (Replica::sample): every `sample_every` steps, labels from step0
  int sample_every;
  uint32_t sample_after;
  double bound_thr;
  const uint32_t* ctrl;
  uint32_t step0;
  int* n_samples;
  int* n_bound;
  SampleHeader* sample_out;
  SamplePose* pose_out;
  unsigned* sample_cursor;  // [0] records, [1] poses, [2] dropped
  unsigned sample_cap, pose_cap;
  int* acc_neg;          // accepted with dE < 0
  int* acc_boltz;        // accepted by the Boltzmann test
  int* rej;
  unsigned long long* evals_kh;     // residue-residue pair evaluations
  unsigned long long* evals_crowd;  // pair evaluations involving a crowder
  int rec_stride, rec_offset;       // records of step s at rec_offset + s
  int n_steps;
  int nmax, mmax, lmax;  // shared-memory capacities
  int mol_in_smem;       // centres resident in shared memory
  int csize;             // CTAs per replica (a thread-block cluster), 1, 2, 4 or 8
  // beads kept in global memory (systems too large for shared memory): trial
  // positions and trial relative positions of each (instance, CTA rank), 6 lmax
  float4* trial_scratch;
  EnergyConsts K;
};

constexpr int kRing = 64;  // proposal records held in shared memory (two halves)

// Shared-memory layout of sweep_kernel, in bytes, for capacities (nmax beads,
// mmax molecules, lmax beads per molecule).
struct SweepSmem {
  size_t tab, beads, centres, trial_pos, trial_rel, ring, red, total;
  static __host__ __device__ size_t take(size_t& off, size_t bytes) {
    size_t o = off;
    off += (bytes + 15) & ~size_t(15);
    return o;
  }
  // mol_in_smem = 0: molecule centres and starts stay in global memory (the
  // largest systems), everything else as usual. beads_in_smem = 0: the beads
  // and the trial buffers stay in global memory too (systems of any size)
  static __host__ __device__ SweepSmem make(int nmax, int mmax, int lmax, int mol_in_smem,
                                            int csize = 1, int beads_in_smem = 1) {
    SweepSmem s;
    size_t off = 0;
    s.tab = take(off, sizeof(float4) * kNT * kNT);
    s.beads = take(off, beads_in_smem ? sizeof(float4) * nmax : 0);
    s.centres = take(off, mol_in_smem ? sizeof(float4) * mmax : 0);
    s.trial_pos = take(off, beads_in_smem ? sizeof(float4) * 4 * lmax : 0);
    s.trial_rel = take(off, beads_in_smem ? sizeof(float4) * 2 * lmax : 0);
    s.ring = take(off, sizeof(StepRec) * kRing);
    s.red = take(off, sizeof(double) * 2 * csize * 2 * 32);  // [parity][rank][dE, dcc][warp]
    s.total = off;
    return s;
  }
};

// Sum of 8 FP64 partials (16-byte aligned) in a fixed pairwise order; the
// entries of warps a smaller CTA does not have hold an exact zero. Every
// thread evaluates it and gets the same value.
__device__ __forceinline__ double tree_sum8(const double* v) {
  const double2* v2 = reinterpret_cast<const double2*>(v);
  const double2 a = v2[0], b = v2[1], c = v2[2], d = v2[3];
  return ((a.x + a.y) + (b.x + b.y)) + ((c.x + c.y) + (d.x + d.y));
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n"); }

// One CTA per replica-instance, persistent over the sweep. The instance's beads
// and molecule centres stay in shared memory for all n_steps steps.
//
// Ownership: in the pair loop thread t reads only beads j = t (mod T), and the
// same thread writes those beads when a move is accepted, so bead updates need
// no barrier. Every thread computes the FP64 sum of the per-warp partials and
// the Metropolis decision itself (same order, same result), and tracks the
// previous step's move to read a molecule moved one step ago from registers or
// the trial buffer rather than from another thread's not-yet-ordered write.
// A step of a one-bead molecule therefore costs one barrier; a chain step
// costs two (trial positions are built by the owners of the chain's beads).
// GB: the beads stay where they are in global memory (updated in place, no
// prologue copy and no write-back) and the trial buffers live in per-instance
// global scratch; every access pattern, owner and barrier is the same as with
// the beads in shared memory (a CTA barrier orders global memory for the CTA,
// a cluster barrier for the cluster; the CTAs of a cluster write identical
// values to the beads they own).
template <bool R12, bool CUT, bool CLUSTER, bool GB>
__global__ void __launch_bounds__(256, 2) sweep_kernel(SweepArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SweepSmem L = SweepSmem::make(A.nmax, A.mmax, A.lmax, A.mol_in_smem, A.csize, !GB);
  float4* s_tab = reinterpret_cast<float4*>(smem_raw + L.tab);
  float4* const sm_beads = reinterpret_cast<float4*>(smem_raw + L.beads);
  float4* s_cent = reinterpret_cast<float4*>(smem_raw + L.centres);
  float4* const sm_tpos = reinterpret_cast<float4*>(smem_raw + L.trial_pos);
  StepRec* s_ring = reinterpret_cast<StepRec*>(smem_raw + L.ring);
  double* s_red = reinterpret_cast<double*>(smem_raw + L.red);

  const int tid = threadIdx.x, nthr = blockDim.x;
  const int tmask = nthr - 1;  // nthr is a power of two
  const int lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
  // A replica may span a cluster of csize CTAs: every CTA holds the whole
  // replica and runs every step, the pair loops split bead j over the
  // cluster's threads (CTA rank r, thread t takes j = r T + t mod csize T;
  // within a CTA that is still j = t mod T, so ownership is unchanged), the
  // warps' partial sums go to every CTA's shared memory, and one cluster
  // barrier per step replaces the CTA barrier. Rank 0 alone writes state that
  // is not idempotent (rotations, counters, samples) and the final state.
  const int csize = CLUSTER ? A.csize : 1;
  const int crank = CLUSTER ? (int)cooperative_groups::this_cluster().block_rank() : 0;
  const int gtid = crank * nthr + tid, gstride = nthr * csize, gmask = gstride - 1;
  __shared__ int s_next;
  for (int it = 0;; ++it) {
  int idx;
  if (A.queue) {
    if (tid == 0) s_next = atomicAdd(A.queue, 1);
    __syncthreads();
    idx = s_next;
    __syncthreads();  // every thread has read s_next before it is rewritten
    if (idx >= A.n_list) break;
  } else {
    if (it > 0) break;
    idx = blockIdx.x / csize;
  }
  const int inst = A.inst_list[idx];
  const int sysid = A.inst_sys[inst];
  const SysDev S = A.sys[sysid];
  const int slot = inst - S.inst0;
  const int N = S.n_beads, M = S.n_mol;
  const int bead_off = S.bead_base + slot * N;
  const int mol_off = S.mol_base + slot * M;
  const float box = S.box, invbox = S.invbox;
  const StepRec* recs = A.recs + (size_t)inst * A.rec_stride + A.rec_offset;
  const int n_steps = A.n_steps;
  float4* const s_beads = GB ? A.pos + bead_off : sm_beads;
  // per-(instance, CTA rank) global scratch of 6 lmax entries: trial
  // positions (used when the beads stay in global memory) and trial
  // relative positions
  float4* const scratch =
      A.trial_scratch + ((size_t)inst * csize + crank) * 6 * (size_t)A.lmax;
  // trial positions of a chain move, two entries per moved bead k, by step
  // parity b: s_tpos[2 (b lmax + k)] = (new x, old x, new y, old y),
  // s_tpos[2 (b lmax + k) + 1] = (new z, old z, meta word, table row offset),
  // so that each (new, old) coordinate pair is a register pair of the packed
  // pair loops as loaded
  float4* const s_tpos = GB ? scratch : sm_tpos;
  // rotated relative positions of the chain's beads, computed with its trial
  // positions by the beads' owners and installed by the same threads (each
  // thread reads back only what it wrote), in shared memory, or in global
  // scratch when the beads stay in global memory. The install writes rel
  // without reading it, so the CTAs of a cluster, which all install the same
  // values, cannot read one another's update. Two buffers by step parity,
  // like the trial positions: the next step's owners (another molecule,
  // other threads) write theirs before any barrier, while slower warps may
  // still install from this step's
  float4* const s_trel =
      GB ? scratch + 4 * (size_t)A.lmax : reinterpret_cast<float4*>(smem_raw + L.trial_rel);

  // ---- prologue: make the instance resident in shared memory
  for (int i = tid; i < kNT * kNT; i += nthr) s_tab[i] = A.tab[i];
  // partial-sum entries of warps this CTA does not have: an exact zero
  for (int i = tid; i < 2 * csize * 2 * 8; i += nthr)
    if ((i & 7) >= nwarps) s_red[(i >> 3) * 32 + (i & 7)] = 0.0;
  if (!GB)
    for (int i = tid; i < N; i += nthr) s_beads[i] = A.pos[bead_off + i];
  // molecule centres: shared memory, or global memory for the largest
  // systems (thread 0 writes a centre; others read it only after a later
  // barrier, which orders global memory within the CTA as well)
  float4* cent = A.mol_in_smem ? s_cent : A.centre + mol_off;
  if (A.mol_in_smem)
    for (int i = tid; i < M; i += nthr) s_cent[i] = A.centre[mol_off + i];
  {
    // first ring fill: records of steps 0..min(kRing, n_steps)-1, 16 B per copy
    const int nrec = min(kRing, n_steps);
    const int chunks = nrec * (int)(sizeof(StepRec) / 16);
    for (int c = tid; c < chunks; c += nthr)
      cp_async16(reinterpret_cast<char*>(s_ring) + 16 * c,
                 reinterpret_cast<const char*>(recs) + 16 * c);
    cp_async_commit();
    cp_async_wait_all();
  }
  // every thread keeps the running energies (all see the same dE and decision)
  double energy = A.energy[inst], ecc = A.ecc[inst];
  int n_neg = 0, n_boltz = 0, n_rej = 0, n_samp = 0, n_bnd = 0;
  unsigned long long ev_kh = 0, ev_crowd = 0;
  const int ncb = S.n_chain_beads;  // beads [0, ncb) belong to chains
  const int ctype = S.crowd_type;   // the crowders' one type, or -1
  const uint32_t step0 = A.ctrl ? A.ctrl[0] : A.step0;
  int to_sample = A.sample_every;  // steps left in the current sampling chunk
  __shared__ long long s_pose_slot;
  // every CTA of a cluster has started before any writes another's shared memory
  if (CLUSTER)
    cooperative_groups::this_cluster().sync();
  else
    __syncthreads();
  float4 next_c = make_float4(0.f, 0.f, 0.f, 0.f);
  if (n_steps > 0 && !A.mol_in_smem) next_c = cent[s_ring[0].m];

  // previous step, known to every thread
  int p_m = -1, p_acc = 0, p_rot = 0, p_n = 0, p_b = 0;
  float4 p_single = make_float4(0.f, 0.f, 0.f, 0.f);  // accepted one-bead position
  float p_nc0 = 0.f, p_nc1 = 0.f, p_nc2 = 0.f;          // accepted new centre

  for (int s = 0; s < n_steps; ++s) {
    // ---- prefetch the next ring half (records s+31 .. s+62). The half it
    // overwrites ends with step s-2's record, which is read until after step
    // s-2's barrier; a thread at step s has passed step s-1's barrier, so no
    // thread reads it any more
    if ((s & 31) == 1 && s > 1 && s + 31 < n_steps) {
      const int first = s + 31;
      const int nrec = min(32, n_steps - first);
      const int chunks = nrec * (int)(sizeof(StepRec) / 16);
      char* dst = reinterpret_cast<char*>(s_ring + (first & (kRing - 1)));
      const char* src = reinterpret_cast<const char*>(recs + first);
      for (int c = tid; c < chunks; c += nthr) cp_async16(dst + 16 * c, src + 16 * c);
      cp_async_commit();
    }
    const StepRec& recs_ = s_ring[s & (kRing - 1)];  // stable for the whole step
    struct {
      int m, rotate, crowd;
      float t[3];
    } rec;
    rec.m = recs_.m;
    rec.rotate = (recs_.info & kRecRotate) != 0;
    rec.crowd = (recs_.info & kRecCrowd) != 0;
    rec.t[0] = recs_.t[0];
    rec.t[1] = recs_.t[1];
    rec.t[2] = recs_.t[2];
    const int m = rec.m;
    const int m0 = recs_.m0, n = recs_.info & kRecCount;
    const int b = s & 1;
    const bool same = (m == p_m) && p_acc;  // moved (and accepted) last step
    // centre of m: the one this step's thread computed last step if m moved
    // then, else the one loaded at the end of the previous step
    float c0, c1, c2;
    if (same && !p_rot) {
      c0 = p_nc0;
      c1 = p_nc1;
      c2 = p_nc2;
    } else {
      const float4 c = A.mol_in_smem ? cent[m] : next_c;
      c0 = c.x;
      c1 = c.y;
      c2 = c.z;
    }
    float nc0 = c0, nc1 = c1, nc2 = c2;
    if (!rec.rotate) {
      const float x0 = __fadd_rn(__fadd_rn(c0, rec.t[0]), box);
      const float x1 = __fadd_rn(__fadd_rn(c1, rec.t[1]), box);
      const float x2 = __fadd_rn(__fadd_rn(c2, rec.t[2]), box);
      // c + t + L almost always lies in [0, 2L), where wrap_box subtracts L
      // or nothing: one test for all three, selects instead of branches
      const float L2 = 2.0f * box;  // exact
      if (x0 >= 0.0f && x0 < L2 && x1 >= 0.0f && x1 < L2 && x2 >= 0.0f && x2 < L2) {
        nc0 = x0 < box ? x0 : __fsub_rn(x0, box);
        nc1 = x1 < box ? x1 : __fsub_rn(x1, box);
        nc2 = x2 < box ? x2 : __fsub_rn(x2, box);
      } else {
        nc0 = wrap_box(x0, box);
        nc1 = wrap_box(x1, box);
        nc2 = wrap_box(x2, box);
      }
    }
    // a one-bead rotation moves nothing (its bead sits at the centre): dE = 0
    const bool skip = rec.rotate && n == 1;
    float4 pold1, pnew1;  // one-bead molecule: old/new position in registers
    if (n == 1) {
      pold1 = same ? p_single : s_beads[m0];
      pnew1 = make_float4(nc0, nc1, nc2, pold1.w);
    } else {
      // trial positions of the chain, built by the owners of its beads
      QuatProducts qp{};
      if (rec.rotate) qp = quat_products(recs_.q[0], recs_.q[1], recs_.q[2], recs_.q[3]);
      int j = m0 + ((tid - m0) & tmask);
      for (; j < m0 + n; j += nthr) {
        const int k = j - m0;
        const float4 rl = A.rel[bead_off + j];
        // the bead's current position: this thread owns it and installed
        // its last move itself
        const float4 ol = s_beads[j];
        float4 np;
        if (rec.rotate) {
          const float3 r2 = rotate_rel(qp, rl.x, rl.y, rl.z);
          np = make_float4(__fadd_rn(r2.x, nc0), __fadd_rn(r2.y, nc1), __fadd_rn(r2.z, nc2), ol.w);
          s_trel[b * A.lmax + k] = make_float4(r2.x, r2.y, r2.z, 0.0f);
        } else {
          np = make_float4(__fadd_rn(rl.x, nc0), __fadd_rn(rl.y, nc1), __fadd_rn(rl.z, nc2), ol.w);
        }
        float4* e = s_tpos + 2 * (b * A.lmax + k);
        e[0] = make_float4(np.x, ol.x, np.y, ol.y);
        e[1] = make_float4(np.z, ol.z, ol.w, __int_as_float(bead_type(ol.w) * kNT));
      }
      __syncthreads();  // trial positions and the previous chain update visible
    }

    // ---- dE over beads j outside the molecule (thread t owns j = t mod T).
    // Beads are chains [0, ncb) then crowders [ncb, N); the moved molecule's
    // own beads [m0, m0 + n) split the range in two. Residue-residue pairs of
    // a chain move are the change of the chain-chain energy sample() adds.
    double dacc = 0.0, dcc = 0.0;
    if (!skip) {
      const int x0 = m0, x1 = m0 + n;
      float acc_c = 0.0f, acc_o = 0.0f;
      if (n == 1) {
        // one bead (a crowder or a one-residue chain), positions in registers
        const int ta = bead_type(pold1.w);
        const float4* trow = s_tab + ta * kNT;
        if (rec.crowd) {
          // a one-bead crowder: every pair is a crowder pair. One loop over
          // the thread's j in increasing order (the order of the per-thread
          // sum), two j per pass with both loads issued first, the moved
          // bead itself (j = m0) left out of the sum
          const bool one_ct = ctype >= 0;
          const float4 Tc = trow[one_ct ? ctype : 0];
          // the two beads of a pass as the two lanes of packed FP32, against
          // the moved bead's new and old position (negated once per step)
          const PackedBox PB1 = packed_box(box, invbox);
          const float2 nnx = make_float2(-pnew1.x, -pnew1.x), nny = make_float2(-pnew1.y, -pnew1.y),
                       nnz = make_float2(-pnew1.z, -pnew1.z);
          const float2 nox = make_float2(-pold1.x, -pold1.x), noy = make_float2(-pold1.y, -pold1.y),
                       noz = make_float2(-pold1.z, -pold1.z);
          int j = gtid;
          // folded minimum image where the system allows it (fold_mi)
          auto pass1 = [&](auto fold) {
            constexpr bool F = decltype(fold)::value;
            for (; j + gstride < N; j += 2 * gstride) {
              const int j2 = j + gstride;
              const float4 pa = s_beads[j], pb = s_beads[j2];
              const float4 Ta = (one_ct && j >= ncb) ? Tc : trow[bead_type(pa.w)];
              const float4 Tb = (one_ct && j2 >= ncb) ? Tc : trow[bead_type(pb.w)];
              const float2 xj = make_float2(pa.x, pb.x), yj = make_float2(pa.y, pb.y),
                           zj = make_float2(pa.z, pb.z);
              const float2 A2 = make_float2(Ta.x, Tb.x), C2 = make_float2(Ta.z, Tb.z);
              const float2 en =
                  crowd_energy2<R12, CUT>(pair_r2_2<F>(xj, yj, zj, nnx, nny, nnz, PB1), A2, C2);
              const float2 eo =
                  crowd_energy2<R12, CUT>(pair_r2_2<F>(xj, yj, zj, nox, noy, noz, PB1), A2, C2);
              const float2 d = __fadd2_rn(en, make_float2(-eo.x, -eo.y));
              if (j != m0) acc_o += d.x;
              if (j2 != m0) acc_o += d.y;
            }
          };
          if (S.fold_mi) pass1(std::true_type{}); else pass1(std::false_type{});
          if (j < N && j != m0) {
            const float4 pa = s_beads[j];
            const float4 Ta = (one_ct && j >= ncb) ? Tc : trow[bead_type(pa.w)];
            const float en = crowd_energy<R12, CUT>(pair_r2(pnew1, pa, box, invbox), Ta.x, Ta.z);
            const float eo = crowd_energy<R12, CUT>(pair_r2(pold1, pa, box, invbox), Ta.x, Ta.z);
            acc_o += en - eo;
          }
        } else {
          // a one-residue chain: residue pairs with the chains' beads,
          // crowder pairs with the rest
          for (int part = 0; part < 2; ++part) {
            const int lo = part ? x1 : 0, hi = part ? N : x0;
            if (lo >= hi) continue;
            const int cb = min(hi, ncb);
            int j = lo + ((gtid - lo) & gmask);  // first j >= lo in this thread's class
            for (; j < cb; j += gstride) {
              const float4 pj = s_beads[j];
              const float4 Tj = trow[bead_type(pj.w)];
              const float en = pair_energy_r2(pair_r2(pnew1, pj, box, invbox), Tj, false, A.K);
              const float eo = pair_energy_r2(pair_r2(pold1, pj, box, invbox), Tj, false, A.K);
              acc_c += en - eo;
            }
            const float4 Tc = trow[ctype >= 0 ? ctype : 0];
            for (; j < hi; j += gstride) {
              const float4 pj = s_beads[j];
              const float4 Tj = ctype >= 0 ? Tc : trow[bead_type(pj.w)];
              const float en = crowd_energy<R12, CUT>(pair_r2(pnew1, pj, box, invbox), Tj.x, Tj.z);
              const float eo = crowd_energy<R12, CUT>(pair_r2(pold1, pj, box, invbox), Tj.x, Tj.z);
              acc_o += en - eo;
            }
          }
        }
      } else {
        // a chain (or a multi-bead crowder): each thread takes its beads j and
        // runs over the n moved beads k, the same k in every lane. Two j per
        // pass where the class has them, so each k's positions and table row
        // serve two beads; each j's sum over k is added on its own, in j order
        const float4* tp = s_tpos + 2 * b * A.lmax;
        for (int part = 0; part < 2; ++part) {
          const int lo = part ? x1 : 0, hi = part ? N : x0;
          if (lo >= hi) continue;
          const int cb = min(hi, ncb);
          int j = lo + ((gtid - lo) & gmask);
          if (!rec.crowd) {
            // residue pairs: the new and the old evaluation of a pair as the
            // two lanes of packed FP32
            const PackedBox PB = packed_box(box, invbox);
            auto pass2 = [&](auto fold) {
              constexpr bool F = decltype(fold)::value;
              for (; j + gstride < cb; j += 2 * gstride) {
                const float4 pa = s_beads[j], pb = s_beads[j + gstride];
                const int ta = bead_type(pa.w), tb = bead_type(pb.w);
                const float2 nax = make_float2(-pa.x, -pa.x), nay = make_float2(-pa.y, -pa.y),
                             naz = make_float2(-pa.z, -pa.z);
                const float2 nbx = make_float2(-pb.x, -pb.x), nby = make_float2(-pb.y, -pb.y),
                             nbz = make_float2(-pb.z, -pb.z);
                float a = 0.0f, c = 0.0f;
#pragma unroll 2
                for (int k = 0; k < n; ++k) {
                  const float4 P = tp[2 * k], Q = tp[2 * k + 1];
                  const float2 kx = make_float2(P.x, P.y), ky = make_float2(P.z, P.w),
                               kz = make_float2(Q.x, Q.y);
                  const float4* row = s_tab + __float_as_int(Q.w);
                  const float4 Ta = row[ta], Tb = row[tb];
                  const float2 ea =
                      kh_energy2(pair_r2_2<F>(kx, ky, kz, nax, nay, naz, PB), Ta, A.K.c_xi);
                  const float2 eb =
                      kh_energy2(pair_r2_2<F>(kx, ky, kz, nbx, nby, nbz, PB), Tb, A.K.c_xi);
                  a += ea.x - ea.y;
                  c += eb.x - eb.y;
                }
                acc_c += a;
                acc_c += c;
              }
            };
            if (S.fold_mi) pass2(std::true_type{}); else pass2(std::false_type{});
          }
          for (; j < cb; j += gstride) {
            const float4 pj = s_beads[j];
            const int tb = bead_type(pj.w);
            float a = 0.0f;
            if (!rec.crowd) {
              for (int k = 0; k < n; ++k) {
                const float4 P = tp[2 * k], Q = tp[2 * k + 1];
                const float4 pn = make_float4(P.x, P.z, Q.x, 0.0f), po = make_float4(P.y, P.w, Q.y, 0.0f);
                const float4 T = s_tab[__float_as_int(Q.w) + tb];
                const float en = pair_energy_r2(pair_r2(pn, pj, box, invbox), T, false, A.K);
                const float eo = pair_energy_r2(pair_r2(po, pj, box, invbox), T, false, A.K);
                a += en - eo;
              }
              acc_c += a;
            } else {
              for (int k = 0; k < n; ++k) {
                const float4 P = tp[2 * k], Q = tp[2 * k + 1];
                const float4 pn = make_float4(P.x, P.z, Q.x, 0.0f), po = make_float4(P.y, P.w, Q.y, 0.0f);
                const float4 T = s_tab[__float_as_int(Q.w) + tb];
                const float en = crowd_energy<R12, CUT>(pair_r2(pn, pj, box, invbox), T.x, T.z);
                const float eo = crowd_energy<R12, CUT>(pair_r2(po, pj, box, invbox), T.x, T.z);
                a += en - eo;
              }
              acc_o += a;
            }
          }
          const bool one_ct = ctype >= 0;
          const PackedBox PBc = packed_box(box, invbox);
          auto pass3 = [&](auto fold) {
            constexpr bool F = decltype(fold)::value;
            for (; j + gstride < hi; j += 2 * gstride) {
              const float4 pa = s_beads[j], pb = s_beads[j + gstride];
              const int ta = bead_type(pa.w), tb = bead_type(pb.w);
              const float2 nax = make_float2(-pa.x, -pa.x), nay = make_float2(-pa.y, -pa.y),
                           naz = make_float2(-pa.z, -pa.z);
              const float2 nbx = make_float2(-pb.x, -pb.x), nby = make_float2(-pb.y, -pb.y),
                           nbz = make_float2(-pb.z, -pb.z);
              float a = 0.0f, c = 0.0f;
#pragma unroll 2
              for (int k = 0; k < n; ++k) {
                const float4 P = tp[2 * k], Q = tp[2 * k + 1];
                const float2 kx = make_float2(P.x, P.y), ky = make_float2(P.z, P.w),
                             kz = make_float2(Q.x, Q.y);
                const float4* row = s_tab + __float_as_int(Q.w);
                const float4 Ta = row[ta];
                const float4 Tb = one_ct ? Ta : row[tb];  // one crowder species: ta == tb
                const float2 ea = crowd_energy2<R12, CUT>(pair_r2_2<F>(kx, ky, kz, nax, nay, naz, PBc),
                                                          make_float2(Ta.x, Ta.x),
                                                          make_float2(Ta.z, Ta.z));
                const float2 eb = crowd_energy2<R12, CUT>(pair_r2_2<F>(kx, ky, kz, nbx, nby, nbz, PBc),
                                                          make_float2(Tb.x, Tb.x),
                                                          make_float2(Tb.z, Tb.z));
                a += ea.x - ea.y;
                c += eb.x - eb.y;
              }
              acc_o += a;
              acc_o += c;
            }
          };
          if (S.fold_mi) pass3(std::true_type{}); else pass3(std::false_type{});
          for (; j < hi; j += gstride) {
            const float4 pj = s_beads[j];
            const int tb = bead_type(pj.w);
            float a = 0.0f;
            for (int k = 0; k < n; ++k) {
              const float4 P = tp[2 * k], Q = tp[2 * k + 1];
              const float4 pn = make_float4(P.x, P.z, Q.x, 0.0f), po = make_float4(P.y, P.w, Q.y, 0.0f);
              const float4 T = s_tab[__float_as_int(Q.w) + tb];
              const float en = crowd_energy<R12, CUT>(pair_r2(pn, pj, box, invbox), T.x, T.z);
              const float eo = crowd_energy<R12, CUT>(pair_r2(po, pj, box, invbox), T.x, T.z);
              a += en - eo;
            }
            acc_o += a;
          }
        }
      }
      dcc = (double)acc_c;
      dacc = (double)acc_o;
    }
    dacc = warp_sum(dacc);
    if (!rec.crowd) dcc = warp_sum(dcc);
    if (lane == 0) {
      if (!CLUSTER) {
        s_red[b * 64 + warp] = dacc;
        s_red[b * 64 + 32 + warp] = dcc;
      } else {
        cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
        for (int r = 0; r < csize; ++r) {
          double* dst = cl.map_shared_rank(s_red, r) + (b * csize + crank) * 64;
          dst[warp] = dacc;
          dst[32 + warp] = dcc;
        }
      }
    }
    if ((s & 31) == 31) cp_async_wait_all();  // next ring half has landed
    // R: partial sums (and the prefetched records) visible
    if (!CLUSTER)
      __syncthreads();
    else
      cooperative_groups::this_cluster().sync();

    // ---- every thread: the same FP64 sums (a fixed pairwise tree over the
    // warps' partials) and the same Metropolis decision
    if (s + 1 < n_steps && A.mol_in_smem == 0) {
      next_c = cent[s_ring[(s + 1) & (kRing - 1)].m];
    }
    double dE = tree_sum8(s_red + b * csize * 64);
    double dE_cc = 0.0;
    if (!rec.crowd) dE_cc = tree_sum8(s_red + b * csize * 64 + 32);
    for (int r = 1; r < csize; ++r) {  // the other CTAs' sums, in rank order
      dE += tree_sum8(s_red + (b * csize + r) * 64);
      if (!rec.crowd) dE_cc += tree_sum8(s_red + (b * csize + r) * 64 + 32);
    }
    if (!rec.crowd) dE += dE_cc;
    const int acc = dE < 0.0 ? 1 : (dE < recs_.thr ? 2 : 0);
    if (acc) {
      energy += dE;
      ecc += dE_cc;
      if (n == 1) {
        if (tid == (m0 & tmask)) s_beads[m0] = pnew1;
        p_single = pnew1;
      } else {
        // the owners install the chain (and its relative positions)
        int j = m0 + ((tid - m0) & tmask);
        for (; j < m0 + n; j += nthr) {
          const float4* e = s_tpos + 2 * (b * A.lmax + (j - m0));
          const float4 P = e[0], Q = e[1];
          s_beads[j] = make_float4(P.x, P.z, Q.x, Q.z);
          if (rec.rotate) A.rel[bead_off + j] = s_trel[b * A.lmax + (j - m0)];
        }
      }
      if (tid == 0 && rec.rotate && crank == 0) {
        double* qd = A.quat + 4 * (size_t)(mol_off + m);
        double out[4];
        quat_mul(recs_.q[0], recs_.q[1], recs_.q[2], recs_.q[3], qd[0], qd[1], qd[2], qd[3], out);
        qd[0] = out[0];
        qd[1] = out[1];
        qd[2] = out[2];
        qd[3] = out[3];
      }
      if (tid == 0 && !rec.rotate) cent[m] = make_float4(nc0, nc1, nc2, 0.0f);
    }
    // counters: every thread keeps them (no branch on the thread index);
    // thread 0 of rank 0 writes them out
    n_neg += acc == 1;
    n_boltz += acc == 2;
    n_rej += acc == 0;
    if (!skip) {
      // two evaluations (old and new position) per pair
      const unsigned nn2 = 2u * (unsigned)n;
      if (rec.crowd) {
        ev_crowd += (unsigned long long)nn2 * (unsigned)(N - n);
      } else {
        ev_kh += (unsigned long long)nn2 * (unsigned)(S.n_chain_beads - n);
        ev_crowd += (unsigned long long)nn2 * (unsigned)(N - S.n_chain_beads);
      }
    }
    // ---- Replica::sample at the end of every sampling chunk (main.cpp:975-989):
    // bound if potential (+ chain-chain energy when crowders exist) < threshold
    if (to_sample > 0 && --to_sample == 0) {
      to_sample = A.sample_every;
      const uint32_t label = step0 + (uint32_t)(s + 1 - A.sample_every);
      if (label >= A.sample_after) {
        const double enc = (ncb < N) ? energy + ecc : energy;
        const bool bound = enc < A.bound_thr;
        ++n_samp;  // every thread; thread 0 of rank 0 writes them out
        n_bnd += bound ? 1 : 0;
        if (bound && A.sample_out && crank == 0) {
          __syncthreads();  // this step's centre / rotation writes visible
          if (tid == 0) {
            const unsigned r = atomicAdd(&A.sample_cursor[0], 1u);
            const unsigned p0 = atomicAdd(&A.sample_cursor[1], (unsigned)M);
            if (r < A.sample_cap && (unsigned long long)p0 + M <= A.pose_cap) {
              SampleHeader hd;
              hd.inst = inst;
              hd.label = label;
              hd.e_nc = enc;
              hd.e = energy;
              hd.temperature = A.ladder[S.inst0 + A.temp_idx[inst]];
              hd.n_mol = M;
              hd.pose_offset = p0;
              hd.pad = 0;
              A.sample_out[r] = hd;
              s_pose_slot = p0;
            } else {
              atomicAdd(&A.sample_cursor[2], 1u);
              s_pose_slot = -1;
            }
          }
          __syncthreads();
          const long long p0 = s_pose_slot;
          if (p0 >= 0) {
            for (int i = tid; i < M; i += nthr) {
              const double* qd = A.quat + 4 * (size_t)(mol_off + i);
              const float4 c = cent[i];
              SamplePose ps;
              ps.q[0] = qd[0];
              ps.q[1] = qd[1];
              ps.q[2] = qd[2];
              ps.q[3] = qd[3];
              ps.c[0] = c.x;
              ps.c[1] = c.y;
              ps.c[2] = c.z;
              ps.pad = 0.0f;
              A.pose_out[p0 + i] = ps;
            }
          }
          __syncthreads();  // poses read before the next step moves anything
        }
      }
    }
    p_m = m;
    p_acc = acc != 0;
    p_rot = rec.rotate;
    p_n = n;
    p_b = b;
    p_nc0 = nc0;
    p_nc1 = nc1;
    p_nc2 = nc2;
  }
  (void)p_n;
  __syncthreads();

  // ---- epilogue: write the instance back (every CTA of a cluster holds the
  // same state; rank 0 writes it)
  if (crank == 0) {
  if (!GB)
    for (int i = tid; i < N; i += nthr) A.pos[bead_off + i] = s_beads[i];
  if (A.mol_in_smem)
    for (int i = tid; i < M; i += nthr) A.centre[mol_off + i] = s_cent[i];
  }
  if (tid == 0 && crank == 0) {
    A.energy[inst] = energy;
    A.ecc[inst] = ecc;
    A.n_samples[inst] += n_samp;
    A.n_bound[inst] += n_bnd;
    A.acc_neg[inst] += n_neg;
    A.acc_boltz[inst] += n_boltz;
    A.rej[inst] += n_rej;
    A.evals_kh[inst] += ev_kh;
    A.evals_crowd[inst] += ev_crowd;
  }
  __syncthreads();  // shared memory is reused by the next instance
  }  // instance loop
  // no CTA leaves while another may still write into its shared memory
  if (CLUSTER) cooperative_groups::this_cluster().sync();
}

// ------------------------------------------------------------------ state staging
// Host layout (3 floats per bead and molecule) <-> device layout (float4 with
// the bead meta word), converted on the device so that uploads and downloads
// are plain copies of the caller's buffers.
__global__ void state_check_kernel(const float* __restrict__ pos3, const float* __restrict__ rel3,
                                   const float* __restrict__ cen3, const int* __restrict__ info,
                                   long long nb, long long nm,
                                   unsigned long long* __restrict__ bad) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nb; i += stride) {
    const float* p = pos3 + 3 * i;
    const float* r = rel3 + 3 * i;
    bool fin = true;
    for (int k = 0; k < 3; ++k) fin = fin && isfinite(p[k]) && isfinite(r[k]);
    if (!fin) atomicMin(&bad[0], (unsigned long long)i);
    if ((info[i] & (int)0x80000000u) && (r[0] != 0.0f || r[1] != 0.0f || r[2] != 0.0f))
      atomicMin(&bad[1], (unsigned long long)i);
  }
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < nm; m += stride) {
    const float* c = cen3 + 3 * m;
    if (!(isfinite(c[0]) && isfinite(c[1]) && isfinite(c[2])))
      atomicMin(&bad[2], (unsigned long long)m);
  }
}

__global__ void state_pack_kernel(const float* __restrict__ pos3, const float* __restrict__ rel3,
                                  const float* __restrict__ cen3, const int* __restrict__ info,
                                  long long nb, long long nm, float4* __restrict__ pos,
                                  float4* __restrict__ rel, float4* __restrict__ cen) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nb; i += stride) {
    pos[i] = make_float4(pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2],
                         __int_as_float(info[i] & 0x7fffffff));
    rel[i] = make_float4(rel3[3 * i], rel3[3 * i + 1], rel3[3 * i + 2], 0.0f);
  }
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < nm; m += stride)
    cen[m] = make_float4(cen3[3 * m], cen3[3 * m + 1], cen3[3 * m + 2], 0.0f);
}

__global__ void state_unpack_kernel(const float4* __restrict__ pos, const float4* __restrict__ rel,
                                    const float4* __restrict__ cen, long long nb, long long nm,
                                    float* __restrict__ pos3, float* __restrict__ rel3,
                                    float* __restrict__ cen3) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nb; i += stride) {
    const float4 p = pos[i], r = rel[i];
    pos3[3 * i] = p.x;
    pos3[3 * i + 1] = p.y;
    pos3[3 * i + 2] = p.z;
    rel3[3 * i] = r.x;
    rel3[3 * i + 1] = r.y;
    rel3[3 * i + 2] = r.z;
  }
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < nm; m += stride) {
    const float4 c = cen[m];
    cen3[3 * m] = c.x;
    cen3[3 * m + 1] = c.y;
    cen3[3 * m + 2] = c.z;
  }
}

// May the sweep fold the minimum image of a system? A bead the sweep has not
// moved is where it was uploaded; a moved molecule has its centre in [0, L)
// (translations wrap it, rotations leave it) and each bead within R of it (a
// rotation of rel keeps |rel|), R the largest |rel| over all instances. So on
// each axis every bead lies in [min(p_min, -R), max(p_max, L + R)], and no two
// are further apart than that interval is long. fold_image2 needs less than
// 1.5 L; the test keeps a margin (1.01 R, 1.49 L) for the rounding of repeated
// rotations. fold_part_kernel: one CTA per instance, its largest |rel|^2 and
// bead extent (part[inst][0..6]: R^2, -p_min xyz, p_max xyz, all combined by
// max); fold_flag_kernel: one CTA per system combines its instances.
__global__ void fold_part_kernel(const SysDev* __restrict__ sys, const int* __restrict__ inst_sys,
                                 const float4* __restrict__ pos, const float4* __restrict__ rel,
                                 float* __restrict__ part) {
  __shared__ float s_v[7][32];
  const int inst = blockIdx.x;
  const SysDev S = sys[inst_sys[inst]];
  const size_t base = S.bead_base + (size_t)(inst - S.inst0) * S.n_beads;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const float lowest = -3.0e38f;
  float v[7] = {0.0f, lowest, lowest, lowest, lowest, lowest, lowest};
  for (int i = tid; i < S.n_beads; i += blockDim.x) {
    const float4 q = rel[base + i], p = pos[base + i];
    v[0] = fmaxf(v[0], fmaf(q.x, q.x, fmaf(q.y, q.y, q.z * q.z)));
    v[1] = fmaxf(v[1], -p.x);
    v[2] = fmaxf(v[2], -p.y);
    v[3] = fmaxf(v[3], -p.z);
    v[4] = fmaxf(v[4], p.x);
    v[5] = fmaxf(v[5], p.y);
    v[6] = fmaxf(v[6], p.z);
  }
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    for (int off = 16; off > 0; off >>= 1) v[k] = fmaxf(v[k], __shfl_down_sync(0xffffffffu, v[k], off));
    if (lane == 0) s_v[k][warp] = v[k];
  }
  __syncthreads();
  if (tid < 7) {
    float w = s_v[tid][0];
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) w = fmaxf(w, s_v[tid][q]);
    part[(size_t)inst * 8 + tid] = w;
  }
}

__global__ void fold_flag_kernel(SysDev* __restrict__ sys, const float* __restrict__ part) {
  __shared__ float s_v[7][32];
  const SysDev S = sys[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const float lowest = -3.0e38f;
  float v[7] = {0.0f, lowest, lowest, lowest, lowest, lowest, lowest};
  for (int i = tid; i < S.n_rep; i += blockDim.x)
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] = fmaxf(v[k], part[(size_t)(S.inst0 + i) * 8 + k]);
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    for (int off = 16; off > 0; off >>= 1) v[k] = fmaxf(v[k], __shfl_down_sync(0xffffffffu, v[k], off));
    if (lane == 0) s_v[k][warp] = v[k];
  }
  __syncthreads();
  if (tid == 0) {
    float w[7];
    for (int k = 0; k < 7; ++k) {
      w[k] = s_v[k][0];
      for (int q = 1; q < (int)(blockDim.x >> 5); ++q) w[k] = fmaxf(w[k], s_v[k][q]);
    }
    const float R = 1.01f * sqrtf(w[0]), lim = 1.49f * S.box;
    bool ok = true;
    for (int a = 0; a < 3; ++a)  // max(p_max, L + R) - min(p_min, -R)
      ok = ok && fmaxf(w[4 + a], S.box + R) + fmaxf(w[1 + a], R) <= lim;
    sys[blockIdx.x].fold_mi = ok ? 1 : 0;
  }
}

// ------------------------------------------------------------------ full E
struct TileItem {
  int inst, ti, tj;
  int slot;  // the item's place in the instance-grouped list (its partial's slot)
};

constexpr int kTile = 128;

// Crowder-wall energy of bead i against the tile's beads [a, b), added to acc
// in ascending j: two beads per pass in packed FP32 from the tile's
// coordinate arrays (an odd first bead, and a last one, alone). FIXED: one
// table entry for every j (crowders of the system's one species), else the
// entry of each j's type. FOLD: the folded minimum image (the system's every
// bead pair is within 1.5 box lengths on each axis).
template <bool R12, bool CUT, bool FIXED, bool FOLD>
__device__ __forceinline__ void crowd_run(const float* __restrict__ sx, const float* __restrict__ sy,
                                          const float* __restrict__ sz, const int* __restrict__ st,
                                          const float4* __restrict__ s_tab, int ta, float4 Tfix,
                                          int j0, int a, int b, float4 pi, float2 npx, float2 npy,
                                          float2 npz, const PackedBox& B, float box, float invbox,
                                          float& acc) {
  int j = a;
  if (j < b && ((j - j0) & 1)) {
    const int o = j - j0;
    const float4 T = FIXED ? Tfix : s_tab[st[o] * kNT + ta];
    acc += crowd_energy<R12, CUT>(pair_r2_f<FOLD>(pi, make_float4(sx[o], sy[o], sz[o], 0.0f), box, invbox),
                                  T.x, T.z);
    ++j;
  }
  const float2 Af = make_float2(Tfix.x, Tfix.x), Cf = make_float2(Tfix.z, Tfix.z);
#pragma unroll 2
  for (; j + 1 < b; j += 2) {
    const int o = j - j0;  // even: 8-byte aligned pairs
    const float2 r2 = pair_r2_2<FOLD>(*reinterpret_cast<const float2*>(sx + o),
                                *reinterpret_cast<const float2*>(sy + o),
                                *reinterpret_cast<const float2*>(sz + o), npx, npy, npz, B);
    float2 A2 = Af, C2 = Cf;
    if (!FIXED) {
      const float4 Ta = s_tab[st[o] * kNT + ta], Tb = s_tab[st[o + 1] * kNT + ta];
      A2 = make_float2(Ta.x, Tb.x);
      C2 = make_float2(Ta.z, Tb.z);
    }
    const float2 e = crowd_energy2<R12, CUT>(r2, A2, C2);
    acc += e.x;
    acc += e.y;
  }
  if (j < b) {
    const int o = j - j0;
    const float4 T = FIXED ? Tfix : s_tab[st[o] * kNT + ta];
    acc += crowd_energy<R12, CUT>(pair_r2_f<FOLD>(pi, make_float4(sx[o], sy[o], sz[o], 0.0f), box, invbox),
                                  T.x, T.z);
  }
}

// Energy of bead i (position pi, type ta) against the j beads [lo, hi) of the
// tile (s_j, and by coordinate sx, sy, sz with types st), in ascending j,
// leaving out the beads [xa, xb) of its own molecule. Beads are stored chains
// first, crowders after, so the range splits into a chain part [lo, ncb) and a
// crowder part [ncb, hi), and each part runs a loop specialised to its pair
// class:
//   chain i, chain j ..... Kim-Hummer + Debye-Hueckel, table entry per pair
//                          (added to the chain-chain sum as well);
//   any i, crowder j ..... crowder wall with the table entry fixed per i when
//                          the system has one crowder species;
//   crowder i, chain j ... crowder wall, table entry per residue type.
// The crowder-wall loops take two beads per pass in packed FP32. The single
// accumulator runs in ascending j, as one unspecialised loop would. FOLD: the
// folded minimum image (the system's fold flag is set).
template <bool R12, bool CUT, bool FOLD>
__device__ __forceinline__ void energy_row(const float4* __restrict__ s_j,
                                           const float* __restrict__ sx,
                                           const float* __restrict__ sy,
                                           const float* __restrict__ sz,
                                           const int* __restrict__ st, int j0, int lo, int hi,
                                           int xa, int xb, int ncb, int ctype, float4 pi, int ta,
                                           const float4* __restrict__ s_tab, float box,
                                           float invbox, const EnergyConsts& K, float& acc,
                                           float& acc_cc) {
  const bool a_crowd = ta >= kNumAmino;
  const PackedBox B = packed_box(box, invbox);
  const float2 npx = make_float2(-pi.x, -pi.x), npy = make_float2(-pi.y, -pi.y),
               npz = make_float2(-pi.z, -pi.z);
  const float4 Tc = s_tab[(ctype >= 0 ? ctype : 0) * kNT + ta];
  // two sub-ranges of [lo, hi) outside the own molecule
  const int r0a = lo, r0b = min(hi, xa);
  const int r1a = max(lo, xb), r1b = hi;
  for (int part = 0; part < 2; ++part) {
    const int a = part ? r1a : r0a, b = part ? r1b : r0b;
    if (a >= b) continue;
    const int cb = min(b, ncb);  // [a, cb): chain beads; [max(a, ncb), b): crowders
    if (!a_crowd) {
#pragma unroll 4
      for (int j = a; j < cb; ++j) {
        const float4 pj = s_j[j - j0];
        const float4 T = s_tab[bead_type(pj.w) * kNT + ta];
        const float e = pair_energy_r2(pair_r2_f<FOLD>(pi, pj, box, invbox), T, false, K);
        acc += e;
        acc_cc += e;
      }
    } else {
      crowd_run<R12, CUT, false, FOLD>(sx, sy, sz, st, s_tab, ta, Tc, j0, a, cb, pi, npx, npy, npz, B,
                                 box, invbox, acc);
    }
    const int ca = max(a, ncb);
    if (ctype >= 0)
      crowd_run<R12, CUT, true, FOLD>(sx, sy, sz, st, s_tab, ta, Tc, j0, ca, b, pi, npx, npy, npz, B,
                                box, invbox, acc);
    else
      crowd_run<R12, CUT, false, FOLD>(sx, sy, sz, st, s_tab, ta, Tc, j0, ca, b, pi, npx, npy, npz, B,
                                 box, invbox, acc);
  }
}

// Polls of a bounded mbarrier wait (each poll may suspend the thread for a
// while); reaching the limit means the copy never completed.
constexpr int kWaitLimit = 1 << 22;

// Location of an item's j-tile in pos (contiguous, 16-byte aligned, 16 bytes
// per bead).
__device__ __forceinline__ const float4* tile_src(const SysDev* __restrict__ sys,
                                                  const int* __restrict__ inst_sys,
                                                  const float4* __restrict__ pos, TileItem W,
                                                  unsigned* bytes) {
  const SysDev S = sys[inst_sys[W.inst]];
  const int N = S.n_beads;
  const int j0 = W.tj * kTile;
  *bytes = 16u * (unsigned)min(kTile, N - j0);
  return pos + S.bead_base + (W.inst - S.inst0) * N + j0;
}

// Two-stage pipeline over the CTA's items with one CTA barrier per item:
// while item k is computed, the bulk copy (TMA, no multicast) of item k+1's
// j-tile lands in the other buffer. Item k's barrier, after every thread's
// own wait for its tile and its share of the by-coordinate copy, also shows
// that every thread has finished item k-1: only then does thread 0 issue the
// copy into item k-1's buffer and add up item k-1's warp partials. The
// by-coordinate copies and the warp partials are double-buffered like the
// tiles.
__global__ void __launch_bounds__(kTile) energy_tile_kernel(
    const SysDev* __restrict__ sys, const int* __restrict__ inst_sys,
    const float4* __restrict__ pos, const float4* __restrict__ tab,
    const int* __restrict__ mol_start, const TileItem* __restrict__ items, int n_items,
    int* __restrict__ queue, double* __restrict__ scratch, double* __restrict__ scratch_cc,
    EnergyConsts K, int* __restrict__ err) {
  __shared__ float4 s_tab[kNT * kNT];
  __shared__ __align__(128) float4 s_j[2][kTile];  // two stages
  // the tile by coordinate, and its bead types, per stage
  __shared__ __align__(16) float s_jx[2][kTile], s_jy[2][kTile], s_jz[2][kTile];
  __shared__ int s_jt[2][kTile];
  __shared__ double s_red[2][kTile / 32];
  __shared__ double s_red_cc[2][kTile / 32];
  __shared__ __align__(8) unsigned long long s_bar[2];
  // the items whose tiles are (or go next) in buffers 0 and 1, from a work
  // queue over the list sorted by decreasing cost; each item's partials go
  // to its slot in the instance-grouped list, so the per-instance reduction
  // does not depend on which CTA took which item, or when
  __shared__ int s_item[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < kNT * kNT; i += kTile) s_tab[i] = tab[i];
  if (tid == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    const int first = atomicAdd(queue, 1);
    s_item[0] = first;
    s_item[1] = atomicAdd(queue, 1);
    if (first < n_items) {
      unsigned bytes;
      const float4* src = tile_src(sys, inst_sys, pos, items[first], &bytes);
      bulk_load(s_j[0], src, bytes, &s_bar[0]);
    }
  }
  __syncthreads();  // barriers initialised, s_item set
  unsigned phases = 0;  // bit b: parity of buffer b's next completion
  int buf = 0;
  int prev = -1;  // the previous item's slot, whose partials thread 0 writes out
  for (;; buf ^= 1) {
    // s_item[buf] was written before a barrier every thread has passed
    const int it = s_item[buf];
    if (it >= n_items) break;
    const TileItem W = items[it];
    const SysDev S = sys[inst_sys[W.inst]];
    const int N = S.n_beads;
    const int base = S.bead_base + (W.inst - S.inst0) * N;
    const int j0 = W.tj * kTile;
    const int jn = min(kTile, N - j0);
    // this thread's i bead, loaded while the tile is still in flight
    const int i = W.ti * kTile + tid;
    const bool ivalid = i < N;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    int xa = 0, xb = 0;
    if (ivalid) {
      pi = pos[base + i];
      const int mi = bead_mol(pi.w);
      xa = mol_start[S.mstart_off + mi];
      xb = mol_start[S.mstart_off + mi + 1];
    }
    const bool ok = mbar_wait(&s_bar[buf], (phases >> buf) & 1u, kWaitLimit);
    phases ^= 1u << buf;
    const float4* tile = s_j[buf];
    if (ok && tid < jn) {
      const float4 p = tile[tid];
      s_jx[buf][tid] = p.x;
      s_jy[buf][tid] = p.y;
      s_jz[buf][tid] = p.z;
      s_jt[buf][tid] = bead_type(p.w);
    }
    // this item's coordinate copy is complete and every thread is done with
    // the previous item (its tile buffer, coordinate copy and partials)
    if (__syncthreads_or(!ok)) {  // the copy never landed: report and stop
      if (tid == 0) {
        atomicOr(err, 1);
        // the copy given up on still writes this CTA's shared memory (the
        // next one is not issued yet): wait for it again, bounded, before
        // the CTA leaves; it can leave with the copy in flight only if this
        // wait runs out as well
        mbar_wait(&s_bar[buf], ((phases >> buf) & 1u) ^ 1u, kWaitLimit);
      }
      return;
    }
    if (tid == 0) {
      const int next = s_item[buf ^ 1];  // written by this thread
      if (prev >= 0) {
        double v = 0.0, c = 0.0;
        for (int w = 0; w < kTile / 32; ++w) {
          v += s_red[buf ^ 1][w];
          c += s_red_cc[buf ^ 1][w];
        }
        scratch[prev] = v;
        scratch_cc[prev] = c;
      }
      if (next < n_items) {
        unsigned bytes;
        const float4* src = tile_src(sys, inst_sys, pos, items[next], &bytes);
        bulk_load(s_j[buf ^ 1], src, bytes, &s_bar[buf ^ 1]);
      }
      // the item after next, for this buffer: every thread read s_item[buf]
      // before this item's barrier
      s_item[buf] = atomicAdd(queue, 1);
    }
    double dsum = 0.0, dcc = 0.0;
    if (ivalid) {
      const int ta = bead_type(pi.w);
      const int lo = (W.ti == W.tj) ? i + 1 : j0;
      float acc = 0.0f, acc_cc = 0.0f;  // all pairs; chain-chain pairs
#define REMC_ENERGY_ROW(R12_, CUT_, FOLD_)                                                        \
  energy_row<R12_, CUT_, FOLD_>(tile, s_jx[buf], s_jy[buf], s_jz[buf], s_jt[buf], j0, lo, j0 + jn, \
                                xa, xb, S.n_chain_beads, S.crowd_type, pi, ta, s_tab, S.box,     \
                                S.invbox, K, acc, acc_cc)
      if (K.crowder_mode) {
        if (K.crowder_cut) {
          if (S.fold_mi) REMC_ENERGY_ROW(true, true, true); else REMC_ENERGY_ROW(true, true, false);
        } else {
          if (S.fold_mi) REMC_ENERGY_ROW(true, false, true); else REMC_ENERGY_ROW(true, false, false);
        }
      } else {
        if (K.crowder_cut) {
          if (S.fold_mi) REMC_ENERGY_ROW(false, true, true); else REMC_ENERGY_ROW(false, true, false);
        } else {
          if (S.fold_mi) REMC_ENERGY_ROW(false, false, true); else REMC_ENERGY_ROW(false, false, false);
        }
      }
#undef REMC_ENERGY_ROW
      dsum = (double)acc;
      dcc = (double)acc_cc;
    }
    dsum = warp_sum(dsum);
    dcc = warp_sum(dcc);
    if (lane == 0) {
      s_red[buf][warp] = dsum;
      s_red_cc[buf][warp] = dcc;
    }
    prev = W.slot;
  }
  __syncthreads();  // the last item's partials are written
  if (tid == 0 && prev >= 0) {
    double v = 0.0, c = 0.0;
    for (int w = 0; w < kTile / 32; ++w) {
      v += s_red[buf ^ 1][w];
      c += s_red_cc[buf ^ 1][w];
    }
    scratch[prev] = v;
    scratch_cc[prev] = c;
  }
}

// One warp waits, with the energy kernel's bounded mbarrier wait, for a
// phase that nothing completes (no copy is issued, nothing arrives): after
// `polls` polls the wait gives up and the error word is set, as when a tile's
// bulk copy never lands. Nothing is in flight when the kernel returns.
__global__ void wait_probe_kernel(int* __restrict__ err, int polls) {
  __shared__ __align__(8) unsigned long long s_bar;
  if (threadIdx.x == 0) mbar_init(&s_bar, 1);
  __syncthreads();
  const bool ok = mbar_wait(&s_bar, 0u, polls);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(err, 1);
}

// Per-instance fixed-order sum of the tile partials.
__global__ void energy_reduce_kernel(const int* __restrict__ item_off, int n_inst,
                                     const double* __restrict__ scratch,
                                     const double* __restrict__ scratch_cc,
                                     double* __restrict__ energy, double* __restrict__ ecc) {
  const int inst = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (inst >= n_inst) return;
  const int a = item_off[inst], b = item_off[inst + 1];
  double v = 0.0, c = 0.0;
  for (int i = a + lane; i < b; i += 32) {
    v += scratch[i];
    c += scratch_cc[i];
  }
  v = warp_sum(v);
  c = warp_sum(c);
  if (lane == 0) {
    energy[inst] = v;
    ecc[inst] = c;
  }
}


// ------------------------------------------------------------------ adjoint
// Forces and parameter derivatives of the full energy: same upper-triangle
// items as energy_tile_kernel. Thread i keeps its bead's force in registers;
// the force on each j bead is warp-reduced per j into per-warp shared rows and
// added to global memory once per item. dE/deps comes from the per-type-pair
// sums G_ab = sum d e / d eps_ab (eps enters each residue pair linearly),
// dE/dXi from sum e_DH r / Xi^2.
struct AdjConsts {
  float inv_xi;   // 1/Xi
  float c_lj;     // LJ_CF * KBT_CF (d e / d eps per unit of the 4 s6 (1 - s6) form)
  float inv_xi2;  // 1/Xi^2
};

// Forces of one j group of 8 on this lane's bead i, and the group's j forces
// summed over the warp into s_fj. Lane L takes the 8 beads in the order
// j = jg + (q ^ r), r = (L >> 2) & 7, so that every level of the
// recursive-halving transpose-reduce keeps and sends fixed registers:
// after the xor-16, xor-8 and xor-4 levels and the xor-2/xor-1 sums, the four
// lanes of group r hold the warp's total force from bead jg + r.
// CHAIN: beads [jg, jend) are residues (Kim-Hummer + Debye-Hueckel against a
// residue i, crowder wall against a crowder i); else crowders (wall).
// CHECK = false when every lane's 8 pairs are known to count.
template <bool R12, bool CUT, bool CHAIN, bool CHECK>
__device__ __forceinline__ void adjoint_group(
    const float4* __restrict__ s_j, const float4* __restrict__ s_tab, float* __restrict__ s_G,
    float (*__restrict__ s_fjw)[3], int jg, int jend, int jlo, int ex0, int ex1, bool ivalid,
    float4 pi, int ta, bool a_crowd, float4 Tc, bool tc_fixed, float box, float invbox,
    const EnergyConsts& K, const AdjConsts& C, int lane, float& fx, float& fy, float& fz,
    float& acc_e, float& acc_x) {
  const int r = (lane >> 2) & 7;
  float g[8][3];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    g[q][0] = g[q][1] = g[q][2] = 0.0f;
    const int jj = jg + (q ^ r);
    if (CHECK) {
      const bool valid = ivalid && jj < jend && jj >= jlo &&
                         (unsigned)(jj - ex0) >= (unsigned)(ex1 - ex0);
      if (!valid) continue;
    }
    const float4 pj = s_j[jj];
    const float dx = min_image(pi.x - pj.x, box, invbox);
    const float dy = min_image(pi.y - pj.y, box, invbox);
    const float dz = min_image(pi.z - pj.z, box, invbox);
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const float rinv = fast_rsqrt(r2);
    const float rinv2 = rinv * rinv;
    float f;  // -(de/dr)/r
    if (CHAIN && !a_crowd) {
      const int tb = bead_type(pj.w);
      const float4 T = s_tab[tb * kNT + ta];
      const float s2 = T.y * rinv2;
      const float s6 = s2 * s2 * s2;
      const float gg = fmaf(-s6, s6, s6);  // s6 (1 - s6)
      float lj = T.x * gg;
      float dlj = 6.0f * T.x * s6 * fmaf(-2.0f, s6, 1.0f) * rinv2;  // -(dLJ/dr)/r
      float dg = 4.0f * gg;                                          // d e_LJ / d eps per c_lj
      if (r2 < T.z) {
        lj = fmaf(0.5f, T.x, -lj);
        dlj = -dlj;
        dg = 2.0f - dg;
      }
      const float rr = r2 * rinv;
      const float dh = T.w * fast_ex2(rr * K.c_xi) * rinv;
      acc_e += lj + dh;
      acc_x += dh * rr;  // * 1/Xi^2 by the caller
      f = dlj + dh * (C.inv_xi + rinv) * rinv;
      atomicAdd(&s_G[ta * kNumAmino + tb], dg * C.c_lj);
    } else {
      const float4 T = (!CHAIN && tc_fixed) ? Tc : s_tab[bead_type(pj.w) * kNT + ta];
      const float e = crowd_energy<R12, CUT>(r2, T.x, T.z);
      acc_e += e;
      f = (R12 ? 12.0f : 6.0f) * e * rinv2;
    }
    const float gx = f * dx, gy = f * dy, gz = f * dz;
    fx += gx;
    fy += gy;
    fz += gz;
    g[q][0] = gx;
    g[q][1] = gy;
    g[q][2] = gz;
  }
  float h4[4][3];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) h4[q][c] = g[q][c] + __shfl_xor_sync(0xffffffffu, g[q + 4][c], 16);
  float h2[2][3];
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) h2[q][c] = h4[q][c] + __shfl_xor_sync(0xffffffffu, h4[q + 2][c], 8);
  float h1[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    h1[c] = h2[0][c] + __shfl_xor_sync(0xffffffffu, h2[1][c], 4);
    h1[c] += __shfl_xor_sync(0xffffffffu, h1[c], 2);
    h1[c] += __shfl_xor_sync(0xffffffffu, h1[c], 1);
  }
  if ((lane & 3) == 0 && jg + r < jend) {
    // force on j = -(sum of the forces this warp's i beads feel from j)
    s_fjw[jg + r][0] -= h1[0];
    s_fjw[jg + r][1] -= h1[1];
    s_fjw[jg + r][2] -= h1[2];
  }
}

// The common case of adjoint_group: crowder beads j of one species (fixed
// table entry Tc) and a group that needs no per-pair tests, evaluated two
// pairs at a time in packed FP32 (f32x2: one instruction per operation on
// both pairs, each element rounded as the scalar operation would be). The
// lane pairs its beads q and q + 4 (j = jg + (q ^ r) and jg + ((q + 4) ^ r)),
// exactly the two the first transpose-reduce level combines, so the j forces
// land in the same registers as in adjoint_group. Coordinates come from the
// tile's structure-of-arrays copy, so both beads' x (y, z) load straight into
// one register pair: gx, gy, gz hold the group's coordinates with beads q
// and q + 4 side by side (q < 4), in the order this lane's half-warp pairs
// them (see adjoint_tile_kernel), so each pair is one 8-byte load per
// coordinate. Works with e = p_j - p_i = -d: the forces it sums are the
// negated pair forces (the caller negates the i-force sums; the j beads
// receive them as they are).
// MASK: a group with pairs to leave out (j <= i in a diagonal tile, the i
// bead's own molecule, j past the tile's end; coordinates there may be stale):
// every pair is evaluated and the left-out ones' energy and forces are
// replaced by zero, which costs less than the scalar checked path.
template <bool R12, bool CUT, bool MASK>
__device__ __forceinline__ void adjoint_group_crowd2(
    const float* __restrict__ gx8, const float* __restrict__ gy8,
    const float* __restrict__ gz8, float (*__restrict__ s_fjw)[3], int jg, int jend,
    float2 npx, float2 npy, float2 npz, float A, float cut2, float box, float invbox, int lane,
    float2& nfx, float2& nfy, float2& nfz, float2& acc_e2, bool ivalid = true, int jlo = 0,
    int ex0 = 0, int ex1 = 0) {
  const int r = (lane >> 2) & 7;
  const float kMagic = 12582912.0f;  // 1.5 * 2^23, as in min_image
  const float2 iL = make_float2(invbox, invbox), nL = make_float2(-box, -box);
  const float2 M = make_float2(kMagic, kMagic), nM = make_float2(-kMagic, -kMagic);
  const float2 A2 = make_float2(A, A);
  const float2 cf = make_float2(R12 ? 12.0f : 6.0f, R12 ? 12.0f : 6.0f);
  float g[8][3];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    // beads jg + (q ^ r) and jg + ((q + 4) ^ r), in that order
    const int o = 2 * ((q ^ r) & 3);
    float2 ex = __fadd2_rn(*reinterpret_cast<const float2*>(gx8 + o), npx);
    float2 ey = __fadd2_rn(*reinterpret_cast<const float2*>(gy8 + o), npy);
    float2 ez = __fadd2_rn(*reinterpret_cast<const float2*>(gz8 + o), npz);
    ex = __ffma2_rn(nL, __fadd2_rn(__ffma2_rn(ex, iL, M), nM), ex);
    ey = __ffma2_rn(nL, __fadd2_rn(__ffma2_rn(ey, iL, M), nM), ey);
    ez = __ffma2_rn(nL, __fadd2_rn(__ffma2_rn(ez, iL, M), nM), ez);
    const float2 r2 = __ffma2_rn(ex, ex, __ffma2_rn(ey, ey, __fmul2_rn(ez, ez)));
    const float2 rinv2 = make_float2(fast_rcp(r2.x), fast_rcp(r2.y));
    const float2 i6 = __fmul2_rn(__fmul2_rn(rinv2, rinv2), rinv2);
    float2 e = __fmul2_rn(A2, i6);
    if (R12) e = __fmul2_rn(e, i6);
    if (CUT) {
      e.x = (r2.x < cut2) ? e.x : 0.0f;
      e.y = (r2.y < cut2) ? e.y : 0.0f;
    }
    bool va = true, vb = true;
    if (MASK) {
      const int ja = jg + (q ^ r), jb = jg + ((q + 4) ^ r);
      va = ivalid && ja < jend && ja >= jlo && (unsigned)(ja - ex0) >= (unsigned)(ex1 - ex0);
      vb = ivalid && jb < jend && jb >= jlo && (unsigned)(jb - ex0) >= (unsigned)(ex1 - ex0);
      e.x = va ? e.x : 0.0f;
      e.y = vb ? e.y : 0.0f;
    }
    acc_e2 = __fadd2_rn(acc_e2, e);
    const float2 f = __fmul2_rn(__fmul2_rn(cf, e), rinv2);  // -(de/dr)/r
    float2 gx = __fmul2_rn(f, ex), gy = __fmul2_rn(f, ey), gz = __fmul2_rn(f, ez);
    if (MASK) {  // e = 0 can still meet rinv2 = inf (j = i, or stale coordinates)
      gx = make_float2(va ? gx.x : 0.0f, vb ? gx.y : 0.0f);
      gy = make_float2(va ? gy.x : 0.0f, vb ? gy.y : 0.0f);
      gz = make_float2(va ? gz.x : 0.0f, vb ? gz.y : 0.0f);
    }
    nfx = __fadd2_rn(nfx, gx);
    nfy = __fadd2_rn(nfy, gy);
    nfz = __fadd2_rn(nfz, gz);
    g[q][0] = gx.x;
    g[q][1] = gy.x;
    g[q][2] = gz.x;
    g[q + 4][0] = gx.y;
    g[q + 4][1] = gy.y;
    g[q + 4][2] = gz.y;
  }
  float h4[4][3];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) h4[q][c] = g[q][c] + __shfl_xor_sync(0xffffffffu, g[q + 4][c], 16);
  float h2[2][3];
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) h2[q][c] = h4[q][c] + __shfl_xor_sync(0xffffffffu, h4[q + 2][c], 8);
  float h1[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    h1[c] = h2[0][c] + __shfl_xor_sync(0xffffffffu, h2[1][c], 4);
    h1[c] += __shfl_xor_sync(0xffffffffu, h1[c], 2);
    h1[c] += __shfl_xor_sync(0xffffffffu, h1[c], 1);
  }
  if ((lane & 3) == 0 && jg + r < jend) {
    // force on j = sum over this warp's i beads of the negated pair forces
    s_fjw[jg + r][0] += h1[0];
    s_fjw[jg + r][1] += h1[1];
    s_fjw[jg + r][2] += h1[2];
  }
}

template <bool R12, bool CUT>
__global__ void __launch_bounds__(kTile, 8) adjoint_tile_kernel(
    const SysDev* __restrict__ sys, const int* __restrict__ inst_sys,
    const float4* __restrict__ pos, const float4* __restrict__ tab,
    const int* __restrict__ mol_start, const TileItem* __restrict__ items, int n_items,
    int* __restrict__ queue, float* __restrict__ forces, double* __restrict__ G,
    double* __restrict__ dxi, double* __restrict__ e_out, EnergyConsts K, AdjConsts C) {
  __shared__ float4 s_tab[kNT * kNT];
  __shared__ float4 s_j[kTile];
  __shared__ int s_it;  // the CTA's next item, from the work queue
  // the tile's crowder part [jc, jn) again, by coordinate, in groups of 8
  // from jc with beads q and q + 4 side by side: copy 0 in the order
  // (q, q + 4) for lanes 0-15, copy 1 in the order (q + 4, q) for lanes 16-31
  // (adjoint_group's bead order j = jg + (q ^ r), r = (lane >> 2) & 7, puts
  // the bead of the pair with the smaller index first for r < 4, last for
  // r >= 4). 8 entries of slack: a partial last group is stored, not read
  __shared__ __align__(16) float s_px[2][kTile + 8], s_py[2][kTile + 8], s_pz[2][kTile + 8];
  __shared__ float s_fj[kTile / 32][kTile][3];
  __shared__ float s_G[kNumAmino * kNumAmino];
  __shared__ double s_red[kTile / 32][2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < kNT * kNT; i += kTile) s_tab[i] = tab[i];
  // items come from a work queue over a list ordered by decreasing cost, so
  // the CTAs finish together (the outputs are sums of atomics: any item
  // order gives them)
  if (tid == 0) s_it = atomicAdd(queue, 1);
  for (;;) {
    __syncthreads();  // the previous item is done with the shared buffers; s_it is set
    const int it = s_it;
    if (it >= n_items) break;
    const TileItem W = items[it];
    const SysDev S = sys[inst_sys[W.inst]];
    const int N = S.n_beads;
    const int base = S.bead_base + (W.inst - S.inst0) * N;
    const float box = S.box, invbox = S.invbox;
    const int j0 = W.tj * kTile;
    const int jn = min(kTile, N - j0);
    const int jc = max(0, min(jn, S.n_chain_beads - j0));  // [0, jc) residues, [jc, jn) crowders
    if (tid < jn) {
      const float4 p = pos[base + j0 + tid];
      s_j[tid] = p;
      if (tid >= jc) {
        const int o = tid - jc, w = o & 7, g = (o & ~7) + 2 * (w & 3);
        const int p0 = g + (w >> 2), p1 = g + 1 - (w >> 2);
        s_px[0][p0] = p.x;
        s_py[0][p0] = p.y;
        s_pz[0][p0] = p.z;
        s_px[1][p1] = p.x;
        s_py[1][p1] = p.y;
        s_pz[1][p1] = p.z;
      }
    }
    for (int k = tid; k < (kTile / 32) * kTile * 3; k += kTile) (&s_fj[0][0][0])[k] = 0.0f;
    for (int k = tid; k < kNumAmino * kNumAmino; k += kTile) s_G[k] = 0.0f;
    __syncthreads();
    const int i = W.ti * kTile + tid;
    const bool ivalid = i < N;
    float4 pi = ivalid ? pos[base + i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int ta = bead_type(pi.w);
    const bool a_crowd = ta >= kNumAmino;
    // j (relative to j0) runs from jlo, leaving out the own molecule [ex0, ex1)
    const int jlo = (W.ti == W.tj) ? tid + 1 : 0;
    int ex0 = 0, ex1 = 0;
    if (ivalid) {
      const int mi = bead_mol(pi.w);
      ex0 = mol_start[S.mstart_off + mi] - j0;
      ex1 = mol_start[S.mstart_off + mi + 1] - j0;
    }
    const bool tc_fixed = S.crowd_type >= 0;
    const int half = lane >> 4;
    const float4 Tc = s_tab[(tc_fixed ? S.crowd_type : 0) * kNT + ta];
    float fx = 0.f, fy = 0.f, fz = 0.f, acc_e = 0.f, acc_x = 0.f;
    // packed crowder groups: negated force sums and energy, two pairs per lane
    float2 nfx = make_float2(0.f, 0.f), nfy = nfx, nfz = nfx, acc_e2 = nfx;
    const float2 npx = make_float2(-pi.x, -pi.x), npy = make_float2(-pi.y, -pi.y),
                 npz = make_float2(-pi.z, -pi.z);
    // a group needs no per-pair tests when, for every lane, it is full, past
    // the lane's first j and clear of its own molecule (a warp vote)
#define REMC_ADJ_GROUP(CHAIN_, jend_)                                                           \
  {                                                                                          \
    const bool clean = ivalid && jg + 8 <= (jend_) && jg >= jlo && (ex1 <= jg || ex0 >= jg + 8); \
    if (__all_sync(0xffffffffu, clean))                                                      \
      adjoint_group<R12, CUT, CHAIN_, false>(s_j, s_tab, s_G, s_fj[warp], jg, jend_, jlo, ex0, \
                                             ex1, ivalid, pi, ta, a_crowd, Tc, tc_fixed, box, \
                                             invbox, K, C, lane, fx, fy, fz, acc_e, acc_x);   \
    else                                                                                     \
      adjoint_group<R12, CUT, CHAIN_, true>(s_j, s_tab, s_G, s_fj[warp], jg, jend_, jlo, ex0, \
                                            ex1, ivalid, pi, ta, a_crowd, Tc, tc_fixed, box,  \
                                            invbox, K, C, lane, fx, fy, fz, acc_e, acc_x);    \
  }
    // in a diagonal tile every lane of warp w takes j > i >= 32 w: groups
    // wholly below that add nothing and are left out (warp-uniform starts,
    // group alignment kept: from 0 for residues, from jc for crowders)
    const int jmin = (W.ti == W.tj) ? 32 * warp + 1 : 0;
    const int jg_chain = (jmin >> 3) << 3;
    const int jg_crowd = jc + (jmin > jc ? ((jmin - jc) >> 3) << 3 : 0);
    for (int jg = jg_chain; jg < jc; jg += 8) REMC_ADJ_GROUP(true, jc)  // uniform trip counts
    if (tc_fixed) {
      for (int jg = jg_crowd; jg < jn; jg += 8) {
        const bool clean = ivalid && jg + 8 <= jn && jg >= jlo && (ex1 <= jg || ex0 >= jg + 8);
        if (__all_sync(0xffffffffu, clean))
          adjoint_group_crowd2<R12, CUT, false>(s_px[half] + (jg - jc), s_py[half] + (jg - jc),
                                                s_pz[half] + (jg - jc), s_fj[warp], jg, jn, npx,
                                                npy, npz, Tc.x, Tc.z, box, invbox, lane, nfx, nfy,
                                                nfz, acc_e2);
        else
          adjoint_group_crowd2<R12, CUT, true>(s_px[half] + (jg - jc), s_py[half] + (jg - jc),
                                               s_pz[half] + (jg - jc), s_fj[warp], jg, jn, npx,
                                               npy, npz, Tc.x, Tc.z, box, invbox, lane, nfx, nfy,
                                               nfz, acc_e2, ivalid, jlo, ex0, ex1);
      }
    } else {
      for (int jg = jg_crowd; jg < jn; jg += 8) REMC_ADJ_GROUP(false, jn)
    }
#undef REMC_ADJ_GROUP
    fx -= nfx.x + nfx.y;
    fy -= nfy.x + nfy.y;
    fz -= nfz.x + nfz.y;
    acc_e += acc_e2.x + acc_e2.y;
    double de = warp_sum((double)acc_e), dxv = warp_sum((double)acc_x);
    if (lane == 0) {
      s_red[warp][0] = de;
      s_red[warp][1] = dxv;
    }
    __syncthreads();
    if (ivalid) {
      atomicAdd(&forces[3 * (size_t)(base + i)], fx);
      atomicAdd(&forces[3 * (size_t)(base + i) + 1], fy);
      atomicAdd(&forces[3 * (size_t)(base + i) + 2], fz);
    }
    if (tid < jn) {
      float sx = 0.f, sy = 0.f, sz = 0.f;
      for (int w = 0; w < kTile / 32; ++w) {
        sx += s_fj[w][tid][0];
        sy += s_fj[w][tid][1];
        sz += s_fj[w][tid][2];
      }
      atomicAdd(&forces[3 * (size_t)(base + j0 + tid)], sx);
      atomicAdd(&forces[3 * (size_t)(base + j0 + tid) + 1], sy);
      atomicAdd(&forces[3 * (size_t)(base + j0 + tid) + 2], sz);
    }
    for (int k = tid; k < kNumAmino * kNumAmino; k += kTile)
      if (s_G[k] != 0.0f) atomicAdd(&G[(size_t)W.inst * kNumAmino * kNumAmino + k], (double)s_G[k]);
    if (tid == 0) {
      double e = 0.0, x = 0.0;
      for (int w = 0; w < kTile / 32; ++w) {
        e += s_red[w][0];
        x += s_red[w][1];
      }
      atomicAdd(&e_out[W.inst], e);
      atomicAdd(&dxi[W.inst], x * (double)C.inv_xi2);
      s_it = atomicAdd(queue, 1);  // every thread read s_it before this item's barriers
    }
  }
}

// Per-molecule force and torque about the centre (torque = sum rel x F):
// one thread per molecule, grid (instance, molecule chunk). A one-bead
// molecule is a copy widened to FP64; a chain's thread sums its beads in
// order (FP64). Memory-bound: forces, rel and the six doubles per molecule.
__global__ void __launch_bounds__(128) molecule_force_torque_kernel(
    const SysDev* __restrict__ sys, const int* __restrict__ inst_sys,
    const int* __restrict__ mol_start, const float4* __restrict__ rel,
    const float* __restrict__ forces, double* __restrict__ out) {
  const int inst = blockIdx.x;
  const SysDev S = sys[inst_sys[inst]];
  const int m = blockIdx.y * blockDim.x + threadIdx.x;
  if (m >= S.n_mol) return;
  const int slot = inst - S.inst0;
  const int base = S.bead_base + slot * S.n_beads;
  const int* ms = mol_start + S.mstart_off;
  const int a = ms[m], b = ms[m + 1];
  double fx = 0.0, fy = 0.0, fz = 0.0, tx = 0.0, ty = 0.0, tz = 0.0;
  for (int k = a; k < b; ++k) {
    const float4 rl = rel[base + k];
    const double Fx = forces[3 * (size_t)(base + k)], Fy = forces[3 * (size_t)(base + k) + 1],
                 Fz = forces[3 * (size_t)(base + k) + 2];
    fx += Fx;
    fy += Fy;
    fz += Fz;
    tx += (double)rl.y * Fz - (double)rl.z * Fy;
    ty += (double)rl.z * Fx - (double)rl.x * Fz;
    tz += (double)rl.x * Fy - (double)rl.y * Fx;
  }
  double2* o = reinterpret_cast<double2*>(out + 6 * (size_t)(S.mol_base + slot * S.n_mol + m));
  o[0] = make_double2(fx, fy);
  o[1] = make_double2(fz, tx);
  o[2] = make_double2(ty, tz);
}

// ------------------------------------------------------------------ exchange
__global__ void exchange_kernel(const SysDev* __restrict__ sys, const float* __restrict__ ladder,
                                const double* __restrict__ energy, int* __restrict__ temp_idx,
                                int* __restrict__ slot_of_temp, int* __restrict__ ex_tests,
                                int* __restrict__ ex_acc, const uint32_t* ctrl, uint32_t round_arg,
                                int offset_arg, uint32_t seed_lo, uint32_t seed_hi) {
  const int sysid = blockIdx.x;
  const SysDev S = sys[sysid];
  const int R = S.n_rep;
  const uint32_t round = ctrl ? ctrl[1] : round_arg;
  const int offset = ctrl ? (int)(ctrl[2] & 1u) : offset_arg;
  int tests = 0, accs = 0;
  for (int p = threadIdx.x; offset + 2 * p < R - 1; p += blockDim.x) {
    const int t = offset + 2 * p;
    const int a = slot_of_temp[S.inst0 + t], b = slot_of_temp[S.inst0 + t + 1];
    const double Ti = (double)ladder[S.inst0 + t], Tj = (double)ladder[S.inst0 + t + 1];
    const double delta = (1.0 / Ti - 1.0 / Tj) * (energy[S.inst0 + a] - energy[S.inst0 + b]) *
                         (double)(4184.0f / 8.314472f);
    uint4 x = philox4x32_10(make_uint4(round, (uint32_t)p, (uint32_t)sysid, 2u),
                            make_uint2(seed_lo, seed_hi));
    const double u = u32_unit(x.x);
    double pacc = exp(delta);
    if (pacc > 1.0) pacc = 1.0;
    ++tests;
    if (u < pacc) {
      ++accs;
      slot_of_temp[S.inst0 + t] = b;
      slot_of_temp[S.inst0 + t + 1] = a;
      temp_idx[S.inst0 + a] = t + 1;
      temp_idx[S.inst0 + b] = t;
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    tests += __shfl_down_sync(0xffffffffu, tests, off);
    accs += __shfl_down_sync(0xffffffffu, accs, off);
  }
  if (threadIdx.x == 0) {
    ex_tests[sysid] += tests;
    ex_acc[sysid] += accs;
  }
}

// Set the device step/round/offset counters from kernel arguments (stream
// ordered, no host copy).
__global__ void ctrl_set_kernel(uint32_t* ctrl, uint32_t step0, uint32_t round0) {
  ctrl[0] = step0;
  ctrl[1] = round0;
  ctrl[2] = round0 & 1u;
  ctrl[3] = 0u;
}

// Advance the device step/round/offset counters between graph replays.
__global__ void ctrl_advance_kernel(uint32_t* ctrl, uint32_t steps) {
  ctrl[0] += steps;
  ctrl[1] += 1u;
  ctrl[2] ^= 1u;
}

// ------------------------------------------------------------------ dE API
__global__ void delta_kernel(const SysDev* __restrict__ sys, const int* __restrict__ inst_sys,
                             const float4* __restrict__ pos, const float4* __restrict__ tab,
                             const int* __restrict__ mol_start, int inst, int mol,
                             const float4* __restrict__ newpos, double* __restrict__ out,
                             EnergyConsts K) {
  __shared__ double s_red[32];
  const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const SysDev S = sys[inst_sys[inst]];
  const int N = S.n_beads;
  const int base = S.bead_base + (inst - S.inst0) * N;
  const int m0 = mol_start[S.mstart_off + mol], n = mol_start[S.mstart_off + mol + 1] - m0;
  double dacc = 0.0;
  for (int k = 0; k < n; ++k) {
    const float4 pold = pos[base + m0 + k];
    float4 pnew = newpos[k];
    const int ta = bead_type(pold.w);
    float acc = 0.0f;
    for (int jj = tid; jj < N - n; jj += nthr) {
      const int j = jj < m0 ? jj : jj + n;
      const float4 pj = pos[base + j];
      const int tb = bead_type(pj.w);
      const float4 T = tab[ta * kNT + tb];
      const bool crowd = ta >= kNumAmino || tb >= kNumAmino;
      acc += pair_energy_r2(pair_r2(pnew, pj, S.box, S.invbox), T, crowd, K) -
             pair_energy_r2(pair_r2(pold, pj, S.box, S.invbox), T, crowd, K);
    }
    dacc += (double)acc;
  }
  dacc = warp_sum(dacc);
  if (lane == 0) s_red[warp] = dacc;
  __syncthreads();
  if (tid == 0) {
    double v = 0.0;
    for (int w = 0; w < nthr / 32; ++w) v += s_red[w];
    *out = v;
  }
}

}  // namespace

// =================================================================== host
struct remc_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  remc_params params{};
  int n_sys = 0, n_inst = 0;
  std::vector<SysDev> h_sys;
  std::vector<int> h_inst_sys;
  std::vector<int> h_mol_start;  // concatenated per system
  std::vector<int> h_mol_role;
  std::vector<int> h_bead_type;  // concatenated per system
  std::vector<int> h_bead_off_static;
  size_t total_beads = 0, total_mols = 0;
  int nmax = 0, mmax = 0, lmax = 0;
  // tables
  float vdw[kNT] = {}, charge[kNT] = {}, rho[kNT] = {};
  float pair_table[400] = {};
  bool tables_set = false, state_set = false, replica_params_set = false;
  // device
  SysDev* d_sys = nullptr;
  int* d_inst_sys = nullptr;
  int* d_inst_list = nullptr;
  long long* d_inst_cost = nullptr;  // per instance: cost of the current block of steps
  int* d_inst_order = nullptr;       // work order of the persistent sweep, by that cost
  int work_order = 1;                // 1: by the block's proposal costs; 0: static order
  float4* d_pos = nullptr;
  float4* d_rel = nullptr;
  float4* d_centre = nullptr;
  double* d_quat = nullptr;
  int* d_mol_start = nullptr;
  int* d_mol_role = nullptr;
  int* d_mrole_off = nullptr;
  StepRec* d_recs = nullptr;
  size_t recs_cap = 0;  // records per instance the buffer holds
  int recs_gen = 0;     // bumped on every reallocation (captured graphs hold the pointer)
  float4* d_tab = nullptr;
  double* d_energy = nullptr;
  int* d_temp_idx = nullptr;
  int* d_slot_of_temp = nullptr;
  float* d_ladder = nullptr;
  float* d_tstep = nullptr;
  double* d_rot_cs = nullptr;
  int* d_acc_neg = nullptr;
  int* d_acc_boltz = nullptr;
  int* d_rej = nullptr;
  unsigned long long* d_evals_kh = nullptr;
  unsigned long long* d_evals_crowd = nullptr;
  int* d_ex_tests = nullptr;
  int* d_ex_acc = nullptr;
  uint32_t* d_ctrl = nullptr;
  int* d_queue = nullptr;
  int sweep_grid = 0;  // resident CTAs of the persistent sweep
  int mol_in_smem = 1; // molecule centres/starts in shared memory (else global)
  int sweep_csize = 1; // CTAs per replica (thread-block cluster size)
  int sweep_cluster_slots = 0;  // clusters of that size the GPU holds at once
  int beads_in_smem = 1; // beads resident in shared memory (else updated in place in global)
  float4* d_trial_scratch = nullptr;  // sweep trial buffers, 6 lmax per (instance, CTA rank)
  float* d_fold_part = nullptr;       // per instance: the fold test's partial extents [8]
  size_t trial_scratch_cap = 0;       // float4 entries
  int max_dyn_smem = 0;
  int config_gen = 0;  // bumped when the sweep schedule changes
  TileItem* d_items_by_cost = nullptr;  // the items by decreasing cost (work-queue order)
  int* d_adj_queue = nullptr;  // in d_adj_acc
  int* d_energy_queue = nullptr;
  int* d_item_off = nullptr;
  double* d_scratch = nullptr;
  double* d_scratch_cc = nullptr;
  // adjoint accumulators, one allocation (made on first use) so that one
  // memset clears them all: forces, G, dxi, energy and the work counter
  unsigned char* d_adj_acc = nullptr;
  size_t adj_acc_bytes = 0;
  float* d_forces = nullptr;
  double* d_G = nullptr;
  double* d_dxi = nullptr;
  double* d_eadj = nullptr;
  double* d_mft = nullptr;
  double* d_ecc = nullptr;
  int* d_n_samples = nullptr;
  int* d_n_bound = nullptr;
  SampleHeader* d_sample_out = nullptr;
  SamplePose* d_pose_out = nullptr;
  unsigned* d_sample_cursor = nullptr;
  unsigned sample_cap = 0, pose_cap = 0;
  int sample_every = 0;
  uint32_t sample_after = 0;
  double bound_thr = -1.1844;
  int sample_gen = 0;  // bumped when sampling changes (captured graphs hold it)
  int n_items = 0;
  float4* d_newpos = nullptr;
  double* d_dE = nullptr;
  int* d_bead_info = nullptr;  // per bead per instance: meta word | (one-bead molecule << 31)
  float* d_stage = nullptr;    // host-layout staging: pos[3n], rel[3n], centre[3m]
  double* d_stage_q = nullptr; // quaternions [4m]
  unsigned long long* d_bad = nullptr;  // first invalid bead / one-bead offset / molecule
  int* d_err = nullptr;        // set by a kernel whose bounded wait gave up
  int sweep_threads = 128;
  int num_sms = 148;
  // graph
  cudaGraphExec_t graph_exec = nullptr;
  int graph_steps = -1;
  uint64_t graph_seed = 0;
  int graph_recs_gen = -1;
  int graph_sample_gen = -1;
  int graph_config_gen = -1;
};

namespace {

template <typename T>
int dev_alloc(T** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess)
    return set_error(REMC_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", n * sizeof(T),
                     cudaGetErrorString(e));
  return REMC_OK;
}

void free_all(remc_handle* h) {
  void* ptrs[] = {h->d_sys,      h->d_inst_sys,  h->d_inst_list,  h->d_inst_cost,  h->d_inst_order,
                  h->d_pos,        h->d_rel,
                  h->d_centre,   h->d_quat,      h->d_mol_start,  h->d_tab,        h->d_energy,
                  h->d_temp_idx, h->d_slot_of_temp, h->d_ladder,  h->d_tstep,      h->d_rot_cs,
                  h->d_acc_neg,  h->d_acc_boltz, h->d_rej,        h->d_ex_tests,   h->d_ex_acc,
                  h->d_evals_kh, h->d_evals_crowd, h->d_mol_role, h->d_mrole_off, h->d_recs,
                  h->d_queue,      h->d_scratch_cc, h->d_ecc,     h->d_n_samples,  h->d_n_bound,
                  h->d_sample_out, h->d_pose_out, h->d_sample_cursor, h->d_adj_acc,
                  h->d_mft,
                  h->d_ctrl,     h->d_items_by_cost, h->d_energy_queue,
                  h->d_item_off,   h->d_scratch,    h->d_newpos,
                  h->d_dE,       h->d_bead_info, h->d_stage,      h->d_stage_q,    h->d_bad,
                  h->d_err,      h->d_trial_scratch, h->d_fold_part};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  if (h->stream) cudaStreamDestroy(h->stream);
}

int build_tables(remc_handle* h) {
  const remc_params& P = h->params;
  std::vector<float4> tab(kNT * kNT);
  const float c_lj = (float)((double)P.lj_cf * (double)P.kbt_cf);
  const float c_dh = (float)((double)P.dh_const * (double)P.kbt_cf);
  const float two_third = 1.2599210498948732f;  // 2^(1/3): (2^(1/6) sigma)^2 = 2^(1/3) sigma^2
  for (int a = 0; a < kNT; ++a) {
    for (int b = 0; b < kNT; ++b) {
      float4 t;
      if (a < kNumAmino && b < kNumAmino) {
        // eps = lambda (M - e0) in FP32, as the reference evaluates it
        float eps = P.lambda_ * (h->pair_table[a * 20 + b] - P.e0);
        float epsc = eps * c_lj;
        float sig = 0.5f * (h->vdw[a] + h->vdw[b]);
        t.x = 4.0f * epsc;
        t.y = sig * sig;
        t.z = eps > 0.0f ? sig * sig * two_third : -1.0f;
        t.w = h->charge[a] * h->charge[b] * c_dh;
      } else {
        double A;
        if (P.crowder_mode == 0) {
          A = 46656.0 * (double)c_lj;  // (6/r)^6 = 46656 r^-6
        } else {
          double sg = (double)h->rho[a] + (double)h->rho[b];
          double s2 = sg * sg, s6 = s2 * s2 * s2;
          A = (double)P.crowder_eps * s6 * s6 * (double)c_lj;
        }
        t.x = (float)A;
        t.y = 0.0f;
        t.z = P.crowder_cutoff > 0.0f ? P.crowder_cutoff * P.crowder_cutoff : INFINITY;
        t.w = 0.0f;
      }
      tab[a * kNT + b] = t;
    }
  }
  REMC_CUDA_TRY(cudaMemcpyAsync(h->d_tab, tab.data(), sizeof(float4) * tab.size(),
                                cudaMemcpyHostToDevice, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return REMC_OK;
}

EnergyConsts consts_of(const remc_handle* h) {
  EnergyConsts K;
  K.c_xi = (float)(-1.4426950408889634 / (double)h->params.debye_length);
  K.crowder_mode = h->params.crowder_mode;
  K.crowder_cut = h->params.crowder_cutoff > 0.0f ? 1 : 0;
  return K;
}

// NVTX range over one API call, for timelines (a no-op unless a tool is attached).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Report (and clear) the error word a kernel sets when a bounded wait gives up.
int check_device_error(remc_handle* h) {
  int e = 0;
  REMC_CUDA_TRY(cudaMemcpyAsync(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (e) {
    REMC_CUDA_TRY(cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream));
    return set_error(REMC_ERR_TIMEOUT, "a device-side wait for a bulk copy gave up");
  }
  return REMC_OK;
}

int check_ready(const remc_handle* h) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (!h->tables_set) return set_error(REMC_ERR_STATE, "type tables not set");
  if (!h->state_set) return set_error(REMC_ERR_STATE, "state not uploaded");
  if (!h->replica_params_set) return set_error(REMC_ERR_STATE, "replica parameters not set");
  return REMC_OK;
}

// Grow the proposal-record buffer to hold `steps` records per instance.
int ensure_recs(remc_handle* h, size_t steps) {
  if (steps <= h->recs_cap) return REMC_OK;
  if (h->d_recs) {
    cudaStreamSynchronize(h->stream);
    cudaFree(h->d_recs);
    h->d_recs = nullptr;
    h->recs_cap = 0;
  }
  int rc = dev_alloc(&h->d_recs, steps * (size_t)h->n_inst);
  if (rc) return rc;
  h->recs_cap = steps;
  h->recs_gen++;
  return REMC_OK;
}

// The sweep kernel compiled for the handle's crowder model, single CTAs or
// clusters of CTAs per replica, beads in shared or in global memory.
using SweepFn = void (*)(SweepArgs);
template <bool CLUSTER, bool GB>
SweepFn sweep_fn_model(const remc_params& p) {
  const bool cut = p.crowder_cutoff > 0.0f;
  if (p.crowder_mode)
    return cut ? sweep_kernel<true, true, CLUSTER, GB> : sweep_kernel<true, false, CLUSTER, GB>;
  return cut ? sweep_kernel<false, true, CLUSTER, GB> : sweep_kernel<false, false, CLUSTER, GB>;
}
SweepFn sweep_fn(const remc_params& p, bool cluster, bool global_beads) {
  if (global_beads)
    return cluster ? sweep_fn_model<true, true>(p) : sweep_fn_model<false, true>(p);
  return cluster ? sweep_fn_model<true, false>(p) : sweep_fn_model<false, false>(p);
}

// Set the sweep schedule: threads per replica, where molecule data lives,
// CTAs per replica, and whether the beads are resident in shared memory.
int configure_sweep(remc_handle* h, int threads, int mol_in_smem, int csize, int beads_in_smem) {
  if (threads < 32 || threads > 256 || (threads & (threads - 1)) != 0)
    return set_error(REMC_ERR_INVALID, "threads per replica must be 32, 64, 128 or 256");
  if (csize != 1 && csize != 2 && csize != 4 && csize != 8)
    return set_error(REMC_ERR_INVALID, "cluster size must be 1, 2, 4 or 8");
  const size_t smem =
      SweepSmem::make(h->nmax, h->mmax, h->lmax, mol_in_smem, csize, beads_in_smem).total;
  if (smem > (size_t)h->max_dyn_smem)
    return set_error(REMC_ERR_INVALID,
                     "largest system needs %zu bytes of shared memory, device allows %d", smem,
                     h->max_dyn_smem);
  const SweepFn fn = sweep_fn(h->params, csize > 1, !beads_in_smem);
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
  if (e != cudaSuccess || per_sm < 1)
    return set_error(REMC_ERR_CUDA, "sweep kernel does not fit on an SM: %s",
                     cudaGetErrorString(e));
  if (csize > 1) {
    // the cluster must be schedulable: csize CTAs of this size in one GPC
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(csize);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    e = cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg);
    if (e != cudaSuccess || clusters < 1)
      return set_error(REMC_ERR_INVALID, "a cluster of %d sweep CTAs does not fit: %s", csize,
                       cudaGetErrorString(e));
    h->sweep_cluster_slots = clusters;
  }
  {
    // trial buffers of every (instance, CTA rank): 6 lmax float4 each (the
    // trial relative positions, and the trial positions when the beads stay
    // in global memory)
    const size_t need = (size_t)h->n_inst * csize * 6 * (size_t)h->lmax;
    if (need > h->trial_scratch_cap) {
      float4* p = nullptr;
      if (dev_alloc(&p, need)) return REMC_ERR_NOMEM;
      if (h->d_trial_scratch) {
        cudaStreamSynchronize(h->stream);
        cudaFree(h->d_trial_scratch);
      }
      h->d_trial_scratch = p;
      h->trial_scratch_cap = need;
    }
  }
  h->sweep_threads = threads;
  h->mol_in_smem = mol_in_smem;
  h->sweep_csize = csize;
  h->beads_in_smem = beads_in_smem;
  h->sweep_grid = per_sm * h->num_sms;
  h->config_gen++;
  return REMC_OK;
}

// Largest number of steps per launch whose records fit the buffer budget.
size_t max_chunk_steps(const remc_handle* h) {
  const size_t budget = (size_t)1 << 30;  // 1 GiB of proposal records
  size_t c = budget / (sizeof(StepRec) * (size_t)h->n_inst);
  return c < 64 ? 64 : c;
}

int launch_proposals(remc_handle* h, int n_steps, uint64_t seed, uint32_t step0,
                     const uint32_t* ctrl) {
  ProposalArgs P;
  P.sys = h->d_sys;
  P.inst_sys = h->d_inst_sys;
  P.mol_start = h->d_mol_start;
  P.mol_role = h->d_mol_role;
  P.mrole_off = h->d_mrole_off;
  P.tstep = h->d_tstep;
  P.rot_cs = h->d_rot_cs;
  P.ladder = h->d_ladder;
  P.temp_idx = h->d_temp_idx;
  P.recs = h->d_recs;
  P.ctrl = ctrl;
  P.step0 = step0;
  P.seed_lo = (uint32_t)seed;
  P.seed_hi = (uint32_t)(seed >> 32);
  P.n_inst = h->n_inst;
  P.n_steps = n_steps;
  P.rec_stride = (int)h->recs_cap;
  const long long total = (long long)h->n_inst * n_steps;
  const int grid = (int)((total + 255) / 256);
  proposal_kernel<<<grid, 256, 0, h->stream>>>(P);
  REMC_CUDA_TRY(cudaGetLastError());
  return REMC_OK;
}

int launch_sweep_kernel(remc_handle* h, int n_steps, int rec_offset, const int* inst_list,
                        int n_blocks, bool persistent, uint32_t step0, const uint32_t* ctrl) {
  SweepArgs A;
  A.sys = h->d_sys;
  A.inst_sys = h->d_inst_sys;
  A.inst_list = inst_list;
  // a cluster schedule runs one cluster per replica (no work queue); the
  // one-replica-per-launch path always runs single CTAs
  const int csize = persistent ? h->sweep_csize : 1;
  if (csize > 1) persistent = false;
  A.queue = persistent ? h->d_queue : nullptr;
  A.n_list = n_blocks;
  A.csize = csize;
  if (persistent) {
    REMC_CUDA_TRY(cudaMemsetAsync(h->d_queue, 0, sizeof(int), h->stream));
    n_blocks = std::min(n_blocks, h->sweep_grid);
  }
  A.pos = h->d_pos;
  A.rel = h->d_rel;
  A.centre = h->d_centre;
  A.quat = h->d_quat;
  A.mol_start = h->d_mol_start;
  A.tab = h->d_tab;
  A.recs = h->d_recs;
  A.energy = h->d_energy;
  A.ecc = h->d_ecc;
  A.temp_idx = h->d_temp_idx;
  A.ladder = h->d_ladder;
  A.sample_every = h->sample_every;
  A.sample_after = h->sample_after;
  A.bound_thr = h->bound_thr;
  A.ctrl = ctrl;
  A.step0 = step0;
  A.n_samples = h->d_n_samples;
  A.n_bound = h->d_n_bound;
  A.sample_out = h->d_sample_out;
  A.pose_out = h->d_pose_out;
  A.sample_cursor = h->d_sample_cursor;
  A.sample_cap = h->sample_cap;
  A.pose_cap = h->pose_cap;
  A.acc_neg = h->d_acc_neg;
  A.acc_boltz = h->d_acc_boltz;
  A.rej = h->d_rej;
  A.evals_kh = h->d_evals_kh;
  A.evals_crowd = h->d_evals_crowd;
  A.rec_stride = (int)h->recs_cap;
  A.rec_offset = rec_offset;
  A.n_steps = n_steps;
  A.nmax = h->nmax;
  A.mmax = h->mmax;
  A.mol_in_smem = h->mol_in_smem;
  A.lmax = h->lmax;
  A.trial_scratch = h->d_trial_scratch;
  A.K = consts_of(h);
  const bool gb = !h->beads_in_smem;
  const size_t smem =
      SweepSmem::make(h->nmax, h->mmax, h->lmax, h->mol_in_smem, csize, h->beads_in_smem).total;
  if (csize == 1) {
    sweep_fn(h->params, false, gb)<<<n_blocks, h->sweep_threads, smem, h->stream>>>(A);
  } else {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(csize * n_blocks);
    cfg.blockDim = dim3(h->sweep_threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = h->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    REMC_CUDA_TRY(cudaLaunchKernelEx(&cfg, sweep_fn(h->params, true, gb), A));
  }
  REMC_CUDA_TRY(cudaGetLastError());
  return REMC_OK;
}

// A step's fixed work (record, reductions, barrier, decision) in pair
// evaluations, per thread of the replica: about 1,500 pair evaluations at 256
// threads, from per-step clock64 timings of one-bead and chain steps on the
// 64-system batch (a step costs about 1,700 cycles plus 1.1 per pair there).
constexpr long long kStepCostPerThread = 6;

// The persistent sweep takes its work in cost order (remc_set_work_order).
bool uses_cost_order(const remc_handle* h) {
  return h->work_order == 1 && h->sweep_csize == 1 && h->n_inst > 1 &&
         h->n_inst <= kMaxRankedInst;
}

// Proposals then one persistent sweep over all instances, for n_steps steps
// (the record buffer must already hold n_steps records per instance).
int launch_sweep(remc_handle* h, int n_steps, uint64_t seed, uint32_t step0,
                 const uint32_t* ctrl) {
  int rc = launch_proposals(h, n_steps, seed, step0, ctrl);
  if (rc) return rc;
  // the work queue in decreasing order of what each replica's proposals cost
  // (single CTAs per replica: a cluster schedule runs every replica at once)
  const int* list = h->d_inst_list;
  if (uses_cost_order(h) && n_steps > 0) {
    block_cost_kernel<<<h->n_inst, 256, 0, h->stream>>>(
        h->d_sys, h->d_inst_sys, h->d_recs, (int)h->recs_cap, n_steps,
        kStepCostPerThread * (long long)h->sweep_threads, h->d_inst_cost);
    REMC_CUDA_TRY(cudaGetLastError());
    rank_kernel<<<(h->n_inst + 7) / 8, 256, 0, h->stream>>>(h->d_inst_cost, h->n_inst,
                                                             h->d_inst_order);
    REMC_CUDA_TRY(cudaGetLastError());
    list = h->d_inst_order;
  }
  return launch_sweep_kernel(h, n_steps, 0, list, h->n_inst, true, step0, ctrl);
}

}  // namespace

extern "C" {

void remc_default_params(remc_params* p) {
  if (!p) return;
  p->lambda_ = 0.159f;
  p->e0 = -2.27f;
  p->debye_length = 10.0f;
  p->dh_const = 0.948f * 1.602176487f * 1.602176487f;  // Replica.cpp:624 (float arithmetic)
  p->lj_cf = 0.3507221006079f;
  p->kbt_cf = 1.0f / (294.0f * 8.314472f / 4184.0f);
  p->crowder_mode = 0;
  p->crowder_cutoff = 15.0f;
  p->crowder_eps = 1.0f;
}

const char* remc_last_error_string(void) { return g_last_error.c_str(); }

int remc_create(const remc_system_desc* systems, int n_systems, const remc_params* params,
                remc_handle** out) {
  if (!out) return set_error(REMC_ERR_INVALID, "out is null");
  *out = nullptr;
  if (!systems || n_systems <= 0) return set_error(REMC_ERR_INVALID, "no systems");
  remc_handle* h = new (std::nothrow) remc_handle();
  if (!h) return set_error(REMC_ERR_NOMEM, "host allocation failed");
  if (params)
    h->params = *params;
  else
    remc_default_params(&h->params);
  // ---- validate and lay out
  size_t bead_cursor = 0, mol_cursor = 0;
  int inst_cursor = 0, mstart_cursor = 0;
  for (int s = 0; s < n_systems; ++s) {
    const remc_system_desc& d = systems[s];
    if (d.n_beads <= 0 || d.n_mol <= 0 || d.n_replicas <= 0 || !d.mol_start || !d.mol_role ||
        !d.bead_type || !(d.box > 0.0f) || !std::isfinite(d.box)) {
      delete h;
      return set_error(REMC_ERR_INVALID, "system %d: bad descriptor", s);
    }
    if (d.n_mol >= (1 << 22)) {
      delete h;
      return set_error(REMC_ERR_INVALID, "system %d: too many molecules", s);
    }
    if (d.mol_start[0] != 0 || d.mol_start[d.n_mol] != d.n_beads) {
      delete h;
      return set_error(REMC_ERR_INVALID, "system %d: mol_start must run 0..n_beads", s);
    }
    int lmax = 0;
    for (int m = 1; m < d.n_mol; ++m) {
      if (d.mol_role[m] == 0 && d.mol_role[m - 1] == -1) {
        delete h;
        return set_error(REMC_ERR_INVALID,
                         "system %d: chains must precede crowders (the reference's files "
                         "section precedes its crowders section)", s);
      }
    }
    for (int m = 0; m < d.n_mol; ++m) {
      int n = d.mol_start[m + 1] - d.mol_start[m];
      if (n <= 0) {
        delete h;
        return set_error(REMC_ERR_INVALID, "system %d: molecule %d is empty", s, m);
      }
      if (d.mol_role[m] != 0 && d.mol_role[m] != -1) {
        delete h;
        return set_error(REMC_ERR_INVALID, "system %d: molecule %d role must be 0 or -1", s, m);
      }
      for (int b = d.mol_start[m]; b < d.mol_start[m + 1]; ++b) {
        int t = d.bead_type[b];
        bool crowd_t = t >= kNumAmino;
        if (t < 0 || t >= kNT || crowd_t != (d.mol_role[m] == -1)) {
          delete h;
          return set_error(REMC_ERR_INVALID,
                           "system %d: bead %d type %d does not match molecule role", s, b, t);
        }
      }
      lmax = std::max(lmax, n);
    }
    SysDev S{};
    S.n_beads = d.n_beads;
    S.n_mol = d.n_mol;
    S.n_rep = d.n_replicas;
    S.lmax = lmax;
    S.inst0 = inst_cursor;
    S.bead_base = (int)bead_cursor;
    S.mol_base = (int)mol_cursor;
    S.mstart_off = mstart_cursor;
    S.box = d.box;
    S.invbox = 1.0f / d.box;
    S.translate_only_crowders = d.translate_only_crowders ? 1 : 0;
    S.n_chain_beads = 0;
    S.crowd_type = -1;
    bool mixed = false;
    for (int b = 0; b < d.n_beads; ++b) {
      const int t = d.bead_type[b];
      if (t < kNumAmino) {
        ++S.n_chain_beads;
      } else if (S.crowd_type < 0) {
        S.crowd_type = t;
      } else if (S.crowd_type != t) {
        mixed = true;
      }
    }
    if (mixed) S.crowd_type = -1;
    h->h_sys.push_back(S);
    for (int k = 0; k < d.n_replicas; ++k) h->h_inst_sys.push_back(s);
    h->h_mol_start.insert(h->h_mol_start.end(), d.mol_start, d.mol_start + d.n_mol + 1);
    h->h_mol_role.insert(h->h_mol_role.end(), d.mol_role, d.mol_role + d.n_mol);
    h->h_bead_off_static.push_back((int)h->h_bead_type.size());
    h->h_bead_type.insert(h->h_bead_type.end(), d.bead_type, d.bead_type + d.n_beads);
    bead_cursor += (size_t)d.n_beads * d.n_replicas;
    mol_cursor += (size_t)d.n_mol * d.n_replicas;
    inst_cursor += d.n_replicas;
    mstart_cursor += d.n_mol + 1;
    h->nmax = std::max(h->nmax, d.n_beads);
    h->mmax = std::max(h->mmax, d.n_mol);
    h->lmax = std::max(h->lmax, lmax);
  }
  if (bead_cursor >= (size_t)1 << 31) {
    delete h;
    return set_error(REMC_ERR_INVALID, "too many beads in one handle");
  }
  h->n_sys = n_systems;
  h->n_inst = inst_cursor;
  h->total_beads = bead_cursor;
  h->total_mols = mol_cursor;
  cudaError_t e = cudaGetDevice(&h->device);
  if (e != cudaSuccess) {
    delete h;
    return set_error(REMC_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  }
  int max_smem = 0;
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
  const SweepFn kSweeps[16] = {
      sweep_kernel<false, false, false, false>, sweep_kernel<false, true, false, false>,
      sweep_kernel<true, false, false, false>,  sweep_kernel<true, true, false, false>,
      sweep_kernel<false, false, true, false>,  sweep_kernel<false, true, true, false>,
      sweep_kernel<true, false, true, false>,   sweep_kernel<true, true, true, false>,
      sweep_kernel<false, false, false, true>,  sweep_kernel<false, true, false, true>,
      sweep_kernel<true, false, false, true>,   sweep_kernel<true, true, false, true>,
      sweep_kernel<false, false, true, true>,   sweep_kernel<false, true, true, true>,
      sweep_kernel<true, false, true, true>,    sweep_kernel<true, true, true, true>};
  int static_smem = 0;
  for (SweepFn f : kSweeps) {
    cudaFuncAttributes fattr;
    e = cudaFuncGetAttributes(&fattr, f);
    if (e != cudaSuccess) {
      delete h;
      return set_error(REMC_ERR_CUDA, "cudaFuncGetAttributes: %s", cudaGetErrorString(e));
    }
    static_smem = std::max(static_smem, (int)fattr.sharedSizeBytes);
  }
  const int max_dyn = max_smem - static_smem;
  h->max_dyn_smem = max_dyn;
  for (SweepFn f : kSweeps) {
    e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn);
    if (e != cudaSuccess) {
      delete h;
      return set_error(REMC_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    }
  }
  // default schedule (the autotuner may replace it): molecule data in shared
  // memory when it fits, more threads per replica for larger systems, and the
  // beads left in global memory for systems too large for shared memory
  {
    const int threads = h->nmax <= 2048 ? 128 : 256;
    int rc0 = configure_sweep(h, threads, 1, 1, 1);
    if (rc0) rc0 = configure_sweep(h, threads, 0, 1, 1);
    if (rc0) rc0 = configure_sweep(h, threads, 0, 1, 0);
    if (rc0) {
      delete h;
      return rc0;
    }
  }
  // ---- work list of the full-energy kernel (upper-triangle tiles)
  std::vector<TileItem> items;
  std::vector<int> item_off;
  for (int g = 0; g < h->n_inst; ++g) {
    item_off.push_back((int)items.size());
    const SysDev& S = h->h_sys[h->h_inst_sys[g]];
    int nt = (S.n_beads + kTile - 1) / kTile;
    for (int ti = 0; ti < nt; ++ti)
      for (int tj = ti; tj < nt; ++tj) items.push_back(TileItem{g, ti, tj, (int)items.size()});
  }
  item_off.push_back((int)items.size());
  h->n_items = (int)items.size();
  // the order of the energy and adjoint work queues: decreasing estimated
  // cost (pairs, residue pairs weighted up), stable
  std::vector<TileItem> items_by_cost(items);
  {
    auto cost = [&](const TileItem& W) {
      const SysDev& S = h->h_sys[h->h_inst_sys[W.inst]];
      const int N = S.n_beads, ncb = S.n_chain_beads;
      const long long in = std::min(kTile, N - W.ti * kTile), jn = std::min(kTile, N - W.tj * kTile);
      const long long ir = std::max(0, std::min((int)in, ncb - W.ti * kTile));
      const long long jr = std::max(0, std::min((int)jn, ncb - W.tj * kTile));
      const long long pairs = W.ti == W.tj ? in * (in - 1) / 2 : in * jn;
      const long long rr = W.ti == W.tj ? ir * (ir - 1) / 2 : ir * jr;
      return 2 * pairs + rr;
    };
    std::stable_sort(items_by_cost.begin(), items_by_cost.end(),
                     [&](const TileItem& a, const TileItem& b) { return cost(a) > cost(b); });
  }
  // ---- device memory
  int rc = REMC_OK;
  e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) rc = set_error(REMC_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
  std::vector<int> inst_list(h->n_inst);
  for (int g = 0; g < h->n_inst; ++g) inst_list[g] = g;
  // largest expected cost first (longest-processing-time order for the work
  // queue): expected pair evaluations per step = sum_m n_m (N - n_m) / M
  std::vector<double> sys_cost(h->n_sys, 0.0);
  for (int s2 = 0; s2 < h->n_sys; ++s2) {
    const SysDev& S = h->h_sys[s2];
    const int* ms = &h->h_mol_start[S.mstart_off];
    double c = 0.0;
    for (int m = 0; m < S.n_mol; ++m) {
      const double n = ms[m + 1] - ms[m];
      c += n * (S.n_beads - n);
    }
    sys_cost[s2] = c / S.n_mol + S.n_beads;  // + per-step bookkeeping
  }
  std::stable_sort(inst_list.begin(), inst_list.end(), [&](int a, int b) {
    return sys_cost[h->h_inst_sys[a]] > sys_cost[h->h_inst_sys[b]];
  });
  if (!rc) rc = dev_alloc(&h->d_sys, h->h_sys.size());
  if (!rc) rc = dev_alloc(&h->d_inst_sys, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_inst_list, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_inst_cost, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_inst_order, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_pos, h->total_beads);
  if (!rc) rc = dev_alloc(&h->d_bead_info, h->total_beads);
  if (!rc) rc = dev_alloc(&h->d_stage, 6 * h->total_beads + 3 * h->total_mols);
  if (!rc) rc = dev_alloc(&h->d_stage_q, 4 * h->total_mols);
  if (!rc) rc = dev_alloc(&h->d_bad, 3);
  if (!rc) rc = dev_alloc(&h->d_err, 1);
  if (!rc) rc = dev_alloc(&h->d_rel, h->total_beads);
  if (!rc) rc = dev_alloc(&h->d_centre, h->total_mols);
  if (!rc) rc = dev_alloc(&h->d_quat, 4 * h->total_mols);
  if (!rc) rc = dev_alloc(&h->d_mol_start, h->h_mol_start.size());
  if (!rc) rc = dev_alloc(&h->d_mol_role, h->h_mol_role.size());
  if (!rc) rc = dev_alloc(&h->d_mrole_off, h->n_sys);
  if (!rc) rc = dev_alloc(&h->d_tab, (size_t)kNT * kNT);
  if (!rc) rc = dev_alloc(&h->d_energy, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_temp_idx, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_slot_of_temp, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_ladder, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_tstep, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_rot_cs, 2 * (size_t)h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_acc_neg, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_acc_boltz, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_rej, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_evals_kh, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_evals_crowd, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_ex_tests, h->n_sys);
  if (!rc) rc = dev_alloc(&h->d_ex_acc, h->n_sys);
  if (!rc) rc = dev_alloc(&h->d_ctrl, 4);
  if (!rc) rc = dev_alloc(&h->d_queue, 1);
  if (!rc) rc = dev_alloc(&h->d_items_by_cost, items.size());
  if (!rc) rc = dev_alloc(&h->d_energy_queue, 1);
  if (!rc) rc = dev_alloc(&h->d_item_off, item_off.size());
  if (!rc) rc = dev_alloc(&h->d_scratch, items.size());
  if (!rc) rc = dev_alloc(&h->d_scratch_cc, items.size());
  if (!rc) rc = dev_alloc(&h->d_ecc, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_n_samples, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_n_bound, h->n_inst);
  if (!rc) rc = dev_alloc(&h->d_sample_cursor, 4);
  if (!rc) rc = dev_alloc(&h->d_newpos, h->lmax);
  if (!rc) rc = dev_alloc(&h->d_dE, 1);
  if (!rc) rc = dev_alloc(&h->d_fold_part, (size_t)h->n_inst * 8);
  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (rc) return;
    cudaError_t ee = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream);
    if (ee != cudaSuccess) rc = set_error(REMC_ERR_CUDA, "upload: %s", cudaGetErrorString(ee));
  };
  up(h->d_sys, h->h_sys.data(), sizeof(SysDev) * h->h_sys.size());
  up(h->d_inst_sys, h->h_inst_sys.data(), sizeof(int) * h->n_inst);
  up(h->d_inst_list, inst_list.data(), sizeof(int) * h->n_inst);
  up(h->d_mol_start, h->h_mol_start.data(), sizeof(int) * h->h_mol_start.size());
  up(h->d_mol_role, h->h_mol_role.data(), sizeof(int) * h->h_mol_role.size());
  std::vector<int> mrole_off(h->n_sys);
  for (int s2 = 0, off = 0; s2 < h->n_sys; ++s2) {
    mrole_off[s2] = off;
    off += h->h_sys[s2].n_mol;
  }
  up(h->d_mrole_off, mrole_off.data(), sizeof(int) * h->n_sys);
  up(h->d_items_by_cost, items_by_cost.data(), sizeof(TileItem) * items_by_cost.size());
  up(h->d_item_off, item_off.data(), sizeof(int) * item_off.size());
  // per bead per instance: the meta word of pos.w, and bit 31 for beads of
  // one-bead molecules (whose relative position must be zero)
  std::vector<int> bead_info(h->total_beads);
  for (int g = 0; g < h->n_inst; ++g) {
    const int s2 = h->h_inst_sys[g];
    const SysDev& S = h->h_sys[s2];
    const size_t b0 = (size_t)S.bead_base + (size_t)(g - S.inst0) * S.n_beads;
    const int* ms = &h->h_mol_start[S.mstart_off];
    const int* bt = &h->h_bead_type[h->h_bead_off_static[s2]];
    for (int m = 0; m < S.n_mol; ++m)
      for (int b = ms[m]; b < ms[m + 1]; ++b)
        bead_info[b0 + b] =
            pack_meta(m, bt[b]) | (ms[m + 1] - ms[m] == 1 ? (int)0x80000000u : 0);
  }
  up(h->d_bead_info, bead_info.data(), sizeof(int) * bead_info.size());
  if (!rc) {
    cudaMemsetAsync(h->d_acc_neg, 0, sizeof(int) * h->n_inst, h->stream);
    cudaMemsetAsync(h->d_acc_boltz, 0, sizeof(int) * h->n_inst, h->stream);
    cudaMemsetAsync(h->d_rej, 0, sizeof(int) * h->n_inst, h->stream);
    cudaMemsetAsync(h->d_evals_kh, 0, sizeof(unsigned long long) * h->n_inst, h->stream);
    cudaMemsetAsync(h->d_evals_crowd, 0, sizeof(unsigned long long) * h->n_inst, h->stream);
    cudaMemsetAsync(h->d_ex_tests, 0, sizeof(int) * h->n_sys, h->stream);
    cudaMemsetAsync(h->d_ex_acc, 0, sizeof(int) * h->n_sys, h->stream);
    cudaMemsetAsync(h->d_energy, 0, sizeof(double) * h->n_inst, h->stream);
    cudaMemsetAsync(h->d_ecc, 0, sizeof(double) * h->n_inst, h->stream);
    cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream);
    cudaMemsetAsync(h->d_n_samples, 0, sizeof(int) * h->n_inst, h->stream);
    cudaMemsetAsync(h->d_n_bound, 0, sizeof(int) * h->n_inst, h->stream);
    cudaMemsetAsync(h->d_sample_cursor, 0, sizeof(unsigned) * 4, h->stream);
    cudaMemsetAsync(h->d_ctrl, 0, sizeof(uint32_t) * 4, h->stream);
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = set_error(REMC_ERR_CUDA, "create sync: %s", cudaGetErrorString(e));
  }
  if (rc) {
    free_all(h);
    delete h;
    return rc;
  }
  *out = h;
  return REMC_OK;
}

int remc_destroy(remc_handle* h) {
  if (!h) return REMC_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_all(h);
  delete h;
  return REMC_OK;
}

int remc_set_params(remc_handle* h, const remc_params* p) {
  if (!h || !p) return set_error(REMC_ERR_INVALID, "null argument");
  if (!(p->debye_length > 0.0f) || (p->crowder_mode != 0 && p->crowder_mode != 1))
    return set_error(REMC_ERR_INVALID, "bad parameters");
  h->params = *p;
  h->config_gen++;  // a captured graph holds the old constants and kernel
  if (h->tables_set) return build_tables(h);
  return REMC_OK;
}

int remc_set_type_tables(remc_handle* h, const float* vdw, const float* charge, const float* rho,
                         const float* pair_table) {
  if (!h || !vdw || !charge || !rho || !pair_table)
    return set_error(REMC_ERR_INVALID, "null argument");
  memcpy(h->vdw, vdw, sizeof(h->vdw));
  memcpy(h->charge, charge, sizeof(h->charge));
  memcpy(h->rho, rho, sizeof(h->rho));
  memcpy(h->pair_table, pair_table, sizeof(h->pair_table));
  int rc = build_tables(h);
  if (rc == REMC_OK) h->tables_set = true;
  return rc;
}

int remc_upload_state(remc_handle* h, const float* pos, const float* rel, const float* centre,
                      const double* quat) {
  NvtxRange nvtx_range("remc_upload_state");
  if (!h || !pos || !rel || !centre || !quat) return set_error(REMC_ERR_INVALID, "null argument");
  const size_t nb = h->total_beads, nm = h->total_mols;
  float* sp = h->d_stage;
  float* sr = sp + 3 * nb;
  float* sc = sr + 3 * nb;
  // the caller's buffers go to staging as they are; the state changes only
  // after every coordinate has been checked
  REMC_CUDA_TRY(cudaMemcpyAsync(sp, pos, sizeof(float) * 3 * nb, cudaMemcpyHostToDevice, h->stream));
  REMC_CUDA_TRY(cudaMemcpyAsync(sr, rel, sizeof(float) * 3 * nb, cudaMemcpyHostToDevice, h->stream));
  REMC_CUDA_TRY(cudaMemcpyAsync(sc, centre, sizeof(float) * 3 * nm, cudaMemcpyHostToDevice,
                                h->stream));
  REMC_CUDA_TRY(cudaMemcpyAsync(h->d_stage_q, quat, sizeof(double) * 4 * nm,
                                cudaMemcpyHostToDevice, h->stream));
  REMC_CUDA_TRY(cudaMemsetAsync(h->d_bad, 0x7f, sizeof(unsigned long long) * 3, h->stream));
  const int grid = h->num_sms * 4;
  state_check_kernel<<<grid, 256, 0, h->stream>>>(sp, sr, sc, h->d_bead_info, (long long)nb,
                                                  (long long)nm, h->d_bad);
  REMC_CUDA_TRY(cudaGetLastError());
  unsigned long long bad[3];
  REMC_CUDA_TRY(cudaMemcpyAsync(bad, h->d_bad, sizeof(bad), cudaMemcpyDeviceToHost, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  const unsigned long long none = 0x7f7f7f7f7f7f7f7full;
  if (bad[0] != none || bad[1] != none || bad[2] != none) {
    // name the instance and bead / molecule of the first offender
    for (int g = 0; g < h->n_inst; ++g) {
      const SysDev& S = h->h_sys[h->h_inst_sys[g]];
      const unsigned long long b0 =
          (unsigned long long)S.bead_base + (unsigned long long)(g - S.inst0) * S.n_beads;
      const unsigned long long m0 =
          (unsigned long long)S.mol_base + (unsigned long long)(g - S.inst0) * S.n_mol;
      if (bad[2] != none && bad[2] >= m0 && bad[2] < m0 + S.n_mol)
        return set_error(REMC_ERR_NUMERIC, "instance %d molecule %d: non-finite centre", g,
                         (int)(bad[2] - m0));
      if (bad[0] != none && bad[0] >= b0 && bad[0] < b0 + S.n_beads)
        return set_error(REMC_ERR_NUMERIC, "instance %d bead %d: non-finite coordinate", g,
                         (int)(bad[0] - b0));
      if (bad[1] != none && bad[1] >= b0 && bad[1] < b0 + S.n_beads)
        return set_error(REMC_ERR_INVALID,
                         "instance %d bead %d: a one-bead molecule must sit at its centre", g,
                         (int)(bad[1] - b0));
    }
    return set_error(REMC_ERR_INVALID, "invalid state");
  }
  state_pack_kernel<<<grid, 256, 0, h->stream>>>(sp, sr, sc, h->d_bead_info, (long long)nb,
                                                 (long long)nm, h->d_pos, h->d_rel, h->d_centre);
  REMC_CUDA_TRY(cudaGetLastError());
  fold_part_kernel<<<h->n_inst, 256, 0, h->stream>>>(h->d_sys, h->d_inst_sys, h->d_pos,
                                                     h->d_rel, h->d_fold_part);
  REMC_CUDA_TRY(cudaGetLastError());
  fold_flag_kernel<<<h->n_sys, 256, 0, h->stream>>>(h->d_sys, h->d_fold_part);
  REMC_CUDA_TRY(cudaGetLastError());
  REMC_CUDA_TRY(cudaMemcpyAsync(h->d_quat, h->d_stage_q, sizeof(double) * 4 * nm,
                                cudaMemcpyDeviceToDevice, h->stream));
  h->state_set = true;
  return REMC_OK;
}

int remc_download_state(remc_handle* h, float* pos, float* rel, float* centre, double* quat) {
  NvtxRange nvtx_range("remc_download_state");
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (!h->state_set) return set_error(REMC_ERR_STATE, "state not uploaded");
  const size_t nb = h->total_beads, nm = h->total_mols;
  float* sp = h->d_stage;
  float* sr = sp + 3 * nb;
  float* sc = sr + 3 * nb;
  state_unpack_kernel<<<h->num_sms * 4, 256, 0, h->stream>>>(h->d_pos, h->d_rel, h->d_centre,
                                                             (long long)nb, (long long)nm, sp, sr,
                                                             sc);
  REMC_CUDA_TRY(cudaGetLastError());
  if (pos)
    REMC_CUDA_TRY(cudaMemcpyAsync(pos, sp, sizeof(float) * 3 * nb, cudaMemcpyDeviceToHost,
                                  h->stream));
  if (rel)
    REMC_CUDA_TRY(cudaMemcpyAsync(rel, sr, sizeof(float) * 3 * nb, cudaMemcpyDeviceToHost,
                                  h->stream));
  if (centre)
    REMC_CUDA_TRY(cudaMemcpyAsync(centre, sc, sizeof(float) * 3 * nm, cudaMemcpyDeviceToHost,
                                  h->stream));
  if (quat)
    REMC_CUDA_TRY(cudaMemcpyAsync(quat, h->d_quat, sizeof(double) * 4 * nm,
                                  cudaMemcpyDeviceToHost, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return REMC_OK;
}

int remc_set_replica_params(remc_handle* h, const float* ladder, const float* tstep,
                            const double* rstep) {
  if (!h || !ladder || !tstep || !rstep) return set_error(REMC_ERR_INVALID, "null argument");
  std::vector<int> ti(h->n_inst);
  std::vector<double> cs(2 * (size_t)h->n_inst);
  for (int g = 0; g < h->n_inst; ++g) {
    const SysDev& S = h->h_sys[h->h_inst_sys[g]];
    if (!(ladder[g] > 0.0f) || !std::isfinite(ladder[g]))
      return set_error(REMC_ERR_INVALID, "instance %d: temperature must be positive", g);
    if (g > S.inst0 && !(ladder[g] >= ladder[g - 1]))
      return set_error(REMC_ERR_INVALID, "ladder must be non-decreasing within a system");
    ti[g] = g - S.inst0;
    // Molecule::rotateQ evaluates sin/cos(angle/2.0) in FP64 (Molecule.cpp:290-291)
    cs[2 * g] = cos(rstep[g] / 2.0);
    cs[2 * g + 1] = sin(rstep[g] / 2.0);
  }
  REMC_CUDA_TRY(cudaMemcpyAsync(h->d_ladder, ladder, sizeof(float) * h->n_inst,
                                cudaMemcpyHostToDevice, h->stream));
  REMC_CUDA_TRY(cudaMemcpyAsync(h->d_tstep, tstep, sizeof(float) * h->n_inst,
                                cudaMemcpyHostToDevice, h->stream));
  REMC_CUDA_TRY(cudaMemcpyAsync(h->d_rot_cs, cs.data(), sizeof(double) * cs.size(),
                                cudaMemcpyHostToDevice, h->stream));
  REMC_CUDA_TRY(cudaMemcpyAsync(h->d_temp_idx, ti.data(), sizeof(int) * h->n_inst,
                                cudaMemcpyHostToDevice, h->stream));
  // slot_of_temp is the identity at start (temperature index t held by slot t)
  REMC_CUDA_TRY(cudaMemcpyAsync(h->d_slot_of_temp, ti.data(), sizeof(int) * h->n_inst,
                                cudaMemcpyHostToDevice, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->replica_params_set = true;
  return REMC_OK;
}

int remc_energy_full(remc_handle* h, double* out) {
  NvtxRange nvtx_range("remc_energy_full");
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (!h->tables_set || !h->state_set) return set_error(REMC_ERR_STATE, "tables/state not set");
  int grid = std::min(h->n_items, h->num_sms * 8);
  REMC_CUDA_TRY(cudaMemsetAsync(h->d_energy_queue, 0, sizeof(int), h->stream));
  energy_tile_kernel<<<grid, kTile, 0, h->stream>>>(
      h->d_sys, h->d_inst_sys, h->d_pos, h->d_tab, h->d_mol_start, h->d_items_by_cost,
      h->n_items, h->d_energy_queue, h->d_scratch, h->d_scratch_cc, consts_of(h), h->d_err);
  REMC_CUDA_TRY(cudaGetLastError());
  energy_reduce_kernel<<<(h->n_inst + 7) / 8, 256, 0, h->stream>>>(
      h->d_item_off, h->n_inst, h->d_scratch, h->d_scratch_cc, h->d_energy, h->d_ecc);
  REMC_CUDA_TRY(cudaGetLastError());
  if (out) {
    REMC_CUDA_TRY(cudaMemcpyAsync(out, h->d_energy, sizeof(double) * h->n_inst,
                                  cudaMemcpyDeviceToHost, h->stream));
    return check_device_error(h);
  }
  return REMC_OK;
}

int remc_get_energies(remc_handle* h, double* out) {
  if (!h || !out) return set_error(REMC_ERR_INVALID, "null argument");
  REMC_CUDA_TRY(cudaMemcpyAsync(out, h->d_energy, sizeof(double) * h->n_inst,
                                cudaMemcpyDeviceToHost, h->stream));
  return check_device_error(h);
}

int remc_sweep(remc_handle* h, int n_steps, uint64_t seed, uint32_t step0) {
  NvtxRange nvtx_range("remc_sweep");
  int rc = check_ready(h);
  if (rc) return rc;
  if (n_steps < 0) return set_error(REMC_ERR_INVALID, "n_steps < 0");
  const size_t chunk_max = max_chunk_steps(h);
  for (int done = 0; done < n_steps;) {
    const int chunk = (int)std::min((size_t)(n_steps - done), chunk_max);
    rc = ensure_recs(h, (size_t)chunk);
    if (rc) return rc;
    rc = launch_sweep(h, chunk, seed, step0 + (uint32_t)done, nullptr);
    if (rc) return rc;
    done += chunk;
  }
  return REMC_OK;
}

int remc_sweep_plain(remc_handle* h, int n_steps, uint64_t seed, uint32_t step0) {
  NvtxRange nvtx_range("remc_sweep_plain");
  int rc = check_ready(h);
  if (rc) return rc;
  if (n_steps < 0) return set_error(REMC_ERR_INVALID, "n_steps < 0");
  const size_t chunk_max = max_chunk_steps(h);
  for (int done = 0; done < n_steps;) {
    const int chunk = (int)std::min((size_t)(n_steps - done), chunk_max);
    rc = ensure_recs(h, (size_t)chunk);
    if (rc) return rc;
    rc = launch_proposals(h, chunk, seed, step0 + (uint32_t)done, nullptr);
    if (rc) return rc;
    for (int s = 0; s < chunk; ++s) {
      for (int g = 0; g < h->n_inst; ++g) {
        // one single-CTA launch per replica per step; d_inst_list + g names one
        // instance (instances are independent within a step, so order is free)
        rc = launch_sweep_kernel(h, 1, s, h->d_inst_list + g, 1, false,
                                 step0 + (uint32_t)(done + s), nullptr);
        if (rc) return rc;
      }
    }
    done += chunk;
  }
  return REMC_OK;
}

int remc_exchange(remc_handle* h, uint64_t seed, uint32_t round, int offset) {
  NvtxRange nvtx_range("remc_exchange");
  int rc = check_ready(h);
  if (rc) return rc;
  if (offset != 0 && offset != 1) return set_error(REMC_ERR_INVALID, "offset must be 0 or 1");
  exchange_kernel<<<h->n_sys, 32, 0, h->stream>>>(h->d_sys, h->d_ladder, h->d_energy,
                                                  h->d_temp_idx, h->d_slot_of_temp,
                                                  h->d_ex_tests, h->d_ex_acc, nullptr, round,
                                                  offset, (uint32_t)seed, (uint32_t)(seed >> 32));
  REMC_CUDA_TRY(cudaGetLastError());
  return REMC_OK;
}

int remc_get_temperature_map(remc_handle* h, int* temp_of_slot) {
  if (!h || !temp_of_slot) return set_error(REMC_ERR_INVALID, "null argument");
  REMC_CUDA_TRY(cudaMemcpyAsync(temp_of_slot, h->d_temp_idx, sizeof(int) * h->n_inst,
                                cudaMemcpyDeviceToHost, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return REMC_OK;
}

int remc_set_temperature_map(remc_handle* h, const int* temp_of_slot) {
  if (!h || !temp_of_slot) return set_error(REMC_ERR_INVALID, "null argument");
  if (!h->replica_params_set) return set_error(REMC_ERR_STATE, "replica parameters not set");
  std::vector<int> slot_of(h->n_inst, -1);
  for (int s = 0; s < h->n_sys; ++s) {
    const SysDev& S = h->h_sys[s];
    for (int k = 0; k < S.n_rep; ++k) {
      const int t = temp_of_slot[S.inst0 + k];
      if (t < 0 || t >= S.n_rep || slot_of[S.inst0 + t] >= 0)
        return set_error(REMC_ERR_INVALID,
                         "system %d: temperature map is not a permutation of 0..%d", s,
                         S.n_rep - 1);
      slot_of[S.inst0 + t] = k;
    }
  }
  REMC_CUDA_TRY(cudaMemcpyAsync(h->d_temp_idx, temp_of_slot, sizeof(int) * h->n_inst,
                                cudaMemcpyHostToDevice, h->stream));
  REMC_CUDA_TRY(cudaMemcpyAsync(h->d_slot_of_temp, slot_of.data(), sizeof(int) * h->n_inst,
                                cudaMemcpyHostToDevice, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return REMC_OK;
}

int remc_set_energies(remc_handle* h, const double* energy, const double* noncrowder) {
  if (!h || !energy) return set_error(REMC_ERR_INVALID, "null argument");
  for (int g = 0; g < h->n_inst; ++g)
    if (!std::isfinite(energy[g]) || (noncrowder && !std::isfinite(noncrowder[g])))
      return set_error(REMC_ERR_NUMERIC, "instance %d: non-finite energy", g);
  REMC_CUDA_TRY(cudaMemcpyAsync(h->d_energy, energy, sizeof(double) * h->n_inst,
                                cudaMemcpyHostToDevice, h->stream));
  if (noncrowder)
    REMC_CUDA_TRY(cudaMemcpyAsync(h->d_ecc, noncrowder, sizeof(double) * h->n_inst,
                                  cudaMemcpyHostToDevice, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return REMC_OK;
}

int remc_get_counters(remc_handle* h, int* accept, int* acceptA, int* reject) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (accept)
    REMC_CUDA_TRY(cudaMemcpyAsync(accept, h->d_acc_neg, sizeof(int) * h->n_inst,
                                  cudaMemcpyDeviceToHost, h->stream));
  if (acceptA)
    REMC_CUDA_TRY(cudaMemcpyAsync(acceptA, h->d_acc_boltz, sizeof(int) * h->n_inst,
                                  cudaMemcpyDeviceToHost, h->stream));
  if (reject)
    REMC_CUDA_TRY(cudaMemcpyAsync(reject, h->d_rej, sizeof(int) * h->n_inst,
                                  cudaMemcpyDeviceToHost, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return REMC_OK;
}

int remc_reset_counters(remc_handle* h) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  REMC_CUDA_TRY(cudaMemsetAsync(h->d_acc_neg, 0, sizeof(int) * h->n_inst, h->stream));
  REMC_CUDA_TRY(cudaMemsetAsync(h->d_acc_boltz, 0, sizeof(int) * h->n_inst, h->stream));
  REMC_CUDA_TRY(cudaMemsetAsync(h->d_rej, 0, sizeof(int) * h->n_inst, h->stream));
  REMC_CUDA_TRY(cudaMemsetAsync(h->d_evals_kh, 0, sizeof(unsigned long long) * h->n_inst,
                                h->stream));
  REMC_CUDA_TRY(cudaMemsetAsync(h->d_evals_crowd, 0, sizeof(unsigned long long) * h->n_inst,
                                h->stream));
  REMC_CUDA_TRY(cudaMemsetAsync(h->d_n_samples, 0, sizeof(int) * h->n_inst, h->stream));
  REMC_CUDA_TRY(cudaMemsetAsync(h->d_n_bound, 0, sizeof(int) * h->n_inst, h->stream));
  return REMC_OK;
}

int remc_set_sampling(remc_handle* h, int sample_every, uint32_t sample_after,
                      double bound_threshold, int max_records, int max_poses) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (sample_every < 0 || max_records < 0 || max_poses < 0)
    return set_error(REMC_ERR_INVALID, "negative sampling argument");
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if ((unsigned)max_records != h->sample_cap || (unsigned)max_poses != h->pose_cap) {
    if (h->d_sample_out) cudaFree(h->d_sample_out);
    if (h->d_pose_out) cudaFree(h->d_pose_out);
    h->d_sample_out = nullptr;
    h->d_pose_out = nullptr;
    h->sample_cap = h->pose_cap = 0;
    if (max_records > 0 && max_poses > 0) {
      int rc = dev_alloc(&h->d_sample_out, (size_t)max_records);
      if (!rc) rc = dev_alloc(&h->d_pose_out, (size_t)max_poses);
      if (rc) return rc;
      h->sample_cap = (unsigned)max_records;
      h->pose_cap = (unsigned)max_poses;
    }
  }
  h->sample_every = sample_every;
  h->sample_after = sample_after;
  h->bound_thr = bound_threshold;
  h->sample_gen++;
  REMC_CUDA_TRY(cudaMemsetAsync(h->d_sample_cursor, 0, sizeof(unsigned) * 4, h->stream));
  return REMC_OK;
}

int remc_get_sample_counters(remc_handle* h, int* samples, int* bound) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (samples)
    REMC_CUDA_TRY(cudaMemcpyAsync(samples, h->d_n_samples, sizeof(int) * h->n_inst,
                                  cudaMemcpyDeviceToHost, h->stream));
  if (bound)
    REMC_CUDA_TRY(cudaMemcpyAsync(bound, h->d_n_bound, sizeof(int) * h->n_inst,
                                  cudaMemcpyDeviceToHost, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return REMC_OK;
}

int remc_read_samples(remc_handle* h, remc_sample* records, int max_records,
                      remc_sample_pose* poses, int max_poses, int* n_records, int* n_poses,
                      int* n_dropped) {
  if (!h || !n_records || !n_poses) return set_error(REMC_ERR_INVALID, "null argument");
  unsigned cur[4] = {0, 0, 0, 0};
  REMC_CUDA_TRY(cudaMemcpyAsync(cur, h->d_sample_cursor, sizeof(cur), cudaMemcpyDeviceToHost,
                                h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  const unsigned nr = std::min(cur[0], h->sample_cap);
  // poses of the records kept (a reservation that did not fit wrote nothing)
  std::vector<SampleHeader> hd(nr);
  if (nr)
    REMC_CUDA_TRY(cudaMemcpyAsync(hd.data(), h->d_sample_out, sizeof(SampleHeader) * nr,
                                  cudaMemcpyDeviceToHost, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  unsigned np = 0;
  for (unsigned i = 0; i < nr; ++i) np = std::max(np, hd[i].pose_offset + (unsigned)hd[i].n_mol);
  if ((int)nr > max_records || (int)np > max_poses)
    return set_error(REMC_ERR_INVALID, "output buffers too small: need %u records, %u poses",
                     nr, np);
  for (unsigned i = 0; i < nr; ++i) {
    records[i].inst = hd[i].inst;
    records[i].label = hd[i].label;
    records[i].e_noncrowder = hd[i].e_nc;
    records[i].e_total = hd[i].e;
    records[i].temperature = hd[i].temperature;
    records[i].n_mol = hd[i].n_mol;
    records[i].pose_offset = (int)hd[i].pose_offset;
  }
  if (np) {
    std::vector<SamplePose> ps(np);
    REMC_CUDA_TRY(cudaMemcpyAsync(ps.data(), h->d_pose_out, sizeof(SamplePose) * np,
                                  cudaMemcpyDeviceToHost, h->stream));
    REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (unsigned i = 0; i < np; ++i) {
      for (int k = 0; k < 4; ++k) poses[i].q[k] = ps[i].q[k];
      for (int k = 0; k < 3; ++k) poses[i].centre[k] = ps[i].c[k];
    }
  }
  *n_records = (int)nr;
  *n_poses = (int)np;
  if (n_dropped) *n_dropped = (int)cur[2] + (int)(cur[0] - nr);
  REMC_CUDA_TRY(cudaMemsetAsync(h->d_sample_cursor, 0, sizeof(unsigned) * 4, h->stream));
  return REMC_OK;
}

int remc_energy_adjoint(remc_handle* h, float* forces, double* mol_force_torque,
                        double* dE_dlambda, double* dE_dxi, double* dE_deps, double* energy) {
  NvtxRange nvtx_range("remc_energy_adjoint");
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (!h->tables_set || !h->state_set) return set_error(REMC_ERR_STATE, "tables/state not set");
  int rc = REMC_OK;
  if (!h->d_adj_acc) {
    // forces first, every part on a 256-byte boundary
    auto up256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t nG = (size_t)kNumAmino * kNumAmino * h->n_inst;
    const size_t off_f = 0;
    const size_t off_G = up256(off_f + sizeof(float) * 3 * h->total_beads);
    const size_t off_dxi = up256(off_G + sizeof(double) * nG);
    const size_t off_e = up256(off_dxi + sizeof(double) * h->n_inst);
    const size_t off_q = up256(off_e + sizeof(double) * h->n_inst);
    h->adj_acc_bytes = off_q + 16;
    rc = dev_alloc(&h->d_adj_acc, h->adj_acc_bytes);
    if (!rc) rc = dev_alloc(&h->d_mft, 6 * h->total_mols);
    if (rc) return rc;
    h->d_G = reinterpret_cast<double*>(h->d_adj_acc + off_G);
    h->d_dxi = reinterpret_cast<double*>(h->d_adj_acc + off_dxi);
    h->d_eadj = reinterpret_cast<double*>(h->d_adj_acc + off_e);
    h->d_adj_queue = reinterpret_cast<int*>(h->d_adj_acc + off_q);
    h->d_forces = reinterpret_cast<float*>(h->d_adj_acc + off_f);
  }
  REMC_CUDA_TRY(cudaMemsetAsync(h->d_adj_acc, 0, h->adj_acc_bytes, h->stream));
  AdjConsts C;
  C.inv_xi = 1.0f / h->params.debye_length;
  C.inv_xi2 = C.inv_xi * C.inv_xi;
  C.c_lj = (float)((double)h->params.lj_cf * (double)h->params.kbt_cf);
  const bool cut = h->params.crowder_cutoff > 0.0f;
  auto adj = h->params.crowder_mode ? (cut ? adjoint_tile_kernel<true, true>
                                           : adjoint_tile_kernel<true, false>)
                                    : (cut ? adjoint_tile_kernel<false, true>
                                           : adjoint_tile_kernel<false, false>);
  // a persistent grid: as many CTAs as fit on the GPU at once
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adj, kTile, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 8;
  const int grid = std::min(h->n_items, h->num_sms * per_sm);
  adj<<<grid, kTile, 0, h->stream>>>(h->d_sys, h->d_inst_sys, h->d_pos, h->d_tab, h->d_mol_start,
                                     h->d_items_by_cost, h->n_items, h->d_adj_queue, h->d_forces,
                                     h->d_G, h->d_dxi, h->d_eadj, consts_of(h), C);
  REMC_CUDA_TRY(cudaGetLastError());
  molecule_force_torque_kernel<<<dim3(h->n_inst, (h->mmax + 127) / 128), 128, 0, h->stream>>>(
      h->d_sys, h->d_inst_sys, h->d_mol_start, h->d_rel, h->d_forces, h->d_mft);
  REMC_CUDA_TRY(cudaGetLastError());
  if (forces)
    REMC_CUDA_TRY(cudaMemcpyAsync(forces, h->d_forces, sizeof(float) * 3 * h->total_beads,
                                  cudaMemcpyDeviceToHost, h->stream));
  if (mol_force_torque)
    REMC_CUDA_TRY(cudaMemcpyAsync(mol_force_torque, h->d_mft, sizeof(double) * 6 * h->total_mols,
                                  cudaMemcpyDeviceToHost, h->stream));
  if (dE_dxi)
    REMC_CUDA_TRY(cudaMemcpyAsync(dE_dxi, h->d_dxi, sizeof(double) * h->n_inst,
                                  cudaMemcpyDeviceToHost, h->stream));
  if (energy)
    REMC_CUDA_TRY(cudaMemcpyAsync(energy, h->d_eadj, sizeof(double) * h->n_inst,
                                  cudaMemcpyDeviceToHost, h->stream));
  std::vector<double> G;
  if (dE_deps || dE_dlambda) {
    G.resize((size_t)kNumAmino * kNumAmino * h->n_inst);
    REMC_CUDA_TRY(cudaMemcpyAsync(G.data(), h->d_G, sizeof(double) * G.size(),
                                  cudaMemcpyDeviceToHost, h->stream));
  }
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  // symmetric parameter eps_ab = eps_ba: both table entries carry the full
  // derivative; eps = lambda (M - e0) gives dE/dlambda = sum G_ab (M_ab - e0)
  for (int g = 0; g < h->n_inst && !G.empty(); ++g) {
    const double* Gi = &G[(size_t)g * kNumAmino * kNumAmino];
    double dl = 0.0;
    for (int a = 0; a < kNumAmino; ++a) {
      for (int b = 0; b < kNumAmino; ++b) {
        const double d = (a == b) ? Gi[a * kNumAmino + a]
                                  : Gi[a * kNumAmino + b] + Gi[b * kNumAmino + a];
        if (dE_deps) dE_deps[(size_t)g * kNumAmino * kNumAmino + a * kNumAmino + b] = d;
        dl += Gi[a * kNumAmino + b] *
              ((double)h->pair_table[a * 20 + b] - (double)h->params.e0);
      }
    }
    if (dE_dlambda) dE_dlambda[g] = dl;
  }
  return REMC_OK;
}

int remc_get_noncrowder_energies(remc_handle* h, double* out) {
  if (!h || !out) return set_error(REMC_ERR_INVALID, "null argument");
  REMC_CUDA_TRY(cudaMemcpyAsync(out, h->d_ecc, sizeof(double) * h->n_inst,
                                cudaMemcpyDeviceToHost, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return REMC_OK;
}

int remc_get_pair_evaluations(remc_handle* h, uint64_t* residue_pairs, uint64_t* crowder_pairs) {
  if (!h || !residue_pairs || !crowder_pairs) return set_error(REMC_ERR_INVALID, "null argument");
  std::vector<unsigned long long> a(h->n_inst), b(h->n_inst);
  REMC_CUDA_TRY(cudaMemcpyAsync(a.data(), h->d_evals_kh, sizeof(unsigned long long) * h->n_inst,
                                cudaMemcpyDeviceToHost, h->stream));
  REMC_CUDA_TRY(cudaMemcpyAsync(b.data(), h->d_evals_crowd,
                                sizeof(unsigned long long) * h->n_inst, cudaMemcpyDeviceToHost,
                                h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  uint64_t sa = 0, sb = 0;
  for (int i = 0; i < h->n_inst; ++i) {
    sa += a[i];
    sb += b[i];
  }
  *residue_pairs = sa;
  *crowder_pairs = sb;
  return REMC_OK;
}

int remc_get_stream(remc_handle* h, void** stream) {
  if (!h || !stream) return set_error(REMC_ERR_INVALID, "null argument");
  *stream = (void*)h->stream;
  return REMC_OK;
}

int remc_delta_energy(remc_handle* h, int inst, int mol, const float* new_pos, double* dE) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (!h->tables_set || !h->state_set) return set_error(REMC_ERR_STATE, "tables/state not set");
  if (inst < 0 || inst >= h->n_inst || !new_pos || !dE)
    return set_error(REMC_ERR_INVALID, "bad instance or null pointer");
  const int s = h->h_inst_sys[inst];
  const SysDev& S = h->h_sys[s];
  if (mol < 0 || mol >= S.n_mol) return set_error(REMC_ERR_INVALID, "bad molecule index");
  const int* ms = &h->h_mol_start[S.mstart_off];
  const int n = ms[mol + 1] - ms[mol];
  std::vector<float4> np(n);
  for (int k = 0; k < n; ++k) {
    for (int c = 0; c < 3; ++c)
      if (!std::isfinite(new_pos[3 * k + c]))
        return set_error(REMC_ERR_NUMERIC, "non-finite new position");
    np[k] = make_float4(new_pos[3 * k], new_pos[3 * k + 1], new_pos[3 * k + 2], 0.0f);
  }
  REMC_CUDA_TRY(cudaMemcpyAsync(h->d_newpos, np.data(), sizeof(float4) * n,
                                cudaMemcpyHostToDevice, h->stream));
  delta_kernel<<<1, 256, 0, h->stream>>>(h->d_sys, h->d_inst_sys, h->d_pos, h->d_tab,
                                         h->d_mol_start, inst, mol, h->d_newpos, h->d_dE,
                                         consts_of(h));
  REMC_CUDA_TRY(cudaGetLastError());
  REMC_CUDA_TRY(cudaMemcpyAsync(dE, h->d_dE, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return REMC_OK;
}

int remc_run(remc_handle* h, int n_blocks, int steps_per_block, uint64_t seed, uint32_t step0,
             uint32_t round0) {
  NvtxRange nvtx_range("remc_run");
  int rc = check_ready(h);
  if (rc) return rc;
  if (n_blocks < 0 || steps_per_block <= 0)
    return set_error(REMC_ERR_INVALID, "bad block counts");
  // device control block: step counter, round counter, offset parity
  ctrl_set_kernel<<<1, 1, 0, h->stream>>>(h->d_ctrl, step0, round0);
  REMC_CUDA_TRY(cudaGetLastError());
  if ((size_t)steps_per_block > max_chunk_steps(h))
    return set_error(REMC_ERR_INVALID, "steps_per_block too large for the record buffer");
  rc = ensure_recs(h, (size_t)steps_per_block);
  if (rc) return rc;
  if (!h->graph_exec || h->graph_steps != steps_per_block || h->graph_seed != seed ||
      h->graph_recs_gen != h->recs_gen || h->graph_sample_gen != h->sample_gen ||
      h->graph_config_gen != h->config_gen) {
    if (h->graph_exec) {
      cudaGraphExecDestroy(h->graph_exec);
      h->graph_exec = nullptr;
    }
    cudaGraph_t graph;
    REMC_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    rc = launch_sweep(h, steps_per_block, seed, 0, h->d_ctrl);
    if (!rc) {
      exchange_kernel<<<h->n_sys, 32, 0, h->stream>>>(
          h->d_sys, h->d_ladder, h->d_energy, h->d_temp_idx, h->d_slot_of_temp, h->d_ex_tests,
          h->d_ex_acc, h->d_ctrl, 0, 0, (uint32_t)seed, (uint32_t)(seed >> 32));
      ctrl_advance_kernel<<<1, 1, 0, h->stream>>>(h->d_ctrl, (uint32_t)steps_per_block);
    }
    cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    if (rc) return rc;
    if (e != cudaSuccess) return set_error(REMC_ERR_CUDA, "capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&h->graph_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return set_error(REMC_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e));
    h->graph_steps = steps_per_block;
    h->graph_seed = seed;
    h->graph_recs_gen = h->recs_gen;
    h->graph_sample_gen = h->sample_gen;
    h->graph_config_gen = h->config_gen;
  }
  for (int b = 0; b < n_blocks; ++b) REMC_CUDA_TRY(cudaGraphLaunch(h->graph_exec, h->stream));
  return REMC_OK;
}

int remc_autotune(remc_handle* h, int probe_steps, uint64_t seed, int* threads_out,
                  int* mol_in_smem_out, float* best_ms_out) {
  NvtxRange nvtx_range("remc_autotune");
  int rc = check_ready(h);
  if (rc) return rc;
  if (probe_steps <= 0) return set_error(REMC_ERR_INVALID, "probe_steps must be positive");
  // snapshot everything a sweep changes, so tuning leaves the state as it was
  struct Buf {
    void* dev;
    size_t bytes;
    void* save;
  };
  Buf bufs[] = {{h->d_pos, sizeof(float4) * h->total_beads, nullptr},
                {h->d_rel, sizeof(float4) * h->total_beads, nullptr},
                {h->d_centre, sizeof(float4) * h->total_mols, nullptr},
                {h->d_quat, sizeof(double) * 4 * h->total_mols, nullptr},
                {h->d_energy, sizeof(double) * h->n_inst, nullptr},
                {h->d_ecc, sizeof(double) * h->n_inst, nullptr},
                {h->d_acc_neg, sizeof(int) * h->n_inst, nullptr},
                {h->d_acc_boltz, sizeof(int) * h->n_inst, nullptr},
                {h->d_rej, sizeof(int) * h->n_inst, nullptr},
                {h->d_evals_kh, sizeof(unsigned long long) * h->n_inst, nullptr},
                {h->d_evals_crowd, sizeof(unsigned long long) * h->n_inst, nullptr},
                {h->d_n_samples, sizeof(int) * h->n_inst, nullptr},
                {h->d_n_bound, sizeof(int) * h->n_inst, nullptr}};
  const int nb = (int)(sizeof(bufs) / sizeof(bufs[0]));
  auto release = [&]() {
    for (int i = 0; i < nb; ++i)
      if (bufs[i].save) cudaFree(bufs[i].save);
  };
  for (int i = 0; i < nb; ++i) {
    if (cudaMalloc(&bufs[i].save, bufs[i].bytes) != cudaSuccess) {
      release();
      return set_error(REMC_ERR_NOMEM, "autotune snapshot allocation failed");
    }
    REMC_CUDA_TRY(cudaMemcpyAsync(bufs[i].save, bufs[i].dev, bufs[i].bytes,
                                  cudaMemcpyDeviceToDevice, h->stream));
  }
  const int saved_every = h->sample_every;
  h->sample_every = 0;
  rc = ensure_recs(h, (size_t)probe_steps);
  const int cand_threads[2] = {128, 256};
  // clusters of CTAs per replica only pay when replicas are fewer than the
  // CTAs the GPU can hold
  int cand_c[4] = {1, 0, 0, 0}, n_c = 1;
  for (int c = 2; c <= 8; c *= 2)
    if ((long long)h->n_inst * c <= 2LL * h->num_sms) cand_c[n_c++] = c;
  int best_t = h->sweep_threads, best_m = h->mol_in_smem, best_c = h->sweep_csize;
  int best_b = h->beads_in_smem;
  float best = 1e30f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // beads in shared memory wherever some schedule allows it; in global memory
  // (any size, slower) only when no schedule does
  bool any_fit = false;
  for (int bi = 1; bi >= 0 && !rc && !any_fit; --bi) {
  for (int ci = 0; ci < n_c && !rc; ++ci) {
  for (int ti = 0; ti < 2 && !rc; ++ti) {
    for (int mi = 1; mi >= 0 && !rc; --mi) {
      if (configure_sweep(h, cand_threads[ti], mi, cand_c[ci], bi) != REMC_OK) continue;
      // a cluster size whose clusters cannot all be resident would run the
      // replicas in waves: not a candidate
      if (cand_c[ci] > 1 && h->n_inst > h->sweep_cluster_slots) continue;
      any_fit = true;
      float ms = 1e30f;
      for (int rep = 0; rep < 3 && !rc; ++rep) {  // first launch warms up; best of two
        float t_rep = 0.0f;
        cudaEventRecord(e0, h->stream);
        rc = launch_sweep(h, probe_steps, seed, 0, nullptr);
        cudaEventRecord(e1, h->stream);
        if (!rc && cudaEventSynchronize(e1) != cudaSuccess)
          rc = set_error(REMC_ERR_CUDA, "autotune probe failed");
        if (!rc) cudaEventElapsedTime(&t_rep, e0, e1);
        if (!rc && rep > 0) ms = std::min(ms, t_rep);
        for (int i = 0; i < nb && !rc; ++i)
          if (cudaMemcpyAsync(bufs[i].dev, bufs[i].save, bufs[i].bytes, cudaMemcpyDeviceToDevice,
                              h->stream) != cudaSuccess)
            rc = set_error(REMC_ERR_CUDA, "autotune restore failed");
      }
      if (!rc && ms < best) {
        best = ms;
        best_t = cand_threads[ti];
        best_m = mi;
        best_c = cand_c[ci];
        best_b = bi;
      }
    }
  }
  }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->sample_every = saved_every;
  cudaStreamSynchronize(h->stream);
  release();
  if (rc) return rc;
  rc = configure_sweep(h, best_t, best_m, best_c, best_b);
  if (rc) return rc;
  if (threads_out) *threads_out = best_t;
  if (mol_in_smem_out) *mol_in_smem_out = best_m;
  if (best_ms_out) *best_ms_out = best;
  return REMC_OK;
}

int remc_set_schedule(remc_handle* h, int threads, int mol_in_smem) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return configure_sweep(h, threads, mol_in_smem ? 1 : 0, h->sweep_csize, h->beads_in_smem);
}

int remc_set_cluster(remc_handle* h, int cluster) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return configure_sweep(h, h->sweep_threads, h->mol_in_smem, cluster, h->beads_in_smem);
}

int remc_set_bead_storage(remc_handle* h, int in_shared_memory) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return configure_sweep(h, h->sweep_threads, h->mol_in_smem, h->sweep_csize,
                         in_shared_memory ? 1 : 0);
}

int remc_set_work_order(remc_handle* h, int by_cost) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (by_cost != 0 && by_cost != 1) return set_error(REMC_ERR_INVALID, "work order must be 0 or 1");
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->work_order = by_cost;
  h->config_gen++;  // captured graphs hold the launch sequence
  return REMC_OK;
}

int remc_get_work_order(remc_handle* h, int* by_cost, int* launches_per_sweep) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (by_cost) *by_cost = h->work_order;
  if (launches_per_sweep) *launches_per_sweep = uses_cost_order(h) ? 4 : 2;
  return REMC_OK;
}

int remc_get_bead_storage(remc_handle* h, int* in_shared_memory) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (in_shared_memory) *in_shared_memory = h->beads_in_smem;
  return REMC_OK;
}

int remc_get_schedule(remc_handle* h, int* threads, int* mol_in_smem, int* cluster) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (threads) *threads = h->sweep_threads;
  if (mol_in_smem) *mol_in_smem = h->mol_in_smem;
  if (cluster) *cluster = h->sweep_csize;
  return REMC_OK;
}

int remc_get_fold_flags(remc_handle* h, int* per_system) {
  if (!h || !per_system) return set_error(REMC_ERR_INVALID, "null argument");
  std::vector<SysDev> sd(h->n_sys);
  REMC_CUDA_TRY(cudaMemcpyAsync(sd.data(), h->d_sys, sizeof(SysDev) * h->n_sys,
                                cudaMemcpyDeviceToHost, h->stream));
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  for (int s2 = 0; s2 < h->n_sys; ++s2) per_system[s2] = sd[s2].fold_mi;
  return REMC_OK;
}

int remc_check_wait_timeout(remc_handle* h, int polls) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  if (polls < 1 || polls > (1 << 20))
    return set_error(REMC_ERR_INVALID, "polls must be in [1, 2^20]");
  wait_probe_kernel<<<1, 32, 0, h->stream>>>(h->d_err, polls);
  REMC_CUDA_TRY(cudaGetLastError());
  return check_device_error(h);
}

int remc_sync(remc_handle* h) {
  if (!h) return set_error(REMC_ERR_INVALID, "null handle");
  REMC_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return check_device_error(h);
}

int remc_num_instances(const remc_handle* h) { return h ? h->n_inst : 0; }

}  // extern "C"
