// galpy_b200/csrc/orbit_kernel.cuh
//
// The persistent orbit-integration kernel (one thread per orbit, work
// stealing, one force evaluation per loop iteration; machines.cuh) and the
// selection of its instantiations.  Included by the library's translation
// units that instantiate it: galpy_cuda.cu (leapfrog, rk4, symplec4, dop853)
// and orbit_kernels_more.cu (rk6, symplec6, dopr54), which compile in
// parallel.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

#include "../../include/galpy_cuda.h"
#include "machines.cuh"

namespace gpc {

// ----------------------------------------------------------------------------
// kernel
// ----------------------------------------------------------------------------
struct KArgs {
  long long nobj;
  int nt, indiv_t;
  const double* t;
  const double* w0;
  int in_layout;
  OutSpec out;
  int* err;
  long long* nsteps;
  const GpComp* comps;
  int ncomp;
  const int* group;
  double dt, rtol, atol;
  long long max_attempts;
  unsigned long long* counter;
  const int* abort_flag;
  unsigned long long* done_count;
  const int* order;  // work-queue order (longest first), or NULL
  int variational_nv; // values per input row of variational runs (0 otherwise)
  // the first tail_len queue entries (the longest orbits) go to one warp on
  // each of the SMs 0..tail_sms-1, which run nothing else (0: no reservation)
  long long tail_len;
  int tail_sms;
  unsigned long long* tail_counter;
  unsigned* sm_claim;
  // DOP853 dense-output request queues, one ring of M::kQueueSlots records
  // per warp of the grid (NULL: dense output in the warp's slot cycle)
  double* dense_q;
  // Streaming of finished orbits (blocking host entry points, AoS output):
  // the rows of the orbit at work-queue position q are written at output
  // position q (the output holds the rows in queue order); once they are
  // all written, stage_idx[q] records the orbit and stage_ready[q /
  // kStageChunk] counts the complete positions of each chunk, so that the
  // host can copy finished chunks while the kernel runs.  pend[q] counts
  // the writers of those rows that have not finished (the orbit's own lane,
  // and its queued dense-output requests).  NULL: no streaming (rows at the
  // orbit's index).
  int* stage_idx;
  unsigned* stage_ready;
  int* pend;
  // scalar parameters of the (single) potential, read from the constant bank
  // by the kernels whose POT takes them directly
  double scal[kMaxComp * kScalarStride];
};

// Whether machine M can queue its dense output (M::kQueue, default false).
template <class M, class = void>
struct QueueOf {
  static constexpr bool value = false;
};
template <class M>
struct QueueOf<M, std::void_t<decltype(M::kQueue)>> {
  static constexpr bool value = M::kQueue;
};

template <int NV, int D, bool CYL_OK, int ROW>
struct DevRows {
  const OutSpec* o;
  long long i;
  __device__ __forceinline__ void operator()(int j, const double* v) const
  {
    write_row<NV, D, CYL_OK, ROW>(*o, i, j, v);
  }
};

template <class M>
__device__ __forceinline__ void load_state(const KArgs& A, long long i, double* w)
{
  if (A.in_layout == GALPY_CUDA_IN_SOA) {
#pragma unroll
    for (int k = 0; k < M::NV; k++) w[k] = A.w0[(long long)k * A.nobj + i];
  } else {
#pragma unroll
    for (int k = 0; k < M::NV; k++) w[k] = A.w0[i * M::NV + k];
  }
}

// Whether any reserved SM has taken its tail warp.
__device__ __forceinline__ bool tail_claimed(const KArgs& A)
{
  for (int k = 0; k < A.tail_sms; k++)
    if (*reinterpret_cast<const volatile unsigned*>(&A.sm_claim[k])) return true;
  return false;
}

// Staged slots per chunk of the streaming of finished orbits.
constexpr int kStageChunk = 4096;

// Output position of the orbit i at work-queue position q: q when rows are
// streamed (the output then holds them in queue order), else i.
__device__ __forceinline__ long long out_pos(const KArgs& A, long long q, long long i)
{
  return A.stage_idx ? q : i;
}

// The orbit whose rows are at output position p.
__device__ __forceinline__ long long orbit_at(const KArgs& A, long long p)
{
  return A.stage_idx && A.order ? (long long)A.order[p] : p;
}

#if defined(__CUDACC__)
// The rows at output position p (orbit i) are all written, by whichever lanes
// wrote them, and made visible with __threadfence: publish the position.
__device__ __forceinline__ void publish_rows(const KArgs& A, long long p, long long i)
{
  A.stage_idx[p] = (int)i;
  __threadfence();
  atomicAdd(&A.stage_ready[p / kStageChunk], 1u);
}

// One writer of the rows at output position p has finished: the last one
// publishes them.
__device__ __forceinline__ void release_rows(const KArgs& A, long long p)
{
  __threadfence();  // this writer's rows before the count
  if (atomicSub(&A.pend[p], 1) == 1) {
    __threadfence();  // the other writers' rows before the publication
    publish_rows(A, p, orbit_at(A, p));
  }
}
#endif

// Next work-queue position of a worker: the reserved-SM tail queue first
// (tail role), then the main queue; -1 when both are exhausted.  The orbit
// at position q is order[q] (q without an order).
__device__ __forceinline__ long long next_orbit(const KArgs& A, int& my_role)
{
  long long q = -1;
  if (my_role == 1) {
    q = (long long)atomicAdd(A.tail_counter, 1ULL);
    if (q >= A.tail_len) {
      q = -1;
      my_role = 0;
    }
  }
  if (q < 0 && A.tail_len > 0 && !tail_claimed(A)) {
    // no reserved SM hosts a tail warp: the longest orbits go first here
    q = (long long)atomicAdd(A.tail_counter, 1ULL);
    if (q >= A.tail_len) q = -1;
  }
  if (q < 0) {
    q = (long long)atomicAdd(A.counter, 1ULL) + A.tail_len;
    if (q >= A.nobj) {
      if (A.tail_len == 0) return -1;
      q = (long long)atomicAdd(A.tail_counter, 1ULL);
      if (q >= A.tail_len) return -1;
    }
  }
  return q;
}

#if defined(__CUDACC__)
// The persistent loop of a machine whose dense output goes through the
// warp's request queue (Dop853Machine with KArgs::dense_q set).  The slot
// cycle of an attempt is slots 0..10 (stages 2..12) and 11 (the FSAL
// evaluation); after slot 11 the lanes whose step contains output times
// append a request to the warp's ring (ballot + prefix count, so the
// records are contiguous), and whenever 32 or more requests wait -- or the
// warp has no orbits left -- slots 12..14 are a dense round: lane L runs the
// three dense stages of request head + L and writes its rows.  Every lane of
// the warp stays in the loop until the warp has no orbit and no request
// left (the ballots need all 32 lanes), so a lane without an orbit idles
// instead of leaving.
template <class M, int D, int PREC, bool VAR, class POT>
__device__ __forceinline__ void queued_loop(const KArgs& A, double* slot_store, int my_role)
{
  constexpr bool CYL_OK = !VAR;
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int QS = M::kQueueSlots;
  using Rows = DevRows<M::NV, D, CYL_OK, M::kRow>;
  const int lane = threadIdx.x & 31;
  const long long warp_id = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  double* const q = A.dense_q + warp_id * (long long)(M::kQueueFields * QS);
  M m;
  m.bind(slot_store + threadIdx.x, true);
  long long i = 0, pos = 0;  // the active orbit and its output position
  bool active = false, aborting = false, idle = false;
  const GpComp* comps = A.comps;
  unsigned iter = 0;
  int slot = 0, qhead = 0, qcount = 0, nround = 0;
  for (;;) {
    const bool dense = slot >= 12;
    if (!dense && !active && !idle) {
      const long long qpos = next_orbit(A, my_role);
      if (qpos < 0) {
        idle = true;
      } else {
        i = A.order ? (long long)A.order[qpos] : qpos;
        pos = out_pos(A, qpos, i);
        if (aborting) {
          A.err[i] = E_ABORT;
          write_nan_rows<M::NV, D, CYL_OK, M::kRow>(A.out, pos, 0);
          if (A.stage_idx) {
            __threadfence();
            publish_rows(A, pos, i);
          }
        } else {
          if (A.pend) A.pend[pos] = 1;  // its own lane writes rows until it is done
          double w[M::NV];
          load_state<M>(A, i, w);
          comps = A.comps + (A.group ? (long long)A.group[i] * A.ncomp : 0LL);
          Rows rows{&A.out, pos};
          m.init(w, A.t + (A.indiv_t ? i * (long long)A.nt : 0LL), A.nt, A.dt, A.rtol, A.atol,
                 A.max_attempts, rows);
          active = true;
        }
      }
    }
    const int p = (qhead + lane) & (QS - 1);
    if (dense ? lane < nround : (active && !m.done)) {
      double y[M::NY], qq[M::NA], a[M::NA];
      long long o = i, opos = pos;
      const GpComp* cp = comps;
      double tf = 0.0;  // the force's time (read by time-dependent component lists only)
      if (dense) {  // the request's output position, orbit and parameter group
        opos = reinterpret_cast<const long long*>(q)[(11 * M::N + 2) * QS + p];
        o = orbit_at(A, opos);
        cp = A.comps + (A.group ? (long long)A.group[o] * A.ncomp : 0LL);
        m.req_point(y, slot + 2, q, p);
        if constexpr (POT::kTimeDep) tf = m.req_tpoint(y, slot + 2, q, p);
      } else {
        m.point(y, slot);
        if constexpr (POT::kTimeDep) tf = m.tpoint(y, slot);
      }
      M::pos(y, qq);
      eval_force<D, PREC, VAR, POT>(cp, A.ncomp, qq, a, A.scal, tf);
      Rows rows{&A.out, opos};
      if (dense) {
        m.req_consume(y, a, slot + 2, q, p, A.t + (A.indiv_t ? o * (long long)A.nt : 0LL), rows);
        if (A.stage_idx && slot == 14) release_rows(A, opos);  // its rows are written
      } else {
        m.consume(y, a, rows, slot);
      }
    }
    // the requests of this slot's accepted steps (only the FSAL slot makes any)
    if (slot == 11) {
      const unsigned want = __ballot_sync(FULL, m.want_enqueue);
      if (m.want_enqueue) {
        const int rank = __popc(want & ((1u << lane) - 1u));
        if (A.pend) atomicAdd(&A.pend[pos], 1);  // the request writes rows at pos
        m.write_request(q, (qhead + qcount + rank) & (QS - 1), pos);
        m.want_enqueue = false;
        Rows rows{&A.out, pos};
        m.finish_step(rows);
      }
      qcount += __popc(want);
    }
    const bool all_idle = __all_sync(FULL, idle);
    // next slot (uniform over the warp)
    if (slot == 14) {
      __syncwarp();  // every lane has read its request before the slots are reused
      qhead = (qhead + nround) & (QS - 1);
      qcount -= nround;
      nround = 0;
    }
    if (slot == 11 || slot == 14 || (all_idle && !dense)) {
      if (qcount >= 32 || (all_idle && qcount > 0)) {
        __syncwarp();  // the records of the ring are visible to every lane
        nround = qcount < 32 ? qcount : 32;
        slot = 12;
      } else {
        slot = 0;
      }
    } else {
      slot++;
    }
    if (all_idle && qcount == 0 && nround == 0) break;
    ++iter;
    if (A.abort_flag && ((iter & 255u) == 0u) &&
        *reinterpret_cast<const volatile int*>(A.abort_flag)) {
      aborting = true;
      if (active && !m.done) {
        m.err = E_ABORT;
        m.done = true;
      }
    }
    if (active && m.done) {
      Rows rows{&A.out, pos};
      fill_unreached_rows(m, rows);
      A.err[i] = m.err;
      if (A.nsteps) A.nsteps[i] = m.nsteps;
      if (A.done_count) atomicAdd(A.done_count, 1ULL);
      if (A.stage_idx) release_rows(A, pos);
      active = false;
    }
  }
}
#endif

// MINB: minimum resident blocks per SM requested from the register
// allocator (1 = no cap; larger values trade registers for occupancy).
template <class M, int D, int PREC, bool VAR, class POT, int MINB>
__global__ void __launch_bounds__(128, MINB) orbit_kernel(const __grid_constant__ KArgs A)
{
  constexpr bool CYL_OK = !VAR;
  using Rows = DevRows<M::NV, D, CYL_OK, M::kRow>;
  extern __shared__ double slot_store[];
  // Reserved SMs for the longest orbits: the first block resident on each of
  // SMs 0..tail_sms-1 keeps one warp, which takes the tail queue (then helps
  // with the main queue); any other block there leaves, so those orbits do
  // not share their SM with the bulk of the batch.  Main workers drain tail
  // entries left unclaimed (no block landed on a reserved SM).
  __shared__ int role;  // 0 main queue, 1 tail warp, 2 leave
  if (threadIdx.x == 0) {
    role = 0;
    if (A.tail_len > 0) {
      unsigned smid;
      asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
      if (smid < (unsigned)A.tail_sms) role = atomicExch(&A.sm_claim[smid], 1u) == 0u ? 1 : 2;
    }
  }
  __syncthreads();
  int my_role = role;
  if (my_role == 2 || (my_role == 1 && threadIdx.x >= 32)) return;
  if constexpr (QueueOf<M>::value) {
    if (A.dense_q) {
      queued_loop<M, D, PREC, VAR, POT>(A, slot_store, my_role);
      return;
    }
  }
  M m;
  m.bind(slot_store + threadIdx.x);
  long long i = 0, pos = 0;  // the active orbit and its output position
  bool active = false, aborting = false;
  const GpComp* comps = A.comps;
  unsigned iter = 0;
  int slot = 0;
  for (;;) {
    if (!active) {
      const long long qpos = next_orbit(A, my_role);
      if (qpos < 0) break;
      i = A.order ? (long long)A.order[qpos] : qpos;
      pos = out_pos(A, qpos, i);
      if (aborting) {
        A.err[i] = E_ABORT;
        write_nan_rows<M::NV, D, CYL_OK, M::kRow>(A.out, pos, 0);
        if (A.stage_idx) {
          __threadfence();
          publish_rows(A, pos, i);
        }
        continue;
      }
      double w[M::NV];
      load_state<M>(A, i, w);
      comps = A.comps + (A.group ? (long long)A.group[i] * A.ncomp : 0LL);
      Rows rows{&A.out, pos};
      m.init(w, A.t + (A.indiv_t ? i * (long long)A.nt : 0LL), A.nt, A.dt, A.rtol, A.atol,
             A.max_attempts, rows);
      active = true;
    }
    if (!m.done) {
      double y[M::NY], q[M::NA], a[M::NA];
      m.point(y, slot);
      double tf = 0.0;
      if constexpr (POT::kTimeDep) tf = m.tpoint(y, slot);
      M::pos(y, q);
      eval_force<D, PREC, VAR, POT>(comps, A.ncomp, q, a, A.scal, tf);
      Rows rows{&A.out, pos};
      m.consume(y, a, rows, slot);
    }
    // advance the warp's stage slot (DOP853): the dense-output slots run only
    // if some lane of the warp needs them
#if defined(__CUDA_ARCH__)
    slot = M::next_slot(slot, __any_sync(__activemask(), m.wants_dense()));
#endif
    ++iter;
    if (A.abort_flag && ((iter & 255u) == 0u) &&
        *reinterpret_cast<const volatile int*>(A.abort_flag)) {
      aborting = true;
      if (!m.done) {
        m.err = E_ABORT;
        m.done = true;
      }
    }
    if (m.done) {
      Rows rows{&A.out, pos};
      fill_unreached_rows(m, rows);
      A.err[i] = m.err;
      if (A.nsteps) A.nsteps[i] = m.nsteps;
      if (A.done_count) atomicAdd(A.done_count, 1ULL);
      if (A.stage_idx) {
        __threadfence();
        publish_rows(A, pos, i);
      }
      active = false;
    }
  }
}

// ----------------------------------------------------------------------------
// instantiation and selection
// ----------------------------------------------------------------------------
using KernelFn = void (*)(const KArgs);

struct KernelInfo {
  KernelFn fn = nullptr;
  int slot_doubles = 0;   // per-thread shared-memory slot store (doubles)
  int queue_doubles = 0;  // per-warp dense-output request ring (doubles; 0: none)
};

template <class M>
constexpr int queue_doubles_of()
{
  if constexpr (QueueOf<M>::value)
    return M::kQueueFields * M::kQueueSlots;
  else
    return 0;
}

// Register-budget variants (chosen by the autotuner, galpy_b200/autotune.py):
// variant 0 lets the compiler use up to 255 registers; variant 1 caps them
// so that more blocks are resident (3 blocks/SM for DOP853, whose shared
// slot store allows at most 3; 4 blocks/SM for the lighter integrators).
template <class M, int D, int PREC, bool VAR, class POT>
static KernelInfo info_of(int variant)
{
  KernelInfo k;
  constexpr int capped = M::kSlotDoubles > 0 ? 3 : 4;
  if constexpr (VAR) {  // variational runs: one variant
    k.fn = orbit_kernel<M, D, PREC, VAR, POT, 1>;
  } else {
    if (variant == 1)
      k.fn = orbit_kernel<M, D, PREC, VAR, POT, capped>;
    else
      k.fn = orbit_kernel<M, D, PREC, VAR, POT, 1>;
  }
  k.slot_doubles = M::kSlotDoubles;
  k.queue_doubles = queue_doubles_of<M>();
  return k;
}

// Set::pick<D, PREC, VAR, POT>(method, variant): the kernel of one of the
// set's methods, or an empty KernelInfo.
template <class Set, int PREC, class POT>
static KernelInfo pick_plain(int planar, int method, int variant)
{
  return planar ? Set::template pick<2, PREC, false, POT>(method, variant)
                : Set::template pick<3, PREC, false, POT>(method, variant);
}

// sig: GALPY_CUDA_SIG_MW14 selects the kernels with the MWPotential2014
// component list fixed at compile time (plain runs), GALPY_CUDA_SIG_COMMON
// the float64 kernels whose run-time list leaves out the ellipsoidal family;
// variational runs and float32 forces walk the full list at run time.
template <class Set>
static KernelInfo pick_kernel_in(int planar, int var, int prec, int method, int sig,
                                 int variant, bool direct)
{
  if (var) {
    if (prec != GALPY_CUDA_FP64) return KernelInfo();  // variational runs are float64 only
    return planar ? Set::template pick<2, PREC_FP64, true, DynPot>(method, 0)
                  : Set::template pick<3, PREC_FP64, true, DynPot>(method, 0);
  }
  const bool mw14 = sig == GALPY_CUDA_SIG_MW14;
  if (prec == GALPY_CUDA_F32FORCE) {
    if (!mw14) return pick_plain<Set, PREC_F32, DynPot>(planar, method, variant);
    return direct ? pick_plain<Set, PREC_F32, MW14Pot>(planar, method, variant)
                  : pick_plain<Set, PREC_F32, MW14GroupPot>(planar, method, variant);
  }
  if (sig == GALPY_CUDA_SIG_COMMON)
    return pick_plain<Set, PREC_FP64, DynPotCommon>(planar, method, variant);
  if (!mw14) return pick_plain<Set, PREC_FP64, DynPot>(planar, method, variant);
  return direct ? pick_plain<Set, PREC_FP64, MW14Pot>(planar, method, variant)
                : pick_plain<Set, PREC_FP64, MW14GroupPot>(planar, method, variant);
}

// rk6, symplec6 and dopr54 (orbit_kernels_more.cu; not exported)
__attribute__((visibility("hidden"))) KernelInfo pick_kernel_more(int planar, int var, int prec,
                                                                  int method, int sig,
                                                                  int variant, bool direct);
// the mixed-precision forms (GALPY_CUDA_F64_TAIL32, _F32BULGE,
// _F32FORCE_DF) of the MWPotential2014 kernels (orbit_kernels_prec.cu; not
// exported)
__attribute__((visibility("hidden"))) KernelInfo pick_kernel_prec(int planar, int var, int prec,
                                                                  int method, int sig,
                                                                  int variant, bool direct);
// surface-of-section kernels: rk4, rk6, dopr54, dop853 on the 3D or planar
// (surface x = 0 / y = 0) system, FP64, run-time component list
// (orbit_kernels_more.cu; not exported)
__attribute__((visibility("hidden"))) KernelInfo pick_kernel_sos(int method, int variant,
                                                                 int system);

}  // namespace gpc
