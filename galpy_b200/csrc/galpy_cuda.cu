// galpy_b200/csrc/galpy_cuda.cu
//
// libgalpy_cuda.so: batched orbit integration on sm_100a behind the C ABI of
// include/galpy_cuda.h.
//
// Execution model
//   * One thread integrates one orbit at a time in float64 state.  Threads
//     pull orbit indices from a device work counter (work stealing) until the
//     batch is exhausted, so orbits with very different step counts (inner
//     vs outer orbits, ragged integration times, adaptive DOP853) keep every
//     lane busy instead of leaving warps waiting for their slowest orbit.
//   * The kernel is persistent: one wave of blocks sized from the occupancy
//     of the instantiated kernel on this device's SMs.
//   * Every loop iteration of a thread performs exactly one force evaluation
//     (machines.cuh), so all lanes of a warp meet at a single inlined force
//     call whatever stage of whatever orbit they are in.
//   * Potential parameters are compiled on the host into per-component
//     records (compile_potential.h) read through the read-only cache; a batch
//     may hold many parameter groups (ragged multi-potential runs).
//   * Output rows are written directly in the requested layout: galpy's AoS
//     cylindrical rows for the drop-in entry points, or coalesced SoA rows
//     for device-resident batch use.
#include <cub/device/device_radix_sort.cuh>
#include <cuda.h>  // CUcontext and CUresult only; no driver symbol is linked
#include <cuda_runtime.h>
#include <signal.h>
#include <stddef.h>
#include <stdio.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/galpy_cuda.h"
#include "compile_potential.h"
#include "orbit_kernel.cuh"

using namespace gpc;

// ----------------------------------------------------------------------------
// error reporting
// ----------------------------------------------------------------------------
static thread_local std::string g_last_error;

static int set_error(int code, const std::string& msg)
{
  g_last_error = msg;
  return code;
}

// for the library's other translation units (not exported)
__attribute__((visibility("hidden"))) int gpc_report_error(int code, const char* msg)
{
  return set_error(code, msg);
}

#define GPC_CUDA_TRY(expr)                                                              \
  do {                                                                                  \
    cudaError_t e_ = (expr);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return set_error(GALPY_CUDA_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// The context current on the calling thread: the driver's cuCtxGetCurrent,
// reached through the runtime (cudaGetDriverEntryPoint) so that the library
// does not link libcuda itself.  NULL when no context is current yet.
static CUcontext current_context()
{
  typedef CUresult (*GetCurrentFn)(CUcontext*);
  static const GetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (GetCurrentFn) nullptr;
    return reinterpret_cast<GetCurrentFn>(p);
  }();
  CUcontext c = nullptr;
  if (fn && fn(&c) != CUDA_SUCCESS) c = nullptr;
  return c;
}

// ----------------------------------------------------------------------------
// longest-first scheduling: estimated cost of each orbit
// ----------------------------------------------------------------------------
// cost ~ |t_end - t_0| * Omega, Omega^2 = |a . x| / |x|^2 at the initial
// point (the local orbital frequency): the number of steps of any of the
// integrators grows with the number of orbital periods covered.  Orbits are
// handed out in decreasing order of this estimate so that the longest ones
// start first and the batch does not end with a few long orbits running
// alone.
template <int D>
__global__ void __launch_bounds__(256) cost_kernel(const KArgs A, float* key, int* idx)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= A.nobj) return;
  double q[3] = {0.0, 0.0, 0.0}, a[3] = {0.0, 0.0, 0.0};
  const int nv = 2 * D;
  for (int k = 0; k < D; k++)
    q[k] = A.in_layout == GALPY_CUDA_IN_SOA ? A.w0[(long long)k * A.nobj + i]
                                             : A.w0[i * (long long)(A.variational_nv ? A.variational_nv : nv) + k];
  const GpComp* comps = A.comps + (A.group ? (long long)A.group[i] * A.ncomp : 0LL);
  eval_force<D, PREC_FP64, false, DynPot>(comps, A.ncomp, q, a);
  double ax = 0.0, xx = 0.0;
  for (int k = 0; k < D; k++) {
    ax += a[k] * q[k];
    xx += q[k] * q[k];
  }
  const double* tt = A.t + (A.indiv_t ? i * (long long)A.nt : 0LL);
  const double span = fabs(tt[A.nt - 1] - tt[0]);
  const double om = sqrt(fabs(ax) / (xx > 0.0 ? xx : 1e-300));
  float k = (float)(span * om);
  if (!isfinite(k)) k = 0.f;
  key[i] = k;
  idx[i] = (int)i;
}

// Parameter-group launches: the cost estimate in 64 logarithmic buckets
// (4 log2(1 + cost): each a factor 2^(1/4) wide) as the high bits of the key
// and the orbit's group (complemented) as the low bits, so that the
// descending sort still hands out the longest orbits first, while the orbits
// of one bucket come group by group: the lanes of a warp then read the same
// potential records (on the ragged workload, 512 groups: 1,235 ms per launch
// with the plain cost order, 1,026 ms in index order, where groups are
// contiguous).
constexpr int kCostBuckets = 64;
template <int D>
__global__ void __launch_bounds__(256) cost_group_kernel(const KArgs A, unsigned* key, int* idx)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= A.nobj) return;
  double q[3] = {0.0, 0.0, 0.0}, a[3] = {0.0, 0.0, 0.0};
  const int nv = 2 * D;
  for (int k = 0; k < D; k++)
    q[k] = A.in_layout == GALPY_CUDA_IN_SOA ? A.w0[(long long)k * A.nobj + i]
                                             : A.w0[i * (long long)(A.variational_nv ? A.variational_nv : nv) + k];
  const int g = A.group[i];
  const GpComp* comps = A.comps + (long long)g * A.ncomp;
  eval_force<D, PREC_FP64, false, DynPot>(comps, A.ncomp, q, a);
  double ax = 0.0, xx = 0.0;
  for (int k = 0; k < D; k++) {
    ax += a[k] * q[k];
    xx += q[k] * q[k];
  }
  const double* tt = A.t + (A.indiv_t ? i * (long long)A.nt : 0LL);
  const double cost = fabs(tt[A.nt - 1] - tt[0]) * sqrt(fabs(ax) / (xx > 0.0 ? xx : 1e-300));
  int b = isfinite(cost) ? (int)(4.0 * log2(1.0 + cost)) : 0;
  b = b < 0 ? 0 : (b > kCostBuckets - 1 ? kCostBuckets - 1 : b);
  const unsigned gl = (unsigned)(g < 0 ? 0 : (g > 0xffffff ? 0xffffff : g));
  key[i] = ((unsigned)b << 24) | (0xffffffu - gl);
  idx[i] = (int)i;
}

// ----------------------------------------------------------------------------
// launch plumbing
// ----------------------------------------------------------------------------
struct CoreMethods {
  template <int D, int PREC, bool VAR, class POT>
  static KernelInfo pick(int method, int variant)
  {
    switch (method) {
      case M_LEAPFROG: return info_of<SymplecticMachine<D, VAR, 2>, D, PREC, VAR, POT>(variant);
      case M_SYMPLEC4: return info_of<SymplecticMachine<D, VAR, 4>, D, PREC, VAR, POT>(variant);
      case M_RK4: return info_of<RKMachine<D, VAR, 4>, D, PREC, VAR, POT>(variant);
      case M_DOP853: return info_of<Dop853Machine<D, VAR>, D, PREC, VAR, POT>(variant);
    }
    return KernelInfo();
  }
};

// The ODE system of a launch (the field exists when size_ext >= 2).
static int launch_system(const galpy_cuda_launch* L)
{
  return L->size_ext >= 2 ? L->system : GALPY_CUDA_SYS_ORBIT;
}

static KernelInfo pick_kernel(int planar, int var, int prec, int method, int sig, int variant,
                              bool direct, int system = GALPY_CUDA_SYS_ORBIT)
{
  if (system != GALPY_CUDA_SYS_ORBIT) return pick_kernel_sos(method, variant, system);
  if (prec >= GALPY_CUDA_F64_TAIL32)
    return pick_kernel_prec(planar, var, prec, method, sig, variant, direct);
  if (method == M_RK6 || method == M_SYMPLEC6 || method == M_DOPR54)
    return pick_kernel_more(planar, var, prec, method, sig, variant, direct);
  return pick_kernel_in<CoreMethods>(planar, var, prec, method, sig, variant, direct);
}

static int signature_of(int npot, const int* pot_type)
{
  if (npot == 3 && pot_type[0] == T_PSWC && pot_type[1] == T_MN && pot_type[2] == T_NFW)
    return GALPY_CUDA_SIG_MW14;
  for (int k = 0; k < npot; k++)
    if (needs_full_list(pot_type[k])) return GALPY_CUDA_SIG_GENERIC;
  return GALPY_CUDA_SIG_COMMON;
}

// The signature a launch runs with: GALPY_CUDA_SIG_COMMON falls back to the
// full run-time list when the host copy of the records shows a component
// only that list carries (ellipsoidal, DehnenBar, SCF).
static int launch_signature(const galpy_cuda_launch* L)
{
  if (L->signature != GALPY_CUDA_SIG_COMMON || !L->comps_host) return L->signature;
  const GpComp* hc = static_cast<const GpComp*>(L->comps_host);
  for (int k = 0; k < L->ncomp; k++)
    if (needs_full_list(hc[k].type)) return GALPY_CUDA_SIG_GENERIC;
  return GALPY_CUDA_SIG_COMMON;
}

static bool method_supported(int m)
{
  return m >= M_LEAPFROG && m <= M_DOP853;  // galpy's 0..6; 7 (ias15) is not implemented
}

constexpr int kMaxTailSms = 16;
struct Scratch {  // device scratch of one launch (128 bytes)
  unsigned long long counter;
  unsigned long long done_count;
  unsigned long long tail_counter;
  unsigned long long spare;
  int abort_flag;
  unsigned sm_claim[kMaxTailSms];  // first block resident on each reserved SM
  int pad[7];
};
static_assert(sizeof(Scratch) == 128, "Scratch layout");

// Device buffers of the streaming of finished orbits (RowStreamer); the
// launch's output then holds the rows in work-queue order.
struct Staging {
  int* idx = nullptr;         // [nobj] orbit at each output position
  unsigned* ready = nullptr;  // [nchunk] complete positions per chunk
  int* pend = nullptr;        // [nobj] unfinished row writers per position
};

// Launch on `stream`.  scratch: device Scratch (counter zeroed here).
// Scalars of a single-potential launch for the kernel-parameter path.
static bool direct_scalars(const galpy_cuda_launch* L, double* scal)
{
  if (L->group || !L->comps_host || L->signature != GALPY_CUDA_SIG_MW14) return false;
  const GpComp* hc = static_cast<const GpComp*>(L->comps_host);
  for (int k = 0; k < L->ncomp && k < kMaxComp; k++)
    for (int j = 0; j < kScalarStride; j++) scal[k * kScalarStride + j] = hc[k].c[j];
  return true;
}

// Stream-ordered allocation from `pool`, or from the device's default pool
// when pool is NULL (the device entry point's documented behaviour).
static cudaError_t alloc_async(void** p, size_t bytes, cudaMemPool_t pool, cudaStream_t s)
{
  return pool ? cudaMallocFromPoolAsync(p, bytes, pool, s) : cudaMallocAsync(p, bytes, s);
}

// Kernel and kernel arguments of a launch, with the control words pointed
// into `scratch` (a Scratch in device memory, cleared by the caller).
static int prepare_launch(const galpy_cuda_launch* L, Scratch* scratch, bool progress,
                          KernelInfo& ki, KArgs& A, const Staging* stg = nullptr)
{
  double scal[kMaxComp * kScalarStride] = {0.0};
  const bool direct = direct_scalars(L, scal);
  ki = pick_kernel(L->planar, L->variational, L->precision, L->odeint_type, launch_signature(L),
                   L->variant, direct, launch_system(L));
  if (!ki.fn) return set_error(GALPY_CUDA_ERR_METHOD, "method/precision combination not implemented");
  memset(&A, 0, sizeof(A));
  A.nobj = L->nobj;
  A.nt = L->nt;
  A.indiv_t = L->indiv_t;
  A.t = L->t;
  A.w0 = L->w0;
  A.in_layout = L->in_layout;
  A.out.out = L->out;
  A.out.layout = L->out_layout;
  A.out.nt = L->nt;
  A.out.row0 = L->out_row0;
  A.out.nobj = L->nobj;
  A.err = L->err;
  A.nsteps = L->nsteps;
  A.comps = static_cast<const GpComp*>(L->comps);
  A.ncomp = L->ncomp;
  A.group = L->group;
  A.dt = L->dt;
  A.rtol = L->rtol;
  A.atol = L->atol;
  A.max_attempts = L->max_attempts;
  A.counter = &scratch->counter;
  A.tail_counter = &scratch->tail_counter;
  A.sm_claim = scratch->sm_claim;
  A.abort_flag = L->abort_flag ? L->abort_flag : &scratch->abort_flag;
  A.done_count = progress ? &scratch->done_count : nullptr;
  A.variational_nv = L->variational ? (L->planar ? 8 : 12) : 0;
  memcpy(A.scal, scal, sizeof(scal));
  if (stg) {
    A.stage_idx = stg->idx;
    A.stage_ready = stg->ready;
    A.pend = stg->pend;
  }
  return GALPY_CUDA_OK;
}

// Grid of the persistent kernel (one wave: SMs x resident blocks), its
// shared memory and carveout, the SMs reserved for the longest orbits, and
// the launch.  Shared by the allocating and the allocation-free entry points.
// queue: give DOP853 kernels their dense-output request rings (allocated
// stream-ordered from `pool`, or the default pool when NULL, and freed after
// the launch); without it their dense output runs in the warps' slot cycle.
static int launch_persistent(const galpy_cuda_launch* L, const KernelInfo& ki, KArgs& A,
                             cudaStream_t stream, bool queue = false,
                             cudaMemPool_t pool = nullptr)
{
  KernelFn fn = ki.fn;
  int dev = 0;
  GPC_CUDA_TRY(cudaGetDevice(&dev));
  int nsm = 0;
  GPC_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int block = L->block_size > 0 ? L->block_size : 128;
  if (block > 128 || block % 32) return set_error(GALPY_CUDA_ERR_ARG, "block_size must be 32..128, multiple of 32");
  // machines with a slot store keep it strided by kSlotStride threads
  // whatever the block size (smaller blocks leave part of it unused)
  const size_t smem = (size_t)ki.slot_doubles * sizeof(double) * kSlotStride;
  if (smem > 48 * 1024)
    GPC_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // slot-store machines: all of the unified L1/shared array as shared memory
  // for the register-capped variant and for blocks below 128, so that 3
  // blocks' slot stores (3 x 66 KB for 3D DOP853) fit per SM; the hot
  // potential tables are a few KB
  // (the attribute belongs to the kernel, so it is set on every launch)
  if (smem > 0)
    GPC_CUDA_TRY(cudaFuncSetAttribute(
        fn, cudaFuncAttributePreferredSharedMemoryCarveout,
        (int)(L->variant == 1 || block < kSlotStride ? cudaSharedmemCarveoutMaxShared
                                                     : cudaSharedmemCarveoutDefault)));
  int per_sm = 0;
  GPC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, smem));
  if (per_sm < 1) per_sm = 1;
  long long grid = L->grid_size > 0 ? L->grid_size : (long long)nsm * per_sm;
  const long long need = (L->nobj + block - 1) / block;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  // reserve SMs for the longest orbits of a large longest-first batch (one
  // warp each); worthwhile only when the batch is many waves deep.  On the
  // batching workload one SM was best (1,035 ms per step; 2: 1,041, 4:
  // 1,052, 8: 1,072, none: 1,167).
  int tail_sms = L->size_ext >= 1 && L->tail_sms >= 0 ? L->tail_sms : 1;
  if (tail_sms > kMaxTailSms) tail_sms = kMaxTailSms;
  if (tail_sms > nsm / 16) tail_sms = nsm / 16;
  if (A.order && tail_sms > 0 && L->grid_size <= 0 &&
      L->nobj >= 8LL * grid * block && grid == (long long)nsm * per_sm) {
    A.tail_sms = tail_sms;
    A.tail_len = 32LL * tail_sms;
  }
  void* dq = nullptr;
  A.dense_q = nullptr;
  if (queue && ki.queue_doubles > 0) {
    const size_t bytes = (size_t)grid * (block / 32) * ki.queue_doubles * sizeof(double);
    GPC_CUDA_TRY(alloc_async(&dq, bytes, pool, stream));
    A.dense_q = static_cast<double*>(dq);
  }
  fn<<<(unsigned)grid, block, smem, stream>>>(A);
  cudaError_t le = cudaGetLastError();
  if (dq) cudaFreeAsync(dq, stream);
  if (le != cudaSuccess)
    return set_error(GALPY_CUDA_ERR_CUDA, std::string("orbit kernel launch: ") + cudaGetErrorString(le));
  return GALPY_CUDA_OK;
}

static int launch_kernel(const galpy_cuda_launch* L, Scratch* scratch, bool progress,
                         cudaStream_t stream, cudaMemPool_t pool = nullptr,
                         const Staging* stg = nullptr)
{
  KernelInfo ki;
  KArgs A;
  int rc = prepare_launch(L, scratch, progress, ki, A, stg);
  if (rc) return rc;
  const int system = launch_system(L);
  GPC_CUDA_TRY(cudaMemsetAsync(scratch, 0, sizeof(Scratch), stream));

  // longest-first work queue (stream-ordered scratch, freed after the launch);
  // surface-of-section runs go in order (the cost pass reads orbit states)
  void* sched = nullptr;
  if (L->schedule == GALPY_CUDA_SCHED_LONGEST_FIRST && L->nobj > 1 && L->nobj < (1LL << 31) &&
      system == GALPY_CUDA_SYS_ORBIT) {
    const int n = (int)L->nobj;
    size_t tmp_bytes = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp_bytes, (float*)nullptr, (float*)nullptr,
                                              (int*)nullptr, (int*)nullptr, n, 0, 32, stream);
    if (A.group) {  // parameter groups sort 32-bit unsigned keys (cost_group_kernel)
      size_t ubytes = 0;
      cub::DeviceRadixSort::SortPairsDescending(nullptr, ubytes, (unsigned*)nullptr,
                                                (unsigned*)nullptr, (int*)nullptr, (int*)nullptr,
                                                n, 0, 32, stream);
      tmp_bytes = std::max(tmp_bytes, ubytes);
    }
    const size_t keys = (size_t)n * sizeof(float), vals = (size_t)n * sizeof(int);
    const size_t off_k2 = keys, off_v1 = 2 * keys, off_v2 = 2 * keys + vals,
                 off_tmp = (2 * keys + 2 * vals + 255) & ~(size_t)255;
    GPC_CUDA_TRY(alloc_async(&sched, off_tmp + tmp_bytes, pool, stream));
    char* base = static_cast<char*>(sched);
    float* k1 = reinterpret_cast<float*>(base);
    float* k2 = reinterpret_cast<float*>(base + off_k2);
    int* v1 = reinterpret_cast<int*>(base + off_v1);
    int* v2 = reinterpret_cast<int*>(base + off_v2);
    const unsigned cb = (unsigned)((L->nobj + 255) / 256);
    cudaError_t se;
    if (A.group) {  // bucketed cost, then group (cost_group_kernel)
      unsigned* u1 = reinterpret_cast<unsigned*>(k1);
      unsigned* u2 = reinterpret_cast<unsigned*>(k2);
      if (L->planar)
        cost_group_kernel<2><<<cb, 256, 0, stream>>>(A, u1, v1);
      else
        cost_group_kernel<3><<<cb, 256, 0, stream>>>(A, u1, v1);
      GPC_CUDA_TRY(cudaGetLastError());
      se = cub::DeviceRadixSort::SortPairsDescending(base + off_tmp, tmp_bytes, u1, u2, v1, v2, n,
                                                     0, 32, stream);
    } else {
      if (L->planar)
        cost_kernel<2><<<cb, 256, 0, stream>>>(A, k1, v1);
      else
        cost_kernel<3><<<cb, 256, 0, stream>>>(A, k1, v1);
      GPC_CUDA_TRY(cudaGetLastError());
      se = cub::DeviceRadixSort::SortPairsDescending(base + off_tmp, tmp_bytes, k1, k2, v1, v2, n,
                                                     0, 32, stream);
    }
    if (se != cudaSuccess) {
      cudaFreeAsync(sched, stream);
      return set_error(GALPY_CUDA_ERR_CUDA, std::string("radix sort: ") + cudaGetErrorString(se));
    }
    A.order = v2;
  }
  rc = launch_persistent(L, ki, A, stream, true, pool);
  if (sched) cudaFreeAsync(sched, stream);
  return rc;
}

static int check_launch(const galpy_cuda_launch* L)
{
  if (!L) return set_error(GALPY_CUDA_ERR_ARG, "launch is NULL");
  const int system = launch_system(L);
  if (system < GALPY_CUDA_SYS_ORBIT || system > GALPY_CUDA_SYS_SOS_PLANAR_Y)
    return set_error(GALPY_CUDA_ERR_ARG, "unknown system");
  if (system != GALPY_CUDA_SYS_ORBIT) {
    const int m = L->odeint_type;
    if (m != M_RK4 && m != M_RK6 && m != M_DOPR54 && m != M_DOP853)
      return set_error(GALPY_CUDA_ERR_METHOD,
                       "surface-of-section integration takes rk4, rk6, dopr54 or dop853");
    if (L->planar != (system != GALPY_CUDA_SYS_SOS) || L->variational ||
        L->precision != GALPY_CUDA_FP64)
      return set_error(GALPY_CUDA_ERR_ARG,
                       "surface-of-section integration is plain float64, 3D for "
                       "GALPY_CUDA_SYS_SOS and planar for the planar systems");
  }
  if (!method_supported(L->odeint_type))
    return set_error(GALPY_CUDA_ERR_METHOD, "odeint_type not implemented on the GPU");
  if (L->nobj < 0 || L->nt < 1 || !L->t || !L->w0 || !L->out || !L->err || !L->comps ||
      L->ncomp < 1 || L->ncomp > kMaxComp || L->out_row0 < 0 || L->out_row0 >= L->nt)
    return set_error(GALPY_CUDA_ERR_ARG, "invalid launch arguments");
  if (L->precision < GALPY_CUDA_FP64 || L->precision > GALPY_CUDA_F32FORCE_DF)
    return set_error(GALPY_CUDA_ERR_ARG, "unknown precision");
  return GALPY_CUDA_OK;
}

// ----------------------------------------------------------------------------
// SIGINT handling of the galpy-facing blocking calls (the reference polls a
// process-global flag set by its handler, bovy_symplecticode.c:38-45)
// ----------------------------------------------------------------------------
static volatile sig_atomic_t g_sigint = 0;
static void on_sigint(int) { g_sigint = 1; }

struct SigintGuard {
  struct sigaction old_action;
  bool installed = false;
  explicit SigintGuard(bool install = true)
  {
    if (!install) return;
    struct sigaction a;
    memset(&a, 0, sizeof(a));
    a.sa_handler = on_sigint;
    g_sigint = 0;
    installed = sigaction(SIGINT, &a, &old_action) == 0;
  }
  ~SigintGuard()
  {
    if (installed) sigaction(SIGINT, &old_action, nullptr);
  }
};

// RAII device buffers for the host-pointer entry points
struct DevBuf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  ~DevBuf()
  {
    if (p) cudaFreeAsync(p, s);
  }
};

// The blocking entry points allocate their device buffers stream-ordered
// from a memory pool private to the library (one per device and context),
// whose release threshold keeps freed memory in the pool: with a threshold
// of 0 every call would hand gigabytes back to the driver at its final
// synchronisation and map them again on the next call (e2e 4.3e8 vs 9.7e8
// steps/s on the batching workload).  Being private, the pool changes
// nothing in the caller's own allocators (the device's default pool keeps
// its settings); galpy_cuda_trim_memory returns the cached memory.
static std::mutex g_pool_mutex;
static cudaMemPool_t g_pool[64] = {nullptr};
static CUcontext g_pool_ctx[64] = {nullptr};

static int library_pool(cudaMemPool_t* out)
{
  int dev = 0;
  GPC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(GALPY_CUDA_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  CUcontext ctx = current_context();
  if (!ctx) {  // no context yet: cudaSetDevice initialises the primary one
    GPC_CUDA_TRY(cudaSetDevice(dev));
    ctx = current_context();
  }
  if (!g_pool[dev] || ctx != g_pool_ctx[dev]) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    GPC_CUDA_TRY(cudaMemPoolCreate(&pool, &props));
    unsigned long long keep = ~0ULL;
    GPC_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pool[dev] = pool;
    g_pool_ctx[dev] = ctx;
  }
  *out = g_pool[dev];
  return GALPY_CUDA_OK;
}

// The same pool for the library's other translation units (the orbit
// interpolation's scratch).
__attribute__((visibility("hidden"))) int gpc_library_pool(cudaMemPool_t* out)
{
  return library_pool(out);
}

static int select_device(const galpy_cuda_opts* o)
{
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1)
    return set_error(GALPY_CUDA_ERR_NODEVICE, "no CUDA device visible");
  if (o && o->device >= 0) GPC_CUDA_TRY(cudaSetDevice(o->device));
  return GALPY_CUDA_OK;
}

// ----------------------------------------------------------------------------
// streaming of finished orbits to the host
// ----------------------------------------------------------------------------
// The blocking entry points return galpy's AoS result rows in host memory
// (pinned or pageable numpy arrays).  Copying the whole result after the
// kernel would add the full device->host transfer (5 GB for the batching
// workload) to the call.  Instead the kernel writes the rows in work-queue
// order (the orbit at queue position q at output position q) and publishes
// each position once its rows are complete; while it runs, this streamer
// copies every 4096-position chunk whose positions are all published
// through pinned bounce buffers on a copy stream, in any order, and worker
// threads scatter the rows to the orbits' places in the caller's result
// array.  Positions are taken in longest-first order, so a chunk holds
// orbits of similar length, which finish at similar times.
// Pinned bounce buffers of RowStreamer, kept for later calls (pinning host
// memory is slow); at most kBounceCache of them stay cached.
static std::mutex g_bounce_mu;
static std::vector<void*> g_bounce_free;
constexpr size_t kBounceCache = 8;

static cudaError_t bounce_get(void** p, size_t bytes)
{
  {
    std::lock_guard<std::mutex> lk(g_bounce_mu);
    if (!g_bounce_free.empty()) {
      *p = g_bounce_free.back();
      g_bounce_free.pop_back();
      return cudaSuccess;
    }
  }
  return cudaMallocHost(p, bytes);
}

static void bounce_put(void* p)
{
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_bounce_mu);
  if (g_bounce_free.size() < kBounceCache)
    g_bounce_free.push_back(p);
  else
    cudaFreeHost(p);
}

class RowStreamer {
 public:
  static constexpr size_t kBounceBytes = 32u << 20;
  static constexpr int kBuffers = 4;

  // rows: the launch's output, [nobj][row] in work-queue order
  RowStreamer(const Staging& st, const double* rows, long long nobj, size_t row, double* result,
              cudaStream_t side)
      : st_(st), rows_(rows), nobj_(nobj), row_(row), result_(result), side_(side)
  {
    nchunk_ = (int)((nobj + kStageChunk - 1) / kStageChunk);
    issued_.assign(nchunk_, 0);
    per_buf_ = (long long)(kBounceBytes / (row * sizeof(double)));
    if (per_buf_ < 1) per_buf_ = 1;
    if (per_buf_ > kStageChunk) per_buf_ = kStageChunk;
  }

  ~RowStreamer()
  {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
    if (copy_) cudaStreamDestroy(copy_);
    for (auto& b : buf_) {
      if (b.ev) cudaEventDestroy(b.ev);
      bounce_put(b.rows);
      if (b.idx) cudaFreeHost(b.idx);
    }
    if (ready_h_) cudaFreeHost(ready_h_);
  }

  cudaError_t start()
  {
    cudaError_t e = cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    if ((e = cudaMallocHost(&ready_h_, nchunk_ * sizeof(unsigned))) != cudaSuccess) return e;
    for (auto& b : buf_) {
      void* p = nullptr;
      if ((e = bounce_get(&p, kBounceBytes)) != cudaSuccess) return e;
      b.rows = static_cast<double*>(p);
      if ((e = cudaMallocHost(&b.idx, per_buf_ * sizeof(int))) != cudaSuccess) return e;
      if ((e = cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming)) != cudaSuccess) return e;
    }
    unsigned nt = std::thread::hardware_concurrency();
    nworkers_ = nt < 2 ? 1 : (nt > 16 ? 16 : (int)nt);
    for (int k = 0; k < nworkers_; k++) workers_.emplace_back([this] { work(); });
    return cudaSuccess;
  }

  // Issue the copies of finished chunks and hand finished copies to the
  // workers; returns whether every orbit has been delivered.
  cudaError_t poll(bool& all_done)
  {
    cudaError_t e;
    if (issued_total_ < nobj_) {
      if ((e = cudaMemcpyAsync(ready_h_, st_.ready, nchunk_ * sizeof(unsigned),
                               cudaMemcpyDeviceToHost, side_)) != cudaSuccess)
        return e;
      if ((e = cudaStreamSynchronize(side_)) != cudaSuccess) return e;
    }
    for (auto& b : buf_) {
      if (b.state != 1) continue;
      e = cudaEventQuery(b.ev);
      if (e == cudaErrorNotReady) continue;
      if (e != cudaSuccess) return e;
      b.state = 2;
      enqueue(b);
    }
    // copies of complete chunks, lowest chunk first
    while (scan_ < nchunk_ && issued_[scan_] == chunk_size(scan_)) scan_++;
    int c = scan_;
    for (auto& b : buf_) {
      if (issued_total_ >= nobj_) break;
      if (b.state != 0) continue;
      while (c < nchunk_ && (issued_[c] == chunk_size(c) || ready_h_[c] < (unsigned)chunk_size(c)))
        c++;
      if (c >= nchunk_) break;
      const long long first = (long long)c * kStageChunk + issued_[c];
      const long long n = std::min<long long>(per_buf_, chunk_size(c) - issued_[c]);
      if ((e = cudaMemcpyAsync(b.rows, rows_ + first * row_, n * row_ * sizeof(double),
                               cudaMemcpyDeviceToHost, copy_)) != cudaSuccess)
        return e;
      if ((e = cudaMemcpyAsync(b.idx, st_.idx + first, n * sizeof(int),
                               cudaMemcpyDeviceToHost, copy_)) != cudaSuccess)
        return e;
      if ((e = cudaEventRecord(b.ev, copy_)) != cudaSuccess) return e;
      b.count = n;
      b.state = 1;
      issued_[c] += (int)n;
      issued_total_ += n;
    }
    all_done = issued_total_ >= nobj_ && delivered_.load() >= nobj_;
    return cudaSuccess;
  }

 private:
  int chunk_size(int c) const
  {
    return (int)std::min<long long>(kStageChunk, nobj_ - (long long)c * kStageChunk);
  }

  struct Buf {
    double* rows = nullptr;
    int* idx = nullptr;
    cudaEvent_t ev = nullptr;
    long long count = 0;
    std::atomic<int> state{0};  // 0 free, 1 copying, 2 scattering (workers free it)
    std::atomic<int> parts{0};
  };
  struct Job {
    Buf* b;
    long long k0, k1;
  };

  void enqueue(Buf& b)
  {
    const int parts = (int)std::min<long long>(nworkers_, b.count);
    b.parts.store(parts);
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (int p = 0; p < parts; p++)
        jobs_.push_back({&b, b.count * p / parts, b.count * (p + 1) / parts});
    }
    cv_.notify_all();
  }

  void work()
  {
    for (;;) {
      Job j;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [this] { return stop_ || !jobs_.empty(); });
        if (jobs_.empty()) return;
        j = jobs_.back();
        jobs_.pop_back();
      }
      for (long long k = j.k0; k < j.k1; k++)
        memcpy(result_ + (size_t)j.b->idx[k] * row_, j.b->rows + (size_t)k * row_,
               row_ * sizeof(double));
      delivered_.fetch_add(j.k1 - j.k0);
      if (j.b->parts.fetch_sub(1) == 1) j.b->state = 0;  // the buffer is free again
    }
  }

  Staging st_;
  const double* rows_;
  long long nobj_;
  size_t row_;
  double* result_;
  cudaStream_t side_, copy_ = nullptr;
  int nchunk_ = 0, nworkers_ = 1;
  long long per_buf_ = 1, issued_total_ = 0;
  std::vector<int> issued_;  // positions of each chunk whose copy is issued
  int scan_ = 0;             // chunks below are fully issued
  unsigned* ready_h_ = nullptr;
  Buf buf_[kBuffers];
  std::vector<std::thread> workers_;
  std::vector<Job> jobs_;
  std::mutex mu_;
  std::condition_variable cv_;
  bool stop_ = false;
  std::atomic<long long> delivered_{0};
};

// Streaming pays off when the result is large (its transfer is then a
// sizeable part of the call) and spans several chunks.
static bool stream_rows_for(long long nobj, size_t n_out)
{
  return nobj >= 4LL * kStageChunk && n_out * sizeof(double) >= (size_t)(256u << 20);
}

// One device's share of a multi-device blocking call.  The caller's thread
// holds the SIGINT handler and drives the progress callback from the orbit
// counts each device reports; a device that fails raises `stop`, which the
// others forward to their kernels like a SIGINT.
struct SplitCtl {
  std::atomic<unsigned long long> done{0};
  std::atomic<int>* stop = nullptr;
};

// Blocking host-pointer integration shared by the galpy-facing entry points.
// One potential's records (a component may take continuation records: an
// SCF expansion's coefficients).
static int compile_records(int planar, int /*var*/, int npot, const int* pot_type,
                           const double* pot_args, std::vector<GpComp>& comps)
{
  const int n = group_records(planar, npot, pot_type, pot_args);
  if (n == -3) return set_error(GALPY_CUDA_ERR_POTENTIAL, "potential type not implemented on the GPU");
  if (n < 1) return set_error(GALPY_CUDA_ERR_ARG, "invalid potential arguments");
  comps.assign((size_t)n, GpComp{});
  const int rc = compile_group(planar, npot, pot_type, pot_args, comps.data(), nullptr);
  if (rc == -3) return set_error(GALPY_CUDA_ERR_POTENTIAL, "potential type not implemented on the GPU");
  if (rc) return set_error(GALPY_CUDA_ERR_ARG, "invalid potential arguments");
  return GALPY_CUDA_OK;
}

// w: rectangular initial states [nobj][nv]; result written in galpy's layout
// (cylindrical rows) unless rect_out.
static int run_host(int planar, int var, long long nobj, const double* w, int nv, int nt,
                    const double* t, int indiv_t, int npot, const int* pot_type,
                    const double* pot_args, double dt, double rtol, double atol, double* result,
                    int* err, int odeint_type, galpy_cuda_callback cb, const galpy_cuda_opts* o,
                    bool rect_out, int system = GALPY_CUDA_SYS_ORBIT, SplitCtl* ctl = nullptr)
{
  int rc = select_device(o);
  if (rc) return rc;
  if (!method_supported(odeint_type))
    return set_error(GALPY_CUDA_ERR_METHOD, "odeint_type not implemented on the GPU");
  if (nobj == 0) return GALPY_CUDA_OK;
  std::vector<GpComp> comps;
  rc = compile_records(planar, var, npot, pot_type, pot_args, comps);
  if (rc) return rc;
  cudaMemPool_t pool = nullptr;
  rc = library_pool(&pool);
  if (rc) return rc;

  cudaStream_t stream, side;
  GPC_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  GPC_CUDA_TRY(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t a, b;
    ~StreamGuard()
    {
      cudaStreamSynchronize(a);
      cudaStreamDestroy(a);
      cudaStreamDestroy(b);
    }
  } sg{stream, side};

  const size_t n_w = (size_t)nobj * nv, n_t = (size_t)(indiv_t ? nobj : 1) * nt;
  const size_t n_out = (size_t)nobj * nt * nv;
  DevBuf dw, dt_, dout, derr, dsteps, dcomp, dscr;
  dw.s = dt_.s = dout.s = derr.s = dsteps.s = dcomp.s = dscr.s = stream;
  GPC_CUDA_TRY(alloc_async(&dw.p, n_w * sizeof(double), pool, stream));
  GPC_CUDA_TRY(alloc_async(&dt_.p, n_t * sizeof(double), pool, stream));
  GPC_CUDA_TRY(alloc_async(&dout.p, n_out * sizeof(double), pool, stream));
  GPC_CUDA_TRY(alloc_async(&derr.p, (size_t)nobj * sizeof(int), pool, stream));
  GPC_CUDA_TRY(alloc_async(&dcomp.p, comps.size() * sizeof(GpComp), pool, stream));
  GPC_CUDA_TRY(alloc_async(&dscr.p, sizeof(Scratch), pool, stream));
  if (o && o->nsteps) GPC_CUDA_TRY(alloc_async(&dsteps.p, (size_t)nobj * sizeof(long long), pool, stream));
  // streaming of finished orbits (RowStreamer; the output then holds the
  // rows in work-queue order): the orbit at each output position, per-chunk
  // counts of complete positions, per-position writer counts
  const int stream_opt =
      o && o->size >= (int)(offsetof(galpy_cuda_opts, stream_rows) + sizeof(int))
          ? o->stream_rows
          : -1;
  const bool stream_rows = stream_opt == 1 || (stream_opt < 0 && stream_rows_for(nobj, n_out));
  DevBuf sidx, sready, spend;
  sidx.s = sready.s = spend.s = stream;
  Staging stg;
  if (stream_rows) {
    const size_t nchunk = (size_t)((nobj + kStageChunk - 1) / kStageChunk);
    GPC_CUDA_TRY(alloc_async(&sidx.p, (size_t)nobj * sizeof(int), pool, stream));
    GPC_CUDA_TRY(alloc_async(&sready.p, nchunk * sizeof(unsigned), pool, stream));
    GPC_CUDA_TRY(alloc_async(&spend.p, (size_t)nobj * sizeof(int), pool, stream));
    GPC_CUDA_TRY(cudaMemsetAsync(sready.p, 0, nchunk * sizeof(unsigned), stream));
    stg.idx = static_cast<int*>(sidx.p);
    stg.ready = static_cast<unsigned*>(sready.p);
    stg.pend = static_cast<int*>(spend.p);
  }
  GPC_CUDA_TRY(cudaMemcpyAsync(dw.p, w, n_w * sizeof(double), cudaMemcpyHostToDevice, stream));
  GPC_CUDA_TRY(cudaMemcpyAsync(dt_.p, t, n_t * sizeof(double), cudaMemcpyHostToDevice, stream));
  GPC_CUDA_TRY(cudaMemcpyAsync(dcomp.p, comps.data(), comps.size() * sizeof(GpComp),
                               cudaMemcpyHostToDevice, stream));

  galpy_cuda_launch L;
  memset(&L, 0, sizeof(L));
  L.planar = planar;
  L.variational = var;
  L.odeint_type = odeint_type;
  L.precision = o ? o->precision : GALPY_CUDA_FP64;
  L.nobj = nobj;
  L.nt = nt;
  L.indiv_t = indiv_t;
  L.t = static_cast<double*>(dt_.p);
  L.w0 = static_cast<double*>(dw.p);
  L.in_layout = GALPY_CUDA_IN_AOS;
  L.out = static_cast<double*>(dout.p);
  L.out_layout = rect_out ? GALPY_CUDA_OUT_AOS_RECT : GALPY_CUDA_OUT_GALPY;
  L.out_row0 = 0;
  L.err = static_cast<int*>(derr.p);
  L.nsteps = static_cast<long long*>(dsteps.p);
  L.comps = dcomp.p;
  L.comps_host = comps.data();
  L.ncomp = (int)comps.size();
  L.dt = dt;
  L.rtol = rtol;
  L.atol = atol;
  L.max_attempts = o ? o->max_attempts : 0;
  L.block_size = o ? o->block_size : 0;
  L.signature = signature_of(npot, pot_type);
  const bool has_sched = o && o->size >= (int)(offsetof(galpy_cuda_opts, schedule) + sizeof(int));
  L.schedule = has_sched ? o->schedule : GALPY_CUDA_SCHED_LONGEST_FIRST;
  L.variant = has_sched ? o->variant : 0;
  L.size_ext = 2;
  L.tail_sms = -1;
  L.system = system;
  rc = check_launch(&L);
  if (rc) return rc;

  Scratch* scr = static_cast<Scratch*>(dscr.p);
  cudaEvent_t e0, e1;
  GPC_CUDA_TRY(cudaEventCreate(&e0));
  GPC_CUDA_TRY(cudaEventCreate(&e1));
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard()
    {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } eg{e0, e1};
  SigintGuard sig(ctl == nullptr);
  RowStreamer streamer(stg, static_cast<const double*>(dout.p), nobj, (size_t)nt * nv, result,
                       side);
  if (stream_rows) GPC_CUDA_TRY(streamer.start());
  const bool track = cb != nullptr || ctl != nullptr;
  GPC_CUDA_TRY(cudaEventRecord(e0, stream));
  rc = launch_kernel(&L, scr, track, stream, pool, stream_rows ? &stg : nullptr);
  if (rc) return rc;
  GPC_CUDA_TRY(cudaEventRecord(e1, stream));

  // wait: poll completion, forward SIGINT to the device, drive the progress
  // callback, stream the finished orbits' rows to the result
  unsigned long long reported = 0, *pinned_done = nullptr;
  if (track) GPC_CUDA_TRY(cudaMallocHost(&pinned_done, sizeof(unsigned long long)));
  struct PinGuard {
    unsigned long long* p;
    ~PinGuard()
    {
      if (p) cudaFreeHost(p);
    }
  } pg{pinned_done};
  bool abort_sent = false, kernel_done = false, rows_done = !stream_rows;
  for (;;) {
    if (!kernel_done) {
      cudaError_t q = cudaEventQuery(e1);
      if (q == cudaSuccess)
        kernel_done = true;
      else if (q != cudaErrorNotReady)
        return set_error(GALPY_CUDA_ERR_CUDA,
                         std::string("integration kernel: ") + cudaGetErrorString(q));
    }
    if (stream_rows && !rows_done) {
      cudaError_t q = streamer.poll(rows_done);
      if (q != cudaSuccess)
        return set_error(GALPY_CUDA_ERR_CUDA,
                         std::string("result streaming: ") + cudaGetErrorString(q));
    }
    if (kernel_done && rows_done) break;
    if ((g_sigint || (ctl && ctl->stop->load())) && !abort_sent) {
      static const int one = 1;
      cudaMemcpyAsync(&scr->abort_flag, &one, sizeof(int), cudaMemcpyHostToDevice, side);
      abort_sent = true;
    }
    if (track && !kernel_done) {
      cudaMemcpyAsync(pinned_done, &scr->done_count, sizeof(unsigned long long),
                      cudaMemcpyDeviceToHost, side);
      cudaStreamSynchronize(side);
      if (ctl)
        ctl->done.store(*pinned_done);
      else
        for (; reported < *pinned_done; reported++) cb();
    }
    struct timespec ts = {0, stream_rows ? 500000 : 2000000};
    nanosleep(&ts, nullptr);
  }
  if (ctl)
    ctl->done.store((unsigned long long)nobj);
  else if (cb)
    for (; reported < (unsigned long long)nobj; reported++) cb();
  if (o && o->elapsed_ms) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    *o->elapsed_ms = ms;
  }
  if (!stream_rows)
    GPC_CUDA_TRY(cudaMemcpyAsync(result, dout.p, n_out * sizeof(double), cudaMemcpyDeviceToHost,
                                 stream));
  GPC_CUDA_TRY(cudaMemcpyAsync(err, derr.p, (size_t)nobj * sizeof(int), cudaMemcpyDeviceToHost, stream));
  if (o && o->nsteps)
    GPC_CUDA_TRY(cudaMemcpyAsync(o->nsteps, dsteps.p, (size_t)nobj * sizeof(long long),
                                 cudaMemcpyDeviceToHost, stream));
  GPC_CUDA_TRY(cudaStreamSynchronize(stream));
  if (abort_sent) return GALPY_CUDA_ERR_INTERRUPTED;
  return GALPY_CUDA_OK;
}

// ----------------------------------------------------------------------------
// one blocking call over several devices
// ----------------------------------------------------------------------------
// The orbits of a batch are independent, so a batch spread over devices needs
// no exchange: each device integrates a contiguous range of orbits, whose
// states, times and result rows are contiguous slices of the caller's arrays.
// The ranges hold equal shares of the estimated cost -- the longest-first
// estimate |t_end - t_0| * Omega(x_0) of cost_kernel, evaluated here on the
// host with the same force code -- rather than equal orbit counts, so that a
// batch ordered by energy or radius (a grid of orbits, say) still loads the
// devices evenly.  Within its range each device schedules longest-first as a
// one-device call does.

// Estimated cost of each orbit (cost_kernel's estimate; 1 for every orbit of
// a surface-of-section run, whose states are not positions).  group: the
// potential group of each orbit (comps holds ngroup * ncomp records), or null.
static void orbit_costs(int planar, long long nobj, const double* w, int nv, int nt,
                        const double* t, int indiv_t, const GpComp* comps, int ncomp,
                        const int* group, int system, double* cost)
{
  const int D = planar ? 2 : 3;
  auto one = [&](long long i) {
    if (system != GALPY_CUDA_SYS_ORBIT) return 1.0;
    double q[3] = {0.0, 0.0, 0.0}, a[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < D; k++) q[k] = w[i * nv + k];
    const GpComp* c = comps + (group ? (long long)group[i] * ncomp : 0LL);
    if (D == 3)
      eval_force<3, PREC_FP64, false, DynPot>(c, ncomp, q, a);
    else
      eval_force<2, PREC_FP64, false, DynPot>(c, ncomp, q, a);
    double ax = 0.0, xx = 0.0;
    for (int k = 0; k < D; k++) {
      ax += a[k] * q[k];
      xx += q[k] * q[k];
    }
    const double* tt = t + (indiv_t ? i * (long long)nt : 0LL);
    const double est = fabs(tt[nt - 1] - tt[0]) * sqrt(fabs(ax) / (xx > 0.0 ? xx : 1e-300));
    // a floor keeps orbits with a zero estimate (at the centre, or of zero
    // duration) from being free: each still costs its launch share
    return std::isfinite(est) ? est + 1e-3 : 1e-3;
  };
  const long long per = 1 << 15;
  const int nthr = (int)std::min<long long>(
      std::max(1u, std::min(std::thread::hardware_concurrency(), 32u)), (nobj + per - 1) / per);
  if (nthr <= 1) {
    for (long long i = 0; i < nobj; i++) cost[i] = one(i);
    return;
  }
  std::vector<std::thread> th;
  for (int k = 0; k < nthr; k++)
    th.emplace_back([&, k] {
      const long long a = nobj * k / nthr, b = nobj * (k + 1) / nthr;
      for (long long i = a; i < b; i++) cost[i] = one(i);
    });
  for (auto& x : th) x.join();
}

// Cut [0, nobj) into nparts contiguous ranges of equal cost: bounds[k] is the
// first orbit of part k (bounds[0] = 0, bounds[nparts] = nobj).  Part k ends
// where the running cost first reaches k+1 nparts-ths of the total; a part
// may be empty when single orbits dominate the cost.
static void cut_ranges(long long nobj, const double* cost, int nparts, long long* bounds)
{
  double total = 0.0;
  for (long long i = 0; i < nobj; i++) total += cost[i];
  bounds[0] = 0;
  long long i = 0;
  double run = 0.0;
  for (int k = 1; k < nparts; k++) {
    const double target = total * k / nparts;
    // take orbit i while that brings the running cost closer to the target
    while (i < nobj && run + 0.5 * cost[i] <= target) run += cost[i++];
    bounds[k] = i;
  }
  bounds[nparts] = nobj;
}

// The devices of a multi-device call (empty: one device, opts.device).
static int device_list(const galpy_cuda_opts* o, std::vector<int>& devs)
{
  devs.clear();
  const bool has = o && o->size >= (int)(offsetof(galpy_cuda_opts, devices) + sizeof(o->devices));
  if (!has || o->ndevices == 0 || o->ndevices == 1) return GALPY_CUDA_OK;
  if (o->ndevices < -1) return set_error(GALPY_CUDA_ERR_ARG, "invalid ndevices");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1)
    return set_error(GALPY_CUDA_ERR_NODEVICE, "no CUDA device visible");
  const int want = o->ndevices < 0 ? n : o->ndevices;
  for (int k = 0; k < want; k++) {
    const int d = o->ndevices > 0 && o->devices ? o->devices[k] : k;
    if (d < 0 || d >= n) return set_error(GALPY_CUDA_ERR_ARG, "device ordinal out of range");
    devs.push_back(d);  // a repeated ordinal runs several ranges concurrently on that device
  }
  return GALPY_CUDA_OK;
}

// run_host over the devices opts names: one thread per device, each running
// the one-device path on its range; this thread forwards SIGINT, reports
// progress and collects the first error.
static int run_host_split(int planar, int var, long long nobj, const double* w, int nv, int nt,
                          const double* t, int indiv_t, int npot, const int* pot_type,
                          const double* pot_args, double dt, double rtol, double atol,
                          double* result, int* err, int odeint_type, galpy_cuda_callback cb,
                          const galpy_cuda_opts* o, bool rect_out,
                          int system = GALPY_CUDA_SYS_ORBIT)
{
  std::vector<int> devs;
  int rc = device_list(o, devs);
  if (rc) return rc;
  if (devs.size() < 2 || nobj < (long long)devs.size())
    return run_host(planar, var, nobj, w, nv, nt, t, indiv_t, npot, pot_type, pot_args, dt, rtol,
                    atol, result, err, odeint_type, cb, o, rect_out, system);
  if (!method_supported(odeint_type))
    return set_error(GALPY_CUDA_ERR_METHOD, "odeint_type not implemented on the GPU");
  std::vector<GpComp> comps;
  rc = compile_records(planar, var, npot, pot_type, pot_args, comps);
  if (rc) return rc;

  const int nd = (int)devs.size();
  std::vector<double> cost((size_t)nobj);
  orbit_costs(planar, nobj, w, nv, nt, t, indiv_t, comps.data(), (int)comps.size(), nullptr, system,
              cost.data());
  std::vector<long long> bounds(nd + 1);
  cut_ranges(nobj, cost.data(), nd, bounds.data());

  std::atomic<int> stop{0};
  std::vector<SplitCtl> ctl(nd);
  std::vector<int> rcs(nd, GALPY_CUDA_OK);
  std::vector<std::string> msgs(nd);
  std::vector<double> ms(nd, 0.0);
  std::vector<std::atomic<int>> finished(nd);
  SigintGuard sig;
  std::vector<std::thread> th;
  for (int k = 0; k < nd; k++) {
    ctl[k].stop = &stop;
    finished[k].store(0);
    th.emplace_back([&, k] {
      const long long a = bounds[k], n = bounds[k + 1] - a;
      galpy_cuda_opts ok = *o;
      ok.size = (int)sizeof(galpy_cuda_opts);
      ok.device = devs[k];
      ok.ndevices = 0;
      ok.devices = nullptr;
      ok.nsteps = o->nsteps ? o->nsteps + a : nullptr;
      ok.elapsed_ms = &ms[k];
      int r = GALPY_CUDA_OK;
      if (n > 0)
        r = run_host(planar, var, n, w + a * nv, nv, nt, t + (indiv_t ? a * nt : 0), indiv_t,
                     npot, pot_type, pot_args, dt, rtol, atol, result + a * (long long)nt * nv,
                     err + a, odeint_type, nullptr, &ok, rect_out, system, &ctl[k]);
      ctl[k].done.store((unsigned long long)n);
      if (r != GALPY_CUDA_OK && r != GALPY_CUDA_ERR_INTERRUPTED) {
        msgs[k] = g_last_error;
        stop.store(1);
      }
      rcs[k] = r;
      finished[k].store(1);
    });
  }
  unsigned long long reported = 0;
  for (;;) {
    bool all = true;
    unsigned long long done = 0;
    for (int k = 0; k < nd; k++) {
      all = all && finished[k].load();
      done += ctl[k].done.load();
    }
    if (cb)
      for (; reported < done; reported++) cb();
    if (all) break;
    struct timespec ts = {0, 2000000};
    nanosleep(&ts, nullptr);
  }
  for (auto& x : th) x.join();
  if (cb)
    for (; reported < (unsigned long long)nobj; reported++) cb();
  if (o->elapsed_ms) *o->elapsed_ms = *std::max_element(ms.begin(), ms.end());
  for (int k = 0; k < nd; k++)
    if (rcs[k] != GALPY_CUDA_OK && rcs[k] != GALPY_CUDA_ERR_INTERRUPTED)
      return set_error(rcs[k], "device " + std::to_string(devs[k]) + ": " + msgs[k]);
  for (int k = 0; k < nd; k++)
    if (rcs[k] == GALPY_CUDA_ERR_INTERRUPTED) return GALPY_CUDA_ERR_INTERRUPTED;
  return GALPY_CUDA_OK;
}

// f(i0, i1) over [0, n) in contiguous pieces on up to 16 host threads (one
// thread below 65,536 items): the per-orbit coordinate conversions of large
// batches (1M orbits: ~40 ms of sin/cos on one core).
template <class F>
static void host_parallel_for(long long n, F f)
{
  const int nthr = n < 65536 ? 1 : (int)std::max(1u, std::min(std::thread::hardware_concurrency(), 16u));
  if (nthr <= 1) {
    f(0LL, n);
    return;
  }
  std::vector<std::thread> th;
  for (int k = 0; k < nthr; k++) th.emplace_back([&, k] { f(n * k / nthr, n * (k + 1) / nthr); });
  for (auto& x : th) x.join();
}

// (R, vR, vT, z, vz, phi, t) -> surface-of-section state (x, y, vx, vy, A,
// t, psi), in place, exactly as cyl_to_sos_galpy (bovy_coords.c:149-163)
static void cyl_to_sos_inplace(long long nobj, double* yo)
{
  host_parallel_for(nobj, [yo](long long i0, long long i1) {
    for (long long i = i0; i < i1; i++) {
      double* v = yo + 7 * i;
      const double R = v[0], cp = cos(v[5]), sp = sin(v[5]), vR = v[1], vT = v[2];
      v[5] = v[6];
      v[6] = atan2(v[3], v[4]);
      v[4] = sqrt(v[3] * v[3] + v[4] * v[4]);
      v[0] = R * cp;
      v[1] = R * sp;
      v[2] = vR * cp - vT * sp;
      v[3] = vR * sp + vT * cp;
    }
  });
}

// (R, vR, vT, phi, t) -> planar surface-of-section state, in place, exactly
// as polar_to_sos_galpy (bovy_coords.c:200-226): surface 1 (y = 0) gives
// (x, vx, A, t, psi), otherwise (x = 0) (y, vy, A, t, psi)
static void polar_to_sos_inplace(long long nobj, double* yo, int surface)
{
  host_parallel_for(nobj, [yo, surface](long long i0, long long i1) {
    for (long long i = i0; i < i1; i++) {
      double* v = yo + 5 * i;
      const double R = v[0], cp = cos(v[3]), sp = sin(v[3]), vR = v[1], vT = v[2];
      if (surface == 1) {
        v[0] = R * cp;
        v[1] = vR * cp - vT * sp;
        const double y = R * sp, vy = vR * sp + vT * cp;
        v[2] = sqrt(y * y + vy * vy);
        v[3] = v[4];
        v[4] = atan2(y, vy);
      } else {
        v[0] = R * sp;
        v[1] = vR * sp + vT * cp;
        const double x = R * cp, vx = vR * cp - vT * sp;
        v[2] = sqrt(x * x + vx * vx);
        v[3] = v[4];
        v[4] = atan2(x, vx);
      }
    }
  });
}

// cylindrical -> rectangular initial conditions, in place, exactly as
// cyl_to_rect_galpy / polar_to_rect_galpy (bovy_coords.c:57-124)
static void cyl_to_rect_inplace(int planar, long long nobj, double* yo)
{
  host_parallel_for(nobj, [yo, planar](long long i0, long long i1) {
    for (long long i = i0; i < i1; i++) {
      double* v = yo + (planar ? 4 : 6) * i;
      if (planar) {
        const double R = v[0], phi = v[3], cp = cos(phi), sp = sin(phi), vR = v[1], vT = v[2];
        v[0] = R * cp;
        v[1] = R * sp;
        v[2] = vR * cp - vT * sp;
        v[3] = vR * sp + vT * cp;
      } else {
        const double R = v[0], phi = v[5], cp = cos(phi), sp = sin(phi), vR = v[1], vT = v[2];
        v[0] = R * cp;
        v[1] = R * sp;
        v[2] = v[3];
        v[5] = v[4];
        v[3] = vR * cp - vT * sp;
        v[4] = vR * sp + vT * cp;
      }
    }
  });
}

// ----------------------------------------------------------------------------
// energies of stored states (output-side check of the integrations)
// ----------------------------------------------------------------------------
// E = v^2/2 + Phi(x), minus Omega . (x cross v) when Omega is not zero (the
// Jacobi integral in a frame rotating with pattern speed Omega).
__global__ void __launch_bounds__(256) energy_kernel(const GpComp* comps, int ncomp,
                                                     const int* group, int planar,
                                                     const double* w, long long n, long long sc,
                                                     long long so, double ox, double oy,
                                                     double oz, double* E)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* v = w + i * so;
  const GpComp* c = comps + (group ? (long long)group[i] * ncomp : 0LL);
  double x, y, z, vx, vy, vz;
  if (planar) {
    x = v[0];
    y = v[sc];
    z = 0.0;
    vx = v[2 * sc];
    vy = v[3 * sc];
    vz = 0.0;
  } else {
    x = v[0];
    y = v[sc];
    z = v[2 * sc];
    vx = v[3 * sc];
    vy = v[4 * sc];
    vz = v[5 * sc];
  }
  double e = 0.5 * (vx * vx + vy * vy + vz * vz) + potential_value(c, ncomp, x, y, z);
  if (ox != 0.0 || oy != 0.0 || oz != 0.0)
    e -= ox * (y * vz - z * vy) + oy * (z * vx - x * vz) + oz * (x * vy - y * vx);
  E[i] = e;
}

// Accelerations at points (positions SoA [3][n], z ignored when planar) with
// the integrators' own force code: run-time component list, or the
// compile-time MWPotential2014 list when mw14 (the headline kernels' path).
template <class POT, int PREC>
__global__ void __launch_bounds__(256) accel_kernel(const GpComp* comps, int ncomp,
                                                    const int* group, int planar,
                                                    const double* pos, long long n, double* acc)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const GpComp* c = comps + (group ? (long long)group[i] * ncomp : 0LL);
  const double q[3] = {pos[i], pos[n + i], planar ? 0.0 : pos[2 * n + i]};
  double a[3] = {0.0, 0.0, 0.0};
  if (planar)
    eval_force<2, PREC, false, POT>(c, ncomp, q, a);
  else
    eval_force<3, PREC, false, POT>(c, ncomp, q, a);
  acc[i] = a[0];
  acc[n + i] = a[1];
  acc[2 * n + i] = a[2];
}

// ----------------------------------------------------------------------------
// FP64 pipe peak: independent fused multiply-add chains per thread
// ----------------------------------------------------------------------------
__global__ void __launch_bounds__(256) fp64_fma_peak_kernel(double* sink, int iters, double mul)
{
  double a0 = 1e-3 * threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4,
         a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  const double add = 1e-9;
  for (int i = 0; i < iters; i++) {
    a0 = fma(a0, mul, add);
    a1 = fma(a1, mul, add);
    a2 = fma(a2, mul, add);
    a3 = fma(a3, mul, add);
    a4 = fma(a4, mul, add);
    a5 = fma(a5, mul, add);
    a6 = fma(a6, mul, add);
    a7 = fma(a7, mul, add);
  }
  const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.678) sink[threadIdx.x] = s;  // keeps the chains alive
}

// ----------------------------------------------------------------------------
// Allocation-free variant of the device entry point
// ----------------------------------------------------------------------------
// galpy_cuda_integrate_device allocates its scratch (the work-stealing
// counter and the longest-first work queue) with cudaMallocAsync on every
// call.  Some callers cannot let a library allocate: applications that run
// the integrator inside a loop that must not touch the CUDA allocator (an
// allocation can implicitly synchronise the device, or grow a memory pool the
// application has sized and locked for its own use), and embedding hosts
// whose allocation policy forbids third-party device allocations.  For them,
// galpy_cuda_integrate_device_noalloc keeps all of its scratch in the fixed
// array below, which is part of the loaded module: every GPU that loads the
// library holds these ~5 MiB until the process exits.
constexpr long long kNoAllocMaxOrbits = 1LL << 20;  // largest batch it accepts
constexpr int kNoAllocBuckets = 64;                 // cost buckets of the work queue
constexpr size_t kNoAllocCtl = 0;                   // Scratch control words
constexpr size_t kNoAllocCount = 256;               // unsigned[64] bucket sizes
constexpr size_t kNoAllocNext = 512;                // unsigned[64] bucket fill positions
constexpr size_t kNoAllocBucket = 1024;             // unsigned char[max] bucket of each orbit
constexpr size_t kNoAllocOrder = kNoAllocBucket + kNoAllocMaxOrbits;  // int[max] work queue
constexpr size_t kNoAllocBytes = kNoAllocOrder + 4 * kNoAllocMaxOrbits;
static_assert(sizeof(Scratch) <= kNoAllocCount, "control block too large");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch, looked up once per device and
// context (host code must not use the symbol itself: on the host it is only
// a stand-in for the device object).  The cache is keyed on the context as
// well as the ordinal: after cudaDeviceReset the module is loaded again into
// a new primary context, possibly at another address, and the next call
// looks the array up again instead of using a stale pointer.
static std::mutex g_noalloc_mutex;
static void* g_noalloc_ptr[64] = {nullptr};
static CUcontext g_noalloc_ctx[64] = {nullptr};

static int noalloc_scratch(void** out)
{
  int dev = 0;
  GPC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(GALPY_CUDA_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  CUcontext ctx = current_context();
  if (!g_noalloc_ptr[dev] || !ctx || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return set_error(GALPY_CUDA_ERR_CUDA,
                       std::string("cudaGetSymbolAddress(noalloc scratch): ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = p;
    g_noalloc_ctx[dev] = current_context();  // the lookup made the primary context current
  }
  *out = g_noalloc_ptr[dev];
  return GALPY_CUDA_OK;
}

// Bucketed longest-first order without a sort: bucket = 4 log2(1 + cost)
// (64 buckets, largest cost first), counted, scanned and scattered.
template <int D>
__global__ void __launch_bounds__(256) noalloc_bucket_kernel(const KArgs A, unsigned char* scr)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= A.nobj) return;
  double q[3] = {0.0, 0.0, 0.0}, a[3] = {0.0, 0.0, 0.0};
  const int nv = A.variational_nv ? A.variational_nv : 2 * D;
  for (int k = 0; k < D; k++)
    q[k] = A.in_layout == GALPY_CUDA_IN_SOA ? A.w0[(long long)k * A.nobj + i] : A.w0[i * nv + k];
  const GpComp* comps = A.comps + (A.group ? (long long)A.group[i] * A.ncomp : 0LL);
  eval_force<D, PREC_FP64, false, DynPot>(comps, A.ncomp, q, a);
  double ax = 0.0, xx = 0.0;
  for (int k = 0; k < D; k++) {
    ax += a[k] * q[k];
    xx += q[k] * q[k];
  }
  const double* tt = A.t + (A.indiv_t ? i * (long long)A.nt : 0LL);
  const double cost = fabs(tt[A.nt - 1] - tt[0]) * sqrt(fabs(ax) / (xx > 0.0 ? xx : 1e-300));
  int b = isfinite(cost) ? (int)(4.0 * log2(1.0 + cost)) : 0;
  b = b < 0 ? 0 : (b > kNoAllocBuckets - 1 ? kNoAllocBuckets - 1 : b);
  const int key = kNoAllocBuckets - 1 - b;  // descending cost
  scr[kNoAllocBucket + i] = (unsigned char)key;
  atomicAdd(reinterpret_cast<unsigned*>(scr + kNoAllocCount) + key, 1u);
}

__global__ void noalloc_scan_kernel(unsigned char* scr)
{
  if (threadIdx.x != 0) return;
  const unsigned* count = reinterpret_cast<const unsigned*>(scr + kNoAllocCount);
  unsigned* next = reinterpret_cast<unsigned*>(scr + kNoAllocNext);
  unsigned s = 0;
  for (int b = 0; b < kNoAllocBuckets; b++) {
    next[b] = s;
    s += count[b];
  }
}

__global__ void __launch_bounds__(256) noalloc_scatter_kernel(long long n, unsigned char* scr)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int key = scr[kNoAllocBucket + i];
  const unsigned pos = atomicAdd(reinterpret_cast<unsigned*>(scr + kNoAllocNext) + key, 1u);
  reinterpret_cast<int*>(scr + kNoAllocOrder)[pos] = (int)i;
}

// ----------------------------------------------------------------------------
// exported C ABI
// ----------------------------------------------------------------------------
extern "C" {

int galpy_cuda_energy_device(const void* comps, int ncomp, const int* group, int planar,
                             const double* w, long long n, long long comp_stride,
                             long long orbit_stride, double* E, void* stream)
{
  if (!comps || !w || !E || n < 0 || ncomp < 1 || ncomp > kMaxComp)
    return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  if (n == 0) return GALPY_CUDA_OK;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  energy_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const GpComp*>(comps), ncomp, group, planar, w, n, comp_stride, orbit_stride,
      0.0, 0.0, 0.0, E);
  GPC_CUDA_TRY(cudaGetLastError());
  return GALPY_CUDA_OK;
}

int galpy_cuda_jacobi_device(const void* comps, int ncomp, const int* group, int planar,
                             const double* w, long long n, long long comp_stride,
                             long long orbit_stride, const double* omega, double* J,
                             void* stream)
{
  if (!comps || !w || !J || !omega || n < 0 || ncomp < 1 || ncomp > kMaxComp)
    return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  if (n == 0) return GALPY_CUDA_OK;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  // planar states have no z: only the z component of Omega acts on them
  energy_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const GpComp*>(comps), ncomp, group, planar, w, n, comp_stride, orbit_stride,
      planar ? 0.0 : omega[0], planar ? 0.0 : omega[1], omega[2], J);
  GPC_CUDA_TRY(cudaGetLastError());
  return GALPY_CUDA_OK;
}

int galpy_cuda_accel_device(const void* comps, int ncomp, const int* group, int planar,
                            int signature, int precision, const double* pos, long long n,
                            double* acc, void* stream)
{
  if (!comps || !pos || !acc || n < 0 || ncomp < 1 || ncomp > kMaxComp)
    return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  if (precision < GALPY_CUDA_FP64 || precision > GALPY_CUDA_F32FORCE_DF)
    return set_error(GALPY_CUDA_ERR_ARG, "unknown precision");
  const bool mw14 = signature == GALPY_CUDA_SIG_MW14 && ncomp == 3;
  if ((precision == GALPY_CUDA_F64_TAIL32 || precision == GALPY_CUDA_F32BULGE) && !mw14)
    return set_error(GALPY_CUDA_ERR_METHOD,
                     "the mixed float64/float32 forces are built for MWPotential2014 only");
  if (n == 0) return GALPY_CUDA_OK;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const GpComp* c = static_cast<const GpComp*>(comps);
  if (precision == GALPY_CUDA_F64_TAIL32) {
    accel_kernel<MW14MixedPot<false, MIX_TAIL32>, PREC_FP64>
        <<<blocks, 256, 0, s>>>(c, ncomp, group, planar, pos, n, acc);
  } else if (precision == GALPY_CUDA_F32BULGE) {
    accel_kernel<MW14MixedPot<false, MIX_F32BULGE>, PREC_FP64>
        <<<blocks, 256, 0, s>>>(c, ncomp, group, planar, pos, n, acc);
  } else if (precision == GALPY_CUDA_FP64) {
    if (mw14)
      accel_kernel<MW14GroupPot, PREC_FP64><<<blocks, 256, 0, s>>>(c, ncomp, group, planar, pos, n, acc);
    else
      accel_kernel<DynPot, PREC_FP64><<<blocks, 256, 0, s>>>(c, ncomp, group, planar, pos, n, acc);
  } else {
    if (mw14)
      accel_kernel<MW14GroupPot, PREC_F32><<<blocks, 256, 0, s>>>(c, ncomp, group, planar, pos, n, acc);
    else
      accel_kernel<DynPot, PREC_F32><<<blocks, 256, 0, s>>>(c, ncomp, group, planar, pos, n, acc);
  }
  GPC_CUDA_TRY(cudaGetLastError());
  return GALPY_CUDA_OK;
}

int galpy_cuda_fp64_peak(double* tflops, double* ms)
{
  int dev = 0, nsm = 0;
  GPC_CUDA_TRY(cudaGetDevice(&dev));
  GPC_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  double* sink = nullptr;
  GPC_CUDA_TRY(cudaMalloc(&sink, 256 * sizeof(double)));
  const int blocks = nsm * 8, threads = 256, iters = 1 << 16;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(e0);
    fp64_fma_peak_kernel<<<blocks, threads>>>(sink, iters, 0.9999999);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (rep > 0 && t < best) best = t;
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (e != cudaSuccess) return set_error(GALPY_CUDA_ERR_CUDA, cudaGetErrorString(e));
  const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
  if (tflops) *tflops = flops / (best * 1e-3) / 1e12;
  if (ms) *ms = best;
  return GALPY_CUDA_OK;
}

int galpy_cuda_abi_version(void) { return GALPY_CUDA_ABI_VERSION; }

const char* galpy_cuda_last_error(void) { return g_last_error.c_str(); }

int galpy_cuda_device_count(void)
{
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int galpy_cuda_trim_memory(int device)
{
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1)
    return set_error(GALPY_CUDA_ERR_NODEVICE, "no CUDA device visible");
  int prev = 0;
  GPC_CUDA_TRY(cudaGetDevice(&prev));
  const int first = device >= 0 ? device : 0, last = device >= 0 ? device : n - 1;
  if (first >= n) return set_error(GALPY_CUDA_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  for (int d = first; d <= last && d < 64; d++) {
    if (!g_pool[d]) continue;
    GPC_CUDA_TRY(cudaSetDevice(d));
    // only the pool of the context it was made in (a reset dropped it)
    if (current_context() == g_pool_ctx[d]) {
      GPC_CUDA_TRY(cudaDeviceSynchronize());
      GPC_CUDA_TRY(cudaMemPoolTrimTo(g_pool[d], 0));
    }
  }
  GPC_CUDA_TRY(cudaSetDevice(prev));
  return GALPY_CUDA_OK;
}

int galpy_cuda_comp_size(void) { return (int)sizeof(GpComp); }

int galpy_cuda_signature(int npot, const int* pot_type)
{
  if (!pot_type || npot < 1) return GALPY_CUDA_SIG_GENERIC;
  return signature_of(npot, pot_type);
}

int galpy_cuda_comp_records(int planar, int npot, const int* pot_type, const double* pot_args)
{
  if (!pot_type || !pot_args) return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  const int n = group_records(planar, npot, pot_type, pot_args);
  if (n == -3) return set_error(GALPY_CUDA_ERR_POTENTIAL, "potential type not implemented on the GPU");
  if (n < 1) return set_error(GALPY_CUDA_ERR_ARG, "invalid potential arguments");
  return n;
}

int galpy_cuda_compile_potential(int planar, int npot, const int* pot_type,
                                 const double* pot_args, int ngroup, void* out)
{
  if (!pot_type || !pot_args || !out || ngroup < 1)
    return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  GpComp* c = static_cast<GpComp*>(out);
  const double* p = pot_args;
  const int nrec = group_records(planar, npot, pot_type, pot_args);
  if (nrec == -3) return set_error(GALPY_CUDA_ERR_POTENTIAL, "potential type not implemented on the GPU");
  if (nrec < 1) return set_error(GALPY_CUDA_ERR_ARG, "invalid potential arguments");
  for (int g = 0; g < ngroup; g++) {
    int used = 0;
    if (group_records(planar, npot, pot_type, p) != nrec)  // groups share one stride
      return set_error(GALPY_CUDA_ERR_ARG, "parameter groups of different sizes");
    int rc = compile_group(planar, npot, pot_type, p, c + (size_t)g * nrec, &used);
    if (rc == -3) return set_error(GALPY_CUDA_ERR_POTENTIAL, "potential type not implemented on the GPU");
    if (rc) return set_error(GALPY_CUDA_ERR_ARG, "invalid potential arguments");
    p += used;
  }
  share_tables(c, ngroup * nrec);
  return GALPY_CUDA_OK;
}

int galpy_cuda_split_orbits(int planar, long long nobj, const double* w, int nv, int nt,
                            const double* t, int indiv_t, int npot, const int* pot_type,
                            const double* pot_args, int ngroup, const int* group, int nparts,
                            long long* bounds)
{
  if (nobj < 0 || nt < 1 || nparts < 1 || nv < (planar ? 4 : 6) || !bounds ||
      (nobj && (!w || !t)) || npot < 1 || !pot_type || !pot_args || ngroup < 1 ||
      (ngroup > 1 && !group))
    return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  if (group)
    for (long long i = 0; i < nobj; i++)
      if (group[i] < 0 || group[i] >= ngroup)
        return set_error(GALPY_CUDA_ERR_ARG, "group index out of range");
  const int nrec = galpy_cuda_comp_records(planar, npot, pot_type, pot_args);
  if (nrec < 0) return nrec;
  std::vector<GpComp> comps((size_t)nrec * ngroup);
  const int rc = galpy_cuda_compile_potential(planar, npot, pot_type, pot_args, ngroup,
                                              comps.data());
  if (rc) return rc;
  std::vector<double> cost((size_t)nobj);
  orbit_costs(planar, nobj, w, nv, nt, t, indiv_t, comps.data(), nrec, group,
              GALPY_CUDA_SYS_ORBIT, cost.data());
  cut_ranges(nobj, cost.data(), nparts, bounds);
  return GALPY_CUDA_OK;
}

int galpy_cuda_integrate_device(const galpy_cuda_launch* L)
{
  int rc = check_launch(L);
  if (rc) return rc;
  if (L->nobj == 0) return GALPY_CUDA_OK;
  cudaStream_t s = static_cast<cudaStream_t>(L->stream);
  Scratch* scr = nullptr;
  GPC_CUDA_TRY(cudaMallocAsync((void**)&scr, sizeof(Scratch), s));
  rc = launch_kernel(L, scr, false, s);
  cudaFreeAsync(scr, s);
  return rc;
}

int galpy_cuda_integrate_device_noalloc(const galpy_cuda_launch* L)
{
  int rc = check_launch(L);
  if (rc) return rc;
  if (L->nobj > kNoAllocMaxOrbits)
    return set_error(GALPY_CUDA_ERR_ARG,
                     "galpy_cuda_integrate_device_noalloc: nobj = " + std::to_string(L->nobj) +
                         " exceeds its fixed scratch of " + std::to_string(kNoAllocMaxOrbits) +
                         " orbits; split the batch or use galpy_cuda_integrate_device");
  if (L->nobj == 0) return GALPY_CUDA_OK;
  void* base = nullptr;
  rc = noalloc_scratch(&base);
  if (rc) return rc;
  unsigned char* scr = static_cast<unsigned char*>(base);
  Scratch* ctl = reinterpret_cast<Scratch*>(scr + kNoAllocCtl);
  cudaStream_t stream = static_cast<cudaStream_t>(L->stream);
  KernelInfo ki;
  KArgs A;
  rc = prepare_launch(L, ctl, false, ki, A);
  if (rc) return rc;
  // the array keeps the previous call's contents: zero the control words
  // and the bucket counters (a memset, not an allocation)
  GPC_CUDA_TRY(cudaMemsetAsync(scr, 0, kNoAllocBucket, stream));
  if (L->schedule == GALPY_CUDA_SCHED_LONGEST_FIRST && L->nobj > 1 &&
      launch_system(L) == GALPY_CUDA_SYS_ORBIT) {
    const unsigned nb = (unsigned)((L->nobj + 255) / 256);
    if (L->planar)
      noalloc_bucket_kernel<2><<<nb, 256, 0, stream>>>(A, scr);
    else
      noalloc_bucket_kernel<3><<<nb, 256, 0, stream>>>(A, scr);
    noalloc_scan_kernel<<<1, 32, 0, stream>>>(scr);
    noalloc_scatter_kernel<<<nb, 256, 0, stream>>>(L->nobj, scr);
    GPC_CUDA_TRY(cudaGetLastError());
    A.order = reinterpret_cast<const int*>(scr + kNoAllocOrder);
  }
  return launch_persistent(L, ki, A, stream);
}

int integrateFullOrbit_cuda(int nobj, double* yo, int nt, double* t, int indiv_t, int npot,
                            int* pot_type, double* pot_args, void* /*pot_tfuncs*/, double dt,
                            double rtol, double atol, double* result, int* err, int odeint_type,
                            galpy_cuda_callback cb, const galpy_cuda_opts* opts)
{
  if (nobj < 0 || nt < 1 || (nobj && (!yo || !t || !result || !err)) || !pot_type || !pot_args)
    return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  if (!method_supported(odeint_type))
    return set_error(GALPY_CUDA_ERR_METHOD, "odeint_type not implemented on the GPU");
  cyl_to_rect_inplace(0, nobj, yo);
  return run_host_split(0, 0, nobj, yo, 6, nt, t, indiv_t, npot, pot_type, pot_args, dt, rtol, atol,
                  result, err, odeint_type, cb, opts, false);
}

int integrateFullOrbit_sos_cuda(int nobj, double* yo, int npsi, double* psi, int indiv_psi,
                                int npot, int* pot_type, double* pot_args, void* /*pot_tfuncs*/,
                                double dpsi, double rtol, double atol, double* result, int* err,
                                int odeint_type, galpy_cuda_callback cb,
                                const galpy_cuda_opts* opts)
{
  if (nobj < 0 || npsi < 1 || (nobj && (!yo || !psi || !result || !err)) || !pot_type ||
      !pot_args)
    return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  if (odeint_type != M_RK4 && odeint_type != M_RK6 && odeint_type != M_DOPR54 &&
      odeint_type != M_DOP853)
    return set_error(GALPY_CUDA_ERR_METHOD,
                     "surface-of-section integration takes rk4, rk6, dopr54 or dop853");
  cyl_to_sos_inplace(nobj, yo);
  return run_host_split(0, 0, nobj, yo, 7, npsi, psi, indiv_psi, npot, pot_type, pot_args, dpsi, rtol,
                  atol, result, err, odeint_type, cb, opts, false, GALPY_CUDA_SYS_SOS);
}

int integratePlanarOrbit_sos_cuda(int nobj, double* yo, int npsi, double* psi, int indiv_psi,
                                  int surface, int npot, int* pot_type, double* pot_args,
                                  void* /*pot_tfuncs*/, double dpsi, double rtol, double atol,
                                  double* result, int* err, int odeint_type,
                                  galpy_cuda_callback cb, const galpy_cuda_opts* opts)
{
  if (nobj < 0 || npsi < 1 || (nobj && (!yo || !psi || !result || !err)) || !pot_type ||
      !pot_args)
    return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  if (odeint_type != M_RK4 && odeint_type != M_RK6 && odeint_type != M_DOPR54 &&
      odeint_type != M_DOP853)
    return set_error(GALPY_CUDA_ERR_METHOD,
                     "surface-of-section integration takes rk4, rk6, dopr54 or dop853");
  polar_to_sos_inplace(nobj, yo, surface);
  return run_host_split(1, 0, nobj, yo, 5, npsi, psi, indiv_psi, npot, pot_type, pot_args, dpsi, rtol,
                  atol, result, err, odeint_type, cb, opts, false,
                  surface == 1 ? GALPY_CUDA_SYS_SOS_PLANAR_Y : GALPY_CUDA_SYS_SOS_PLANAR_X);
}

int integratePlanarOrbit_cuda(int nobj, double* yo, int nt, double* t, int indiv_t, int npot,
                              int* pot_type, double* pot_args, void* /*pot_tfuncs*/, double dt,
                              double rtol, double atol, double* result, int* err,
                              int odeint_type, galpy_cuda_callback cb,
                              const galpy_cuda_opts* opts)
{
  if (nobj < 0 || nt < 1 || (nobj && (!yo || !t || !result || !err)) || !pot_type || !pot_args)
    return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  if (!method_supported(odeint_type))
    return set_error(GALPY_CUDA_ERR_METHOD, "odeint_type not implemented on the GPU");
  cyl_to_rect_inplace(1, nobj, yo);
  return run_host_split(1, 0, nobj, yo, 4, nt, t, indiv_t, npot, pot_type, pot_args, dt, rtol, atol,
                  result, err, odeint_type, cb, opts, false);
}

int integrateFullOrbit_dxdv_cuda(double* yo, int nt, double* t, int npot, int* pot_type,
                                 double* pot_args, void* /*pot_tfuncs*/, double dt, double rtol,
                                 double atol, double* result, int* err, int odeint_type,
                                 const galpy_cuda_opts* opts)
{
  if (!yo || nt < 1 || !t || !result || !err || !pot_type || !pot_args)
    return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  return run_host(0, 1, 1, yo, 12, nt, t, 0, npot, pot_type, pot_args, dt, rtol, atol, result,
                  err, odeint_type, nullptr, opts, true);
}

int integratePlanarOrbit_dxdv_cuda(double* yo, int nt, double* t, int npot, int* pot_type,
                                   double* pot_args, void* /*pot_tfuncs*/, double dt, double rtol,
                                   double atol, double* result, int* err, int odeint_type,
                                   galpy_cuda_callback cb, const galpy_cuda_opts* opts)
{
  if (!yo || nt < 1 || !t || !result || !err || !pot_type || !pot_args)
    return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  return run_host(1, 1, 1, yo, 8, nt, t, 0, npot, pot_type, pot_args, dt, rtol, atol, result,
                  err, odeint_type, cb, opts, true);
}

int integrateOrbit_dxdv_batch_cuda(int planar, int nobj, double* yo, int nt, double* t,
                                   int indiv_t, int npot, int* pot_type, double* pot_args,
                                   double dt, double rtol, double atol, double* result, int* err,
                                   int odeint_type, const galpy_cuda_opts* opts)
{
  if (nobj < 0 || nt < 1 || (nobj && (!yo || !t || !result || !err)) || !pot_type || !pot_args)
    return set_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  return run_host_split(planar ? 1 : 0, 1, nobj, yo, planar ? 8 : 12, nt, t, indiv_t, npot, pot_type,
                  pot_args, dt, rtol, atol, result, err, odeint_type, nullptr, opts, true);
}

}  // extern "C"
