// galpy_b200/csrc/adjoint.cu
//
// Kernels and C-ABI entry points of the reverse-mode gradient of DOP853
// orbit integration (the per-orbit algorithms are in adjoint.cuh).
//
// One thread owns one orbit for a whole pass.  Arrays are SoA ([value][orbit])
// so that the 32 lanes of a warp touch consecutive addresses; the per-orbit
// segment buffers of the backward pass (64 step start states) are
// thread-local arrays, which the hardware interleaves across the lanes of a
// warp the same way.  A checkpoint record holds a segment's start state and
// its 64 accepted step sizes ([ckpt_cap][nv + 1 + 64][nobj]).  Compile-time component lists (MWPotential2014's
// PowerSphericalwCutoff + MiyamotoNagai + NFW) are inlined like in the
// integration kernels; the tidal tensors and parameter derivatives of the
// backward pass walk the component list at run time.
#include <cuda_runtime.h>

#include <string>

#include "../../include/galpy_cuda.h"
#include "adjoint.cuh"
#include "compile_potential.h"

using namespace gpc;

int gpc_report_error(int code, const char* msg);  // galpy_cuda.cu

namespace {

struct AdjK {
  long long nobj;
  double t0, T, rtol, atol;
  long long max_att;
  const GpComp* comps;
  int ncomp;
  const int* group;
  const double* w0;
  double* yT;
  long long* nsteps;
  int* err;
  double* ckpt;
  int ccap;
  double* hrec;
  long long hcap;
  const double* gyT;
  double* gw0;
  double* gparam;
  const int* order;
};

// Orbit handled by thread j of the launch.
__device__ __forceinline__ long long orbit_of(const AdjK& A, long long j)
{
  return A.order ? (long long)A.order[j] : j;
}

template <class POT>
__device__ __forceinline__ adj::Field<POT> field_of(const AdjK& A, long long i)
{
  const int g = A.group ? A.group[i] : 0;
  return adj::Field<POT>{A.comps + (long long)g * A.ncomp, A.ncomp, nullptr};
}

template <int D, class POT>
__global__ void __launch_bounds__(128) adj_forward_kernel(const AdjK A)
{
  constexpr int N = 2 * D;
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= A.nobj) return;
  const long long i = orbit_of(A, j);
  if (i < 0 || i >= A.nobj) return;
  const adj::Field<POT> F = field_of<POT>(A, i);
  double w[N], y[N];
#pragma unroll
  for (int c = 0; c < N; c++) w[c] = A.w0[c * A.nobj + i];
  long long ns = 0;
  const int st = adj::forward_orbit<D, POT>(F, w, A.t0, A.T, A.rtol, A.atol, A.max_att,
                                            A.ckpt + i, A.nobj, A.ccap,
                                            A.hrec ? A.hrec + i : nullptr, A.nobj, A.hcap, y, &ns);
#pragma unroll
  for (int c = 0; c < N; c++) A.yT[c * A.nobj + i] = st == E_OK ? y[c] : NAN;
  A.nsteps[i] = ns;
  A.err[i] = st;
}

template <int D, class POT>
__global__ void __launch_bounds__(128) adj_replay_kernel(const AdjK A)
{
  constexpr int N = 2 * D;
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= A.nobj) return;
  const long long i = orbit_of(A, j);
  if (i < 0 || i >= A.nobj) return;
  const adj::Field<POT> F = field_of<POT>(A, i);
  double w[N], y[N];
#pragma unroll
  for (int c = 0; c < N; c++) w[c] = A.w0[c * A.nobj + i];
  const long long ns = A.nsteps[i];
  if (ns > A.hcap) {
#pragma unroll
    for (int c = 0; c < N; c++) A.yT[c * A.nobj + i] = NAN;
    return;
  }
  adj::replay_orbit<D, POT>(F, w, A.t0, A.T, A.hrec + i, A.nobj, ns, y);
#pragma unroll
  for (int c = 0; c < N; c++) A.yT[c * A.nobj + i] = y[c];
}

// MINB: minimum resident blocks per SM asked of the register allocator
// (1: no cap; 4: at most 128 registers a thread at 128 threads a block).
template <int D, class POT, int MINB>
__global__ void __launch_bounds__(128, MINB) adj_backward_kernel(const AdjK A)
{
  constexpr int N = 2 * D;
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= A.nobj) return;
  const long long i = orbit_of(A, j);
  if (i < 0 || i >= A.nobj) return;
  const adj::Field<POT> F = field_of<POT>(A, i);
  const int np = adj::group_nparam(F.comp, F.ncomp);
  double lam[N], g[adj::kMaxParam];
  for (int p = 0; p < np; p++) g[p] = 0.0;
  const long long nseg = (A.nsteps[i] + adj::kCkptEvery - 1) / adj::kCkptEvery;
  if (A.err[i] != E_OK || A.nsteps[i] < 0 || nseg > A.ccap) {
#pragma unroll
    for (int c = 0; c < N; c++) lam[c] = NAN;
    for (int p = 0; p < np; p++) g[p] = NAN;
  } else {
#pragma unroll
    for (int c = 0; c < N; c++) lam[c] = A.gyT[c * A.nobj + i];
    adj::backward_orbit<D, POT>(F, A.T, A.ckpt + i, A.nobj, A.nsteps[i], lam, g);
  }
#pragma unroll
  for (int c = 0; c < N; c++) A.gw0[c * A.nobj + i] = lam[c];
  if (A.gparam)
    for (int p = 0; p < np; p++) A.gparam[p * A.nobj + i] = g[p];
}

enum Pass { P_FORWARD, P_REPLAY, P_BACKWARD };

template <int D, class POT>
void launch_pass(Pass pass, int variant, const AdjK& K, unsigned blocks, unsigned threads,
                 cudaStream_t s)
{
  switch (pass) {
    case P_FORWARD: adj_forward_kernel<D, POT><<<blocks, threads, 0, s>>>(K); break;
    case P_REPLAY: adj_replay_kernel<D, POT><<<blocks, threads, 0, s>>>(K); break;
    case P_BACKWARD:
      if (variant == 1)
        adj_backward_kernel<D, POT, 4><<<blocks, threads, 0, s>>>(K);
      else
        adj_backward_kernel<D, POT, 1><<<blocks, threads, 0, s>>>(K);
      break;
  }
}

using MW14Adj = FixedPot<false, T_PSWC, T_MN, T_NFW>;

int run_pass(Pass pass, const galpy_cuda_adjoint* a)
{
  if (!a || a->size < (int)sizeof(galpy_cuda_adjoint))
    return gpc_report_error(GALPY_CUDA_ERR_ARG, "galpy_cuda_adjoint: NULL or wrong size");
  if (a->nobj < 0 || !a->comps || a->ncomp < 1 || a->ncomp > kMaxComp || !a->w0 || !a->nsteps)
    return gpc_report_error(GALPY_CUDA_ERR_ARG, "galpy_cuda_adjoint: invalid arguments");
  if (pass == P_FORWARD && (!a->yT || !a->err || !a->ckpt || a->ckpt_cap < 1 ||
                            (a->hrec && a->hcap < 1)))
    return gpc_report_error(GALPY_CUDA_ERR_ARG, "adjoint forward: yT, err and ckpt are required");
  if (pass == P_REPLAY && (!a->yT || !a->hrec || a->hcap < 1))
    return gpc_report_error(GALPY_CUDA_ERR_ARG, "adjoint replay: yT and hrec are required");
  if (pass == P_BACKWARD && (!a->err || !a->ckpt || !a->gyT || !a->gw0))
    return gpc_report_error(GALPY_CUDA_ERR_ARG,
                            "adjoint backward: err, ckpt, gyT and gw0 are required");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
    return gpc_report_error(GALPY_CUDA_ERR_NODEVICE, "no CUDA device visible");
  if (a->nobj == 0) return GALPY_CUDA_OK;
  AdjK K;
  K.nobj = a->nobj;
  K.t0 = a->t0;
  K.T = a->tend;
  K.rtol = a->rtol;
  K.atol = a->atol;
  K.max_att = a->max_attempts;
  K.comps = static_cast<const GpComp*>(a->comps);
  K.ncomp = a->ncomp;
  K.group = a->group;
  K.w0 = a->w0;
  K.yT = a->yT;
  K.nsteps = a->nsteps;
  K.err = a->err;
  K.ckpt = a->ckpt;
  K.ccap = a->ckpt_cap;
  K.hrec = a->hrec;
  K.hcap = a->hcap;
  K.gyT = a->gyT;
  K.gw0 = a->gw0;
  K.gparam = a->gparam;
  K.order = a->order;
  const unsigned threads = a->block_size > 0 ? (unsigned)a->block_size : 64u;
  if (threads > 128 || threads % 32)
    return gpc_report_error(GALPY_CUDA_ERR_ARG, "adjoint: block_size must be 32..128, a multiple of 32");
  const unsigned blocks = (unsigned)((a->nobj + threads - 1) / threads);
  cudaStream_t s = static_cast<cudaStream_t>(a->stream);
  const bool mw14 = a->signature == GALPY_CUDA_SIG_MW14 && a->ncomp == 3;
  const int v = a->variant;
  if (a->planar)
    mw14 ? launch_pass<2, MW14Adj>(pass, v, K, blocks, threads, s)
         : launch_pass<2, DynPot>(pass, v, K, blocks, threads, s);
  else
    mw14 ? launch_pass<3, MW14Adj>(pass, v, K, blocks, threads, s)
         : launch_pass<3, DynPot>(pass, v, K, blocks, threads, s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return gpc_report_error(GALPY_CUDA_ERR_CUDA, (std::string("adjoint launch: ") +
                                                  cudaGetErrorString(e)).c_str());
  return GALPY_CUDA_OK;
}

}  // namespace

extern "C" {

int galpy_cuda_adjoint_forward(const galpy_cuda_adjoint* a) { return run_pass(P_FORWARD, a); }

int galpy_cuda_adjoint_replay(const galpy_cuda_adjoint* a) { return run_pass(P_REPLAY, a); }

int galpy_cuda_adjoint_backward(const galpy_cuda_adjoint* a) { return run_pass(P_BACKWARD, a); }

int galpy_cuda_adjoint_params(int planar, int npot, const int* pot_type, const double* pot_args,
                              int* arg_index)
{
  if (!pot_type || npot < 1 || npot > kMaxComp)
    return gpc_report_error(GALPY_CUDA_ERR_ARG, "invalid arguments");
  int n = 0, off = 0;
  for (int k = 0; k < npot; k++) {
    // an ellipsoidal component's argument count is read from its arguments
    const int na = galpy_nargs(pot_type[k], planar, pot_args ? pot_args + off : nullptr);
    if (na < 0)
      return gpc_report_error(GALPY_CUDA_ERR_POTENTIAL, "potential type not implemented on the GPU");
    // the adjoint's DOP853 evaluates static forces and needs the tidal
    // tensor, which the device does not have for an SCF expansion
    if (pot_type[k] == T_DEHNENBAR || pot_type[k] == T_SCF || pot_type[k] == T_SPIRALARMS ||
        pot_type[k] == T_NEEDLEBAR ||
        is_wrapper(pot_type[k]) || is_disk_pert(pot_type[k]))
      return gpc_report_error(GALPY_CUDA_ERR_POTENTIAL,
                              "gradients through a time-dependent or SCF potential are not "
                              "available");
    // a rotated ellipsoid: the tidal tensor follows the reference's second
    // derivatives, which ignore the rotation, so they are not the derivative
    // of its force and the adjoint would return wrong gradients
    if (is_ellipsoidal(pot_type[k])) {
      const double* e = pot_args + off + 17 + (int)pot_args[off + 16];
      if (e[2] == 0.0)
        return gpc_report_error(GALPY_CUDA_ERR_POTENTIAL,
                                "gradients through a rotated ellipsoidal potential are not "
                                "available (its second derivatives ignore the rotation)");
    }
    const int np = adj::comp_nparam(pot_type[k]);
    for (int p = 0; p < np; p++, n++)
      if (arg_index) arg_index[n] = off + adj::comp_param_arg(pot_type[k], p);
    off += na;
  }
  return n;
}

}  // extern "C"
