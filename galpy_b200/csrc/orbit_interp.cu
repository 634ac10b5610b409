// galpy_b200/csrc/orbit_interp.cu
//
// Orbit interpolation between stored rows on the device: galpy's
// Orbit.__call__ at times that are not integration times
// (galpy/orbit/Orbits.py:6460-6575) through the interpolants that
// _setupOrbitInterp builds (:6739-6830): per orbit and phase component --
// x = R cos(phi) and y = R sin(phi) in place of R and phi, to avoid phase
// wrapping -- the interpolating cubic spline through the rows
// (InterpolatedUnivariateSpline(k=3) per orbit, or RectBivariateSpline(kx=3,
// ky=1, s=0) over (t, orbit index), whose value at an integer orbit index is
// that orbit's cubic), R = sqrt(x^2 + y^2) and phi = atan2(y, x) after.
//
// FITPACK's interpolating cubic (s = 0) places its interior knots at the
// data points but the second and the second to last: the not-a-knot spline,
// whose third derivative is continuous at t_1 and t_{m-2}.  It is computed
// here from the standard second-derivative (moment) form: with h_i =
// t_{i+1} - t_i and moments M_i,
//   h_{i-1} M_{i-1} + 2 (h_{i-1} + h_i) M_i + h_i M_{i+1}
//       = 6 ((y_{i+1} - y_i) / h_i - (y_i - y_{i-1}) / h_{i-1}),  0 < i < m-1,
//   h_1 M_0 - (h_0 + h_1) M_1 + h_0 M_2 = 0                     (not-a-knot),
//   h_{m-2} M_{m-3} - (h_{m-3} + h_{m-2}) M_{m-2} + h_{m-3} M_{m-1} = 0;
// M_0 and M_{m-1} are eliminated with the end conditions, which leaves a
// tridiagonal system in M_1 .. M_{m-2}, solved by the Thomas algorithm.  With
// fewer than 4 points galpy uses degree m - 1: the interpolating line or
// parabola.  Queries outside [t_0, t_{m-1}] extrapolate the end pieces (as
// FITPACK's splev does by default; galpy refuses them before interpolating).
//
// Four passes:
//   transpose_kernel  the rows [n][nt][nv] to component-major values
//                     X[nv][nt][n] (x, y in place of R, phi), through a
//                     shared-memory tile: each orbit's rows are read as one
//                     contiguous run and the values written orbit-contiguous
//   sweep_kernel      per orbit (one thread for shared times): the Thomas
//                     factors c'_i, which depend on the times only
//   moments_kernel    per (orbit, component): the right-hand side, forward
//                     elimination and back substitution -> M_i
//   eval_kernel       per (orbit, block of queries): interval search, the
//                     cubic of each component, conversion back to (R, phi);
//                     the thread writes its orbit's consecutive output rows
// X, the moments M[nv][nt][n] and the Thomas factors [nt][n] are
// orbit-contiguous, so that consecutive threads (orbits) touch consecutive
// doubles.
#include <cuda_runtime.h>
#include <stddef.h>

#include <string>

#include "../../include/galpy_cuda.h"

int gpc_report_error(int code, const char* msg);  // galpy_cuda.cu
int gpc_library_pool(cudaMemPool_t* out);         // galpy_cuda.cu

namespace {

__device__ __forceinline__ double tq_of(const double* t, int indiv, long long i, int nt, int j)
{
  return t[(indiv ? i * (long long)nt : 0LL) + j];
}

// Value of component k at row j of orbit i in the component-major array X.
__device__ __forceinline__ double xval(const double* X, long long n, int nt, int k, int j,
                                       long long i)
{
  return X[((long long)k * nt + j) * n + i];
}

// Rows [n][nt][NV] (galpy cylindrical) -> X[NV][nt][n] with x = R cos(phi),
// y = R sin(phi) in the places of R and phi.  Block: kTileO orbits x kTileJ
// rows; the load walks each orbit's kTileJ * NV contiguous doubles, the
// store walks orbits.
constexpr int kTileO = 32, kTileJ = 8;
template <int NV>
__global__ void __launch_bounds__(256) transpose_kernel(long long n, int nt, const double* rows,
                                                        double* X)
{
  constexpr int W = kTileJ * NV + 1;  // padded row of the tile (bank spread)
  __shared__ double tile[kTileO * W];
  const long long i0 = (long long)blockIdx.x * kTileO;
  const int j0 = blockIdx.y * kTileJ;
  const int jn = nt - j0 < kTileJ ? nt - j0 : kTileJ;
  for (int e = threadIdx.x; e < kTileO * kTileJ * NV; e += blockDim.x) {
    const int o = e / (kTileJ * NV), r = e - o * (kTileJ * NV);
    if (i0 + o < n && r < jn * NV) tile[o * W + r] = rows[((i0 + o) * nt + j0) * NV + r];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kTileO * kTileJ * NV; e += blockDim.x) {
    const int o = e % kTileO, rest = e / kTileO;
    const int jj = rest % kTileJ, k = rest / kTileJ;
    if (i0 + o >= n || jj >= jn) continue;
    const double* v = tile + o * W + jj * NV;
    double val = v[k];
    if (k == 0)
      val = v[0] * cos(v[NV - 1]);
    else if (k == NV - 1)
      val = v[0] * sin(v[NV - 1]);
    X[((long long)k * nt + j0 + jj) * n + i0 + o] = val;
  }
}

// Coefficients of row i (1 <= i <= m-2) of the reduced system
// a_i M_{i-1} + b_i M_i + c_i M_{i+1} = r_i (a_1 and c_{m-2} unused).
__device__ __forceinline__ void row_coefs(const double* tt, int m, int i, double& a, double& b,
                                          double& c)
{
  const double h0 = tt[i] - tt[i - 1], h1 = tt[i + 1] - tt[i];
  a = h0;
  b = 2.0 * (h0 + h1);
  c = h1;
  if (i == 1) {  // M_0 = ((h0 + h1) M_1 - h0 M_2) / h1 substituted
    b = (h0 + h1) * (h0 + 2.0 * h1) / h1;
    c = (h1 * h1 - h0 * h0) / h1;
    a = 0.0;
  }
  if (i == m - 2) {  // M_{m-1} = ((hl + hr) M_{m-2} - hr M_{m-3}) / hl, hl = h0, hr = h1
    // (m >= 4 here, so row m - 2 is never row 1: with m = 4 the two rows
    // carry one end condition each)
    a = (h0 * h0 - h1 * h1) / h0;
    b = (h0 + h1) * (2.0 * h0 + h1) / h0;
    c = 0.0;
  }
}

__global__ void sweep_kernel(long long n, int nt, const double* t, int indiv, double* cp)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* tt = t + (indiv ? i * (long long)nt : 0LL);
  const int m = nt;
  double prev = 0.0;
  for (int r = 1; r <= m - 2; r++) {
    double a, b, c;
    row_coefs(tt, m, r, a, b, c);
    const double den = b - a * prev;
    prev = c / den;
    cp[(long long)r * n + i] = prev;
  }
}

template <int NV>
__global__ void moments_kernel(long long n, int nt, const double* t, int indiv,
                               const double* X, const double* cp, long long ncp, double* M)
{
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= n * NV) return;
  const int k = (int)(g / n);
  const long long i = g - (long long)k * n;
  const double* tt = t + (indiv ? i * (long long)nt : 0LL);
  const long long ci = indiv ? i : 0LL;
  const int m = nt;
  double* Mk = M + (long long)k * nt * n;
  // forward elimination: d'_r stored in M_r
  double ym = xval(X, n, nt, k, 0, i), y0 = xval(X, n, nt, k, 1, i);
  double dprev = 0.0, cprev = 0.0;
  for (int r = 1; r <= m - 2; r++) {
    const double yp = xval(X, n, nt, k, r + 1, i);
    const double h0 = tt[r] - tt[r - 1], h1 = tt[r + 1] - tt[r];
    const double rhs = 6.0 * ((yp - y0) / h1 - (y0 - ym) / h0);
    double a, b, c;
    row_coefs(tt, m, r, a, b, c);
    const double den = b - a * cprev;
    const double d = (rhs - a * dprev) / den;
    Mk[(long long)r * n + i] = d;
    dprev = d;
    cprev = cp[(long long)r * ncp + ci];
    ym = y0;
    y0 = yp;
  }
  // back substitution
  double Mnext = Mk[(long long)(m - 2) * n + i];
  for (int r = m - 3; r >= 1; r--) {
    const double Mr = Mk[(long long)r * n + i] - cp[(long long)r * ncp + ci] * Mnext;
    Mk[(long long)r * n + i] = Mr;
    Mnext = Mr;
  }
  // the end moments from the not-a-knot conditions
  const double h0 = tt[1] - tt[0], h1 = tt[2] - tt[1];
  const double M1 = Mk[1LL * n + i], M2 = Mk[2LL * n + i];
  Mk[i] = ((h0 + h1) * M1 - h0 * M2) / h1;
  const double hl = tt[m - 2] - tt[m - 3], hr = tt[m - 1] - tt[m - 2];
  const double Ma = Mk[(long long)(m - 3) * n + i], Mb = Mk[(long long)(m - 2) * n + i];
  Mk[(long long)(m - 1) * n + i] = ((hl + hr) * Mb - hr * Ma) / hl;
}

// Interval of tq in the increasing grid tt[0..m-1]: j with tt[j] <= tq <
// tt[j+1], clamped to [0, m-2] (extrapolation uses the end pieces).
__device__ __forceinline__ int interval(const double* tt, int m, double tq)
{
  int lo = 0, hi = m - 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (tt[mid] <= tq)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Queries per thread of eval_kernel: a thread writes kQueryBlock
// consecutive output rows of its orbit, whose partial 32-byte sectors then
// merge in L2.
constexpr int kQueryBlock = 16;
template <int NV>
__global__ void __launch_bounds__(128) eval_kernel(long long n, int nt, const double* t, int indiv,
                                                   const double* X, const double* M, int nq,
                                                   const double* tq, int indiv_q, double* out)
{
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long i = g % n;  // consecutive threads: consecutive orbits
  const long long qb = g / n;
  const int q0 = (int)(qb * kQueryBlock);
  if (q0 >= nq) return;
  const int q1 = nq - q0 < kQueryBlock ? nq : q0 + kQueryBlock;
  const double* tt = t + (indiv ? i * (long long)nt : 0LL);
  const int m = nt;
  for (int q = q0; q < q1; q++) {
    const double x = tq_of(tq, indiv_q, i, nq, q);
    double v[NV];
    if (m == 1) {
#pragma unroll
      for (int k = 0; k < NV; k++) v[k] = xval(X, n, nt, k, 0, i);
    } else if (m == 2) {  // the line through both rows
      const double s = (x - tt[0]) / (tt[1] - tt[0]);
#pragma unroll
      for (int k = 0; k < NV; k++) {
        const double a = xval(X, n, nt, k, 0, i), b = xval(X, n, nt, k, 1, i);
        v[k] = a + s * (b - a);
      }
    } else if (m == 3) {  // the parabola through the three rows (Newton form)
      const double t0 = tt[0], t1 = tt[1], t2 = tt[2];
#pragma unroll
      for (int k = 0; k < NV; k++) {
        const double y0 = xval(X, n, nt, k, 0, i), y1 = xval(X, n, nt, k, 1, i);
        const double y2 = xval(X, n, nt, k, 2, i);
        const double d01 = (y1 - y0) / (t1 - t0), d12 = (y2 - y1) / (t2 - t1);
        const double d012 = (d12 - d01) / (t2 - t0);
        v[k] = y0 + (x - t0) * (d01 + (x - t1) * d012);
      }
    } else {
      const int j = interval(tt, m, x);
      const double h = tt[j + 1] - tt[j], A = tt[j + 1] - x, B = x - tt[j];
#pragma unroll
      for (int k = 0; k < NV; k++) {
        const double Mj = xval(M, n, nt, k, j, i), Mj1 = xval(M, n, nt, k, j + 1, i);
        const double yj = xval(X, n, nt, k, j, i), yj1 = xval(X, n, nt, k, j + 1, i);
        v[k] = (Mj * A * A * A + Mj1 * B * B * B) / (6.0 * h) + (yj / h - Mj * h / 6.0) * A +
               (yj1 / h - Mj1 * h / 6.0) * B;
      }
    }
    // (x, y) -> (R, phi), galpy's unpacking of the interpolated x and y
    const double px = v[0], py = v[NV - 1];
    double* o = out + (i * nq + q) * NV;
    o[0] = sqrt(px * px + py * py);
#pragma unroll
    for (int k = 1; k < NV - 1; k++) o[k] = v[k];
    o[NV - 1] = atan2(py, px);
  }
}

int fail(const char* what, cudaError_t e)
{
  return gpc_report_error(GALPY_CUDA_ERR_CUDA, (std::string(what) + cudaGetErrorString(e)).c_str());
}

template <int NV>
int run(long long n, int nt, const double* t, int indiv_t, const double* rows, int nq,
        const double* tq, int indiv_q, double* out, cudaStream_t s)
{
  double* X = nullptr;
  double* M = nullptr;
  double* cp = nullptr;
  cudaError_t e;
  // scratch from the library's private pool, which keeps freed memory
  // mapped for the next call (galpy_cuda_trim_memory returns it): with a
  // release threshold of 0 every call would map its gigabytes again
  cudaMemPool_t pool = nullptr;
  const int prc = gpc_library_pool(&pool);
  if (prc) return prc;
  const long long ncp = indiv_t ? n : 1;
  const size_t vals = (size_t)NV * nt * n;
  if ((e = cudaMallocFromPoolAsync((void**)&X, vals * sizeof(double), pool, s)) != cudaSuccess)
    return fail("interpolation scratch: ", e);
  const dim3 tgrid((unsigned)((n + kTileO - 1) / kTileO), (unsigned)((nt + kTileJ - 1) / kTileJ));
  transpose_kernel<NV><<<tgrid, 256, 0, s>>>(n, nt, rows, X);
  if (nt >= 4) {
    if ((e = cudaMallocFromPoolAsync((void**)&M, vals * sizeof(double), pool, s)) != cudaSuccess ||
        (e = cudaMallocFromPoolAsync((void**)&cp, (size_t)nt * ncp * sizeof(double), pool, s)) !=
            cudaSuccess) {
      if (M) cudaFreeAsync(M, s);
      cudaFreeAsync(X, s);
      return fail("interpolation scratch: ", e);
    }
    sweep_kernel<<<(unsigned)((ncp + 127) / 128), 128, 0, s>>>(ncp, nt, t, indiv_t, cp);
    moments_kernel<NV><<<(unsigned)((n * NV + 127) / 128), 128, 0, s>>>(n, nt, t, indiv_t, X, cp,
                                                                         ncp, M);
  }
  const long long items = n * (long long)((nq + kQueryBlock - 1) / kQueryBlock);
  eval_kernel<NV><<<(unsigned)((items + 127) / 128), 128, 0, s>>>(n, nt, t, indiv_t, X, M, nq, tq,
                                                                   indiv_q, out);
  e = cudaGetLastError();
  cudaFreeAsync(X, s);
  if (M) cudaFreeAsync(M, s);
  if (cp) cudaFreeAsync(cp, s);
  if (e != cudaSuccess) return fail("interpolation kernels: ", e);
  return GALPY_CUDA_OK;
}

}  // namespace

extern "C" int galpy_cuda_orbit_interp_device(int nv, long long n, int nt, const double* t,
                                              int indiv_t, const double* rows, int nq,
                                              const double* tq, int indiv_q, double* out,
                                              void* stream)
{
  if ((nv != 4 && nv != 6) || n < 0 || nt < 1 || nq < 0 || (n > 0 && nq > 0 && (!t || !rows ||
                                                                                !tq || !out)))
    return gpc_report_error(GALPY_CUDA_ERR_ARG, "orbit interpolation: invalid arguments");
  if (n == 0 || nq == 0) return GALPY_CUDA_OK;
  if (n * (long long)nq >= (1LL << 31) * 128LL || n * nv >= (1LL << 31) * 128LL)
    return gpc_report_error(GALPY_CUDA_ERR_ARG, "orbit interpolation: too many items");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return nv == 6 ? run<6>(n, nt, t, indiv_t, rows, nq, tq, indiv_q, out, s)
                 : run<4>(n, nt, t, indiv_t, rows, nq, tq, indiv_q, out, s);
}
