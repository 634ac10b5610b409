// galpy_b200/csrc/adjoint.cuh
//
// Reverse-mode differentiation of DOP853 orbit integration: gradients of a
// loss on the final states y(T) with respect to the initial conditions and
// the potential parameters.  The reference has no adjoint; its gradient
// information comes from the variational equations (integrate_dxdv,
// galpy/orbit/orbit_c_ext/integratePlanarOrbit.c:940-1014), one tangent
// vector per input direction.  The adjoint gives the whole gradient of a
// scalar loss in one backward sweep per orbit.
//
// What is differentiated: the discrete map that the forward integrator
// applies, with its accepted step sizes held fixed (they are not
// differentiated; this is the standard discrete adjoint of an adaptive
// method and is exact for the frozen step sequence).
//
//   * Forward: galpy's DOP853 (same tableau, initial step, controller and
//     dense output as Dop853Machine, leung_dop853.c:231-517) from t0 to T;
//     y(T) is the dense-output value inside the step that passes T, as in
//     the reference (it does not shorten the last step).  Every 64 accepted
//     steps the state (y, t) is saved, a checkpoint, together with the
//     segment's 64 accepted step sizes.
//   * Backward, per orbit, segment by segment from the last: restore the
//     segment's checkpoint, recompute the start state of each of its steps
//     with the recorded step sizes (no step-size control runs again, so a
//     marginal accept/reject decision cannot come out differently), then
//     sweep the steps in reverse.  Each step recomputes its stages and
//     applies the adjoint of an explicit Runge-Kutta step:
//         kappa_i = h W_i lambda + h sum_{j>i} A_ji mu_j
//         mu_i    = J(Y_i)^T kappa_i = (K(q_i) kappa_v, kappa_q)
//         lambda <- lambda + sum_i mu_i,   g_theta += sum_i (da/dtheta)^T kappa_v
//     with K the tidal tensor (potentials.cuh, accel_tidal) and da/dtheta
//     the analytic parameter derivatives below.  W = b (8th-order weights)
//     for full steps; the last step is the 16-stage dense-output map with
//     weights W(s), s = (T - t_n) / h_n.
//
// All functions are host/device portable so that the CPU test harness runs
// the same code against finite differences and the reference's variational
// integration.
#pragma once
#include "dop853_tableau.cuh"
#include "gpc_common.cuh"
#include "potentials.cuh"

namespace gpc {
namespace adj {

constexpr int kCkptEvery = 64;              // accepted steps per checkpointed segment
constexpr int kMaxParam = 3 * kMaxComp;     // differentiable parameters per group
constexpr int kMaxRejects = 1000;           // consecutive rejected attempts per step

// ------------------------------------------------------- parameters ---
// Differentiable parameters of a component, in this order:
//   PowerSphericalPotentialwCutoff: amp, rc        (galpy args 0, 2)
//   MiyamotoNagai:                  amp, a, b      (args 0, 1, 2)
//   NFW, Hernquist:                 amp, a         (args 0, 1)
//   LogarithmicHalo:                amp, q, core^2 (args 0, 1, 2)
GPC_HD GPC_FI int comp_nparam(int type)
{
  switch (type) {
    case T_PSWC: return 2;
    case T_MN: return 3;
    case T_NFW: return 2;
    case T_HERNQUIST: return 2;
    case T_LOGHALO: return 3;
    default: return 0;
  }
}
inline int comp_param_arg(int type, int p) { return (type == T_PSWC && p == 1) ? 2 : p; }

GPC_HD GPC_FI int group_nparam(const GpComp* comp, int ncomp)
{
  int n = 0;
  for (int k = 0; k < ncomp; k++) n += comp_nparam(ldg(&comp[k].type));
  return n;
}

// g[p] += lambda . d a(x) / d theta_p for the parameters of one group
// (a = the acceleration; lambda = (lx, ly, lz), lz unused when PLANAR).
template <bool PLANAR>
GPC_HD void accel_param_vjp(const GpComp* __restrict__ comp, int ncomp, double x, double y,
                            double z, double lx, double ly, double lz, double* g)
{
  if (PLANAR) z = lz = 0.0;
  const double R2 = x * x + y * y, z2 = z * z, r2 = R2 + z2;
  const double xl = x * lx + y * ly + z * lz;  // x . lambda: spherical terms a = f(r) x
  int p = 0;
  for (int k = 0; k < ncomp; k++) {
    const GpComp* cp = comp + k;
    const double amp = ldg(&cp->c[0]);
    switch (ldg(&cp->type)) {
      case T_PSWC: {
        // f = -amp M(r)/r^3, M = 2 pi rc^(3-alpha) gamma(a, r^2/rc^2):
        // dM/drc = ((3 - alpha) M - 4 pi r^(3-alpha) e^(-u)) / rc
        const double u = r2 * ldg(&cp->c[1]);
        const double pw = exp(ldg(&cp->c[3]) * log(r2));  // (r^2)^(-alpha/2)
        double Mr3;
        if (u < ldg(&cp->c[5])) {
          Mr3 = ldg(&cp->c[2]) * pw * gamma_star<double>(tables(cp), u, ldg(&cp->c[6]));
        } else {
          const double ir = rsq(r2);
          Mr3 = ldg(&cp->c[4]) * ir * ir * ir;
        }
        const double alpha = -2.0 * ldg(&cp->c[3]), rc = ldg(&cp->c[9]);
        g[p] -= Mr3 * xl;
        g[p + 1] -= amp * ((3.0 - alpha) * Mr3 - ldg(&cp->c[7]) * pw * exp(-u)) / rc * xl;
        p += 2;
        break;
      }
      case T_MN: {
        // a = (x gR, y gR, z gz): gR = -amp D^-3/2, gz = -amp (s/zeta) D^-3/2,
        // zeta = sqrt(z^2 + b^2), s = a + zeta, D = R^2 + s^2
        const double a = ldg(&cp->c[1]), b2 = ldg(&cp->c[2]), b = sqrt(b2);
        const double zb2 = z2 + b2, izb = rsq(zb2), zeta = zb2 * izb, s = a + zeta;
        const double iD = rsq(R2 + s * s), iD3 = iD * iD * iD, iD5 = iD3 * iD * iD;
        const double xyl = x * lx + y * ly, zl = z * lz;
        g[p] += -iD3 * xyl - s * izb * iD3 * zl;
        g[p + 1] += 3.0 * amp * s * iD5 * xyl - amp * (iD3 - 3.0 * s * s * iD5) * izb * zl;
        const double bz = b * izb;  // d zeta / d b = d s / d b
        g[p + 2] += 3.0 * amp * s * iD5 * bz * xyl -
                    amp * bz * (iD3 * izb - s * iD3 * izb * izb - 3.0 * s * s * iD5 * izb) * zl;
        p += 3;
        break;
      }
      case T_NFW: {
        // f = amp / r^2 (1/(a+r) - ln(1+r/a)/r);  df/da = amp / (r a (a+r)^2)
        const double a = ldg(&cp->c[1]);
        const double ir = rsq(r2), r = r2 * ir, iar = 1.0 / (a + r);
        g[p] += ir * ir * (iar - log1p(r * ldg(&cp->c[2])) * ir) * xl;
        g[p + 1] += amp * ir * ldg(&cp->c[2]) * iar * iar * xl;
        p += 2;
        break;
      }
      case T_HERNQUIST: {
        // f = -amp / (2 r (r+a)^2);  df/da = amp / (r (r+a)^3)
        const double a = ldg(&cp->c[1]);
        const double ir = rsq(r2), ira = 1.0 / (r2 * ir + a);
        g[p] -= 0.5 * ir * ira * ira * xl;
        g[p + 1] += amp * ir * ira * ira * ira * xl;
        p += 2;
        break;
      }
      case T_LOGHALO: {
        // a = g (x, e y, z/q^2), g = -amp / D, D = x^2 + e y^2 + z^2/q^2 + core^2
        const double iq2 = ldg(&cp->c[1]), ye = ldg(&cp->c[3]);
        const double D = x * x + ye * y * y + z2 * iq2 + ldg(&cp->c[2]);
        const double iDl = 1.0 / D, gl = -amp * iDl;
        const double vl = x * lx + ye * y * ly + iq2 * z * lz;
        const double diq2 = -2.0 * iq2 * sqrt(iq2);  // d(1/q^2)/dq
        g[p] -= iDl * vl;
        g[p + 1] += amp * iDl * iDl * z2 * diq2 * vl + gl * diq2 * z * lz;
        g[p + 2] += amp * iDl * iDl * vl;
        p += 3;
        break;
      }
      default:
        break;
    }
  }
}

// The per-point force and vector-Jacobian functions are called, not
// inlined, in device code: a DOP853 step unrolls 12-16 stages, and inlining
// a force or tidal evaluation into every one of them made the kernels too
// large for the instruction cache (warps stalled on instruction fetch).
// Arguments and results travel in registers (scalars and a small struct).
#if defined(__CUDACC__)
#define GPC_NI __noinline__
#else
#define GPC_NI
#endif

struct V3 {
  double x, y, z;
};

// mu_q = K(q) lv (K the symmetric tidal tensor); g += (da/dtheta)^T lv.
template <bool PLANAR>
GPC_HD GPC_NI V3 vjp_at(const GpComp* __restrict__ comp, int ncomp, double x, double y, double z,
                        double lx, double ly, double lz, double* g)
{
  double ax, ay, az, K[6];
  if (PLANAR) z = lz = 0.0;
  accel_tidal<PLANAR>(comp, ncomp, x, y, z, ax, ay, az, K);
  V3 r;
  r.x = K[0] * lx + K[1] * ly + K[3] * lz;
  r.y = K[1] * lx + K[2] * ly + K[4] * lz;
  r.z = K[3] * lx + K[4] * ly + K[5] * lz;
  accel_param_vjp<PLANAR>(comp, ncomp, x, y, z, lx, ly, lz, g);
  return r;
}

template <int D>
GPC_HD GPC_FI void accel_vjp(const GpComp* __restrict__ comp, int ncomp, const double* q,
                             const double* lv, double* Kv, double* g)
{
  const V3 r = vjp_at<D == 2>(comp, ncomp, q[0], q[1], D == 3 ? q[D - 1] : 0.0, lv[0], lv[1],
                              D == 3 ? lv[D - 1] : 0.0, g);
  Kv[0] = r.x;
  Kv[1] = r.y;
  if (D == 3) Kv[D - 1] = r.z;
}

// ---------------------------------------------------------- tableau ---
// The DOP853 stages as one 16-stage explicit scheme (0-based stage index;
// stage 12 is the evaluation at the new state, whose input weights are the
// 8th-order solution weights b; stages 13-15 are the dense-output stages).
// A(i, j) is the weight of stage j in the input of stage i (Hairer's a_ij).
GPC_HD constexpr double A(int i, int j)
{
  using namespace dp;
  switch (i * 16 + j) {
    case 1 * 16 + 0: return a21;
    case 2 * 16 + 0: return a31;
    case 2 * 16 + 1: return a32;
    case 3 * 16 + 0: return a41;
    case 3 * 16 + 2: return a43;
    case 4 * 16 + 0: return a51;
    case 4 * 16 + 2: return a53;
    case 4 * 16 + 3: return a54;
    case 5 * 16 + 0: return a61;
    case 5 * 16 + 3: return a64;
    case 5 * 16 + 4: return a65;
    case 6 * 16 + 0: return a71;
    case 6 * 16 + 3: return a74;
    case 6 * 16 + 4: return a75;
    case 6 * 16 + 5: return a76;
    case 7 * 16 + 0: return a81;
    case 7 * 16 + 3: return a84;
    case 7 * 16 + 4: return a85;
    case 7 * 16 + 5: return a86;
    case 7 * 16 + 6: return a87;
    case 8 * 16 + 0: return a91;
    case 8 * 16 + 3: return a94;
    case 8 * 16 + 4: return a95;
    case 8 * 16 + 5: return a96;
    case 8 * 16 + 6: return a97;
    case 8 * 16 + 7: return a98;
    case 9 * 16 + 0: return a101;
    case 9 * 16 + 3: return a104;
    case 9 * 16 + 4: return a105;
    case 9 * 16 + 5: return a106;
    case 9 * 16 + 6: return a107;
    case 9 * 16 + 7: return a108;
    case 9 * 16 + 8: return a109;
    case 10 * 16 + 0: return a111;
    case 10 * 16 + 3: return a114;
    case 10 * 16 + 4: return a115;
    case 10 * 16 + 5: return a116;
    case 10 * 16 + 6: return a117;
    case 10 * 16 + 7: return a118;
    case 10 * 16 + 8: return a119;
    case 10 * 16 + 9: return a1110;
    case 11 * 16 + 0: return a121;
    case 11 * 16 + 3: return a124;
    case 11 * 16 + 4: return a125;
    case 11 * 16 + 5: return a126;
    case 11 * 16 + 6: return a127;
    case 11 * 16 + 7: return a128;
    case 11 * 16 + 8: return a129;
    case 11 * 16 + 9: return a1210;
    case 11 * 16 + 10: return a1211;
    case 12 * 16 + 0: return b1;
    case 12 * 16 + 5: return b6;
    case 12 * 16 + 6: return b7;
    case 12 * 16 + 7: return b8;
    case 12 * 16 + 8: return b9;
    case 12 * 16 + 9: return b10;
    case 12 * 16 + 10: return b11;
    case 12 * 16 + 11: return b12;
    case 13 * 16 + 0: return a141;
    case 13 * 16 + 6: return a147;
    case 13 * 16 + 7: return a148;
    case 13 * 16 + 8: return a149;
    case 13 * 16 + 9: return a1410;
    case 13 * 16 + 10: return a1411;
    case 13 * 16 + 11: return a1412;
    case 13 * 16 + 12: return a1413;
    case 14 * 16 + 0: return a151;
    case 14 * 16 + 5: return a156;
    case 14 * 16 + 6: return a157;
    case 14 * 16 + 7: return a158;
    case 14 * 16 + 10: return a1511;
    case 14 * 16 + 11: return a1512;
    case 14 * 16 + 12: return a1513;
    case 14 * 16 + 13: return a1514;
    case 15 * 16 + 0: return a161;
    case 15 * 16 + 5: return a166;
    case 15 * 16 + 6: return a167;
    case 15 * 16 + 7: return a168;
    case 15 * 16 + 8: return a169;
    case 15 * 16 + 12: return a1613;
    case 15 * 16 + 13: return a1614;
    case 15 * 16 + 14: return a1615;
    default: return 0.0;
  }
}

// Dense-output coefficient d_{m+4, j} of stage j (m = 0..3).
GPC_HD constexpr double Dc(int m, int j)
{
  using namespace dp;
  switch (m * 16 + j) {
    case 0 * 16 + 0: return d41;
    case 0 * 16 + 5: return d46;
    case 0 * 16 + 6: return d47;
    case 0 * 16 + 7: return d48;
    case 0 * 16 + 8: return d49;
    case 0 * 16 + 9: return d410;
    case 0 * 16 + 10: return d411;
    case 0 * 16 + 11: return d412;
    case 0 * 16 + 12: return d413;
    case 0 * 16 + 13: return d414;
    case 0 * 16 + 14: return d415;
    case 0 * 16 + 15: return d416;
    case 1 * 16 + 0: return d51;
    case 1 * 16 + 5: return d56;
    case 1 * 16 + 6: return d57;
    case 1 * 16 + 7: return d58;
    case 1 * 16 + 8: return d59;
    case 1 * 16 + 9: return d510;
    case 1 * 16 + 10: return d511;
    case 1 * 16 + 11: return d512;
    case 1 * 16 + 12: return d513;
    case 1 * 16 + 13: return d514;
    case 1 * 16 + 14: return d515;
    case 1 * 16 + 15: return d516;
    case 2 * 16 + 0: return d61;
    case 2 * 16 + 5: return d66;
    case 2 * 16 + 6: return d67;
    case 2 * 16 + 7: return d68;
    case 2 * 16 + 8: return d69;
    case 2 * 16 + 9: return d610;
    case 2 * 16 + 10: return d611;
    case 2 * 16 + 11: return d612;
    case 2 * 16 + 12: return d613;
    case 2 * 16 + 13: return d614;
    case 2 * 16 + 14: return d615;
    case 2 * 16 + 15: return d616;
    case 3 * 16 + 0: return d71;
    case 3 * 16 + 5: return d76;
    case 3 * 16 + 6: return d77;
    case 3 * 16 + 7: return d78;
    case 3 * 16 + 8: return d79;
    case 3 * 16 + 9: return d710;
    case 3 * 16 + 10: return d711;
    case 3 * 16 + 11: return d712;
    case 3 * 16 + 12: return d713;
    case 3 * 16 + 13: return d714;
    case 3 * 16 + 14: return d715;
    case 3 * 16 + 15: return d716;
    default: return 0.0;
  }
}

// Weights W_j(s) of the dense output y(t_n + s h) = y_n + h sum_j W_j k_j.
// Hairer's continuous extension
//   y + s (dy + s' (bspl + s (r4 + s' (r5 + s (r6 + s' (r7 + s r8))))))
// (s' = 1 - s, dy = h sum b_j k_j, bspl = h k_0 - dy,
// r4 = dy - h k_12 - bspl, r_{m} = h sum_j d_{m,j} k_j) is linear in the
// stages; expanding the products gives these weights.
GPC_HD GPC_FI void dense_weights(double s, double* W)
{
  const double s1 = 1.0 - s;
  const double P1 = s, P2 = s * s1, P3 = s * P2, P4 = P3 * s1, P5 = P4 * s, P6 = P5 * s1,
               P7 = P6 * s;
  const double cb = P1 - P2 + 2.0 * P3;
#pragma unroll
  for (int j = 0; j < 16; j++)
    W[j] = cb * A(12, j) + P4 * Dc(0, j) + P5 * Dc(1, j) + P6 * Dc(2, j) + P7 * Dc(3, j);
  W[0] += P2 - P3;
  W[12] -= P3;
}

// ------------------------------------------------------------ field ---
template <class POT>
struct Field {
  const GpComp* comp;
  int ncomp;
  const double* scal;
};

template <bool PLANAR, class POT>
GPC_HD GPC_NI V3 accel_at(const GpComp* __restrict__ comp, int ncomp, const double* scal,
                          double x, double y, double z)
{
  V3 a = {0.0, 0.0, 0.0};
  accel<double, PLANAR, POT>(comp, ncomp, x, y, z, a.x, a.y, a.z, scal);
  return a;
}

// k = f(Y) = (velocities, accelerations); state (x, y[, z], vx, vy[, vz]).
template <int D, class POT>
GPC_HD GPC_FI void rhs(const Field<POT>& F, const double* Y, double* k)
{
  const V3 a = accel_at<D == 2, POT>(F.comp, F.ncomp, F.scal, Y[0], Y[1],
                                     D == 3 ? Y[D - 1] : 0.0);
#pragma unroll
  for (int c = 0; c < D; c++) k[c] = Y[D + c];
  k[D] = a.x;
  k[D + 1] = a.y;
  if (D == 3) k[2 * D - 1] = a.z;
}

// Stages I0..I1-1 from y with step h (k[0..I0-1] given).  Q, if not null,
// receives the stage positions.
template <int D, class POT, int I0, int I1>
GPC_HD GPC_FI void run_stages(const Field<POT>& F, const double* y, double h, double (*k)[2 * D],
                              double (*Q)[D])
{
  constexpr int N = 2 * D;
#pragma unroll
  for (int i = I0; i < I1; i++) {
    double acc[N];
#pragma unroll
    for (int c = 0; c < N; c++) acc[c] = 0.0;
#pragma unroll
    for (int j = 0; j < i; j++) {
      const double a = A(i, j);
      if (a != 0.0) {
#pragma unroll
        for (int c = 0; c < N; c++) acc[c] += a * k[j][c];
      }
    }
    double Y[N];
#pragma unroll
    for (int c = 0; c < N; c++) Y[c] = y[c] + h * acc[c];
    if (Q) {
#pragma unroll
      for (int c = 0; c < D; c++) Q[i][c] = Y[c];
    }
    rhs<D, POT>(F, Y, k[i]);
  }
}

// ------------------------------------------------------- controller ---
struct Ctl {
  double h, hnew, hmax, pos_neg, facold, rtol, atol, t;
  bool reject;
};

GPC_HD GPC_FI void begin_attempt(Ctl& c) { c.h = c.pos_neg * dmax(fabs(c.h), 1e3 * 2.3e-16); }

// Initial step (leung_dop853.c:296-324); leaves k[0] = f(y).
template <int D, class POT>
GPC_HD void hinit(const Field<POT>& F, const double* y, double (*k)[2 * D], Ctl& c)
{
  constexpr int N = 2 * D;
  rhs<D, POT>(F, y, k[0]);
  double dnf = 0.0, dny = 0.0;
#pragma unroll
  for (int i = 0; i < N; i++) {
    const double sk = c.atol + c.rtol * fabs(y[i]);
    double sqr = k[0][i] / sk;
    dnf += sqr * sqr;
    sqr = y[i] / sk;
    dny += sqr * sqr;
  }
  c.h = csign(dmin(sqrt(dny / dnf) * 0.01, fabs(c.hmax)), c.pos_neg);
  double y1[N];
#pragma unroll
  for (int i = 0; i < N; i++) y1[i] = y[i] + c.h * k[0][i];
  rhs<D, POT>(F, y1, k[1]);
  double der2 = 0.0;
#pragma unroll
  for (int i = 0; i < N; i++) {
    const double sk = c.atol + c.rtol * fabs(y[i]);
    const double sqr = (k[1][i] - k[0][i]) / sk;
    der2 += sqr * sqr;
  }
  der2 = sqrt(der2) / c.h;
  const double der12 = dmax(fabs(der2), sqrt(dnf));
  const double h1 = pow(0.01 / der12, 1.0 / 8.0);
  c.h = csign(dmin(100.0 * fabs(c.h), dmin(fabs(h1), fabs(c.hmax))), c.pos_neg);
  begin_attempt(c);
}

// The new state of a step, y + h sum_j b_j k_j, in the reference's order of
// summation; also returns the combined increment (used by the error test).
template <int D>
GPC_HD GPC_FI void new_state(const double* y, double h, const double (*k)[2 * D], double* inc,
                             double* ynew)
{
  using namespace dp;
#pragma unroll
  for (int i = 0; i < 2 * D; i++) {
    inc[i] = b1 * k[0][i] + b6 * k[5][i] + b7 * k[6][i] + b8 * k[7][i] + b9 * k[8][i] +
             b10 * k[9][i] + b11 * k[10][i] + b12 * k[11][i];
    ynew[i] = y[i] + h * inc[i];
  }
}

// One attempt with step c.h from y (k[0] = f(y) given): stages 1..11, the
// error estimate and the controller decision (leung_dop853.c:330-440).
// Returns 1 accepted (ynew set, c.hnew proposed), 0 rejected (c.h reduced
// for the next attempt), -1 non-finite error norm.
template <int D, class POT>
GPC_HD int attempt(const Field<POT>& F, const double* y, double (*k)[2 * D], double* ynew, Ctl& c)
{
  using namespace dp;
  constexpr int N = 2 * D;
  run_stages<D, POT, 1, 12>(F, y, c.h, k, nullptr);
  double inc[N];
  new_state<D>(y, c.h, k, inc, ynew);
  double e = 0.0, e2 = 0.0;
#pragma unroll
  for (int i = 0; i < N; i++) {
    const double sk = c.atol + c.rtol * dmax(fabs(y[i]), fabs(ynew[i]));
    double erri = inc[i] - bhh1 * k[0][i] - bhh2 * k[8][i] - bhh3 * k[11][i];
    double sqr = erri / sk;
    e2 += sqr * sqr;
    erri = er1 * k[0][i] + er6 * k[5][i] + er7 * k[6][i] + er8 * k[7][i] + er9 * k[8][i] +
           er10 * k[9][i] + er11 * k[10][i] + er12 * k[11][i];
    sqr = erri / sk;
    e += sqr * sqr;
  }
  double deno = e + 0.01 * e2;
  if (deno <= 0.0) deno = 1.0;
  e = fabs(c.h) * e * sqrt(1.0 / (deno * (double)N));
  if (!isfinite(e)) return -1;
  const double fac11 = pow(e, 1.0 / 8.0);
  const double fac = dmax(1.0 / 6.0, dmin(1.0 / 0.333, fac11 / 0.9));
  c.hnew = c.h / fac;
  if (e <= 1.0) {
    c.facold = dmax(e, 1.0e-4);
    return 1;
  }
  c.hnew = c.h / dmin(1.0 / 0.333, fac11 / 0.9);
  c.reject = true;
  c.h = c.hnew;
  begin_attempt(c);
  return 0;
}

// Step size of the next step after an accepted one (leung_dop853.c:476-500).
GPC_HD GPC_FI void next_step(Ctl& c)
{
  double hnew = (fabs(c.hnew) > fabs(c.hmax)) ? c.pos_neg * c.hmax : c.hnew;
  if (c.reject) hnew = c.pos_neg * dmin(fabs(hnew), fabs(c.h));
  c.reject = false;
  c.h = hnew;
  begin_attempt(c);
}

GPC_HD GPC_FI void init_ctl(Ctl& c, double t0, double T, double rtol_ln, double atol_ln)
{
  c.rtol = exp(rtol_ln);
  c.atol = exp(atol_ln);
  c.hmax = T - t0;
  c.pos_neg = csign(1.0, c.hmax);
  c.facold = 1.0e-4;
  c.t = t0;
  c.reject = false;
  c.h = c.hnew = 0.0;
}

// y(T) from the start of the step that contains T: stages 12..15 and the
// dense output (k[0..11] of the step given).
template <int D, class POT>
GPC_HD GPC_FI void dense_final(const Field<POT>& F, const double* y, double h, double t_start,
                               double T, double (*k)[2 * D], double* yT)
{
  run_stages<D, POT, 12, 16>(F, y, h, k, nullptr);
  double W[16];
  dense_weights((T - t_start) / h, W);
#pragma unroll
  for (int i = 0; i < 2 * D; i++) {
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < 16; j++) acc += W[j] * k[j][i];
    yT[i] = y[i] + h * acc;
  }
}

// Checkpoint record of a segment: y[N] and t at its start, then the step
// sizes of its (up to) kCkptEvery accepted steps.
template <int D>
struct Ckpt {
  static constexpr int H = 2 * D + 1;  // offset of the step sizes
  static constexpr int W = H + kCkptEvery;
};

// ---------------------------------------------------------- forward ---
// Integrate one orbit from t0 to T.  Checkpoints go to ck[(c*W + f)*cs]
// (c < ccap); the accepted step sizes, if hrec is not null, to
// hrec[n*hs] (n < hcap).  Returns the status (E_OK, E_BUDGET when the
// attempt budget, checkpoint or step capacity is exhausted, E_NONFINITE).
template <int D, class POT>
GPC_HD int forward_orbit(const Field<POT>& F, const double* w0, double t0, double T,
                         double rtol_ln, double atol_ln, long long max_att, double* ck,
                         long long cs, int ccap, double* hrec, long long hs, long long hcap,
                         double* yT, long long* nsteps)
{
  constexpr int N = 2 * D, CW = Ckpt<D>::W;
  double y[N], ynew[N], k[16][N];
#pragma unroll
  for (int i = 0; i < N; i++) y[i] = w0[i];
  *nsteps = 0;
  if (T == t0) {
#pragma unroll
    for (int i = 0; i < N; i++) yT[i] = y[i];
    return E_OK;
  }
  Ctl c;
  init_ctl(c, t0, T, rtol_ln, atol_ln);
  hinit<D, POT>(F, y, k, c);
  long long n = 0, att = 0;
  for (;;) {
    if (n % kCkptEvery == 0) {
      const long long seg = n / kCkptEvery;
      if (seg >= ccap) return E_BUDGET;
      double* p = ck + seg * CW * cs;
#pragma unroll
      for (int i = 0; i < N; i++) p[i * cs] = y[i];
      p[N * cs] = c.t;
    }
    for (int rej = 0;; rej++) {
      // every rejection shrinks h by at least 1/1.11 down to the floor of
      // begin_attempt; an orbit still rejected long after that is stopped
      if (rej >= kMaxRejects) return E_BUDGET;
      const int r = attempt<D, POT>(F, y, k, ynew, c);
      att++;
      if (r < 0) return E_NONFINITE;
      if (r > 0) break;
      if (max_att > 0 && att >= max_att) return E_BUDGET;
    }
    ck[((n / kCkptEvery) * CW + Ckpt<D>::H + n % kCkptEvery) * cs] = c.h;
    if (hrec) {
      if (n >= hcap) return E_BUDGET;
      hrec[n * hs] = c.h;
    }
    const double t_start = c.t;
    c.t = t_start + c.h;
    n++;
    if (c.pos_neg * T < c.pos_neg * c.t) {  // T lies in this step
      dense_final<D, POT>(F, y, c.h, t_start, T, k, yT);
      *nsteps = n;
      return E_OK;
    }
    rhs<D, POT>(F, ynew, k[0]);  // FSAL: f at the new state starts the next step
#pragma unroll
    for (int i = 0; i < N; i++) y[i] = ynew[i];
    next_step(c);
    if (max_att > 0 && att >= max_att) return E_BUDGET;
  }
}

// ------------------------------------------------ replay (fixed steps) ---
// The forward map with the step sizes held at recorded values h[n*hs],
// n < nsteps (the function the adjoint differentiates; finite differences
// of it check the gradients).
template <int D, class POT>
GPC_HD void replay_orbit(const Field<POT>& F, const double* w0, double t0, double T,
                         const double* hrec, long long hs, long long nsteps, double* yT)
{
  constexpr int N = 2 * D;
  double y[N], ynew[N], inc[N], k[16][N];
#pragma unroll
  for (int i = 0; i < N; i++) y[i] = w0[i];
  if (nsteps <= 0) {
#pragma unroll
    for (int i = 0; i < N; i++) yT[i] = y[i];
    return;
  }
  double t = t0;
  for (long long n = 0; n < nsteps; n++) {
    const double h = hrec[n * hs];
    rhs<D, POT>(F, y, k[0]);
    run_stages<D, POT, 1, 12>(F, y, h, k, nullptr);
    if (n == nsteps - 1) {
      dense_final<D, POT>(F, y, h, t, T, k, yT);
      return;
    }
    new_state<D>(y, h, k, inc, ynew);
#pragma unroll
    for (int i = 0; i < N; i++) y[i] = ynew[i];
    t = t + h;
  }
}

// --------------------------------------------------------- backward ---
// Adjoint of one step from y with step h: lam (dL/d output) becomes
// dL/dy; g accumulates dL/dtheta.  LAST: the step is the dense-output map
// to s = (T - t_n)/h.
template <int D, class POT, bool LAST>
GPC_HD void step_vjp(const Field<POT>& F, const double* y, double h, double s, double* lam,
                     double* g)
{
  constexpr int N = 2 * D, S = LAST ? 16 : 12;
  double k[S][N], Q[S][D];
  rhs<D, POT>(F, y, k[0]);
#pragma unroll
  for (int c = 0; c < D; c++) Q[0][c] = y[c];
  run_stages<D, POT, 1, S>(F, y, h, k, Q);
  double W[16];
  if (LAST) {
    dense_weights(s, W);
  } else {
#pragma unroll
    for (int j = 0; j < 16; j++) W[j] = A(12, j);
  }
  double mu[S][N];
#pragma unroll
  for (int i = S - 1; i >= 0; i--) {
    double kap[N];
#pragma unroll
    for (int c = 0; c < N; c++) kap[c] = h * W[i] * lam[c];
#pragma unroll
    for (int j = i + 1; j < S; j++) {
      const double a = A(j, i);
      if (a != 0.0) {
#pragma unroll
        for (int c = 0; c < N; c++) kap[c] += h * a * mu[j][c];
      }
    }
    double Kv[D];
    accel_vjp<D>(F.comp, F.ncomp, Q[i], kap + D, Kv, g);
#pragma unroll
    for (int c = 0; c < D; c++) {
      mu[i][c] = Kv[c];
      mu[i][D + c] = kap[c];
    }
  }
#pragma unroll
  for (int c = 0; c < N; c++) {
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < S; i++) acc += mu[i][c];
    lam[c] += acc;
  }
}

// Backward sweep of one orbit: lam = dL/dy(T) on entry, dL/dy(t0) on exit;
// g (group_nparam entries, zeroed by the caller) accumulates dL/dtheta.
// ck/cs: the forward pass's checkpoints; nsteps its accepted steps.
template <int D, class POT>
GPC_HD void backward_orbit(const Field<POT>& F, double T, const double* ck, long long cs,
                           long long nsteps, double* lam, double* g)
{
  constexpr int N = 2 * D, CW = Ckpt<D>::W;
  if (nsteps <= 0) return;
  double ys[kCkptEvery][N], ts[kCkptEvery];
  const long long nseg = (nsteps + kCkptEvery - 1) / kCkptEvery;
  for (long long seg = nseg - 1; seg >= 0; seg--) {
    // recompute the start states of the segment's steps
    const double* p = ck + seg * CW * cs;
    const double* hs = p + Ckpt<D>::H * cs;
    const long long n0 = seg * kCkptEvery;
    const int m1 = (int)((n0 + kCkptEvery < nsteps ? n0 + kCkptEvery : nsteps) - n0);
    double y[N], ynew[N], inc[N], k[12][N];
#pragma unroll
    for (int i = 0; i < N; i++) y[i] = p[i * cs];
    double t = p[N * cs];
    for (int m = 0; m < m1; m++) {
#pragma unroll
      for (int i = 0; i < N; i++) ys[m][i] = y[i];
      ts[m] = t;
      if (m == m1 - 1) break;
      const double h = hs[m * cs];
      rhs<D, POT>(F, y, k[0]);
      run_stages<D, POT, 1, 12>(F, y, h, k, nullptr);
      new_state<D>(y, h, k, inc, ynew);
#pragma unroll
      for (int i = 0; i < N; i++) y[i] = ynew[i];
      t = t + h;
    }
    // reverse sweep over the segment's steps
    for (int m = m1 - 1; m >= 0; m--) {
      const double h = hs[m * cs];
      if (n0 + m == nsteps - 1)
        step_vjp<D, POT, true>(F, ys[m], h, (T - ts[m]) / h, lam, g);
      else
        step_vjp<D, POT, false>(F, ys[m], h, 0.0, lam, g);
    }
  }
}

}  // namespace adj
}  // namespace gpc
