// galpy_b200/csrc/machines.cuh
//
// Per-orbit integrator state machines.  Each machine advances its orbit by
// exactly one force evaluation per call:
//
//     m.point(y);                // state at which the next force is needed
//     eval_force(..., y, a);     // the ONE force call site of the kernel
//     m.consume(y, a, out);      // advance, maybe write output rows
//
// so that the 32 lanes of a warp always meet at the same force call, whatever
// stage of whatever orbit each lane is in (step-size estimation, a regular
// step, a rejected DOP853 attempt, dense-output stages, or the start of a new
// orbit picked up by work stealing).  Orbits never diverge at the force call;
// only the few bookkeeping instructions around it are lane-specific.
//
// The arithmetic of every stepper follows the reference step by step so that
// the step sequence (and, for fixed-step methods, the chosen step size) is the
// reference's:
//   leapfrog/symplec4/symplec6  galpy/util/bovy_symplecticode.c:132-587
//   their step estimators       galpy/util/bovy_symplecticode.c:588-1052
//   variational (*_dxdv) forms  galpy/util/bovy_symplecticode.c:1053-1400
//   rk4 / rk6 + estimators      galpy/util/bovy_rk.c:66-480
//   dopr54                      galpy/util/bovy_rk.c:501-760
//   dop853                      galpy/util/leung_dop853.c:231-517
// Each machine also reports the time at which the reference evaluates the
// force of its current point (tpoint: the reference stepper's own
// bookkeeping, so that a time-dependent potential sees the same times); the
// kernel asks for it only when the component list reads the time.
// Differences by design: DOP853 skips its three dense-output stages in
// steps that contain no output time (their results are only used for
// output); every orbit has an attempt budget and stops on a non-finite
// state instead of looping forever.
#pragma once
#include <type_traits>

#include "dop853_tableau.cuh"
#include "gpc_common.cuh"
#include "potentials.cuh"

namespace gpc {

constexpr double kDtSentinel = -9999.99;  // galpy's "estimate the step" marker
// Stride (in doubles) between consecutive values of one thread in a
// machine's slot store: the kernel's block size, fixed at compile time so
// that slot addresses are immediate offsets.
constexpr int kSlotStride = 128;
constexpr double kMaxDtReduce = 10000.;

enum : int { M_LEAPFROG = 0, M_RK4 = 1, M_RK6 = 2, M_SYMPLEC4 = 3, M_SYMPLEC6 = 4, M_DOPR54 = 5,
             M_DOP853 = 6 };
enum : int { PREC_FP64 = 0, PREC_F32 = 1 };

// symplec4 coefficients (Kinoshita et al.; bovy_symplecticode.c:96-99)
constexpr double s4c1 = 0.6756035959798289, s4c2 = -0.1756035959798288;
constexpr double s4c3 = -0.1756035959798288, s4c4 = 0.6756035959798289;
constexpr double s4d1 = 1.3512071919596578, s4d2 = -1.7024143839193153;
constexpr double s4d3 = 1.3512071919596578;
// symplec6 coefficients (Yoshida 1990; bovy_symplecticode.c:100-107): the
// drifts c1..c8 and kicks d1..d7 are palindromic
constexpr double s6c1 = 0.392256805238780, s6c2 = 0.510043411918458;
constexpr double s6c3 = -0.471053385409758, s6c4 = 0.687531682525198e-1;
constexpr double s6d1 = 0.784513610477560, s6d2 = 0.235573213359357;
constexpr double s6d3 = -0.117767998417887e1, s6d4 = 0.131518632068391e1;

// ------------------------------------------------------------------------
// output rows
// ------------------------------------------------------------------------
enum : int { L_GALPY_CYL = 0, L_AOS_RECT = 1, L_SOA_RECT = 2, L_SOA_CYL = 3 };
// what a stored state is: an orbit (rectangular), the 3D surface-of-section
// state, or the planar one for the surface x = 0 / y = 0
enum : int { ROW_ORBIT = 0, ROW_SOS = 1, ROW_SOS_PLANAR_X = 2, ROW_SOS_PLANAR_Y = 3 };

struct OutSpec {
  double* out;
  int layout;
  int nt;        // rows per orbit produced by the integrator
  int row0;      // first row stored (0 = all; nt-1 = final state only)
  long long nobj;
};

// Write row j of orbit i.  v is the rectangular state in the reference's row
// order: plain 3D (x,y,z,vx,vy,vz), planar (x,y,vx,vy); variational rows
// (x, v, dx, dv) are always written rectangular.
template <int NV, int D, bool CYL_OK, int ROW = ROW_ORBIT>
GPC_HD GPC_FI void write_row(const OutSpec& o, long long i, int j, const double* v)
{
  if (j < o.row0) return;
  const long long nrow = o.nt - o.row0, jj = j - o.row0;
  double w[NV];
  const bool cyl = CYL_OK && (o.layout == L_GALPY_CYL || o.layout == L_SOA_CYL);
  if constexpr (ROW == ROW_SOS_PLANAR_X || ROW == ROW_SOS_PLANAR_Y) {
    if (cyl) {
      // (u, vu, A, t, psi) -> (R, vR, vT, phi, t): sos_to_polar_galpy
      // (bovy_coords.c:235-260)
      const double w1 = v[2] * sin(v[4]), w2 = v[2] * cos(v[4]);
      const double x = ROW == ROW_SOS_PLANAR_X ? w1 : v[0];
      const double vx = ROW == ROW_SOS_PLANAR_X ? w2 : v[1];
      const double y = ROW == ROW_SOS_PLANAR_X ? v[0] : w1;
      const double vy = ROW == ROW_SOS_PLANAR_X ? v[1] : w2;
      const double phi = atan2(y, x), cp = cos(phi), sp = sin(phi);
      w[0] = sqrt(x * x + y * y);
      w[1] = vx * cp + vy * sp;
      w[2] = -vx * sp + vy * cp;
      w[3] = phi;
      w[4] = v[3];
    } else {
#pragma unroll
      for (int k = 0; k < NV; k++) w[k] = v[k];
    }
  } else if constexpr (ROW == ROW_SOS) {
    if (cyl) {
      // surface of section (x, y, vx, vy, A, t, psi) -> (R, vR, vT, z, vz,
      // phi, t): sos_to_cyl_galpy (bovy_coords.c:173-189)
      const double x = v[0], y = v[1];
      const double phi = atan2(y, x), cp = cos(phi), sp = sin(phi);
      w[0] = sqrt(x * x + y * y);
      w[1] = v[2] * cp + v[3] * sp;
      w[2] = -v[2] * sp + v[3] * cp;
      w[3] = v[4] * sin(v[6]);
      w[4] = v[4] * cos(v[6]);
      w[5] = phi;
      w[6] = v[5];
    } else {
#pragma unroll
      for (int k = 0; k < NV; k++) w[k] = v[k];
    }
  } else if (cyl) {
    // rect_to_cyl_galpy / rect_to_polar_galpy (bovy_coords.c:79-148), with
    // (cos phi, sin phi) = (x, y) / R instead of two more special functions
    // (the same values to an ulp or two; atan2's own convention at R = 0)
    const double x = v[0], y = v[1];
    const double vx = v[D], vy = v[D + 1];
    const double phi = atan2(y, x), R = sqrt(x * x + y * y);
    double cp, sp;
    if (R > 0.0) {
      const double iR = 1.0 / R;
      cp = x * iR;
      sp = y * iR;
    } else {
      cp = cos(phi);
      sp = sin(phi);
    }
    w[0] = R;
    w[1] = vx * cp + vy * sp;
    w[2] = -vx * sp + vy * cp;
    if (D == 3) {
      w[3] = v[2];
      w[4] = v[5];
      w[5] = phi;
    } else {
      w[3] = phi;
    }
  } else {
#pragma unroll
    for (int k = 0; k < NV; k++) w[k] = v[k];
  }
  if (o.layout == L_SOA_RECT || o.layout == L_SOA_CYL) {
#pragma unroll
    for (int k = 0; k < NV; k++) o.out[((long long)k * nrow + jj) * o.nobj + i] = w[k];
  } else {
    double* p = o.out + (i * nrow + jj) * NV;
#pragma unroll
    for (int k = 0; k < NV; k++) p[k] = w[k];
  }
}

template <int NV, int D, bool CYL_OK, int ROW = ROW_ORBIT>
GPC_HD GPC_FI void write_nan_rows(const OutSpec& o, long long i, int from)
{
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = NAN;
  for (int j = from; j < o.nt; j++) write_row<NV, D, CYL_OK, ROW>(o, i, j, v);
}

// ------------------------------------------------------------------------
// force adapter: positions -> accelerations (+ K . dq for variational runs)
// ------------------------------------------------------------------------
template <int D, int PREC, bool VAR, class POT = DynPot>
GPC_HD GPC_FI void eval_force(const GpComp* comp, int ncomp, const double* q, double* a,
                              const double* scal = nullptr, double t = 0.0)
{
  if (!VAR) {
    if (PREC == PREC_FP64) {
      double ax, ay, az = 0.0;
      accel<double, D == 2, POT>(comp, ncomp, q[0], q[1], D == 3 ? q[2] : 0.0, ax, ay, az, scal,
                                 t);
      a[0] = ax;
      a[1] = ay;
      if (D == 3) a[2] = az;
    } else {
      float ax, ay, az = 0.f;
      accel<float, D == 2, POT>(comp, ncomp, (float)q[0], (float)q[1], D == 3 ? (float)q[2] : 0.f,
                                ax, ay, az, scal, t);
      a[0] = ax;
      a[1] = ay;
      if (D == 3) a[2] = az;
    }
  } else {
    double ax, ay, az, K[6];
    accel_tidal<D == 2>(comp, ncomp, q[0], q[1], D == 3 ? q[2] : 0.0, ax, ay, az, K, t);
    a[0] = ax;
    a[1] = ay;
    if (D == 3) {
      a[2] = az;
      const double dx = q[3], dy = q[4], dz = q[5];
      a[3] = K[0] * dx + K[1] * dy + K[3] * dz;
      a[4] = K[1] * dx + K[2] * dy + K[4] * dz;
      a[5] = K[3] * dx + K[4] * dy + K[5] * dz;
    } else {
      const double dx = q[2], dy = q[3];
      a[2] = K[0] * dx + K[1] * dy;
      a[3] = K[1] * dx + K[2] * dy;
    }
  }
}

// log-sum-exp error scale of the fixed-step estimators
// (bovy_symplecticode.c:609-624, bovy_rk.c:346-353)
GPC_HD GPC_FI double est_scale(const double* v, int n, int stride, double rtol, double atol)
{
  double m = log(fabs(v[0]));
  for (int i = 1; i < n; i++) {
    const double l = log(fabs(v[i * stride]));
    if (l > m) m = l;
  }
  const double c = fmax(atol, rtol + m);
  return log(exp(atol - c) + exp(rtol + m - c)) + c;
}

struct OrbitCommon {
  const double* t;  // this orbit's output times
  int nt;
  int iout;         // last row written
  int err;
  bool done;
  long long nsteps;    // accepted steps
  long long attempts;  // force-consuming step attempts (budget)
  long long max_attempts;
};

// ------------------------------------------------------------------------
// leapfrog / symplec4 / symplec6 (optionally variational)
// ------------------------------------------------------------------------
// Drift-kick compositions: ORD 2 (leapfrog: drifts h/2, h/2; kick h), 4
// (symplec4: 4 drifts, 3 kicks) and 6 (symplec6: 8 drifts, 7 kicks).  The last
// drift of a step merges with the first of the next, as in the reference.
template <int ORD>
struct Composition;
template <>
struct Composition<2> {
  static constexpr int kKicks = 1;
  GPC_HD GPC_FI static double first(double h) { return h / 2.; }
  GPC_HD GPC_FI static double kick(int, double h) { return h; }
  // drift after kick j: the step's last (merged with the next step's first
  // unless `last`)
  GPC_HD GPC_FI static double drift(int, bool last, double h) { return last ? h / 2. : h; }
};
template <>
struct Composition<4> {
  static constexpr int kKicks = 3;
  GPC_HD GPC_FI static double first(double h) { return s4c1 * h; }
  GPC_HD GPC_FI static double kick(int j, double h)
  {
    return j == 0 ? s4d1 * h : (j == 1 ? s4d2 * h : s4d3 * h);
  }
  GPC_HD GPC_FI static double drift(int j, bool last, double h)
  {
    return j == 0 ? s4c2 * h : (j == 1 ? s4c3 * h : (last ? s4c4 * h : (s4c4 + s4c1) * h));
  }
};
template <>
struct Composition<6> {
  static constexpr int kKicks = 7;
  GPC_HD GPC_FI static double first(double h) { return s6c1 * h; }
  GPC_HD GPC_FI static double kick(int j, double h)
  {
    const int m = j < 4 ? j : 6 - j;  // d5..d7 mirror d3..d1
    const double d = m == 0 ? s6d1 : (m == 1 ? s6d2 : (m == 2 ? s6d3 : s6d4));
    return d * h;
  }
  GPC_HD GPC_FI static double drift(int j, bool last, double h)
  {
    // after kick j comes drift c_{j+2}; c5..c8 mirror c4..c1
    if (j == 6) return last ? s6c1 * h : (s6c1 + s6c1) * h;  // c8 (+ c1)
    const int m = j < 3 ? j + 1 : 6 - j;
    const double c = m == 1 ? s6c2 : (m == 2 ? s6c3 : s6c4);
    return c * h;
  }
};

// ------------------------------------------------------------------------
// double-float numbers (head + tail floats, ~48 significant bits): the
// compensated state of the symplectic machines' FP32-force form.  Sums by
// Knuth's TwoSum, products by Dekker's with a fused multiply-add for the
// rounding error of the heads' product, each renormalised with Fast2Sum.
// ------------------------------------------------------------------------
struct DFloat {
  float hi, lo;
};
GPC_HD GPC_FI DFloat df_of(double x)
{
  const float h = (float)x;
  return {h, (float)(x - (double)h)};
}
GPC_HD GPC_FI double df_val(DFloat a) { return (double)a.hi + (double)a.lo; }
GPC_HD GPC_FI DFloat df_add(DFloat a, DFloat b)
{
  const float s = a.hi + b.hi;
  const float bb = s - a.hi;
  const float e = ((a.hi - (s - bb)) + (b.hi - bb)) + (a.lo + b.lo);
  const float h = s + e;
  return {h, e - (h - s)};
}
GPC_HD GPC_FI DFloat df_mul(DFloat a, DFloat b)
{
  const float p = a.hi * b.hi;
  const float e = fmaf(a.hi, b.hi, -p) + (a.hi * b.lo + a.lo * b.hi);
  const float h = p + e;
  return {h, e - (h - p)};
}
GPC_HD GPC_FI DFloat df_mulf(DFloat a, float f)
{
  const float p = a.hi * f;
  const float e = fmaf(a.hi, f, -p) + a.lo * f;
  const float h = p + e;
  return {h, e - (h - p)};
}

// Running state of a symplectic advance: float64, or double-float (DFloat).
GPC_HD GPC_FI double state_val(double x) { return x; }
GPC_HD GPC_FI double state_val(DFloat x) { return df_val(x); }

template <int D, bool VAR, int ORD, class S = double>
struct SymplecticMachine : OrbitCommon {
  using C = Composition<ORD>;
  static constexpr bool kDF = !std::is_same<S, double>::value;  // double-float state
  static constexpr int NQ = VAR ? 2 * D : D;  // stepped positions
  static constexpr int NY = NQ;               // size of the force argument
  static constexpr int NV = 2 * NQ;           // values per output row
  static constexpr int NA = NQ;               // force result size
  static constexpr int kRow = ROW_ORBIT;
  static constexpr int kSlotDoubles = 0;      // no slot store needed
  GPC_HD GPC_FI void bind(double*) {}
  GPC_HD GPC_FI bool wants_dense() const { return false; }
  GPC_HD GPC_FI static int next_slot(int slot, bool) { return slot >= 14 ? 0 : slot + 1; }
  GPC_HD GPC_FI static void pos(const double* y, double* q)
  {
#pragma unroll
    for (int k = 0; k < NQ; k++) q[k] = y[k];
  }
  enum { EST_FULL = 0, EST_HALF = 1, MAIN = 2 };
  double qo[NQ], po[NQ];  // state at the last output
  S qw[NQ], pw[NQ];       // state of the running advance
  double q11[D], p11[D];  // estimator: the single-step result (base orbit)
  double dt, init_dt, h, sq, sp, rtol, atol;
  // the reference's time `to` (bovy_symplecticode.c): symplec4 / symplec6
  // add each drift's length to it and kick at it (their estimators take it
  // back by dt after each trial); leapfrog kicks at to + dt/2 and adds dt
  // per step (its estimator kicks at t0 + dt/2, t0 + dt/4, t0 + 3 dt/4)
  double tk;
  long long nrun, kick, nkick;
  int sub, phase;
  // double-float form: the step's kick and drift coefficients, converted
  // once per advance (the drift after the last kick of the advance is dlast)
  DFloat kc0, kc1, kc2, dc0, dc1, dc2, dlast;

  GPC_HD GPC_FI static DFloat pick3(int j, DFloat a, DFloat b, DFloat c)
  {
    return j == 0 ? a : (j == 1 ? b : c);
  }

  GPC_HD GPC_FI void start(double hh, long long nstep)
  {
    h = hh;
    nrun = nstep;
    kick = 0;
    sub = 0;
    nkick = C::kKicks * nstep;
    const double c = C::first(h);
    if (ORD != 2) tk += c;
    if constexpr (kDF) {
      static_assert(C::kKicks <= 3, "double-float state: leapfrog and symplec4");
      kc0 = df_of(C::kick(0, h));
      kc1 = df_of(C::kick(C::kKicks > 1 ? 1 : 0, h));
      kc2 = df_of(C::kick(C::kKicks > 2 ? 2 : 0, h));
      dc0 = df_of(C::drift(0, false, h));
      dc1 = df_of(C::drift(C::kKicks > 1 ? 1 : 0, false, h));
      dc2 = df_of(C::drift(C::kKicks > 2 ? 2 : 0, false, h));
      dlast = df_of(C::drift(C::kKicks - 1, true, h));
      const DFloat cd = df_of(c);
#pragma unroll
      for (int k = 0; k < NQ; k++) {
        qw[k] = df_add(df_of(qo[k]), df_mul(cd, df_of(po[k])));
        pw[k] = df_of(po[k]);
      }
    } else {
#pragma unroll
      for (int k = 0; k < NQ; k++) {
        qw[k] = qo[k] + c * po[k];
        pw[k] = po[k];
      }
    }
  }

  GPC_HD GPC_FI void row(double* v) const
  {
    // output order (x, v) for the base and (dx, dv) for the deviation
#pragma unroll
    for (int k = 0; k < D; k++) {
      v[k] = qo[k];
      v[D + k] = po[k];
      if (VAR) {
        v[2 * D + k] = qo[D + k];
        v[3 * D + k] = po[D + k];
      }
    }
  }

  GPC_HD GPC_FI void begin_main()
  {
    const long long ndt = (long long)(init_dt / dt);
    phase = MAIN;
    tk = t[0];
    start(dt, ndt < 1 ? 1 : ndt);
  }

  // time of the force evaluation of the current kick
  GPC_HD GPC_FI double tpoint(const double* /*y*/, int /*slot*/) const
  {
    if (ORD != 2) return tk;
    if (phase == MAIN) return tk + dt / 2.;
    if (phase == EST_FULL) return t[0] + dt / 2.;
    return kick == 0 ? t[0] + dt / 4. : t[0] + 3. * dt / 4.;
  }

  // w: (x, v) or (x, v, dx, dv) rectangular
  template <class W>
  GPC_HD void init(const double* w, const double* tt, int nt_, double dt_in, double rtol_,
                   double atol_, long long max_att, W& out)
  {
    t = tt;
    nt = nt_;
    iout = 0;
    err = E_OK;
    done = false;
    nsteps = 0;
    attempts = 0;
    max_attempts = max_att;
    rtol = rtol_;
    atol = atol_;
#pragma unroll
    for (int k = 0; k < D; k++) {
      qo[k] = w[k];
      po[k] = w[D + k];
      if (VAR) {
        qo[D + k] = w[2 * D + k];
        po[D + k] = w[3 * D + k];
      }
    }
    double v[NV];
    row(v);
    out(0, v);
    if (nt < 2) {
      done = true;
      return;
    }
    init_dt = tt[1] - tt[0];
    tk = tt[0];
    if (dt_in == kDtSentinel) {
      dt = init_dt;
      sq = est_scale(qo, D, 1, rtol, atol);
      sp = est_scale(po, D, 1, rtol, atol);
      phase = EST_FULL;
      start(dt, 1);
    } else {
      dt = dt_in;
      begin_main();
    }
  }

  GPC_HD GPC_FI void point(double* y, int /*slot*/) const
  {
    // the double-float form hands its head to the single-precision force
#pragma unroll
    for (int k = 0; k < NQ; k++) {
      if constexpr (kDF)
        y[k] = (double)qw[k].hi;
      else
        y[k] = qw[k];
    }
  }

  template <class W>
  GPC_HD void consume(const double* /*y*/, const double* a, W& out, int /*slot*/)
  {
    const bool last = (kick == nkick - 1);
    if constexpr (kDF) {
      const DFloat dk = pick3(sub, kc0, kc1, kc2);
#pragma unroll
      for (int k = 0; k < NQ; k++) pw[k] = df_add(pw[k], df_mulf(dk, (float)a[k]));
      const DFloat dd = last ? dlast : pick3(sub, dc0, dc1, dc2);
#pragma unroll
      for (int k = 0; k < NQ; k++) qw[k] = df_add(qw[k], df_mul(dd, pw[k]));
    } else {
      const double dk = C::kick(sub, h);
#pragma unroll
      for (int k = 0; k < NQ; k++) pw[k] = pw[k] + dk * a[k];
      const double dc = C::drift(sub, last, h);
#pragma unroll
      for (int k = 0; k < NQ; k++) qw[k] = qw[k] + dc * pw[k];
    }
    if (ORD != 2)
      tk += C::drift(sub, last, h);
    else if (phase == MAIN)
      tk = tk + dt;
    kick++;
    sub = sub < C::kKicks - 1 ? sub + 1 : 0;
    if (last) advance_done(out);
  }

  template <class W>
  GPC_HD void advance_done(W& out)
  {
    if (phase != MAIN && ORD != 2) tk -= dt;  // the estimator's `to -= dt`
    if (phase == EST_FULL) {
#pragma unroll
      for (int k = 0; k < D; k++) {
        q11[k] = state_val(qw[k]);
        p11[k] = state_val(pw[k]);
      }
      phase = EST_HALF;
      start(dt / 2., 2);
      return;
    }
    if (phase == EST_HALF) {
      double e = 0.;
#pragma unroll
      for (int k = 0; k < D; k++) {
        e += exp(2. * log(fabs(q11[k] - state_val(qw[k]))) - 2. * sq);
        e += exp(2. * log(fabs(p11[k] - state_val(pw[k]))) - 2. * sp);
      }
      e = sqrt(e / 2. / D);
      if (e > 1. && init_dt / dt < kMaxDtReduce) {
        dt /= 2.;
        phase = EST_FULL;
        start(dt, 1);
      } else {
        begin_main();
      }
      return;
    }
    // MAIN: one output interval completed
    bool fin = true;
#pragma unroll
    for (int k = 0; k < NQ; k++) {
      qo[k] = state_val(qw[k]);
      po[k] = state_val(pw[k]);
      fin = fin && isfinite(qo[k]) && isfinite(po[k]);
    }
    nsteps += nrun;
    attempts += nrun;
    iout++;
    double v[NV];
    row(v);
    out(iout, v);
    if (!fin) {
      err = E_NONFINITE;
      done = true;
    } else if (iout == nt - 1) {
      done = true;
    } else if (max_attempts > 0 && attempts >= max_attempts) {
      err = E_BUDGET;
      done = true;
    } else {
      start(dt, nrun);
    }
  }
};

// ------------------------------------------------------------------------
// classical RK steps as stage machines
// ------------------------------------------------------------------------
// Stage s of one step of size h from yn: d is the derivative at the stage's
// point (yn for s = 0, ynk after), yn1 accumulates the step's result and ynk
// receives the next stage's point.
// bovy_rk4_onestep (bovy_rk.c:142-170)
template <int N>
GPC_HD GPC_FI void rk4_stage(int s, double h, const double* yn, double* yn1, double* ynk,
                             const double* d)
{
  if (s == 0 || s == 3) {
#pragma unroll
    for (int k = 0; k < N; k++) yn1[k] += h * d[k] / 6.;
  } else {
#pragma unroll
    for (int k = 0; k < N; k++) yn1[k] += h * d[k] / 3.;
  }
  if (s < 2) {
#pragma unroll
    for (int k = 0; k < N; k++) ynk[k] = yn[k] + h * d[k] / 2.;
  } else if (s == 2) {
#pragma unroll
    for (int k = 0; k < N; k++) ynk[k] = yn[k] + h * d[k];
  }
}

// bovy_rk6_onestep (bovy_rk.c:256-327): weights (11, 0, 81, 81, -32, -32,
// 11)/120; kk[0..4] hold k1..k5 (k6 is only needed for the last point)
template <int N>
GPC_HD GPC_FI void rk6_stage(int s, double h, const double* yn, double* yn1, double* ynk,
                             double (*kk)[N], const double* d)
{
  switch (s) {
    case 0:
#pragma unroll
      for (int k = 0; k < N; k++) {
        yn1[k] += 11. * h * d[k] / 120.;
        kk[0][k] = h * d[k];
        ynk[k] = yn[k] + kk[0][k] / 3.;
      }
      break;
    case 1:
#pragma unroll
      for (int k = 0; k < N; k++) {
        kk[1][k] = h * d[k];
        ynk[k] = yn[k] + 2. * kk[1][k] / 3.;
      }
      break;
    case 2:
#pragma unroll
      for (int k = 0; k < N; k++) {
        yn1[k] += 81. * h * d[k] / 120.;
        kk[2][k] = h * d[k];
        ynk[k] = yn[k] + (kk[0][k] + 4. * kk[1][k] - kk[2][k]) / 12.;
      }
      break;
    case 3:
#pragma unroll
      for (int k = 0; k < N; k++) {
        yn1[k] += 81. * h * d[k] / 120.;
        kk[3][k] = h * d[k];
        ynk[k] = yn[k] + (-kk[0][k] + 18. * kk[1][k] - 3. * kk[2][k] - 6. * kk[3][k]) / 16.;
      }
      break;
    case 4:
#pragma unroll
      for (int k = 0; k < N; k++) {
        yn1[k] -= 32. * h * d[k] / 120.;
        kk[4][k] = h * d[k];
        ynk[k] = yn[k] + (9. * kk[1][k] - 3. * kk[2][k] - 6. * kk[3][k] + 4. * kk[4][k]) / 8.;
      }
      break;
    case 5:
#pragma unroll
      for (int k = 0; k < N; k++) {
        yn1[k] -= 32. * h * d[k] / 120.;
        const double k6 = h * d[k];
        ynk[k] = yn[k] + (9. * kk[0][k] - 36. * kk[1][k] + 63. * kk[2][k] + 72. * kk[3][k] -
                          64. * k6) / 44.;
      }
      break;
    default:
#pragma unroll
      for (int k = 0; k < N; k++) yn1[k] += 11. * h * d[k] / 120.;
  }
}

// ------------------------------------------------------------------------
// ODE systems of the RK-type machines
// ------------------------------------------------------------------------
// An orbit: y = (x, v[, dx, dv]) in rectangular coordinates; dy/dt from the
// force at the positions (and K . dq for the deviations).
template <int D, bool VAR>
struct OrbitSystem {
  static constexpr int N = VAR ? 4 * D : 2 * D;  // ODE dimension
  static constexpr int NA = VAR ? 2 * D : D;     // force argument / result size
  static constexpr int kRow = ROW_ORBIT;         // output row conversion
  static constexpr int kTimeIndex = -1;          // the time is the machine's, not in y
  // force argument: positions (and deviation positions) of (x, v[, dx, dv])
  GPC_HD GPC_FI static void pos(const double* y, double* q)
  {
#pragma unroll
    for (int k = 0; k < D; k++) {
      q[k] = y[k];
      if (VAR) q[D + k] = y[2 * D + k];
    }
  }
  GPC_HD GPC_FI static void deriv(const double* y, const double* a, double* d)
  {
#pragma unroll
    for (int k = 0; k < D; k++) {
      d[k] = y[D + k];
      d[D + k] = a[k];
      if (VAR) {
        d[2 * D + k] = y[3 * D + k];
        d[3 * D + k] = a[D + k];
      }
    }
  }
};

// Surface-of-section integration (evalSOSDeriv, integrateFullOrbit.c:
// 1353-1390): y = (x, y, vx, vy, A, t, psi) with z = A sin(psi) and
// vz = A cos(psi); the independent variable is the increment of psi, and
// y[6] carries the absolute angle (d y[6] = 1).  The force is evaluated at
// (x, y, A sin psi).
struct SosSystem {
  static constexpr int N = 7, NA = 3;
  static constexpr int kRow = ROW_SOS;
  static constexpr int kTimeIndex = 5;  // the force's time is the state's
  GPC_HD GPC_FI static void pos(const double* y, double* q)
  {
    q[0] = y[0];
    q[1] = y[1];
    q[2] = y[4] * sin(y[6]);
  }
  GPC_HD GPC_FI static void deriv(const double* y, const double* a, double* d)
  {
    const double sp = sin(y[6]), cp = cos(y[6]);
    const double ipd = 1.0 / (cp * cp - sp * a[2] / y[4]);  // d psi / dt = cos^2 - sin az / A
    d[0] = y[2] * ipd;
    d[1] = y[3] * ipd;
    d[2] = a[0] * ipd;
    d[3] = a[1] * ipd;
    d[4] = cp * (y[4] * sp + a[2]) * ipd;
    d[5] = ipd;
    d[6] = 1.0;
  }
};

// Planar surface of section (evalPlanarSOSDerivx / evalPlanarSOSDerivy,
// integratePlanarOrbit.c:1056-1123): y = (u, vu, A, t, psi).  SURF 0
// (surface x = 0): (u, vu) = (y, vy), x = A sin psi, vx = A cos psi;
// SURF 1 (y = 0): (u, vu) = (x, vx), y = A sin psi, vy = A cos psi.
template <int SURF>
struct PlanarSosSystem {
  static constexpr int N = 5, NA = 2;
  static constexpr int kRow = SURF == 0 ? ROW_SOS_PLANAR_X : ROW_SOS_PLANAR_Y;
  static constexpr int kTimeIndex = 3;
  GPC_HD GPC_FI static void pos(const double* y, double* q)
  {
    const double w = y[2] * sin(y[4]);
    q[0] = SURF == 0 ? w : y[0];
    q[1] = SURF == 0 ? y[0] : w;
  }
  GPC_HD GPC_FI static void deriv(const double* y, const double* a, double* d)
  {
    const double sp = sin(y[4]), cp = cos(y[4]);
    const double aw = SURF == 0 ? a[0] : a[1];  // along the surface normal
    const double au = SURF == 0 ? a[1] : a[0];
    const double ipd = 1.0 / (cp * cp - sp * aw / y[2]);
    d[0] = y[1] * ipd;
    d[1] = au * ipd;
    d[2] = cp * (y[2] * sp + aw) * ipd;
    d[3] = ipd;
    d[4] = 1.0;
  }
};

// ------------------------------------------------------------------------
// RK4 / RK6 (optionally variational)
// ------------------------------------------------------------------------
template <int D, bool VAR, int ORD, class SYS = OrbitSystem<D, VAR>>
struct RKMachine : OrbitCommon {
  static_assert(ORD == 4 || ORD == 6, "rk4 or rk6");
  static constexpr int N = SYS::N;  // ODE dimension
  static constexpr int NY = N;
  static constexpr int NV = N;
  static constexpr int NA = SYS::NA;  // force result size
  static constexpr int kRow = SYS::kRow;
  static constexpr int kStages = ORD == 4 ? 4 : 7;
  GPC_HD GPC_FI static void pos(const double* y, double* q) { SYS::pos(y, q); }
  static constexpr int kSlotDoubles = 0;
  GPC_HD GPC_FI void bind(double*) {}
  GPC_HD GPC_FI bool wants_dense() const { return false; }
  GPC_HD GPC_FI static int next_slot(int slot, bool) { return slot >= 14 ? 0 : slot + 1; }
  enum { EST_A = 0, EST_B = 1, EST_C = 2, MAIN = 3 };
  double yo[N];    // orbit state at the last completed step
  double yn[N], yn1[N], ynk[N];
  double y1[N];    // estimator: the one-step result
  double kk[ORD == 6 ? 5 : 1][N];  // rk6 stage increments k1..k5
  double dt, init_dt, h, s, rtol, atol;
  double tk;  // the reference's `to` of the main loop (bovy_rk.c: += dt per step)
  long long nrun, step;
  int stage, phase;

  // time of the current stage's force evaluation: the step's start tb
  // (rk4_estimate_step's to, to, to + dt/2 for its three trial steps) plus
  // the stage offset of bovy_rk4_onestep / bovy_rk6_onestep
  GPC_HD GPC_FI double tpoint(const double* y, int /*slot*/) const
  {
    if constexpr (SYS::kTimeIndex >= 0) {
      return y[SYS::kTimeIndex];
    } else {
      const double tb = phase == MAIN ? tk : (phase == EST_C ? t[0] + dt / 2. : t[0]);
      if (stage == 0) return tb;
      if (ORD == 4) return stage == 3 ? tb + h : tb + h / 2.;
      switch (stage) {
        case 1: case 3: return tb + h / 3.;
        case 2: return tb + 2. * h / 3.;
        case 4: case 5: return tb + h / 2.;
        default: return tb + h;
      }
    }
  }

  GPC_HD GPC_FI void start(const double* from, double hh)
  {
    h = hh;
    stage = 0;
#pragma unroll
    for (int k = 0; k < N; k++) yn[k] = yn1[k] = from[k];
  }

  GPC_HD GPC_FI void begin_main()
  {
    const long long ndt = (long long)(init_dt / dt);
    nrun = ndt < 1 ? 1 : ndt;
    step = 0;
    phase = MAIN;
    tk = t[0];
    start(yo, dt);
  }

  template <class W>
  GPC_HD void init(const double* w, const double* tt, int nt_, double dt_in, double rtol_,
                   double atol_, long long max_att, W& out)
  {
    t = tt;
    nt = nt_;
    iout = 0;
    err = E_OK;
    done = false;
    nsteps = 0;
    attempts = 0;
    max_attempts = max_att;
    rtol = rtol_;
    atol = atol_;
#pragma unroll
    for (int k = 0; k < N; k++) yo[k] = w[k];
    out(0, yo);
    if (nt < 2) {
      done = true;
      return;
    }
    init_dt = tt[1] - tt[0];
    if (dt_in == kDtSentinel) {
      dt = init_dt;
      s = est_scale(yo, N, 1, rtol, atol);
      phase = EST_A;
      start(yo, dt);
    } else {
      dt = dt_in;
      begin_main();
    }
  }

  GPC_HD GPC_FI void point(double* y, int /*slot*/) const
  {
    const bool first = stage == 0;
#pragma unroll
    for (int k = 0; k < N; k++) y[k] = first ? yn[k] : ynk[k];
  }

  template <class W>
  GPC_HD void consume(const double* y, const double* a, W& out, int /*slot*/)
  {
    double d[N];
    SYS::deriv(y, a, d);
    if (ORD == 4)
      rk4_stage<N>(stage, h, yn, yn1, ynk, d);
    else
      rk6_stage<N>(stage, h, yn, yn1, ynk, kk, d);
    if (++stage < kStages) return;
    onestep_done(out);
  }

  template <class W>
  GPC_HD void onestep_done(W& out)
  {
    // rk4_estimate_step / rk6_estimate_step (bovy_rk.c:328-480): one step of
    // dt against two of dt/2
    if (phase == EST_A) {
#pragma unroll
      for (int k = 0; k < N; k++) y1[k] = yn1[k];
      phase = EST_B;
      start(yo, dt / 2.);
      return;
    }
    if (phase == EST_B) {
      phase = EST_C;
      start(yn1, dt / 2.);
      return;
    }
    if (phase == EST_C) {
      double e = 0.;
#pragma unroll
      for (int k = 0; k < N; k++) e += exp(2. * log(fabs(y1[k] - yn1[k])) - 2. * s);
      e = sqrt(e / N);
      const double c = ceil(pow(e, ORD == 4 ? 1. / 5. : 1. / 7.));
      if (c > 1. && init_dt / dt * c < kMaxDtReduce) {
        dt /= c;
        phase = EST_A;
        start(yo, dt);
      } else {
        begin_main();
      }
      return;
    }
    bool fin = true;
#pragma unroll
    for (int k = 0; k < N; k++) {
      yo[k] = yn1[k];
      fin = fin && isfinite(yn1[k]);
    }
    tk += dt;
    nsteps++;
    attempts++;
    if (++step < nrun) {
      if (!fin) {
        err = E_NONFINITE;
        done = true;
        return;
      }
      start(yo, dt);
      return;
    }
    step = 0;
    iout++;
    out(iout, yo);
    if (!fin) {
      err = E_NONFINITE;
      done = true;
    } else if (iout == nt - 1) {
      done = true;
    } else if (max_attempts > 0 && attempts >= max_attempts) {
      err = E_BUDGET;
      done = true;
    } else {
      start(yo, dt);
    }
  }
};

template <int D, bool VAR>
using RK4Machine = RKMachine<D, VAR, 4>;

// ------------------------------------------------------------------------
// DOPR54 (optionally variational)
// ------------------------------------------------------------------------
// Dormand-Prince 5(4) tableau (bovy_rk.c:630-665)
namespace dp5 {
constexpr double a21 = 0.2, a31 = 3. / 40., a32 = 9. / 40.;
constexpr double a41 = 44. / 45., a42 = -56. / 15., a43 = 32. / 9.;
constexpr double a51 = 19372. / 6561., a52 = -25360. / 2187., a53 = 64448. / 6561.,
                 a54 = -212. / 729.;
constexpr double a61 = 9017. / 3168., a62 = -355. / 33., a63 = 46732. / 5247., a64 = 49. / 176.,
                 a65 = -5103. / 18656.;
constexpr double b1 = 35. / 384., b3 = 500. / 1113., b4 = 125. / 192., b5 = -2187. / 6784.,
                 b6 = 11. / 84.;
constexpr double e1 = b1 - 5179. / 57600., e3 = b3 - 7571. / 16695., e4 = b4 - 393. / 640.,
                 e5 = b5 + 92097. / 339200., e6 = b6 - 187. / 2100., e7 = -1. / 40.;
}  // namespace dp5

// bovy_dopr54 (bovy_rk.c:501-616) and bovy_dopr54_actualstep (:617-760):
// adaptive steps with a first-same-as-last derivative; the step factor is
// 0.85 err^(-1/5) rounded to a power of two in [1/8, 8] and an attempt is
// accepted when that power is >= 0.  Each output interval ends with a step
// clipped to its end (no interpolation).  A step that would shrink below
// the interval's first step / 10000 (or is NaN) is taken at that size and
// accepted, and the orbit's err becomes 1 as in the reference.  The first
// step comes from rk4_estimate_step.  Every attempt either advances the
// time or shrinks the step (at most 5 times in a row before a forced step),
// and an accepted step that no longer advances the time ends the orbit
// (err 2), so an orbit always finishes.
template <int D, bool VAR, class SYS = OrbitSystem<D, VAR>>
struct Dopr54Machine : OrbitCommon {
  static constexpr int N = SYS::N;
  static constexpr int NY = N;
  static constexpr int NV = N;
  static constexpr int NA = SYS::NA;
  static constexpr int kRow = SYS::kRow;
  GPC_HD GPC_FI static void pos(const double* y, double* q) { SYS::pos(y, q); }
  static constexpr int kSlotDoubles = 0;
  GPC_HD GPC_FI void bind(double*) {}
  GPC_HD GPC_FI bool wants_dense() const { return false; }
  GPC_HD GPC_FI static int next_slot(int slot, bool) { return slot >= 14 ? 0 : slot + 1; }
  enum { EST_A = 0, EST_B = 1, EST_C = 2, FSAL0 = 3, MAIN = 4 };
  double yo[N];    // state at time `to`
  double a1[N];    // derivative at yo
  // k1..k6 of an attempt; during the step estimation kk[0] is the RK4 step's
  // start and kk[1] the one-step result
  double kk[6][N];
  double yn1[N], yerr[N], ynk[N];
  double to, dtout, init_to, dt_one, init_dt_one, h, s, rtol, atol, est_dt, est_init;
  int stage, phase;
  bool forced;

  // time of the current force evaluation: the step estimation's rk4 trial
  // steps from to (to + est_dt/2 for the third), the first derivative at to,
  // then bovy_dopr54_actualstep's to + c_i dt (c = 1/5, 3/10, 4/5, 8/9, 1, 1)
  GPC_HD GPC_FI double tpoint(const double* y, int /*slot*/) const
  {
    if constexpr (SYS::kTimeIndex >= 0) {
      return y[SYS::kTimeIndex];
    } else {
      if (phase < FSAL0) {
        const double tb = phase == EST_C ? to + est_dt / 2. : to;
        if (stage == 0) return tb;
        return stage == 3 ? tb + h : tb + h / 2.;
      }
      if (phase == FSAL0) return to;
      switch (stage) {
        case 1: return to + 0.2 * h;
        case 2: return to + 0.3 * h;
        case 3: return to + 0.8 * h;
        case 4: return to + 8. / 9. * h;
        default: return to + h;
      }
    }
  }

  GPC_HD GPC_FI void est_start(const double* from, double hh)
  {
    h = hh;
    stage = 0;
#pragma unroll
    for (int k = 0; k < N; k++) kk[0][k] = yn1[k] = from[k];
  }

  template <class W>
  GPC_HD void init(const double* w, const double* tt, int nt_, double dt_in, double rtol_,
                   double atol_, long long max_att, W& out)
  {
    t = tt;
    nt = nt_;
    iout = 0;
    err = E_OK;
    done = false;
    nsteps = 0;
    attempts = 0;
    max_attempts = max_att;
    rtol = rtol_;
    atol = atol_;
#pragma unroll
    for (int k = 0; k < N; k++) yo[k] = w[k];
    out(0, yo);
    if (nt < 2) {
      done = true;
      return;
    }
    dtout = tt[1] - tt[0];
    to = tt[0];
    if (dt_in == kDtSentinel) {
      est_dt = est_init = dtout;
      s = est_scale(yo, N, 1, rtol, atol);
      phase = EST_A;
      est_start(yo, est_dt);
    } else {
      dt_one = dt_in;
      phase = FSAL0;
    }
  }

  GPC_HD GPC_FI void point(double* y, int /*slot*/) const
  {
    if (phase == FSAL0) {
#pragma unroll
      for (int k = 0; k < N; k++) y[k] = yo[k];
      return;
    }
    const bool first = phase < FSAL0 && stage == 0;
#pragma unroll
    for (int k = 0; k < N; k++) y[k] = first ? kk[0][k] : ynk[k];
  }

  template <class W>
  GPC_HD void consume(const double* y, const double* a, W& out, int /*slot*/)
  {
    double d[N];
    SYS::deriv(y, a, d);
    if (phase < FSAL0) {
      rk4_stage<N>(stage, h, kk[0], yn1, ynk, d);
      if (++stage == 4) est_step_done();
      return;
    }
    if (phase == FSAL0) {
#pragma unroll
      for (int k = 0; k < N; k++) a1[k] = d[k];
      phase = MAIN;
      init_dt_one = dt_one;
      init_to = to;
      next_attempt(out);
      return;
    }
    using namespace dp5;
    switch (stage) {
      case 1:
#pragma unroll
        for (int k = 0; k < N; k++) {
          kk[1][k] = h * d[k];
          ynk[k] = yo[k] + a31 * kk[0][k] + a32 * kk[1][k];
        }
        break;
      case 2:
#pragma unroll
        for (int k = 0; k < N; k++) {
          kk[2][k] = h * d[k];
          yn1[k] += b3 * kk[2][k];
          yerr[k] += e3 * kk[2][k];
          ynk[k] = yo[k] + a41 * kk[0][k] + a42 * kk[1][k] + a43 * kk[2][k];
        }
        break;
      case 3:
#pragma unroll
        for (int k = 0; k < N; k++) {
          kk[3][k] = h * d[k];
          yn1[k] += b4 * kk[3][k];
          yerr[k] += e4 * kk[3][k];
          ynk[k] = yo[k] + a51 * kk[0][k] + a52 * kk[1][k] + a53 * kk[2][k] + a54 * kk[3][k];
        }
        break;
      case 4:
#pragma unroll
        for (int k = 0; k < N; k++) {
          kk[4][k] = h * d[k];
          yn1[k] += b5 * kk[4][k];
          yerr[k] += e5 * kk[4][k];
          ynk[k] = yo[k] + a61 * kk[0][k] + a62 * kk[1][k] + a63 * kk[2][k] + a64 * kk[3][k] +
                   a65 * kk[4][k];
        }
        break;
      case 5:
#pragma unroll
        for (int k = 0; k < N; k++) {
          kk[5][k] = h * d[k];
          yn1[k] += b6 * kk[5][k];
          yerr[k] += e6 * kk[5][k];
          // the seventh point's a7j are the b weights (a72 = 0)
          ynk[k] = yo[k] + b1 * kk[0][k] + b3 * kk[2][k] + b4 * kk[3][k] + b5 * kk[4][k] +
                   b6 * kk[5][k];
        }
        break;
      default:
        attempt_done(d, out);
        return;
    }
    stage++;
  }

  // rk4_estimate_step (bovy_rk.c:328-395), run on kk[0] / kk[1]
  GPC_HD void est_step_done()
  {
    if (phase == EST_A) {
#pragma unroll
      for (int k = 0; k < N; k++) kk[1][k] = yn1[k];
      phase = EST_B;
      est_start(yo, est_dt / 2.);
      return;
    }
    if (phase == EST_B) {
      phase = EST_C;
      est_start(yn1, est_dt / 2.);
      return;
    }
    double e = 0.;
#pragma unroll
    for (int k = 0; k < N; k++) e += exp(2. * log(fabs(kk[1][k] - yn1[k])) - 2. * s);
    e = sqrt(e / N);
    const double c = ceil(pow(e, 1. / 5.));
    if (c > 1. && est_init / est_dt * c < kMaxDtReduce) {
      est_dt /= c;
      phase = EST_A;
      est_start(yo, est_dt);
      return;
    }
    dt_one = est_dt;
    phase = FSAL0;
  }

  // bovy_dopr54_onestep's loop (bovy_rk.c:584-616): output the intervals
  // that are complete, then set up the next attempt (its k1 from a1)
  template <class W>
  GPC_HD void next_attempt(W& out)
  {
    for (;;) {
      const bool more = (dtout >= 0. && to < (init_to + dtout)) ||
                        (dtout < 0. && to > (init_to + dtout));
      if (more) break;
      iout++;
      out(iout, yo);
      if (iout == nt - 1) {
        done = true;
        return;
      }
      init_dt_one = dt_one;
      init_to = to;
    }
    if (max_attempts > 0 && attempts >= max_attempts) {
      err = E_BUDGET;
      done = true;
      return;
    }
    forced = false;
    if (init_dt_one / dt_one > kMaxDtReduce || dt_one != dt_one) {
      dt_one = init_dt_one / kMaxDtReduce;
      forced = true;
      err = E_MINSTEP;
    }
    if (dtout >= 0. && dt_one > (init_to + dtout - to)) dt_one = (init_to + dtout - to);
    if (dtout < 0. && dt_one < (init_to + dtout - to)) dt_one = (init_to + dtout - to);
    h = dt_one;
    using namespace dp5;
#pragma unroll
    for (int k = 0; k < N; k++) {
      kk[0][k] = h * a1[k];
      yn1[k] = yo[k] + b1 * kk[0][k];
      yerr[k] = e1 * kk[0][k];
      ynk[k] = yo[k] + a21 * kk[0][k];
    }
    stage = 1;
  }

  // the seventh stage's derivative d: error norm, controller, accept
  template <class W>
  GPC_HD void attempt_done(const double* d, W& out)
  {
    // The reference's norm sqrt(sum_i exp(2 ln|e_i| - 2 s) / N) with the
    // scale s from max_i ln|yo_i| (bovy_rk.c:723-738), evaluated as
    // sqrt(sum_i e_i^2 exp(-2 s) / N) with max_i ln|yo_i| = ln max_i |yo_i|:
    // the same values up to rounding, with 2 logs and 3 exps instead of
    // 2N + 1 logs and N + 2 exps per attempt (which had kept the FP64 pipe
    // busy with the controller rather than the force).
    double ymax = fabs(yo[0]), e = 0.;
#pragma unroll
    for (int k = 0; k < N; k++) {
      yerr[k] += dp5::e7 * h * d[k];
      ymax = fmax(ymax, fabs(yo[k]));
      e += yerr[k] * yerr[k];
    }
    const double m = log(ymax), c = fmax(atol, rtol + m);
    const double sc = log(exp(atol - c) + exp(rtol + m - c)) + c;
    e = sqrt(e * exp(-2. * sc) / N);
    const double corr = 0.85 * pow(e, -.2);
    double p2 = round(log(corr) / log(2.));
    if (p2 > 3.)
      p2 = 3.;
    else if (p2 < -3.)
      p2 = -3.;
    attempts++;
    if (p2 >= 0. || forced) {
      bool fin = true;
#pragma unroll
      for (int k = 0; k < N; k++) {
        a1[k] = d[k];
        yo[k] = yn1[k];
        fin = fin && isfinite(yn1[k]);
      }
      const double to_before = to;
      to += h;
      nsteps++;
      if (!fin) {
        err = E_NONFINITE;
        done = true;
        return;
      }
      // a step below half an ulp of `to` leaves it unchanged: the reference
      // would loop forever here; the orbit stops as out of budget instead
      if (to == to_before) {
        err = E_BUDGET;
        done = true;
        return;
      }
    }
    dt_one = h * pow(2., p2);
    next_attempt(out);
  }
};

// ------------------------------------------------------------------------
// DOP853 (optionally variational)
// ------------------------------------------------------------------------
// Stage inputs as data: stage s's input is y0 + h * sum_t coef[s][t] *
// K[slot[s][t]] (terms in the reference's order, leung_dop853.c:351-388 and
// :446-462), and its derivative goes to slot dst[s].  Slots: 0 k1, 1 k2, 2 k3,
// 3 k4, 4 k5, 5 k6, 6 k7, 7 k8, 8 k9, 9 k10, 10 s14, 11 s15 -- the reference's
// k1..k10 with its reuse (stage 11 -> k2, stage 12 -> k3, the FSAL derivative
// -> k4, the new state -> k5), plus two slots for the first dense-output
// stages so that k10/k2/k3 stay available for the interpolation.  Because
// every lane of a warp is in the same stage (see kCycle below) the table
// reads are uniform constant-cache broadcasts and one small loop serves all
// stages.
struct DopStageTable {
  int nterm[17];
  int slot[17][9];
  double coef[17][9];
  int dst[17];
};
#define GPC_DOP853_STAGE_TABLE \
  {{0, 0, 1, 2, 2, 3, 3, 4, 5, 6, 7, 8, 9, 0, 8, 8, 8}, \
   {{0, 0, 0, 0, 0, 0, 0, 0, 0}, \
    {0, 0, 0, 0, 0, 0, 0, 0, 0}, \
    {0, 0, 0, 0, 0, 0, 0, 0, 0}, \
    {0, 1, 0, 0, 0, 0, 0, 0, 0}, \
    {0, 2, 0, 0, 0, 0, 0, 0, 0}, \
    {0, 2, 3, 0, 0, 0, 0, 0, 0}, \
    {0, 3, 4, 0, 0, 0, 0, 0, 0}, \
    {0, 3, 4, 5, 0, 0, 0, 0, 0}, \
    {0, 3, 4, 5, 6, 0, 0, 0, 0}, \
    {0, 3, 4, 5, 6, 7, 0, 0, 0}, \
    {0, 3, 4, 5, 6, 7, 8, 0, 0}, \
    {0, 3, 4, 5, 6, 7, 8, 9, 0}, \
    {0, 3, 4, 5, 6, 7, 8, 9, 1}, \
    {0, 0, 0, 0, 0, 0, 0, 0, 0}, \
    {0, 6, 7, 8, 9, 1, 2, 3, 0}, \
    {0, 5, 6, 7, 1, 2, 3, 10, 0}, \
    {0, 5, 6, 7, 8, 3, 10, 11, 0}}, \
   {{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, \
    {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, \
    {dp::a21, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, \
    {dp::a31, dp::a32, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, \
    {dp::a41, dp::a43, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, \
    {dp::a51, dp::a53, dp::a54, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, \
    {dp::a61, dp::a64, dp::a65, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, \
    {dp::a71, dp::a74, dp::a75, dp::a76, 0.0, 0.0, 0.0, 0.0, 0.0}, \
    {dp::a81, dp::a84, dp::a85, dp::a86, dp::a87, 0.0, 0.0, 0.0, 0.0}, \
    {dp::a91, dp::a94, dp::a95, dp::a96, dp::a97, dp::a98, 0.0, 0.0, 0.0}, \
    {dp::a101, dp::a104, dp::a105, dp::a106, dp::a107, dp::a108, dp::a109, 0.0, 0.0}, \
    {dp::a111, dp::a114, dp::a115, dp::a116, dp::a117, dp::a118, dp::a119, dp::a1110, 0.0}, \
    {dp::a121, dp::a124, dp::a125, dp::a126, dp::a127, dp::a128, dp::a129, dp::a1210, dp::a1211}, \
    {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, \
    {dp::a141, dp::a147, dp::a148, dp::a149, dp::a1410, dp::a1411, dp::a1412, dp::a1413, 0.0}, \
    {dp::a151, dp::a156, dp::a157, dp::a158, dp::a1511, dp::a1512, dp::a1513, dp::a1514, 0.0}, \
    {dp::a161, dp::a166, dp::a167, dp::a168, dp::a169, dp::a1613, dp::a1614, dp::a1615, 0.0}}, \
   {-1, -1, 1, 2, 3, 4, 5, 6, 7, 8, 9, 1, 2, 3, 10, 11, -1}}

#if defined(__CUDACC__)
__constant__ DopStageTable kDopTableDev = GPC_DOP853_STAGE_TABLE;
#endif
static const DopStageTable kDopTableHost = GPC_DOP853_STAGE_TABLE;

GPC_HD GPC_FI const DopStageTable& dop_table()
{
#if defined(__CUDA_ARCH__)
  return kDopTableDev;
#else
  return kDopTableHost;
#endif
}

template <int D, bool VAR, class SYS = OrbitSystem<D, VAR>>
struct Dop853Machine : OrbitCommon {
  static constexpr int N = SYS::N;
  static constexpr int NY = N;
  static constexpr int NV = N;
  static constexpr int NA = SYS::NA;  // force result size
  static constexpr int kRow = SYS::kRow;
  GPC_HD GPC_FI static void pos(const double* y, double* q) { SYS::pos(y, q); }
  enum {
    ST_INIT1 = 0, ST_INIT2 = 1,
    // ST_S2..ST_S12 = 2..12
    ST_FSAL = 13, ST_S14 = 14, ST_S15 = 15, ST_S16 = 16
  };
  enum { K1 = 0, K2 = 1, K3 = 2, K4 = 3, K5 = 4, K6 = 5, K7 = 6, K8 = 7, K9 = 8, K10 = 9,
         S14 = 10, S15 = 11 };
  // Stage slots K2..K10, S14, S15 live in a per-thread slot store (shared
  // memory in the kernel, strided by the block size: bank-conflict free); y0
  // and K1 -- the first term of every stage input -- stay in registers.
  static constexpr int kSlots = 11;
  static constexpr int kSlotDoubles = kSlots * N;
  double y0[N], k1[N];
  double* ks;  // slot store: slot s >= 1 at ks[((s - 1) * N + i) * kSlotStride]
  GPC_HD GPC_FI void bind(double* base, bool queue = false)
  {
    ks = base;
    queued = queue;
    want_enqueue = false;
  }
  GPC_HD GPC_FI double& K(int s, int i) const { return ks[((s - 1) * N + i) * kSlotStride]; }
  double h, hnew, hmax, pos_neg, rtol, atol;
  double t_current, t_old;
  int stage;
  bool reject;

  // Lanes of a warp run the stages of their (different) orbits in lock step:
  // an attempt occupies slots 0..10 (stages 2..12), slot 11 (the FSAL
  // evaluation) and, only when some lane of the warp has an output time in
  // its step, slots 12..14 (the dense-output stages); the kernel advances
  // the slot for the whole warp (next_slot).  A lane with nothing to compute
  // in a slot (a rejected attempt, a step without output time, a new orbit
  // waiting for slot 0) evaluates the force at y0 and discards it.  The two
  // start-up evaluations of a new orbit run in whatever slots follow its
  // pick-up.
  GPC_HD GPC_FI static int slot_stage(int slot) { return slot + 2; }
  GPC_HD GPC_FI bool active_in(int slot) const { return stage < 2 || stage == slot_stage(slot); }
  GPC_HD GPC_FI bool wants_dense() const { return !done && stage == ST_S14; }
  GPC_HD GPC_FI static int next_slot(int slot, bool any_dense)
  {
    if (slot == 11) return any_dense ? 12 : 0;
    return slot >= 14 ? 0 : slot + 1;
  }

  GPC_HD GPC_FI void begin_attempt()
  {
    h = pos_neg * dmax(fabs(h), 1e3 * 2.3e-16);
    stage = 2;
  }

  template <class W>
  GPC_HD void init(const double* w, const double* tt, int nt_, double /*dt*/, double rtol_,
                   double atol_, long long max_att, W& out)
  {
    t = tt;
    nt = nt_;
    iout = 0;
    err = E_OK;
    done = false;
    nsteps = 0;
    attempts = 0;
    max_attempts = max_att;
    rtol = exp(rtol_);
    atol = exp(atol_);
#pragma unroll
    for (int k = 0; k < N; k++) y0[k] = w[k];
    out(0, y0);
    if (nt < 2) {
      done = true;
      return;
    }
    hmax = tt[nt - 1] - tt[0];
    pos_neg = csign(1.0, hmax);
    reject = false;
    t_current = t_old = tt[0];
    stage = ST_INIT1;
  }

  GPC_HD GPC_FI void point(double* y, int slot) const
  {
    if (!active_in(slot) || stage == ST_INIT1) {
#pragma unroll
      for (int i = 0; i < N; i++) y[i] = y0[i];
      return;
    }
    if (stage == ST_INIT2) {  // explicit Euler step (leung_dop853.c:310)
#pragma unroll
      for (int i = 0; i < N; i++) y[i] = y0[i] + h * k1[i];
      return;
    }
    if (stage == ST_FSAL) {  // the new state
#pragma unroll
      for (int i = 0; i < N; i++) y[i] = K(K5, i);
      return;
    }
    const DopStageTable& tb = dop_table();
    const int n = tb.nterm[stage];
    double acc[N];
    {  // the first term of every stage input is K1 (table slot 0)
      const double c0 = tb.coef[stage][0];
#pragma unroll
      for (int i = 0; i < N; i++) acc[i] = c0 * k1[i];
    }
    // unrolled by 4 (with a remainder): the table reads of later terms are
    // issued ahead of the shared-memory loads and FMAs of earlier ones
#pragma unroll 4
    for (int tt = 1; tt < n; tt++) {
      const int s = tb.slot[stage][tt];
      const double c = tb.coef[stage][tt];
#pragma unroll
      for (int i = 0; i < N; i++) acc[i] += c * K(s, i);
    }
#pragma unroll
    for (int i = 0; i < N; i++) y[i] = y0[i] + h * acc[i];
  }

  GPC_HD GPC_FI bool output_pending() const
  {
    return iout < nt - 1 && pos_neg * t[iout + 1] < pos_neg * t_current;
  }

  // c_s of the stage whose input is evaluated (leung_dop853.c:351-462)
  GPC_HD GPC_FI static double stage_c(int stage)
  {
    using namespace dp;
    switch (stage) {
      case 2: return c2;
      case 3: return c3;
      case 4: return c4;
      case 5: return c5;
      case 6: return c6;
      case 7: return c7;
      case 8: return c8;
      case 9: return c9;
      case 10: return c10;
      case 11: return c11;
      case ST_S14: return c14;
      case ST_S15: return c15;
      default: return c16;
    }
  }

  // time of the current force evaluation as the reference passes it:
  // t0 and t0 + h for the start-up, t_current + c_s h for stages 2..11,
  // t_current + h for stage 12, the new t_current for the FSAL derivative,
  // t_old + c_s h for the dense-output stages (a lane idle in the slot:
  // any time, its result is discarded)
  GPC_HD GPC_FI double tpoint(const double* y, int slot) const
  {
    if constexpr (SYS::kTimeIndex >= 0) {
      return y[SYS::kTimeIndex];
    } else {
      if (!active_in(slot) || stage == ST_INIT1 || stage == ST_FSAL) return t_current;
      if (stage == ST_INIT2 || stage == 12) return t_current + h;
      if (stage >= ST_S14) return t_old + stage_c(stage) * h;
      return t_current + stage_c(stage) * h;
    }
  }

  template <class W>
  GPC_HD void consume(const double* y, const double* a, W& out, int slot)
  {
    using namespace dp;
    if (!active_in(slot)) return;
    double d[N];
    SYS::deriv(y, a, d);
    if (stage == ST_INIT1) {  // leung_dop853.c:296-308
      double dny = 0.0, dnf = 0.0;
#pragma unroll
      for (int i = 0; i < N; i++) {
        k1[i] = d[i];
        const double sk = atol + rtol * fabs(y0[i]);
        double sqr = d[i] / sk;
        dnf += sqr * sqr;
        sqr = y0[i] / sk;
        dny += sqr * sqr;
      }
      h = csign(dmin(sqrt(dny / dnf) * 0.01, fabs(hmax)), pos_neg);
      hnew = dnf;  // kept for the second start-up evaluation (hnew is free until the first step)
      stage = ST_INIT2;
      return;
    }
    if (stage == ST_INIT2) {  // leung_dop853.c:309-324
      double der2 = 0.0;
#pragma unroll
      for (int i = 0; i < N; i++) {
        const double sk = atol + rtol * fabs(y0[i]);
        const double sqr = (d[i] - k1[i]) / sk;
        der2 += sqr * sqr;
      }
      der2 = sqrt(der2) / h;
      const double der12 = dmax(fabs(der2), sqrt(hnew));  // hnew: dnf of the first evaluation
      const double h1 = pow(0.01 / der12, 1.0 / 8.0);
      h = csign(dmin(100.0 * fabs(h), dmin(fabs(h1), fabs(hmax))), pos_neg);
      begin_attempt();
      return;
    }
    const int dst = dop_table().dst[stage];
    if (dst >= 0) {
#pragma unroll
      for (int i = 0; i < N; i++) K(dst, i) = d[i];
    }
    if (stage < 12) {
      stage++;
      return;
    }
    if (stage == 12) {
      after_stage12();
      return;
    }
    if (stage == ST_FSAL) {
      nsteps++;
      if (output_pending()) {
        if (queued) {
          // the rows of this step go to the warp's queue: the kernel writes
          // the request, then calls finish_step
          jf = iout + 1;
          while (output_pending()) iout++;
          jl = iout;
          want_enqueue = true;
          return;
        }
        stage = ST_S14;
        return;
      }
      finish_step(out);
      return;
    }
    if (stage < ST_S16) {
      stage++;
      return;
    }
    // ST_S16: dense output (leung_dop853.c:441-474), d = stage-16 derivative
    while (output_pending()) {
      const double sv = (t[iout + 1] - t_old) / h;
      double v[N];
#pragma unroll
      for (int i = 0; i < N; i++)
        v[i] = dense_value(sv, h, y0[i], K(K5, i), k1[i], K(K2, i), K(K3, i), K(K4, i),
                           K(K6, i), K(K7, i), K(K8, i), K(K9, i), K(K10, i), K(S14, i),
                           K(S15, i), d[i]);
      iout++;
      out(iout, v);
    }
    finish_step(out);
  }

  // One component of the dense output at s = sv of a step of size h from
  // y0 to y1 (leung_dop853.c:441-474): k1 the step's first derivative,
  // k2 / k3 the stage-11 / stage-12 derivatives (kept in the K2 / K3 slots,
  // as the reference reuses k2 and k3), k4 = f(y1), k6..k10 the stage
  // derivatives, s14..s16 the three dense-output stages.  Shared by the
  // in-slot and the queued dense output, so both give the same rows.
  GPC_HD GPC_FI static double dense_value(double sv, double h, double y0, double y1, double k1,
                                          double k2, double k3, double k4, double k6,
                                          double k7, double k8, double k9, double k10,
                                          double s14, double s15, double s16)
  {
    using namespace dp;
    const double s1 = 1.0 - sv;
    const double rc1 = y0;
    const double ydiff = y1 - y0;
    const double bspl = h * k1 - ydiff;
    const double rc4 = ydiff - h * k4 - bspl;
    double rc5 = d41 * k1 + d46 * k6 + d47 * k7 + d48 * k8 + d49 * k9 + d410 * k10 +
                 d411 * k2 + d412 * k3;
    double rc6 = d51 * k1 + d56 * k6 + d57 * k7 + d58 * k8 + d59 * k9 + d510 * k10 +
                 d511 * k2 + d512 * k3;
    double rc7 = d61 * k1 + d66 * k6 + d67 * k7 + d68 * k8 + d69 * k9 + d610 * k10 +
                 d611 * k2 + d612 * k3;
    double rc8 = d71 * k1 + d76 * k6 + d77 * k7 + d78 * k8 + d79 * k9 + d710 * k10 +
                 d711 * k2 + d712 * k3;
    rc5 = h * (rc5 + d413 * k4 + d414 * s14 + d415 * s15 + d416 * s16);
    rc6 = h * (rc6 + d513 * k4 + d514 * s14 + d515 * s15 + d516 * s16);
    rc7 = h * (rc7 + d613 * k4 + d614 * s14 + d615 * s15 + d616 * s16);
    rc8 = h * (rc8 + d713 * k4 + d714 * s14 + d715 * s15 + d716 * s16);
    return rc1 +
           sv * (ydiff + s1 * (bspl + sv * (rc4 + s1 * (rc5 + sv * (rc6 + s1 * (rc7 + sv * rc8))))));
  }

  // ---- queued dense output ---------------------------------------------
  // With a request queue (the kernel's per-warp ring in global memory), a
  // step that contains output times does not run the three dense-output
  // stages in the warp's slot cycle, where the other lanes of the warp would
  // sit idle for them: the lane writes the step's data to the queue and goes
  // on with its next step, and the warp later runs the dense stages of 32
  // queued requests side by side (one per lane).  The rows are the same as
  // the in-slot dense output's (same arithmetic, dense_value).
  //
  // Request record, field-major with kQueueSlots slots per field (component
  // i of vector field f of slot p at q[(f * N + i) * kQueueSlots + p]):
  //   vector fields 0 y0, 1 k1, 2..10 the slot store K2..K10 (K5 = y1,
  //   K4 = f(y1)); then scalars h, t_old, the orbit index and the row range
  //   (first << 32 | last) at q[(11 N + k) * kQueueSlots + p], k = 0..3.
  static constexpr int kQueueSlots = 64;
  static constexpr int kQueueFields = 11 * N + 4;  // doubles per slot
  static constexpr bool kQueue = SYS::kRow == ROW_ORBIT && !VAR;
  bool queued;        // dense output through the warp's queue
  bool want_enqueue;  // this step's dense output waits for the queue
  int jf, jl;         // rows of the pending request

  GPC_HD GPC_FI void write_request(double* q, int p, long long orbit) const
  {
    constexpr int QS = kQueueSlots;
#pragma unroll
    for (int i = 0; i < N; i++) {
      q[(0 * N + i) * QS + p] = y0[i];
      q[(1 * N + i) * QS + p] = k1[i];
    }
#pragma unroll
    for (int s = 1; s <= 9; s++)
#pragma unroll
      for (int i = 0; i < N; i++) q[((1 + s) * N + i) * QS + p] = K(s, i);
    q[(11 * N + 0) * QS + p] = h;
    q[(11 * N + 1) * QS + p] = t_old;
    long long* qi = reinterpret_cast<long long*>(q);
    qi[(11 * N + 2) * QS + p] = orbit;
    qi[(11 * N + 3) * QS + p] = ((long long)jf << 32) | (long long)(unsigned)jl;
  }

  // Slot s of request p: s = 0 its k1, 1..9 its K2..K10, 10 / 11 the dense
  // stages S14 / S15, which the round keeps in this lane's own slot store
  // (unused by the lane's orbit when dense output is queued).
  GPC_HD GPC_FI double req_k(const double* q, int p, int s, int i) const
  {
    return s <= 9 ? q[((1 + s) * N + i) * kQueueSlots + p] : K(s, i);
  }

  // Input of dense stage `stage` (14, 15, 16) of request p: the table loop
  // of point() over the request's slots.
  GPC_HD GPC_FI void req_point(double* y, int stage, const double* q, int p) const
  {
    const DopStageTable& tb = dop_table();
    const int n = tb.nterm[stage];
    double acc[N];
    {
      const double c0 = tb.coef[stage][0];
#pragma unroll
      for (int i = 0; i < N; i++) acc[i] = c0 * q[(1 * N + i) * kQueueSlots + p];
    }
#pragma unroll 4
    for (int tt = 1; tt < n; tt++) {
      const int s = tb.slot[stage][tt];
      const double c = tb.coef[stage][tt];
#pragma unroll
      for (int i = 0; i < N; i++) acc[i] += c * req_k(q, p, s, i);
    }
    const double hq = q[(11 * N) * kQueueSlots + p];
#pragma unroll
    for (int i = 0; i < N; i++) y[i] = q[(0 * N + i) * kQueueSlots + p] + hq * acc[i];
  }

  // Time of dense stage `stage` of request p (t_old + c_s h of its step).
  GPC_HD GPC_FI double req_tpoint(const double* y, int stage, const double* q, int p) const
  {
    if constexpr (SYS::kTimeIndex >= 0) {
      return y[SYS::kTimeIndex];
    } else {
      return q[(11 * N + 1) * kQueueSlots + p] + stage_c(stage) * q[(11 * N) * kQueueSlots + p];
    }
  }

  // Derivative of dense stage `stage` at request p: stages 14 and 15 are
  // kept for the next stage inputs; stage 16 completes the rows.
  template <class W>
  GPC_HD void req_consume(const double* y, const double* a, int stage, const double* q, int p,
                          const double* tt, W& out)
  {
    double d[N];
    SYS::deriv(y, a, d);
    if (stage < ST_S16) {
      const int s = stage == ST_S14 ? S14 : S15;
#pragma unroll
      for (int i = 0; i < N; i++) K(s, i) = d[i];
      return;
    }
    constexpr int QS = kQueueSlots;
    const double hq = q[(11 * N) * QS + p], told = q[(11 * N + 1) * QS + p];
    const long long rr = reinterpret_cast<const long long*>(q)[(11 * N + 3) * QS + p];
    const int j0 = (int)(rr >> 32), j1 = (int)(unsigned)(rr & 0xffffffffLL);
    for (int j = j0; j <= j1; j++) {
      const double sv = (tt[j] - told) / hq;
      double v[N];
#pragma unroll
      for (int k = 0; k < N; k++) v[k] = 0.0;
      // one component at a time: unrolled, the compiler would issue all
      // 14 N loads of the record at once and hold them in registers.  The
      // component index of this loop is a run-time value, so d and v are
      // read and written through selects over compile-time indices: indexed
      // by it they would live in local memory.
#pragma unroll 1
      for (int i = 0; i < N; i++) {
        double di = d[0];
#pragma unroll
        for (int k = 1; k < N; k++) di = i == k ? d[k] : di;
        const double vi =
            dense_value(sv, hq, q[(0 * N + i) * QS + p], q[((1 + K5) * N + i) * QS + p],
                        q[(1 * N + i) * QS + p], q[((1 + K2) * N + i) * QS + p],
                        q[((1 + K3) * N + i) * QS + p], q[((1 + K4) * N + i) * QS + p],
                        q[((1 + K6) * N + i) * QS + p], q[((1 + K7) * N + i) * QS + p],
                        q[((1 + K8) * N + i) * QS + p], q[((1 + K9) * N + i) * QS + p],
                        q[((1 + K10) * N + i) * QS + p], K(S14, i), K(S15, i), di);
#pragma unroll
        for (int k = 0; k < N; k++) v[k] = i == k ? vi : v[k];
      }
      out(j, v);
    }
  }

  GPC_HD void after_stage12()
  {
    using namespace dp;
    attempts++;
    double e = 0.0, e2 = 0.0;
#pragma unroll
    for (int i = 0; i < N; i++) {
      const double k1 = this->k1[i], k2 = K(K2, i), k3 = K(K3, i), k6 = K(K6, i), k7 = K(K7, i);
      const double k8 = K(K8, i), k9 = K(K9, i), k10 = K(K10, i);
      const double k4 =
          b1 * k1 + b6 * k6 + b7 * k7 + b8 * k8 + b9 * k9 + b10 * k10 + b11 * k2 + b12 * k3;
      const double k5 = y0[i] + h * k4;
      K(K4, i) = k4;
      K(K5, i) = k5;
      const double sk = atol + rtol * dmax(fabs(y0[i]), fabs(k5));
      double erri = k4 - bhh1 * k1 - bhh2 * k9 - bhh3 * k3;
      double sqr = erri / sk;
      e2 += sqr * sqr;
      erri = er1 * k1 + er6 * k6 + er7 * k7 + er8 * k8 + er9 * k9 + er10 * k10 + er11 * k2 +
             er12 * k3;
      sqr = erri / sk;
      e += sqr * sqr;
    }
    double deno = e + 0.01 * e2;
    if (deno <= 0.0) deno = 1.0;
    e = fabs(h) * e * sqrt(1.0 / (deno * (double)N));
    if (!isfinite(e)) {
      err = E_NONFINITE;
      done = true;
      return;
    }
    const double fac11 = pow(e, 1.0 / 8.0);
    // Lund stabilisation with beta = 0 divides by pow(facold, 0) == 1, so the
    // reference's facold (max(e, 1e-4) of the last accepted step) drops out
    double fac = fac11;
    fac = dmax(1.0 / 6.0, dmin(1.0 / 0.333, fac / 0.9));
    hnew = h / fac;
    if (e <= 1.0) {
      // accepted: the step runs from t_old to t_current (the reference
      // advances both before the test and restores them on rejection)
      t_old = t_current;
      t_current = t_current + h;
      stage = ST_FSAL;
    } else {
      // an attempt rejected at the smallest step (begin_attempt's floor)
      // repeats exactly -- same state, same step, same error -- so the
      // reference rejects it forever; the orbit stops as out of budget
      if (fabs(h) <= 1e3 * 2.3e-16) {
        err = E_BUDGET;
        done = true;
        return;
      }
      hnew = h / dmin(1.0 / 0.333, fac11 / 0.9);
      reject = true;
      h = hnew;
      if (max_attempts > 0 && attempts >= max_attempts) {
        err = E_BUDGET;
        done = true;
        return;
      }
      begin_attempt();
    }
  }

  template <class W>
  GPC_HD void finish_step(W& /*out*/)
  {
#pragma unroll
    for (int i = 0; i < N; i++) {
      k1[i] = K(K4, i);
      y0[i] = K(K5, i);
    }
    hnew = (fabs(hnew) > fabs(hmax)) ? pos_neg * hmax : hnew;
    if (reject) hnew = pos_neg * dmin(fabs(hnew), fabs(h));
    reject = false;
    h = hnew;
    if (iout == nt - 1) {
      done = true;
      return;
    }
    if (max_attempts > 0 && attempts >= max_attempts) {
      err = E_BUDGET;
      done = true;
      return;
    }
    begin_attempt();
  }
};

// Rows the integrator did not reach (stopped by the budget, a non-finite
// state or an abort) are written as NaN.
template <class M, class W>
GPC_HD void fill_unreached_rows(const M& m, W& out)
{
  if (m.err == E_OK) return;
  double v[M::NV];
#pragma unroll
  for (int k = 0; k < M::NV; k++) v[k] = NAN;
  for (int j = m.iout + 1; j < m.nt; j++) out(j, v);
}

// One orbit through the queued dense output with a queue of one request
// that is served as soon as it is written (the host test harness's check of
// the request record and the dense rounds' arithmetic; the kernel serves 32
// requests of a warp at a time).  m must be bound with queue = true; q holds
// Dop853Machine::kQueueFields * kQueueSlots doubles; tt are the orbit's
// output times.
template <class M, class F, class W>
GPC_HD void run_orbit_queued(M& m, F& force, W& out, double* q, const double* tt,
                             long long orbit)
{
  double y[M::NY], qq[M::NA], a[M::NA];
  int slot = 0;
  while (!m.done) {
    m.point(y, slot);
    M::pos(y, qq);
    force(qq, a, m.tpoint(y, slot));
    m.consume(y, a, out, slot);
    if (slot == 11 && m.want_enqueue) {
      m.write_request(q, 0, orbit);
      m.want_enqueue = false;
      m.finish_step(out);
      for (int stage = 14; stage <= 16; stage++) {
        m.req_point(y, stage, q, 0);
        M::pos(y, qq);
        force(qq, a, m.req_tpoint(y, stage, q, 0));
        m.req_consume(y, a, stage, q, 0, tt, out);
      }
    }
    slot = slot == 11 ? 0 : slot + 1;
  }
  fill_unreached_rows(m, out);
}

// Per-orbit driver used by the host test harness: run one machine to
// completion with the force evaluated by `force` (positions, result, time).
template <class M, class F, class W>
GPC_HD void run_orbit(M& m, F& force, W& out)
{
  double y[M::NY], q[M::NA], a[M::NA];
  int slot = 0;
  while (!m.done) {
    m.point(y, slot);
    M::pos(y, q);
    force(q, a, m.tpoint(y, slot));
    m.consume(y, a, out, slot);
    slot = M::next_slot(slot, m.wants_dense());
  }
  fill_unreached_rows(m, out);
}

}  // namespace gpc
