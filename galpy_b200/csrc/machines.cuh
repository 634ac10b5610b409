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
//   leapfrog / symplec4         galpy/util/bovy_symplecticode.c:132-377
//   their step estimators       galpy/util/bovy_symplecticode.c:588-809
//   variational (*_dxdv) forms  galpy/util/bovy_symplecticode.c:1053-1268
//   rk4 + estimator             galpy/util/bovy_rk.c:66-170, 328-395
//   dop853                      galpy/util/leung_dop853.c:231-517
// Differences by design: the time variable of the reference's symplectic and
// RK loops is not tracked (the supported potentials are static); DOP853
// skips its three dense-output stages in steps that contain no output time
// (their results are only used for output); every orbit has an attempt budget
// and stops on a non-finite state instead of looping forever.
#pragma once
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

enum : int { M_LEAPFROG = 0, M_RK4 = 1, M_SYMPLEC4 = 3, M_DOP853 = 6 };
enum : int { PREC_FP64 = 0, PREC_F32 = 1 };

// symplec4 coefficients (Kinoshita et al.; bovy_symplecticode.c:96-99)
constexpr double s4c1 = 0.6756035959798289, s4c2 = -0.1756035959798288;
constexpr double s4c3 = -0.1756035959798288, s4c4 = 0.6756035959798289;
constexpr double s4d1 = 1.3512071919596578, s4d2 = -1.7024143839193153;
constexpr double s4d3 = 1.3512071919596578;

// ------------------------------------------------------------------------
// output rows
// ------------------------------------------------------------------------
enum : int { L_GALPY_CYL = 0, L_AOS_RECT = 1, L_SOA_RECT = 2, L_SOA_CYL = 3 };

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
template <int NV, int D, bool CYL_OK>
GPC_HD GPC_FI void write_row(const OutSpec& o, long long i, int j, const double* v)
{
  if (j < o.row0) return;
  const long long nrow = o.nt - o.row0, jj = j - o.row0;
  double w[NV];
  const bool cyl = CYL_OK && (o.layout == L_GALPY_CYL || o.layout == L_SOA_CYL);
  if (cyl) {
    // rect_to_cyl_galpy / rect_to_polar_galpy (bovy_coords.c:79-148)
    const double x = v[0], y = v[1];
    const double vx = v[D], vy = v[D + 1];
    const double phi = atan2(y, x), cp = cos(phi), sp = sin(phi);
    w[0] = sqrt(x * x + y * y);
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

template <int NV, int D, bool CYL_OK>
GPC_HD GPC_FI void write_nan_rows(const OutSpec& o, long long i, int from)
{
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = NAN;
  for (int j = from; j < o.nt; j++) write_row<NV, D, CYL_OK>(o, i, j, v);
}

// ------------------------------------------------------------------------
// force adapter: positions -> accelerations (+ K . dq for variational runs)
// ------------------------------------------------------------------------
template <int D, int PREC, bool VAR, class POT = DynPot>
GPC_HD GPC_FI void eval_force(const GpComp* comp, int ncomp, const double* q, double* a,
                              const double* scal = nullptr)
{
  if (!VAR) {
    if (PREC == PREC_FP64) {
      double ax, ay, az = 0.0;
      accel<double, D == 2, POT>(comp, ncomp, q[0], q[1], D == 3 ? q[2] : 0.0, ax, ay, az, scal);
      a[0] = ax;
      a[1] = ay;
      if (D == 3) a[2] = az;
    } else {
      float ax, ay, az = 0.f;
      accel<float, D == 2, POT>(comp, ncomp, (float)q[0], (float)q[1], D == 3 ? (float)q[2] : 0.f,
                                ax, ay, az, scal);
      a[0] = ax;
      a[1] = ay;
      if (D == 3) a[2] = az;
    }
  } else {
    double ax, ay, az, K[6];
    accel_tidal<D == 2>(comp, ncomp, q[0], q[1], D == 3 ? q[2] : 0.0, ax, ay, az, K);
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
// leapfrog / symplec4 (optionally variational)
// ------------------------------------------------------------------------
template <int D, bool VAR, bool S4>
struct SymplecticMachine : OrbitCommon {
  static constexpr int NQ = VAR ? 2 * D : D;  // stepped positions
  static constexpr int NY = NQ;               // size of the force argument
  static constexpr int NV = 2 * NQ;           // values per output row
  static constexpr int NA = NQ;               // force result size
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
  double qw[NQ], pw[NQ];  // state of the running advance
  double q11[D], p11[D];  // estimator: the single-step result (base orbit)
  double dt, init_dt, h, sq, sp, rtol, atol;
  long long nrun, kick, nkick;
  int sub, phase;

  GPC_HD GPC_FI void start(double hh, long long nstep)
  {
    h = hh;
    nrun = nstep;
    kick = 0;
    sub = 0;
    nkick = (S4 ? 3 : 1) * nstep;
    const double c = S4 ? s4c1 * h : h / 2.;
#pragma unroll
    for (int k = 0; k < NQ; k++) {
      qw[k] = qo[k] + c * po[k];
      pw[k] = po[k];
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
    start(dt, ndt < 1 ? 1 : ndt);
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
#pragma unroll
    for (int k = 0; k < NQ; k++) y[k] = qw[k];
  }

  template <class W>
  GPC_HD void consume(const double* /*y*/, const double* a, W& out, int /*slot*/)
  {
    const double dk = S4 ? (sub == 0 ? s4d1 * h : (sub == 1 ? s4d2 * h : s4d3 * h)) : h;
#pragma unroll
    for (int k = 0; k < NQ; k++) pw[k] = pw[k] + dk * a[k];
    const bool last = (kick == nkick - 1);
    double dc;
    if (S4)
      dc = sub == 0 ? s4c2 * h : (sub == 1 ? s4c3 * h : (last ? s4c4 * h : (s4c4 + s4c1) * h));
    else
      dc = last ? h / 2. : h;
#pragma unroll
    for (int k = 0; k < NQ; k++) qw[k] = qw[k] + dc * pw[k];
    kick++;
    sub = (S4 && sub < 2) ? sub + 1 : 0;
    if (last) advance_done(out);
  }

  template <class W>
  GPC_HD void advance_done(W& out)
  {
    if (phase == EST_FULL) {
#pragma unroll
      for (int k = 0; k < D; k++) {
        q11[k] = qw[k];
        p11[k] = pw[k];
      }
      phase = EST_HALF;
      start(dt / 2., 2);
      return;
    }
    if (phase == EST_HALF) {
      double e = 0.;
#pragma unroll
      for (int k = 0; k < D; k++) {
        e += exp(2. * log(fabs(q11[k] - qw[k])) - 2. * sq);
        e += exp(2. * log(fabs(p11[k] - pw[k])) - 2. * sp);
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
      qo[k] = qw[k];
      po[k] = pw[k];
      fin = fin && isfinite(qw[k]) && isfinite(pw[k]);
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
// RK4 (optionally variational)
// ------------------------------------------------------------------------
template <int D, bool VAR>
struct RK4Machine : OrbitCommon {
  static constexpr int N = VAR ? 4 * D : 2 * D;  // ODE dimension
  static constexpr int NY = N;
  static constexpr int NV = N;
  static constexpr int NA = VAR ? 2 * D : D;  // force result size
  // force argument: positions (and deviation positions) of (x, v[, dx, dv])
  GPC_HD GPC_FI static void pos(const double* y, double* q)
  {
#pragma unroll
    for (int k = 0; k < D; k++) {
      q[k] = y[k];
      if (VAR) q[D + k] = y[2 * D + k];
    }
  }
  static constexpr int kSlotDoubles = 0;
  GPC_HD GPC_FI void bind(double*) {}
  GPC_HD GPC_FI bool wants_dense() const { return false; }
  GPC_HD GPC_FI static int next_slot(int slot, bool) { return slot >= 14 ? 0 : slot + 1; }
  enum { EST_A = 0, EST_B = 1, EST_C = 2, MAIN = 3 };
  double yo[N];    // orbit state at the last completed step
  double yn[N], yn1[N], ynk[N];
  double y1[N], ya[N];  // estimator: one-step result; midpoint of the two half steps
  double dt, init_dt, h, s, rtol, atol;
  long long nrun, step;
  int stage, phase;

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
    // derivative of the state at the evaluation point (x, v[, dx, dv])
    double d[N];
#pragma unroll
    for (int k = 0; k < D; k++) {
      d[k] = y[D + k];
      d[D + k] = a[k];
      if (VAR) {
        d[2 * D + k] = y[3 * D + k];
        d[3 * D + k] = a[D + k];
      }
    }
    // bovy_rk4_onestep (bovy_rk.c:142-170)
    if (stage == 0 || stage == 3) {
#pragma unroll
      for (int k = 0; k < N; k++) yn1[k] += h * d[k] / 6.;
    } else {
#pragma unroll
      for (int k = 0; k < N; k++) yn1[k] += h * d[k] / 3.;
    }
    if (stage < 2) {
#pragma unroll
      for (int k = 0; k < N; k++) ynk[k] = yn[k] + h * d[k] / 2.;
    } else if (stage == 2) {
#pragma unroll
      for (int k = 0; k < N; k++) ynk[k] = yn[k] + h * d[k];
    }
    if (++stage < 4) return;
    onestep_done(out);
  }

  template <class W>
  GPC_HD void onestep_done(W& out)
  {
    if (phase == EST_A) {
#pragma unroll
      for (int k = 0; k < N; k++) y1[k] = yn1[k];
      phase = EST_B;
      start(yo, dt / 2.);
      return;
    }
    if (phase == EST_B) {
#pragma unroll
      for (int k = 0; k < N; k++) ya[k] = yn1[k];
      phase = EST_C;
      start(ya, dt / 2.);
      return;
    }
    if (phase == EST_C) {
      double e = 0.;
#pragma unroll
      for (int k = 0; k < N; k++) e += exp(2. * log(fabs(y1[k] - yn1[k])) - 2. * s);
      e = sqrt(e / N);
      const double c = ceil(pow(e, 1. / 5.));
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

template <int D, bool VAR>
struct Dop853Machine : OrbitCommon {
  static constexpr int N = VAR ? 4 * D : 2 * D;
  static constexpr int NY = N;
  static constexpr int NV = N;
  static constexpr int NA = VAR ? 2 * D : D;  // force result size
  // force argument: positions (and deviation positions) of (x, v[, dx, dv])
  GPC_HD GPC_FI static void pos(const double* y, double* q)
  {
#pragma unroll
    for (int k = 0; k < D; k++) {
      q[k] = y[k];
      if (VAR) q[D + k] = y[2 * D + k];
    }
  }
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
  GPC_HD GPC_FI void bind(double* base) { ks = base; }
  GPC_HD GPC_FI double& K(int s, int i) const { return ks[((s - 1) * N + i) * kSlotStride]; }
  double h, hnew, hmax, pos_neg, facold, rtol, atol;
  double t_current, t_old, t_old_older, dnf;
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
    facold = 1.0e-4;
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
    t_current = t_old = t_old_older = tt[0];
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

  template <class W>
  GPC_HD void consume(const double* y, const double* a, W& out, int slot)
  {
    using namespace dp;
    if (!active_in(slot)) return;
    double d[N];
#pragma unroll
    for (int k = 0; k < D; k++) {
      d[k] = y[D + k];
      d[D + k] = a[k];
      if (VAR) {
        d[2 * D + k] = y[3 * D + k];
        d[3 * D + k] = a[D + k];
      }
    }
    if (stage == ST_INIT1) {  // leung_dop853.c:296-308
      double dny = 0.0;
      dnf = 0.0;
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
      const double der12 = dmax(fabs(der2), sqrt(dnf));
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
      const double sv = (t[iout + 1] - t_old) / h, s1 = 1.0 - sv;
      double v[N];
#pragma unroll
      for (int i = 0; i < N; i++) {
        const double k1 = this->k1[i], k2 = K(K2, i), k3 = K(K3, i), k4 = K(K4, i);
        const double k6 = K(K6, i), k7 = K(K7, i), k8 = K(K8, i), k9 = K(K9, i);
        const double k10 = K(K10, i), s14 = K(S14, i), s15 = K(S15, i);
        const double rc1 = y0[i];
        const double ydiff = K(K5, i) - y0[i];
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
        rc5 = h * (rc5 + d413 * k4 + d414 * s14 + d415 * s15 + d416 * d[i]);
        rc6 = h * (rc6 + d513 * k4 + d514 * s14 + d515 * s15 + d516 * d[i]);
        rc7 = h * (rc7 + d613 * k4 + d614 * s14 + d615 * s15 + d616 * d[i]);
        rc8 = h * (rc8 + d713 * k4 + d714 * s14 + d715 * s15 + d716 * d[i]);
        v[i] = rc1 +
               sv * (ydiff +
                     s1 * (bspl + sv * (rc4 + s1 * (rc5 + sv * (rc6 + s1 * (rc7 + sv * rc8))))));
      }
      iout++;
      out(iout, v);
    }
    finish_step(out);
  }

  GPC_HD void after_stage12()
  {
    using namespace dp;
    attempts++;
    t_old_older = t_old;
    t_old = t_current;
    t_current = t_current + h;
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
    double fac = fac11;  // Lund stabilisation with beta = 0: / pow(facold, 0) == / 1
    fac = dmax(1.0 / 6.0, dmin(1.0 / 0.333, fac / 0.9));
    hnew = h / fac;
    if (e <= 1.0) {
      facold = dmax(e, 1.0e-4);
      stage = ST_FSAL;
    } else {
      hnew = h / dmin(1.0 / 0.333, fac11 / 0.9);
      reject = true;
      t_current = t_old;
      t_old = t_old_older;
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

// Per-orbit driver used by the kernels and by the host test harness: run one
// machine to completion with the force evaluated by `force`.
template <class M, class F, class W>
GPC_HD void run_orbit(M& m, F& force, W& out)
{
  double y[M::NY], q[M::NA], a[M::NA];
  int slot = 0;
  while (!m.done) {
    m.point(y, slot);
    M::pos(y, q);
    force(q, a);
    m.consume(y, a, out, slot);
    slot = M::next_slot(slot, m.wants_dense());
  }
  fill_unreached_rows(m, out);
}

}  // namespace gpc
