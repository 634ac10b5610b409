// tests/harness/host_harness.cpp -- TEST ONLY.
//
// Runs the engine's own per-orbit state machines and force library
// (galpy_b200/csrc/machines.cuh, potentials.cuh) as plain host C++, one
// orbit after another, so the device code's logic can be compared with the
// CPU oracle in the CPU-only test suite.  It is never part of the product:
// the package has no CPU path and refuses to run without its CUDA library.
#include <vector>

#include "../../galpy_b200/csrc/compile_potential.h"
#include "../../galpy_b200/csrc/machines.cuh"

using namespace gpc;

namespace {
// one group's compiled records (a component may take continuation records)
int records(int planar, int npot, const int* pot_type, const double* pot_args,
            std::vector<GpComp>& comps)
{
  const int n = group_records(planar, npot, pot_type, pot_args);
  if (n < 1) return n < 0 ? n : -1;
  comps.assign((size_t)n, GpComp{});
  return compile_group(planar, npot, pot_type, pot_args, comps.data(), nullptr);
}

struct Rows {
  double* out;
  int nv, nt;
  long long i;
  void operator()(int j, const double* v) const
  {
    for (int k = 0; k < nv; k++) out[(i * nt + j) * nv + k] = v[k];
  }
};

template <int D, int PREC, bool VAR, class POT>
struct Force {
  const GpComp* c;
  int n;
  double scal[kMaxComp * kScalarStride];  // the kernel-parameter copy of the scalars
  void operator()(const double* q, double* a, double t) const
  {
    eval_force<D, PREC, VAR, POT>(c, n, q, a, scal, t);
  }
};

template <class M, int D, int PREC, bool VAR, class POT>
void run_all(int nobj, const double* w, int nt, const double* t, int indiv_t, const GpComp* comps,
             int ncomp, double dt, double rtol, double atol, long long max_att, double* out,
             int* err, long long* nsteps)
{
  Force<D, PREC, VAR, POT> f{comps, ncomp, {}};
  for (int k = 0; k < ncomp && k < kMaxComp; k++)
    for (int j = 0; j < kScalarStride; j++) f.scal[k * kScalarStride + j] = comps[k].c[j];
  std::vector<double> store((size_t)M::kSlotDoubles * kSlotStride + 1);
  for (long long i = 0; i < nobj; i++) {
    M m;
    m.bind(store.data());
    Rows r{out, M::NV, nt, i};
    m.init(w + i * M::NV, t + (indiv_t ? i * nt : 0), nt, dt, rtol, atol, max_att, r);
    run_orbit(m, f, r);
    err[i] = m.err;
    if (nsteps) nsteps[i] = m.nsteps;
  }
}

template <int D, int PREC, bool VAR, class POT>
int dispatch(int method, int nobj, const double* w, int nt, const double* t, int indiv_t,
             const GpComp* c, int n, double dt, double rtol, double atol, long long ma,
             double* out, int* err, long long* ns)
{
  switch (method) {
#define HARNESS_CASE(code, ...)                                                                  \
  case code:                                                                                     \
    run_all<__VA_ARGS__, D, PREC, VAR, POT>(nobj, w, nt, t, indiv_t, c, n, dt, rtol, atol, ma, \
                                            out, err, ns);                                       \
    return 0;
    HARNESS_CASE(M_LEAPFROG, SymplecticMachine<D, VAR, 2>)
    HARNESS_CASE(M_SYMPLEC4, SymplecticMachine<D, VAR, 4>)
    HARNESS_CASE(M_SYMPLEC6, SymplecticMachine<D, VAR, 6>)
    HARNESS_CASE(M_RK4, RKMachine<D, VAR, 4>)
    HARNESS_CASE(M_RK6, RKMachine<D, VAR, 6>)
    HARNESS_CASE(M_DOPR54, Dopr54Machine<D, VAR>)
    HARNESS_CASE(M_DOP853, Dop853Machine<D, VAR>)
#undef HARNESS_CASE
  }
  return -2;
}
}  // namespace

extern "C" int harness_integrate(int planar, int var, int method, int prec, int nobj,
                                 const double* w, int nt, const double* t, int indiv_t,
                                 int npot, const int* pot_type, const double* pot_args, double dt,
                                 double rtol, double atol, long long max_att, double* out,
                                 int* err, long long* nsteps)
{
  std::vector<GpComp> comps;
  int rc = records(planar, npot, pot_type, pot_args, comps);
  if (rc) return rc;
  const GpComp* c = comps.data();
  // the kernels' compile-time MWPotential2014 specialisation
  const bool mw14 = npot == 3 && pot_type[0] == T_PSWC && pot_type[1] == T_MN &&
                    pot_type[2] == T_NFW;
  const int nrec = (int)comps.size();
#define HARNESS_ARGS method, nobj, w, nt, t, indiv_t, c, nrec, dt, rtol, atol, max_att, out, err, nsteps
  if (var) return planar ? dispatch<2, PREC_FP64, true, DynPot>(HARNESS_ARGS)
                         : dispatch<3, PREC_FP64, true, DynPot>(HARNESS_ARGS);
  if (planar) {
    if (prec) return mw14 ? dispatch<2, PREC_F32, false, MW14Pot>(HARNESS_ARGS)
                          : dispatch<2, PREC_F32, false, DynPot>(HARNESS_ARGS);
    return mw14 ? dispatch<2, PREC_FP64, false, MW14Pot>(HARNESS_ARGS)
                : dispatch<2, PREC_FP64, false, DynPot>(HARNESS_ARGS);
  }
  if (prec) return mw14 ? dispatch<3, PREC_F32, false, MW14Pot>(HARNESS_ARGS)
                        : dispatch<3, PREC_F32, false, DynPot>(HARNESS_ARGS);
  return mw14 ? dispatch<3, PREC_FP64, false, MW14Pot>(HARNESS_ARGS)
              : dispatch<3, PREC_FP64, false, DynPot>(HARNESS_ARGS);
#undef HARNESS_ARGS
}

// DOP853 with its dense output through the request record (the kernels'
// queued dense output, served one request at a time): same outputs as
// harness_integrate's in-slot dense output, bit for bit.
template <int D, class POT>
static void run_dop853_queued(int nobj, const double* w, int nt, const double* t, int indiv_t,
                              const GpComp* comps, int ncomp, double rtol, double atol,
                              long long max_att, double* out, int* err, long long* nsteps)
{
  using M = Dop853Machine<D, false>;
  Force<D, PREC_FP64, false, POT> f{comps, ncomp, {}};
  for (int k = 0; k < ncomp && k < kMaxComp; k++)
    for (int j = 0; j < kScalarStride; j++) f.scal[k * kScalarStride + j] = comps[k].c[j];
  std::vector<double> store((size_t)M::kSlotDoubles * kSlotStride + 1);
  std::vector<double> q((size_t)M::kQueueFields * M::kQueueSlots);
  for (long long i = 0; i < nobj; i++) {
    M m;
    m.bind(store.data(), true);
    Rows r{out, M::NV, nt, i};
    const double* tt = t + (indiv_t ? i * nt : 0);
    m.init(w + i * M::NV, tt, nt, kDtSentinel, rtol, atol, max_att, r);
    run_orbit_queued(m, f, r, q.data(), tt, i);
    err[i] = m.err;
    if (nsteps) nsteps[i] = m.nsteps;
  }
}

extern "C" int harness_dop853_queued(int planar, int nobj, const double* w, int nt,
                                     const double* t, int indiv_t, int npot, const int* pot_type,
                                     const double* pot_args, double rtol, double atol,
                                     long long max_att, double* out, int* err, long long* nsteps)
{
  std::vector<GpComp> comps;
  int rc = records(planar, npot, pot_type, pot_args, comps);
  if (rc) return rc;
  const bool mw14 = npot == 3 && pot_type[0] == T_PSWC && pot_type[1] == T_MN &&
                    pot_type[2] == T_NFW;
  if (planar) {
    if (mw14)
      run_dop853_queued<2, MW14Pot>(nobj, w, nt, t, indiv_t, comps.data(), (int)comps.size(), rtol, atol,
                                    max_att, out, err, nsteps);
    else
      run_dop853_queued<2, DynPot>(nobj, w, nt, t, indiv_t, comps.data(), (int)comps.size(), rtol, atol,
                                   max_att, out, err, nsteps);
  } else {
    if (mw14)
      run_dop853_queued<3, MW14Pot>(nobj, w, nt, t, indiv_t, comps.data(), (int)comps.size(), rtol, atol,
                                    max_att, out, err, nsteps);
    else
      run_dop853_queued<3, DynPot>(nobj, w, nt, t, indiv_t, comps.data(), (int)comps.size(), rtol, atol,
                                   max_att, out, err, nsteps);
  }
  return 0;
}

// Surface-of-section machines (FP64, run-time component list) on SOS states:
// system 1 (3D): w [nobj][7] = (x, y, vx, vy, A, t, psi); 2 / 3 (planar,
// surface x = 0 / y = 0): w [nobj][5] = (u, vu, A, t, psi); out raw rows.
template <class SYS, int D>
static int run_sos(int method, int nobj, const double* w, int nt, const double* t, int indiv_t,
                   const GpComp* c, int npot, double dt, double rtol, double atol,
                   long long max_att, double* out, int* err, long long* nsteps)
{
  switch (method) {
    case M_RK4:
      run_all<RKMachine<D, false, 4, SYS>, D, PREC_FP64, false, DynPot>(
          nobj, w, nt, t, indiv_t, c, npot, dt, rtol, atol, max_att, out, err, nsteps);
      return 0;
    case M_RK6:
      run_all<RKMachine<D, false, 6, SYS>, D, PREC_FP64, false, DynPot>(
          nobj, w, nt, t, indiv_t, c, npot, dt, rtol, atol, max_att, out, err, nsteps);
      return 0;
    case M_DOPR54:
      run_all<Dopr54Machine<D, false, SYS>, D, PREC_FP64, false, DynPot>(
          nobj, w, nt, t, indiv_t, c, npot, dt, rtol, atol, max_att, out, err, nsteps);
      return 0;
    case M_DOP853:
      run_all<Dop853Machine<D, false, SYS>, D, PREC_FP64, false, DynPot>(
          nobj, w, nt, t, indiv_t, c, npot, dt, rtol, atol, max_att, out, err, nsteps);
      return 0;
  }
  return -2;
}

extern "C" int harness_integrate_sos(int system, int method, int nobj, const double* w, int nt,
                                     const double* t, int indiv_t, int npot, const int* pot_type,
                                     const double* pot_args, double dt, double rtol, double atol,
                                     long long max_att, double* out, int* err, long long* nsteps)
{
  const int planar = system != 1;
  std::vector<GpComp> comps;
  int rc = records(planar, npot, pot_type, pot_args, comps);
  if (rc) return rc;
  const GpComp* c = comps.data();
  const int nrec = (int)comps.size();
#define SOS_ARGS method, nobj, w, nt, t, indiv_t, c, nrec, dt, rtol, atol, max_att, out, err, nsteps
  if (system == 1) return run_sos<SosSystem, 3>(SOS_ARGS);
  if (system == 2) return run_sos<PlanarSosSystem<0>, 2>(SOS_ARGS);
  if (system == 3) return run_sos<PlanarSosSystem<1>, 2>(SOS_ARGS);
#undef SOS_ARGS
  return -1;
}

// accelerations (and tidal tensors) at points, for force-level tests
// gamma*(a, u) from a compiled PowerSphericalwCutoff record (table check)
extern "C" int harness_gamma_star(double alpha, double rc, int n, const double* u, double* out)
{
  const int pt = T_PSWC;
  const double pa[3] = {1.0, alpha, rc};
  GpComp c;
  int rc_ = compile_group(1, 1, &pt, pa, &c, nullptr);
  if (rc_) return rc_;
  for (int i = 0; i < n; i++) out[i] = gamma_star<double>(&c, u[i], c.c[6]);
  return 0;
}

// potential values at points (energy kernel's device function, on the host),
// from galpy's 3D or planar argument list
extern "C" int harness_potential_in(int planar, int n, const double* x, const double* y,
                                    const double* z, int npot, const int* pot_type,
                                    const double* pot_args, double* out)
{
  std::vector<GpComp> comps;
  int rc = records(planar, npot, pot_type, pot_args, comps);
  if (rc) return rc;
  const int nrec = (int)comps.size();
  for (int i = 0; i < n; i++) out[i] = potential_value(comps.data(), nrec, x[i], y[i], z[i]);
  return 0;
}

extern "C" int harness_potential(int n, const double* x, const double* y, const double* z,
                                 int npot, const int* pot_type, const double* pot_args,
                                 double* out)
{
  return harness_potential_in(0, n, x, y, z, npot, pot_type, pot_args, out);
}

// accelerations (tidal tensors, FP32 accelerations) at points at time t
extern "C" int harness_forces_at(int planar, int n, const double* x, const double* y,
                                 const double* z, double t, int npot, const int* pot_type,
                                 const double* pot_args, double* acc /*[n][3]*/,
                                 double* tidal /*[n][6] or NULL*/,
                                 double* acc32 /*[n][3] or NULL*/)
{
  std::vector<GpComp> comps;
  int rc = records(planar, npot, pot_type, pot_args, comps);
  if (rc) return rc;
  const int nrec = (int)comps.size();
  for (int i = 0; i < n; i++) {
    double ax = 0, ay = 0, az = 0, K[6];
    if (planar)
      accel<double, true>(comps.data(), nrec, x[i], y[i], 0.0, ax, ay, az, nullptr, t);
    else
      accel<double, false>(comps.data(), nrec, x[i], y[i], z[i], ax, ay, az, nullptr, t);
    acc[3 * i] = ax;
    acc[3 * i + 1] = ay;
    acc[3 * i + 2] = az;
    if (tidal) {
      double bx, by, bz;
      if (planar)
        accel_tidal<true>(comps.data(), nrec, x[i], y[i], 0.0, bx, by, bz, K, t);
      else
        accel_tidal<false>(comps.data(), nrec, x[i], y[i], z[i], bx, by, bz, K, t);
      for (int k = 0; k < 6; k++) tidal[6 * i + k] = K[k];
    }
    if (acc32) {
      float fx = 0, fy = 0, fz = 0;
      if (planar)
        accel<float, true>(comps.data(), nrec, (float)x[i], (float)y[i], 0.f, fx, fy, fz,
                           nullptr, t);
      else
        accel<float, false>(comps.data(), nrec, (float)x[i], (float)y[i], (float)z[i], fx, fy,
                            fz, nullptr, t);
      acc32[3 * i] = fx;
      acc32[3 * i + 1] = fy;
      acc32[3 * i + 2] = fz;
    }
  }
  return 0;
}

extern "C" int harness_forces(int planar, int n, const double* x, const double* y,
                              const double* z, int npot, const int* pot_type,
                              const double* pot_args, double* acc, double* tidal, double* acc32)
{
  return harness_forces_at(planar, n, x, y, z, 0.0, npot, pot_type, pot_args, acc, tidal, acc32);
}

// The mixed float64 / float32 MWPotential2014 forces (MIX_TAIL32 = 1,
// MIX_F32BULGE = 2) at n points, [n][3].
extern "C" int harness_forces_mixed(int mix, int planar, int n, const double* x, const double* y,
                                    const double* z, const double* pot_args, double* acc)
{
  const int pot_type[3] = {T_PSWC, T_MN, T_NFW};
  std::vector<GpComp> comps(3);
  int rc = compile_group(planar, 3, pot_type, pot_args, comps.data(), nullptr);
  if (rc) return rc;
  for (int i = 0; i < n; i++) {
    double ax = 0, ay = 0, az = 0;
    const double zi = planar ? 0.0 : z[i];
    if (mix == MIX_TAIL32) {
      if (planar)
        accel<double, true, MW14MixedPot<false, MIX_TAIL32>>(comps.data(), 3, x[i], y[i], zi,
                                                            ax, ay, az);
      else
        accel<double, false, MW14MixedPot<false, MIX_TAIL32>>(comps.data(), 3, x[i], y[i], zi,
                                                             ax, ay, az);
    } else {
      if (planar)
        accel<double, true, MW14MixedPot<false, MIX_F32BULGE>>(comps.data(), 3, x[i], y[i], zi,
                                                              ax, ay, az);
      else
        accel<double, false, MW14MixedPot<false, MIX_F32BULGE>>(comps.data(), 3, x[i], y[i],
                                                               zi, ax, ay, az);
    }
    acc[3 * i] = ax;
    acc[3 * i + 1] = ay;
    acc[3 * i + 2] = az;
  }
  return 0;
}

// ------------------------------------------------------------- adjoint ---
#include "../../galpy_b200/csrc/adjoint.cuh"

namespace {
struct AdjPot {
  std::vector<GpComp> comps;
  int rc = 0;
  AdjPot(int planar, int npot, const int* pot_type, const double* pot_args) : comps(npot)
  {
    rc = compile_group(planar, npot, pot_type, pot_args, comps.data(), nullptr);
  }
  adj::Field<DynPot> field() const { return {comps.data(), (int)comps.size(), nullptr}; }
};
}  // namespace

extern "C" int harness_adj_nparam(int planar, int npot, const int* pot_type,
                                  const double* pot_args)
{
  AdjPot P(planar, npot, pot_type, pot_args);
  if (P.rc) return P.rc;
  return adj::group_nparam(P.comps.data(), npot);
}

// g[i][p] = lambda_i . d a(x_i) / d theta_p
extern "C" int harness_adj_param_vjp(int planar, int n, const double* x, const double* y,
                                     const double* z, const double* lam /*[n][3]*/, int npot,
                                     const int* pot_type, const double* pot_args, double* g)
{
  AdjPot P(planar, npot, pot_type, pot_args);
  if (P.rc) return P.rc;
  const int np = adj::group_nparam(P.comps.data(), npot);
  for (int i = 0; i < n; i++) {
    double* gi = g + (size_t)i * np;
    for (int p = 0; p < np; p++) gi[p] = 0.0;
    if (planar)
      adj::accel_param_vjp<true>(P.comps.data(), npot, x[i], y[i], 0.0, lam[3 * i],
                                 lam[3 * i + 1], 0.0, gi);
    else
      adj::accel_param_vjp<false>(P.comps.data(), npot, x[i], y[i], z[i], lam[3 * i],
                                  lam[3 * i + 1], lam[3 * i + 2], gi);
  }
  return np;
}

// Forward pass per orbit (w0, yT: [nobj][nv]); hrec [nobj][hcap] (may be
// NULL); nsteps, err [nobj].
extern "C" int harness_adj_forward(int planar, int nobj, const double* w0, double t0, double T,
                                   double rtol, double atol, int npot, const int* pot_type,
                                   const double* pot_args, double* yT, long long* nsteps,
                                   int* err, double* hrec, long long hcap)
{
  AdjPot P(planar, npot, pot_type, pot_args);
  if (P.rc) return P.rc;
  const int nv = planar ? 4 : 6;
  const int ccap = 4096;
  std::vector<double> ck((size_t)ccap * (nv + 1 + adj::kCkptEvery));
  for (int i = 0; i < nobj; i++) {
    double* h = hrec ? hrec + (size_t)i * hcap : nullptr;
    if (planar)
      err[i] = adj::forward_orbit<2, DynPot>(P.field(), w0 + (size_t)i * nv, t0, T, rtol, atol, 0,
                                             ck.data(), 1, ccap, h, 1, hcap,
                                             yT + (size_t)i * nv, nsteps + i);
    else
      err[i] = adj::forward_orbit<3, DynPot>(P.field(), w0 + (size_t)i * nv, t0, T, rtol, atol, 0,
                                             ck.data(), 1, ccap, h, 1, hcap,
                                             yT + (size_t)i * nv, nsteps + i);
  }
  return 0;
}

// The forward map with frozen steps hrec [nobj][hcap], nsteps [nobj].
extern "C" int harness_adj_replay(int planar, int nobj, const double* w0, double t0, double T,
                                  int npot, const int* pot_type, const double* pot_args,
                                  const double* hrec, long long hcap, const long long* nsteps,
                                  double* yT)
{
  AdjPot P(planar, npot, pot_type, pot_args);
  if (P.rc) return P.rc;
  const int nv = planar ? 4 : 6;
  for (int i = 0; i < nobj; i++) {
    if (planar)
      adj::replay_orbit<2, DynPot>(P.field(), w0 + (size_t)i * nv, t0, T, hrec + (size_t)i * hcap,
                                   1, nsteps[i], yT + (size_t)i * nv);
    else
      adj::replay_orbit<3, DynPot>(P.field(), w0 + (size_t)i * nv, t0, T, hrec + (size_t)i * hcap,
                                   1, nsteps[i], yT + (size_t)i * nv);
  }
  return 0;
}

// Forward + backward: gw0 [nobj][nv] = dL/dw0, gth [nobj][np] = dL/dtheta
// for dL/dyT = gyT [nobj][nv].  Returns np.
extern "C" int harness_adj_gradient(int planar, int nobj, const double* w0, double t0, double T,
                                    double rtol, double atol, int npot, const int* pot_type,
                                    const double* pot_args, const double* gyT, double* gw0,
                                    double* gth, int* err)
{
  AdjPot P(planar, npot, pot_type, pot_args);
  if (P.rc) return P.rc;
  const int nv = planar ? 4 : 6;
  const int np = adj::group_nparam(P.comps.data(), npot);
  const int ccap = 4096;
  std::vector<double> ck((size_t)ccap * (nv + 1 + adj::kCkptEvery));
  double yT[6];
  long long ns;
  for (int i = 0; i < nobj; i++) {
    double* lam = gw0 + (size_t)i * nv;
    double* g = gth + (size_t)i * np;
    for (int c = 0; c < nv; c++) lam[c] = gyT[(size_t)i * nv + c];
    for (int p = 0; p < np; p++) g[p] = 0.0;
    if (planar) {
      err[i] = adj::forward_orbit<2, DynPot>(P.field(), w0 + (size_t)i * nv, t0, T, rtol, atol, 0,
                                             ck.data(), 1, ccap, nullptr, 1, 0, yT, &ns);
      if (err[i] == 0)
        adj::backward_orbit<2, DynPot>(P.field(), T, ck.data(), 1, ns, lam, g);
    } else {
      err[i] = adj::forward_orbit<3, DynPot>(P.field(), w0 + (size_t)i * nv, t0, T, rtol, atol, 0,
                                             ck.data(), 1, ccap, nullptr, 1, 0, yT, &ns);
      if (err[i] == 0)
        adj::backward_orbit<3, DynPot>(P.field(), T, ck.data(), 1, ns, lam, g);
    }
  }
  return np;
}

namespace {
// Checkpoints of the frozen-step map (state and time at each segment start,
// the step sizes), then the device's backward sweep.
template <int D>
void backward_frozen(const AdjPot& P, const double* w0, double t0, double T, const double* h,
                     long long ns, double* lam, double* g)
{
  constexpr int N = 2 * D, CW = N + 1 + adj::kCkptEvery;
  std::vector<double> ck((size_t)((ns + adj::kCkptEvery - 1) / adj::kCkptEvery + 1) * CW);
  double y[N], k[12][N], inc[N], ynew[N], t = t0;
  for (int c = 0; c < N; c++) y[c] = w0[c];
  for (long long n = 0; n < ns; n++) {
    double* p = ck.data() + (n / adj::kCkptEvery) * CW;
    if (n % adj::kCkptEvery == 0) {
      for (int c = 0; c < N; c++) p[c] = y[c];
      p[N] = t;
    }
    p[N + 1 + n % adj::kCkptEvery] = h[n];
    adj::rhs<D, DynPot>(P.field(), y, k[0]);
    adj::run_stages<D, DynPot, 1, 12>(P.field(), y, h[n], k, nullptr);
    adj::new_state<D>(y, h[n], k, inc, ynew);
    for (int c = 0; c < N; c++) y[c] = ynew[c];
    t = t + h[n];
  }
  adj::backward_orbit<D, DynPot>(P.field(), T, ck.data(), 1, ns, lam, g);
}
}  // namespace

// Backward pass with given frozen steps hrec [nobj][hcap] (nsteps [nobj]).
// Returns np.
extern "C" int harness_adj_backward_frozen(int planar, int nobj, const double* w0, double t0,
                                           double T, int npot, const int* pot_type,
                                           const double* pot_args, const double* hrec,
                                           long long hcap, const long long* nsteps,
                                           const double* gyT, double* gw0, double* gth)
{
  AdjPot P(planar, npot, pot_type, pot_args);
  if (P.rc) return P.rc;
  const int nv = planar ? 4 : 6;
  const int np = adj::group_nparam(P.comps.data(), npot);
  for (int i = 0; i < nobj; i++) {
    double* lam = gw0 + (size_t)i * nv;
    double* g = gth + (size_t)i * np;
    for (int c = 0; c < nv; c++) lam[c] = gyT[(size_t)i * nv + c];
    for (int p = 0; p < np; p++) g[p] = 0.0;
    if (planar)
      backward_frozen<2>(P, w0 + (size_t)i * nv, t0, T, hrec + (size_t)i * hcap, nsteps[i], lam, g);
    else
      backward_frozen<3>(P, w0 + (size_t)i * nv, t0, T, hrec + (size_t)i * hcap, nsteps[i], lam, g);
  }
  return np;
}

// Binade-table functions of the force path: kind 0 = (x)^(-alpha/2) from a
// PowerSphericalwCutoff record, kind 1 = log1p(x) from an NFW record, kind 2
// the single-precision log1p.
extern "C" int harness_binade(int kind, double alpha, int n, const double* x, double* out)
{
  GpComp c;
  if (kind == 0) {
    const int pt = T_PSWC;
    const double pa[3] = {1.0, alpha, 0.5};
    if (compile_group(1, 1, &pt, pa, &c, nullptr)) return -1;
    for (int i = 0; i < n; i++) out[i] = pswc_power(&c, x[i]);
  } else {
    const int pt = T_NFW;
    const double pa[2] = {1.0, 2.0};
    if (compile_group(1, 1, &pt, pa, &c, nullptr)) return -1;
    for (int i = 0; i < n; i++)
      out[i] = kind == 1 ? nfw_log1p(&c, x[i]) : (double)nfw_log1pf(&c, (float)x[i]);
  }
  return 0;
}
