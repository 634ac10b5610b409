/*
 * galpy_cuda.h -- C ABI of libgalpy_cuda.so, the B200 orbit-integration engine
 * behind galpy's Orbit.integrate methods 'leapfrog_cuda', 'rk4_cuda',
 * 'rk6_cuda', 'symplec4_cuda', 'symplec6_cuda', 'dopr54_cuda' and
 * 'dop853_cuda'.
 *
 * The galpy-facing entry points take exactly the arguments of the libgalpy
 * functions they stand in for, with galpy's conventions: AoS arrays owned by
 * the caller (host memory), yo overwritten with the rectangular initial
 * conditions, t either shared (nt) or per orbit (nobj*nt, indiv_t = 1),
 * rtol/atol as natural logarithms, dt = -9999.99 meaning "estimate the step",
 * odeint_type 0 leapfrog, 1 rk4, 2 rk6, 3 symplec4, 4 symplec6, 5 dopr54,
 * 6 dop853 (galpy's numbering; 7 ias15 returns GALPY_CUDA_ERR_METHOD so the
 * caller can fall back), pot_type/pot_args as produced by galpy's _parse_pot
 * (types 0 LogarithmicHalo, 5 MiyamotoNagai, 8 Hernquist, 9 NFW,
 * 15 PowerSphericalwCutoff, and the spherical 7 PowerSpherical/Kepler,
 * 10 Jaffe, 14 Isochrone, 17 Plummer, 18 PseudoIsothermal, 20 Burkert,
 * 33 DehnenCoreSpherical, 34 DehnenSpherical, 35 HomogeneousSphere, 40 Null,
 * 41 Einasto, 46 ExpTruncNFW, and the axisymmetric 12 FlattenedPower,
 * 16 KuzminKutuzovStaeckel, 19 KuzminDisk, the ellipsoidal 21 TriaxialHernquist, 22 TriaxialNFW,
 * 23 TriaxialJaffe, 30 PerfectEllipsoid, 37 TriaxialGaussian, 38 PowerTriaxial,
 * 43 TwoPowerTriaxial (at most 96 Gauss-Legendre nodes), and in the planar
 * entry points 29 HenonHeiles;
 * others return GALPY_CUDA_ERR_POTENTIAL), per-orbit err[] (0 ok, -10 interrupted by
 * SIGINT, 1 = dopr54 forced a step at its smallest allowed size, as the
 * reference does; the orbit is complete).  Two additions: every entry point returns a status code instead
 * of void, and takes a trailing options pointer (NULL = defaults).
 *
 * Per-orbit err values beyond the reference's: 2 = attempt budget exhausted
 * (or, in dopr54, a step too small to advance the time, where the reference
 * loops forever), 3 = the state became non-finite (the reference loops
 * forever on NaN in DOP853; rows after the failure are NaN here).
 */
#ifndef GALPY_CUDA_H
#define GALPY_CUDA_H
#ifdef __cplusplus
extern "C" {
#endif

#define GALPY_CUDA_ABI_VERSION 2

/* return codes */
#define GALPY_CUDA_OK 0
#define GALPY_CUDA_ERR_ARG (-1)         /* invalid argument */
#define GALPY_CUDA_ERR_METHOD (-2)      /* odeint_type not implemented on the GPU */
#define GALPY_CUDA_ERR_POTENTIAL (-3)   /* a pot_type not implemented on the GPU */
#define GALPY_CUDA_ERR_CUDA (-4)        /* CUDA runtime failure; see galpy_cuda_last_error */
#define GALPY_CUDA_ERR_NODEVICE (-5)    /* no CUDA device visible */
#define GALPY_CUDA_ERR_INTERRUPTED (-10) /* SIGINT during the call; err[] holds -10 */

/* precision of the force evaluation and the state.  FP64 and F32FORCE apply
 * to every method and potential; the three mixed forms to plain (not
 * variational) runs in MWPotential2014-type potentials
 * (GALPY_CUDA_SIG_MW14), other combinations return GALPY_CUDA_ERR_METHOD. */
#define GALPY_CUDA_FP64 0       /* float64 force and state */
#define GALPY_CUDA_F32FORCE 1   /* float32 force, float64 state */
#define GALPY_CUDA_F64_TAIL32 2 /* float64 force with the high-order terms of its special-
                                   function table polynomials in float32 (~1e-11 relative
                                   force error), float64 state; leapfrog, symplec4, rk4,
                                   dop853 */
#define GALPY_CUDA_F32BULGE 3   /* as F64_TAIL32 with the bulge (PowerSphericalwCutoff) term in
                                   float32; leapfrog, symplec4, rk4, dop853 */
#define GALPY_CUDA_F32FORCE_DF 4 /* float32 force, compensated double-float (two float32)
                                    state; leapfrog, symplec4 */

/* array layouts of the device-pointer entry point */
#define GALPY_CUDA_IN_AOS 0      /* [nobj][nv] rectangular */
#define GALPY_CUDA_IN_SOA 1      /* [nv][nobj] rectangular */
#define GALPY_CUDA_OUT_GALPY 0   /* [nobj][nrow][nv], galpy's cylindrical coordinates */
#define GALPY_CUDA_OUT_AOS_RECT 1 /* [nobj][nrow][nv] rectangular */
#define GALPY_CUDA_OUT_SOA_RECT 2 /* [nv][nrow][nobj] rectangular */
#define GALPY_CUDA_OUT_SOA_CYL 3  /* [nv][nrow][nobj] cylindrical */

/* potential signatures (kernels specialised at compile time) */
#define GALPY_CUDA_SIG_GENERIC 0 /* any list of supported components */
#define GALPY_CUDA_SIG_MW14 1    /* exactly (15, 5, 9): MWPotential2014's component types */
#define GALPY_CUDA_SIG_COMMON 2  /* a list without ellipsoidal components (types 21, 22, 23,
                                    30, 37, 38, 43): float64 kernels whose run-time list
                                    leaves that family out (fewer registers).  Orbits of a
                                    launch given this signature for a potential with such a
                                    component stop with err 3 (non-finite force); when the
                                    launch carries comps_host the engine checks the types and
                                    uses the full list instead. */

/* order in which orbits are handed to the GPU threads */
/* the ODE system of a device launch (galpy_cuda_launch.system) */
#define GALPY_CUDA_SYS_ORBIT 0 /* orbit in time: the 2*dim (or 4*dim variational) state */
#define GALPY_CUDA_SYS_SOS 1   /* 3D surface of section: (x,y,vx,vy,A,t,psi) in the psi increment */
#define GALPY_CUDA_SYS_SOS_PLANAR_X 2 /* planar, surface x = 0: (y,vy,A,t,psi) */
#define GALPY_CUDA_SYS_SOS_PLANAR_Y 3 /* planar, surface y = 0: (x,vx,A,t,psi) */

#define GALPY_CUDA_SCHED_IN_ORDER 0
#define GALPY_CUDA_SCHED_LONGEST_FIRST 1 /* by estimated cost: integration time x orbital frequency */

typedef void (*galpy_cuda_callback)(void);

typedef struct galpy_cuda_opts {
  int size;                /* sizeof(galpy_cuda_opts) */
  int device;              /* CUDA device ordinal, -1 = current */
  int precision;           /* a GALPY_CUDA_* precision form (default GALPY_CUDA_FP64) */
  int block_size;          /* threads per block, 0 = tuned default */
  long long max_attempts;  /* per-orbit step-attempt budget, 0 = unlimited */
  long long *nsteps;       /* optional out, host [nobj]: accepted steps per orbit */
  double *elapsed_ms;      /* optional out: device time of the integration kernel */
  int variant;             /* register-budget variant of the kernel (see galpy_cuda_launch) */
  int schedule;            /* GALPY_CUDA_SCHED_* (default longest-first) */
  int stream_rows;         /* the blocking entry points' result transfer: -1 (or a shorter
                              struct) automatic -- for large results the rows of finished
                              orbits are copied to the host while the kernel runs; 0 one copy
                              after the kernel; 1 streamed whatever the size */
  int ndevices;            /* devices one blocking call spreads its orbits over: 0 or 1 (or a
                              shorter struct) one device (`device`); n > 1 the first n of
                              `devices` (or ordinals 0..n-1 when `devices` is NULL); -1 every
                              visible device.  The orbits are cut into contiguous ranges of
                              equal estimated cost (the longest-first estimate), one per
                              device, integrated concurrently, each range's results written
                              straight into its rows of the caller's arrays; no data crosses
                              between devices.  elapsed_ms then reports the slowest device. */
  const int *devices;      /* optional device ordinals for ndevices > 1; an ordinal may
                              repeat (its ranges then run concurrently on that device) */
} galpy_cuda_opts;

/* Compiled potential record size in bytes. */
int galpy_cuda_comp_size(void);

/* Records one potential group compiles to: one per component, plus
 * continuation records that hold an SCF expansion's coefficients (galpy
 * type 24); the stride of a parameter group in the compiled array and the
 * launch's ncomp.  Returns the count, or GALPY_CUDA_ERR_POTENTIAL /
 * GALPY_CUDA_ERR_ARG. */
int galpy_cuda_comp_records(int planar, int npot, const int *pot_type, const double *pot_args);

/* Signature of a component-type list (GALPY_CUDA_SIG_*), for the device
 * entry point's launch.signature. */
int galpy_cuda_signature(int npot, const int *pot_type);

/* Translate galpy's (pot_type, pot_args) for ngroup potential groups with the
 * same component types (pot_args holds ngroup consecutive argument blocks)
 * into compiled records written to out (host memory of ngroup *
 * galpy_cuda_comp_records(...) * galpy_cuda_comp_size() bytes; every group
 * must compile to the same number of records).  Returns 0 or
 * GALPY_CUDA_ERR_POTENTIAL / GALPY_CUDA_ERR_ARG. */
int galpy_cuda_compile_potential(int planar, int npot, const int *pot_type,
                                 const double *pot_args, int ngroup, void *out);

/* Contiguous orbit ranges of equal estimated cost, as a multi-device call
 * (galpy_cuda_opts.ndevices) cuts them; for callers that spread a batch over
 * processes themselves (one per device, e.g. torch.distributed ranks).
 * w [nobj][nv] rectangular states (positions first), t [nt] or [nobj][nt];
 * pot_args holds ngroup consecutive argument blocks (as for
 * galpy_cuda_compile_potential) and group [nobj] each orbit's block (NULL
 * when ngroup is 1); writes bounds[nparts+1]: part k is orbits
 * [bounds[k], bounds[k+1]).  The cost of an orbit is |t_end - t_0| *
 * Omega(x_0), Omega^2 = |a.x|/|x|^2 in its group's potential (the
 * longest-first schedule's estimate).  Host only: needs no device. */
int galpy_cuda_split_orbits(int planar, long long nobj, const double *w, int nv, int nt,
                            const double *t, int indiv_t, int npot, const int *pot_type,
                            const double *pot_args, int ngroup, const int *group, int nparts,
                            long long *bounds);

/* Stands in for integrateFullOrbit (galpy/orbit/orbit_c_ext/integrateFullOrbit.c:1046). */
int integrateFullOrbit_cuda(int nobj, double *yo, int nt, double *t, int indiv_t, int npot,
                            int *pot_type, double *pot_args, void *pot_tfuncs, double dt,
                            double rtol, double atol, double *result, int *err,
                            int odeint_type, galpy_cuda_callback cb,
                            const galpy_cuda_opts *opts);

/* Stands in for integratePlanarOrbit (galpy/orbit/orbit_c_ext/integratePlanarOrbit.c:743). */
int integratePlanarOrbit_cuda(int nobj, double *yo, int nt, double *t, int indiv_t, int npot,
                              int *pot_type, double *pot_args, void *pot_tfuncs, double dt,
                              double rtol, double atol, double *result, int *err,
                              int odeint_type, galpy_cuda_callback cb,
                              const galpy_cuda_opts *opts);

/* Stands in for integrateFullOrbit_sos (integrateFullOrbit.c:1151-1167):
 * yo [nobj][7] = (R,vR,vT,z,vz,phi,t0), overwritten with the surface-of-
 * section state (x,y,vx,vy,A,t0,psi0) like the reference
 * (cyl_to_sos_galpy); psi [npsi] or [nobj][npsi] angle increments; dpsi the
 * step (-9999.99 = estimate); odeint_type 1 rk4, 2 rk6, 5 dopr54, 6 dop853
 * (the symplectic ones and ias15 return GALPY_CUDA_ERR_METHOD, as the
 * reference does not integrate them here); result [nobj][npsi][7] =
 * (R,vR,vT,z,vz,phi,t). */
int integrateFullOrbit_sos_cuda(int nobj, double *yo, int npsi, double *psi, int indiv_psi,
                                int npot, int *pot_type, double *pot_args, void *pot_tfuncs,
                                double dpsi, double rtol, double atol, double *result, int *err,
                                int odeint_type, galpy_cuda_callback cb,
                                const galpy_cuda_opts *opts);

/* Stands in for integratePlanarOrbit_sos (integratePlanarOrbit.c:848-866):
 * yo [nobj][5] = (R,vR,vT,phi,t0), overwritten with the surface-of-section
 * state (polar_to_sos_galpy); surface 0: x = 0 (state (y,vy,A,t,psi)),
 * 1: y = 0 (state (x,vx,A,t,psi)); result [nobj][npsi][5] =
 * (R,vR,vT,phi,t); methods as integrateFullOrbit_sos_cuda. */
int integratePlanarOrbit_sos_cuda(int nobj, double *yo, int npsi, double *psi, int indiv_psi,
                                  int surface, int npot, int *pot_type, double *pot_args,
                                  void *pot_tfuncs, double dpsi, double rtol, double atol,
                                  double *result, int *err, int odeint_type,
                                  galpy_cuda_callback cb, const galpy_cuda_opts *opts);

/* Stands in for integrateFullOrbit_dxdv (integrateFullOrbit.c:1234): one
 * orbit, yo = (x,y,z,vx,vy,vz,dx,dy,dz,dvx,dvy,dvz), result [nt][12]. */
int integrateFullOrbit_dxdv_cuda(double *yo, int nt, double *t, int npot, int *pot_type,
                                 double *pot_args, void *pot_tfuncs, double dt, double rtol,
                                 double atol, double *result, int *err, int odeint_type,
                                 const galpy_cuda_opts *opts);

/* Stands in for integratePlanarOrbit_dxdv (integratePlanarOrbit.c:940): one
 * orbit, yo = (x,y,vx,vy,dx,dy,dvx,dvy), result [nt][8]. */
int integratePlanarOrbit_dxdv_cuda(double *yo, int nt, double *t, int npot, int *pot_type,
                                   double *pot_args, void *pot_tfuncs, double dt, double rtol,
                                   double atol, double *result, int *err, int odeint_type,
                                   galpy_cuda_callback cb, const galpy_cuda_opts *opts);

/* Batched variational integration (galpy runs the single-orbit functions
 * above once per orbit from Python, galpy/orbit/Orbits.py:2445): nobj orbits
 * with one deviation column each, yo [nobj][4*dim] rectangular, t shared or
 * per orbit, result [nobj][nt][4*dim]. */
int integrateOrbit_dxdv_batch_cuda(int planar, int nobj, double *yo, int nt, double *t,
                                   int indiv_t, int npot, int *pot_type, double *pot_args,
                                   double dt, double rtol, double atol, double *result, int *err,
                                   int odeint_type, const galpy_cuda_opts *opts);

/* Device-pointer entry point: all arrays live on the device, the call is
 * asynchronous on `stream`.  Needs 64 bytes of device scratch for the
 * work-stealing counter (plus the scheduling scratch, see `schedule`),
 * allocated stream-ordered per call. */
typedef struct galpy_cuda_launch {
  int planar, variational, odeint_type, precision;
  long long nobj;
  int nt, indiv_t;
  const double *t;          /* nt or nobj*nt */
  const double *w0;         /* initial rectangular states */
  int in_layout;            /* GALPY_CUDA_IN_* */
  double *out;
  int out_layout;           /* GALPY_CUDA_OUT_* */
  int out_row0;             /* first row stored (nt-1: final state only) */
  int *err;                 /* [nobj] */
  long long *nsteps;        /* [nobj] or NULL */
  const void *comps;        /* compiled potential, ngroup*ncomp records */
  int ncomp;
  const int *group;         /* [nobj] group of each orbit, or NULL (one group) */
  double dt, rtol, atol;    /* galpy conventions */
  long long max_attempts;
  const int *abort_flag;    /* device int polled by the kernel, or NULL */
  void *stream;             /* cudaStream_t */
  int block_size, grid_size; /* 0 = defaults */
  int signature;            /* galpy_cuda_signature(pot_type) */
  int schedule;             /* GALPY_CUDA_SCHED_*; longest-first sorts the work queue
                               (needs ~13 bytes/orbit of stream-ordered scratch) */
  int variant;              /* register budget: 0 compiler default, 1 capped for occupancy */
  const void *comps_host;   /* optional host copy of `comps` (ncomp records, one group):
                               its scalars are passed as kernel parameters */
  int size_ext;             /* 1 if tail_sms is set, 2 if system is set too (0: defaults) */
  int tail_sms;             /* SMs reserved for the longest orbits of a large longest-first
                               batch, one warp each (-1: default 1, 0: none) */
  int system;               /* GALPY_CUDA_SYS_* (size_ext >= 2; default the orbit); SOS runs
                               are float64, rk4/rk6/dopr54/dop853, w0 rows of 7 (3D) or 5
                               (planar) */
} galpy_cuda_launch;

int galpy_cuda_integrate_device(const galpy_cuda_launch *launch);

/* Same integration as galpy_cuda_integrate_device, for callers that must not
 * let a library allocate device memory while they run (an allocation can
 * synchronise the device or grow a pool the application sized for itself).
 * No counterpart in the reference.  It calls no cudaMalloc/cudaFree or other
 * allocating routine: its scratch (work-stealing counter, abort word and a
 * bucketed longest-first work queue) lives in a fixed ~5 MiB array compiled
 * into the library, held by every GPU that loads it until the process exits.
 * Limit: at most 1,048,576 orbits per call (GALPY_CUDA_ERR_ARG beyond that;
 * split the batch).  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress), and so does the first call after the
 * device's context was reset (cudaDeviceReset); make those calls before any
 * stream capture.  The launch shape (grid, shared-memory carveout, SMs
 * reserved for the longest orbits) is that of galpy_cuda_integrate_device;
 * only the longest-first order differs in detail (64 cost buckets instead of
 * a sort).  Every call reuses the same array (the control words are cleared
 * at the start of each call), so calls that overlap on the GPU -- on
 * different streams or from different threads -- race: serialise them. */
int galpy_cuda_integrate_device_noalloc(const galpy_cuda_launch *launch);

/* Energies E = v^2/2 + Phi(x) of n stored rectangular states on the device
 * (galpy's Orbit.E for these potentials, galpy/orbit/Orbits.py:2902):
 * component k of orbit i at w[i*orbit_stride + k*comp_stride]; group as in
 * galpy_cuda_launch.  Asynchronous on `stream`.  The bulge term needs
 * alpha < 2. */
int galpy_cuda_energy_device(const void *comps, int ncomp, const int *group, int planar,
                             const double *w, long long n, long long comp_stride,
                             long long orbit_stride, double *E, void *stream);

/* The Jacobi integral J = v^2/2 + Phi(x) - Omega . (x cross v) of n stored
 * rectangular states on the device (galpy's Orbit.Jacobi, E - OmegaP . L,
 * galpy/orbit/Orbits.py:3298-3375), states and group as in
 * galpy_cuda_energy_device; omega: host double[3], the pattern-speed vector
 * (planar states use its z component).  Omega = 0 gives the energy.
 * Asynchronous on `stream`. */
int galpy_cuda_jacobi_device(const void *comps, int ncomp, const int *group, int planar,
                             const double *w, long long n, long long comp_stride,
                             long long orbit_stride, const double *omega, double *J,
                             void *stream);

/* Orbits between their stored rows (galpy's Orbit.__call__ at times that are
 * not integration times, galpy/orbit/Orbits.py:6460-6575, through the
 * interpolants of _setupOrbitInterp, :6739-6830): per orbit and component --
 * x = R cos(phi), y = R sin(phi) in place of R and phi -- the interpolating
 * cubic spline through the rows with not-a-knot ends (FITPACK's s = 0, k = 3
 * spline, which galpy's InterpolatedUnivariateSpline / RectBivariateSpline
 * evaluate; degree nt - 1 below 4 rows), then R = sqrt(x^2 + y^2), phi =
 * atan2(y, x).  nv 6 (R,vR,vT,z,vz,phi) or 4 (R,vR,vT,phi); rows [n][nt][nv]
 * (galpy's result layout); t [nt] or [n][nt] (indiv_t), increasing; tq [nq]
 * or [n][nq] (indiv_q); out [n][nq][nv].  Queries outside [t_0, t_end]
 * extrapolate the end pieces (galpy refuses them before it interpolates).
 * Device pointers, asynchronous on `stream`; scratch of 2*n*nt*nv doubles
 * (n*nt*nv below 4 rows; plus n*nt with per-orbit times) allocated
 * stream-ordered on it from the library's private memory pool (kept for the
 * next call; galpy_cuda_trim_memory returns it). */
int galpy_cuda_orbit_interp_device(int nv, long long n, int nt, const double *t, int indiv_t,
                                   const double *rows, int nq, const double *tq, int indiv_q,
                                   double *out, void *stream);

/* ---------------------------------------------------------------------------
 * Gradients of a loss on final states (reverse mode).  No counterpart in the
 * reference: galpy's gradient information is the variational integration
 * (integrate_dxdv, integratePlanarOrbit.c:940), one tangent vector per input
 * direction; these entry points give dL/d(initial state) and
 * dL/d(potential parameters) of a scalar loss L(y(T)) with one backward
 * sweep per orbit.
 *
 * The forward pass is galpy's DOP853 (the same step sequence as
 * odeint_type 6, y(T) from its dense output) from t0 to tend.  It saves the
 * state every 64 accepted steps together with those steps' sizes
 * (checkpoints).  The backward pass recomputes each 64-step segment from its
 * checkpoint with the recorded step sizes and applies the exact adjoint of
 * the Runge-Kutta stages with the step sizes held fixed (the discrete adjoint
 * of the forward map).  All arrays are device memory
 * owned by the caller; the calls are asynchronous on `stream` and allocate
 * nothing.  nv = 4 (planar: x, y, vx, vy) or 6 (x, y, z, vx, vy, vz).
 *
 * Differentiable parameters, per component in pot_type order (the pot_args
 * index of each: galpy_cuda_adjoint_params):
 *   15 PowerSphericalwCutoff: amp, rc;  5 MiyamotoNagai: amp, a, b;
 *   9 NFW: amp, a;  8 Hernquist: amp, a;  0 LogarithmicHalo: amp, q, core^2.
 * ------------------------------------------------------------------------- */
typedef struct galpy_cuda_adjoint {
  int size;                 /* sizeof(galpy_cuda_adjoint) */
  int planar;
  long long nobj;
  double t0, tend;          /* integration interval, shared by all orbits */
  double rtol, atol;        /* natural logarithms, as galpy passes them */
  long long max_attempts;   /* per-orbit attempt budget, 0 = unlimited */
  const void *comps;        /* galpy_cuda_compile_potential records (device) */
  int ncomp;
  const int *group;         /* [nobj] group of each orbit, or NULL */
  int signature;            /* galpy_cuda_signature(pot_type) */
  const double *w0;         /* [nv][nobj] initial rectangular states */
  double *yT;               /* [nv][nobj] out (forward, replay): states at tend */
  long long *nsteps;        /* [nobj] accepted steps: out of forward, in of replay/backward */
  int *err;                 /* [nobj] status: out of forward (0 ok, 2 budget or
                               checkpoint capacity exhausted, 3 non-finite), in of backward */
  double *ckpt;             /* [ckpt_cap][nv+1+64][nobj] checkpoints (segment start state and
                               its 64 step sizes): out of forward, in of backward */
  int ckpt_cap;             /* checkpoints per orbit: at most 64*ckpt_cap steps */
  double *hrec;             /* [hcap][nobj] accepted step sizes: optional out of forward,
                               in of replay; NULL to skip */
  long long hcap;
  const double *gyT;        /* [nv][nobj] dL/dy(tend) (backward) */
  double *gw0;              /* [nv][nobj] out (backward): dL/dw0 */
  double *gparam;           /* [nparam][nobj] out (backward): per-orbit dL/dparam, or NULL */
  void *stream;             /* cudaStream_t */
  int block_size;           /* 0 = default */
  const int *order;         /* optional [nobj] permutation: thread j takes orbit order[j]
                               (e.g. orbits by decreasing nsteps for the backward pass,
                               so that the lanes of a warp have similar work), or NULL */
  int variant;              /* backward register budget: 0 compiler default, 1 capped for
                               occupancy (at most 128 registers a thread) */
} galpy_cuda_adjoint;

/* Forward pass: yT, nsteps, err, checkpoints (and hrec if set). */
int galpy_cuda_adjoint_forward(const galpy_cuda_adjoint *a);

/* Backward pass: gw0 and gparam for gyT, from the forward pass's nsteps, err
 * and checkpoints (same w0 interval, tolerances and potential).  Orbits with
 * err != 0 get NaN gradients. */
int galpy_cuda_adjoint_backward(const galpy_cuda_adjoint *a);

/* The forward map with frozen steps: yT from w0 with the nsteps[i] step
 * sizes in hrec (the function the backward pass differentiates exactly;
 * finite differences of it check the gradients). */
int galpy_cuda_adjoint_replay(const galpy_cuda_adjoint *a);

/* Number of differentiable parameters of a component list (>= 0), or
 * GALPY_CUDA_ERR_POTENTIAL; arg_index (may be NULL) receives the pot_args
 * index of each parameter.  pot_args (may be NULL) is needed where a
 * component's argument count depends on its arguments (the ellipsoidal
 * types); without it such lists return GALPY_CUDA_ERR_POTENTIAL.  A rotated
 * ellipsoidal component also returns GALPY_CUDA_ERR_POTENTIAL: the tidal
 * tensor follows the reference's second derivatives, which ignore the
 * rotation, so the adjoint's gradients would not be those of its force.
 * (ABI 2 added pot_args.) */
int galpy_cuda_adjoint_params(int planar, int npot, const int *pot_type, const double *pot_args,
                              int *arg_index);

/* Accelerations at n points (positions SoA [3][n] device memory, z ignored
 * when planar) written to acc [3][n], with the integrators' own force code
 * (galpy's evaluateRforces/zforces in Cartesian form; the acceleration that
 * evalRectForce, integrateFullOrbit.c:1307, hands to the steppers).
 * signature GALPY_CUDA_SIG_MW14 selects the compile-time MWPotential2014
 * path of the integration kernels; precision as galpy_cuda_opts.
 * Asynchronous on `stream`. */
int galpy_cuda_accel_device(const void *comps, int ncomp, const int *group, int planar,
                            int signature, int precision, const double *pos, long long n,
                            double *acc, void *stream);

/* Diagnostic: measured float64 fused-multiply-add throughput of the current
 * device in TFLOP/s (2 flops per FMA), the roofline denominator of the
 * integration kernels. */
int galpy_cuda_fp64_peak(double *tflops, double *ms);

/* Version, last error message of this thread, device count. */
int galpy_cuda_abi_version(void);
const char *galpy_cuda_last_error(void);
int galpy_cuda_device_count(void);

/* Device memory of the blocking (host-pointer) entry points.  They allocate
 * their buffers stream-ordered from a memory pool private to this library
 * (one per device), which keeps freed memory cached for the next call
 * instead of unmapping and mapping it again each time; the caller's own
 * allocators, the device's default memory pool included, are left as they
 * are.  This returns the cached memory of `device` (-1: every device) to
 * the driver; it synchronises those devices.  No counterpart in the
 * reference (galpy's C allocates host memory only). */
int galpy_cuda_trim_memory(int device);

#ifdef __cplusplus
}
#endif
#endif /* GALPY_CUDA_H */
