// galpy_b200/csrc/orbit_kernels_prec.cu
//
// Instantiations of the orbit kernel in the mixed-precision forms beside the
// plain float64 and the FP32-force / float64-state ones, for the
// MWPotential2014 component list (the configurations that specify mixed
// precision), in a translation unit of their own so that they compile in
// parallel with the rest:
//
//   GALPY_CUDA_F64_TAIL32    float64 force with the high-order terms of its
//                            table polynomials in float32 (force error
//                            ~1e-11 relative); leapfrog, symplec4, rk4,
//                            dop853
//   GALPY_CUDA_F32BULGE      as F64_TAIL32, with the bulge term in float32;
//                            leapfrog, symplec4, rk4, dop853
//   GALPY_CUDA_F32FORCE_DF   float32 force with a double-float (two-float)
//                            compensated state; leapfrog, symplec4
//
// Plain orbits only (no variational or surface-of-section runs).
#include "orbit_kernel.cuh"

namespace gpc {

template <int MIX>
struct MixedMethods {
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

struct DFStateMethods {
  template <int D, int PREC, bool VAR, class POT>
  static KernelInfo pick(int method, int variant)
  {
    switch (method) {
      case M_LEAPFROG:
        return info_of<SymplecticMachine<D, VAR, 2, DFloat>, D, PREC, VAR, POT>(variant);
      case M_SYMPLEC4:
        return info_of<SymplecticMachine<D, VAR, 4, DFloat>, D, PREC, VAR, POT>(variant);
    }
    return KernelInfo();
  }
};

template <int MIX>
static KernelInfo pick_mixed(int planar, int method, int variant, bool direct)
{
  using Set = MixedMethods<MIX>;
  if (direct)
    return pick_plain<Set, PREC_FP64, MW14MixedPot<true, MIX>>(planar, method, variant);
  return pick_plain<Set, PREC_FP64, MW14MixedPot<false, MIX>>(planar, method, variant);
}

KernelInfo pick_kernel_prec(int planar, int var, int prec, int method, int sig, int variant,
                            bool direct)
{
  if (var || sig != GALPY_CUDA_SIG_MW14) return KernelInfo();
  switch (prec) {
    case GALPY_CUDA_F64_TAIL32: return pick_mixed<MIX_TAIL32>(planar, method, variant, direct);
    case GALPY_CUDA_F32BULGE: return pick_mixed<MIX_F32BULGE>(planar, method, variant, direct);
    case GALPY_CUDA_F32FORCE_DF:
      return direct ? pick_plain<DFStateMethods, PREC_F32, MW14Pot>(planar, method, variant)
                    : pick_plain<DFStateMethods, PREC_F32, MW14GroupPot>(planar, method, variant);
  }
  return KernelInfo();
}

}  // namespace gpc
