// galpy_b200/csrc/orbit_kernels_more.cu
//
// Instantiations of the orbit kernel for rk6, symplec6 and dopr54, and for
// surface-of-section integration, in a translation unit of their own so
// that the library's kernels compile in parallel.
#include "orbit_kernel.cuh"

namespace gpc {

struct MoreMethods {
  template <int D, int PREC, bool VAR, class POT>
  static KernelInfo pick(int method, int variant)
  {
    switch (method) {
      case M_RK6: return info_of<RKMachine<D, VAR, 6>, D, PREC, VAR, POT>(variant);
      case M_SYMPLEC6: return info_of<SymplecticMachine<D, VAR, 6>, D, PREC, VAR, POT>(variant);
      case M_DOPR54: return info_of<Dopr54Machine<D, VAR>, D, PREC, VAR, POT>(variant);
    }
    return KernelInfo();
  }
};

KernelInfo pick_kernel_more(int planar, int var, int prec, int method, int sig, int variant,
                            bool direct)
{
  return pick_kernel_in<MoreMethods>(planar, var, prec, method, sig, variant, direct);
}

// Surface of section (integrateFullOrbit_sos): the RK-type machines on the
// 7-D system, 3D and float64, any potential.
KernelInfo pick_kernel_sos(int method, int variant)
{
  switch (method) {
    case M_RK4: return info_of<RKMachine<3, false, 4, SosSystem>, 3, PREC_FP64, false, DynPot>(variant);
    case M_RK6: return info_of<RKMachine<3, false, 6, SosSystem>, 3, PREC_FP64, false, DynPot>(variant);
    case M_DOPR54:
      return info_of<Dopr54Machine<3, false, SosSystem>, 3, PREC_FP64, false, DynPot>(variant);
    case M_DOP853:
      return info_of<Dop853Machine<3, false, SosSystem>, 3, PREC_FP64, false, DynPot>(variant);
  }
  return KernelInfo();
}

}  // namespace gpc
