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

// Surface of section (integrateFullOrbit_sos, integratePlanarOrbit_sos): the
// RK-type machines on the 7-D (3D) or 5-D (planar) system, float64, any
// potential.
template <class SYS, int D>
static KernelInfo pick_sos_system(int method, int variant)
{
  switch (method) {
    case M_RK4: return info_of<RKMachine<D, false, 4, SYS>, D, PREC_FP64, false, DynPot>(variant);
    case M_RK6: return info_of<RKMachine<D, false, 6, SYS>, D, PREC_FP64, false, DynPot>(variant);
    case M_DOPR54:
      return info_of<Dopr54Machine<D, false, SYS>, D, PREC_FP64, false, DynPot>(variant);
    case M_DOP853:
      return info_of<Dop853Machine<D, false, SYS>, D, PREC_FP64, false, DynPot>(variant);
  }
  return KernelInfo();
}

KernelInfo pick_kernel_sos(int method, int variant, int system)
{
  switch (system) {
    case GALPY_CUDA_SYS_SOS: return pick_sos_system<SosSystem, 3>(method, variant);
    case GALPY_CUDA_SYS_SOS_PLANAR_X: return pick_sos_system<PlanarSosSystem<0>, 2>(method, variant);
    case GALPY_CUDA_SYS_SOS_PLANAR_Y: return pick_sos_system<PlanarSosSystem<1>, 2>(method, variant);
  }
  return KernelInfo();
}

}  // namespace gpc
