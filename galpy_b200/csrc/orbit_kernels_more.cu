// galpy_b200/csrc/orbit_kernels_more.cu
//
// Instantiations of the orbit kernel for rk6, symplec6 and dopr54, in a
// translation unit of their own so that the library's kernels compile in
// parallel.
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

}  // namespace gpc
