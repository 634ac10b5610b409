// galpy_b200/csrc/compile_potential.h
//
// Host-side "potential compiler": turns galpy's flat (pot_type, pot_args)
// stream (as built by galpy/orbit/integrateFullOrbit.py:43-614 and
// integratePlanarOrbit.py:33-663, decoded in C by
// integrateFullOrbit.c:69-1040 / integratePlanarOrbit.c:55-742) into the
// device records of potentials.cuh, with every per-component constant
// precomputed once per call instead of once per force evaluation.
#pragma once
#include <math.h>
#include <string.h>

#include "potentials.cuh"

namespace gpc {

// number of galpy arguments of a supported type (3D PowerSphericalwCutoff
// carries two extra cache slots, integrateFullOrbit.py:178-180)
inline int galpy_nargs(int type, int planar)
{
  switch (type) {
    case T_LOGHALO: return 4;
    case T_MN: return 3;
    case T_HERNQUIST: return 2;
    case T_NFW: return 2;
    case T_PSWC: return planar ? 3 : 5;
    default: return -1;
  }
}

// Compile one group.  Returns 0, -3 (unsupported type) or -1 (bad args).
// *consumed receives the number of pot_args read.
inline int compile_group(int planar, int npot, const int* pot_type, const double* pot_args,
                         GpComp* out, int* consumed)
{
  if (npot < 1 || npot > kMaxComp) return -1;
  const double* p = pot_args;
  for (int k = 0; k < npot; k++) {
    const int type = pot_type[k];
    const int na = galpy_nargs(type, planar);
    if (na < 0) return -3;
    GpComp c;
    memset(&c, 0, sizeof(c));
    c.type = type;
    const double amp = p[0];
    c.c[0] = amp;
    switch (type) {
      case T_PSWC: {
        const double alpha = p[1], rc = p[2];
        const double a = 1.5 - 0.5 * alpha;
        if (!(a > 0.0) || !(rc > 0.0)) return -1;
        c.c[1] = 1.0 / (rc * rc);
        c.c[2] = a;
        c.c[3] = lgamma(a);
        c.c[4] = 2.0 * M_PI * pow(rc, 3.0 - alpha) * tgamma(a);
        c.c[5] = -0.5 * alpha;
        c.c[6] = 4.0 * M_PI;
        c.c[7] = alpha;
        for (int n = 1; n <= kSeriesTerms; n++) c.inv_ap[n - 1] = 1.0 / (a + n);
        break;
      }
      case T_MN:
        c.c[1] = p[1];
        c.c[2] = p[2] * p[2];
        break;
      case T_HERNQUIST:
      case T_NFW:
        if (!(p[1] > 0.0)) return -1;
        c.c[1] = p[1];
        c.c[2] = 1.0 / p[1];
        break;
      case T_LOGHALO: {
        const double q = p[1], core2 = p[2], om = p[3];
        if (!(q > 0.0)) return -1;
        c.c[1] = 1.0 / (q * q);
        c.c[2] = core2;
        // galpy passes 1 - 1/b^2 for a triaxial halo and 2.0 (> 1) when
        // axisymmetric (integrateFullOrbit.py:69-73)
        const bool tri = om < 1.0;
        c.c[3] = tri ? 1.0 - om : 1.0;
        c.c[4] = tri ? 1.0 : 0.0;
        break;
      }
    }
    out[k] = c;
    p += na;
  }
  if (consumed) *consumed = (int)(p - pot_args);
  return 0;
}

}  // namespace gpc
