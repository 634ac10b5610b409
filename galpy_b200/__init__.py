"""galpy_b200 -- B200-native batched orbit integration for galpy.

The engine (libgalpy_cuda.so, built from galpy_b200/csrc for sm_100a) runs
galpy's C integrators (leapfrog, symplec4, symplec6, rk4, rk6, dopr54,
dop853) -- plain and variational (dxdv) -- in MWPotential2014-type
potentials on the GPU.  Its galpy-facing entry points mirror galpy's own C
wrappers (galpy/orbit/integrateFullOrbit.py, integratePlanarOrbit.py);
``galpy_hooks`` plugs them into ``galpy.orbit.Orbit.integrate`` as the
methods 'leapfrog_cuda', 'symplec4_cuda', 'symplec6_cuda', 'rk4_cuda',
'rk6_cuda', 'dopr54_cuda' and 'dop853_cuda'.

There is no CPU fallback: calls raise CudaLibraryMissing when the library is
not built and CudaError when no GPU is available.
"""
from ._lib import (CudaError, CudaLibraryMissing, MethodNotSupported,  # noqa: F401
                   PotentialNotSupported)
from .integrate import (CUDA_METHODS, accel_device, compile_potential,  # noqa: F401
                        energy_device,
                        integrate_device,
                        integrate_dxdv_batch, integrateFullOrbit_cuda,
                        integrateFullOrbit_sos_cuda, integratePlanarOrbit_sos_cuda,
                        integrateFullOrbit_dxdv_cuda, integratePlanarOrbit_cuda,
                        integratePlanarOrbit_dxdv_cuda, parse_integrator, parse_tol,
                        shard_of, signature, split_orbits)
from .adjoint import final_state  # noqa: F401
from .potentials import (HernquistPotential, LogarithmicHaloPotential,  # noqa: F401
                         MiyamotoNagaiPotential, MWPotential2014, NFWPotential,
                         PowerSphericalPotentialwCutoff, parse_pot)

__version__ = "0.1.0"
