"""Child process of tests/test_gpu_interrupt.py (TEST ONLY).

Runs one long blocking integration through the galpy-facing wrapper and
reports how it ended; the parent sends SIGINT while the kernel runs.  The
same pattern as the reference's tests/orbitint4sigint.py driven by
test_orbit_c_sigint_full / _planar (tests/test_orbit.py:12211-12420).

usage: python sigint_child.py <method> full|planar [split]

With `split` the call spreads its orbits over two ranges on device 0
(devices=[0, 0]), whose threads the calling thread's handler stops.
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def main():
    import galpy_b200 as gb
    from galpy_b200 import potentials
    from helpers import seeded_ics

    method, kind = sys.argv[1], sys.argv[2]
    devices = [0, 0] if len(sys.argv) > 3 and sys.argv[3] == "split" else None
    planar = kind == "planar"
    pot = potentials.MWPotential2014()
    fn = gb.integratePlanarOrbit_cuda if planar else gb.integrateFullOrbit_cuda
    # warm-up: CUDA context, module load and memory pool outside the timed call
    ics = seeded_ics(64, 3, planar=planar)
    fn(pot, ics.copy(), np.linspace(0, 1, 3), method, progressbar=False)
    n = 1 << 16
    ics = seeded_ics(n, 4, planar=planar)
    t = np.array([0.0, 1.0e4])
    print("Starting long integration ...", flush=True)
    t0 = time.time()
    try:
        fn(pot, ics, t, method, progressbar=False, dt=0.001 if "dop" not in method else None,
           devices=devices)
    except KeyboardInterrupt:
        print(f"KeyboardInterrupt after {time.time() - t0:.3f} s", flush=True)
        return 0
    print(f"completed after {time.time() - t0:.3f} s", flush=True)
    return 5


if __name__ == "__main__":
    sys.exit(main())
