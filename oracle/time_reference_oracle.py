"""Recipe: time one 64^3 step of the reference's own pure-Python oracles.

    FLUXFX_SOURCE=/path/to/FluxFX_Source python oracle/time_reference_oracle.py [n]

One step = ``thermal_reference.step`` (semi-Lagrangian velocity and scalar
transport + buoyancy; ``fluxfx/physics/thermal_reference.py:22-32``) followed
by ``pressure_reference.project`` with its default 80 Jacobi iterations
(``fluxfx/physics/pressure_reference.py:90-97``) -- the reference's CPU
restatement of its step, on one host thread. It needs the reference checkout,
so it runs only where that is present; the printed JSON is a measurement
recorded beside the CPU baseline, not a product path.
"""
import json
import os
import sys
import time
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))


def main(n=64):
    from oracle.glsl_ref.build import REFERENCE_CHECKOUT
    sys.path.insert(0, str(REFERENCE_CHECKOUT))
    from fluxfx.physics import pressure_reference, thermal_reference
    from fluxfx.physics.config import GridSpec
    from fluxfx.physics.thermal import ThermalSettings
    import random
    grid = GridSpec((n, n, n))
    settings = ThermalSettings(thermal_lift=1.0, density_weight=0.05)
    rnd = random.Random(0)
    vel = [[rnd.uniform(-1e-3, 1e-3) for _ in range(s[0] * s[1] * s[2])] for s in grid.face_shapes]
    cells = n * n * n
    dens = [0.0] * cells
    temp = [0.0] * cells
    t0 = time.perf_counter()
    dens, temp, vel = thermal_reference.step(dens, temp, vel, grid, settings, 0.02)
    t1 = time.perf_counter()
    vel, _, _ = pressure_reference.project(vel, grid, 0.02)
    t2 = time.perf_counter()
    print(json.dumps({"n": n, "transport_s": t1 - t0, "projection_s": t2 - t1, "step_s": t2 - t0,
                      "steps_per_s": 1.0 / (t2 - t0), "threads": 1, "host_cpu_count": os.cpu_count()}))


if __name__ == '__main__':
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 64)
