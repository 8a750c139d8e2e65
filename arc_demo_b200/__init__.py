"""B200-native batched world step for arc-demo's quadruped environment.

`native.Sim` binds libarcsim.so (built by `arc_demo_b200.build`) with the
reference's `Sim` interface; the library's C ABI is include/arc_sim.h.
"""

from .native import Model, Sim  # noqa: F401
