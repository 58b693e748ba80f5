"""molscat_b200: B200-native (sm_100a, FP64) drop-in for the MOLSCAT / BOUND /
FIELD log-derivative propagator hot path (MDPROP / LDPROP).

The compute lives in libmolscat_gpu.so (C ABI: include/molscat_gpu.h); this
package is the host-side mirror of the reference's propagator interface.
"""
from .propagators import (Coupling, Plan, PropagatorError, Segment, hammat_pvec, ldprop, mdprop,
                          propagate, radial_grid)

__all__ = ["Coupling", "Segment", "Plan", "PropagatorError", "mdprop", "ldprop", "propagate",
           "hammat_pvec", "radial_grid"]
