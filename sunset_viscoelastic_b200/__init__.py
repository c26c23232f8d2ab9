"""B200-native LABFM time-step path of SUNSET (viscoelastic): neighbour search, LABFM
weights, stencil operators, viscoelastic right-hand sides and the RK3(2)4[2R+]C step as
CUDA kernels for sm_100a behind a C-ABI (include/sunset_gpu.h).

``labfm.Sunset`` mirrors the reference's subroutines over that C-ABI; ``nodesets`` holds
the IPART format and the synthetic workloads.
"""
from .nodesets import NodeSet, Workload, WORKLOADS, jittered_lattice, read_ipart, write_ipart, initial_state  # noqa: F401

__all__ = ["NodeSet", "Workload", "WORKLOADS", "jittered_lattice", "read_ipart", "write_ipart", "initial_state"]
