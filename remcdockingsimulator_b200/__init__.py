"""B200-native replica-exchange Monte Carlo engine for rigid-body docking of
residue-level protein chains among crowders.

The hot path (pair energy, dE, Metropolis sweep, replica exchange) runs in
hand-written sm_100a CUDA kernels behind the C ABI of include/remc_b200.h;
this package holds the host-side model, file formats and Python bindings.
"""
__version__ = "0.1.0"
