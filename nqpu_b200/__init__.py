"""B200-native statevector engine: a drop-in for the circuit-run path of
nQPU's Rust statevector backend (QuantumState / GateOperations / C FFI).

The compute path is the CUDA library `libnqpu_b200.so` (sm_100a); this package
is its Python binding.  Importing the package does not touch the GPU; creating a
StateVector without a CUDA device raises.
"""
from ._lib import NqpuErrorException, load  # noqa: F401
from .circuits import brickwork, hea, hea_batch, serving_mix, tfim_trotter  # noqa: F401
from .state import Circuit, StateVector  # noqa: F401

__all__ = ["StateVector", "Circuit", "load", "NqpuErrorException", "brickwork", "tfim_trotter",
           "hea", "hea_batch", "serving_mix"]
