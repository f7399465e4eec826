"""B200-native GEMINI frequency-wavenumber hot path.

Radial ODE solves per (omega, l) on an FP64 persistent CUDA kernel, degree sums
and the batched inverse FFT to seismograms, behind a C ABI
(``include/gemini_fk.h``).  This package holds the host-side mirror of the
reference's interfaces (earth model, external nodes, frequency grid) and the
ctypes binding of the CUDA library.
"""
from .model import (ExternalRadialNodes, FKParams, FrequencyGrid, GeminiError, NodeEarthModel,
                    frequency_grid, load_node_model, nsp_for)

__all__ = ["ExternalRadialNodes", "FKParams", "FrequencyGrid", "GeminiError", "NodeEarthModel",
           "frequency_grid", "load_node_model", "nsp_for"]
