"""sloth_b200: SLOTH's ray-propagation hot path on NVIDIA B200 (sm_100a).

Python host code mirrors SLOTH's core.domain / core.beam / core.propagator
API; the compute runs in hand-written CUDA kernels in libsloth_b200.so,
called through the C ABI declared in include/sloth_b200.h. There is no CPU
fallback.
"""
__version__ = "0.1.0"
