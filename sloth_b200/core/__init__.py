"""core.domain / core.beam / core.propagator of SLOTH, on B200 kernels."""
