"""Host-side helpers shared by the propagator (src/shared/ of the reference)."""
