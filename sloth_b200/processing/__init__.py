"""Post-processing of traced rays on the GPU (the reference's src/processing)."""
