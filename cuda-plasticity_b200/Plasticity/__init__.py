"""Drop-in facades of the reference Plasticity package (filled in below)."""
