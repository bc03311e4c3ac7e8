"""Drop-in facades of the reference's ``Plasticity`` package (mattbierbaum/cuda-plasticity).

Module paths, class names, signatures and defaults follow the reference so that RunPython-style
drivers run unchanged; the time step, flux and stress are computed by libcdd.so on the GPU
(package ``cdd``). Host-side helpers (field algebra, k tables, raw file I/O) are plain numpy.
"""
