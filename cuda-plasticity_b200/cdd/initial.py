"""Seeded Gaussian-random-field initial conditions for the nine-component plastic distortion.

The workloads this package is measured on are defined by a construction of their own rather than
by the reference's ``GaussianRandomInitializer`` (Plasticity/FieldInitializers/FieldInitializer.py
L153-209, which always draws at 128^d and Fourier-resamples). The construction here is:

1. each of the 9 components is i.i.d. N(0, 1) per cell, drawn from ``numpy.random.default_rng(seed)``
   as one array of shape ``(9,) + shape`` (component order xx, xy, xz, yx, yy, yz, zx, zy, zz);
2. each component is Fourier-filtered by ``exp(-|k|^2 s^2 / 2)`` with ``k_d = 2 pi m_d`` for the
   wrapped integer index ``m_d`` in ``[-n_d/2, n_d/2)`` (box length 1) and ``s = sigma`` in box units;
3. the whole field is rescaled so that its rms over all components and cells is ``rms``.

The result is FP64, laid out ``[component][axis0][axis1][(axis2)]`` with the last axis contiguous,
which is the numpy C order of the reference's per-component ``GridArray``.
"""
import numpy as np


def gaussian_random_field(shape, sigma, rms=0.05, seed=0):
    """Return a float64 array of shape ``(9,) + shape``; see the module docstring."""
    shape = tuple(int(n) for n in shape)
    if len(shape) not in (2, 3):
        raise ValueError("grid must be 2-D or 3-D, got shape %r" % (shape,))
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((9,) + shape)
    axes = tuple(range(1, len(shape) + 1))
    spec = np.fft.rfftn(white, axes=axes)
    ksq = np.zeros(spec.shape[1:])
    for d, n in enumerate(shape):
        if d == len(shape) - 1:
            m = np.arange(n // 2 + 1, dtype=np.float64)
        else:
            m = np.fft.fftfreq(n) * n
        k = 2.0 * np.pi * m
        view = [1] * len(shape)
        view[d] = k.size
        ksq = ksq + (k * k).reshape(view)
    spec *= np.exp(-0.5 * ksq * sigma * sigma)
    field = np.fft.irfftn(spec, s=shape, axes=axes)
    field *= rms / np.sqrt(np.mean(field * field))
    return np.ascontiguousarray(field)


def gaussian_random_field_torch(shape, sigma, rms=0.05, seed=0, device="cuda", dtype=None):
    """The same construction drawn with torch's generator on ``device`` (fast at 256^3).

    The white noise comes from ``torch.Generator`` rather than numpy, so the field differs from
    ``gaussian_random_field`` for the same seed; the filter and normalisation are identical.
    Used to build large synthetic inputs without a host round trip.
    """
    import torch
    shape = tuple(int(n) for n in shape)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    white = torch.randn((9,) + shape, generator=gen, device=device, dtype=torch.float64)
    dims = tuple(range(1, len(shape) + 1))
    spec = torch.fft.rfftn(white, dim=dims)
    del white
    ksq = torch.zeros(spec.shape[1:], dtype=torch.float64, device=device)
    for d, n in enumerate(shape):
        if d == len(shape) - 1:
            m = torch.arange(n // 2 + 1, dtype=torch.float64, device=device)
        else:
            m = torch.fft.fftfreq(n, device=device, dtype=torch.float64) * n
        k = 2.0 * np.pi * m
        view = [1] * len(shape)
        view[d] = k.numel()
        ksq = ksq + (k * k).reshape(view)
    spec *= torch.exp(-0.5 * ksq * sigma * sigma)
    field = torch.fft.irfftn(spec, s=shape, dim=dims)
    del spec
    field *= rms / torch.sqrt(torch.mean(field * field))
    return field.contiguous() if dtype is None else field.to(dtype).contiguous()
