"""Initial primitive fields (rho, u, v, w, p) on an interior-only periodic box.

Every generator returns a float64 array of shape ``(5, nz, ny, nx)`` (x fastest,
the reference's ``idx3`` order without ghosts), ready for
``Solver.upload_primitive`` -- the equivalent of the reference's
``initialize_*`` + ``apply_boundary`` + ``primitiveToConserved`` sequence
(main.cpp:67-71).

The reference has no Taylor-Green initializer and its isotropic generator
hard-codes k0 = 8 and an amplitude (isotropic_ini.cpp:34-35); the generators
here are parameterised restatements of the formulas the workloads name.
"""
from __future__ import annotations

import math

import numpy as np


def grid_coords(n: int, L: float = 2.0 * math.pi, x0: float = 0.0) -> np.ndarray:
    """Node positions x_i = x0 + i*dx with dx = L/n (as initialization.cpp:324 and
    the Tecplot writer's x = x0 + i*dx, output.cpp:62)."""
    return x0 + np.arange(n, dtype=np.float64) * (L / n)


def taylor_green(n: int, gamma: float = 1.4, Ma: float = 0.1, L: float = 2.0 * math.pi,
                 perturb: float = 0.0, seed: int = 0, k0: float = 4.0) -> np.ndarray:
    """Taylor-Green vortex on [0, L)^3:

        rho = 1, u = sin x cos y cos z, v = -cos x sin y cos z, w = 0,
        p = 1/(gamma Ma^2) + (cos 2x + cos 2y)(cos 2z + 2)/16.

    With ``perturb > 0`` a seeded solenoidal random velocity field (spectrum
    peaked at ``k0``) of that rms amplitude is added, as the adjoint workload
    asks ("a seeded 1e-3-amplitude random solenoidal velocity perturbation").
    """
    x = grid_coords(n, L)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    W = np.empty((5, n, n, n))
    W[0] = 1.0
    W[1] = np.sin(X) * np.cos(Y) * np.cos(Z)
    W[2] = -np.cos(X) * np.sin(Y) * np.cos(Z)
    W[3] = 0.0
    W[4] = 1.0 / (gamma * Ma * Ma) + (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0) / 16.0
    if perturb > 0.0:
        du = solenoidal_field(n, k0=k0, seed=seed)
        rms = math.sqrt(float(np.mean(du[0] ** 2 + du[1] ** 2 + du[2] ** 2)) / 3.0)
        W[1:4] += du * (perturb / rms)
    return W


def solenoidal_field(n: int, k0: float = 4.0, seed: int = 12345) -> np.ndarray:
    """Random-phase solenoidal velocity field with E(k) ~ k^4 exp(-2 (k/k0)^2).

    Follows generate_full_turbulence (isotropic_ini.cpp:42-122): per mode an
    amplitude sqrt(2/3) sqrt(kk exp(-2 kk/k0^2) / 4pi) (kk = |k|^2), three random
    phases, projection onto the plane normal to k (u_k - k (k.u_k)/kk), inverse
    complex transform, real part. The phases come from a seeded numpy generator
    instead of a fixed-seed mt19937_64, and k0 is a parameter. Returns
    (3, n, n, n) with unit-free amplitude; callers rescale.
    """
    rng = np.random.default_rng(seed)
    phases = 2.0 * math.pi * rng.random((3, n, n, n))   # the one random draw
    try:
        import torch
        use_gpu = n >= 128 and torch.cuda.is_available()
    except Exception:  # torch is optional here
        use_gpu = False
    if use_gpu:
        xp = torch
        dev = "cuda"
        a = torch.from_numpy(phases).to(dev)
        k = torch.fft.fftfreq(n, 1.0 / n, dtype=torch.float64, device=dev)
    else:
        xp = np
        a = phases
        k = np.fft.fftfreq(n, 1.0 / n)
    K1 = k.reshape(1, 1, n)
    K2 = k.reshape(1, n, 1)
    K3 = k.reshape(n, 1, 1)
    kk = K1 * K1 + K2 * K2 + K3 * K3
    kk_safe = xp.where(kk == 0, xp.ones_like(kk), kk)
    Ak = math.sqrt(2.0 / 3.0) * xp.sqrt(kk * xp.exp(-2.0 * kk / (k0 * k0)) / (4.0 * math.pi))
    vr = Ak * xp.sin(a)
    vi = Ak * xp.cos(a)
    del a
    vkr = K1 * vr[0] + K2 * vr[1] + K3 * vr[2]
    vki = K1 * vi[0] + K2 * vi[1] + K3 * vi[2]
    out = np.empty((3, n, n, n))
    for c, Kc in enumerate((K1, K2, K3)):
        re = Kc * vkr / kk_safe - vr[c]
        im = Kc * vki / kk_safe - vi[c]
        zero = kk == 0
        if use_gpu:
            spec = torch.complex(torch.where(zero, 0.0, re), torch.where(zero, 0.0, im))
            out[c] = torch.fft.ifftn(spec).real.cpu().numpy()
        else:
            spec = np.where(zero, 0.0, re + 1j * im)
            out[c] = np.fft.ifftn(spec).real
    return out


def isotropic(n: int, mach_t: float, Ma: float, gamma: float = 1.4, k0: float = 4.0,
              seed: int = 12345, L: float = 2.0 * math.pi) -> np.ndarray:
    """Decaying isotropic turbulence: rho = 1, T = 1 (p = Rgas rho T, as
    init_isotropic_turbulence sets it, isotropic_ini.cpp:184-189) and the
    solenoidal field of :func:`solenoidal_field` scaled so that the turbulent Mach
    number sqrt(<|u|^2>) / <c> of compute_turbulence_statistics
    (ana_isotropic.cpp:289) equals ``mach_t``; at T = 1, c = sqrt(gamma Rgas) = 1/Ma.
    """
    del L  # the spectrum is defined on the integer wavenumbers of a 2*pi box
    u = solenoidal_field(n, k0=k0, seed=seed)
    Rgas = 1.0 / (Ma * Ma * gamma)
    c = math.sqrt(gamma * Rgas * 1.0)
    urms_total = math.sqrt(float(np.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2)))
    u *= (mach_t * c) / urms_total
    W = np.empty((5, n, n, n))
    W[0] = 1.0
    W[1:4] = u
    W[4] = Rgas * 1.0 * 1.0
    return W
