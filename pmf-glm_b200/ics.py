"""Seeded synthetic turbulent boxes for the benchmark workloads (host-side, not timed).

The reference's only random initial condition is a Batchelor magnetic field from a random
vector potential over uniform gas (lib/MHDKernels/src/pmf.jl:300-591): B = i s(k) x A(k)
with the centred-difference symbol s_d = sin(k_d dx)/dx (pmf.jl:426-428), a power-law
amplitude and a cutoff, normalised to a target rms. This module keeps that convention for
B and adds Gaussian-random-field density and velocity:

  * density  rho = 1 + sigma*g (or exp(sigma*g - sigma^2/2)), g a unit-variance GRF with
    P(k) ~ k^-2 cut at |m| > kcut_rho (m the integer mode vector);
  * velocity three independent GRFs of the same spectrum scaled to rms |v| = mach * c_s,
    with c_s = 1 for the mean state (p0 = rho_mean c_s^2 / gamma);
  * vector potential A white in k with amplitude |m|^((n-2)/2), sharp cutoff at |m| = kc,
    so that P_B(k) ~ k^n; B scaled to plasma beta = 2 p0 / <B^2>.

Cell B (GLM) is the centred curl of the cell-centred A; CT faces are the staggered curl of
the same A read as an edge-centred potential (ct.jl:310-345 semantics). Random numbers come
from numpy's PCG64 generator seeded per field (seed, seed+1, ...), so a box is reproducible
from (N, seed) alone.
"""
from __future__ import annotations

import numpy as np

try:
    import scipy.fft as _fft

    def _rfftn(a):
        return _fft.rfftn(a, workers=-1)

    def _irfftn(a, s):
        return _fft.irfftn(a, s=s, workers=-1)
except ImportError:  # pragma: no cover
    def _rfftn(a):
        return np.fft.rfftn(a)

    def _irfftn(a, s):
        return np.fft.irfftn(a, s=s)

from problems import prim2cons


def _modes(n):
    """Integer mode numbers (mz, my, mx) on the rfft grid of an n^3 box, axes (z, y, x)."""
    m = np.fft.fftfreq(n, 1.0 / n)
    mx = np.arange(n // 2 + 1, dtype=np.float64)
    return np.meshgrid(m, m, mx, indexing="ij", sparse=True)


def grf(n, seed, index=-2.0, kcut=None):
    """Unit-variance Gaussian random field with P(k) ~ |m|^index, sharp cut at |m| > kcut."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((n, n, n))
    mz, my, mx = _modes(n)
    k = np.sqrt(mx * mx + my * my + mz * mz)
    amp = np.where(k > 0, np.power(np.where(k > 0, k, 1.0), index / 2.0), 0.0)
    if kcut is not None:
        amp = np.where(k > kcut, 0.0, amp)
    f = _irfftn(_rfftn(w) * amp, (n, n, n))
    f -= f.mean()
    return f / f.std()


def vector_potential(n, seed, spec_index=2.0, kc=16.0):
    """Three potential components with amplitude |m|^((n_B-2)/2), sharp cutoff at kc."""
    rng = np.random.default_rng(seed)
    mz, my, mx = _modes(n)
    k = np.sqrt(mx * mx + my * my + mz * mz)
    amp = np.where((k > 0) & (k <= kc), np.power(np.where(k > 0, k, 1.0), (spec_index - 2.0) / 2.0), 0.0)
    return [_irfftn(_rfftn(rng.standard_normal((n, n, n))) * amp, (n, n, n)) for _ in range(3)]


def _curl_centred(A, dx):
    """Cell-centred B = centred curl of a cell-centred A; arrays indexed (z, y, x)."""
    Ax, Ay, Az = A
    d = lambda a, ax: (np.roll(a, -1, axis=ax) - np.roll(a, 1, axis=ax)) / (2 * dx)
    return [d(Az, 1) - d(Ay, 0), d(Ax, 0) - d(Az, 2), d(Ay, 2) - d(Ax, 1)]


def _curl_staggered(A, dx):
    """Lower-face B = staggered curl of an edge-centred A (ct.jl:310-320)."""
    Ax, Ay, Az = A
    d = lambda a, ax: (np.roll(a, -1, axis=ax) - a) / dx
    return [d(Az, 1) - d(Ay, 0), d(Ax, 0) - d(Az, 2), d(Ay, 2) - d(Ax, 1)]


def turbulent_box(n, seed=0, mach=0.5, beta=1.0, rho_sigma=0.1, lognormal=False, kcut_rho=None,
                  b_index=2.0, kc=16.0, gamma=5.0 / 3.0, with_ct=False, dtype=np.float32):
    """Conserved SoA fields (9, n^3) of a periodic unit box, dx = 1/n.

    Seeds: seed (density), seed+1..seed+3 (velocity components), seed+4 (potential).
    Returns ``{"U": ..., "A_edge": (3, n^3) or None, "faces": (3, n^3) or None, "p0": p0}``;
    with ``with_ct`` the cell B and E of ``U`` are the CT face average and its energy.
    """
    dx = 1.0 / n
    kcut_rho = n / 4 if kcut_rho is None else kcut_rho
    g = grf(n, seed, -2.0, kcut_rho)
    rho = np.exp(rho_sigma * g - 0.5 * rho_sigma ** 2) if lognormal else 1.0 + rho_sigma * g
    p0 = 1.0 / gamma  # rho_mean = 1, c_s = 1
    v = [grf(n, seed + 1 + c, -2.0, kcut_rho) for c in range(3)]
    vrms = np.sqrt(sum((vc ** 2).mean() for vc in v))
    v = [vc * (mach / vrms) for vc in v]
    A = vector_potential(n, seed + 4, b_index, kc)
    target_b2 = 2.0 * p0 / beta
    if with_ct:
        F = _curl_staggered(A, dx)
        bc = [0.5 * (F[0] + np.roll(F[0], -1, axis=2)), 0.5 * (F[1] + np.roll(F[1], -1, axis=1)),
              0.5 * (F[2] + np.roll(F[2], -1, axis=0))]
        scale = np.sqrt(target_b2 / sum((b ** 2).mean() for b in bc))
        faces = np.stack([f.ravel() * scale for f in F]).astype(dtype)
        A_edge = np.stack([a.ravel() * scale for a in A]).astype(dtype)
        B = [b * scale for b in bc]
    else:
        B = _curl_centred(A, dx)
        scale = np.sqrt(target_b2 / sum((b ** 2).mean() for b in B))
        B = [b * scale for b in B]
        faces = None
        A_edge = None
    q = np.stack([rho.ravel(), v[0].ravel(), v[1].ravel(), v[2].ravel(), np.full(n ** 3, p0),
                  B[0].ravel(), B[1].ravel(), B[2].ravel(), np.zeros(n ** 3)])
    U = prim2cons(q, gamma).astype(dtype)
    return {"U": U, "A_edge": A_edge, "faces": faces, "p0": p0}


def batch_mix(nbox=64, seed=2024, sizes=(32, 48, 64, 96, 128), weights=(5, 4, 3, 2, 1)):
    """Box specifications of the batched workload: side lengths drawn from `sizes` with
    uneven weights, plasma beta log-uniform in [0.01, 10], magnetic spectral index
    uniform in [-2.9, 2], cutoff uniform in [N/8, N/3], GLM and CT alternating at random,
    and a seed per box. Deterministic in `seed`."""
    rng = np.random.default_rng(seed)
    p = np.asarray(weights, dtype=np.float64)
    p /= p.sum()
    specs = []
    for i in range(nbox):
        n = int(rng.choice(sizes, p=p))
        specs.append({"n": n, "beta": float(10 ** rng.uniform(-2.0, 1.0)), "b_index": float(rng.uniform(-2.9, 2.0)),
                      "kc": float(rng.uniform(n / 8, n / 3)), "seed": int(seed + 101 * i),
                      "ct": bool(rng.integers(0, 2))})
    return specs
