"""NumPy restatement of the reference's initial-condition generators — TEST INFRASTRUCTURE ONLY.

Only the tests use this module, as the checker of the device generators in libpmfmhd.so:

* ``pmf_batchelor_field`` follows lib/MHDKernels/src/pmf.jl:300-591 (with the physical-hash
  realizations of pmf.jl:109-191 and the zero padding of :205-224). The spectral
  coefficients are built with the reference's single-precision complex arithmetic (NumPy
  rounds every operation, as Julia does without @fastmath); the inverse transform is FP64
  (the reference's is FFTW single precision), rounded to FP32.
* ``ct_faces_from_cells`` follows ct.jl:246-308 (FP64, like the reference's host FFTW code)
  and returns the faces and the installed cell field.
"""
from __future__ import annotations

import numpy as np

_U64 = np.uint64


def mix64(x):
    """SplitMix64 output function after a golden-ratio increment (pmf.jl:109-114)."""
    with np.errstate(over="ignore"):
        z = x + _U64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> _U64(30))) * _U64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> _U64(27))) * _U64(0x94D049BB133111EB)
        return z ^ (z >> _U64(31))


def _u64(v):
    return np.asarray(v, dtype=np.int64).astype(np.uint64)


def hash_uniform(seed, qx, qy, qz, comp, lane):
    """pmf.jl:116-128: six SplitMix rounds over (seed, qx, qy, qz, component, lane)."""
    h = mix64(_u64(seed))
    for v in (qx, qy, qz, comp, lane):
        h = mix64(h ^ _u64(v))
    return ((h >> _U64(11)).astype(np.float64) + 0.5) * 2.0 ** -53


def hash_normal(seed, qx, qy, qz, comp, real_only):
    """pmf.jl:130-141: Box-Muller of two hashed uniforms, rounded to ComplexF32."""
    u1 = hash_uniform(seed, qx, qy, qz, comp, 1)
    u2 = hash_uniform(seed, qx, qy, qz, comp, 2)
    r = np.sqrt(-2.0 * np.log(u1))
    phase = (2.0 * np.pi) * u2
    re = np.where(real_only, r * np.cos(np.pi * (2.0 * u2)), r * np.cos(phase)).astype(np.float32)
    im = np.where(real_only, 0.0, r * np.sin(phase)).astype(np.float32)
    return re + np.complex64(1j) * im


def _mode(i, n):
    return np.where(i <= n // 2, i, i - n)


def hash_potential(dims, seed, box, realization_box, zero_phase=False):
    """_physical_hash_vector_potential_k (pmf.jl:149-191): three (nz, ny, nx//2+1) complex64
    arrays (x fastest, the reference's column-major (nx//2+1, ny, nz) memory order)."""
    nx, ny, nz = dims
    ratio = realization_box / box
    qscale = int(round(ratio))
    if not (qscale > 0 and abs(ratio - qscale) <= 32 * np.finfo(float).eps * max(1, abs(ratio))):
        raise ValueError("physical-hash reference_box/box must be a positive integer")
    nxh = nx // 2 + 1
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nxh), indexing="ij")
    mx, my, mz = ii, _mode(jj, ny), _mode(kk, nz)
    boundary = (ii == 0) | (ii == nxh - 1)
    pj, pk = np.mod(-my, ny), np.mod(-mz, nz)
    earlier = (pj < jj) | ((pj == jj) & (pk < kk))
    conj = boundary & earlier
    real_only = boundary & (pj == jj) & (pk == kk)
    key_my = np.where(conj, _mode(pj, ny), my)
    key_mz = np.where(conj, _mode(pk, nz), mz)
    out = []
    for c in (1, 2, 3):
        v = hash_normal(seed, qscale * mx, qscale * key_my, qscale * key_mz, c, real_only | zero_phase)
        out.append(np.where(conj, np.conj(v), v).astype(np.complex64))
    return out


def _zero_pad(ak, source_dims, target_dims):
    """_rfft_zero_pad_complex (pmf.jl:205-224)."""
    ox, oy, oz = source_dims
    nx, ny, nz = target_dims
    out = np.zeros((nz, ny, nx // 2 + 1), np.complex64)
    scale = np.float32((nx * ny * nz) / (ox * oy * oz))
    for kk in range(oz):
        mz = kk if kk <= oz // 2 else kk - oz
        tk = mz if mz >= 0 else nz + mz
        for jj in range(oy):
            my = jj if jj <= oy // 2 else jj - oy
            tj = my if my >= 0 else ny + my
            out[tk, tj, : ox // 2 + 1] = scale * ak[kk, jj, :]
    return out


def pmf_batchelor_field(dims, box=1.0, brms=1.0, seed=1, kcut=None, kmin=0.0, kmax=None, energy_index=4.0,
                        cutoff_order=2.0, mode_lock_n=None, high_mode_lock_n=None, preserve_low_kmax=None,
                        preserve_low_kcut=None, normalization_kind="auto", curl_symbol="centered",
                        curl_reference_n=None, fixed_mode_power=False, mode_realization="physical_hash",
                        realization_box=None, invariant_axis=0):
    """pmf.jl:300-591 for the physical-hash realizations. Returns (Bx, By, Bz, stats) with
    (nx*ny*nz,) float32 fields in x-fastest order."""
    nx, ny, nz = dims
    if nx % 2:
        raise ValueError("even nx required")
    L = float(box)
    zero_phase = mode_realization == "physical_hash_zero_phase"
    RL = L if realization_box is None else float(realization_box)
    kc = np.pi * min(dims) / L if kcut is None else float(kcut)
    km = np.inf if kmax is None else float(kmax)
    preserve_low = preserve_low_kmax is not None
    low_km = float(preserve_low_kmax) if preserve_low else None
    low_kc = kc if preserve_low_kcut is None else float(preserve_low_kcut)
    norm = normalization_kind
    if norm == "auto":
        norm = "reference_band_rms" if preserve_low else "total_band_rms"
    source_lock = high_mode_lock_n if high_mode_lock_n is not None else (None if preserve_low else mode_lock_n)
    source_dims = tuple(dims)
    if source_lock is not None and int(source_lock) != min(dims):
        source_dims = (int(source_lock),) * 3
    amp_exp = 0.5 * (energy_index - 4.0)
    nxh = nx // 2 + 1

    def realization(sd):
        a = hash_potential(sd, seed, L, RL, zero_phase)
        return a if tuple(sd) == tuple(dims) else [_zero_pad(x, sd, dims) for x in a]

    high = realization(source_dims)
    low_source_dims = tuple(dims)
    if preserve_low:
        if mode_lock_n is not None and int(mode_lock_n) != min(dims):
            low_source_dims = (int(mode_lock_n),) * 3
        low = realization(low_source_dims)
    else:
        low = high
    hss = np.float32(np.sqrt(np.prod(source_dims) / np.prod(low_source_dims))) if preserve_low else np.float32(1)
    dx = L / nx
    tpl = (2.0 * np.pi) / L
    kxv = np.arange(nxh) * tpl
    kyv = _mode(np.arange(ny), ny) * tpl
    kzv = _mode(np.arange(nz), nz) * tpl
    centered = curl_symbol == "centered"
    cref = 0 if curl_reference_n is None else int(curl_reference_n)

    def sym(k, h):
        return (np.sin(k * h) / h if centered else k).astype(np.float32)

    rdx = dx if cref == 0 else L / cref
    sx, sy, sz = sym(kxv, dx), sym(kyv, dx), sym(kzv, dx)
    rx, ry, rz = sym(kxv, rdx), sym(kyv, rdx), sym(kzv, rdx)
    project = cref != 0 and cref != min(dims)
    KZ, KY, KX = np.meshgrid(kzv, kyv, kxv, indexing="ij")
    k2 = KX * KX + KY * KY + KZ * KZ
    SZ, SY, SX = np.meshgrid(sz, sy, sx, indexing="ij")
    RZ, RY, RX = np.meshgrid(rz, ry, rx, indexing="ij")
    MZ, MY, MX = np.meshgrid(_mode(np.arange(nz), nz), _mode(np.arange(ny), ny), np.arange(nxh), indexing="ij")
    inv = [None, MX, MY, MZ][invariant_axis] if invariant_axis else None
    dead = (k2 == 0) | (k2 > km * km)
    if inv is not None:
        dead |= inv != 0
    with np.errstate(divide="ignore", invalid="ignore"):
        kmag = np.sqrt(k2)
        if preserve_low:
            thr = np.float32(np.float32(low_km) * np.float32(low_km)) * np.float32(1 + 8 * np.finfo(np.float32).eps)
            use_low = (k2 <= float(thr)) & ~dead
        else:
            use_low = np.zeros_like(dead)
        lkc = np.where(use_low, low_kc, kc)
        amp = (kmag / lkc) ** amp_exp * np.exp(-0.5 * (kmag / lkc) ** cutoff_order)
        w = (amp * np.where(use_low, np.float32(1), hss).astype(np.float64)).astype(np.float32)
        w = np.where(dead, np.float32(0), w)
    A = [np.where(use_low, low[c], high[c]) for c in range(3)]
    wa = [(w * a.real).astype(np.float32) + np.complex64(1j) * (w * a.imag).astype(np.float32) for a in A]

    def rmul(r, z):
        with np.errstate(invalid="ignore", over="ignore"):
            return (r * z.real) + np.complex64(1j) * (r * z.imag)

    def ti(z):
        return -z.imag + np.complex64(1j) * z.real

    b = [ti(rmul(RY, wa[2]) - rmul(RZ, wa[1])), ti(rmul(RZ, wa[0]) - rmul(RX, wa[2])),
         ti(rmul(RX, wa[1]) - rmul(RY, wa[0]))]
    b = [x.astype(np.complex64) for x in b]
    if project:
        s2 = (SX * SX + SY * SY + SZ * SZ).astype(np.float32)
        dot = rmul(SX, b[0]) + rmul(SY, b[1]) + rmul(SZ, b[2])
        with np.errstate(divide="ignore", invalid="ignore"):
            par = (dot.real / s2) + np.complex64(1j) * (dot.imag / s2)
        ok = s2 > 0
        b = [np.where(ok, (x - rmul(S, par)).astype(np.complex64), x) for x, S in zip(b, (SX, SY, SZ))]
    b = [np.where(dead, np.complex64(0), x) for x in b]
    lo = [np.where(use_low, x, np.complex64(0)) for x in b]
    kmin2 = float(kmin) ** 2
    if kmin > 0:
        b = [np.where(k2 <= kmin2, np.complex64(0), x) for x in b]
    if fixed_mode_power:
        live = ~((k2 == 0) | (k2 > km * km) | (k2 <= kmin2))
        raw = (b[0].real * b[0].real + b[0].imag * b[0].imag) + (b[1].real * b[1].real + b[1].imag * b[1].imag)
        raw = (raw + (b[2].real * b[2].real + b[2].imag * b[2].imag)).astype(np.float32)
        with np.errstate(divide="ignore", invalid="ignore"):
            target = (kmag / lkc) ** (energy_index - 2.0) * np.exp(-((kmag / lkc) ** cutoff_order))
            sm = np.sqrt(target / raw.astype(np.float64)).astype(np.float32)
        go = live & (raw > 0)
        b = [np.where(go, rmul(sm, x), x) for x in b]
        lo = [np.where(go & use_low, rmul(sm, x), x) for x in lo]
    n = nx * ny * nz
    B = [np.fft.irfftn(x.astype(np.complex128), s=(nz, ny, nx), axes=(0, 1, 2)).astype(np.float32).ravel()
         for x in b]
    rms0 = np.sqrt(sum((x.astype(np.float64) ** 2).sum() for x in B) / n)
    if not rms0 > 0:
        raise ValueError("generated zero PMF field")
    if preserve_low:
        Lw = [np.fft.irfftn(x.astype(np.complex128), s=(nz, ny, nx), axes=(0, 1, 2)).astype(np.float32).ravel()
              for x in lo]
        ref_rms0 = np.sqrt(sum((x.astype(np.float64) ** 2).sum() for x in Lw) / n)
    else:
        ref_rms0 = rms0
    scale = np.float32(brms / (ref_rms0 if norm == "reference_band_rms" else rms0))
    B = [x * scale for x in B]
    total = np.sqrt(sum((x.astype(np.float64) ** 2).sum() for x in B) / n)
    stats = {"brms_measured": total, "reference_band_brms_measured": float(scale) * ref_rms0,
             "normalization_kind": norm, "kcut": kc, "kmax": km, "high_source_scale": float(hss)}
    return B[0], B[1], B[2], stats


def ct_faces_from_cells(U, dims):
    """ct.jl:246-308 in FP64: faces (3, nc) float32 and the installed cell field (9, nc) float32
    (cell B = face average, E keeps the thermal pressure, psi = 0), plus the stats."""
    nx, ny, nz = dims
    Bold = [U[5 + d].astype(np.float64).reshape(nz, ny, nx) for d in range(3)]
    Bh = [np.fft.rfftn(b) for b in Bold]

    def half_phase(n, m):
        mm = np.where(m > n / 2, m - n, m)
        nyq = (n % 2 == 0) & (m == n // 2)
        return np.where(nyq, 0.0, np.pi * mm / n), nyq

    tx, qx = half_phase(nx, np.arange(nx // 2 + 1))
    ty, qy = half_phase(ny, np.arange(ny))
    tz, qz = half_phase(nz, np.arange(nz))
    THZ, THY, THX = np.meshgrid(tz, ty, tx, indexing="ij")
    QZ, QY, QX = np.meshgrid(qz, qy, qx, indexing="ij")
    bx = np.where(QX, 0, Bh[0]); by = np.where(QY, 0, Bh[1]); bz = np.where(QZ, 0, Bh[2])
    Tx, Ty, Tz = np.tan(THX), np.tan(THY), np.tan(THZ)
    t2 = Tx * Tx + Ty * Ty + Tz * Tz
    with np.errstate(divide="ignore", invalid="ignore"):
        dot = np.where(t2 > 0, (Tx * bx + Ty * by + Tz * bz) / np.where(t2 > 0, t2, 1.0), 0)
    bx = bx - Tx * dot; by = by - Ty * dot; bz = bz - Tz * dot
    F = [bx * np.exp(-1j * THX) / np.cos(THX), by * np.exp(-1j * THY) / np.cos(THY), bz * np.exp(-1j * THZ) / np.cos(THZ)]
    faces = np.stack([np.fft.irfftn(f, s=(nz, ny, nx), axes=(0, 1, 2)).ravel() for f in F]).astype(np.float32)
    f3 = [faces[d].reshape(nz, ny, nx) for d in range(3)]
    h = np.float32(0.5)
    bc = [(h * (f3[0] + np.roll(f3[0], -1, axis=2))).ravel(), (h * (f3[1] + np.roll(f3[1], -1, axis=1))).ravel(),
          (h * (f3[2] + np.roll(f3[2], -1, axis=0))).ravel()]
    out = U.astype(np.float32).copy()
    ox, oy, oz = out[5], out[6], out[7]
    out[4] = out[4] + h * ((bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]) - (ox * ox + oy * oy + oz * oz))
    out[5], out[6], out[7], out[8] = bc[0], bc[1], bc[2], 0
    Bnew = [out[5 + d].astype(np.float64) for d in range(3)]
    num = sum(((Bnew[d] - Bold[d].ravel()) ** 2).sum() for d in range(3))
    den = sum((Bold[d] ** 2).sum() for d in range(3))
    enew = sum((Bnew[d] ** 2).sum() for d in range(3))
    return faces, out, {"cell_b_rel_l2_change": float(np.sqrt(num / den)) if den > 0 else 0.0,
                        "magnetic_energy_ratio": float(enew / den) if den > 0 else 1.0}
