"""The NumPy restatement of the PMF initial-condition generator reproduces the reference's
own checks of it (test/inherited/runtests.jl:322-430) before it is trusted as the checker
of the device generator. The realization is the physical-hash one (the reference's
reproducible realization; its MersenneTwister `:legacy` draws are not reproducible
outside Julia), so the checks that the reference runs on legacy fields are run on hashed
ones: they test properties of the construction, not of the random draws."""
import numpy as np

import pmf_oracle as po

TWO_PI = 2 * np.pi


def test_hash_is_keyed_by_physical_mode():
    """runtests.jl:355-395: a half box keyed to the same realization box carries identical
    vector-potential coefficients on every shared mode."""
    a1 = po.hash_potential((32, 32, 32), 42, 1.0, 1.0)
    ah = po.hash_potential((16, 16, 16), 42, 0.5, 1.0)
    errs = []
    for mz in range(-2, 3):
        for my in range(-2, 3):
            for mx in range(0, 3):
                if mx == my == mz == 0 or 4 * np.pi * np.sqrt(mx * mx + my * my + mz * mz) > 12 * np.pi:
                    continue
                jh, kh = my % 16, mz % 16
                j1, k1 = (2 * my) % 32, (2 * mz) % 32
                for c in range(3):
                    errs.append(abs(ah[c][kh, jh, mx] - a1[c][k1, j1, 2 * mx]))
    assert errs and max(errs) == 0


def test_zero_phase_realization_is_real():
    a = po.hash_potential((16, 16, 16), 42, 1.0, 1.0, zero_phase=True)
    assert all(np.all(x.imag == 0) for x in a)


def _rfft3(f, n):
    return np.fft.rfftn(f.astype(np.float64).reshape(n, n, n))


def test_fixed_mode_power_scatter():
    """runtests.jl:322-341: with fixed_mode_power every mode carries the analytic envelope."""
    n = 32
    B = po.pmf_batchelor_field((n, n, n), box=1, brms=1e-3, seed=42, kcut=8 * np.pi, kmax=12 * np.pi,
                               fixed_mode_power=True)
    K = [_rfft3(B[c], n) for c in range(3)]
    vals = []
    for kk in range(n):
        for jj in range(n):
            for ii in range(n // 2 + 1):
                my = jj if jj <= 16 else jj - 32
                mz = kk if kk <= 16 else kk - 32
                k = TWO_PI * np.sqrt(ii * ii + my * my + mz * mz)
                if not 0 < k <= 8 * np.pi:
                    continue
                shape = (k / (8 * np.pi)) ** 2 * np.exp(-(k / (8 * np.pi)) ** 2)
                vals.append(sum(abs(K[c][kk, jj, ii]) ** 2 for c in range(3)) / shape)
    vals = np.array(vals)
    assert vals.std() / vals.mean() < 2e-5


def physical_pair():
    l1 = po.pmf_batchelor_field((32, 32, 32), box=1, brms=1e-3, seed=42, kcut=8 * np.pi, kmax=12 * np.pi,
                                mode_lock_n=32, curl_reference_n=32, fixed_mode_power=True, realization_box=1)
    lh = po.pmf_batchelor_field((32, 32, 32), box=0.5, brms=1e-3, seed=42, kcut=8 * np.pi, kmax=12 * np.pi,
                                mode_lock_n=16, curl_reference_n=16, fixed_mode_power=True, realization_box=1)
    return l1, lh


def common_mode_errors(l1, lh, n=32):
    k1 = [_rfft3(l1[c], n) for c in range(3)]
    kh = [_rfft3(lh[c], n) for c in range(3)]
    errs = []
    for mz in range(-2, 3):
        for my in range(-2, 3):
            for mx in range(0, 3):
                if mx == my == mz == 0 or 4 * np.pi * np.sqrt(mx * mx + my * my + mz * mz) > 12 * np.pi:
                    continue
                coarse = np.array([kh[c][mz % n, my % n, mx] for c in range(3)])
                ref = np.array([k1[c][(2 * mz) % n, (2 * my) % n, 2 * mx] for c in range(3)])
                cn, rn = np.linalg.norm(coarse), np.linalg.norm(ref)
                if cn > 0 and rn > 0:
                    errs.append(np.linalg.norm(coarse / cn - ref / rn))
    return errs


def test_matched_boxes_share_their_common_modes():
    """runtests.jl:343-395: boxes of side 1 and 1/2 keyed to one realization box agree on
    their common physical modes up to each grid's own solenoidal projection."""
    errs = common_mode_errors(*physical_pair())
    assert errs and max(errs) < 0.035


def test_reference_band_normalisation_at_a_rounded_fundamental():
    """runtests.jl:404-412: a preserved band cut infinitesimally below 2pi/L keeps that shell."""
    box = 1.03
    f = po.pmf_batchelor_field((16, 16, 16), box=box, brms=1e-3, seed=42, kcut=20 * np.pi / box,
                               kmax=8 * np.pi / box, preserve_low_kmax=6.100179909883,
                               normalization_kind="reference_band_rms", fixed_mode_power=True, realization_box=box)
    assert abs(f[3]["reference_band_brms_measured"] / 1e-3 - 1) < 2e-6


def nested(n):
    return po.pmf_batchelor_field((n, n, n), brms=1e-3, seed=42, kcut=8 * np.pi, kmax=16 * np.pi, mode_lock_n=16,
                                  high_mode_lock_n=32, preserve_low_kmax=4 * np.pi, preserve_low_kcut=8 * np.pi,
                                  curl_symbol="continuum")


def test_nested_grids_agree():
    """runtests.jl:414-428: the same locked modes on 32^3 and 64^3 give the same field at the
    common points."""
    c, f = nested(32), nested(64)
    for d in range(3):
        coarse = c[d].astype(np.float64).reshape(32, 32, 32)
        fine = f[d].astype(np.float64).reshape(64, 64, 64)[::2, ::2, ::2]
        rel = np.sqrt(((coarse - fine) ** 2).sum() / (coarse ** 2).sum())
        corr = (coarse * fine).sum() / np.sqrt((coarse ** 2).sum() * (fine ** 2).sum())
        assert rel < 2e-5 and corr > 1 - 2e-6


def test_centred_field_is_solenoidal_and_normalised():
    n = 32
    B = po.pmf_batchelor_field((n, n, n), brms=2e-3, seed=7, kcut=8 * np.pi)
    assert abs(B[3]["brms_measured"] / 2e-3 - 1) < 1e-6
    f = [B[c].astype(np.float64).reshape(n, n, n) for c in range(3)]
    dx = 1.0 / n
    div = ((np.roll(f[0], -1, 2) - np.roll(f[0], 1, 2)) + (np.roll(f[1], -1, 1) - np.roll(f[1], 1, 1)) +
           (np.roll(f[2], -1, 0) - np.roll(f[2], 1, 0))) / (2 * dx)
    assert np.abs(div).max() * dx / 2e-3 < 1e-5
