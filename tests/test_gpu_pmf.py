"""The device initial-condition generators (through the C ABI) against the NumPy oracle of
pmf.jl / ct.jl and the reference's own checks of them (test/inherited/runtests.jl:322-430,
ct.jl:246-308): the Batchelor PMF field with the physical-hash realizations, mode locking,
the preserved low band, fixed mode power and the invariant axis; the uniform-gas install;
the tiled variant; and ct_faces_from_cells on cuFFT."""
import numpy as np
import pytest
import torch

import pmf_oracle as po
import pmfmhd
import problems
from mhd_cases import within_parity
from test_pmf_oracle import common_mode_errors

pytestmark = pytest.mark.gpu
PI = np.pi

CASES = {
    "centred": dict(dims=(32, 32, 32), box=1, brms=1e-3, seed=42, kcut=8 * PI, kmax=12 * PI),
    "locked_half_box": dict(dims=(32, 32, 32), box=0.5, brms=1e-3, seed=42, kcut=8 * PI, kmax=12 * PI,
                            mode_lock_n=16, curl_reference_n=16, fixed_mode_power=True, realization_box=1),
    "zero_phase": dict(dims=(16, 16, 16), box=1, brms=1e-3, seed=42, kcut=8 * PI, kmax=2 * PI,
                       mode_realization="physical_hash_zero_phase", realization_box=1),
    "rounded_fundamental": dict(dims=(16, 16, 16), box=1.03, brms=1e-3, seed=42, kcut=20 * PI / 1.03,
                                kmax=8 * PI / 1.03, preserve_low_kmax=6.100179909883,
                                normalization_kind="reference_band_rms", fixed_mode_power=True, realization_box=1.03),
    "nested64": dict(dims=(64, 64, 64), brms=1e-3, seed=42, kcut=8 * PI, kmax=16 * PI, mode_lock_n=16,
                     high_mode_lock_n=32, preserve_low_kmax=4 * PI, preserve_low_kcut=8 * PI,
                     curl_symbol="continuum"),
    "ragged_invariant": dict(dims=(48, 32, 24), box=1.5, brms=2e-2, seed=-5, kcut=6 * PI, kmin=3 * PI,
                             energy_index=2.0, cutoff_order=4.0, invariant_axis=3),
}


def host(B):
    return np.stack([b.cpu().numpy() for b in B[:3]])


@pytest.mark.parametrize("name", list(CASES))
def test_pmf_field_matches_oracle(name):
    kw = dict(CASES[name])
    dims = kw.pop("dims")
    g = pmfmhd.pmf_batchelor_field(dims, **kw)
    o = po.pmf_batchelor_field(dims, **kw)
    hg, ho = host(g), np.stack(o[:3])
    assert np.isfinite(hg).all()
    # cuFFT single precision against an FP64 inverse transform of the same coefficients
    assert np.abs(hg - ho).max() <= 1e-5 * np.abs(ho).max(), np.abs(hg - ho).max() / np.abs(ho).max()
    assert abs(g[3]["brms_measured"] / o[3]["brms_measured"] - 1) < 1e-5
    assert abs(g[3]["reference_band_brms_measured"] / o[3]["reference_band_brms_measured"] - 1) < 1e-5


def test_pmf_known_answers_on_the_device():
    """runtests.jl:322-412 on the device's fields: fixed-mode scatter, common modes of matched
    boxes, reference-band normalisation at a rounded fundamental, nested grids."""
    n = 32
    fx = host(pmfmhd.pmf_batchelor_field((n, n, n), box=1, brms=1e-3, seed=42, kcut=8 * PI, kmax=12 * PI,
                                         fixed_mode_power=True))
    K = [np.fft.rfftn(fx[c].astype(np.float64).reshape(n, n, n)) for c in range(3)]
    kz, ky, kx = np.meshgrid(np.fft.fftfreq(n, 1 / n), np.fft.fftfreq(n, 1 / n), np.arange(n // 2 + 1), indexing="ij")
    k = 2 * PI * np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    sel = (k > 0) & (k <= 8 * PI)
    shape = (k[sel] / (8 * PI)) ** 2 * np.exp(-(k[sel] / (8 * PI)) ** 2)
    vals = sum(np.abs(K[c][sel]) ** 2 for c in range(3)) / shape
    assert vals.std() / vals.mean() < 2e-5
    l1 = host(pmfmhd.pmf_batchelor_field((32, 32, 32), box=1, brms=1e-3, seed=42, kcut=8 * PI, kmax=12 * PI,
                                         mode_lock_n=32, curl_reference_n=32, fixed_mode_power=True,
                                         realization_box=1))
    lh = host(pmfmhd.pmf_batchelor_field((32, 32, 32), **{k_: v for k_, v in CASES["locked_half_box"].items()
                                                           if k_ != "dims"}))
    errs = common_mode_errors(l1, lh)
    assert errs and max(errs) < 0.035
    kw = dict(CASES["rounded_fundamental"])
    kw.pop("dims")
    st = pmfmhd.pmf_batchelor_field((16, 16, 16), **kw)[3]
    assert abs(st["reference_band_brms_measured"] / 1e-3 - 1) < 2e-6
    kw = dict(CASES["nested64"])
    kw.pop("dims")
    c32 = host(pmfmhd.pmf_batchelor_field((32, 32, 32), **kw))
    c64 = host(pmfmhd.pmf_batchelor_field((64, 64, 64), **kw))
    for d in range(3):
        coarse = c32[d].astype(np.float64).reshape(32, 32, 32)
        fine = c64[d].astype(np.float64).reshape(64, 64, 64)[::2, ::2, ::2]
        assert np.sqrt(((coarse - fine) ** 2).sum() / (coarse ** 2).sum()) < 2e-5
        assert (coarse * fine).sum() / np.sqrt((coarse ** 2).sum() * (fine ** 2).sum()) > 1 - 2e-6


def test_init_pmf_glm_and_ct_states():
    """init_pmf_batchelor! (pmf.jl:602-642): uniform gas around the field; CT states get
    divergence-free faces from ct_faces_from_cells! (compared with the FP64 oracle)."""
    n = 32
    kw = dict(brms=0.05, seed=3, kcut=8 * PI, kmax=12 * PI, mode_realization="physical_hash")
    s = pmfmhd.allocate_state((n, n, n), 1.0 / n)
    st = pmfmhd.init_pmf_batchelor(s, rho0=1.3, p0=0.7, **kw)
    h = pmfmhd.fields_to_host(s)
    B = np.stack(po.pmf_batchelor_field((n, n, n), box=1.0, **kw)[:3])
    assert np.abs(h[5:8] - B).max() <= 1e-5 * np.abs(B).max()
    assert np.all(h[0] == np.float32(1.3)) and np.all(h[1:4] == 0) and np.all(h[8] == 0)
    E = np.float32(0.7) / np.float32(5 / 3 - 1) + np.float32(0.5) * (h[5] ** 2 + h[6] ** 2 + h[7] ** 2)
    assert np.abs(h[4] - E).max() <= 1e-6 * E.max()
    assert abs(st["brms_measured"] / 0.05 - 1) < 1e-5 and st["rho0"] == 1.3
    c = pmfmhd.allocate_state((n, n, n), 1.0 / n, mhd_solver="ct")
    st = pmfmhd.init_pmf_batchelor(c, rho0=1.3, p0=0.7, **kw)
    assert st["ct_faces"]["max_divb_face_dx_over_brms"] < 1e-5
    # the oracle's ct_faces_from_cells on the same installed cell field
    g = pmfmhd.allocate_state((n, n, n), 1.0 / n)
    pmfmhd.init_pmf_batchelor(g, rho0=1.3, p0=0.7, **kw)
    faces, cells, ost = po.ct_faces_from_cells(pmfmhd.fields_to_host(g), (n, n, n))
    fg = c.ct.packed[: 3 * n ** 3].cpu().numpy().reshape(3, -1)
    assert np.abs(fg - faces).max() <= 1e-6 * np.abs(faces).max()
    assert not within_parity(cells, pmfmhd.fields_to_host(c))
    assert abs(st["ct_faces"]["cell_b_rel_l2_change"] - ost["cell_b_rel_l2_change"]) <= 1e-6
    assert abs(st["ct_faces"]["magnetic_energy_ratio"] / ost["magnetic_energy_ratio"] - 1) <= 1e-6
    assert torch.count_nonzero(c.ct.rbx) == 0


def test_ct_faces_from_cells_matches_oracle_on_a_smooth_field():
    n = 24
    U = problems.smooth_fields(n)
    s = pmfmhd.set_fields(pmfmhd.allocate_state((n, n, n), 1.0 / n, mhd_solver="ct"), U)
    st = pmfmhd.ct_faces_from_cells(s)
    faces, cells, ost = po.ct_faces_from_cells(U, (n, n, n))
    fg = s.ct.packed[: 3 * n ** 3].cpu().numpy().reshape(3, -1)
    assert np.abs(fg - faces).max() <= 1e-6 * np.abs(faces).max()
    assert not within_parity(cells, pmfmhd.fields_to_host(s))
    assert st["max_divb_face_dx_over_brms"] < 1e-5


def test_tiled_pmf_repeats_the_tile():
    """init_pmf_batchelor_tiled! (pmf.jl:652-710): the box holds the tile's field repeated."""
    n = 32
    s = pmfmhd.allocate_state((n, n, n), 1.0 / n)
    st = pmfmhd.init_pmf_batchelor_tiled(s, tile_box=0.5, brms=0.02, seed=9, kcut=8 * PI, realization_box=0.5)
    assert st["tile_n"] == 16
    h = pmfmhd.fields_to_host(s)[5:8].reshape(3, n, n, n)
    assert np.array_equal(h[:, :16, :16, :16], h[:, 16:, 16:, 16:])
    assert np.array_equal(h[:, :16, :16, :16], h[:, :16, 16:, :16])
    t = po.pmf_batchelor_field((16, 16, 16), box=0.5, brms=0.02, seed=9, kcut=8 * PI, realization_box=0.5)
    tile = np.stack(t[:3]).reshape(3, 16, 16, 16)
    assert np.abs(h[:, :16, :16, :16] - tile).max() <= 1e-5 * np.abs(tile).max()


def test_pmf_argument_errors():
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.pmf_batchelor_field((16, 16, 16), mode_realization="legacy")
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.pmf_batchelor_field((15, 16, 16))
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.pmf_batchelor_field((16, 16, 16), brms=0)
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.pmf_batchelor_field((16, 16, 16), normalization_kind="reference_band_rms")
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.pmf_batchelor_field((32, 32, 32), kmax=12 * PI, minimum_cells_per_wavelength=16)
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.pmf_batchelor_field((16, 16, 16), box=1.0, realization_box=1.5)
    s = pmfmhd.allocate_state((32, 32, 32), 1.0 / 32)
    with pytest.raises(pmfmhd.PMFMHDError):
        pmfmhd.init_pmf_batchelor_tiled(s, tile_box=0.3, brms=1.0)


def test_checkpoint_round_trip_of_a_device_state(tmp_path):
    """runner.jl:26-140 semantics on device arrays: a CT state written and restored into a
    fresh state steps to the same bits."""
    import checkpoint
    n = 16
    a = pmfmhd.allocate_state((n, n, n), 1.0 / n, mhd_solver="ct")
    pmfmhd.init_pmf_batchelor(a, brms=0.3, seed=5, kcut=6 * PI)
    cfg = {"N": n, "mhd_solver": "ct", "cfl": 0.3}
    path = str(tmp_path / "ck.bin")
    checkpoint.write_pmf_checkpoint(path, cfg, {"cycle": 11}, checkpoint.state_arrays(a))
    b = pmfmhd.allocate_state((n, n, n), 1.0 / n, mhd_solver="ct")
    rt = checkpoint.restore_pmf_checkpoint(path, cfg, checkpoint.state_arrays(b))
    assert rt["cycle"] == 11
    for _ in range(3):
        dt, _ = pmfmhd.compute_dt(a, 0.3)
        pmfmhd.step(a, float(dt), integrator="ref")
        pmfmhd.step(b, float(dt), integrator="ref")
    assert np.array_equal(pmfmhd.fields_to_host(a), pmfmhd.fields_to_host(b))
    assert torch.equal(a.ct.packed[: 3 * n ** 3], b.ct.packed[: 3 * n ** 3])
