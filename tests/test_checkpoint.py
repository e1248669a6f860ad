"""Checkpoint write/restore rules of the production runner (runner.jl:26-140), as checked by
the reference's test/inherited/test_pmf_checkpoint_helpers.jl:14-86, on host arrays."""
import numpy as np
import pytest

from checkpoint import CheckpointError, restore_pmf_checkpoint, write_pmf_checkpoint


def test_endpoint_extension_optional_fields_and_allowed_changes(tmp_path):
    path = str(tmp_path / "checkpoint.bin")
    stored = dict(N=4, zstart=3.0e6, zend=1.0e5, cfl=0.1)
    expected = dict(N=4, zstart=3.0e6, zend=500.0, cfl=0.1)
    source = np.array([1, 2, 3], np.float32)
    assert write_pmf_checkpoint(path, stored, {"cycle": 7}, [("field", source)]) > 0
    dest = np.zeros(3, np.float32)
    assert restore_pmf_checkpoint(path, expected, [("field", dest)])["cycle"] == 7
    assert np.array_equal(dest, source)
    opt = np.ones(3, np.float32)
    rt = restore_pmf_checkpoint(path, expected, [("field", dest), ("magnetic_residual_1", opt)],
                                optional_missing_arrays=("magnetic_residual_1",))
    assert rt["cycle"] == 7 and np.all(opt == 0)
    with pytest.raises(CheckpointError):
        restore_pmf_checkpoint(path, expected, [("field", dest), ("required_trailing", np.zeros(3, np.float32))])
    incompatible = dict(N=4, zstart=3.0e6, zend=500.0, cfl=0.2)
    with pytest.raises(CheckpointError):
        restore_pmf_checkpoint(path, incompatible, [("field", np.zeros(3, np.float32))])
    dest[:] = 0
    with pytest.warns(UserWarning):
        rt = restore_pmf_checkpoint(path, incompatible, [("field", dest)], allowed_config_changes=("cfl",))
    assert rt["cycle"] == 7 and np.array_equal(dest, source)
    physical = dict(N=8, zstart=3.0e6, zend=500.0, cfl=0.2)
    with pytest.raises(CheckpointError):
        restore_pmf_checkpoint(path, physical, [("field", np.zeros(3, np.float32))], allowed_config_changes=("cfl",))
    # a validator can veto an allowed change
    with pytest.raises(CheckpointError):
        restore_pmf_checkpoint(path, incompatible, [("field", dest)], allowed_config_changes=("cfl",),
                               allowed_config_validator=lambda s, e, r, changed: False)


def test_solver_guard_and_exact_round_trip(tmp_path):
    base = dict(N=4, zstart=3.0e6, zend=1.0e5, cfl=0.1)
    src = np.array([1, 2, 3], np.float32)
    legacy, glm, ct = (str(tmp_path / n) for n in ("legacy.bin", "glm.bin", "ct.bin"))
    write_pmf_checkpoint(legacy, base, {"cycle": 1}, [("field", src)])
    write_pmf_checkpoint(glm, {**base, "mhd_solver": "glm"}, {"cycle": 2}, [("field", src)])
    write_pmf_checkpoint(ct, {**base, "mhd_solver": "ct"}, {"cycle": 3}, [("field", src), ("ct_bxf", src)])

    def want(s):
        return {**base, "mhd_solver": s}

    def restore(p, cfg, arrays=None):
        return restore_pmf_checkpoint(p, cfg, arrays or [("field", np.zeros(3, np.float32))])
    assert restore(legacy, want("glm"))["cycle"] == 1
    assert restore(legacy, {**want("glm"), "zend": 5.0e4})["cycle"] == 1
    assert restore(glm, want("glm"))["cycle"] == 2
    for p in (legacy, glm):
        with pytest.raises(CheckpointError, match="mhd_solver mismatch"):
            restore(p, want("ct"))
    with pytest.raises(CheckpointError, match="mhd_solver mismatch"):
        restore(ct, want("glm"))
    faces, field = np.zeros(3, np.float32), np.zeros(3, np.float32)
    assert restore(ct, want("ct"), [("field", field), ("ct_bxf", faces)])["cycle"] == 3
    assert np.array_equal(faces, src)


def test_shape_dtype_name_and_magic_checks(tmp_path):
    path = str(tmp_path / "c.bin")
    cfg = dict(N=4)
    a = np.arange(12, dtype=np.float32).reshape(3, 4)
    b = np.arange(5, dtype=np.float64)
    write_pmf_checkpoint(path, cfg, {"t": 0.5, "measured": [1, 2]}, [("a", a), ("b", b)])
    da, db = np.zeros((3, 4), np.float32), np.zeros(5, np.float64)
    rt = restore_pmf_checkpoint(path, cfg, [("a", da), ("b", db)])
    assert rt == {"t": 0.5, "measured": [1, 2]}
    assert np.array_equal(da, a) and np.array_equal(db, b)
    with pytest.raises(CheckpointError, match="size mismatch"):
        restore_pmf_checkpoint(path, cfg, [("a", np.zeros(12, np.float32)), ("b", db)])
    with pytest.raises(CheckpointError, match="type mismatch"):
        restore_pmf_checkpoint(path, cfg, [("a", da), ("b", np.zeros(5, np.float32))])
    with pytest.raises(CheckpointError, match="field mismatch"):
        restore_pmf_checkpoint(path, cfg, [("b", db), ("a", da)])
    with pytest.raises(CheckpointError, match="array-count"):
        restore_pmf_checkpoint(path, cfg, [("a", da)])
    with open(str(tmp_path / "bad.bin"), "wb") as f:
        f.write(b"not a checkpoint")
    with pytest.raises(CheckpointError, match="unsupported"):
        restore_pmf_checkpoint(str(tmp_path / "bad.bin"), cfg, [("a", da)])
    assert not (tmp_path / "c.bin.tmp").exists()


def test_truncated_checkpoint_is_rejected(tmp_path):
    """A file cut short anywhere (header, field metadata or field data) raises CheckpointError
    rather than failing in reshape or restoring part of a state."""
    path = str(tmp_path / "c.bin")
    cfg = dict(N=4)
    a = np.arange(12, dtype=np.float32).reshape(3, 4)
    b = np.arange(5, dtype=np.float64)
    write_pmf_checkpoint(path, cfg, {"t": 0.5}, [("a", a), ("b", b)])
    full = open(path, "rb").read()
    for cut in (len(full) - 1, len(full) - 5 * 8, len(full) - 45, 40):
        bad = str(tmp_path / f"cut{cut}.bin")
        with open(bad, "wb") as f:
            f.write(full[:cut])
        with pytest.raises(CheckpointError, match="truncated"):
            restore_pmf_checkpoint(bad, cfg, [("a", np.zeros((3, 4), np.float32)), ("b", np.zeros(5, np.float64))])
