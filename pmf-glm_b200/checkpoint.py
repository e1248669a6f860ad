"""Run checkpoints of a PMF run: the semantics of the production runner's checkpoint helpers
(src/production/runner.jl:26-140, `_write_pmf_checkpoint` / `_restore_pmf_checkpoint!`).

The reference writes Julia's `Serialization` stream, which only Julia can read; this module
keeps the same content and rules in a self-describing binary container:

    b"pmfmhd PMF checkpoint v1\\n"
    u64 length + JSON {"config": ..., "runtime": ..., "narrays": n}
    n times: u64 length + JSON {"name", "dtype", "shape"}, then the raw little-endian array bytes

* fields are streamed one at a time (a device array is copied to the host, written and
  released before the next), so checkpointing never holds a second full state in host memory;
* the file is written to ``path + ".tmp"``, flushed to stable storage (fsync) and renamed
  over ``path``, so a crash or power loss mid-write leaves the previous checkpoint intact;
* a file cut short (a copy interrupted, a full disk) is rejected with CheckpointError, not
  half-restored;
* restoring checks the solver (a checkpoint without an ``mhd_solver`` key is a GLM one and
  never resumes as CT, nor the other way round), the configuration fingerprint (equal, or a
  legacy subset, or only ``zend`` changed, or only explicitly allowed keys changed and accepted
  by an optional validator), the array count, names, shapes and dtypes; trailing arrays named
  as optional may be missing and are zero-filled.

Configuration values may be numbers, strings, booleans, None or lists of them.
"""
from __future__ import annotations

import json
import math
import os
import struct
import warnings
from typing import Callable, Iterable, Optional, Sequence, Tuple

import numpy as np

MAGIC = b"pmfmhd PMF checkpoint v1\n"


class CheckpointError(RuntimeError):
    pass


def _to_host(a) -> np.ndarray:
    try:
        import torch
        if isinstance(a, torch.Tensor):
            return a.detach().cpu().numpy()
    except ImportError:  # pragma: no cover
        pass
    return np.asarray(a)


def _write_block(f, obj) -> None:
    data = json.dumps(obj, sort_keys=False).encode()
    f.write(struct.pack("<Q", len(data)))
    f.write(data)


def _read_exact(f, n: int) -> bytes:
    data = f.read(n)
    if len(data) != n:
        raise CheckpointError("truncated PMF checkpoint")
    return data


def _read_block(f):
    (n,) = struct.unpack("<Q", _read_exact(f, 8))
    return json.loads(_read_exact(f, n).decode())


def write_pmf_checkpoint(path: str, config: dict, runtime: dict, arrays: Sequence[Tuple[str, object]]) -> int:
    """Write a checkpoint; returns its size in bytes (0 and nothing written for an empty path)."""
    if not path:
        return 0
    parent = os.path.dirname(path)
    if parent:
        os.makedirs(parent, exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(MAGIC)
        _write_block(f, {"config": config, "runtime": runtime, "narrays": len(arrays)})
        for name, arr in arrays:
            h = np.ascontiguousarray(_to_host(arr))
            dt = h.dtype.newbyteorder("<")
            _write_block(f, {"name": str(name), "dtype": dt.str, "shape": list(h.shape)})
            f.write(h.astype(dt, copy=False).tobytes())
            del h
        f.flush()
        os.fsync(f.fileno())
    os.replace(tmp, path)
    # the rename reaches stable storage with its directory entry (not possible everywhere)
    try:
        d = os.open(os.path.dirname(os.path.abspath(path)), os.O_RDONLY)
        try:
            os.fsync(d)
        finally:
            os.close(d)
    except OSError:
        pass
    return os.path.getsize(path)


def _isequal(a, b) -> bool:
    """Julia's isequal on configuration values: NaN equals NaN, -0.0 differs from 0.0."""
    if isinstance(a, float) and isinstance(b, float):
        if math.isnan(a) and math.isnan(b):
            return True
        return a == b and math.copysign(1.0, a) == math.copysign(1.0, b)
    if isinstance(a, (list, tuple)) and isinstance(b, (list, tuple)):
        return len(a) == len(b) and all(_isequal(x, y) for x, y in zip(a, b))
    if isinstance(a, bool) != isinstance(b, bool):
        return False
    return a == b


def _config_equal(a: dict, b: dict) -> bool:
    return list(a.keys()) == list(b.keys()) and all(_isequal(a[k], b[k]) for k in a)


def _copy_into(dest, host: np.ndarray) -> None:
    try:
        import torch
        if isinstance(dest, torch.Tensor):
            dest.copy_(torch.from_numpy(host).to(dest.device))
            return
    except ImportError:  # pragma: no cover
        pass
    dest[...] = host


def _dtype_of(dest) -> np.dtype:
    try:
        import torch
        if isinstance(dest, torch.Tensor):
            return np.dtype(str(dest.dtype).replace("torch.", ""))
    except ImportError:  # pragma: no cover
        pass
    return np.asarray(dest).dtype


def _zero(dest) -> None:
    try:
        import torch
        if isinstance(dest, torch.Tensor):
            dest.zero_()
            return
    except ImportError:  # pragma: no cover
        pass
    dest[...] = 0


def restore_pmf_checkpoint(path: str, expected_config: dict, arrays: Sequence[Tuple[str, object]],
                           allowed_config_changes: Iterable[str] = (),
                           allowed_config_validator: Optional[Callable] = None,
                           optional_missing_arrays: Iterable[str] = ()) -> dict:
    """Restore `arrays` (host or device arrays, filled in place) and return the runtime record."""
    with open(path, "rb") as f:
        if f.read(len(MAGIC)) != MAGIC:
            raise CheckpointError(f"unsupported PMF checkpoint format: {path}")
        head = _read_block(f)
        stored, runtime = dict(head["config"]), head["runtime"]
        expected = dict(expected_config)
        if "mhd_solver" in expected:
            has_key = "mhd_solver" in stored
            stored_solver = str(stored["mhd_solver"]) if has_key else "glm"
            expected_solver = str(expected["mhd_solver"])
            if stored_solver != expected_solver:
                raise CheckpointError(
                    f"PMF checkpoint mhd_solver mismatch: checkpoint was written by mhd_solver={stored_solver}"
                    + ("" if has_key else " (no mhd_solver key: legacy GLM)")
                    + f" but this run requests mhd_solver={expected_solver}; resume with the same solver "
                      "or start a new run")
            if not has_key:
                stored["mhd_solver"] = "glm"
        if not _config_equal(stored, expected):
            sk = list(stored.keys())

            def same(k):
                return k in expected and _isequal(stored[k], expected[k])
            compatible_legacy = all(same(k) for k in sk)
            compatible_endpoint = (all(k == "zend" or same(k) for k in sk)
                                   and all(k == "zend" or k in stored for k in expected))
            allowed = set(str(k) for k in allowed_config_changes)
            structural = (bool(allowed) and all(k == "zend" or k in allowed or same(k) for k in sk)
                          and all(k == "zend" or k in allowed or k in stored for k in expected)
                          and all(k in stored and k in expected for k in allowed))
            changed = [k for k in allowed if not _isequal(stored[k], expected[k])] if structural else []
            compatible_override = structural and (
                allowed_config_validator is None or allowed_config_validator(stored, expected, runtime, changed))
            if not (compatible_legacy or compatible_endpoint or compatible_override):
                raise CheckpointError(f"PMF checkpoint configuration mismatch\nstored:   {stored}\nexpected: {expected}")
            if compatible_legacy:
                if "velocity_transport_version" in expected and "velocity_transport_version" not in stored:
                    raise CheckpointError("checkpoint predates corrected photon velocity evolution; restart this "
                                          "trajectory from a consistent initial state")
                warnings.warn("restoring legacy PMF checkpoint without newer fingerprint fields "
                              f"(missing: {[k for k in expected if k not in stored]})")
            elif not compatible_endpoint:
                warnings.warn(f"restoring PMF checkpoint with explicitly allowed configuration changes {changed}")
        narrays = int(head["narrays"])
        if narrays > len(arrays):
            raise CheckpointError(f"PMF checkpoint array-count mismatch: stored={narrays} expected={len(arrays)}")
        optional = set(str(x) for x in optional_missing_arrays)
        for index, (expected_name, dest) in enumerate(arrays):
            if index >= narrays:
                if str(expected_name) not in optional:
                    raise CheckpointError(f"PMF checkpoint is missing required trailing field {expected_name}")
                _zero(dest)
                continue
            meta = _read_block(f)
            if meta["name"] != str(expected_name):
                raise CheckpointError(f"PMF checkpoint field mismatch: stored={meta['name']} expected={expected_name}")
            dt = np.dtype(meta["dtype"])
            shape = tuple(meta["shape"])
            data = _read_exact(f, int(np.prod(shape, dtype=np.int64)) * dt.itemsize)
            host = np.frombuffer(data, dtype=dt).reshape(shape)
            dshape = tuple(dest.shape)
            if shape != dshape:
                raise CheckpointError(f"PMF checkpoint size mismatch for {meta['name']}: stored={shape} "
                                      f"expected={dshape}")
            if dt.newbyteorder("=") != _dtype_of(dest).newbyteorder("="):
                raise CheckpointError(f"PMF checkpoint type mismatch for {meta['name']}: stored={dt} "
                                      f"expected={_dtype_of(dest)}")
            _copy_into(dest, host.astype(dt.newbyteorder("="), copy=True))
        return runtime


def state_arrays(s) -> list:
    """The arrays of an MHDState in checkpoint order: the nine conserved fields, the CT faces
    and their remainders (CT states), the compensation remainders (compensated states)."""
    out = [(f"U{v + 1}", s.U[v]) for v in range(9)]
    if s.ct is not None:
        out += [("ct_bxf", s.ct.slot(0)), ("ct_byf", s.ct.slot(1)), ("ct_bzf", s.ct.slot(2)),
                ("ct_residual_1", s.ct.slot(18)), ("ct_residual_2", s.ct.slot(19)), ("ct_residual_3", s.ct.slot(20))]
    if s.resid is not None:
        out += [(f"residual_{i + 1}", r) for i, r in enumerate(s.resid)]
    return out
