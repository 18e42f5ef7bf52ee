"""Binary checkpoint files of a session, read and written on the host.

The same format as ``tara_checkpoint_write`` / ``tara_checkpoint_read`` of
the CUDA library (``csrc/checkpoint.cu``), for tools that inspect or prepare
checkpoints without a GPU.  Little-endian throughout:

* header, 192 bytes: ``b"TARA2DCK"``, uint32 version (1), int32 model,
  precision, Nx, Ny, nf, fix_curlB, flags (bit 0: history present), int64
  step, float64 time, float64 params[17] in the order of ``PARAM_NAMES``;
* nf state fields, then (flags bit 0) nf history fields, each a
  ``complex128`` array of shape (Ny, Nx/2 + 1);
* checksum, 16 bytes: uint64 s1 = sum of every preceding 8-byte word w_i and
  uint64 s2 = sum of (i + 1) * w_i, both modulo 2**64.

The reference has no restart (its drivers always start from an initial
condition, src/main2com.f95:215-343, src/main2coh.f95:176-257).
"""
from __future__ import annotations

import os
import struct

import numpy as np

MAGIC = b"TARA2DCK"
VERSION = 1
HEADER_BYTES = 192
PARAM_NAMES = ("Lx", "Ly", "pi", "dt", "mux", "muy", "ms", "CS", "spheat", "mu", "mu_0", "eta", "kf", "A",
               "nu", "alpha", "lambda")
_HEAD = struct.Struct("<8sI7iqd17d")
assert _HEAD.size == HEADER_BYTES


class CheckpointError(ValueError):
    pass


def checksum(words: np.ndarray) -> tuple[int, int]:
    """(s1, s2) of a uint64 word array: sum w_i and sum (i + 1) w_i modulo 2**64."""
    w = np.asarray(words, dtype="<u8")
    idx = np.arange(1, w.size + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        s1 = int(np.sum(w, dtype=np.uint64))
        s2 = int(np.sum(w * idx, dtype=np.uint64))
    return s1, s2


def write(path, model: int, precision: int, Nx: int, Ny: int, state, history=None, step: int = 0,
          time: float = 0.0, params: dict | None = None, fix_curlB: int = 0) -> None:
    """Write a checkpoint; state/history are lists of (Ny, Nx//2+1) complex arrays."""
    Nh = Nx // 2 + 1
    fields = [np.ascontiguousarray(f, dtype="<c16") for f in state]
    nf = len(fields)
    if history is not None:
        hist = [np.ascontiguousarray(f, dtype="<c16") for f in history]
        if len(hist) != nf:
            raise CheckpointError("history and state differ in field count")
        fields += hist
    if any(f.shape != (Ny, Nh) for f in fields):
        raise CheckpointError(f"fields must have shape ({Ny}, {Nh})")
    p = dict(params or {})
    prm = [float(p.get(k, 0.0)) for k in PARAM_NAMES]
    head = _HEAD.pack(MAGIC, VERSION, model, precision, Nx, Ny, nf, fix_curlB, 1 if history is not None else 0,
                      int(step), float(time), *prm)
    body = head + b"".join(f.tobytes() for f in fields)
    s1, s2 = checksum(np.frombuffer(body, dtype="<u8"))
    tmp = os.fspath(path) + ".tmp"
    with open(tmp, "wb") as fh:
        fh.write(body)
        fh.write(struct.pack("<QQ", s1, s2))
    os.replace(tmp, path)


def read_header(path) -> dict:
    """The header fields of a checkpoint (no field data, no checksum check)."""
    with open(path, "rb") as fh:
        data = fh.read(HEADER_BYTES)
    if len(data) < HEADER_BYTES or data[:8] != MAGIC:
        raise CheckpointError(f"{path}: not a checkpoint file")
    (_, version, model, precision, Nx, Ny, nf, fix_curlB, flags, step, time, *prm) = _HEAD.unpack_from(data)
    return dict(version=version, model=model, precision=precision, Nx=Nx, Ny=Ny, nf=nf, fix_curlB=fix_curlB,
                history=bool(flags & 1), step=step, time=time, params=dict(zip(PARAM_NAMES, prm)))


def read(path) -> dict:
    """Read and verify a checkpoint: a dict with model, precision, Nx, Ny, nf,
    fix_curlB, step, time, params (dict), state (list) and history (list or None)."""
    with open(path, "rb") as fh:
        data = fh.read()
    if len(data) < HEADER_BYTES + 16 or data[:8] != MAGIC:
        raise CheckpointError(f"{path}: not a checkpoint file")
    (_, version, model, precision, Nx, Ny, nf, fix_curlB, flags, step, time, *prm) = _HEAD.unpack_from(data)
    if version != VERSION:
        raise CheckpointError(f"{path}: unsupported version {version}")
    Nh = Nx // 2 + 1
    nfields = nf * (2 if flags & 1 else 1)
    size = HEADER_BYTES + nfields * Ny * Nh * 16
    if len(data) != size + 16:
        raise CheckpointError(f"{path}: truncated or oversized ({len(data)} bytes, expected {size + 16})")
    s1, s2 = struct.unpack_from("<QQ", data, size)
    if (s1, s2) != checksum(np.frombuffer(data, dtype="<u8", count=size // 8)):
        raise CheckpointError(f"{path}: checksum mismatch")
    arr = np.frombuffer(data, dtype="<c16", count=nfields * Ny * Nh, offset=HEADER_BYTES).reshape(nfields, Ny, Nh)
    fields = [arr[k].copy() for k in range(nfields)]
    return dict(model=model, precision=precision, Nx=Nx, Ny=Ny, nf=nf, fix_curlB=fix_curlB, step=step, time=time,
                params=dict(zip(PARAM_NAMES, prm)), state=fields[:nf], history=fields[nf:] if flags & 1 else None)
