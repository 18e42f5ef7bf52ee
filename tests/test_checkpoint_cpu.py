"""Checkpoint file format on the host (tara2d_b200.checkpoint): round trip,
header layout, and rejection of corrupted, truncated and foreign files.
No GPU needed; the library's own reader and writer are checked against this
module in tests/test_checkpoint_gpu.py."""
import struct

import numpy as np
import pytest

from tara2d_b200 import checkpoint as ck


def fields(n, Ny, Nh, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((Ny, Nh)) + 1j * rng.standard_normal((Ny, Nh)) for _ in range(n)]


def test_round_trip(tmp_path):
    Nx, Ny = 16, 12
    st, hi = fields(3, Ny, Nx // 2 + 1, 1), fields(3, Ny, Nx // 2 + 1, 2)
    p = tmp_path / "a.ck"
    ck.write(p, 1, 0, Nx, Ny, st, hi, step=17, time=1.7e-3, params={"dt": 1e-4, "mux": 2e-4, "lambda": 10.0},
             fix_curlB=1)
    r = ck.read(p)
    assert (r["model"], r["precision"], r["Nx"], r["Ny"], r["nf"], r["fix_curlB"]) == (1, 0, Nx, Ny, 3, 1)
    assert r["step"] == 17 and r["time"] == 1.7e-3
    assert r["params"]["dt"] == 1e-4 and r["params"]["mux"] == 2e-4 and r["params"]["lambda"] == 10.0
    for a, b in zip(r["state"] + r["history"], st + hi):
        assert np.array_equal(a, b)
    assert not (tmp_path / "a.ck.tmp").exists()


def test_without_history(tmp_path):
    p = tmp_path / "b.ck"
    st = fields(6, 8, 9, 3)
    ck.write(p, 2, 1, 16, 8, st)
    r = ck.read(p)
    assert r["history"] is None and all(np.array_equal(a, b) for a, b in zip(r["state"], st))


def test_header_layout(tmp_path):
    """The byte offsets the library's reader and writer use."""
    p = tmp_path / "c.ck"
    ck.write(p, 2, 0, 16, 16, fields(6, 16, 9, 4), fields(6, 16, 9, 5), step=123456789012, time=0.25,
             params={"Lx": 6.5, "lambda": -1.0})
    raw = p.read_bytes()
    assert raw[:8] == b"TARA2DCK"
    assert struct.unpack_from("<I7i", raw, 8) == (1, 2, 0, 16, 16, 6, 0, 1)
    assert struct.unpack_from("<qd", raw, 40) == (123456789012, 0.25)
    assert struct.unpack_from("<d", raw, 56)[0] == 6.5 and struct.unpack_from("<d", raw, 56 + 16 * 8)[0] == -1.0
    assert len(raw) == 192 + 12 * 16 * 9 * 16 + 16


def test_checksum_definition():
    w = np.array([1, 2, 2 ** 63, 2 ** 64 - 1], dtype=np.uint64)
    s1 = (1 + 2 + 2 ** 63 + 2 ** 64 - 1) % 2 ** 64
    s2 = (1 * 1 + 2 * 2 + 3 * 2 ** 63 + 4 * (2 ** 64 - 1)) % 2 ** 64
    assert ck.checksum(w) == (s1, s2)


@pytest.mark.parametrize("where", [0, 100, 191, 192, 1000, -17])
def test_corruption_is_detected(tmp_path, where):
    p = tmp_path / "d.ck"
    ck.write(p, 1, 0, 16, 16, fields(3, 16, 9, 6), fields(3, 16, 9, 7))
    raw = bytearray(p.read_bytes())
    raw[where] ^= 0x10
    p.write_bytes(bytes(raw))
    with pytest.raises(ck.CheckpointError):
        ck.read(p)


def test_truncated_and_foreign_files(tmp_path):
    p = tmp_path / "e.ck"
    ck.write(p, 1, 0, 16, 16, fields(3, 16, 9, 8))
    raw = p.read_bytes()
    p.write_bytes(raw[:-1])
    with pytest.raises(ck.CheckpointError, match="truncated"):
        ck.read(p)
    p.write_bytes(b"NOTACKPT" + raw[8:])
    with pytest.raises(ck.CheckpointError, match="not a checkpoint"):
        ck.read(p)
    with pytest.raises(ck.CheckpointError):
        ck.write(tmp_path / "f.ck", 1, 0, 16, 16, fields(3, 16, 8, 9))  # wrong Nh
