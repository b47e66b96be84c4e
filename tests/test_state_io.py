"""Restart / snapshot format of read_state.cpp / write_state.cpp (no GPU)."""
import struct

import numpy as np
import pytest

from cudasph_b200 import ics, state_io


def test_roundtrip(tmp_path):
    ic = ics.polytrope(500, seed=2)
    ic["ax"] = np.linspace(-1, 1, 500)
    ic["phi"] = -np.ones(500)
    hdr = state_io.default_header(500, global_time=0.25, dt=1e-3, iteration_number=7)
    path = tmp_path / "restart.bin"
    state_io.write_state(str(path), hdr, ic)
    assert path.stat().st_size == 124 + 23 * 8 * 500
    h2, p2 = state_io.read_state(str(path))
    assert h2["n_bodies"] == 500 and h2["iteration_number"] == 7 and h2["global_time"] == 0.25
    for k in ("x", "y", "z", "vx", "m", "u", "ax", "phi"):
        assert np.array_equal(p2[k], ic[k]), k
    assert np.allclose(p2["range"], ic["range"], rtol=1e-15)
    assert np.allclose(p2["mu"], ic["mu"], rtol=1e-15)
    assert p2["dt"] == 1e-3 and p2["time"] == 0.25


def test_header_field_order(tmp_path):
    """The header is the field-by-field fread sequence of read_state.cpp:5-23."""
    hdr = state_io.default_header(3, nnopt=11, hmin=0.5, hmax=2.5, sep0=3.5, t_end=9.0, dt_out=0.1,
                                  snapshot_number=4, iteration_number=5, global_time=1.5, nav=6, alpha=1.0,
                                  beta=2.0, eta2=0.01, ngr=7, nrelax=8, trelax=1e30, dt=0.002, omega2=0.3)
    p = {k: np.arange(3, dtype=float) + 1 for k in ("x", "y", "z", "m", "range", "vx", "vy", "vz", "u", "mu")}
    path = tmp_path / "s.bin"
    state_io.write_state(str(path), hdr, p)
    raw = path.read_bytes()
    fmt = "<ii ddddd ii d i ddd ii ddd".replace(" ", "")
    vals = struct.unpack(fmt, raw[:struct.calcsize(fmt)])
    assert struct.calcsize(fmt) == 124
    assert vals == (3, 11, 0.5, 2.5, 3.5, 9.0, 0.1, 4, 5, 1.5, 6, 1.0, 2.0, 0.01, 7, 8, 1e30, 0.002, 0.3)
    rec = struct.unpack("<23d", raw[124:124 + 184])
    # x y z m h rho ...: h is range/2 (write_state.cpp:34); aa bb cc = -1; mu in grams
    assert rec[0] == 1.0 and rec[3] == 1.0 and rec[4] == 0.5
    assert rec[19:22] == (-1.0, -1.0, -1.0)
    assert rec[18] == pytest.approx(1.66054e-24)


def test_truncated_file_is_rejected(tmp_path):
    ic = ics.polytrope(50, seed=2)
    path = tmp_path / "t.bin"
    state_io.write_state(str(path), state_io.default_header(50), ic)
    data = path.read_bytes()
    (tmp_path / "cut.bin").write_bytes(data[:-100])
    with pytest.raises(ValueError, match="truncated"):
        state_io.read_state(str(tmp_path / "cut.bin"))
    (tmp_path / "hdr.bin").write_bytes(data[:50])
    with pytest.raises(ValueError, match="truncated header"):
        state_io.read_state(str(tmp_path / "hdr.bin"))
