""".sphs v1 snapshot format and validation order (Snapshot::save/load,
src/cuda/SPH/snapshot.cu:10-106), host-only paths of the C ABI."""
import json
import struct
from pathlib import Path

import numpy as np
import pytest

import wcsph

GOLDEN = Path(__file__).resolve().parent / "golden"


def _state(n=10, seed=0):
    rng = np.random.default_rng(seed)
    pos = rng.random((n, 4)).astype(np.float32)
    pos[:, 3] = 1
    vel = rng.standard_normal((n, 4)).astype(np.float32)
    vel[:, 3] = 0
    return pos, vel


def test_layout_is_byte_exact(tmp_path):
    pos, vel = _state(7)
    f = tmp_path / "a.sphs"
    wcsph.snapshot_write(f, "surface_tension", pos, vel)
    raw = f.read_bytes()
    assert len(raw) == 76 + 32 * 7
    assert raw[:4] == b"SPHS" and struct.unpack("<I", raw[4:8])[0] == 1
    assert raw[8:72] == b"surface_tension".ljust(64, b"\0")
    assert struct.unpack("<I", raw[72:76])[0] == 7
    assert raw[76:76 + 16 * 7] == pos.tobytes() and raw[76 + 16 * 7:] == vel.tobytes()
    p2, v2 = wcsph.snapshot_read(f, "surface_tension", 7)
    assert np.array_equal(p2, pos) and np.array_equal(v2, vel)
    assert wcsph.snapshot_header(f) == ("surface_tension", 7)


def test_app_name_too_long(tmp_path):
    pos, vel = _state(2)
    with pytest.raises(wcsph.SnapshotError) as e:
        wcsph.snapshot_write(tmp_path / "b.sphs", "x" * 64, pos, vel)
    assert "app_name too long (max 63 chars)" in e.value.message
    wcsph.snapshot_write(tmp_path / "c.sphs", "x" * 63, pos, vel)


@pytest.mark.parametrize("case,status,text", [
    ("missing", wcsph.ERR_IO, "cannot open"),
    ("short_header", wcsph.ERR_SNAPSHOT_TRUNCATED, "header read failed"),
    ("magic", wcsph.ERR_SNAPSHOT_MAGIC, "bad magic"),
    ("version", wcsph.ERR_SNAPSHOT_VERSION, "version mismatch (file=2, expected=1)"),
    ("app", wcsph.ERR_SNAPSHOT_APP_NAME, "app_name mismatch (file='other', expected='surface_tension')"),
    ("count", wcsph.ERR_SNAPSHOT_COUNT, "fluid count mismatch (file=5, expected=6)"),
    ("body", wcsph.ERR_SNAPSHOT_TRUNCATED, "body read failed"),
])
def test_load_validation_order(tmp_path, case, status, text):
    pos, vel = _state(6)
    f = tmp_path / "s.sphs"
    wcsph.snapshot_write(f, "surface_tension", pos, vel)
    raw = bytearray(f.read_bytes())
    n_expected = 6
    if case == "missing":
        f = tmp_path / "nope.sphs"
    elif case == "short_header":
        f.write_bytes(bytes(raw[:40]))
    elif case == "magic":
        raw[0:4] = b"SPHX"
        f.write_bytes(bytes(raw))
    elif case == "version":
        raw[4:8] = struct.pack("<I", 2)
        raw[0:4] = b"SPHS"
        f.write_bytes(bytes(raw))
    elif case == "app":
        wcsph.snapshot_write(f, "other", pos, vel)
    elif case == "count":
        wcsph.snapshot_write(f, "surface_tension", pos[:5], vel[:5])
    elif case == "body":
        f.write_bytes(bytes(raw[:-4]))
    with pytest.raises(wcsph.SnapshotError) as e:
        wcsph.snapshot_read(f, "surface_tension", n_expected)
    assert e.value.status == status
    assert text in e.value.message


def test_corrupt_app_name_is_terminated(tmp_path):
    # snapshot.cu:73 forces app_name[63] = 0 before comparing
    pos, vel = _state(3)
    f = tmp_path / "t.sphs"
    wcsph.snapshot_write(f, "a", pos, vel)
    raw = bytearray(f.read_bytes())
    raw[8:72] = b"b" * 64
    f.write_bytes(bytes(raw))
    with pytest.raises(wcsph.SnapshotError) as e:
        wcsph.snapshot_read(f, "a", 3)
    assert "file='" + "b" * 63 + "'" in e.value.message


def test_reference_snapshot_subsets_match_known_answers():
    info = json.loads((GOLDEN / "reference_snapshots.json").read_text())
    assert len(info) == 6 and all(v["bytes"] == 76 + 32 * v["fluid_n"] for v in info.values())
    for stem, app in (("surface_settled", "surface_tension"), ("tilting_chaotic", "tilting_box")):
        rec = info[f"{stem}.sphs"]
        assert rec["app_name"] == app and rec["fluid_n"] == 27000
        pos, vel = wcsph.snapshot_read(GOLDEN / f"{stem}_2048.sphs", app, 2048)
        assert np.array_equal(pos[0], np.float32(rec["pos0"])) and np.array_equal(vel[0], np.float32(rec["vel0"]))
        assert np.all(pos[:, 3] == 1) and np.all(vel[:, 3] == 0)
