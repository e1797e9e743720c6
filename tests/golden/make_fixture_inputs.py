#!/usr/bin/env python3
"""Writes the golden fixture INPUTS from a reference checkout:

    python tests/golden/make_fixture_inputs.py <petbab/fluid-simulation checkout>

(or with WCSPH_REFERENCE_DIR set).

* surface_settled_2048.sphs / tilting_chaotic_2048.sphs: the first 2048
  particles (a Morton-compact chunk) of the reference's shipped snapshots
  measurements/snapshots/{surface_settled,tilting_chaotic}.sphs, written in
  the same .sphs v1 format with the same app_name.
* reference_snapshots.json: header, size, sha256 and the first particle of
  every shipped snapshot (known answers for the snapshot reader).
The dam-break fixture input is generated, not stored (fixtures.py).
"""
from __future__ import annotations

import hashlib
import json
import struct
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def snapshot_dir() -> Path:
    import os

    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WCSPH_REFERENCE_DIR")
    if not root:
        raise SystemExit("usage: make_fixture_inputs.py <reference checkout> (or set WCSPH_REFERENCE_DIR)")
    return Path(root) / "measurements" / "snapshots"


def read_sphs(path: Path):
    raw = path.read_bytes()
    magic, version = raw[:4], struct.unpack("<I", raw[4:8])[0]
    name = raw[8:72].split(b"\0")[0].decode()
    n = struct.unpack("<I", raw[72:76])[0]
    body = np.frombuffer(raw[76:76 + 32 * n], np.float32).reshape(2, n, 4)
    return magic, version, name, n, body[0].copy(), body[1].copy(), raw


def write_sphs(path: Path, name: str, pos: np.ndarray, vel: np.ndarray):
    hdr = b"SPHS" + struct.pack("<I", 1) + name.encode().ljust(64, b"\0") + struct.pack("<I", pos.shape[0])
    path.write_bytes(hdr + pos.astype(np.float32).tobytes() + vel.astype(np.float32).tobytes())


def main():
    info = {}
    for f in sorted(snapshot_dir().glob("*.sphs")):
        magic, version, name, n, pos, vel, raw = read_sphs(f)
        info[f.name] = {"magic": magic.decode(), "version": version, "app_name": name, "fluid_n": n,
                        "bytes": len(raw), "sha256": hashlib.sha256(raw).hexdigest(),
                        "pos0": [float(x) for x in pos[0]], "vel0": [float(x) for x in vel[0]],
                        "pos_min": [float(x) for x in pos[:, :3].min(0)],
                        "pos_max": [float(x) for x in pos[:, :3].max(0)]}
        if f.stem in ("surface_settled", "tilting_chaotic"):
            write_sphs(HERE / f"{f.stem}_2048.sphs", name, pos[:2048], vel[:2048])
    (HERE / "reference_snapshots.json").write_text(json.dumps(info, indent=1) + "\n")
    print("wrote", sorted(p.name for p in HERE.glob("*_2048.sphs")), len(info), "snapshot records")


if __name__ == "__main__":
    main()
