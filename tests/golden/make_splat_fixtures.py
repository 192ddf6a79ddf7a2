"""Writes tests/golden/splat_fixtures.json from the reference's own splat
fixtures, tests/data/splats/tiny.ply (64 splats, degree 0) and sh3.ply (64
splats, degree 3), in the lucabRTrender tree.

Each file's binary little-endian float properties are read by name and laid
out as this library's raw records (the 3DGS PLY encoding of lrt_pack_splats:
x y z, logit opacity, three log scales, rotation w x y z, three DC, then the
rest coefficients all red, then green, then blue), stored as base64 float32.
The reference tree is read only here; the tests use the JSON.

    python tests/golden/make_splat_fixtures.py <reference root>
"""
from __future__ import annotations

import base64
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def read_ply(path: Path) -> dict[str, np.ndarray]:
    data = path.read_bytes()
    end = data.index(b"end_header\n") + len(b"end_header\n")
    header = data[:end].decode("ascii").splitlines()
    assert "format binary_little_endian 1.0" in header
    count = 0
    names = []
    for line in header:
        parts = line.split()
        if parts[:2] == ["element", "vertex"]:
            count = int(parts[2])
        elif parts[:2] == ["property", "float"]:
            names.append(parts[2])
    table = np.frombuffer(data[end:end + 4 * count * len(names)], dtype="<f4").reshape(count, len(names))
    return {n: table[:, k].copy() for k, n in enumerate(names)}


def records(fields: dict[str, np.ndarray]) -> tuple[np.ndarray, int]:
    rest = sum(1 for n in fields if n.startswith("f_rest_"))
    per_colour = rest // 3
    order = ["x", "y", "z", "opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3",
             "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{k}" for k in range(rest)]
    out = np.stack([fields[n] for n in order], axis=1).astype(np.float32)
    return out, per_colour


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_splat_fixtures.py <reference root>")
    root = Path(sys.argv[1])
    out = {}
    for name in ("tiny", "sh3"):
        recs, per_colour = records(read_ply(root / "tests" / "data" / "splats" / f"{name}.ply"))
        out[name] = {"source": f"tests/data/splats/{name}.ply", "count": int(recs.shape[0]),
                     "rest_per_colour": per_colour, "floats_per_record": int(recs.shape[1]),
                     "records_f32_base64": base64.b64encode(recs.tobytes()).decode("ascii")}
    (HERE / "splat_fixtures.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
