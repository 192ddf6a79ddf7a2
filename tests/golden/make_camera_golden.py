"""Regenerate tests/golden/camera_ref.json from the reference's own camera code.

The reference's modules/render/src/Camera.cpp (with aofx/Transform.h) compiles
here unchanged; ``make -C oracle ref`` builds it from its sources into
oracle/_ref/libref_camera.so behind a C entry point (oracle/ref_camera_shim.cpp).
This script calls it for the camera set-ups the reference's own render tests
use (tests/render/test_splat_render.cpp) plus the benchmark cameras, and
writes what projectionFor returned. Run in a container that has the
reference tree; the JSON it writes is committed so the tests need neither.
"""
import ctypes as C
import json
import math
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
LIB = ROOT / "oracle" / "_ref" / "libref_camera.so"

# (name, eye, target, up, orthographic, focal_mm, window_tx, window_ty, window_sx, window_sy, roll, near, w, h)
CASES = [
    ("perspective", (1.5, 1.0, 6.0), (0, 0, 0), (0, 1, 0), 0, 30.0, 0, 0, 1, 1, 0, 0.1, 250, 190),
    ("frustum_edge", (0.3, -0.2, 2.2), (0, 0, 0), (0, 1, 0), 0, 18.0, 0, 0, 1, 1, 0, 0.1, 250, 190),
    ("orthographic", (0.0, 3.0, 5.0), (0, 0, 0), (0, 1, 0), 1, 5.0, 0, 0, 1, 1, 0, 0.1, 250, 190),
    ("window_roll", (-2.0, 0.5, 5.0), (0, 0, 0), (0, 1, 0), 0, 50.0, 0.2, 0, 1, 1.3, 25.0, 0.1, 250, 190),
    ("two_instances", (2.0, 1.5, 7.0), (0, 0, -0.5), (0, 1, 0), 0, 50.0, 0, 0, 1, 1, 0, 0.1, 250, 190),
    ("straight_down", (0.0, 5.0, 0.0), (0, 0, 0), (0, 1, 0), 0, 35.0, 0, 0, 1, 1, 0, 0.1, 64, 48),
    ("bench_512", (0.0, 0.0, 4.0), (0, 0, 0), (0, 1, 0), 0, 443.40500673763256 * 24.576 / 512, 0, 0, 1, 1, 0, 0.01,
     512, 512),
]
for k in range(20):
    th = 2 * math.pi * k / 20
    CASES.append((f"orbit_{k}", (4 * math.sin(th), 0.0, 4 * math.cos(th)), (0, 0, 0), (0, 1, 0), 0,
                  (540.0 / math.tan(math.radians(30))) * 24.576 / 1920, 0, 0, 1, 1, 0, 0.01, 1920, 1080))


def main() -> None:
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref"], check=True)
    lib = C.CDLL(str(LIB))
    d3 = C.c_double * 3
    lib.ref_camera_projection.argtypes = [d3, d3, d3, C.c_int] + [C.c_double] * 7 + [C.c_uint32, C.c_uint32,
                                                                                       C.c_void_p, C.c_void_p,
                                                                                       C.c_void_p]
    out = []
    for (name, eye, target, up, ortho, focal, tx, ty, sx, sy, roll, near, w, h) in CASES:
        m = (C.c_double * 16)()
        f6 = (C.c_double * 6)()
        e3 = (C.c_double * 3)()
        lib.ref_camera_projection(d3(*eye), d3(*target), d3(*up), ortho, focal, tx, ty, sx, sy, roll, near, w, h,
                                  m, f6, e3)
        out.append(dict(name=name, eye=list(eye), target=list(target), up=list(up), orthographic=ortho,
                        focal=focal, window_translate=[tx, ty], window_scale=[sx, sy], window_roll=roll,
                        near_z=near, width=w, height=h, world_to_view=[float(v).hex() for v in m],
                        focal_centre_near_far=[float(v).hex() for v in f6], eye_world=[float(v).hex() for v in e3]))
    path = Path(__file__).resolve().parent / "camera_ref.json"
    path.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {len(out)} cases to {path}")


if __name__ == "__main__":
    main()
