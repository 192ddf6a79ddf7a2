"""The C-ABI boundary without a GPU: the library loads, exports every symbol
include/lrt_raster.h declares, its struct layouts match the ctypes mirror,
host-only entry points work, and device entry points fail cleanly."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

import lucabrtrender_b200 as L
from lucabrtrender_b200 import _abi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "lrt_raster.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(lrt_\w+)\s*\(", text, flags=re.M)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = _abi.load()
    assert lib.lrt_abi_version() == _abi.ABI_VERSION
    names = declared_functions()
    assert len(names) >= 10
    assert sorted(names) == sorted(_abi.EXPORTS)
    out = subprocess.run(["nm", "-D", "--defined-only", str(_abi.LIBRARY_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (lrt_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing


PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "lrt_raster.h"
#define S(t) printf(#t " %zu\n", sizeof(t));
#define O(t, f) printf(#t "." #f " %zu\n", offsetof(t, f));
int main(void) {
  S(lrt_projection) O(lrt_projection, eye_world) O(lrt_projection, orthographic)
  S(lrt_lens) S(lrt_camera) O(lrt_camera, lens)
  S(lrt_splat_edit) O(lrt_splat_edit, max_scale)
  S(lrt_gpu_splats) O(lrt_gpu_splats, sh)
  S(lrt_splat_instance) O(lrt_splat_instance, edit)
  S(lrt_render_settings) O(lrt_render_settings, time_stages)
  S(lrt_frame_stats) O(lrt_frame_stats, total_ms)
  S(lrt_targets) S(lrt_debug_view) O(lrt_debug_view, visible)
  S(lrt_train_params) O(lrt_train_params, sh) S(lrt_train_grads) O(lrt_train_grads, sh)
  S(lrt_gpu_points) O(lrt_gpu_points, colours) S(lrt_point_style) O(lrt_point_style, colour)
  S(lrt_point_instance) O(lrt_point_instance, style)
  S(lrt_lod_build_settings) O(lrt_lod_build_settings, chunk_splats)
  S(lrt_lod_info) O(lrt_lod_info, extent) O(lrt_lod_info, level_groups)
  S(lrt_lod_instance) O(lrt_lod_instance, edit) O(lrt_lod_instance, threshold)
  S(lrt_cut_stats) O(lrt_cut_stats, available)
  return 0;
}
"""

CTYPES = {
    "lrt_projection": _abi.Projection, "lrt_lens": _abi.Lens, "lrt_camera": _abi.CameraStruct,
    "lrt_splat_edit": _abi.SplatEdit, "lrt_gpu_splats": _abi.GpuSplatsStruct,
    "lrt_splat_instance": _abi.SplatInstanceStruct, "lrt_render_settings": _abi.RenderSettingsStruct,
    "lrt_frame_stats": _abi.FrameStatsStruct, "lrt_targets": _abi.TargetsStruct, "lrt_debug_view": _abi.DebugView,
    "lrt_train_params": _abi.TrainParams, "lrt_train_grads": _abi.TrainGrads,
    "lrt_gpu_points": _abi.GpuPointsStruct, "lrt_point_style": _abi.PointStyleStruct,
    "lrt_point_instance": _abi.PointInstanceStruct, "lrt_lod_build_settings": _abi.LodBuildSettings,
    "lrt_lod_info": _abi.LodInfo, "lrt_lod_instance": _abi.LodInstanceStruct, "lrt_cut_stats": _abi.CutStatsStruct,
}


def test_struct_layouts_match_the_header(tmp_path):
    src = tmp_path / "probe.c"
    src.write_text(PROBE)
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        name, value = line.split()
        value = int(value)
        if "." in name:
            t, f = name.split(".")
            assert getattr(CTYPES[t], f).offset == value, name
        else:
            assert C.sizeof(CTYPES[name]) == value, name


def test_cpp_host_compiles_against_the_header(tmp_path):
    """A C++ host links the library through the header alone (the binding a
    maintainer adds in the reference's C++ tree)."""
    src = tmp_path / "host.cpp"
    src.write_text(r"""
#include "lrt_raster.h"
#include <cstdio>
int main() {
    lrt_camera cam;
    const double eye[3] = {0, 0, 4}, target[3] = {0, 0, 0}, up[3] = {0, 1, 0};
    if (lrt_camera_looking_at(eye, target, up, &cam) != LRT_OK) return 1;
    lrt_projection p;
    if (lrt_projection_for(&cam, 512, 512, &p) != LRT_OK) return 2;
    std::printf("%.6f %.1f\n", p.focal_x, p.centre_x);
    return lrt_abi_version() == LRT_ABI_VERSION ? 0 : 3;
}
""")
    exe = tmp_path / "host"
    subprocess.run(["g++", "-std=c++17", "-I", str(ROOT / "include"), str(src), "-o", str(exe),
                    str(_abi.LIBRARY_PATH), f"-Wl,-rpath,{_abi.LIBRARY_PATH.parent}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert out.stdout.split() == [f"{512 * 50 / 24.576:.6f}", "256.0"]


def test_host_entry_points_validate_arguments():
    lib = _abi.load()
    kept = C.c_uint32()
    assert lib.lrt_pack_splats(None, 1, 59, 15, 15, None, None, None, C.byref(kept)) == _abi.INVALID_ARGUMENT
    assert lib.lrt_pack_splats(None, 0, 59, 3, 15, None, None, None, C.byref(kept)) == _abi.INVALID_ARGUMENT
    assert lib.lrt_projection_for(None, 1, 1, None) == _abi.INVALID_ARGUMENT
    assert lib.lrt_rast_create(None, 0) == _abi.INVALID_ARGUMENT
    assert lib.lrt_rast_render(None, None, None, 0, None, None, None, None) == _abi.INVALID_ARGUMENT
    assert lib.lrt_math_eval(7, None, None, 0, None) == _abi.INVALID_ARGUMENT
    settings = _abi.LodBuildSettings()
    assert lib.lrt_lod_build_settings_default(C.byref(settings)) == _abi.OK
    assert (round(settings.max_group_fraction, 6), settings.coarsest_level, settings.chunk_splats) == (0.5, 1, 65536)
    assert lib.lrt_lod_build(None, None, None, None, None, None) == _abi.INVALID_ARGUMENT
    assert lib.lrt_lod_select(None, None, None, 0, 0.0, None, None, None, None) == _abi.INVALID_ARGUMENT
    assert lib.lrt_lod_get_info(None, None) == _abi.INVALID_ARGUMENT
    lib.lrt_lod_destroy(None)


def test_device_entry_points_fail_cleanly_without_a_device():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a device is present")
    h = C.c_void_p()
    assert _abi.load().lrt_rast_create(C.byref(h), 0) == _abi.DEVICE_FAILURE
    assert not h.value


@pytest.mark.gpu
def test_cpp_host_renders_a_frame_through_the_header(tmp_path):
    """A C++ host does what the reference-side binding does: packs raw
    records with lrt_pack_splats, copies them into cudaMalloc'd buffers,
    renders one frame with lrt_rast_render into cudaMalloc'd targets and reads
    it back. Its image equals the Python path's bit for bit."""
    import numpy as np
    import torch
    import lucabrtrender_b200 as L

    raw = L.synthetic_records(30_000, 12)
    raw_path = tmp_path / "raw.f32"
    raw.astype(np.float32).tofile(raw_path)
    W, H = 320, 240
    src = tmp_path / "render_host.cpp"
    src.write_text(r"""
#include "lrt_raster.h"
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <vector>
int main(int argc, char** argv) {
    const uint32_t W = 320, H = 240, fpr = 59;
    FILE* f = std::fopen(argv[1], "rb");
    std::vector<float> raw;
    float v;
    while (std::fread(&v, 4, 1, f) == 1) raw.push_back(v);
    std::fclose(f);
    const uint32_t count = static_cast<uint32_t>(raw.size() / fpr);
    const uint32_t words = (15 * 3 + 1) / 2;
    std::vector<float> pos(size_t{count} * 4);
    std::vector<uint32_t> shape(size_t{count} * 4), sh(size_t{count} * words);
    uint32_t kept = 0;
    if (lrt_pack_splats(raw.data(), count, fpr, 15, 15, pos.data(), shape.data(), sh.data(), &kept) != LRT_OK) return 1;
    void *dPos, *dShape, *dSh, *dColour, *dDepth;
    cudaMalloc(&dPos, kept * 16ull);
    cudaMalloc(&dShape, kept * 16ull);
    cudaMalloc(&dSh, kept * 4ull * words);
    cudaMalloc(&dColour, W * H * 16ull);
    cudaMalloc(&dDepth, W * H * 4ull);
    cudaMemcpy(dPos, pos.data(), kept * 16ull, cudaMemcpyHostToDevice);
    cudaMemcpy(dShape, shape.data(), kept * 16ull, cudaMemcpyHostToDevice);
    cudaMemcpy(dSh, sh.data(), kept * 4ull * words, cudaMemcpyHostToDevice);
    lrt_gpu_splats cloud{};
    cloud.count = kept;
    cloud.rest_per_colour = 15;
    cloud.sh_words = words;
    cloud.positions = dPos;
    cloud.shape = dShape;
    cloud.sh = dSh;
    lrt_splat_instance inst{};
    inst.splats = &cloud;
    for (int k = 0; k < 4; ++k) inst.object_to_world[5 * k] = 1.0;
    lrt_camera cam;
    const double eye[3] = {1.0, 0.5, 4.0}, target[3] = {0, 0, 0}, up[3] = {0, 1, 0};
    if (lrt_camera_looking_at(eye, target, up, &cam) != LRT_OK) return 2;
    const double focalPx = (H / 2.0) / std::tan(60.0 * (3.14159265358979323846 / 180.0) / 2.0);
    cam.lens.focal = focalPx * cam.lens.haperture / W;
    cam.lens.near_z = 0.01;
    lrt_projection proj;
    if (lrt_projection_for(&cam, W, H, &proj) != LRT_OK) return 3;
    lrt_render_settings s{};
    s.width = W;
    s.height = H;
    s.antialias = 1;
    s.max_sh_degree = 3;
    s.depth_threshold = 0.5f;
    s.linearise = 1;
    lrt_targets t{W, H, dColour, dDepth};
    lrt_frame_stats stats{};
    lrt_rast* r = nullptr;
    if (lrt_rast_create(&r, 0) != LRT_OK) return 4;
    if (lrt_rast_render(r, &proj, &inst, 1, &s, &t, &stats, nullptr) != LRT_OK) {
        std::fprintf(stderr, "%s\n", lrt_rast_last_error(r));
        return 5;
    }
    std::vector<float> colour(size_t{W} * H * 4);
    cudaMemcpy(colour.data(), dColour, colour.size() * 4, cudaMemcpyDeviceToHost);
    FILE* o = std::fopen(argv[2], "wb");
    std::fwrite(colour.data(), 4, colour.size(), o);
    std::fclose(o);
    std::printf("%u %u %u\n", stats.splats, stats.visible, stats.pairs);
    lrt_rast_destroy(r);
    for (void* p : {dPos, dShape, dSh, dColour, dDepth}) cudaFree(p);
    return 0;
}
""")
    exe = tmp_path / "render_host"
    cuda = "/usr/local/cuda"
    subprocess.run(["g++", "-std=c++17", "-I", str(ROOT / "include"), "-I", f"{cuda}/include", str(src), "-o",
                    str(exe), str(_abi.LIBRARY_PATH), f"-Wl,-rpath,{_abi.LIBRARY_PATH.parent}", f"-L{cuda}/lib64",
                    "-lcudart", f"-Wl,-rpath,{cuda}/lib64"], check=True)
    out_path = tmp_path / "colour.f32"
    run = subprocess.run([str(exe), str(raw_path), str(out_path)], capture_output=True, text=True)
    assert run.returncode == 0, run.stderr
    splats, visible, pairs = map(int, run.stdout.split())
    host_colour = np.fromfile(out_path, np.float32).reshape(H, W, 4)

    packed = L.pack_splats(raw, 15, 3)
    cam = L.square_pixel_camera((1.0, 0.5, 4.0), (0.0, 0.0, 0.0), W, H, 60.0, 0.01)
    r = L.TileRasterizer.create(0)
    try:
        t = L.RenderTargets()
        stats = r.render(cam, [L.SplatInstance(L.to_device(packed))], L.RenderSettings(width=W, height=H), t)
        assert (stats.splats, stats.visible, stats.pairs) == (splats, visible, pairs)
        assert pairs > 0
        assert np.array_equal(t.colour.cpu().numpy().view(np.uint32), host_colour.view(np.uint32))
    finally:
        r.close()
