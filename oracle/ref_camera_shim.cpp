// ORACLE -- test infrastructure. A C entry point over the reference's own
// camera code (modules/render/src/Camera.cpp with
// modules/aofx/sdk/include/aofx/Transform.h), compiled from the reference's
// sources where they lie into oracle/_ref/ by oracle/Makefile. It exists to
// produce golden projection vectors (tests/golden/make_camera_golden.py) that
// pin the restated camera maths in the product and in the oracle.
#include <cstdint>
#include <cstring>

#include "lrt/render/Camera.h"

extern "C" int ref_camera_projection(const double eye[3], const double target[3], const double up[3],
                                     int orthographic, double focal, double window_tx, double window_ty,
                                     double window_sx, double window_sy, double window_roll, double near_z,
                                     uint32_t width, uint32_t height, double* world_to_view16,
                                     double* focal_centre_near_far6, double* eye3) {
    using namespace lrt::render;
    Camera camera = Camera::lookingAt({eye[0], eye[1], eye[2]}, {target[0], target[1], target[2]},
                                      {up[0], up[1], up[2]});
    camera.lens.projection = orthographic ? Lens::Projection::Orthographic : Lens::Projection::Perspective;
    camera.lens.focal = focal;
    camera.lens.windowTranslate[0] = window_tx;
    camera.lens.windowTranslate[1] = window_ty;
    camera.lens.windowScale[0] = window_sx;
    camera.lens.windowScale[1] = window_sy;
    camera.lens.windowRoll = window_roll;
    camera.lens.nearZ = near_z;
    const Projection p = projectionFor(camera, width, height);
    std::memcpy(world_to_view16, p.worldToView.m.data(), 16 * sizeof(double));
    focal_centre_near_far6[0] = p.focalX;
    focal_centre_near_far6[1] = p.focalY;
    focal_centre_near_far6[2] = p.centreX;
    focal_centre_near_far6[3] = p.centreY;
    focal_centre_near_far6[4] = p.nearZ;
    focal_centre_near_far6[5] = p.farZ;
    eye3[0] = p.eyeWorld.x;
    eye3[1] = p.eyeWorld.y;
    eye3[2] = p.eyeWorld.z;
    return 0;
}
