// Linux portability shim for framework/3d/CameraControls.hpp.  CameraParams
// (reconstruction_lib/common/CameraParams.hpp:74-107) embeds a CameraControls
// member; the blurred/pinhole reconstruction path never touches it (only the
// shadow path calls camera.getFar() and the camera matrices, Reconstruction.cpp:
// 374-378, 732).  This stub keeps the constructor signature and those accessors,
// which return what the test driver sets (the GL camera's own state is not
// modelled).
//
// Test infrastructure only (oracle/_ref/).
#pragma once
#include "base/Math.hpp"

namespace FW
{

class CommonControls;

class CameraControls
{
public:
    enum Feature { Feature_Default = 0 };

                    CameraControls  (CommonControls* commonControls = NULL, U32 features = Feature_Default) { (void)commonControls; (void)features; m_far = 1.0e4f; }
    F32             getFar          (void) const    { return m_far; }
    Mat4f           getWorldToCamera(void) const    { return m_worldToCamera; }
    Mat4f           getCameraToWorld(void) const    { return m_cameraToWorld; }

    void            setFar          (F32 f)         { m_far = f; }
    void            setMatrices     (const Mat4f& cameraToWorld, const Mat4f& worldToCamera) { m_cameraToWorld = cameraToWorld; m_worldToCamera = worldToCamera; }

private:
    F32             m_far;
    Mat4f           m_cameraToWorld;
    Mat4f           m_worldToCamera;
};

} // namespace FW
