// Handle shared by the reference build's C entry points (ref_driver.cpp,
// ref_gpu_toggle.cpp).  Test infrastructure only.
#pragma once
#include "Reconstruction.hpp"

struct RefHandle
{
    FW::UVTSampleBuffer*    sbuf = nullptr;
    FW::CameraParams*       params = nullptr;
    FW::TreeGather*         tg = nullptr;
};
