// Linux portability shim: SampleBuffer.cpp includes 3d/ConvexPolyhedron.hpp but
// uses nothing from it on the reconstruction path.  Test infrastructure only.
#pragma once
#include "base/Math.hpp"
