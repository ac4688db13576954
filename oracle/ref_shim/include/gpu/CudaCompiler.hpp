// Linux portability shim for the reference framework header gpu/CudaCompiler.hpp.
// The reference's GPU-toggle path (reconstruction/ReconstructionCuda.cpp) compiles
// its kernels at run time with the Fermi-era CUDA 4.0 driver API
// (CudaCompiler / CudaModule / Buffer); that runtime is not part of the CPU
// reference build.  These stand-ins let the translation unit compile so that its
// CPU restatement of the GPU algorithm (CudaReconstruction::reconstructCPU*,
// ReconstructionCuda.cpp:261-872) can run; the GPU launch path fails loudly if
// anything reaches it.
//
// Test infrastructure only: compiled into oracle/_ref/.
#pragma once
#include "base/Defs.hpp"
#include "base/Math.hpp"
#include "base/String.hpp"
#include "base/Timer.hpp"

namespace FW
{

class Buffer
{
public:
    Buffer(const void* ptr = NULL, S64 size = 0) { (void)ptr; (void)size; }
    CUdeviceptr getCudaPtr(void) const         { unavailable(); return 0; }
    CUdeviceptr getMutableCudaPtr(void)        { unavailable(); return 0; }
    void*       getMutablePtr(void)            { unavailable(); return NULL; }
    const void* getPtr(void) const             { unavailable(); return NULL; }
    void        clear(void)                    { unavailable(); }
private:
    static void unavailable(void)              { fail("gpu/Buffer is not part of the CPU reference build"); }
};

class CudaModule
{
public:
    static int  getComputeCapability(void)     { return 20; }
    CUfunction  getKernel(const String& name)  { (void)name; return NULL; }
    Buffer&     getGlobal(const String& name)  { (void)name; static Buffer b; return b; }
    void        updateGlobals(void)            {}
    F32         launchKernelTimed(CUfunction k, const Vec2i& block, const Vec2i& grid)
    {
        (void)k; (void)block; (void)grid;
        fail("kernel launches are not part of the CPU reference build");
        return 0.0f;
    }
};

class CudaCompiler
{
public:
    void        setSourceFile(const String& path)                  { (void)path; }
    void        include(const String& path)                        { (void)path; }
    void        define(const String& key, const String& value)     { (void)key; (void)value; }
    CudaModule* compile(void)
    {
        fail("the runtime CUDA compiler is not part of the CPU reference build");
        return NULL;
    }
};

} // namespace FW
