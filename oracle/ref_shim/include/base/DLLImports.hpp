// Linux portability shim for the reference framework header base/DLLImports.hpp
// (framework/base/DLLImports.hpp:28-263).  The reference version pulls in
// windows.h, mmsystem.h, shlwapi.h and GL/gl.h; the reconstruction path needs none
// of them.  What the path does need from it is the set of CUDA vector struct types
// (int2, float2, ...) that the framework's Vec classes derive from, and the
// FW_USE_CUDA / FW_USE_GLEW switches.  This header supplies exactly those.
//
// Test infrastructure only: compiled into oracle/_ref/ to run the reference's own
// CPU reconstruction for parity checks and the CPU baseline.
#pragma once
#include "base/Defs.hpp"
#include <stddef.h>
#include <stdio.h>
#include <stdarg.h>
#include <time.h>

#ifndef FW_USE_CUDA
#define FW_USE_CUDA 0
#endif
#define FW_USE_GLEW 0

#define CUDA_VERSION 2010
#define CUDAAPI

typedef enum { CUDA_SUCCESS = 0 } CUresult;
typedef struct { FW::S32 x, y; }        int2;
typedef struct { FW::S32 x, y, z; }     int3;
typedef struct { FW::S32 x, y, z, w; }  int4;
typedef struct { FW::F32 x, y; }        float2;
typedef struct { FW::F32 x, y, z; }     float3;
typedef struct { FW::F32 x, y, z, w; }  float4;
typedef struct { FW::F64 x, y; }        double2;
typedef struct { FW::F64 x, y, z; }     double3;
typedef struct { FW::F64 x, y, z, w; }  double4;

typedef void*   CUfunction;
typedef void*   CUmodule;
typedef int     CUdevice;
typedef size_t  CUdeviceptr;
typedef void*   CUcontext;
typedef void*   CUstream;
typedef void*   CUevent;
typedef void*   CUtexref;
typedef void*   CUsurfref;
typedef size_t  CUsize_t;

typedef unsigned int GLuint;
typedef int          GLint;
typedef unsigned int GLenum;

// Microsoft CRT functions used by framework/base/String.cpp, framework/io/Stream.cpp
// and framework/base/Random.cpp, expressed with their C99/POSIX equivalents.
// The va_list is copied before each use because String::setfv (String.cpp:71-78)
// passes the same va_list to two formatting calls, which the Microsoft CRT
// tolerates and glibc does not.
inline int _vscprintf(const char* fmt, va_list args)
{
    va_list c; va_copy(c, args); int n = vsnprintf(NULL, 0, fmt, c); va_end(c); return n;
}
inline int vsprintf_s(char* buf, size_t size, const char* fmt, va_list args)
{
    va_list c; va_copy(c, args); int n = vsnprintf(buf, size, fmt, c); va_end(c); return n;
}
inline int vsnprintf_s(char* buf, size_t size, size_t count, const char* fmt, va_list args)
{
    va_list c; va_copy(c, args); int n = vsnprintf(buf, (count < size) ? count + 1 : size, fmt, c); va_end(c);
    return (n >= 0 && (size_t)n <= count) ? n : -1;
}
inline int ctime_s(char* buf, size_t size, const time_t* t) { (void)size; return ctime_r(t, buf) ? 0 : 1; }

typedef union { struct { unsigned int LowPart; int HighPart; }; long long QuadPart; } LARGE_INTEGER;
inline int QueryPerformanceCounter(LARGE_INTEGER* c)
{
    struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts);
    c->QuadPart = (long long)ts.tv_sec * 1000000000LL + ts.tv_nsec; return 1;
}
