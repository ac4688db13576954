// Linux portability shim for framework/gui/Image.hpp.  The reference Image is a
// GL-backed, multi-format pixel container; the reconstruction path only stores
// RGBA float pixels in it (Reconstruction.cpp:221-295 uses getSize, setVec4f,
// getVec4f, flipY) and exports a screenshot (a no-op here).  This headless
// RGBA32F image keeps that interface.
//
// Test infrastructure only (oracle/_ref/).
#pragma once
#include "base/Math.hpp"
#include "base/String.hpp"

namespace FW
{

class Image
{
public:
                    Image       (const Vec2i& size)             { m_size = size; m_pixels = new Vec4f[(size_t)size.x * size.y]; }
                    ~Image      (void)                          { delete[] m_pixels; }

    const Vec2i&    getSize     (void) const                    { return m_size; }
    Vec4f           getVec4f    (const Vec2i& pos) const        { return m_pixels[(size_t)pos.y * m_size.x + pos.x]; }
    void            setVec4f    (const Vec2i& pos, const Vec4f& v) { m_pixels[(size_t)pos.y * m_size.x + pos.x] = v; }
    void            clear       (U32 abgr = 0)                  { (void)abgr; for (size_t i = 0; i < (size_t)m_size.x * m_size.y; i++) m_pixels[i] = Vec4f(0.0f); }
    void            flipY       (void);
    const Vec4f*    getPtr      (void) const                    { return m_pixels; }

private:
                    Image       (const Image&);
    Image&          operator=   (const Image&);

    Vec2i           m_size;
    Vec4f*          m_pixels;
};

void exportImage(const String& fileName, const Image* image);

} // namespace FW
