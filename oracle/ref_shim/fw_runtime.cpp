// Linux runtime for the reference framework pieces that the reconstruction path
// links against, replacing framework/base/Defs.cpp (Win32 allocator hooks,
// profiler, fail()), framework/base/MulticoreLauncher.cpp (Win32 thread pool) and
// the GL-backed gui/Image.cpp.  Behaviour kept from the reference:
//   - FW::malloc/free/realloc are the C allocator (Defs.cpp:81-120 adds only
//     bookkeeping on top).
//   - fail() ends the current operation (Defs.cpp:257-282 shows a message box and
//     exits); here it throws, so that the C entry points in ref_driver.cpp can
//     report an error instead of terminating the test process.
//   - profilePush/Pop are no-ops (profiling is off unless profileStart() is
//     called, Defs.cpp:531-560, and the path never calls it).
//   - MulticoreLauncher runs queued tasks on hardware_concurrency() threads
//     (MulticoreLauncher.cpp:53, 177-180), overridable with TLFR_REF_THREADS.
//
// Test infrastructure only (oracle/_ref/).
#include "base/Defs.hpp"
#include "base/String.hpp"
#include "base/MulticoreLauncher.hpp"
#include "gui/Image.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstdarg>
#include <cstring>
#include <deque>
#include <mutex>
#include <condition_variable>
#include <thread>
#include <vector>
#include <stdexcept>
#include <string>

namespace FW
{

void* malloc(size_t size)               { return ::malloc(size ? size : 1); }
void  free(void* ptr)                   { ::free(ptr); }
void* realloc(void* ptr, size_t size)   { return ::realloc(ptr, size ? size : 1); }

static bool quiet(void)
{
    static int q = -1;
    if (q < 0)
    {
        const char* e = getenv("TLFR_REF_VERBOSE");
        q = (e && e[0] == '1') ? 0 : 1;
    }
    return q == 1;
}

void printf(const char* fmt, ...)
{
    if (quiet())
        return;
    va_list args;
    va_start(args, fmt);
    vfprintf(stdout, fmt, args);
    va_end(args);
}

String sprintf(const char* fmt, ...)
{
    String str;
    va_list args;
    va_start(args, fmt);
    str.setfv(fmt, args);
    va_end(args);
    return str;
}

static String s_error;
static bool   s_hasError = false;

void setError(const char* fmt, ...)
{
    if (s_hasError)
        return;
    va_list args;
    va_start(args, fmt);
    s_error.setfv(fmt, args);
    va_end(args);
    s_hasError = true;
}

String clearError(void)             { String old = s_error; s_error = ""; s_hasError = false; return old; }
bool restoreError(const String& old){ bool had = s_hasError; s_error = old; s_hasError = (old.getLength() != 0); return had; }
bool hasError(void)                 { return s_hasError; }
const String& getError(void)        { return s_error; }

void fail(const char* fmt, ...)
{
    char buf[2048];
    va_list args;
    va_start(args, fmt);
    vsnprintf(buf, sizeof(buf), fmt, args);
    va_end(args);
    throw std::runtime_error(buf);
}

void failWin32Error(const char* funcName)   { fail("%s failed", funcName); }
void failIfError(void)                       { if (s_hasError) fail("%s", s_error.getPtr()); }

int  incNestingLevel(int delta)             { static int level = 0; int old = level; level += delta; return old; }
bool setDiscardEvents(bool discard)         { (void)discard; return false; }
bool getDiscardEvents(void)                 { return false; }

void profileStart(void)                     {}
void profilePush(const char* id)            { (void)id; }
void profilePop(void)                       {}
void profileEnd(bool printResults)          { (void)printResults; }

//------------------------------------------------------------------------
// Image (headless RGBA32F) and screenshot export (no-op).
//------------------------------------------------------------------------

void Image::flipY(void)
{
    for (int y = 0; y < m_size.y / 2; y++)
        for (int x = 0; x < m_size.x; x++)
        {
            Vec4f a = getVec4f(Vec2i(x, y));
            Vec4f b = getVec4f(Vec2i(x, m_size.y - 1 - y));
            setVec4f(Vec2i(x, y), b);
            setVec4f(Vec2i(x, m_size.y - 1 - y), a);
        }
}

void exportImage(const String& fileName, const Image* image) { (void)fileName; (void)image; }

//------------------------------------------------------------------------
// MulticoreLauncher on std::thread.
//------------------------------------------------------------------------

struct LauncherImpl
{
    std::mutex                          lock;
    std::condition_variable             cv;
    std::deque<MulticoreLauncher::Task> pending;
    std::deque<MulticoreLauncher::Task> finished;
    int                                 running = 0;
    std::string                         error;
};

static int s_numThreads = 0;

int MulticoreLauncher::getNumCores(void)
{
    const char* e = getenv("TLFR_REF_THREADS");
    if (e && atoi(e) > 0)
        return atoi(e);
    unsigned n = std::thread::hardware_concurrency();
    return n ? (int)n : 1;
}

void MulticoreLauncher::setNumThreads(int numThreads) { s_numThreads = numThreads; }

MulticoreLauncher::MulticoreLauncher(void)  { m_impl = new LauncherImpl; }
MulticoreLauncher::~MulticoreLauncher(void) { delete (LauncherImpl*)m_impl; }

MulticoreLauncher& MulticoreLauncher::push(TaskFunc func, void* data, int firstIdx, int numTasks)
{
    LauncherImpl* impl = (LauncherImpl*)m_impl;
    std::lock_guard<std::mutex> g(impl->lock);
    for (int i = 0; i < numTasks; i++)
    {
        Task t;
        t.launcher = this;
        t.func = func;
        t.data = data;
        t.idx = firstIdx + i;
        t.result = NULL;
        impl->pending.push_back(t);
    }
    impl->cv.notify_all();
    return *this;
}

int MulticoreLauncher::getNumTasks(void) const
{
    LauncherImpl* impl = (LauncherImpl*)m_impl;
    std::lock_guard<std::mutex> g(impl->lock);
    return (int)(impl->pending.size() + impl->finished.size()) + impl->running;
}

int MulticoreLauncher::getNumFinished(void) const
{
    LauncherImpl* impl = (LauncherImpl*)m_impl;
    std::lock_guard<std::mutex> g(impl->lock);
    return (int)impl->finished.size();
}

void MulticoreLauncher::popAll(void)
{
    LauncherImpl* impl = (LauncherImpl*)m_impl;
    int n = (s_numThreads > 0) ? s_numThreads : getNumCores();

    auto worker = [impl]()
    {
        for (;;)
        {
            Task t;
            {
                std::unique_lock<std::mutex> g(impl->lock);
                impl->cv.wait(g, [impl] { return !impl->pending.empty() || impl->running == 0; });
                if (impl->pending.empty())
                    return;                 // nothing queued and nothing running: done
                t = impl->pending.front();
                impl->pending.pop_front();
                impl->running++;
            }
            try
            {
                t.func(t);
            }
            catch (const std::exception& e)
            {
                std::lock_guard<std::mutex> g(impl->lock);
                if (impl->error.empty())
                    impl->error = e.what();
            }
            {
                std::lock_guard<std::mutex> g(impl->lock);
                impl->running--;
                impl->cv.notify_all();
            }
        }
    };

    std::vector<std::thread> threads;
    for (int i = 0; i < n; i++)
        threads.emplace_back(worker);
    for (auto& th : threads)
        th.join();

    std::string err;
    {
        std::lock_guard<std::mutex> g(impl->lock);
        impl->finished.clear();
        err.swap(impl->error);
    }
    if (!err.empty())
        throw std::runtime_error(err);
}

MulticoreLauncher::Task MulticoreLauncher::pop(void)
{
    LauncherImpl* impl = (LauncherImpl*)m_impl;
    Task t;
    memset(&t, 0, sizeof(t));
    popAll();
    (void)impl;
    return t;
}

} // namespace FW
