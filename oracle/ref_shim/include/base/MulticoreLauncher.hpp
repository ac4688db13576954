// Linux portability shim for framework/base/MulticoreLauncher.hpp:89-139.
// The reference launcher is a Win32 thread pool built on Thread/Monitor/Spinlock.
// This replacement keeps the same public interface (Task, push, pop, popAll,
// getNumCores, setNumThreads) on std::thread: pushed tasks are queued, and
// pop()/popAll() run the queue on a pool of worker threads.  Tasks may push
// further tasks from inside a worker (Sort.cpp's qsortMulticore does).
//
// The thread count defaults to std::thread::hardware_concurrency(); the
// environment variable TLFR_REF_THREADS overrides it.
//
// Test infrastructure only (oracle/_ref/).
#pragma once
#include "base/Hash.hpp"     // the reference header reached Hash.hpp through Thread.hpp
#include "base/Deque.hpp"
#include "base/String.hpp"

namespace FW
{

class MulticoreLauncher
{
public:
    struct Task;
    typedef void (*TaskFunc)(Task& task);

    struct Task
    {
        MulticoreLauncher*  launcher;
        TaskFunc            func;
        void*               data;
        int                 idx;
        void*               result;
    };

                            MulticoreLauncher   (void);
                            ~MulticoreLauncher  (void);

    MulticoreLauncher&      push                (TaskFunc func, void* data, int firstIdx = 0, int numTasks = 1);
    Task                    pop                 (void);

    int                     getNumTasks         (void) const;
    int                     getNumFinished      (void) const;

    void                    popAll              (void);
    void                    popAll              (const String& progressMessage) { (void)progressMessage; popAll(); }

    static int              getNumCores         (void);
    static void             setNumThreads       (int numThreads);

private:
                            MulticoreLauncher   (const MulticoreLauncher&);
    MulticoreLauncher&      operator=           (const MulticoreLauncher&);

    void*                   m_impl;
};

} // namespace FW
