// Host memory copies split over a few persistent worker threads. One thread
// copies a 4 MB chunk out of pinned staging memory at about 10 GB/s; the
// RGBA32F readback of a 1080p frame (33 MB) needs several threads to stay
// under the reference's 3 ms target while the next chunks arrive by DMA.
#pragma once

#include <condition_variable>
#include <cstddef>
#include <mutex>
#include <thread>
#include <vector>

namespace mrt {

class CopyPool {
public:
    explicit CopyPool(unsigned workers);
    ~CopyPool();
    CopyPool(const CopyPool&) = delete;
    CopyPool& operator=(const CopyPool&) = delete;

    // memcpy(dst, src, n), split into equal parts over the workers and the
    // calling thread; returns when every part is done.
    void copy(void* dst, const void* src, size_t n);

private:
    void run(unsigned id);

    std::vector<std::thread> m_threads;
    std::mutex m_mutex;
    std::condition_variable m_wake, m_done;
    char* m_dst = nullptr;
    const char* m_src = nullptr;
    size_t m_bytes = 0;
    unsigned m_parts = 1;
    unsigned m_pending = 0;
    unsigned long long m_generation = 0;
    bool m_stop = false;
};

}  // namespace mrt
