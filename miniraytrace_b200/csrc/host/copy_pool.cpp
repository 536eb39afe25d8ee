#include "copy_pool.h"

#include <algorithm>
#include <cstring>

namespace mrt {

CopyPool::CopyPool(unsigned workers) {
    m_parts = workers + 1;  // the caller copies one part itself
    for (unsigned i = 0; i < workers; ++i) m_threads.emplace_back([this, i] { run(i + 1); });
}

CopyPool::~CopyPool() {
    {
        std::lock_guard<std::mutex> lock(m_mutex);
        m_stop = true;
    }
    m_wake.notify_all();
    for (std::thread& t : m_threads) t.join();
}

namespace {
void copyPart(char* dst, const char* src, size_t n, unsigned part, unsigned parts) {
    const size_t per = (n + parts - 1) / parts;
    const size_t b = std::min(n, size_t(part) * per), e = std::min(n, b + per);
    if (e > b) std::memcpy(dst + b, src + b, e - b);
}
}  // namespace

void CopyPool::copy(void* dst, const void* src, size_t n) {
    if (m_threads.empty() || n < (size_t(256) << 10)) {
        std::memcpy(dst, src, n);
        return;
    }
    {
        std::lock_guard<std::mutex> lock(m_mutex);
        m_dst = static_cast<char*>(dst);
        m_src = static_cast<const char*>(src);
        m_bytes = n;
        m_pending = unsigned(m_threads.size());
        ++m_generation;
    }
    m_wake.notify_all();
    copyPart(static_cast<char*>(dst), static_cast<const char*>(src), n, 0, m_parts);
    std::unique_lock<std::mutex> lock(m_mutex);
    m_done.wait(lock, [this] { return m_pending == 0; });
}

void CopyPool::run(unsigned id) {
    unsigned long long seen = 0;
    for (;;) {
        char* dst;
        const char* src;
        size_t n;
        {
            std::unique_lock<std::mutex> lock(m_mutex);
            m_wake.wait(lock, [&] { return m_stop || m_generation != seen; });
            if (m_stop) return;
            seen = m_generation;
            dst = m_dst;
            src = m_src;
            n = m_bytes;
        }
        copyPart(dst, src, n, id, m_parts);
        {
            std::lock_guard<std::mutex> lock(m_mutex);
            if (--m_pending == 0) m_done.notify_one();
        }
    }
}

}  // namespace mrt
