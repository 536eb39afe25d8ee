// Host-side checks of the copy pool behind readback and staged uploads
// (compiled and run by tests/test_host_cpu.py, no GPU needed): copies of
// sizes below, at and above the threaded threshold, odd sizes and sizes that
// do not divide among the threads equal memcpy byte for byte, back to back
// and with 0 to 7 workers.
#include <cstdio>
#include <cstring>
#include <vector>

#include "copy_pool.h"

int main() {
    int failures = 0;
    const size_t sizes[] = {0, 1, 7, 4096, (size_t(256) << 10) - 1, size_t(256) << 10, (size_t(4) << 20) + 3,
                            (size_t(33) << 20) + 17};
    std::vector<unsigned char> src((size_t(33) << 20) + 64), dst(src.size());
    for (size_t i = 0; i < src.size(); ++i) src[i] = static_cast<unsigned char>(i * 2654435761u >> 13);
    for (unsigned workers = 0; workers < 8; ++workers) {
        mrt::CopyPool pool(workers);
        for (int rep = 0; rep < 2; ++rep)
            for (size_t n : sizes) {
                std::memset(dst.data(), 0xA5, dst.size());
                pool.copy(dst.data() + 1, src.data() + 3, n);  // unaligned on purpose
                const bool ok = std::memcmp(dst.data() + 1, src.data() + 3, n) == 0 && dst[0] == 0xA5 &&
                                dst[1 + n] == 0xA5;
                if (!ok) {
                    std::printf("FAILED workers %u size %zu\n", workers, n);
                    ++failures;
                }
            }
    }
    if (failures == 0) std::printf("ok\n");
    return failures == 0 ? 0 : 1;
}
