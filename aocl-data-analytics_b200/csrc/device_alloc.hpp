// The library's device allocation entry (host code).
#pragma once
#include <cuda_runtime.h>
#include <cstdlib>
#include <mutex>
#include <string>

namespace b200 {

// Every device allocation of the library goes through here.  Testing hook:
// while the environment variable AOCLDA_B200_FAIL_ALLOC holds N >= 1, the
// N-th device allocation counted from the moment the variable took that
// value fails as a device out of memory would (no cudaMalloc is made), so
// that tests can drive every allocation failure path of a call.
inline cudaError_t device_alloc(void **p, size_t bytes) {
    static std::mutex mu;
    static std::string armed;
    static long long count = 0;
    const char *env = std::getenv("AOCLDA_B200_FAIL_ALLOC");
    {
        std::lock_guard<std::mutex> lock(mu);
        if (env && *env) {
            if (armed != env) {
                armed = env;
                count = 0;
            }
            const long long n = std::atoll(env);
            if (n >= 1 && ++count == n) {
                *p = nullptr;
                return cudaErrorMemoryAllocation;
            }
        } else if (!armed.empty()) {
            armed.clear();
            count = 0;
        }
    }
    return cudaMalloc(p, bytes);
}

} // namespace b200
