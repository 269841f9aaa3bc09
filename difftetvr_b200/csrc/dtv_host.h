// Host-side helpers shared by the C-ABI translation units: status codes as
// exceptions, the guarded call wrapper, grow-only device buffers.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <cuda_runtime.h>
#include "difftetvr_b200.h"

void dtv_set_last_error(const std::string& msg);

namespace dtv_host {

using u64 = unsigned long long;

struct DtvError : std::runtime_error {
    int32_t code;
    DtvError(int32_t c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define DTV_CK(expr)                                                                                   \
    do {                                                                                               \
        cudaError_t err__ = (expr);                                                                    \
        if (err__ != cudaSuccess)                                                                      \
            throw dtv_host::DtvError(DTV_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(err__)); \
    } while (0)

inline void check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw DtvError(DTV_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class F>
int32_t guarded(F&& fn) {
    try {
        fn();
        return DTV_OK;
    } catch (const DtvError& e) {
        dtv_set_last_error(e.what());
        return e.code;
    } catch (const std::invalid_argument& e) {
        dtv_set_last_error(e.what());
        return DTV_ERR_ARG;
    } catch (const std::bad_alloc&) {
        dtv_set_last_error("host allocation failed");
        return DTV_ERR_BUDGET;
    } catch (const std::exception& e) {
        dtv_set_last_error(e.what());
        return DTV_ERR_STATE;
    }
}

inline void require(bool cond, const char* msg) {
    if (!cond) throw DtvError(DTV_ERR_ARG, msg);
}

// Grow-only device buffer.
template <class T>
struct DevBuf {
    T* ptr = nullptr;
    size_t cap = 0;
    bool ensure(size_t n, cudaStream_t s, bool zero_new = false, double headroom = 1.0) {
        if (n <= cap && ptr) return false;
        if (ptr) {
            DTV_CK(cudaStreamSynchronize(s));
            DTV_CK(cudaFree(ptr));
            ptr = nullptr;
            cap = 0;
        }
        size_t want = size_t(double(n) * headroom);
        if (want < n) want = n;
        if (want == 0) want = 1;
        cudaError_t e = cudaMalloc(&ptr, want * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            ptr = nullptr;
            throw DtvError(DTV_ERR_BUDGET, "device allocation of " + std::to_string(want * sizeof(T)) +
                                               " bytes failed: " + cudaGetErrorString(e));
        }
        cap = want;
        if (zero_new) DTV_CK(cudaMemsetAsync(ptr, 0, want * sizeof(T), s));
        return true;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
    }
};

}  // namespace dtv_host
