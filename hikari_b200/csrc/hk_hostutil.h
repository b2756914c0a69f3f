// Host-side helpers shared by the C-ABI translation units: the error type
// that carries an HK_ERR_* code to the ABI boundary, the CUDA-call check, the
// exception guard of every extern "C" entry point and an owning device buffer.
#pragma once
#include <cuda_runtime.h>

#include <exception>
#include <new>
#include <string>
#include <vector>

#include "../../include/hikari_b200.h"

namespace hk {

struct HkError {
    int code;
    std::string msg;
};

// Records msg as the calling thread's hk_last_error() and returns code.
int set_error(int code, const std::string &msg);

// A failing call's error is reported to the caller and then cleared from the
// runtime's last-error slot (a failed cudaMalloc would otherwise surface again
// at the next launch check of an unrelated call on this thread).
#define HK_CUDA(call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) {                                                                        \
            (void)cudaGetLastError();                                                                   \
            throw ::hk::HkError{e_ == cudaErrorMemoryAllocation ? HK_ERR_NOMEM : HK_ERR_CUDA,           \
                                std::string(#call) + ": " + cudaGetErrorString(e_)};                    \
        }                                                                                               \
    } while (0)

// Runs f and turns every exception into an HK_ERR_* status: nothing throws
// across the C ABI.
template <class F>
int guarded(F &&f) {
    try {
        return f();
    } catch (const HkError &e) {
        return set_error(e.code, e.msg);
    } catch (const std::bad_alloc &) {
        return set_error(HK_ERR_NOMEM, "host allocation failed");
    } catch (const std::exception &e) {
        return set_error(HK_ERR_INVALID, e.what());
    }
}

// Owning device allocation (cudaMalloc / cudaFree).
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    void alloc(size_t n) {
        release();
        if (n == 0) n = 16;
        HK_CUDA(cudaMalloc(&p, n));
        bytes = n;
    }
    template <class T>
    void upload(const std::vector<T> &v) {
        alloc(v.size() * sizeof(T));
        if (!v.empty()) HK_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
    template <class T>
    T *as() const { return (T *)p; }
    // take over o's allocation (o ends empty)
    void take(DevBuf &o) {
        release();
        p = o.p;
        bytes = o.bytes;
        o.p = nullptr;
        o.bytes = 0;
    }
};

// Owning pinned host allocation.
template <class T>
struct PinnedBuf {
    T *p = nullptr;
    size_t n = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf &) = delete;
    PinnedBuf &operator=(const PinnedBuf &) = delete;
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
    void alloc(size_t count) {
        if (p) cudaFreeHost(p);
        p = nullptr;
        HK_CUDA(cudaMallocHost((void **)&p, sizeof(T) * (count ? count : 1)));
        n = count;
    }
};

}  // namespace hk
