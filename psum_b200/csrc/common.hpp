// common.hpp -- status codes, error reporting and CUDA helpers shared by the
// B200 backend's translation units.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "../../include/psum_field_solver.h"

namespace psum_b200 {

// Error carrying a psum_status code; converted to a status at the C ABI and
// rethrown as std::runtime_error by the PSuM-compatible func_table entries.
struct Error : public std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);
const std::string& last_error();

// Process-wide count of kernels launched by this library (psum_kernel_launches).
// Kernels enqueued while a stream is being captured into a CUDA graph are
// taken back out (uncount_launches) and counted per graph launch instead.
void count_launch();
void add_launches(unsigned long long n);
void uncount_launches(unsigned long long n);
unsigned long long thread_launches();   // launches counted by the calling thread
// Pinned, device-mapped counter that kernels add to when they start work
// whose launch count the host cannot know in advance (the iterations of a
// conditional graph loop); psum_kernel_launches includes it.
unsigned long long* device_launch_counter();

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(PSUM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Run `f`, translating exceptions into a status code and the thread's last
// error message.
template <class F>
int guarded(F&& f) {
    try {
        f();
        set_last_error("");
        return PSUM_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::invalid_argument& e) {
        set_last_error(e.what());
        return PSUM_ERR_INVALID_ARGUMENT;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return PSUM_ERR_INTERNAL;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return PSUM_ERR_INTERNAL;
    }
}

// Device allocation owned by a host object (cudaMallocAsync-free, plain cudaMalloc).
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            n = o.n;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        if (count == n && p) return;
        release();
        if (count == 0) return;
        cuda_check(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
        n = count;
    }
    void upload(const T* h, size_t count, cudaStream_t s) {
        alloc(count);
        if (count) cuda_check(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s), "cudaMemcpyAsync H2D");
    }
};

}  // namespace psum_b200
