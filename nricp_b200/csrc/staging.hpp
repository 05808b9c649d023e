// Page-locked host memory for bulk copies between host and device: one
// buffer per process, grown on demand and kept (never freed, so that no free
// runs after the CUDA runtime has shut down); one lease holds it at a time.
#pragma once

#include <cstddef>
#include <mutex>

#include <cuda_runtime.h>

namespace nricp_b200 {

class StagingLease {
public:
    explicit StagingLease(size_t bytes) : lock_(mutex()) {
        if (bytes > capacity()) {
            if (buffer()) cudaFreeHost(buffer());
            buffer() = nullptr;
            capacity() = 0;
            const size_t grown = bytes + bytes / 4;
            if (cudaHostAlloc(&buffer(), grown, cudaHostAllocDefault) != cudaSuccess) {
                buffer() = nullptr;
                throw std::bad_alloc();
            }
            capacity() = grown;
        }
    }
    char* data() const { return static_cast<char*>(buffer()); }

private:
    static std::mutex& mutex() {
        static std::mutex m;
        return m;
    }
    static void*& buffer() {
        static void* p = nullptr;
        return p;
    }
    static size_t& capacity() {
        static size_t c = 0;
        return c;
    }
    std::unique_lock<std::mutex> lock_;
};

}  // namespace nricp_b200
