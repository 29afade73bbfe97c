// Host-side runtime pieces shared by the C ABI: errors, device buffers.
#pragma once

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>

#include <cuda_runtime.h>

#include "orrery_b200.h"

namespace ob {

// An error that crosses no ABI boundary: caught in the extern "C" layer and
// turned into a status code plus ob_last_error() text.
class Error : public std::runtime_error {
public:
    Error(int code, const std::string &message) : std::runtime_error(message), code_(code) {}
    [[nodiscard]] int code() const noexcept { return code_; }

private:
    int code_;
};

inline void check(cudaError_t err, const char *what) {
    if (err != cudaSuccess) {
        const int code = err == cudaErrorMemoryAllocation ? OB_ERROR_OUT_OF_MEMORY : OB_ERROR_CUDA;
        throw Error(code, std::string(what) + ": " + cudaGetErrorName(err) + " (" +
                              cudaGetErrorString(err) + ")");
    }
}

// Raises `kernel`'s dynamic shared-memory limit to `bytes` on the current
// device. The attribute belongs to each device's context, so it is set once
// per device: `configured` is the caller's per-kernel set of devices done
// (bit d for device d; devices from 64 on are set on every call).
inline cudaError_t set_smem_limit_once(const void *kernel, int bytes,
                                       std::atomic<uint64_t> &configured) {
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) {
        return err;
    }
    const uint64_t bit = device >= 0 && device < 64 ? (1ull << device) : 0ull;
    if (bit != 0 && (configured.load(std::memory_order_acquire) & bit) != 0) {
        return cudaSuccess;
    }
    err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (err == cudaSuccess && bit != 0) {
        configured.fetch_or(bit, std::memory_order_acq_rel);
    }
    return err;
}

// Sets the calling thread's last-error text and returns `code`.
int set_error(int code, const std::string &message);

// Owning device allocation that grows on demand and never shrinks, the
// capacity policy of the reference's CUDA solvers
// (src/solvers/cuda_direct_solver.cpp:120-137).
template <typename T> class DeviceArray {
public:
    DeviceArray() = default;
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    DeviceArray(DeviceArray &&o) noexcept : ptr_(std::exchange(o.ptr_, nullptr)),
                                           count_(std::exchange(o.count_, 0)) {}
    DeviceArray &operator=(DeviceArray &&o) noexcept {
        if (this != &o) {
            release();
            ptr_ = std::exchange(o.ptr_, nullptr);
            count_ = std::exchange(o.count_, 0);
        }
        return *this;
    }
    ~DeviceArray() { release(); }

    // Returns true when the storage moved (callers holding the old pointer,
    // such as captured graphs, must refresh).
    bool reserve(size_t count) {
        if (count <= count_) {
            return false;
        }
        release();
        void *p = nullptr;
        check(cudaMalloc(&p, count * sizeof(T)), "device allocation");
        ptr_ = static_cast<T *>(p);
        count_ = count;
        return true;
    }
    void release() noexcept {
        if (ptr_ != nullptr) {
            cudaFree(ptr_);
        }
        ptr_ = nullptr;
        count_ = 0;
    }
    [[nodiscard]] T *data() const noexcept { return ptr_; }
    [[nodiscard]] size_t size() const noexcept { return count_; }
    [[nodiscard]] size_t bytes() const noexcept { return count_ * sizeof(T); }

private:
    T *ptr_ = nullptr;
    size_t count_ = 0;
};

// Records `event` on `stream`; `external` makes it a real event-record node
// when the stream is being captured into a graph.
inline void record(cudaEvent_t event, cudaStream_t stream, bool external) {
    check(external ? cudaEventRecordWithFlags(event, stream, cudaEventRecordExternal)
                   : cudaEventRecord(event, stream),
          "recording an event");
}

// Device status word of one solver; see common.cuh for the bits.
unsigned read_and_clear_status(unsigned *device_word, cudaStream_t stream);

} // namespace ob
