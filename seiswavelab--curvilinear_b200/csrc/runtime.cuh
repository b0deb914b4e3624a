// Runtime helpers shared by the engines: the CUDA error convention (a failure throws
// std::runtime_error("CUDA <action>: <message>") inside the library; the C ABI turns it
// into a status, cf. src/common/CudaSupport.cuh:5-8), device selection scope and RAII
// device/pinned buffers.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>

namespace swl {

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};

inline void check(cudaError_t e, const char *action) {
    if (e != cudaSuccess) throw Error(-2, std::string("CUDA ") + action + ": " + cudaGetErrorString(e));
}

// Makes `device` current for the scope and restores the caller's device afterwards.
struct DeviceScope {
    int previous{-1};
    explicit DeviceScope(int device) {
        check(cudaGetDevice(&previous), "query current device");
        if (previous != device) check(cudaSetDevice(device), "select device");
    }
    ~DeviceScope() {
        if (previous >= 0) cudaSetDevice(previous);
    }
    DeviceScope(const DeviceScope &) = delete;
    DeviceScope &operator=(const DeviceScope &) = delete;
};

// Owning device allocation (zeroed on allocation), from the device's stream-ordered memory pool.
// cudaMalloc / cudaFree synchronise the whole device, which stalls every other shot a server
// runs; an allocation here is made and cleared on the calling thread's stream and waited for, so
// it is usable on any stream, and a release returns the memory to the pool without a device-wide
// synchronisation.  The owner must have finished its own work on the buffer before releasing it
// (the engines synchronise their stream first).
struct DeviceBuffer {
    void *ptr{};
    std::size_t bytes{};
    int device{-1};
    DeviceBuffer() = default;
    explicit DeviceBuffer(std::size_t n) { allocate(n); }
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    DeviceBuffer(DeviceBuffer &&o) noexcept
        : ptr(std::exchange(o.ptr, nullptr)), bytes(std::exchange(o.bytes, 0)), device(std::exchange(o.device, -1)) {}
    DeviceBuffer &operator=(DeviceBuffer &&o) noexcept {
        if (this != &o) {
            release();
            ptr = std::exchange(o.ptr, nullptr);
            bytes = std::exchange(o.bytes, 0);
            device = std::exchange(o.device, -1);
        }
        return *this;
    }
    ~DeviceBuffer() { release(); }
    void allocate(std::size_t n) {
        release();
        if (!n) return;
        check(cudaGetDevice(&device), "query current device");
        cudaError_t e = cudaMallocAsync(&ptr, n, cudaStreamPerThread);
        if (e != cudaSuccess) {
            ptr = nullptr;
            cudaGetLastError();
            throw Error(-3, std::string("CUDA allocate ") + std::to_string(n) + " bytes: " + cudaGetErrorString(e));
        }
        bytes = n;
        check(cudaMemsetAsync(ptr, 0, n, cudaStreamPerThread), "clear allocation");
        check(cudaStreamSynchronize(cudaStreamPerThread), "allocation");
    }
    void release() {
        if (ptr) {
            int current = -1;
            cudaGetDevice(&current);
            if (current != device) cudaSetDevice(device);
            cudaFreeAsync(ptr, cudaStreamPerThread);
            if (current != device && current >= 0) cudaSetDevice(current);
        }
        ptr = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// Page-locked host blocks are kept for reuse instead of being freed: cudaFreeHost synchronises the
// device (stalling every running shot), and cudaMallocHost is slow.  Blocks are handed out first
// fit by size; at most `kPinnedCacheBytes` are kept idle.
void *pinnedTake(std::size_t n, std::size_t &got);
void pinnedGive(void *p, std::size_t n);

// Owning pinned host allocation for asynchronous copies.
struct PinnedBuffer {
    void *ptr{};
    std::size_t bytes{};
    PinnedBuffer() = default;
    PinnedBuffer(const PinnedBuffer &) = delete;
    PinnedBuffer &operator=(const PinnedBuffer &) = delete;
    ~PinnedBuffer() { release(); }
    void reserve(std::size_t n) {
        if (n <= bytes) return;
        release();
        ptr = pinnedTake(n, bytes);
    }
    void release() {
        if (ptr) pinnedGive(ptr, bytes);
        ptr = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// Device with the most global memory among sm_100 devices, or -1.
int selectDevice(int requested);

// The calling thread's last failure message, reported by swl_last_error().
std::string &lastErrorRef();

// The 8-step MacCormack direction table of include/SeisCommon/FiniteDifference.hpp:9-13
// (axis 0 = x, 1 = y, 2 = z), flipped at each RK stage.
inline int direction(int step, int stage, int axis) {
    static const int table[8][3] = {{0, 0, 0}, {1, 1, 0}, {1, 1, 1}, {0, 0, 1},
                                    {0, 1, 0}, {1, 0, 0}, {1, 0, 1}, {0, 1, 1}};
    return (table[step % 8][axis] + stage) % 2;
}

// Ricker wavelet of src/two_d/CurvilinearSolver2D.cpp:31-34.
double ricker(double t, double f);

// A 3D tiled tensor map (no swizzle, zero fill outside the tensor) over `base`: dims[0] is the
// contiguous axis; strides are the byte strides of dims 1 and 2 (multiples of 16); box[0] *
// element size must be a multiple of 16 bytes.  The driver's encoder is reached through the
// runtime's entry-point query, so the library does not link libcuda.
void encodeTensorMap3D(CUtensorMap *map, bool fp64, const void *base, const uint64_t dims[3], const uint64_t strides[2],
                       const uint32_t box[3]);

} // namespace swl
