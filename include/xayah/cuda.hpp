// xayah::cuda -- device resource and buffers for the C++ host API.
//
// Header-only counterpart of the reference module xayah.cuda
// (solvers/cuda.ixx:7-59, cuda.cpp:11-66): one non-blocking stream plus a
// stream-ordered memory pool per Resource, RAII buffers allocated from it.
// Errors throw std::runtime_error; destructors terminate on CUDA errors, as
// the reference does.  Requires C++20 and the CUDA runtime.
#pragma once

#include <cuda_runtime_api.h>

#include <cstddef>
#include <cstdint>
#include <exception>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

namespace xayah::cuda {

inline void check(cudaError_t status, const char* what) {
    if (status != cudaSuccess) throw std::runtime_error(std::string{what} + ": " + cudaGetErrorString(status));
}

struct Resource {
    Resource() : native_stream(nullptr), memory_pool_(nullptr) {
        int device;
        check(cudaGetDevice(&device), "cudaGetDevice");
        cudaMemPoolProps properties{};
        properties.allocType = cudaMemAllocationTypePinned;
        properties.handleTypes = cudaMemHandleTypeNone;
        properties.location.type = cudaMemLocationTypeDevice;
        properties.location.id = device;
        cudaMemPool_t pool;
        check(cudaMemPoolCreate(&pool, &properties), "cudaMemPoolCreate");
        memory_pool_ = pool;
        std::uint64_t threshold = std::numeric_limits<std::uint64_t>::max();
        check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold), "cudaMemPoolSetAttribute");
        cudaStream_t stream;
        check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
        native_stream = stream;
    }

    ~Resource() noexcept {
        if (cudaStreamSynchronize(stream()) != cudaSuccess) std::terminate();
        if (cudaStreamDestroy(stream()) != cudaSuccess) std::terminate();
        if (cudaMemPoolDestroy(static_cast<cudaMemPool_t>(memory_pool_)) != cudaSuccess) std::terminate();
    }

    Resource(const Resource&) = delete;
    Resource& operator=(const Resource&) = delete;
    Resource(Resource&&) = delete;
    Resource& operator=(Resource&&) = delete;

    [[nodiscard]] void* allocate(std::size_t bytes) {
        void* p;
        check(cudaMallocFromPoolAsync(&p, bytes, static_cast<cudaMemPool_t>(memory_pool_), stream()), "cudaMallocFromPoolAsync");
        return p;
    }
    void release(void* p) noexcept {
        if (cudaFreeAsync(p, stream()) != cudaSuccess) std::terminate();
    }
    void copy_from_host(void* dst, const void* src, std::size_t bytes) {
        check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream()), "copy_from_host");
    }
    void copy_to_host(void* dst, const void* src, std::size_t bytes) {
        check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream()), "copy_to_host");
    }
    void copy_device(void* dst, const void* src, std::size_t bytes) {
        check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream()), "copy_device");
    }
    void zero(void* dst, std::size_t bytes) { check(cudaMemsetAsync(dst, 0, bytes, stream()), "zero"); }
    void synchronize() { check(cudaStreamSynchronize(stream()), "synchronize"); }

    [[nodiscard]] cudaStream_t stream() const { return static_cast<cudaStream_t>(native_stream); }

    void* native_stream;

private:
    void* memory_pool_;
};

template <typename Element>
    requires std::is_trivially_copyable_v<Element>
struct Buffer {
    Buffer() noexcept : data(nullptr), size(0), resource_() {}
    Buffer(std::shared_ptr<Resource> resource, std::size_t n)
        : data(n == 0 ? nullptr : static_cast<Element*>(resource->allocate(n * sizeof(Element)))), size(n), resource_(std::move(resource)) {}
    ~Buffer() noexcept {
        if (data != nullptr) resource_->release(data);
    }
    Buffer(const Buffer&) = delete;
    Buffer& operator=(const Buffer&) = delete;
    Buffer(Buffer&& o) noexcept : data(std::exchange(o.data, nullptr)), size(std::exchange(o.size, 0u)), resource_(std::move(o.resource_)) {}
    Buffer& operator=(Buffer&& o) noexcept {
        if (this != &o) {
            if (data != nullptr) resource_->release(data);
            resource_ = std::move(o.resource_);
            data = std::exchange(o.data, nullptr);
            size = std::exchange(o.size, 0u);
        }
        return *this;
    }

    Element* data;
    std::size_t size;

private:
    std::shared_ptr<Resource> resource_;
};

}  // namespace xayah::cuda
