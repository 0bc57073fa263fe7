// Test stand-in for the reference's Backend/Buffer.h (DeviceBuffer =
// Buffer<T, BackendPolicy>, src/Backend/Buffer.h): device memory from
// cudaMalloc, with the members Pairlist.h and the adapter test use.
#pragma once
#include "Backend/Resource.h"
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#include <utility>
#include <vector>
namespace MARS {
// The memory calls Types/Bitmask.h makes through BackendPolicy, on the CUDA device.
struct BackendPolicy {
	static void* allocate(const Resource&, size_t n) {
		void* p = nullptr;
		return cudaMalloc(&p, n) == cudaSuccess ? p : nullptr;
	}
	static void deallocate(void* p) { cudaFree(p); }
	static void copy_from_host(void* dst, const void* src, size_t n) {
		cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice);
	}
	static void copy_to_host(void* dst, const void* src, size_t n) {
		cudaMemcpy(dst, src, n, cudaMemcpyDeviceToHost);
	}
};
template <typename T>
class DeviceBuffer {
  public:
	DeviceBuffer() = default;
	explicit DeviceBuffer(size_t n, const Resource& = Resource()) { resize(n); }
	DeviceBuffer(const DeviceBuffer&) = delete;
	DeviceBuffer& operator=(const DeviceBuffer&) = delete;
	DeviceBuffer(DeviceBuffer&& o) noexcept { swap(o); }
	DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
		swap(o);
		return *this;
	}
	~DeviceBuffer() {
		if (p_) cudaFree(p_);
	}
	T* data() { return p_; }
	const T* data() const { return p_; }
	size_t size() const { return n_; }
	bool empty() const { return n_ == 0; }
	void resize(size_t n) {
		if (n == n_) return;
		T* q = nullptr;
		if (n && cudaMalloc(reinterpret_cast<void**>(&q), n * sizeof(T)) != cudaSuccess) {
			std::fprintf(stderr, "DeviceBuffer: cudaMalloc of %zu bytes failed\n", n * sizeof(T));
			std::abort();
		}
		if (p_ && q) cudaMemcpy(q, p_, (n < n_ ? n : n_) * sizeof(T), cudaMemcpyDeviceToDevice);
		if (p_) cudaFree(p_);
		p_ = q;
		n_ = n;
	}
	void copy_from_host(const T* src, size_t n, bool = false) {
		if (n > n_) resize(n);
		cudaMemcpy(p_, src, n * sizeof(T), cudaMemcpyHostToDevice);
	}
	void copy_to_host(T* dst, size_t n, bool = false) const {
		cudaMemcpy(dst, p_, n * sizeof(T), cudaMemcpyDeviceToHost);
	}
	void copy_to_host_sync(T* dst, size_t n) const { copy_to_host(dst, n); }
	void copy_to_host(std::vector<T>& dst) const {
		dst.resize(n_);
		copy_to_host(dst.data(), n_);
	}

  private:
	void swap(DeviceBuffer& o) {
		std::swap(p_, o.p_);
		std::swap(n_, o.n_);
	}
	T* p_ = nullptr;
	size_t n_ = 0;
};
} // namespace MARS
