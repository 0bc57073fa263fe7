// Host-only stand-in for Backend/Buffer.h: "device" memory is host memory.
#pragma once
#include "Backend/Resource.h"
#include <cstdlib>
#include <cstring>
#include <vector>
namespace MARS {
struct BackendPolicy {
	static void* allocate(const Resource&, size_t n) { return std::malloc(n); }
	static void deallocate(void* p) { std::free(p); }
	static void copy_from_host(void* dst, const void* src, size_t n) { std::memcpy(dst, src, n); }
	static void copy_to_host(void* dst, const void* src, size_t n) { std::memcpy(dst, src, n); }
};
template <typename T>
class DeviceBuffer {
  public:
	DeviceBuffer() = default;
	DeviceBuffer(size_t n, const Resource& = Resource()) : v_(n) {}
	T* data() { return v_.data(); }
	const T* data() const { return v_.data(); }
	size_t size() const { return v_.size(); }
	bool empty() const { return v_.empty(); }
	void resize(size_t n) { v_.resize(n); }
	void copy_from_host(const T* src, size_t n, bool = false) { std::memcpy(v_.data(), src, n * sizeof(T)); }
	void copy_to_host(T* dst, size_t n, bool = false) const { std::memcpy(dst, v_.data(), n * sizeof(T)); }
	void copy_to_host_sync(T* dst, size_t n) const { copy_to_host(dst, n); }
	void copy_to_host(std::vector<T>& dst) const { dst = v_; }
	void fill(const T& v, bool = false) { for (auto& x : v_) x = v; }
  private:
	std::vector<T> v_;
};
} // namespace MARS
