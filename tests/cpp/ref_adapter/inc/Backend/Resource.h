// Test stand-in for the reference's Backend/Resource.h (src/Backend/Resource.h):
// one CUDA device and one stream, with the accessors the B200 pairlist adapter
// uses (id(), get_stream()) and the one Pairlist.h uses (get_device_memory()).
// The reference's own Resource needs its multi-backend build; this test only
// needs a device id and a stream.
#pragma once
#include "Header.h"
#include <cuda_runtime.h>
#include <cstddef>
#include <string>
namespace MARS {
enum class StreamType { Compute = 0, Memory = 1, GridCompute = 2, Optional = 3 };
class Resource {
  public:
	Resource() = default;
	explicit Resource(short device_id) : id_(device_id) {}
	short id() const { return id_; }
	void* get_stream(StreamType = StreamType::Compute) const { return nullptr; }  // default stream
	size_t get_device_memory() const {
		size_t free_b = 0, total_b = 0;
		cudaSetDevice(id_);
		cudaMemGetInfo(&free_b, &total_b);
		return total_b;
	}
	std::string toString() const { return "cuda:" + std::to_string(id_); }
	void synchronize_streams() const { cudaDeviceSynchronize(); }
	bool operator==(const Resource& o) const { return id_ == o.id_; }

  private:
	short id_ = 0;
};
} // namespace MARS
