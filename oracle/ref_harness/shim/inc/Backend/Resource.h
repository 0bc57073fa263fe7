// Host-only stand-in for the reference's Backend/Resource.h: the oracle harness
// runs the reference's device functors serially on the CPU, so a resource is
// an empty tag.
#pragma once
#include "Header.h"
#include <cstddef>
#include <string>
namespace MARS {
class Resource {
  public:
	Resource() = default;
	std::string toString() const { return "host"; }
	size_t get_device_memory() const { return size_t(1) << 34; }
	void synchronize_streams() const {}
	bool operator==(const Resource&) const { return true; }
};
} // namespace MARS
