// Host-only stand-in for Backend/KernelConfig.h.
#pragma once
#include "Backend/Events.h"
namespace MARS {
struct KernelConfig {
	size_t n{0};
	static KernelConfig for_1d(size_t size_x, const Resource&) { return KernelConfig{size_x}; }
};
} // namespace MARS
