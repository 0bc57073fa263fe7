// Host-only stand-in for Backend/Kernels.h: launch_kernel runs a functor over
// [0, n) serially on the calling thread (the harness parallelises race-free
// functors itself).
#pragma once
#include "Header.h"
#include "MARSException.h"
#include "MARSLogger.h"
#include "Backend/Buffer.h"
#include "Backend/Events.h"
#include "Backend/KernelConfig.h"
#include "Backend/Resource.h"
namespace MARS {
template <typename F>
Event launch_kernel(const Resource&, const KernelConfig& c, F f) {
	for (size_t i = 0; i < c.n; ++i)
		f(i);
	return Event();
}
} // namespace MARS
