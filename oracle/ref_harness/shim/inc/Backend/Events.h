// Host-only stand-in for Backend/Events.h: launches complete synchronously.
#pragma once
#include "Backend/Resource.h"
#include <vector>
namespace MARS {
class Event {
  public:
	Event() = default;
	Event(std::nullptr_t, const Resource&) {}
	void wait() const {}
};
using EventList = std::vector<Event>;
} // namespace MARS
