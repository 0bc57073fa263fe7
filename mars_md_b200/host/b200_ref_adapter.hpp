// The B200 pairlist as a strategy of the reference's own Pairlist interface.
//
// Unlike b200_pairlist.hpp (a self-contained mirror of the interface), this
// header is compiled against the reference's headers: it includes
// "PatchOperation/Pairlist.h" and "MARSException.h" from the reference source
// tree and derives from MARS::Pairlist itself (src/PatchOperation/Pairlist.h:
// 56-172). A maintainer adds it to the reference build, returns it from
// create_pairlist (src/PatchOperation/Pairlist.cpp:7-31) for a new
// PairlistBuilderType, and links libmarsb200.so. Every override forwards to
// the C ABI (include/marsb200.h); errors come back as MARS::Exception, as the
// reference's builders throw them.
//
// Include paths: the reference's src/ directory, this repository's include/
// directory, and the reference's Backend layer (or a stand-in exposing
// Resource::id(), Resource::get_stream() and DeviceBuffer<T>::data()/size()/
// resize()).
#pragma once

#include "MARSException.h"
#include "PatchOperation/Pairlist.h"
#include "marsb200.h"

#include <algorithm>
#include <cstdint>

namespace MARS {

class B200PairlistAdapter : public Pairlist {
  public:
	B200PairlistAdapter(const Resource& resource, size_t max_particles, size_t max_pairs_ceiling)
		: Pairlist(resource, max_particles, max_pairs_ceiling) {
		create(max_particles);
	}
	B200PairlistAdapter(const B200PairlistAdapter&) = delete;
	B200PairlistAdapter& operator=(const B200PairlistAdapter&) = delete;
	~B200PairlistAdapter() override {
		if (ctx_) mb2_destroy(ctx_);
	}

	// ZOrderPairlist::build_pairlist (ZOrderPairlist.cpp:102-178): the box and
	// the exclusion view set through the base class are handed to the library
	// at each build, as the reference's builder reads them at each build.
	void build_pairlist(const DeviceBuffer<Vector3>& positions, size_t num_particles,
						float cutoff) override {
		if (num_particles > max_particles_)
			MARS_Exception(ExceptionType::ValueError,
						   "B200 pairlist: %zu particles exceed the capacity of %u", num_particles,
						   static_cast<unsigned>(max_particles_));
		const Vector3& size = box_.get_box_size();
		const Vector3& origin = box_.get_origin();
		const float o[3] = {origin.x, origin.y, origin.z};
		const float s[3] = {size.x, size.y, size.z};
		const int p[3] = {box_.is_periodic(0) ? 1 : 0, box_.is_periodic(1) ? 1 : 0,
						  box_.is_periodic(2) ? 1 : 0};
		check(mb2_set_box(ctx_, o, s, p), "set_periodic_box");
		check(mb2_set_exclusions(ctx_, exclusions_.offsets, exclusions_.excluded,
								 static_cast<uint32_t>(exclusions_.num_particles),
								 exclusions_.rigid_body_id),
			  "set_exclusions");
		uint64_t pairs = 0;
		check(mb2_build_pairlist(ctx_, reinterpret_cast<const float*>(positions.data()), nullptr,
								 static_cast<uint32_t>(num_particles), cutoff, interaction_cutoff_,
								 stream(), &pairs),
			  "build_pairlist");
		if (pairs > max_pairs_ceiling_)
			MARS_Exception(ExceptionType::RuntimeError,
						   "B200 pairlist: %llu pairs exceed the pair-buffer ceiling of %zu",
						   static_cast<unsigned long long>(pairs), max_pairs_ceiling_);
		if (materialize_ && pairs > 0) {
			// The reference's consumers read neighbor_pairs_ (int2, smaller
			// original index first, get_neighbor_pairs()).
			if (!grow_pair_capacity(pairs))
				MARS_Exception(ExceptionType::RuntimeError,
							   "B200 pairlist: cannot grow the pair buffer to %llu pairs",
							   static_cast<unsigned long long>(pairs));
			check(mb2_export_pairs(ctx_, reinterpret_cast<int*>(neighbor_pairs_.data()),
								   neighbor_pairs_.size(), stream()),
				  "get_neighbor_pairs");
		}
		num_particles_ = static_cast<uint32_t>(num_particles);
		num_pairs_ = static_cast<uint32_t>(pairs);
		cutoff_ = cutoff;
		cutoff_squared_ = cutoff * cutoff;
	}

	// ZOrderPairlist::needs_update (ZOrderPairlist.cpp:184-190): largest
	// minimum-image displacement since the last build against skin / 2. The
	// library keeps the snapshot of the last build, so old_positions is not
	// read.
	bool needs_update(const DeviceBuffer<Vector3>& positions, const DeviceBuffer<Vector3>&,
					  size_t num_particles, float skin_distance) const override {
		float max_disp = 0.0f;
		int needs = 1;
		check(mb2_needs_update(ctx_, reinterpret_cast<const float*>(positions.data()),
							   static_cast<uint32_t>(num_particles), skin_distance, stream(),
							   &max_disp, &needs),
			  "needs_update");
		return needs != 0;
	}

	// The strategy this class replaces. A maintainer who registers it under a
	// new enumerator returns that one here instead.
	PairlistBuilderType get_type() const override { return PairlistBuilderType::ZOrder; }
	const char* get_name() const override { return "B200 Z-order pairlist (sm_100a)"; }

	// A larger particle capacity needs a new library context; the box and
	// exclusions are handed over again at the next build.
	void resize(size_t new_max_particles, size_t new_max_pairs) override {
		const size_t old = max_particles_;
		Pairlist::resize(new_max_particles, new_max_pairs);
		if (new_max_particles > old) {
			mb2_destroy(ctx_);
			ctx_ = nullptr;
			create(new_max_particles);
		}
	}

	// The nonbonded cutoff the list serves: with it each row stores the pairs
	// likely to interact first (same pair set, see mb2_build_pairlist).
	void set_interaction_cutoff(float cutoff) { interaction_cutoff_ = cutoff; }
	// Whether each build writes the reference's int2 list into
	// neighbor_pairs_ (default on). A caller whose force stage runs through
	// the library reads the context's own list and may turn it off.
	void set_materialize_pairs(bool on) { materialize_ = on; }
	mb2_context* context() const { return ctx_; }

  private:
	void create(size_t max_particles) {
		check(mb2_create(resource_.id(), static_cast<uint32_t>(std::max<size_t>(max_particles, 1)),
						 &ctx_),
			  "mb2_create");
	}
	void* stream() const { return resource_.get_stream(); }
	void check(int rc, const char* what) const {
		if (rc == MB2_OK) return;
		const char* msg = ctx_ ? mb2_last_error(ctx_) : "no context";
		switch (rc) {
			case MB2_ERR_CUDA:
				MARS_Exception(ExceptionType::CUDARuntimeError, "%s: %s", what, msg);
			case MB2_ERR_ARG:
				MARS_Exception(ExceptionType::ValueError, "%s: %s", what, msg);
			default:
				MARS_Exception(ExceptionType::RuntimeError, "%s: %s", what, msg);
		}
	}

	mb2_context* ctx_ = nullptr;
	float interaction_cutoff_ = 0.0f;
	bool materialize_ = true;
};

}  // namespace MARS
