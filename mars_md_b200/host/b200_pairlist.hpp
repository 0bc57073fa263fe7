// C++ host interface over libmarsb200 (include/marsb200.h) that mirrors the
// reference's plug-in points on the BD force-and-integrate path, so a caller
// of the reference can swap it in with the same names, argument meanings and
// error behaviour:
//
//   * Pairlist: the pairlist strategy interface
//     (src/PatchOperation/Pairlist.h:56-252) -- build_pairlist, update_pairlist,
//     needs_update, set_periodic_box, set_exclusions, get_neighbor_pairs,
//     get_num_pairs, get_cutoff, get_type, get_name, resize, get_statistics;
//   * B200Pairlist: a Pairlist backed by the B200 context, registered in
//     create_pairlist (src/PatchOperation/Pairlist.cpp:7-31) under
//     PairlistBuilderType::B200;
//   * B200Patch: the three Patch stages on this path
//     (src/PatchOperation/Patch.h:222-287, Patch.cpp:43-352) --
//     calculate_nonbonded_forces (rebuild schedule + skin check + pair
//     forces), calculate_bonded_forces, integrate_motion (BD or Langevin
//     BAOAB with the deferred closing kick), finish_deferred_kick and
//     reorder_particles (with ExclusionCSR and ParticleReorderManager);
//   * SimOutput: SimManager's DCD, energy and restart output.
//
// Errors are thrown as marsb200::Exception carrying the library's message,
// as the reference throws MARS::Exception; the C ABI underneath never throws.
// Device buffers are caller-owned and passed through as raw pointers, as the
// reference's DeviceBuffer<T>::data() pointers are.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "marsb200.h"

namespace marsb200 {

enum class ExceptionType {
	ValueError,
	CUDAError,
	CapacityError,
	StateError,
	NotImplementedError,
	FileIoError
};

class Exception : public std::runtime_error {
  public:
	Exception(ExceptionType type, const std::string& msg) : std::runtime_error(msg), type_(type) {}
	ExceptionType type() const { return type_; }

  private:
	ExceptionType type_;
};

// Status code of a C-ABI call -> exception (MB2_OK returns).
inline void check(int rc, const mb2_context* ctx, const char* what) {
	if (rc == MB2_OK) return;
	const std::string msg = std::string(what) + ": " + (ctx ? mb2_last_error(ctx) : "no context");
	switch (rc) {
		case MB2_ERR_CUDA: throw Exception(ExceptionType::CUDAError, msg);
		case MB2_ERR_CAPACITY: throw Exception(ExceptionType::CapacityError, msg);
		case MB2_ERR_STATE: throw Exception(ExceptionType::StateError, msg);
		case MB2_ERR_IO: throw Exception(ExceptionType::FileIoError, msg);
		default: throw Exception(ExceptionType::ValueError, msg);
	}
}

inline void cuda_check(cudaError_t e, const char* what) {
	if (e != cudaSuccess)
		throw Exception(ExceptionType::CUDAError, std::string(what) + ": " + cudaGetErrorString(e));
}

// 16-byte vector as the reference stores positions and ForceEnergy
// (src/Types/Vector3.h:41): x, y, z and a fourth word (energy in ForceEnergy).
struct alignas(16) Vector3 {
	float x = 0.0f, y = 0.0f, z = 0.0f, t = 0.0f;
	Vector3() = default;
	Vector3(float x_, float y_, float z_, float t_ = 0.0f) : x(x_), y(y_), z(z_), t(t_) {}
};
static_assert(sizeof(Vector3) == 16, "float4 layout");

// Device and stream a component runs on (the reference's Resource).
struct Resource {
	int device = 0;
	cudaStream_t stream = nullptr;
};

// Owning device array (the reference's DeviceBuffer<T>: data(), size(),
// resize(), copy_from_host(), copy_to_host()).
template <typename T>
class DeviceBuffer {
  public:
	DeviceBuffer() = default;
	explicit DeviceBuffer(size_t count, const Resource& r = Resource{}) : res_(r) { resize(count); }
	DeviceBuffer(const DeviceBuffer&) = delete;
	DeviceBuffer& operator=(const DeviceBuffer&) = delete;
	DeviceBuffer(DeviceBuffer&& o) noexcept { swap(o); }
	DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
		swap(o);
		return *this;
	}
	~DeviceBuffer() {
		if (ptr_) cudaFree(ptr_);
	}
	void resize(size_t count) {
		if (count == count_) return;
		if (ptr_) cuda_check(cudaFree(ptr_), "DeviceBuffer::resize");
		ptr_ = nullptr;
		count_ = 0;
		if (count) {
			cuda_check(cudaSetDevice(res_.device), "DeviceBuffer::resize");
			cuda_check(cudaMalloc(&ptr_, count * sizeof(T)), "DeviceBuffer::resize");
		}
		count_ = count;
	}
	T* data() { return ptr_; }
	const T* data() const { return ptr_; }
	size_t size() const { return count_; }
	void copy_from_host(const T* src, size_t n, bool sync = true) {
		cuda_check(cudaMemcpyAsync(ptr_, src, n * sizeof(T), cudaMemcpyHostToDevice, res_.stream),
				   "DeviceBuffer::copy_from_host");
		if (sync) cuda_check(cudaStreamSynchronize(res_.stream), "DeviceBuffer::copy_from_host");
	}
	void copy_from_host(const std::vector<T>& src) {
		if (src.size() > count_) resize(src.size());
		copy_from_host(src.data(), src.size(), true);
	}
	void copy_to_host(T* dst, size_t n, bool sync = true) const {
		cuda_check(cudaMemcpyAsync(dst, ptr_, n * sizeof(T), cudaMemcpyDeviceToHost, res_.stream),
				   "DeviceBuffer::copy_to_host");
		if (sync) cuda_check(cudaStreamSynchronize(res_.stream), "DeviceBuffer::copy_to_host");
	}
	void copy_to_host(std::vector<T>& dst) const {
		dst.resize(count_);
		copy_to_host(dst.data(), count_, true);
	}
	void copy_to_host_sync(T* dst, size_t n) const { copy_to_host(dst, n, true); }
	void fill_zero() {
		if (count_)
			cuda_check(cudaMemsetAsync(ptr_, 0, count_ * sizeof(T), res_.stream),
					   "DeviceBuffer::fill_zero");
	}

  private:
	void swap(DeviceBuffer& o) noexcept {
		std::swap(ptr_, o.ptr_);
		std::swap(count_, o.count_);
		std::swap(res_, o.res_);
	}
	T* ptr_ = nullptr;
	size_t count_ = 0;
	Resource res_{};
};

// Simulation box: origin, edge lengths and per-axis periodicity
// (src/System/PeriodicBox.h:120-126 constructor arguments).
class PeriodicBox {
  public:
	PeriodicBox() = default;
	PeriodicBox(const Vector3& origin, const Vector3& size, bool px = true, bool py = true,
				bool pz = true)
		: origin_(origin), size_(size), periodic_{px, py, pz} {}
	const Vector3& get_origin() const { return origin_; }
	const Vector3& get_size() const { return size_; }
	bool is_periodic(int dim) const { return periodic_[dim]; }

  private:
	Vector3 origin_{0, 0, 0};
	Vector3 size_{0, 0, 0};
	bool periodic_[3] = {true, true, true};
};

// Borrowed device view of the exclusion CSR (src/Interactions/DeviceExclusions.h:22-75):
// offsets has num_particles + 1 entries; rigid_body_id may be null.
struct ExclusionView {
	const int* offsets = nullptr;
	const int* excluded = nullptr;
	uint32_t num_particles = 0;
	const int* rigid_body_id = nullptr;
};

// Exclusion CSR built on the host from excluded pairs and owned on the device,
// as DeviceBondedInteractions builds it (rebuild_exclusions_after_reorder,
// src/Interactions/DeviceBondedInteraction.h:385-430): pairs canonicalised
// (a < b) and sorted, offsets over 0 .. max index + 1, each particle's
// neighbours in sorted-pair order.
class ExclusionCSR {
  public:
	void build(std::vector<std::pair<int, int>> pairs, const Resource& r = Resource{}) {
		res_ = r;
		for (auto& e : pairs)
			if (e.first > e.second) std::swap(e.first, e.second);
		std::sort(pairs.begin(), pairs.end());
		pairs_ = std::move(pairs);
		num_ = 0;
		if (pairs_.empty()) return;
		int max_idx = 0;
		for (const auto& e : pairs_) max_idx = std::max(max_idx, e.second);
		num_ = static_cast<uint32_t>(max_idx) + 1;
		std::vector<int> off(num_ + 1, 0);
		for (const auto& e : pairs_) {
			off[e.first + 1]++;
			off[e.second + 1]++;
		}
		for (uint32_t p = 0; p < num_; ++p) off[p + 1] += off[p];
		std::vector<int> nb(off[num_]);
		std::vector<int> cur(off.begin(), off.end() - 1);
		for (const auto& e : pairs_) {
			nb[cur[e.first]++] = e.second;
			nb[cur[e.second]++] = e.first;
		}
		offsets_ = DeviceBuffer<int>(off.size(), res_);
		offsets_.copy_from_host(off);
		neighbors_ = DeviceBuffer<int>(std::max<size_t>(nb.size(), 1), res_);
		neighbors_.copy_from_host(nb.data(), nb.size());
	}
	// Endpoints through the old -> new map, then the CSR rebuilt.
	void remap(const std::vector<uint32_t>& inverse) {
		std::vector<std::pair<int, int>> p = pairs_;
		for (auto& e : p) {
			e.first = static_cast<int>(inverse.at(static_cast<size_t>(e.first)));
			e.second = static_cast<int>(inverse.at(static_cast<size_t>(e.second)));
		}
		build(std::move(p), res_);
	}
	ExclusionView view(const int* rigid_body_id = nullptr) const {
		return ExclusionView{num_ ? offsets_.data() : nullptr, num_ ? neighbors_.data() : nullptr,
							 num_, rigid_body_id};
	}
	const std::vector<std::pair<int, int>>& pairs() const { return pairs_; }
	uint32_t num_particles() const { return num_; }

  private:
	std::vector<std::pair<int, int>> pairs_;
	DeviceBuffer<int> offsets_, neighbors_;
	uint32_t num_ = 0;
	Resource res_{};
};

// Per-particle device arrays a reorder permutes: the members DeviceParticle::permute
// gathers (src/Objects/DeviceParticleManager.h:186-208). Null members are skipped;
// force/energy is cleared every step and is not permuted.
struct ParticleArrays {
	Vector3* pos = nullptr;
	Vector3* mom = nullptr;
	Vector3* orient = nullptr;
	int* id = nullptr;
	int* type_id = nullptr;
	uint32_t* flags = nullptr;
	int* attached_rigid_body_id = nullptr;
};

// Device particle indices a reorder remaps (DeviceBondedInteractions::
// remap_particle_indices, src/Interactions/DeviceBondedInteraction.h:364-380).
struct BondedIndices {
	int* bonds2 = nullptr;  // int2 per bond
	size_t num_bonds = 0;
	int* angles4 = nullptr;  // int4 per angle (fourth word unused)
	size_t num_angles = 0;
	int* dihedrals4 = nullptr;  // int4 per dihedral
	size_t num_dihedrals = 0;
	int* restraint_ids = nullptr;  // one particle per restraint
	size_t num_restraints = 0;
};

// ParticleReorderManager::maybe_reorder (src/PatchOperation/ReorderManager.cpp:8-25):
// steps 1, 1 + period, ... once the bonded topology is on the device; a
// period <= 0 falls back to the pairlist rebuild period (SimManager.cpp:345-349).
class ParticleReorderManager {
  public:
	explicit ParticleReorderManager(int reorder_period, size_t rebuild_period = 0)
		: period_(reorder_period > 0 ? static_cast<size_t>(reorder_period) : rebuild_period) {}
	bool should_reorder(size_t step, bool bonded_prepared = true) const {
		if (period_ == 0 || step == 0) return false;
		if ((step - 1) % period_ != 0) return false;
		return bonded_prepared;
	}
	size_t period() const { return period_; }

  private:
	size_t period_;
};

// Pairlist strategies (src/PatchOperation/Pairlist.h:38-43) plus this one.
enum class PairlistBuilderType { ZOrder, CellList, VerletList, Hierarchical, B200 };

// The pairlist strategy interface (src/PatchOperation/Pairlist.h:56-252).
class Pairlist {
  public:
	struct Statistics {
		size_t num_particles;
		size_t num_pairs;
		float cutoff;
		float average_neighbors_per_particle;
		size_t max_neighbors_per_particle;
		double build_time_ms;
	};
	Pairlist(const Resource& resource, size_t max_particles, size_t max_pairs_ceiling)
		: resource_(resource), max_particles_(max_particles), max_pairs_ceiling_(max_pairs_ceiling) {}
	virtual ~Pairlist() = default;
	virtual void build_pairlist(const DeviceBuffer<Vector3>& positions, size_t num_particles,
								float cutoff) = 0;
	virtual void update_pairlist(const DeviceBuffer<Vector3>& positions, size_t num_particles) {
		build_pairlist(positions, num_particles, cutoff_);
	}
	virtual bool needs_update(const DeviceBuffer<Vector3>& positions,
							  const DeviceBuffer<Vector3>& old_positions, size_t num_particles,
							  float skin_distance) const = 0;
	virtual void set_periodic_box(const PeriodicBox& box) { box_ = box; }
	virtual void set_exclusions(const ExclusionView& exclusions) { exclusions_ = exclusions; }
	// Pairs in the reference's format: int2(min, max) of original indices.
	virtual const DeviceBuffer<int2>& get_neighbor_pairs() const = 0;
	size_t get_num_pairs() const { return num_pairs_; }
	float get_cutoff() const { return cutoff_; }
	virtual PairlistBuilderType get_type() const = 0;
	virtual const char* get_name() const = 0;
	virtual void resize(size_t new_max_particles, size_t new_max_pairs) {
		max_particles_ = new_max_particles;
		max_pairs_ceiling_ = new_max_pairs;
	}
	virtual Statistics get_statistics() const {
		return Statistics{num_particles_, num_pairs_, cutoff_,
						  num_particles_ ? static_cast<float>(num_pairs_) / num_particles_ : 0.0f,
						  0, 0.0};
	}

  protected:
	Resource resource_;
	size_t max_particles_;
	size_t max_pairs_ceiling_;
	size_t num_particles_ = 0;
	size_t num_pairs_ = 0;
	float cutoff_ = 0.0f;
	PeriodicBox box_;
	ExclusionView exclusions_;
};

// Owns one library context (create/destroy) and forwards its status codes.
class Context {
  public:
	Context(const Resource& r, size_t max_particles) : res_(r) {
		check(mb2_create(r.device, static_cast<uint32_t>(std::max<size_t>(max_particles, 1)), &ctx_),
			  nullptr, "mb2_create");
	}
	Context(const Context&) = delete;
	Context& operator=(const Context&) = delete;
	~Context() {
		if (ctx_) mb2_destroy(ctx_);
	}
	mb2_context* get() const { return ctx_; }
	void* stream() const { return reinterpret_cast<void*>(res_.stream); }
	const Resource& resource() const { return res_; }
	void set_box(const PeriodicBox& box) {
		const float o[3] = {box.get_origin().x, box.get_origin().y, box.get_origin().z};
		const float s[3] = {box.get_size().x, box.get_size().y, box.get_size().z};
		const int p[3] = {box.is_periodic(0), box.is_periodic(1), box.is_periodic(2)};
		check(mb2_set_box(ctx_, o, s, p), ctx_, "set_periodic_box");
	}
	void set_exclusions(const ExclusionView& e) {
		check(mb2_set_exclusions(ctx_, e.offsets, e.excluded, e.num_particles, e.rigid_body_id),
			  ctx_, "set_exclusions");
	}

  private:
	Resource res_;
	mb2_context* ctx_ = nullptr;
};

// Pairlist on the B200 path: Morton sort + exact pair set in a sliced-ELL
// half list held by the context. get_neighbor_pairs() materialises the
// reference's int2 list on demand (the force path never needs it).
class B200Pairlist : public Pairlist {
  public:
	B200Pairlist(const Resource& resource, size_t max_particles, size_t max_pairs_ceiling)
		: Pairlist(resource, max_particles, max_pairs_ceiling),
		  ctx_(std::make_shared<Context>(resource, max_particles)) {}
	// Share a context with a B200Patch (the patch's force stage reads this list).
	B200Pairlist(std::shared_ptr<Context> ctx, size_t max_particles, size_t max_pairs_ceiling)
		: Pairlist(ctx->resource(), max_particles, max_pairs_ceiling), ctx_(std::move(ctx)) {}

	void build_pairlist(const DeviceBuffer<Vector3>& positions, size_t num_particles,
						float cutoff) override {
		build_with_types(positions.data(), nullptr, num_particles, cutoff, interaction_cutoff_);
	}
	// The force cutoff this list serves (0, the default: none given). Builds
	// through build_pairlist then store the pairs likely to interact first in
	// each row (same pair set; see mb2_build_pairlist).
	void set_interaction_cutoff(float cutoff) { interaction_cutoff_ = cutoff; }
	// Build with type ids (the pair-force stage reads them beside the positions).
	void build_with_types(const Vector3* positions, const int* type_ids, size_t num_particles,
						  float cutoff, float interaction_cutoff) {
		if (num_particles > max_particles_)
			throw Exception(ExceptionType::CapacityError,
							"build_pairlist: more particles than the pairlist was created for");
		uint64_t pairs = 0;
		check(mb2_build_pairlist(ctx_->get(), reinterpret_cast<const float*>(positions), type_ids,
								 static_cast<uint32_t>(num_particles), cutoff, interaction_cutoff,
								 ctx_->stream(), &pairs),
			  ctx_->get(), "build_pairlist");
		if (pairs > max_pairs_ceiling_)
			throw Exception(ExceptionType::CapacityError,
							"build_pairlist: pair count exceeds the pair-buffer ceiling");
		num_particles_ = num_particles;
		num_pairs_ = pairs;
		cutoff_ = cutoff;
		exported_ = false;
	}
	// ZOrderPairlist semantics (ZOrderPairlist.cpp:184-190): the displacement
	// is measured against the snapshot taken at the last build, so
	// old_positions is not read; true when max |dx| > skin / 2.
	bool needs_update(const DeviceBuffer<Vector3>& positions, const DeviceBuffer<Vector3>&,
					  size_t num_particles, float skin_distance) const override {
		float max_disp = 0.0f;
		int needs = 1;
		check(mb2_needs_update(ctx_->get(), reinterpret_cast<const float*>(positions.data()),
							   static_cast<uint32_t>(num_particles), skin_distance, ctx_->stream(),
							   &max_disp, &needs),
			  ctx_->get(), "needs_update");
		last_max_displacement_ = max_disp;
		return needs != 0;
	}
	void set_periodic_box(const PeriodicBox& box) override {
		Pairlist::set_periodic_box(box);
		ctx_->set_box(box);
	}
	void set_exclusions(const ExclusionView& exclusions) override {
		Pairlist::set_exclusions(exclusions);
		ctx_->set_exclusions(exclusions);
	}
	const DeviceBuffer<int2>& get_neighbor_pairs() const override {
		if (!exported_) {
			if (pairs_.size() < num_pairs_) pairs_ = DeviceBuffer<int2>(num_pairs_, resource_);
			if (num_pairs_)
				check(mb2_export_pairs(ctx_->get(), reinterpret_cast<int*>(pairs_.data()),
									   pairs_.size(), ctx_->stream()),
					  ctx_->get(), "get_neighbor_pairs");
			exported_ = true;
		}
		return pairs_;
	}
	PairlistBuilderType get_type() const override { return PairlistBuilderType::B200; }
	const char* get_name() const override { return "B200 Z-order pairlist"; }
	float last_max_displacement() const { return last_max_displacement_; }
	const std::shared_ptr<Context>& context() const { return ctx_; }

  private:
	std::shared_ptr<Context> ctx_;
	mutable DeviceBuffer<int2> pairs_;
	mutable bool exported_ = false;
	mutable float last_max_displacement_ = 0.0f;
	float interaction_cutoff_ = 0.0f;
};

// Factory (src/PatchOperation/Pairlist.cpp:7-31) with the B200 strategy
// registered; the reference's other strategies live in the reference.
inline std::unique_ptr<Pairlist> create_pairlist(PairlistBuilderType type, const Resource& resource,
												 size_t max_particles, size_t max_pairs) {
	switch (type) {
		case PairlistBuilderType::B200:
			return std::make_unique<B200Pairlist>(resource, max_particles, max_pairs);
		default:
			throw Exception(ExceptionType::NotImplementedError,
							"create_pairlist: only PairlistBuilderType::B200 is provided here");
	}
}

// One tabulated table as loaded by the reference (src/Objects/Tables.h:27-120):
// values Y, start X[0] and the step inverse the reference derives from it.
struct Table {
	std::vector<float> values;
	float start = 0.0f;
	float step_inv = 0.0f;
};

// Kinds of tabulated potential (src/Objects/Tables.h:21).
enum class TabulatedType { NonBondedPair, Bond, Angle, Dihedral, Default };

// A table read from the reference's "x y" text files, restating
// Table::read_file, check_same_step_size and convert_angular_abscissa_to_radians
// (src/Objects/Tables.h:27-120): lines whose first character is '#' are
// comments; a line that does not start with two numbers is skipped with a
// warning; numbers are read into float by stream extraction; step = X[1] - X[0]
// and start = X[0] in float, uniform unless some |X[i] - X[i-1]| - step exceeds
// 1e-4 (a warning only, as in the reference); angle and dihedral abscissae are
// degrees, multiplied by float(pi / 180) after the check. The reference's
// warnings are kept in `warnings` instead of being logged.
struct TableFile {
	std::string name;
	TabulatedType type;
	float step_size = 0.0f;
	float start = 0.0f;
	std::vector<float> X, Y;
	std::vector<std::string> warnings;

	explicit TableFile(TabulatedType t) : type(t) {
		if (t == TabulatedType::Dihedral) start = static_cast<float>(-3.14159265358979323846);
	}

	bool check_same_step_size() {
		if (X.size() < 2) {
			warnings.push_back("Table " + name + ": Not enough values to check step size");
			return false;
		}
		step_size = X[1] - X[0];
		start = X[0];
		for (size_t i = 2; i < X.size(); ++i) {
			const float d = std::fabs(X[i] - X[i - 1]) - step_size;
			if (d > 1e-4) {
				warnings.push_back("Table " + name + ": Step size is not the same for all values at index " +
								   std::to_string(i));
				return false;
			}
		}
		return true;
	}

	void read_file(const std::string& file_name, const std::string& name_ = "") {
		if (name_.empty()) {
			const size_t slash = file_name.find_last_of('/');
			std::string stem = slash == std::string::npos ? file_name : file_name.substr(slash + 1);
			const size_t dot = stem.find_last_of('.');
			name = dot == std::string::npos || dot == 0 ? stem : stem.substr(0, dot);
		} else {
			name = name_;
		}
		std::ifstream in(file_name);
		if (!in) throw Exception(ExceptionType::FileIoError, "Table::read_file: cannot open " + file_name);
		std::string line;
		size_t number = 0;
		while (std::getline(in, line)) {
			++number;
			if (!line.empty() && line[0] == '#') continue;
			std::istringstream iss(line);
			float x = 0.0f, y = 0.0f;
			if (iss >> x >> y) {
				X.push_back(x);
				Y.push_back(y);
			} else {
				warnings.push_back("Tables: Failed to parse line " + std::to_string(number) + ": " + line);
			}
		}
		check_same_step_size();
		convert_angular_abscissa_to_radians();
	}

	void convert_angular_abscissa_to_radians() {
		if (type != TabulatedType::Angle && type != TabulatedType::Dihedral) return;
		constexpr float deg_to_rad = static_cast<float>(3.14159265358979323846 / 180.0);
		for (float& x : X) x *= deg_to_rad;
		start *= deg_to_rad;
		step_size *= deg_to_rad;
	}

	// The table as set_pair_tables / set_bonded_tables take it: the non-bonded
	// step inverse is 1.0f / step (DevicePairNonBondedInteraction.h:183), the
	// bonded one float(1.0 / double(step)) (DeviceBondedInteraction.h:213-214).
	Table to_table() const {
		Table t;
		t.values = Y;
		t.start = start;
		t.step_inv = type == TabulatedType::NonBondedPair
						 ? 1.0f / step_size
						 : static_cast<float>(1.0 / static_cast<double>(step_size));
		return t;
	}
};

// Integrators of Patch::integrate_motion on this path (Patch.cpp:238-352).
enum class IntegratorType { BD, Langevin };

// The three Patch stages of the BD path over one context. Set-up mirrors
// what the reference's Patch reads from its registries (tables, types,
// exclusions); the stage calls keep Patch's argument meanings.
class B200Patch {
  public:
	B200Patch(const Resource& resource, size_t max_particles)
		: ctx_(std::make_shared<Context>(resource, max_particles)),
		  pairlist_(ctx_, max_particles, SIZE_MAX) {}

	B200Pairlist& pairlist() { return pairlist_; }
	mb2_context* handle() const { return ctx_->get(); }

	void set_periodic_box(const PeriodicBox& box) { pairlist_.set_periodic_box(box); }
	void set_exclusions(const ExclusionView& e) { pairlist_.set_exclusions(e); }
	// Pair tables: term_matrix[a * num_types + b] = pair tag (bit 5 tabulated,
	// table index << 8; src/Interactions/Nonbonded/Pairwise.h:31-35).
	void set_pair_tables(int num_types, const std::vector<uint32_t>& term_matrix,
						 const std::vector<Table>& tables) {
		Flat f(tables);
		check(mb2_set_pair_tables(ctx_->get(), num_types, term_matrix.data(),
								  static_cast<int>(tables.size()), f.values.data(), f.sizes.data(),
								  f.starts.data(), f.step_invs.data()),
			  ctx_->get(), "set_pair_tables");
	}
	// Analytical pair terms (DevicePairNonBondedInteractions + SolventParams):
	// per-type charge, softcore radius and eps; params null = the reference's
	// solvent and Gaussian defaults.
	void set_pair_terms(const std::vector<float>& charge, const std::vector<float>& radius,
						const std::vector<float>& eps, const mb2_pair_params* params = nullptr) {
		check(mb2_set_pair_terms(ctx_->get(), static_cast<int>(charge.size()), charge.data(),
								 radius.data(), eps.data(), params),
			  ctx_->get(), "set_pair_terms");
	}
	// kind 0 = bonds, 1 = angles, 2 = dihedrals (angle and dihedral tables
	// periodic, abscissa in radians).
	void set_bonded_tables(int kind, const std::vector<Table>& tables) {
		Flat f(tables);
		check(mb2_set_bonded_tables(ctx_->get(), kind, static_cast<int>(tables.size()),
									f.values.data(), f.sizes.data(), f.starts.data(),
									f.step_invs.data()),
			  ctx_->get(), "set_bonded_tables");
	}
	// Per-type charge and diffusion (x, y, z), no grids.
	void set_particle_types(const std::vector<float>& charge, const std::vector<float>& diffusion3) {
		const int t = static_cast<int>(charge.size());
		check(mb2_set_particle_types(ctx_->get(), t, charge.data(), diffusion3.data(), nullptr,
									 nullptr, 0, nullptr, nullptr, nullptr),
			  ctx_->get(), "set_particle_types");
	}

	// DeviceParticle::clear_forces (DeviceParticleManager.h:94-96).
	void clear_forces(DeviceBuffer<Vector3>& force_energy) { force_energy.fill_zero(); }

	// Patch::calculate_nonbonded_forces (Patch.cpp:86-154): rebuild on the
	// first call and every rebuild_period steps when the skin check says so,
	// then add the tabulated pair forces into ForceEnergy. interaction_cutoff
	// <= 0 evaluates every listed pair.
	void calculate_nonbonded_forces(const DeviceBuffer<Vector3>& pos, const DeviceBuffer<int>& types,
									DeviceBuffer<Vector3>& force_energy, size_t num_particles,
									float pairlist_cutoff, float interaction_cutoff, size_t step,
									size_t rebuild_period, bool compute_energy = false) {
		const bool first = !built_ || built_n_ != num_particles;
		bool rebuild = first || rebuild_period == 0 || (step - 1) % rebuild_period == 0;
		const float skin = pairlist_cutoff - interaction_cutoff;
		if (rebuild && !first && rebuild_period != 0 && skin > 0.0f && interaction_cutoff > 0.0f)
			rebuild = pairlist_.needs_update(pos, pos, num_particles, skin);
		if (rebuild) {
			pairlist_.build_with_types(pos.data(), types.data(), num_particles, pairlist_cutoff,
									   interaction_cutoff);
			built_ = true;
			built_n_ = num_particles;
		}
		check(mb2_pair_forces(ctx_->get(), reinterpret_cast<const float*>(pos.data()), types.data(),
							  reinterpret_cast<float*>(force_energy.data()),
							  static_cast<uint32_t>(num_particles), interaction_cutoff,
							  compute_energy ? 1 : 0, ctx_->stream()),
			  ctx_->get(), "calculate_nonbonded_forces");
	}

	// Patch::calculate_bonded_forces (Patch.cpp:156-236): tabulated bonds
	// (int2 per bond) and angles (int4 per angle, fourth word unused).
	void calculate_bonded_forces(const DeviceBuffer<Vector3>& pos, DeviceBuffer<Vector3>& force_energy,
								 const int* bonds2, const int* bond_table_idx, size_t num_bonds,
								 const int* angles4, const int* angle_table_idx, size_t num_angles,
								 bool compute_energy = false) {
		if (num_bonds)
			check(mb2_bond_forces(ctx_->get(), bonds2, bond_table_idx,
								  static_cast<uint32_t>(num_bonds),
								  reinterpret_cast<const float*>(pos.data()),
								  reinterpret_cast<float*>(force_energy.data()),
								  compute_energy ? 1 : 0, ctx_->stream()),
				  ctx_->get(), "calculate_bonded_forces");
		if (num_angles)
			check(mb2_angle_forces(ctx_->get(), angles4, angle_table_idx,
								   static_cast<uint32_t>(num_angles),
								   reinterpret_cast<const float*>(pos.data()),
								   reinterpret_cast<float*>(force_energy.data()),
								   compute_energy ? 1 : 0, ctx_->stream()),
				  ctx_->get(), "calculate_bonded_forces");
	}

	// The rest of Patch::calculate_bonded_forces (Patch.cpp:208-232): tabulated
	// dihedrals (int4 per dihedral) and harmonic restraints (particle id,
	// anchor, spring constant per restraint). A negative table index skips a
	// row, as a non-tabulated form does in the reference.
	void calculate_dihedral_and_restraint_forces(const DeviceBuffer<Vector3>& pos,
												 DeviceBuffer<Vector3>& force_energy,
												 const int* dihedrals4, const int* dihedral_table_idx,
												 size_t num_dihedrals, const int* restraint_ids,
												 const Vector3* restraint_anchors,
												 const float* restraint_k, size_t num_restraints,
												 bool compute_energy = false) {
		if (num_dihedrals)
			check(mb2_dihedral_forces(ctx_->get(), dihedrals4, dihedral_table_idx,
									  static_cast<uint32_t>(num_dihedrals),
									  reinterpret_cast<const float*>(pos.data()),
									  reinterpret_cast<float*>(force_energy.data()),
									  compute_energy ? 1 : 0, ctx_->stream()),
				  ctx_->get(), "calculate_bonded_forces");
		if (num_restraints)
			check(mb2_restraint_forces(ctx_->get(), restraint_ids,
									   reinterpret_cast<const float*>(restraint_anchors),
									   restraint_k, static_cast<uint32_t>(num_restraints),
									   reinterpret_cast<const float*>(pos.data()),
									   reinterpret_cast<float*>(force_energy.data()),
									   compute_energy ? 1 : 0, ctx_->stream()),
				  ctx_->get(), "calculate_bonded_forces");
	}

	// Patch::integrate_motion with the BD integrator (Patch.cpp:238-352,
	// Integrator/BD.h): base seed mixed from (seed, patch_id, step) as the
	// reference mixes it; kT in kcal/mol.
	void integrate_motion(DeviceBuffer<Vector3>& pos, DeviceBuffer<Vector3>& force_energy,
						  const DeviceBuffer<int>& types, const uint32_t* flags,
						  size_t num_particles, float dt, float kT, size_t step, uint64_t seed,
						  uint64_t patch_id = 0, const Vector3& electric_field = Vector3{}) {
		const float e[3] = {electric_field.x, electric_field.y, electric_field.z};
		check(mb2_bd_integrate(ctx_->get(), reinterpret_cast<float*>(pos.data()),
							   reinterpret_cast<float*>(force_energy.data()), types.data(), flags,
							   static_cast<uint32_t>(num_particles), dt, kT, step,
							   mb2_bd_seed(seed, patch_id, step), 0u, e, ctx_->stream()),
			  ctx_->get(), "integrate_motion");
	}

	// Per-type mass and damping for the Langevin integrator.
	void set_langevin_types(const std::vector<float>& mass, const std::vector<float>& damping3) {
		check(mb2_set_langevin_types(ctx_->get(), static_cast<int>(mass.size()), mass.data(),
									 damping3.data()),
			  ctx_->get(), "set_langevin_types");
	}

	// Patch::integrate_motion with either integrator. Langevin keeps the
	// reference's deferred closing kick: it is paid at the start of the next
	// Langevin step, or by finish_deferred_kick (Patch.cpp:290-335, 354-373).
	void integrate_motion(IntegratorType type, DeviceBuffer<Vector3>& pos,
						  DeviceBuffer<Vector3>& mom, DeviceBuffer<Vector3>& force_energy,
						  const DeviceBuffer<int>& types, const uint32_t* flags, size_t num_particles,
						  float dt, float kT, size_t step, uint64_t seed, uint64_t patch_id = 0,
						  const Vector3& electric_field = Vector3{}) {
		if (type == IntegratorType::BD) {
			integrate_motion(pos, force_energy, types, flags, num_particles, dt, kT, step, seed,
							 patch_id, electric_field);
			return;
		}
		const float e[3] = {electric_field.x, electric_field.y, electric_field.z};
		check(mb2_baoab_integrate(ctx_->get(), reinterpret_cast<float*>(pos.data()),
								  reinterpret_cast<float*>(mom.data()),
								  reinterpret_cast<float*>(force_energy.data()), types.data(), flags,
								  static_cast<uint32_t>(num_particles), dt, kT, step,
								  mb2_bd_seed(seed, patch_id, step), 0u, e,
								  deferred_kick_pending_ ? 1 : 0, ctx_->stream()),
			  ctx_->get(), "integrate_motion");
		deferred_kick_pending_ = true;
	}
	void finish_deferred_kick(DeviceBuffer<Vector3>& mom, const DeviceBuffer<Vector3>& force_energy,
							  const uint32_t* flags, size_t num_particles, float dt) {
		if (!deferred_kick_pending_) return;
		deferred_kick_pending_ = false;
		check(mb2_baoab_last_update(ctx_->get(), reinterpret_cast<float*>(mom.data()),
									reinterpret_cast<const float*>(force_energy.data()), flags,
									static_cast<uint32_t>(num_particles), dt, ctx_->stream()),
			  ctx_->get(), "finish_deferred_kick");
	}
	bool has_deferred_kick() const { return deferred_kick_pending_; }

	// Patch::reorder_particles (src/PatchOperation/Patch.cpp:455-480): Morton
	// order over the periodic box, every particle array gathered, every stored
	// index remapped, the exclusion CSR rebuilt and handed to the pairlist, and
	// the next calculate_nonbonded_forces forced to rebuild. A degenerate box
	// or no particles skips the reorder (returns false), as the reference does.
	bool reorder_particles(const PeriodicBox& box, const ParticleArrays& p, size_t num_particles,
						   const BondedIndices& b = BondedIndices{},
						   ExclusionCSR* exclusions = nullptr) {
		if (num_particles == 0 || !p.pos) return false;
		const Vector3& o = box.get_origin();
		const Vector3& sz = box.get_size();
		if (!(o.x + sz.x > o.x && o.y + sz.y > o.y && o.z + sz.z > o.z)) return false;
		mb2_context* c = ctx_->get();
		void* st = ctx_->stream();
		const uint32_t n = static_cast<uint32_t>(num_particles);
		check(mb2_reorder_begin(c, reinterpret_cast<const float*>(p.pos), n, st), c,
			  "reorder_particles");
		auto apply = [&](void* a, uint32_t bytes) {
			if (a) check(mb2_reorder_apply(c, a, bytes, n, st), c, "reorder_particles");
		};
		apply(p.pos, 16);
		apply(p.mom, 16);
		apply(p.orient, 16);
		apply(p.id, 4);
		apply(p.type_id, 4);
		apply(p.flags, 4);
		apply(p.attached_rigid_body_id, 4);
		auto remap = [&](int* a, size_t count) {
			if (a && count) check(mb2_reorder_remap(c, a, count, st), c, "reorder_particles");
		};
		remap(b.bonds2, 2 * b.num_bonds);
		remap(b.angles4, 4 * b.num_angles);
		remap(b.dihedrals4, 4 * b.num_dihedrals);
		remap(b.restraint_ids, b.num_restraints);
		if (exclusions && !exclusions->pairs().empty()) {
			DeviceBuffer<uint32_t> inv(num_particles, ctx_->resource());
			check(mb2_reorder_inverse(c, inv.data(), n, st), c, "reorder_particles");
			std::vector<uint32_t> h;
			inv.copy_to_host(h);
			exclusions->remap(h);
			pairlist_.set_exclusions(exclusions->view(p.attached_rigid_body_id));
		}
		built_ = false;  // force_rebuild_
		return true;
	}

  private:
	struct Flat {
		std::vector<float> values, starts, step_invs;
		std::vector<uint32_t> sizes;
		explicit Flat(const std::vector<Table>& tables) {
			for (const Table& t : tables) {
				values.insert(values.end(), t.values.begin(), t.values.end());
				sizes.push_back(static_cast<uint32_t>(t.values.size()));
				starts.push_back(t.start);
				step_invs.push_back(t.step_inv);
			}
		}
	};
	std::shared_ptr<Context> ctx_;
	B200Pairlist pairlist_;
	bool built_ = false;
	size_t built_n_ = 0;
	bool deferred_kick_pending_ = false;
};

// SimManager's output side for one system (src/SimManager.cpp:318-330,
// 541-575, 596-633, 833-861, 999-1135) over mb2_output: DCD frames (and the
// Langevin momentum DCD), <name>.energy.dat, restart files; rows in global-id
// order through `ids` (may be null). Frames and restarts are written by the
// library's writer thread; flush() waits for them.
class SimOutput {
  public:
	SimOutput(const std::string& output_name, size_t num_particles, int output_period,
			  int energy_output_period, float timestep, const PeriodicBox& box,
			  bool with_momentum = false, const Resource& r = Resource{})
		: res_(r), n_(num_particles), output_period_(output_period),
		  energy_output_period_(energy_output_period) {
		mb2_output_config cfg{};
		cfg.output_name = output_name.c_str();
		cfg.num_particles = static_cast<uint32_t>(num_particles);
		cfg.output_period = output_period;
		cfg.timestep = timestep;
		cfg.box[0] = box.get_size().x;
		cfg.box[1] = box.get_size().y;
		cfg.box[2] = box.get_size().z;
		for (int a = 0; a < 3; ++a) cfg.periodic[a] = box.is_periodic(a) ? 1 : 0;
		cfg.with_momentum = with_momentum ? 1 : 0;
		cfg.device = r.device;
		const int rc = mb2_output_create(&cfg, &out_);
		if (rc != MB2_OK) throw Exception(ExceptionType::ValueError, "SimOutput: mb2_output_create failed");
	}
	SimOutput(const SimOutput&) = delete;
	SimOutput& operator=(const SimOutput&) = delete;
	~SimOutput() {
		if (out_) mb2_output_destroy(out_);
	}
	void write_dcd_frame(const DeviceBuffer<Vector3>& pos, const DeviceBuffer<Vector3>* mom = nullptr,
						 const int* ids = nullptr) {
		ok(mb2_output_frame(out_, reinterpret_cast<const float*>(pos.data()),
							mom ? reinterpret_cast<const float*>(mom->data()) : nullptr, ids,
							static_cast<uint32_t>(n_), stream()),
		   "write_dcd_frame");
	}
	void write_restart_files(const DeviceBuffer<Vector3>& pos, const DeviceBuffer<int>& types,
							 const DeviceBuffer<Vector3>* mom = nullptr, const int* ids = nullptr) {
		ok(mb2_output_restart(out_, reinterpret_cast<const float*>(pos.data()),
							  mom ? reinterpret_cast<const float*>(mom->data()) : nullptr,
							  types.data(), ids, static_cast<uint32_t>(n_), stream()),
		   "write_restart_files");
	}
	// Returns {kinetic (kT), potential (kcal/mol)} and appends them to the file.
	std::pair<double, double> write_energy_output(const DeviceBuffer<Vector3>& force_energy,
												  float kT, const DeviceBuffer<Vector3>* mom = nullptr,
												  const DeviceBuffer<int>* types = nullptr,
												  const std::vector<float>& mass = {}) {
		double e[2] = {0.0, 0.0};
		ok(mb2_output_energy(out_, reinterpret_cast<const float*>(force_energy.data()),
							 mom ? reinterpret_cast<const float*>(mom->data()) : nullptr,
							 types ? types->data() : nullptr, mass.empty() ? nullptr : mass.data(),
							 static_cast<int>(mass.size()), static_cast<uint32_t>(n_), kT, stream(), e),
		   "write_energy_output");
		return {e[0], e[1]};
	}
	// SimManager::handle_output's schedule: a frame every output_period steps;
	// energies, then restart files, every energy_output_period steps.
	void handle_output(size_t step, const DeviceBuffer<Vector3>& pos,
					   const DeviceBuffer<Vector3>& force_energy, const DeviceBuffer<int>& types,
					   float kT, const DeviceBuffer<Vector3>* mom = nullptr,
					   const std::vector<float>& mass = {}, const int* ids = nullptr) {
		if (output_period_ > 0 && step % static_cast<size_t>(output_period_) == 0)
			write_dcd_frame(pos, mom, ids);
		if (energy_output_period_ > 0 && step % static_cast<size_t>(energy_output_period_) == 0) {
			write_energy_output(force_energy, kT, mom, mom ? &types : nullptr, mass);
			write_restart_files(pos, types, mom, ids);
		}
	}
	void flush() { ok(mb2_output_flush(out_), "flush"); }

  private:
	void* stream() const { return reinterpret_cast<void*>(res_.stream); }
	void ok(int rc, const char* what) {
		if (rc == MB2_OK) return;
		const std::string msg = std::string(what) + ": " + mb2_output_last_error(out_);
		switch (rc) {
			case MB2_ERR_ARG: throw Exception(ExceptionType::ValueError, msg);
			case MB2_ERR_IO: throw Exception(ExceptionType::FileIoError, msg);
			case MB2_ERR_CUDA: throw Exception(ExceptionType::CUDAError, msg);
			default: throw Exception(ExceptionType::StateError, msg);
		}
	}
	Resource res_;
	size_t n_;
	int output_period_, energy_output_period_;
	mb2_output* out_ = nullptr;
};

}  // namespace marsb200
