// Drives MARS::B200PairlistAdapter (mars_md_b200/host/b200_ref_adapter.hpp),
// compiled against the reference's own Pairlist.h, the way the reference's
// Patch drives its pairlist (set_periodic_box, set_exclusions, build_pairlist,
// get_num_pairs, get_neighbor_pairs, needs_update).
//
//   ref_adapter_test <case.bin> <pairs.bin>
//
// case.bin: uint32 n; float origin[3], size[3]; int32 periodic[3]; float
// list_radius; uint32 num_offsets (0, or n + 1); float4 pos[n]; then, when
// num_offsets > 0, int32 offsets[n + 1], uint32 num_excluded, int32
// excluded[num_excluded]. pairs.bin: uint64 num_pairs, int32 (i, j)[num_pairs]
// as get_neighbor_pairs() holds them. Prints PASS/FAIL lines; exit 0 when all
// pass.
#include "b200_ref_adapter.hpp"

#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

using namespace MARS;

namespace {

int failures = 0;

void expect(bool ok, const char* what) {
	std::printf("%s %s\n", ok ? "PASS" : "FAIL", what);
	if (!ok) ++failures;
}

template <typename T>
bool read_n(std::FILE* f, T* dst, size_t n) {
	return std::fread(dst, sizeof(T), n, f) == n;
}

}  // namespace

int main(int argc, char** argv) {
	if (argc != 3) {
		std::fprintf(stderr, "usage: %s case.bin pairs.bin\n", argv[0]);
		return 2;
	}
	std::FILE* f = std::fopen(argv[1], "rb");
	if (!f) return 2;
	uint32_t n = 0, num_off = 0;
	float origin[3], size[3], rc = 0.0f;
	int32_t periodic[3];
	bool ok = read_n(f, &n, 1) && read_n(f, origin, 3) && read_n(f, size, 3) &&
			  read_n(f, periodic, 3) && read_n(f, &rc, 1) && read_n(f, &num_off, 1);
	std::vector<Vector3> pos(n);
	ok = ok && read_n(f, reinterpret_cast<float*>(pos.data()), 4 * static_cast<size_t>(n));
	std::vector<int32_t> offsets(num_off), excluded;
	uint32_t num_excl = 0;
	if (ok && num_off) {
		ok = read_n(f, offsets.data(), num_off) && read_n(f, &num_excl, 1);
		excluded.resize(num_excl);
		ok = ok && read_n(f, excluded.data(), num_excl);
	}
	std::fclose(f);
	if (!ok) {
		std::fprintf(stderr, "bad case file\n");
		return 2;
	}

	const Resource res(0);
	DeviceBuffer<Vector3> d_pos(n, res), d_old(n, res);
	d_pos.copy_from_host(pos.data(), n);
	DeviceBuffer<int> d_off(num_off ? num_off : 1, res), d_excl(num_excl ? num_excl : 1, res);
	PeriodicBox box(Vector3(size[0], size[1], size[2]), periodic[0] != 0, periodic[1] != 0,
					periodic[2] != 0);
	box.set_origin(Vector3(origin[0], origin[1], origin[2]));

	std::unique_ptr<Pairlist> pl =
		std::make_unique<B200PairlistAdapter>(res, n, pairlist_max_pairs(res));
	expect(pl->get_type() == PairlistBuilderType::ZOrder, "get_type is the Z-order strategy");
	expect(std::strlen(pl->get_name()) > 0, "get_name");
	pl->set_periodic_box(box);
	if (num_off) {
		d_off.copy_from_host(offsets.data(), num_off);
		d_excl.copy_from_host(excluded.data(), num_excl);
		ExclusionView view;
		view.offsets = d_off.data();
		view.excluded = d_excl.data();
		view.num_particles = static_cast<idx_t>(num_off - 1);
		pl->set_exclusions(view);
	}
	pl->build_pairlist(d_pos, n, rc);
	const size_t np = pl->get_num_pairs();
	std::vector<MARS::int2> pairs(np);
	if (np) pl->get_neighbor_pairs().copy_to_host(pairs.data(), np);
	expect(pl->get_cutoff() == rc, "get_cutoff after build");
	bool ordered = true;
	for (const MARS::int2& p : pairs) ordered = ordered && p.x < p.y && p.x >= 0 && p.y < static_cast<int>(n);
	expect(ordered, "pairs as (smaller, larger) original index");

	// needs_update: unmoved -> false; one particle moved by more than skin / 2 -> true.
	expect(!pl->needs_update(d_pos, d_old, n, 5.0f), "needs_update false before any move");
	if (n > 0) {
		std::vector<Vector3> moved(pos);
		moved[0].x += 2.6f;
		DeviceBuffer<Vector3> d_moved(n, res);
		d_moved.copy_from_host(moved.data(), n);
		expect(pl->needs_update(d_moved, d_old, n, 5.0f), "needs_update true past half the skin");
	}
	// More particles than the capacity: the reference's ValueError.
	bool threw = false;
	try {
		DeviceBuffer<Vector3> big(n + 1, res);
		pl->build_pairlist(big, n + 1, rc);
	} catch (const Exception&) {
		threw = true;
	}
	expect(threw, "build beyond capacity throws MARS::Exception");

	std::FILE* o = std::fopen(argv[2], "wb");
	if (!o) return 2;
	const uint64_t np64 = np;
	std::fwrite(&np64, sizeof(np64), 1, o);
	if (np) std::fwrite(pairs.data(), sizeof(MARS::int2), np, o);
	std::fclose(o);
	std::printf("%s (%zu pairs)\n", failures ? "SOME FAILED" : "ALL PASS", np);
	return failures ? 1 : 0;
}
