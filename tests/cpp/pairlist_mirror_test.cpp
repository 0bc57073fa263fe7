// The C++ host mirror (mars_md_b200/host/b200_pairlist.hpp) used the way the
// reference's own pairlist and patch tests use theirs: a 4x4x4 lattice in an
// open box (Unit_test/Compute/zorder_pairlist_tests.cpp), the skin check,
// exclusions and rigid bodies dropped at build time, a periodic random system
// against an O(N^2) pair set, the error behaviour, and the Patch stages
// against the fused step. One line per check; exit status 0 only if all pass.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <set>
#include <utility>
#include <vector>

#include "b200_pairlist.hpp"

using namespace marsb200;

static int failures = 0;

#define EXPECT(cond, name)                                              \
	do {                                                                \
		if (cond) {                                                     \
			std::printf("PASS %s\n", name);                             \
		} else {                                                        \
			std::printf("FAIL %s (%s:%d)\n", name, __FILE__, __LINE__); \
			++failures;                                                 \
		}                                                               \
	} while (0)

// Minimum image as the reference's PeriodicBox::wrap_diff_scalar rounds it.
static float wrap_diff_scalar(float x, float l) {
	const float image = std::floor(x * (1.0f / l));
	x = x - image * l;
	return x >= 0.5f * l ? x - l : x;
}

static std::set<std::pair<int, int>> host_pairs(const std::vector<Vector3>& p, float l, float rc) {
	std::set<std::pair<int, int>> out;
	const float rc2 = rc * rc;
	for (size_t i = 0; i < p.size(); ++i)
		for (size_t j = i + 1; j < p.size(); ++j) {
			const float dx = wrap_diff_scalar(p[j].x - p[i].x, l);
			const float dy = wrap_diff_scalar(p[j].y - p[i].y, l);
			const float dz = wrap_diff_scalar(p[j].z - p[i].z, l);
			const float xx = dx * dx, yy = dy * dy, zz = dz * dz;
			if ((xx + yy) + zz <= rc2) out.insert({static_cast<int>(i), static_cast<int>(j)});
		}
	return out;
}

static std::set<std::pair<int, int>> device_pairs(const Pairlist& pl) {
	std::vector<int2> h(pl.get_num_pairs());
	if (!h.empty()) pl.get_neighbor_pairs().copy_to_host(h.data(), h.size(), true);
	std::set<std::pair<int, int>> out;
	for (const int2& q : h) out.insert({q.x, q.y});
	return out;
}

static std::vector<Vector3> lattice() {
	std::vector<Vector3> p;
	for (int x = 0; x < 4; ++x)
		for (int y = 0; y < 4; ++y)
			for (int z = 0; z < 4; ++z) p.emplace_back(1.5f * x, 1.5f * y, 1.5f * z);
	return p;
}

static void lattice_tests(const Resource& res) {
	auto pl = create_pairlist(PairlistBuilderType::B200, res, 64, 64 * 64);
	EXPECT(pl->get_type() == PairlistBuilderType::B200, "factory returns the B200 strategy");
	pl->set_periodic_box(PeriodicBox(Vector3(0, 0, 0), Vector3(100, 100, 100), false, false, false));
	const std::vector<Vector3> h = lattice();
	DeviceBuffer<Vector3> pos(h.size(), res);
	pos.copy_from_host(h);
	pl->build_pairlist(pos, h.size(), 2.0f);
	EXPECT(pl->get_num_pairs() == 144, "lattice: 144 nearest-neighbour pairs");
	bool all_bonds = true, ordered = true;
	for (const auto& q : device_pairs(*pl)) {
		const float dx = h[q.second].x - h[q.first].x, dy = h[q.second].y - h[q.first].y,
					dz = h[q.second].z - h[q.first].z;
		all_bonds &= std::fabs(std::sqrt(dx * dx + dy * dy + dz * dz) - 1.5f) < 1e-5f;
		ordered &= q.first < q.second;
	}
	EXPECT(all_bonds, "lattice: every pair is 1.5 A apart");
	EXPECT(ordered, "lattice: pairs stored as (min, max) original indices");
	EXPECT(pl->get_cutoff() == 2.0f, "lattice: cutoff recorded");

	// Skin check against the snapshot taken at the build.
	EXPECT(!pl->needs_update(pos, pos, h.size(), 1.0f), "needs_update: no motion -> no rebuild");
	std::vector<Vector3> moved = h;
	moved[5].x += 0.6f;
	DeviceBuffer<Vector3> pos2(h.size(), res);
	pos2.copy_from_host(moved);
	EXPECT(pl->needs_update(pos2, pos, h.size(), 1.0f), "needs_update: 0.6 A > skin / 2");
	EXPECT(!pl->needs_update(pos2, pos, h.size(), 2.0f), "needs_update: 0.6 A < skin / 2");

	// Exclusions (0,1) and (0,4) are never emitted.
	std::vector<int> offsets(65, 0), excl;
	std::vector<std::vector<int>> rows(64);
	rows[0] = {1, 4};
	rows[1] = {0};
	rows[4] = {0};
	for (int i = 0; i < 64; ++i) {
		offsets[i + 1] = offsets[i] + static_cast<int>(rows[i].size());
		excl.insert(excl.end(), rows[i].begin(), rows[i].end());
	}
	DeviceBuffer<int> d_off(offsets.size(), res), d_ex(excl.size(), res);
	d_off.copy_from_host(offsets);
	d_ex.copy_from_host(excl);
	pl->set_exclusions(ExclusionView{d_off.data(), d_ex.data(), 64, nullptr});
	pl->build_pairlist(pos, h.size(), 2.0f);
	const auto ex_pairs = device_pairs(*pl);
	EXPECT(pl->get_num_pairs() == 142 && !ex_pairs.count({0, 1}) && !ex_pairs.count({0, 4}),
		   "exclusions dropped at build time");
	// A rigid body: particles 16..19 (a lattice row) never pair with each other.
	std::vector<int> body(64, -1);
	for (int i = 16; i < 20; ++i) body[i] = 3;
	DeviceBuffer<int> d_body(64, res);
	d_body.copy_from_host(body);
	pl->set_exclusions(ExclusionView{nullptr, nullptr, 0, d_body.data()});
	pl->build_pairlist(pos, h.size(), 2.0f);
	const auto rb = device_pairs(*pl);
	EXPECT(pl->get_num_pairs() == 141 && !rb.count({16, 17}) && !rb.count({18, 19}),
		   "same-rigid-body pairs dropped");
}

static void periodic_random_test(const Resource& res) {
	const int n = 2000;
	const float l = 60.0f, rc = 8.0f;
	std::mt19937 rng(20261203);
	std::uniform_real_distribution<float> u(0.0f, l);
	std::vector<Vector3> h(n);
	for (auto& p : h) p = Vector3(u(rng), u(rng), u(rng));
	B200Pairlist pl(res, n, static_cast<size_t>(n) * n);
	pl.set_periodic_box(PeriodicBox(Vector3(0, 0, 0), Vector3(l, l, l)));
	DeviceBuffer<Vector3> pos(n, res);
	pos.copy_from_host(h);
	pl.build_pairlist(pos, n, rc);
	const auto want = host_pairs(h, l, rc);
	EXPECT(pl.get_num_pairs() == want.size(), "periodic random: pair count equals O(N^2) count");
	EXPECT(device_pairs(pl) == want, "periodic random: identical pair set");
	const auto st = pl.get_statistics();
	EXPECT(st.num_particles == static_cast<size_t>(n) && st.num_pairs == want.size(),
		   "statistics reflect the build");
}

static void error_tests(const Resource& res) {
	bool threw = false;
	try {
		B200Pairlist pl(res, 16, 256);
		DeviceBuffer<Vector3> pos(16, res);
		pos.fill_zero();
		pl.build_pairlist(pos, 16, 2.0f);  // no box set
	} catch (const Exception& e) {
		threw = e.type() == ExceptionType::StateError;
	}
	EXPECT(threw, "build without a box throws StateError");
	threw = false;
	try {
		create_pairlist(PairlistBuilderType::CellList, res, 16, 256);
	} catch (const Exception& e) {
		threw = e.type() == ExceptionType::NotImplementedError;
	}
	EXPECT(threw, "unknown strategy throws NotImplementedError");
	threw = false;
	try {
		B200Pairlist pl(res, 16, 256);
		pl.set_periodic_box(PeriodicBox(Vector3(0, 0, 0), Vector3(10, 10, 10)));
		DeviceBuffer<Vector3> pos(32, res);
		pos.fill_zero();
		pl.build_pairlist(pos, 32, 2.0f);
	} catch (const Exception& e) {
		threw = e.type() == ExceptionType::CapacityError;
	}
	EXPECT(threw, "more particles than capacity throws CapacityError");
	threw = false;
	try {
		B200Pairlist pl(res, 16, 256);
		pl.set_periodic_box(PeriodicBox(Vector3(0, 0, 0), Vector3(-1, 10, 10)));
	} catch (const Exception& e) {
		threw = e.type() == ExceptionType::ValueError;
	}
	EXPECT(threw, "non-positive box edge throws ValueError");
}

// WCA-like table on 0..19.9 A (sigma 4, eps 0.5, capped at 20).
static Table wca() {
	Table t;
	t.start = 0.0f;
	t.step_inv = 1.0f / 0.1f;
	for (int k = 0; k < 200; ++k) {
		const double r = 0.1 * k, rc = std::pow(2.0, 1.0 / 6.0) * 4.0;
		double v = 0.0;
		if (r < rc) {
			const double s6 = r > 0 ? std::pow(4.0 / r, 6) : 1e30;
			v = std::min(20.0, 4.0 * 0.5 * (s6 * s6 - s6) + 0.5);
		}
		t.values.push_back(static_cast<float>(v));
	}
	return t;
}

static void patch_stage_test(const Resource& res) {
	const int n = 4096;
	const float l = 200.0f;
	std::mt19937 rng(7);
	std::uniform_real_distribution<float> u(0.0f, l);
	std::vector<Vector3> h(n);
	for (auto& p : h) p = Vector3(u(rng), u(rng), u(rng));
	std::vector<int> types(n, 0);
	const float kT = 295.0f * 0.001987191f, dt = 1e-4f;
	auto setup = [&](B200Patch& patch) {
		patch.set_periodic_box(PeriodicBox(Vector3(0, 0, 0), Vector3(l, l, l)));
		patch.set_pair_tables(1, {(1u << 5) | (0u << 8)}, {wca()});
		patch.set_particle_types({0.0f}, {150.0f, 150.0f, 150.0f});
	};
	// Staged: clear, nonbonded, integrate -- three Patch calls per step.
	B200Patch staged(res, n);
	setup(staged);
	DeviceBuffer<Vector3> pos_a(n, res), fe_a(n, res);
	DeviceBuffer<int> d_types(n, res);
	pos_a.copy_from_host(h);
	d_types.copy_from_host(types);
	for (size_t step = 1; step <= 5; ++step) {
		staged.clear_forces(fe_a);
		staged.calculate_nonbonded_forces(pos_a, d_types, fe_a, n, 25.0f, 20.0f, step, 20);
		staged.integrate_motion(pos_a, fe_a, d_types, nullptr, n, dt, kT, step, 99);
	}
	// Fused: one mb2_step per step with the same schedule and seed.
	B200Patch fused(res, n);
	setup(fused);
	DeviceBuffer<Vector3> pos_b(n, res), fe_b(n, res);
	pos_b.copy_from_host(h);
	mb2_step_params prm{};
	prm.pairlist_cutoff = 25.0f;
	prm.cutoff = 20.0f;
	prm.rebuild_period = 20;
	prm.dt = dt;
	prm.kT = kT;
	prm.seed = 99;
	for (uint64_t step = 1; step <= 5; ++step)
		check(mb2_step(fused.handle(), reinterpret_cast<float*>(pos_b.data()),
					   reinterpret_cast<float*>(fe_b.data()), d_types.data(), nullptr, n, step, &prm,
					   nullptr),
			  fused.handle(), "mb2_step");
	std::vector<Vector3> a, b;
	pos_a.copy_to_host(a);
	pos_b.copy_to_host(b);
	float worst = 0.0f, moved = 0.0f;
	for (int i = 0; i < n; ++i) {
		worst = std::max({worst, std::fabs(a[i].x - b[i].x), std::fabs(a[i].y - b[i].y),
						  std::fabs(a[i].z - b[i].z)});
		moved = std::max(moved, std::fabs(a[i].x - h[i].x));
	}
	EXPECT(worst <= 1e-4f && moved > 0.1f, "Patch stages equal the fused step over 5 steps");

	// Many steps in one call (graph-replayed between rebuild checks) against
	// one mb2_step per step, across two rebuild checks.
	B200Patch looped(res, n), ran(res, n);
	setup(looped);
	setup(ran);
	DeviceBuffer<Vector3> pos_c(n, res), fe_c(n, res), pos_d(n, res), fe_d(n, res);
	pos_c.copy_from_host(h);
	pos_d.copy_from_host(h);
	for (uint64_t step = 1; step <= 30; ++step)
		check(mb2_step(looped.handle(), reinterpret_cast<float*>(pos_c.data()),
					   reinterpret_cast<float*>(fe_c.data()), d_types.data(), nullptr, n, step, &prm,
					   nullptr),
			  looped.handle(), "mb2_step");
	check(mb2_run(ran.handle(), reinterpret_cast<float*>(pos_d.data()),
				  reinterpret_cast<float*>(fe_d.data()), d_types.data(), nullptr, n, 1, 30, &prm,
				  nullptr),
		  ran.handle(), "mb2_run");
	std::vector<Vector3> c, d;
	pos_c.copy_to_host(c);
	pos_d.copy_to_host(d);
	float worst_run = 0.0f;
	for (int i = 0; i < n; ++i)
		worst_run = std::max({worst_run, std::fabs(c[i].x - d[i].x), std::fabs(c[i].y - d[i].y),
							  std::fabs(c[i].z - d[i].z)});
	EXPECT(worst_run <= 1e-3f, "mb2_run equals one mb2_step per step over 30 steps");
}

// Langevin through the Patch mirror: the deferred closing kick is owed after a
// step and paid by finish_deferred_kick (momenta change), not twice.
static void langevin_stage_test(const Resource& res) {
	const int n = 1024;
	B200Patch patch(res, n);
	patch.set_periodic_box(PeriodicBox(Vector3(0, 0, 0), Vector3(100, 100, 100)));
	patch.set_particle_types({0.0f}, {150.0f, 150.0f, 150.0f});
	patch.set_langevin_types({12.0f}, {50.0f, 50.0f, 50.0f});
	std::vector<Vector3> h(n), f(n, Vector3(1.0f, -2.0f, 0.5f));
	for (int i = 0; i < n; ++i) h[i] = Vector3(0.09f * i, 50.0f, 50.0f);
	DeviceBuffer<Vector3> pos(n, res), mom(n, res), fe(n, res);
	DeviceBuffer<int> types(n, res);
	pos.copy_from_host(h);
	mom.fill_zero();
	fe.copy_from_host(f);
	types.copy_from_host(std::vector<int>(n, 0));
	const float kT = 295.0f * 0.001987191f;
	patch.integrate_motion(IntegratorType::Langevin, pos, mom, fe, types, nullptr, n, 1e-4f, kT, 1, 5);
	EXPECT(patch.has_deferred_kick(), "Langevin step leaves the closing kick pending");
	std::vector<Vector3> m1, m2;
	mom.copy_to_host(m1);
	patch.finish_deferred_kick(mom, fe, nullptr, n, 1e-4f);
	mom.copy_to_host(m2);
	const float kick = 0.5f * 1e-4f * 1.0f * 4.18679994e4f;
	EXPECT(!patch.has_deferred_kick() && std::fabs((m2[0].x - m1[0].x) - kick) < 1e-3f * kick,
		   "finish_deferred_kick applies one half-kick");
	patch.finish_deferred_kick(mom, fe, nullptr, n, 1e-4f);
	std::vector<Vector3> m3;
	mom.copy_to_host(m3);
	EXPECT(m3[0].x == m2[0].x, "no second closing kick");
}

// Patch::reorder_particles through the mirror: arrays gathered, bonds and the
// exclusion CSR remapped, and the rebuilt pair set equal to the old one
// through the new -> old id map.
static void reorder_stage_test(const Resource& res) {
	const int n = 2000;
	const float l = 60.0f, rc = 8.0f;
	std::mt19937 rng(20261204);
	std::uniform_real_distribution<float> u(0.0f, l);
	std::vector<Vector3> h(n);
	for (auto& p : h) p = Vector3(u(rng), u(rng), u(rng));
	std::vector<std::pair<int, int>> excl;
	std::vector<int> bonds;
	for (int i = 0; i + 1 < n; i += 2) {
		excl.push_back({i + 1, i});
		bonds.push_back(i);
		bonds.push_back(i + 1);
	}
	const PeriodicBox box(Vector3(0, 0, 0), Vector3(l, l, l));
	B200Patch patch(res, n);
	patch.set_periodic_box(box);
	ExclusionCSR ex;
	ex.build(excl, res);
	patch.set_exclusions(ex.view());
	DeviceBuffer<Vector3> pos(n, res);
	DeviceBuffer<int> ids(n, res), bond_dev(bonds.size(), res);
	pos.copy_from_host(h);
	std::vector<int> id0(n);
	for (int i = 0; i < n; ++i) id0[i] = i;
	ids.copy_from_host(id0);
	bond_dev.copy_from_host(bonds);
	patch.pairlist().build_pairlist(pos, n, rc);
	std::set<std::pair<int, int>> before;
	for (const auto& q : device_pairs(patch.pairlist()))
		before.insert({std::min(q.first, q.second), std::max(q.first, q.second)});

	ParticleReorderManager every20(0, 20), every5(5, 20);
	EXPECT(!every20.should_reorder(0) && every20.should_reorder(1) && !every20.should_reorder(2) &&
			   every20.should_reorder(21) && every5.should_reorder(6) &&
			   !every5.should_reorder(6, false),
		   "reorder cadence: steps 1, 1 + period, ...; period falls back to the rebuild period");

	ParticleArrays arrays;
	arrays.pos = pos.data();
	arrays.id = ids.data();
	BondedIndices bi;
	bi.bonds2 = bond_dev.data();
	bi.num_bonds = bonds.size() / 2;
	EXPECT(patch.reorder_particles(box, arrays, n, bi, &ex), "reorder runs on a valid box");
	std::vector<Vector3> h1;
	std::vector<int> id1, b1;
	pos.copy_to_host(h1);
	ids.copy_to_host(id1);
	bond_dev.copy_to_host(b1);
	std::vector<int> inv(n, -1);
	bool perm = true, gathered = true;
	for (int s = 0; s < n; ++s) {
		const int o = id1[s];
		if (o < 0 || o >= n || inv[o] != -1) {
			perm = false;
			break;
		}
		inv[o] = s;
		gathered = gathered && h1[s].x == h[o].x && h1[s].y == h[o].y && h1[s].z == h[o].z;
	}
	EXPECT(perm && gathered, "reorder: ids a permutation, positions gathered by it");
	bool remapped = perm;
	for (size_t k = 0; remapped && k < bonds.size(); ++k) remapped = b1[k] == inv[bonds[k]];
	EXPECT(remapped, "reorder: bond indices through the inverse map");
	patch.pairlist().build_pairlist(pos, n, rc);
	std::set<std::pair<int, int>> after;
	for (const auto& q : device_pairs(patch.pairlist())) {
		const int a = id1[q.first], b = id1[q.second];
		after.insert({std::min(a, b), std::max(a, b)});
	}
	EXPECT(!before.empty() && after == before,
		   "reorder: rebuilt pair set (with remapped exclusions) equals the old one");
	const PeriodicBox flat(Vector3(0, 0, 0), Vector3(l, 0.0f, l));
	EXPECT(!patch.reorder_particles(flat, arrays, n, bi, &ex), "degenerate box skips the reorder");
}

// Analytical pair terms and restraints through the mirror: a Coulomb pair
// and a restrained particle, against the closed forms.
static void analytic_terms_test(const Resource& res) {
	const int n = 3;
	B200Patch patch(res, n);
	patch.set_periodic_box(PeriodicBox(Vector3(0, 0, 0), Vector3(100, 100, 100)));
	// one type, Coulomb only (tag bit 0), no tables
	patch.set_pair_tables(1, {1u}, {});
	patch.set_pair_terms({1.0f}, {2.0f}, {0.5f});
	std::vector<Vector3> h = {Vector3(10, 10, 10), Vector3(14, 10, 10), Vector3(60, 60, 60)};
	DeviceBuffer<Vector3> pos(n, res), fe(n, res);
	DeviceBuffer<int> types(n, res);
	pos.copy_from_host(h);
	fe.fill_zero();
	types.copy_from_host(std::vector<int>(n, 0));
	patch.calculate_nonbonded_forces(pos, types, fe, n, 12.0f, 10.0f, 1, 20, true);
	std::vector<Vector3> f;
	fe.copy_to_host(f);
	const float want = 332.0636f / 16.0f;  // q q C / r^2 at r = 4
	EXPECT(std::fabs(f[1].x - want) < 1e-4f * want && std::fabs(f[0].x + want) < 1e-4f * want &&
			   f[2].x == 0.0f,
		   "Coulomb pair force q1 q2 C / r^2, opposite on the two particles");
	EXPECT(std::fabs(f[0].t - 0.5f * 332.0636f / 4.0f) < 1e-3f, "Coulomb energy halves");
	DeviceBuffer<int> rid(1, res);
	DeviceBuffer<Vector3> anchor(1, res);
	DeviceBuffer<float> rk(1, res);
	rid.copy_from_host(std::vector<int>{2});
	anchor.copy_from_host(std::vector<Vector3>{Vector3(57, 60, 60)});
	rk.copy_from_host(std::vector<float>{2.0f});
	fe.fill_zero();
	patch.calculate_dihedral_and_restraint_forces(pos, fe, nullptr, nullptr, 0, rid.data(),
												  anchor.data(), rk.data(), 1, true);
	fe.copy_to_host(f);
	EXPECT(std::fabs(f[2].x + 6.0f) < 1e-5f && std::fabs(f[2].t - 9.0f) < 1e-5f,
		   "restraint: F = -k (x - x0), E = k |x - x0|^2 / 2");
}

// SimOutput through the mirror: a frame and a restart in global-id order.
static void output_test(const Resource& res) {
	char dir[] = "/tmp/mb2outXXXXXX";
	if (!mkdtemp(dir)) {
		EXPECT(false, "output: temporary directory");
		return;
	}
	const std::string name = std::string(dir) + "/run";
	const int n = 4;
	SimOutput out(name, n, 1, 1, 0.5f, PeriodicBox(Vector3(0, 0, 0), Vector3(10, 10, 10)), false,
				  res);
	std::vector<Vector3> h = {Vector3(1, 2, 3), Vector3(4, 5, 6), Vector3(7, 8, 9),
							  Vector3(0.5f, 0.25f, 0.125f)};
	DeviceBuffer<Vector3> pos(n, res), fe(n, res);
	DeviceBuffer<int> types(n, res), ids(n, res);
	pos.copy_from_host(h);
	fe.copy_from_host(std::vector<Vector3>{Vector3(0, 0, 0, 1.5f), Vector3(0, 0, 0, 2.0f),
										   Vector3(0, 0, 0, -0.5f), Vector3(0, 0, 0, 0.0f)});
	types.copy_from_host(std::vector<int>{0, 1, 2, 3});
	ids.copy_from_host(std::vector<int>{3, 2, 1, 0});  // slot s holds global id 3 - s
	out.handle_output(1, pos, fe, types, 0.6f, nullptr, {}, ids.data());
	out.flush();
	FILE* f = std::fopen((name + ".restart").c_str(), "r");
	char line[128];
	std::string first;
	if (f && std::fgets(line, sizeof(line), f)) first = line;
	if (f) std::fclose(f);
	EXPECT(first == "3 0.5 0.25 0.125\n", "restart rows in global-id order, shortest decimals");
	const auto e = out.write_energy_output(fe, 0.6f);
	EXPECT(e.second == 3.0 && e.first == 0.0, "energy output: potential sum, no kinetic without momenta");
}

int main() {
	Resource res;
	res.device = 0;
	cuda_check(cudaSetDevice(0), "cudaSetDevice");
	try {
		lattice_tests(res);
		periodic_random_test(res);
		error_tests(res);
		patch_stage_test(res);
		langevin_stage_test(res);
		reorder_stage_test(res);
		analytic_terms_test(res);
		output_test(res);
	} catch (const std::exception& e) {
		std::printf("FAIL unexpected exception: %s\n", e.what());
		++failures;
	}
	std::printf(failures ? "FAILED %d\n" : "ALL PASS\n", failures);
	return failures ? 1 : 0;
}
