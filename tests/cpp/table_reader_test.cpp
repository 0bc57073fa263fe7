// Prints a table read by marsb200::TableFile (mars_md_b200/host/b200_pairlist.hpp)
// so the tests can compare it with the Python reader and the reference's
// Table::read_file:
//   table_reader_test <file> <kind: 0 pair, 1 bond, 2 angle, 3 dihedral>
// Output: "n start step uniform step_inv" then one "x y" row per line, all
// floats in hexadecimal (%a).
#include "b200_pairlist.hpp"

#include <cstdio>
#include <cstdlib>

int main(int argc, char** argv) {
	if (argc != 3) return 2;
	using marsb200::TabulatedType;
	static const TabulatedType kinds[4] = {TabulatedType::NonBondedPair, TabulatedType::Bond,
										   TabulatedType::Angle, TabulatedType::Dihedral};
	const int k = std::atoi(argv[2]);
	if (k < 0 || k > 3) return 2;
	marsb200::TableFile t(kinds[k]);
	t.read_file(argv[1]);
	marsb200::TableFile raw(TabulatedType::Bond);
	raw.read_file(argv[1]);
	const bool uniform = raw.check_same_step_size();
	std::printf("%zu %a %a %d %a\n", t.X.size(), t.start, t.step_size, uniform ? 1 : 0,
				t.X.size() >= 2 ? t.to_table().step_inv : 0.0f);
	for (size_t i = 0; i < t.X.size(); ++i) std::printf("%a %a\n", t.X[i], t.Y[i]);
	return 0;
}
