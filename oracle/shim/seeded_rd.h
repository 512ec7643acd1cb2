/*
 * Pre-include (g++ -include) that makes the reference probe generator
 * reproducible without editing it.  Test infrastructure, not product code.
 *
 * DistrRngStd::fill_plusminusone (DistrRngStd.hpp:27-29) builds a fresh
 * std::random_device on every call and seeds std::mt19937 with one rd()
 * draw, so the reference probes are not reproducible.  Here every
 * `std::random_device` in the reference headers names a stand-in whose k-th
 * draw in the process returns SEDI_SEED + k (SEDI_SEED from the environment,
 * default 1234).  Because the reference draws exactly once per probe, probe k
 * (0-based) is generated by std::mt19937(SEDI_SEED + k) followed by
 * std::uniform_real_distribution<double>(0,1) and the x > 0.5 test
 * (DistrRngStd.hpp:32-40), all of it the reference's own unmodified code.
 */
#ifndef SEDI_ORACLE_SEEDED_RD_H
#define SEDI_ORACLE_SEEDED_RD_H

#include <random>
#include <cstdlib>

namespace std {
class sedi_seeded_random_device {
public:
	typedef unsigned int result_type;
	sedi_seeded_random_device() {}
	explicit sedi_seeded_random_device(const std::string &) {}
	result_type operator()() {
		static unsigned long long draws = 0;
		const char *env = getenv("SEDI_SEED");
		unsigned long long base = env ? strtoull(env, 0, 10) : 1234ull;
		return (result_type)(base + draws++);
	}
	double entropy() const { return 0.0; }
	static constexpr result_type min() { return 0; }
	static constexpr result_type max() { return ~0u; }
};
} // namespace std

#define random_device sedi_seeded_random_device

#endif
