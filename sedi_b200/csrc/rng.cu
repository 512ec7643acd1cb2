// Probe generation.
//
// Host path: the reference's own generator, DistrRngStd::fill_plusminusone
// (DistrRngStd.hpp:22-42) -- std::mt19937 seeded with one value, a
// std::uniform_real_distribution<double>(0,1) draw per point, +1 when the draw
// is > 0.5 and -1 otherwise, points visited i1 fastest.  The same standard
// library code runs here, so the probes are the reference's bit for bit.
#include <random>

#include "sedi_internal.h"

namespace sedi {

void host_fill_probe(uint32_t seed, long n, double *out) {
	std::mt19937 engine(seed);
	std::uniform_real_distribution<double> dist(0.0, 1.0);
	for (long i = 0; i < n; i++) {
		const double x = dist(engine);
		out[i] = x > 0.5 ? 1.0 : -1.0;
	}
}

}  // namespace sedi
