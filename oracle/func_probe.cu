// Test infrastructure only: evaluates the reference's own cloud kernel and its inverse window
// (cloud_weight, cloud_filter, cosmictiger/fft.hpp:116-134) and its growth factor
// (cosmos_growth_factor, src/cosmology.cpp:80-87) at fixed points, built from the reference's
// headers and src/cosmology.cpp (oracle/Makefile, target `funcs`).  Its output is the fixture
// tests/golden/ref_functions.json that pins this project's restatements of those functions.
#include <cosmictiger/fft.hpp>
#include <cosmictiger/cosmology.hpp>
#include <cosmictiger/flops.hpp>
#include <cosmictiger/options.hpp>
#include <cstdio>
#include <cstdlib>
void cosmictiger_assert(const char*, bool ok, const char*, int) {
	if (!ok) {
		abort();
	}
}
// host symbols cosmology.cpp takes from the HPX-based parts (not used by cosmos_growth_factor)
static options g_opts;
const options& get_options() {
	return g_opts;
}
void add_cpu_flops(int) {
}
int main() {
	printf("{\"cloud_weight\": [");
	for (int i = 0; i <= 80; i++) {
		const float x = -4.0f + 0.1f * i;
		printf("%s[%.9g, %.9g]", i ? ", " : "", x, cloud_weight(x));
	}
	printf("],\n \"cloud_filter\": [");
	for (int i = 0; i <= 40; i++) {
		const double kh = 0.08 * i;
		printf("%s[%.17g, %.17g]", i ? ", " : "", kh, cloud_filter(kh));
	}
	printf("],\n \"growth_factor\": [");
	const double oms[3] = { 0.25, 0.3111, 0.4 };
	const float as[5] = { 0.02f, 0.1f, 0.3f, 0.6f, 1.0f };
	int first = 1;
	for (double om : oms) {
		for (float a : as) {
			printf("%s[%.17g, %.9g, %.17g]", first ? "" : ", ", om, a, cosmos_growth_factor(om, a));
			first = 0;
		}
	}
	printf("]}\n");
	return 0;
}
