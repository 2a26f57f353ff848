// Test infrastructure only: prints the sizes and field offsets of the reference's checkpoint
// and lightcone records (driver_params, cosmictiger/driver.hpp:26-43; domain_t,
// cosmictiger/domain.hpp:39-48; lc_entry, cosmictiger/lightcone.hpp:54-58) as the compiler lays
// them out, built against the reference's own headers (oracle/Makefile, target `layout`).
// Its output is the fixture tests/golden/ref_layouts.json that pins this project's copies of
// those layouts (cosmictiger_b200/checkpoint.py, ct_lc_entry).
#include <cosmictiger/driver.hpp>
#include <cosmictiger/domain.hpp>
#include <cosmictiger/lightcone.hpp>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
void cosmictiger_assert(const char*, bool ok, const char*, int) {
	if (!ok) {
		abort();
	}
}
int main() {
	printf("{\"driver_params\": {\"size\": %zu, \"energies\": %zu, \"max_rung\": %zu, \"bucket_size\": %zu, \"total_processed\": %zu, \"flops\": %zu, \"itime\": %zu},\n",
		sizeof(driver_params), offsetof(driver_params, energies), offsetof(driver_params, max_rung), offsetof(driver_params, bucket_size),
		offsetof(driver_params, total_processed), offsetof(driver_params, flops), offsetof(driver_params, itime));
	printf(" \"domain_t\": %zu, \"lc_entry\": {\"size\": %zu, \"vx\": %zu, \"pix\": %zu}}\n", sizeof(domain_t), sizeof(lc_entry), offsetof(lc_entry, vx), offsetof(lc_entry, pix));
	return 0;
}
