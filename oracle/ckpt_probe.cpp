// Test infrastructure only (oracle build; never part of the library).
//
// Writes and reads checkpoints with the reference's own code: write_checkpoint and
// read_checkpoint (src/driver.cpp:1143-1200) with particles_save / particles_load
// (src/particles.cpp:1182-1227) and domains_save / domains_load (src/domain.cpp:87-107),
// compiled where they lie against the single-threaded HPX stand-in, for one rank.
//
//   ckpt_probe write <state.bin> <iter> [op...]   op: a minimum rung, "push" or "pop"
//   ckpt_probe resave <iter>
//
// write: loads the state (driver_params as its 176 raw bytes, int64 n, uint32 x[n], y[n], z[n],
// float v[n][3], int8 rung[n]), applies the rung operations with the reference's
// particles_sort_by_rung / particles_push_rungs / particles_pop_rungs from a full active range,
// builds the one-rank domain decomposition (domains_rebound) and writes
// checkpoint.<iter>/checkpoint.0.dat in the working directory (driver_params.iter is set to
// <iter>, as the reference names the directory after it).
// resave: read_checkpoint() of checkpoint.<iter>, then write_checkpoint() of what it loaded to
// the same file (the reference's own re-serialisation of a file it read).
#include "ref_host.h"

#include <cosmictiger/domain.hpp>
#include <cosmictiger/driver.hpp>
#include <cosmictiger/lightcone.hpp>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

// lightcone sections are written only with lightcone output (options.do_lc, off here)
void lc_save(FILE*) {
	abort();
}
void lc_load(FILE*) {
	abort();
}

static int write_main(int argc, char** argv) {
	FILE* f = fopen(argv[2], "rb");
	driver_params params;
	int64_t n = 0;
	if (!f || fread(&params, sizeof(params), 1, f) != 1 || fread(&n, sizeof(n), 1, f) != 1 || n < 0) {
		fprintf(stderr, "ckpt_probe: cannot read %s\n", argv[2]);
		return 2;
	}
	std::vector<uint32_t> X[NDIM];
	std::vector<float> V(3 * n);
	std::vector<int8_t> R(n);
	for (int d = 0; d < NDIM; d++) {
		X[d].resize(n);
		if (fread(X[d].data(), sizeof(uint32_t), n, f) != (size_t) n) {
			return 2;
		}
	}
	if (fread(V.data(), sizeof(float), 3 * n, f) != (size_t) (3 * n) || fread(R.data(), 1, n, f) != (size_t) n) {
		return 2;
	}
	fclose(f);
	g_opts.nparts = n;
	particles_resize(n);
	for (int64_t i = 0; i < n; i++) {
		for (int d = 0; d < NDIM; d++) {
			particles_pos(d, i).raw() = X[d][i];
			particles_vel(d, i) = V[3 * i + d];
		}
		particles_rung(i) = R[i];
	}
	particles_sort_by_rung(0);
	for (int a = 4; a < argc; a++) {
		if (!strcmp(argv[a], "push")) {
			particles_push_rungs();
		} else if (!strcmp(argv[a], "pop")) {
			particles_pop_rungs();
		} else {
			particles_sort_by_rung(atoi(argv[a]));
		}
	}
	domains_rebound();
	params.iter = atoi(argv[3]);
	write_checkpoint(params);
	return 0;
}

static int resave_main(char** argv) {
	g_opts.read_check = atoi(argv[2]);
	const driver_params params = read_checkpoint();
	write_checkpoint(params);
	return 0;
}

int main(int argc, char** argv) {
	ref_set_defaults();
	g_opts.do_lc = false;
	if (argc >= 4 && !strcmp(argv[1], "write")) {
		return write_main(argc, argv);
	}
	if (argc == 3 && !strcmp(argv[1], "resave")) {
		return resave_main(argv);
	}
	fprintf(stderr, "usage: ckpt_probe write <state.bin> <iter> [op...] | ckpt_probe resave <iter>\n");
	return 2;
}
