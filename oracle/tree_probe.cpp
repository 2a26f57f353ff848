// Test infrastructure only (oracle build; never part of the library).
//
// Runs the reference's own tree build -- tree_create (src/tree.cpp:273-601) with its particle
// partition particles_sort (src/particles.cpp:979-1018) -- compiled where the sources lie
// (`make -C oracle tree`, objects in oracle/_ref/), on particles read from a file, and writes
// the resulting tree in the node layout of this project's CPU restatement (ct_or_node,
// oracle/ct_oracle.h: depth first, left child first, heap keys) together with the particle
// order the partition left.  HPX is replaced by the single-threaded stand-in in
// oracle/stub/hpx (every fork runs at once on the calling thread; the reference's node indices
// depend on its threads, its keys, ranges and geometry do not), one locality, and the few
// host services those sources take from the rest of the reference are defined below.
//
//   tree_probe <in> <out> <theta> <hsoft> <bucket>
//   in:  int64 n, then n x, n y, n z (uint32 fixed-point positions)
//   out: int64 node count, the nodes (ct_or_node records), then n x, n y, n z after the build
//
// With --rungs it runs the reference's rung partition instead (particles_sort_by_rung,
// src/particles.cpp:1029-1076, with particles_push_rungs / particles_pop_rungs,
// src/particles.cpp:218-235) for a sequence of operations:
//   tree_probe --rungs <in> <out> <op>...     op: a minimum rung, "push" or "pop"
//   in:  int64 n, then n x, n y, n z (uint32), n x 3 velocities (float), n rungs (int8)
//   out: int64 count of ops, the active-range start after each (int64), then the arrays as read
#include "ref_host.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

static int rungs_main(int argc, char** argv) {
	ref_set_defaults();
	FILE* f = fopen(argv[2], "rb");
	int64_t n = 0;
	if (!f || fread(&n, sizeof(n), 1, f) != 1 || n < 0) {
		fprintf(stderr, "tree_probe: cannot read %s\n", argv[2]);
		return 1;
	}
	std::vector<uint32_t> X[NDIM];
	std::vector<float> V(3 * n);
	std::vector<int8_t> R(n);
	bool ok = true;
	for (int d = 0; d < NDIM; d++) {
		X[d].resize(n);
		ok = ok && fread(X[d].data(), sizeof(uint32_t), n, f) == (size_t) n;
	}
	ok = ok && fread(V.data(), sizeof(float), 3 * n, f) == (size_t) (3 * n) && fread(R.data(), 1, n, f) == (size_t) n;
	fclose(f);
	if (!ok) {
		fprintf(stderr, "tree_probe: short read\n");
		return 1;
	}
	g_opts.nparts = n;
	particles_resize(n);
	for (part_int i = 0; i < n; i++) {
		for (int d = 0; d < NDIM; d++) {
			particles_pos(d, i).raw() = X[d][i];
			particles_vel(d, i) = V[3 * i + d];
		}
		particles_rung(i) = R[i];
	}
	particles_sort_by_rung(0);
	std::vector<int64_t> begins;
	for (int a = 4; a < argc; a++) {
		if (!strcmp(argv[a], "push")) {
			particles_push_rungs();
		} else if (!strcmp(argv[a], "pop")) {
			particles_pop_rungs();
		} else {
			particles_sort_by_rung(atoi(argv[a]));
		}
		begins.push_back(particles_current_range().first);
	}
	for (part_int i = 0; i < n; i++) {
		for (int d = 0; d < NDIM; d++) {
			X[d][i] = particles_pos(d, i).raw();
			V[3 * i + d] = particles_vel(d, i);
		}
		R[i] = particles_rung(i);
	}
	FILE* g = fopen(argv[3], "wb");
	const int64_t cnt = (int64_t) begins.size();
	ok = g && fwrite(&cnt, sizeof(cnt), 1, g) == 1 && fwrite(begins.data(), sizeof(int64_t), begins.size(), g) == begins.size();
	for (int d = 0; d < NDIM && ok; d++) {
		ok = fwrite(X[d].data(), sizeof(uint32_t), n, g) == (size_t) n;
	}
	ok = ok && fwrite(V.data(), sizeof(float), 3 * n, g) == (size_t) (3 * n) && fwrite(R.data(), 1, n, g) == (size_t) n;
	if (!g || !ok || fclose(g) != 0) {
		fprintf(stderr, "tree_probe: cannot write %s\n", argv[3]);
		return 1;
	}
	return 0;
}

int main(int argc, char** argv) {
	if (argc >= 4 && !strcmp(argv[1], "--rungs")) {
		return rungs_main(argc, argv);
	}
	if (argc != 6) {
		fprintf(stderr, "usage: tree_probe <in> <out> <theta> <hsoft> <bucket>\n");
		return 2;
	}
	const double theta = atof(argv[3]);
	g_opts.hsoft = atof(argv[4]);
	g_opts.bucket_size = atoi(argv[5]);
	ref_set_defaults();
	g_opts.theta = theta;
	FILE* f = fopen(argv[1], "rb");
	int64_t n = 0;
	if (!f || fread(&n, sizeof(n), 1, f) != 1 || n < 0) {
		fprintf(stderr, "tree_probe: cannot read %s\n", argv[1]);
		return 1;
	}
	std::vector<uint32_t> X[NDIM];
	for (int d = 0; d < NDIM; d++) {
		X[d].resize(n);
		if (fread(X[d].data(), sizeof(uint32_t), n, f) != (size_t) n) {
			fprintf(stderr, "tree_probe: short read\n");
			return 1;
		}
	}
	fclose(f);
	g_opts.nparts = n;
	particles_resize(n);
	for (part_int i = 0; i < n; i++) {
		for (int d = 0; d < NDIM; d++) {
			particles_pos(d, i).raw() = X[d][i];
			particles_vel(d, i) = 0.f;
		}
		particles_rung(i) = 0;
	}
	particles_sort_by_rung(0);  // the active range is every particle
	tree_create_params params(0, theta, g_opts.hsoft);
	std::vector<ct_or_node> out;
	try {
		const tree_create_return rc = tree_create(params);
		ref_emit_tree(rc.id, 1, 0, out);
	} catch (const std::exception& e) {
		fprintf(stderr, "tree_probe: the reference's tree_create threw: %s\n", e.what());
		return 3;
	}
	FILE* g = fopen(argv[2], "wb");
	const int64_t cnt = (int64_t) out.size();
	bool ok = g && fwrite(&cnt, sizeof(cnt), 1, g) == 1 && fwrite(out.data(), sizeof(ct_or_node), out.size(), g) == out.size();
	for (int d = 0; d < NDIM && ok; d++) {
		for (part_int i = 0; i < n; i++) {
			X[d][i] = particles_pos(d, i).raw();
		}
		ok = fwrite(X[d].data(), sizeof(uint32_t), n, g) == (size_t) n;
	}
	if (!g || !ok || fclose(g) != 0) {
		fprintf(stderr, "tree_probe: cannot write %s\n", argv[2]);
		return 1;
	}
	return 0;
}
