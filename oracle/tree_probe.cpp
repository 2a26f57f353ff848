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
#include <cosmictiger/options.hpp>
#include <cosmictiger/particles.hpp>
#include <cosmictiger/tree.hpp>
#include <cosmictiger/range.hpp>
#include <gsl/gsl_rng.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "ct_oracle.h"

// ---------------------------------------------------------------- host services
static options g_opts;
const options& get_options() {
	return g_opts;
}
int hpx_rank() {
	return 0;
}
int hpx_size() {
	return 1;
}
int hpx_hardware_concurrency() {
	return 1;
}
const vector<hpx::id_type>& hpx_localities() {
	static vector<hpx::id_type> l(1, 0);
	return l;
}
const vector<hpx::id_type>& hpx_children() {
	static vector<hpx::id_type> none;
	return none;
}
void profiler_enter(const char*) {
}
void profiler_exit() {
}
void stack_trace_activate() {
}
void add_cpu_flops(int) {
}
void cuda_set_device() {
}
int cuda_get_device() {
	return 0;
}
// the reference stops on an error here (THROW_ERROR prints its message, then asserts false,
// safe_io.hpp:64-75); the probe exits with status 3 so that the caller can tell it from a crash
void cosmictiger_assert(const char* what, bool ok, const char* file, int line) {
	if (!ok) {
		fflush(stdout);
		fprintf(stderr, "reference assertion failed: %s (%s:%d)\n", what, file, line);
		exit(3);
	}
}
range<double> domains_range(size_t) {
	fprintf(stderr, "tree_probe: domains_range is for several ranks\n");
	abort();
}
// managed memory as host memory (the probe runs on the CPU)
extern "C" {
cudaError_t cudaMallocManaged(void** p, size_t bytes, unsigned int) {
	*p = malloc(bytes ? bytes : 16);
	return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFree(void* p) {
	free(p);
	return cudaSuccess;
}
cudaError_t cudaMemAdvise(const void*, size_t, enum cudaMemoryAdvise, int) {
	return cudaSuccess;
}
cudaError_t cudaMemPrefetchAsync(const void*, size_t, int, cudaStream_t) {
	return cudaSuccess;
}
const char* cudaGetErrorString(cudaError_t) {
	return "tree_probe: no CUDA";
}
}
// the reference's random initial conditions and sampler are not reached
const gsl_rng_type* gsl_rng_taus = nullptr;
gsl_rng* gsl_rng_alloc(const gsl_rng_type*) {
	abort();
}
void gsl_rng_set(const gsl_rng*, unsigned long int) {
	abort();
}
double gsl_rng_uniform(const gsl_rng*) {
	abort();
}
unsigned long int gsl_rng_get(const gsl_rng*) {
	abort();
}
void gsl_rng_free(gsl_rng*) {
	abort();
}

// ---------------------------------------------------------------- tree output
static void emit(tree_id id, uint64_t key, int depth, std::vector<ct_or_node>& out) {
	const tree_node* nd = tree_get_node(id);
	const int me = (int) out.size();
	out.emplace_back();
	ct_or_node r;
	memset(&r, 0, sizeof(r));
	r.key = key;
	r.part_begin = nd->part_range.first;
	r.part_end = nd->part_range.second;
	for (int d = 0; d < NDIM; d++) {
		r.pos[d] = nd->pos[d].raw();
		r.box_begin[d] = nd->box.begin[d].raw();
		r.box_end[d] = nd->box.end[d].raw();
	}
	r.radius = nd->radius;
	r.leaf = nd->leaf;
	r.depth = nd->depth;
	if (depth != (int) nd->depth) {
		fprintf(stderr, "tree_probe: depth %d at key %llu, node says %d\n", depth, (unsigned long long) key, (int) nd->depth);
		abort();
	}
	for (int i = 0; i < 37 && i < MULTIPOLE_SIZE; i++) {
		r.multi[i] = nd->mpos ? nd->mpos->multi[i] : 0.f;
	}
	r.child_left = r.child_right = -1;
	if (!nd->leaf) {
		r.child_left = (int) out.size();
		emit(nd->children[LEFT], key << 1, depth + 1, out);
		r.child_right = (int) out.size();
		emit(nd->children[RIGHT], (key << 1) + 1, depth + 1, out);
	}
	out[me] = r;
}

static void set_defaults() {
	// the reference's defaults (src/options.cpp:173-175)
	g_opts.tree_cache_line_size = 65536 / sizeof(tree_node);
	g_opts.tree_alloc_line_size = 16 * g_opts.tree_cache_line_size;
	g_opts.part_cache_line_size = 131072 / (sizeof(fixed32) * NDIM);
	g_opts.save_force = false;
	g_opts.do_groups = false;
	g_opts.do_tracers = false;
}

static int rungs_main(int argc, char** argv) {
	set_defaults();
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
	set_defaults();
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
		emit(rc.id, 1, 0, out);
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
