// Test infrastructure only (oracle build; never part of the library).
//
// Host services that the reference's src/tree.cpp, src/particles.cpp and src/driver.cpp take
// from the rest of the reference (options, HPX localities, profiler, assertion, CUDA managed
// memory, GSL), for the probes that run those sources where they lie in one process
// (oracle/tree_probe.cpp, oracle/ladder_probe.cpp), and the export of the reference's tree in
// the node layout of this project's CPU restatement (ct_or_node, oracle/ct_oracle.h).
#include "ref_host.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>

// ---------------------------------------------------------------- host services
options g_opts;
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
// weak: the ladder probe defines its own
__attribute__((weak)) void hpx_yield() {
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
// weak: the checkpoint probe links the reference's own src/domain.cpp
__attribute__((weak)) range<double> domains_range(size_t) {
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
// the reference's random initial conditions and sampler are not reached by the tree and ladder
// probes; weak, so that the initial-condition probe (oracle/ic_probe.cpp) supplies the generator
__attribute__((weak)) const gsl_rng_type* gsl_rng_taus = nullptr;
__attribute__((weak)) gsl_rng* gsl_rng_alloc(const gsl_rng_type*) {
	abort();
}
__attribute__((weak)) void gsl_rng_set(const gsl_rng*, unsigned long int) {
	abort();
}
__attribute__((weak)) double gsl_rng_uniform(const gsl_rng*) {
	abort();
}
__attribute__((weak)) double gsl_rng_uniform_pos(const gsl_rng*) {
	abort();
}
__attribute__((weak)) unsigned long int gsl_rng_get(const gsl_rng*) {
	abort();
}
__attribute__((weak)) void gsl_rng_free(gsl_rng*) {
	abort();
}

// ---------------------------------------------------------------- tree output
void ref_emit_tree(tree_id id, uint64_t key, int depth, std::vector<ct_or_node>& out) {
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
		ref_emit_tree(nd->children[LEFT], key << 1, depth + 1, out);
		r.child_right = (int) out.size();
		ref_emit_tree(nd->children[RIGHT], (key << 1) + 1, depth + 1, out);
	}
	out[me] = r;
}


void ref_set_defaults() {
	// the reference's defaults (src/options.cpp:173-175)
	g_opts.tree_cache_line_size = 65536 / sizeof(tree_node);
	g_opts.tree_alloc_line_size = 16 * g_opts.tree_cache_line_size;
	g_opts.part_cache_line_size = 131072 / (sizeof(fixed32) * NDIM);
	g_opts.save_force = false;
	g_opts.do_groups = false;
	g_opts.do_tracers = false;
}

