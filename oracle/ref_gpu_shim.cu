// Test infrastructure only: a harness that runs the reference's OWN CUDA kick and drift.
//
// The reference's device code for the gravity step (src/kick.cu, src/gravity.cu,
// src/drift.cu, src/ewald_indices.cu, src/cuda_mem.cu, src/flops.cu, src/assert.cu,
// src/healpix.cu, src/analytic.cu) compiles as it stands for sm_100a (oracle/Makefile, target
// `refgpu`).  What it takes from the HPX-based host parts of the reference (particles.cpp,
// options.cpp, cuda.cpp, lightcone.cpp, hpx.cpp), which cannot be built here, is supplied
// below.  The harness places caller-given particles in the reference's global particle
// arrays (managed memory, as particles.cpp:774-839 does), lays a caller-given tree out as
// the reference's tree_node array (tree.hpp:98-110) with its multi_pos records, and calls
//   * cuda_execute_kicks (src/kick.cu:508) with one work item for the root, whose check
//     lists are {root} (the call kick() makes at the top of the tree, src/kick.cpp:150), so
//     that the reference's own kernel performs the whole dual tree walk; and
//   * cuda_drift (src/drift.cu:156) for one rung over the active range.
// Nothing here is part of the product; tests/ load it to compare the product with the
// reference.  Inputs must keep the reference's device asserts out of reach (its kernel
// traps on a failed assert): rungs below MAX_RUNG (16), a tree whose leaves satisfy the
// Ewald criterion (the tree_create leaf rule), and small problem sizes (one warp walks).
#define PARTICLES_CPP
#include <cosmictiger/cuda.hpp>
#include <cosmictiger/cuda_mem.hpp>
#include <cosmictiger/drift.hpp>
#include <cosmictiger/ewald_indices.hpp>
#include <cosmictiger/healpix.hpp>
#include <cosmictiger/hpx.hpp>
#include <cosmictiger/kick.hpp>
#include <cosmictiger/lightcone.hpp>
#include <cosmictiger/options.hpp>
#include <cosmictiger/particles.hpp>
#include <cosmictiger/tree.hpp>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ct_gravity.h"

// ---------------------------------------------------------------- host symbols the reference needs
static part_int g_n = 0;
static part_int g_rung_begin = 0;
static options g_opts;

part_int particles_size() {
	return g_n;
}

pair<part_int, part_int> particles_current_range() {
	pair<part_int, part_int> r;
	r.first = g_rung_begin;
	r.second = g_n;
	return r;
}

const options& get_options() {
	return g_opts;
}

int hpx_rank() {
	return 0;
}

int cuda_smp_count() {
	int dev = 0, n = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
	return n;
}

size_t cuda_free_mem() {
	size_t f = 0, t = 0;
	cudaMemGetInfo(&f, &t);
	return f;
}

void cuda_set_device() {
}

void cuda_stream_synchronize(cudaStream_t s) {
	cudaStreamSynchronize(s);
}

void cuda_malloc(void** ptr, size_t size, const char* file, int line) {
	if (cudaMalloc(ptr, size) != cudaSuccess) {
		fprintf(stderr, "reference harness: cudaMalloc of %zu bytes failed (%s:%d)\n", size, file, line);
		abort();
	}
}

void cosmictiger_assert(const char* cond, bool ok, const char* file, int line) {
	if (!ok) {
		fprintf(stderr, "reference assertion \"%s\" failed in %s line %d\n", cond, file, line);
		abort();
	}
}

// Where cuda_drift hands its per-block lightcone lists over (src/drift.cu:188): the harness
// collects the entries (the lists live in the reference's managed heap, readable here after
// the drift's synchronisation) instead of binning them into HEALPix maps and files.
static std::vector<lc_entry> g_lc;

size_t lc_add_parts(const device_vector<device_vector<lc_entry>>& entries, double, double) {
	size_t count = 0;
	for (int b = 0; b < entries.size(); b++) {
		const auto& list = entries[b];
		for (int j = 0; j < list.size(); j++) {
			g_lc.push_back(list[j]);
			count++;
		}
	}
	return count;
}

// ---------------------------------------------------------------- harness
namespace {

bool g_ready = false;

template<class T>
T* managed(size_t count) {
	T* p = nullptr;
	if (cudaMallocManaged(&p, sizeof(T) * (count ? count : 1)) != cudaSuccess) {
		return nullptr;
	}
	return p;
}

int set_particles(int64_t n, const uint32_t* x, const uint32_t* y, const uint32_t* z, const float* vxyz, const int8_t* rung, bool forces) {
	g_n = n;
	const uint32_t* src[3] = { x, y, z };
	for (int d = 0; d < NDIM; d++) {
		particles_x[d] = managed<fixed32>(n);
		if (!particles_x[d]) {
			return -1;
		}
		for (int64_t i = 0; i < n; i++) {
			particles_x[d][i].raw() = src[d][i];
		}
	}
	particles_v = managed<array<float, NDIM>>(n);
	particles_r = managed<char>(n);
	if (!particles_v || !particles_r) {
		return -1;
	}
	for (int64_t i = 0; i < n; i++) {
		for (int d = 0; d < NDIM; d++) {
			particles_v[i][d] = vxyz[3 * i + d];
		}
		particles_r[i] = (char) rung[i];
	}
	for (int d = 0; d < NDIM; d++) {
		particles_g[d] = forces ? managed<float>(n) : nullptr;
	}
	particles_p = forces ? managed<float>(n) : nullptr;
	return 0;
}

void get_particles(int64_t n, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, int8_t* rung) {
	uint32_t* dst[3] = { x, y, z };
	for (int d = 0; d < NDIM; d++) {
		if (dst[d]) {
			for (int64_t i = 0; i < n; i++) {
				dst[d][i] = particles_x[d][i].raw();
			}
		}
	}
	if (vxyz) {
		for (int64_t i = 0; i < n; i++) {
			for (int d = 0; d < NDIM; d++) {
				vxyz[3 * i + d] = particles_v[i][d];
			}
		}
	}
	if (rung) {
		for (int64_t i = 0; i < n; i++) {
			rung[i] = (int8_t) particles_r[i];
		}
	}
}

void free_particles() {
	for (int d = 0; d < NDIM; d++) {
		cudaFree(particles_x[d]);
		cudaFree(particles_g[d]);
		particles_x[d] = nullptr;
		particles_g[d] = nullptr;
	}
	cudaFree(particles_v);
	cudaFree(particles_r);
	cudaFree(particles_p);
	particles_v = nullptr;
	particles_r = nullptr;
	particles_p = nullptr;
	g_n = 0;
}

// The caller's tree (this project's exported node layout: ct_node, root at index 0) as the
// reference's tree_node array with its multi_pos records, in managed memory.
int lay_out_tree(int64_t nnodes, const ct_node* nodes, tree_node** tn_out, multi_pos** mp_out) {
	tree_node* tn = managed<tree_node>(nnodes);
	multi_pos* mp = managed<multi_pos>(nnodes);
	if (!tn || !mp) {
		cudaFree(tn);
		cudaFree(mp);
		return -1;
	}
	for (int64_t i = 0; i < nnodes; i++) {
		const ct_node& s = nodes[i];
		tree_node& t = tn[i];
		memset((void*) &t, 0, sizeof(t));
		for (int d = 0; d < NDIM; d++) {
			t.box.begin[d].raw() = s.box_begin[d];
			t.box.end[d].raw() = s.box_end[d];
			t.pos[d].raw() = s.pos[d];
			mp[i].pos[d].raw() = s.pos[d];
		}
		t.children[LEFT].proc = t.children[RIGHT].proc = 0;
		t.children[LEFT].index = s.child_left;
		t.children[RIGHT].index = s.child_right;
		t.part_range.first = s.part_begin;
		t.part_range.second = s.part_end;
		t.proc_range.first = 0;
		t.proc_range.second = 1;
		t.radius = s.radius;
		t.depth = s.depth;
		t.leaf = s.leaf ? 1 : 0;
		t.local_root = i == 0;
		for (int k = 0; k < MULTIPOLE_SIZE; k++) {
			mp[i].multi[k] = s.multi[k];
		}
		t.mpos = mp + i;
	}
	*tn_out = tn;
	*mp_out = mp;
	return 0;
}

kick_params make_params(const void* pp);

}  // namespace

extern "C" {

// Kick parameters in the reference's own meaning (kick.hpp:138-186).
typedef struct {
	float sign;
	int min_rung;
	float a, t0, theta, h, eta, GM, max_dt;
	int save_force, first_call, ascending, descending, top, do_phi;
} ctref_kick_params;

}  // extern "C"

namespace {
kick_params make_params(const void* pp) {
	const ctref_kick_params* p = (const ctref_kick_params*) pp;
	kick_params kp;
	kp.sign = p->sign;
	kp.min_level = 0;
	kp.min_rung = p->min_rung;
	kp.a = p->a;
	kp.t0 = p->t0;
	kp.theta = p->theta;
	kp.h = p->h;
	kp.eta = p->eta;
	kp.GM = p->GM;
	kp.vel_init = false;
	kp.save_force = p->save_force != 0;
	kp.first_call = p->first_call != 0;
	kp.gpu = true;
	kp.node_load = 0.f;
	kp.max_dt = p->max_dt;
	kp.ascending = p->ascending != 0;
	kp.descending = p->descending != 0;
	kp.top = p->top != 0;
	kp.do_phi = p->do_phi != 0;
	return kp;
}
}  // namespace

extern "C" {

// One-time set-up on the current device: the reference's device heap (cuda_mem_init, as
// cuda_init does, src/cuda.cpp:99-110, with a caller-chosen size) and its Ewald tables in
// __constant__ memory (ewald_const::init_gpu, src/ewald_indices.cu:30).
int ctref_init(double heap_bytes) {
	if (g_ready) {
		return 0;
	}
	g_opts.do_lc = false;
	g_opts.create_glass = false;
	cuda_mem_init((size_t) heap_bytes);
	ewald_const::init_gpu();
	if (cudaDeviceSynchronize() != cudaSuccess) {
		return -1;
	}
	g_ready = true;
	return 0;
}

// The reference's kick of every particle: its kernel walks the whole tree from the root.
// Particles are in tree order (the order the tree's particle ranges refer to); the tree is
// given in this project's exported node layout (ct_node, breadth-first, root at index 0).
// On return vxyz and rung hold the kicked velocities and new rungs; with save_force, gx, gy,
// gz and pot the forces and potentials; ret = {max_rung, pot, kin, dkin, xmom, ymom, zmom,
// nmom} of kick_return.
int ctref_kick(int64_t n, const uint32_t* x, const uint32_t* y, const uint32_t* z, float* vxyz, int8_t* rung, int64_t nnodes, const ct_node* nodes,
		const ctref_kick_params* p, float* gx, float* gy, float* gz, float* pot, double* ret) {
	if (!g_ready || n <= 0 || nnodes <= 0) {
		return -1;
	}
	if (set_particles(n, x, y, z, vxyz, rung, p->save_force != 0)) {
		free_particles();
		return -2;
	}
	tree_node* tn = nullptr;
	multi_pos* mp = nullptr;
	if (lay_out_tree(nnodes, nodes, &tn, &mp)) {
		free_particles();
		return -2;
	}
	const kick_params kp = make_params(p);
	kick_workitem wi;
	for (int k = 0; k < EXPANSION_SIZE; k++) {
		wi.L[k] = 0.f;
	}
	wi.pos = tn[0].pos;
	wi.self.proc = 0;
	wi.self.index = 0;
	wi.dchecklist.push_back(wi.self);
	wi.echecklist.push_back(wi.self);
	vector<kick_workitem> items;
	items.push_back(wi);
	const kick_return kr = cuda_execute_kicks(kp, particles_x[XDIM], particles_x[YDIM], particles_x[ZDIM], tn, items);
	cudaError_t e = cudaGetLastError();  // a failed launch is reported here, not by the sync
	if (e == cudaSuccess) {
		e = cudaDeviceSynchronize();
	}
	if (e == cudaSuccess) {
		get_particles(n, nullptr, nullptr, nullptr, vxyz, rung);
		if (p->save_force) {
			for (int64_t i = 0; i < n; i++) {
				gx[i] = particles_g[XDIM][i];
				gy[i] = particles_g[YDIM][i];
				gz[i] = particles_g[ZDIM][i];
				pot[i] = particles_p[i];
			}
		}
		ret[0] = kr.max_rung;
		ret[1] = kr.pot;
		ret[2] = kr.kin;
		ret[3] = kr.dkin;
		ret[4] = kr.xmom;
		ret[5] = kr.ymom;
		ret[6] = kr.zmom;
		ret[7] = kr.nmom;
	}
	cudaFree(tn);
	cudaFree(mp);
	free_particles();
	return e == cudaSuccess ? 0 : -3;
}

// Blocks of the reference's kick grid (kick_block_count, src/kick.cu:611-624: occupancy x
// SMs); its CPU top hands the GPU subtrees of at most min(16384, max(active / this, bucket))
// particles (kick.cpp:173-177).
int ctref_kick_block_count() {
	return g_ready ? kick_block_count() : -1;
}

// The reference's kick in its production form: cuda_execute_kicks (src/kick.cu:508-609) with
// the caller's work items -- the subtrees below the CPU top of the walk, each with its parent
// expansion, its centre and its direct and Ewald check lists (kick_workitem, kick.hpp:188-194;
// made by kick() at kick.cpp:169-190 and ordered by first particle, kick_workspace.cpp:308-310)
// -- on the caller's tree (ct_node layout; items index into it).  The kick runs `repeats` times
// on the same particle copy (velocities and rungs advance each time); ms[r] receives each call's
// time (CUDA events on the legacy default stream around the call: its host packing of the
// items, the copy to the device, the kernel, the read-back of kick_return and its device
// synchronisation).  Forces, potentials, velocities and rungs are those of the last call.
int ctref_kick_items(int64_t n, const uint32_t* x, const uint32_t* y, const uint32_t* z, float* vxyz, int8_t* rung, int64_t nnodes,
		const ct_node* nodes, const ctref_kick_params* p, int64_t nitems, const int32_t* self, const float* L, const uint32_t* pos,
		const int64_t* doff, const int32_t* dlist, const int64_t* eoff, const int32_t* elist, int repeats, float* gx, float* gy, float* gz,
		float* pot, double* ret, float* ms) {
	if (!g_ready || n <= 0 || nnodes <= 0 || nitems <= 0 || repeats < 1) {
		return -1;
	}
	if (set_particles(n, x, y, z, vxyz, rung, p->save_force != 0)) {
		free_particles();
		return -2;
	}
	tree_node* tn = nullptr;
	multi_pos* mp = nullptr;
	if (lay_out_tree(nnodes, nodes, &tn, &mp)) {
		free_particles();
		return -2;
	}
	const kick_params kp = make_params(p);
	vector<kick_workitem> items(nitems);
	for (int64_t i = 0; i < nitems; i++) {
		kick_workitem& w = items[i];
		for (int k = 0; k < EXPANSION_SIZE; k++) {
			w.L[k] = L[i * EXPANSION_SIZE + k];
		}
		for (int d = 0; d < NDIM; d++) {
			w.pos[d].raw() = pos[3 * i + d];
		}
		w.self.proc = 0;
		w.self.index = self[i];
		for (int64_t j = doff[i]; j < doff[i + 1]; j++) {
			tree_id t;
			t.proc = 0;
			t.index = dlist[j];
			w.dchecklist.push_back(t);
		}
		for (int64_t j = eoff[i]; j < eoff[i + 1]; j++) {
			tree_id t;
			t.proc = 0;
			t.index = elist[j];
			w.echecklist.push_back(t);
		}
	}
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	kick_return kr;
	cudaError_t e = cudaSuccess;
	for (int r = 0; r < repeats && e == cudaSuccess; r++) {
		cudaEventRecord(e0, 0);
		kr = cuda_execute_kicks(kp, particles_x[XDIM], particles_x[YDIM], particles_x[ZDIM], tn, items);
		cudaEventRecord(e1, 0);
		e = cudaGetLastError();
		if (e == cudaSuccess) {
			e = cudaEventSynchronize(e1);
		}
		if (e == cudaSuccess) {
			cudaEventElapsedTime(ms + r, e0, e1);
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	if (e == cudaSuccess) {
		e = cudaDeviceSynchronize();
	}
	if (e == cudaSuccess) {
		get_particles(n, nullptr, nullptr, nullptr, vxyz, rung);
		if (p->save_force) {
			for (int64_t i = 0; i < n; i++) {
				gx[i] = particles_g[XDIM][i];
				gy[i] = particles_g[YDIM][i];
				gz[i] = particles_g[ZDIM][i];
				pot[i] = particles_p[i];
			}
		}
		ret[0] = kr.max_rung;
		ret[1] = kr.pot;
		ret[2] = kr.kin;
		ret[3] = kr.dkin;
		ret[4] = kr.xmom;
		ret[5] = kr.ymom;
		ret[6] = kr.zmom;
		ret[7] = kr.nmom;
	}
	cudaFree(tn);
	cudaFree(mp);
	free_particles();
	return e == cudaSuccess ? 0 : -3;
}

// The reference's drift of the particles in [rung_begin, n) whose rung equals `rung`
// (cuda_drift, src/drift.cu:156; lightcone capture off, no drag).
int ctref_drift(int64_t n, int64_t rung_begin, uint32_t* x, uint32_t* y, uint32_t* z, const float* vxyz, const int8_t* rung, int level, float a, float dt) {
	if (!g_ready || n <= 0) {
		return -1;
	}
	if (set_particles(n, x, y, z, vxyz, rung, false)) {
		free_particles();
		return -2;
	}
	g_rung_begin = rung_begin;
	cuda_drift((char) level, a, dt, 0.f, dt, 1.f, 0.0);
	cudaError_t e = cudaGetLastError();  // a failed launch is reported here, not by the sync
	if (e == cudaSuccess) {
		e = cudaDeviceSynchronize();
	}
	if (e == cudaSuccess) {
		get_particles(n, x, y, z, nullptr, nullptr);
	}
	free_particles();
	g_rung_begin = 0;
	return e == cudaSuccess ? 0 : -3;
}

// The reference's drift with its lightcone capture on (options do_lc, lc_map_size = nside;
// create_glass selects its drag of pi, src/drift.cu:183): particles as in ctref_drift, the
// velocities written back (the drag changes them), and the recorded entries copied to out
// (at most max_out; *nout receives how many there were).  healpix_init fills the pixel tables
// of vec2pix_nest as the reference's start-up does.
int ctref_drift_lc(int64_t n, int64_t rung_begin, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, const int8_t* rung, int level, float a, float dt,
		float tau0, float tau1, float tau_max, int nside, int create_glass, ct_lc_entry* out, int64_t max_out, int64_t* nout) {
	if (!g_ready || n <= 0 || nside < 1 || nside > 8192) {
		return -1;
	}
	healpix_init();
	if (set_particles(n, x, y, z, vxyz, rung, false)) {
		free_particles();
		return -2;
	}
	g_rung_begin = rung_begin;
	g_opts.do_lc = true;
	g_opts.lc_map_size = nside;
	g_opts.create_glass = create_glass != 0;
	g_lc.clear();
	cuda_drift((char) level, a, dt, tau0, tau1, tau_max, 0.0);
	cudaError_t e = cudaGetLastError();
	if (e == cudaSuccess) {
		e = cudaDeviceSynchronize();
	}
	if (e == cudaSuccess) {
		get_particles(n, x, y, z, vxyz, nullptr);
		const int64_t m = std::min<int64_t>(max_out, (int64_t) g_lc.size());
		for (int64_t i = 0; i < m; i++) {
			const lc_entry& s = g_lc[i];
			out[i].x = s.x.raw();
			out[i].y = s.y.raw();
			out[i].z = s.z.raw();
			out[i].vx = s.vx;
			out[i].vy = s.vy;
			out[i].vz = s.vz;
			out[i].pix = s.pix;
		}
		*nout = (int64_t) g_lc.size();
	}
	g_opts.do_lc = false;
	g_opts.create_glass = false;
	free_particles();
	g_rung_begin = 0;
	return e == cudaSuccess ? 0 : -3;
}

}  // extern "C"
