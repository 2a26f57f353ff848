// Internal definitions shared by the gravity-step translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ct_gravity.h"

namespace ct {

constexpr int MAX_ORDER_NEXP = 50;   // order-7 local expansion
constexpr int MAX_ORDER_NMULT = 37;  // order-7 multipole
constexpr int NMULT_STRIDE = 40;     // multipole stride in floats (16-byte aligned rows)
constexpr int NEXP_STRIDE = 52;      // expansion stride in floats (16-byte aligned rows)
constexpr int MAX_DEPTH = 128;       // cosmictiger/defs.hpp:86
constexpr int WARP = 32;
constexpr int MIN_PARTS_PCCP = 38;   // src/kick.cu:32

// Node record read by the walk: one 32-byte load per check.
struct __align__(16) NodeW {
	uint32_t x, y, z;  // expansion centre (fixed32)
	float radius;
	int32_t pbeg, pend;  // particle range
	int32_t child;       // left child index (right = child + 1), -1 for a leaf
	int32_t flags;       // bit 0: leaf
};

// Box of an ensemble that owns particle index p (sub_off has nsub + 1 entries).
__host__ __device__ inline int box_of(const int64_t* sub_off, int nsub, int64_t p) {
	int lo = 0, hi = nsub - 1;
	while (lo < hi) {
		const int mid = (lo + hi + 1) >> 1;
		if (sub_off[mid] <= p) {
			lo = mid;
		} else {
			hi = mid - 1;
		}
	}
	return lo;
}

// fixed32 helpers (cosmictiger/fixed.hpp)
__host__ __device__ inline float fixed_dist(uint32_t a, uint32_t b) {
	return float(int32_t(a - b)) * (1.0f / 4294967296.0f);
}
__host__ __device__ inline double fixed_to_double(uint32_t i) {
	return double(i) * (1.0 / 4294967296.0);
}
// double -> fixed32 by truncation, wrapping modulo 2^32 (x86-64 conversion semantics of the
// reference's fixed32 = double assignment, fixed.hpp:97-101)
__host__ __device__ inline uint32_t fixed_from_double(double x) {
#ifdef __CUDA_ARCH__
	return (uint32_t) __double2ll_rz(x * 4294967296.0);
#else
	return (uint32_t) (int64_t) (x * 4294967296.0);
#endif
}
__host__ __device__ inline int32_t range_fixed_from_double(double x) {
#ifdef __CUDA_ARCH__
	return __double2int_rz(x * 536870912.0);
#else
	return (int32_t) (x * 536870912.0);
#endif
}

struct DevBuf {
	void* p = nullptr;
	size_t bytes = 0;
};

struct Ctx;

// Per-box device state.
struct Box {
	int64_t n = 0;
	int64_t cap = 0;         // particles the x, v, rung arrays hold
	int64_t g_cap = 0;       // particles the g, pot arrays hold
	int sub_cap = 0;         // sub-boxes the per-box arrays hold
	int64_t rung_begin = 0;  // tree covers [rung_begin, n)
	// particles (SoA)
	uint32_t* x[3] = { nullptr, nullptr, nullptr };
	float* v[3] = { nullptr, nullptr, nullptr };
	int8_t* rung = nullptr;
	float* g[3] = { nullptr, nullptr, nullptr };
	float* pot = nullptr;
	// tree
	int64_t nnodes = 0;
	int64_t node_cap = 0;
	std::vector<int64_t> level_start;  // node index where each level begins (host copy)
	NodeW* nodes = nullptr;
	int32_t* nbox = nullptr;    // tight box, fixed<int,29>, 6 per node (b0 b1 b2 e0 e1 e2)
	float* multi = nullptr;     // NMULT_STRIDE per node
	uint64_t* key = nullptr;
	int32_t* depth = nullptr;
	int32_t* parent = nullptr;
	double* gbox = nullptr;     // geometric box, 6 per node (build)
	double* tbox = nullptr;     // tight box in double, 6 per node (upsweep)
	double* cen = nullptr;      // expansion centre in double, 3 per node (upsweep)
	double* multi_d = nullptr;  // multipole in double before rounding, NMULT_STRIDE per node
	bool tree_valid = false;
	ct_tree_params tparams;
	// ensemble: nsub independent periodic unit boxes stored back to back; sub-box s owns
	// particles [sub_off[s], sub_off[s+1]) and tree root node s
	int nsub = 1;
	std::vector<int64_t> sub_off;
	int64_t* d_sub_off = nullptr;
	double* d_sub_sums = nullptr;  // 9 kick sums per sub-box
	int* d_sub_maxrung = nullptr;
	float* d_sub_h = nullptr;      // per-box softening (null: the kick's h for all)
	float* d_sub_GM = nullptr;     // per-box GM (null: the kick's GM for all)
	std::vector<float> sub_h_host;
	int* d_sub_first = nullptr;    // per-box first_call flag (null: the kick's flag for all)
	std::vector<int64_t> rung_stack;  // saved active-range starts (particles_push_rungs)
	// kick results
	ct_counters counters;
	bool have_force = false;
	// lightcone capture (ct_drift_lightcone): entries [0, lc_count) of lc
	ct_lc_entry* lc = nullptr;
	int64_t lc_cap = 0;
	int64_t lc_count = 0;
	int64_t lc_last = 0;           // entries of the last capturing drift (sizes the next one's room)
	uint64_t* lc_cand = nullptr;   // candidate (particle, image) pairs of one drift
	int64_t lc_cand_cap = 0;
	unsigned long long* d_lc_ctr = nullptr;  // [0] candidates, [1] entries
};

// Frees a box's lightcone buffers (ct_lightcone.cu).
void lightcone_release(Ctx* c, Box* b);

struct KickBuffers;  // interaction lists and expansions of the kick (ct_kick.cu)

// Host-visible error state and stream.
struct Ctx {
	int device = 0;
	int order = 7;
	int nsm = 148;
	cudaStream_t stream = nullptr;
	cudaMemPool_t pool = nullptr;   // device memory of the context (stream-ordered on `stream`)
	size_t budget = 0;
	size_t used = 0;
	std::string err;
	std::vector<Box*> boxes;
	// pinned host staging
	void* pinned = nullptr;
	size_t pinned_bytes = 0;
	// scratch (grown on demand)
	std::vector<DevBuf> scratch;
	// device flags / counters
	int* d_flags = nullptr;       // [0] overflow, [1] dropped ewald, [2] depth overflow
	double* d_counters = nullptr; // interaction counters
	void* d_ewald_tab = nullptr;  // device copy of the Ewald tables (when not in __constant__)
	cudaEvent_t ev[16];
	// two more streams for the kick's M2L phase, whose three kernels (Ewald M2L, direct M2L,
	// P2L) run side by side: forked from `stream` by fork_ev and joined back by join_ev
	cudaStream_t side[2] = { nullptr, nullptr };
	cudaEvent_t fork_ev = nullptr, join_ev[2] = { nullptr, nullptr };
	ct_tuning tune = { 128, 1, 32 };  // P2P cell-list size, warps per tile, sinks per tile
	bool drift_timed = false;         // ev[6], ev[7] hold a recorded drift
	unsigned long long launches = 0;  // kernels of this library launched so far
	int compensated = 1;              // Neumaier-compensated P2P batch sums
	int priority = 0;                 // CUDA stream priority of stream and side[] (0: default)
	KickBuffers* kick = nullptr;      // owned; grown by the kick, freed with the context
};

// Device time between two recorded events, 0 if it is not available.  A failed query sets the
// runtime's last error; that error is this call's own and is cleared, so that it cannot
// surface in a later, unrelated check (a library routine that peeks at the last error).
inline float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
	float ms = 0.f;
	if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
		cudaGetLastError();
		ms = 0.f;
	}
	return ms;
}

// Frees the context's kick buffers (called by ct_ctx_destroy).
void kick_buffers_release(Ctx* c);

// Allocation with budget accounting.
ct_status dalloc(Ctx* c, void** p, size_t bytes, const char* what);
void dfree(Ctx* c, void* p, size_t bytes);
ct_status fail(Ctx* c, ct_status code, const std::string& msg);
ct_status cuda_check(Ctx* c, cudaError_t e, const char* what);

// Scratch buffer slot i, at least `bytes` (contents undefined).
void* scratch(Ctx* c, int slot, size_t bytes, ct_status* st);

// Translation-unit entry points.
ct_status tree_build(Ctx* c, Box* b, const ct_tree_params* p);
ct_status kick_run(Ctx* c, Box* b, const ct_kick_params* p, ct_kick_return* out);
ct_status drift_run(Ctx* c, Box* b, int rung, float a, float dt, double drag, bool events = true);
ct_status sort_by_rung_run(Ctx* c, Box* b, int min_rung);
ct_status ewald_init(Ctx* c);
ct_status step_hierarchical(Ctx* c, Box* b, const ct_step_params* p, ct_step_return* out);
ct_status rung_counts(Ctx* c, Box* b, uint64_t* counts);
ct_status direct_ewald_run(Ctx* c, Box* b, int64_t nsink, const uint32_t* sx, const uint32_t* sy, const uint32_t* sz, double h, double* gx,
		double* gy, double* gz, double* pot);

}  // namespace ct

#define CT_CUDA(c, call) do { cudaError_t _e = (call); if (_e != cudaSuccess) return ::ct::cuda_check((c), _e, #call); } while (0)
#define CT_TRY(expr) do { ct_status _s = (expr); if (_s != CT_OK) return _s; } while (0)
