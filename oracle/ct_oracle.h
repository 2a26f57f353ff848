// CPU oracle for the gravity step: test infrastructure only.
//
// A single-source C++ restatement of the reference's tree build (src/tree.cpp:273-601,
// src/particles.cpp:979-1018), kick walk (src/kick.cu:179-506, src/gravity.cu:44-404),
// leaf kick (src/kick.cu:53-177) and drift (src/drift.cu:36-154), plus an FP64 direct
// Ewald summation.  Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg
// load it, always as the checker; the product (libct_gravity.so) never links it.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Operator checks (order selects the 7 or 5 expansion). */
int ct_or_greens(int order, const float* X, float* D);
int ct_or_ewald_greens(int order, const float* X, float* D);
/* Same Ewald operator evaluated in FP64 (accuracy check of the FP32 path). */
int ct_or_ewald_greens_d(int order, const double* X, double* D);
void ct_or_m2l(int order, const float* M, const float* D, float* L, int do_phi);
void ct_or_m2l2(int order, const float* M, const float* D, float* L, int do_phi);
void ct_or_p2m(int order, const float* X, float* M);
void ct_or_m2m_d(int order, const double* M, const double* X, double* Mout);
void ct_or_l2l(int order, const float* L, const float* X, float* Lout, int do_phi);
void ct_or_l2p(int order, const float* L, const float* X, float* Lout, int do_phi);
void ct_or_ewald_tables(int order, float* real_idx, float* four_idx, float* four_exp, float* D0);

/* Mirror of the reference's kick_params (cosmictiger/kick.hpp:138-186). */
typedef struct {
	float sign;
	int min_rung;
	float a;
	float t0;
	float theta;
	float h;
	float eta;
	float GM;
	float max_dt;
	int save_force;
	int first_call;
	int ascending;
	int descending;
	int top;
	int do_phi;
} ct_or_kick_params;

/* Mirror of kick_return (cosmictiger/kick.hpp:92-136). */
typedef struct {
	int max_rung;
	double pot;
	double kin;
	double dkin;
	double xmom;
	double ymom;
	double zmom;
	double nmom;
} ct_or_kick_return;

/* Tree nodes in the oracle's own order (depth-first, left child first). */
typedef struct {
	uint64_t key;
	int32_t part_begin, part_end;
	int32_t child_left, child_right; /* -1 for leaves */
	uint32_t pos[3];
	float radius;
	int32_t box_begin[3], box_end[3]; /* fixed<int,29> raw */
	int32_t leaf;
	int32_t depth;
	float multi[37]; /* order-7 multipole (first NMULT entries used) */
} ct_or_node;

/* Build the tree over particles [begin, n) in place (reorders x,y,z,v,rung exactly as the
 * reference's partition does).  Returns the node count, -1 if max_nodes is too small, or -2
 * if a node at depth 127 still had to split (more than a bucket of coincident particles), where
 * the reference throws "Maximum depth exceeded" (tree.cpp:285-286, MAX_DEPTH 128).
 * Subtrees near the root are built on up to nthreads threads (<= 0: all cores), as the
 * reference forks its right children (tree.cpp:349-350); the result does not depend on it. */
int ct_or_tree_build(int order, int n, int begin, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, int8_t* rung, double theta, double hsoft,
		int bucket, ct_or_node* nodes, int max_nodes, int nthreads);

/* Kick over a tree built by ct_or_tree_build.  g/pot may be null unless save_force.
 * nthreads <= 0 uses every available core. */
int ct_or_kick(int order, const ct_or_kick_params* p, int nnodes, const ct_or_node* nodes, const uint32_t* x, const uint32_t* y, const uint32_t* z,
		float* vxyz, int8_t* rung, float* gx, float* gy, float* gz, float* pot, ct_or_kick_return* rc, int nthreads, double* flops);

/* The kick as work items.  ct_or_kick_plan_create runs the top of the walk (every node holding
 * more than max_parts particles that is not a leaf; max_parts <= 0: total / (16 nthreads)) on
 * nthreads threads, level by level, and keeps the subtrees below it as work items with their
 * check lists and parent expansions, ordered by first particle (the reference's CPU top and its
 * GPU work items, kick.cpp:150-507, kick_workspace.cpp:308-310).  The plan keeps pointers to
 * `nodes` and the positions, which must outlive it.
 * ct_or_kick_plan_items: per item its subtree root, particle count, the particles in its
 * direct check list and the length of its Ewald check list.
 * ct_or_kick_plan_run: walks the items with select[i] != 0 (NULL: all) -- only their particles
 * are kicked -- and stores each walked item's wall time in item_seconds (may be NULL); the
 * return sums the walked items and the top's flops.  A plan may run several times. */
void* ct_or_kick_plan_create(int order, const ct_or_kick_params* p, int nnodes, const ct_or_node* nodes, const uint32_t* x, const uint32_t* y,
		const uint32_t* z, int max_parts, int nthreads, int64_t* nitems, double* top_seconds);
void ct_or_kick_plan_items(const void* plan, int32_t* self, int32_t* nparts, int64_t* near_parts, int32_t* ewald_checks);
int ct_or_kick_plan_run(void* plan, float* vxyz, int8_t* rung, float* gx, float* gy, float* gz, float* pot, const int8_t* select, int nthreads,
		double* item_seconds, ct_or_kick_return* rc, double* flops);
void ct_or_kick_plan_destroy(void* plan);
/* The work items in the form the reference's cuda_execute_kicks takes them (kick_workitem,
 * kick.hpp:188-194): subtree root, parent expansion (nexp floats, zero padded), its centre,
 * and the direct and Ewald check lists (CSR: offsets of nitems + 1 entries). */
void ct_or_kick_plan_list_sizes(const void* plan, int64_t* ndirect, int64_t* newald);
void ct_or_kick_plan_export(const void* plan, int32_t* self, float* L, int nexp, uint32_t* pos, int64_t* doff, int32_t* dlist, int64_t* eoff,
		int32_t* elist);

/* Drift of one rung (src/drift.cu:36-154, lightcone excluded). */
void ct_or_drift(int n, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, const int8_t* rung, int which_rung, float a, float dt, double drag);

/* Lightcone record of one crossing (lc_entry, cosmictiger/lightcone.hpp:54-58). */
typedef struct {
	int32_t x, y, z; /* fixed<int,31>: position of the crossing relative to the observer */
	float vx, vy, vz;
	int32_t pix; /* HEALPix nested pixel */
} ct_or_lc_entry;

/* HEALPix nested pixel of the direction (x, y, z) at nside (vec2pix_nest, src/healpix.cu:55-171). */
int ct_or_healpix_nest(int nside, double x, double y, double z);

/* Drift of one rung with the lightcone capture of cuda_drift_kernel (src/drift.cu:36-154):
 * the particles' crossings of the light cone between tau0 and tau1 (period tau_max) in the 8
 * periodic images next to the observer.  Writes at most max_out entries (in particle order,
 * images in the reference's order) and returns how many crossings there were. */
int64_t ct_or_drift_lc(int n, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, const int8_t* rung, int which_rung, float a, float dt,
		double drag, float tau0, float tau1, float tau_max, int nside, ct_or_lc_entry* out, int64_t max_out);

/* Rung partition of [begin, n): particles with rung >= minrung end up at [return, n)
 * (src/particles.cpp:1029-1076). */
int ct_or_sort_by_rung(int n, int begin, int minrung, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, int8_t* rung);

/* FP64 direct Ewald force and potential on sinks from all n sources (unit mass each,
 * softened nearest image + smooth periodic correction). */
void ct_or_direct_ewald(int n, const uint32_t* x, const uint32_t* y, const uint32_t* z, int nsink, const uint32_t* sx, const uint32_t* sy,
		const uint32_t* sz, double h, double* gx, double* gy, double* gz, double* pot, int nthreads);

#ifdef __cplusplus
}
#endif
