/*
 * ct_gravity.h — C ABI of the B200 gravity step (tree build, kick, drift).
 *
 * Drop-in boundary for the reference's gravity call surface.  Every entry point is
 * extern "C", takes plain pointers and sizes, returns a ct_status (0 = success, negative
 * = error; the message is available from ct_last_error) and never throws.  A context owns
 * one CUDA device, one stream and every box's device-resident state between calls.
 * Calls on one context must come from one host thread at a time.
 *
 * Reference interfaces replaced (paths inside dmarce1/cosmictiger):
 *   particle store       cosmictiger/particles.hpp:159-171 (particles_x/v/r/g/p globals)
 *   sort_by_rung         src/particles.cpp:1029-1076  particles_sort_by_rung(int)
 *   tree_create          cosmictiger/tree.hpp:209-210, src/tree.cpp:273-601
 *   kick                 cosmictiger/kick.hpp:199-200, src/kick.cpp:150-507,
 *                        src/kick.cu:179-609 (cuda_execute_kicks)
 *   drift                cosmictiger/drift.hpp:51-54, src/drift.cu:36-185
 *   ewald_const::init    cosmictiger/ewald_indices.hpp:32-41, src/ewald_indices.cu:30-114
 *   drift with lightcone src/drift.cu:36-195 (do_lc), src/healpix.cu:55-171, lc_add_parts input
 *   initialize           src/initialize.cpp:261-355 (Zel'dovich / 2LPT from power.init)
 *   power spectrum       src/power.cpp:33-77, src/power.cu:32-85, src/fft.cpp:172-360
 */
#ifndef CT_GRAVITY_H
#define CT_GRAVITY_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int ct_status;
#define CT_OK 0
#define CT_ERR_ARG -1        /* invalid argument */
#define CT_ERR_CUDA -2       /* a CUDA runtime call failed */
#define CT_ERR_MEMORY -3     /* device memory or HBM budget exhausted */
#define CT_ERR_CAPACITY -4   /* an internal list overflowed even after regrowth */
#define CT_ERR_STATE -5      /* call out of order (e.g. kick before tree_create) */

typedef struct ct_ctx ct_ctx;

/* Mirror of kick_params (cosmictiger/kick.hpp:138-186); field meaning is the reference's.
 * min_level, gpu, node_load and vel_init have no role on a single device and are absent. */
typedef struct {
	float sign;       /* +1, or -1 for glass creation */
	int min_rung;     /* rung being kicked */
	float a;          /* scale factor */
	float t0;         /* top-level time step */
	float theta;      /* opening angle */
	float h;          /* softening kernel support (box units) */
	float eta;        /* time-step criterion */
	float GM;         /* gravitational constant times particle mass */
	float max_dt;     /* cap on a particle's time step */
	int save_force;   /* keep g and phi per particle */
	int first_call;   /* first kick of a run: no ascending half kick */
	int ascending;    /* apply the ascending half kick */
	int descending;   /* assign rungs and apply the descending half kick */
	int top;          /* top of the rung ladder */
	int do_phi;       /* compute potentials */
} ct_kick_params;

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
} ct_kick_return;

/* Tree-construction parameters (tree_create_params, cosmictiger/tree.hpp:186-207, plus the
 * option values tree_create reads: bucket_size and hsoft, src/options.cpp:107,165,217). */
typedef struct {
	int min_rung;     /* tree over particles with rung >= min_rung, i.e. [rung_begin, n) */
	double theta;
	double hsoft;     /* softening support h, box units */
	int bucket;       /* leaf capacity (reference default 128) */
} ct_tree_params;

/* A tree node as exported for inspection (the reference's tree_node, tree.hpp:98-169,
 * plus its heap key).  Order of export: breadth-first. */
typedef struct {
	uint64_t key;            /* heap key: root 1, children 2k and 2k+1 */
	int32_t part_begin, part_end;
	int32_t child_left, child_right; /* export indices, -1 for leaves */
	uint32_t pos[3];         /* expansion centre, fixed32 */
	float radius;
	int32_t box_begin[3], box_end[3]; /* tight box, fixed<int,29> raw */
	int32_t leaf;
	int32_t depth;
	float multi[37];         /* multipole (first (order-1)^2+1 used) */
} ct_node;

/* Counters of the last kick (interactions by kind and the reference's flop convention). */
typedef struct {
	double pp_pairs;      /* particle-particle pairs */
	double cc_direct;     /* M2L, direct Green's function */
	double cc_ewald;      /* M2L, Ewald Green's function */
	double cp_pairs;      /* P2L (particle -> local expansion) */
	double pc_pairs;      /* M2P (multipole -> particle) */
	double nodes;
	double leaves;
	double flops;         /* total, per the reference's per-interaction counts */
	double flops_pp;
	double flops_cc;
	double ms_tree, ms_walk, ms_m2l, ms_l2l, ms_leaf, ms_drift; /* device time of the last calls */
	double ms_leafkick;   /* M2P + L2P + kick after the P2P kernel */
	double pp_near;       /* pairs from source leaves within the softening length of the sink
	                         leaf (the per-pair softening test runs on these only) */
} ct_counters;

/* ---- context */
ct_status ct_ctx_create(ct_ctx** out, int device, size_t hbm_budget_bytes, int order);
void ct_ctx_destroy(ct_ctx* ctx);
const char* ct_last_error(const ct_ctx* ctx);
int ct_order(const ct_ctx* ctx);
/* Number of this library's kernels launched on the context so far. */
unsigned long long ct_launch_count(const ct_ctx* ctx);

/* ---- boxes (independent periodic unit boxes with their own particles and tree) */
ct_status ct_box_create(ct_ctx* ctx, int64_t n, int* box_id);
ct_status ct_box_destroy(ct_ctx* ctx, int box_id);
int64_t ct_box_size(const ct_ctx* ctx, int box_id);

/* An ensemble: nbox independent periodic unit boxes in one device structure, box s holding
 * counts[s] particles stored after those of boxes 0..s-1.  Every call on it (tree build, kick,
 * drift, transfers of the concatenated arrays) covers all boxes with one set of kernel
 * launches; the boxes never interact.  Kicked with all particles active (min_rung 0). */
ct_status ct_ensemble_create(ct_ctx* ctx, int nbox, const int64_t* counts, int* box_id);
/* Per-box softening h and GM of an ensemble (box s: h[s], GM[s]); without this call every box
 * uses the kick's h and GM.  The tree build's leaf criterion uses the tree parameters' hsoft. */
ct_status ct_ensemble_set_params(ct_ctx* ctx, int box_id, const float* h, const float* GM);
/* New membership for an existing ensemble: nbox boxes of counts[0..nbox) particles.  Device
 * arrays are kept and grown only when the new totals exceed what they hold, so a serving loop
 * can re-batch every step without reallocating; particle contents, per-box parameters and
 * first-call flags are undefined afterwards (gather or upload, set_params, set_first_call). */
ct_status ct_ensemble_reshape(ct_ctx* ctx, int box_id, int nbox, const int64_t* counts);
/* Per-box first_call flags of an ensemble (boxes joining a batch start their own runs). */
ct_status ct_ensemble_set_first_call(ct_ctx* ctx, int box_id, const int* first_call);
/* Copy the particles of plain boxes boxes[0..count) into the ensemble's slots (gather) or
 * back (scatter), device to device; count must equal the ensemble's box count and box s must
 * have the size of slot s. */
ct_status ct_ensemble_gather(ct_ctx* ctx, int ens_id, const int* boxes, int count);
ct_status ct_ensemble_scatter(ct_ctx* ctx, int ens_id, const int* boxes, int count);
/* Device bytes currently allocated by the context (compared against its HBM budget). */
size_t ct_bytes_in_use(const ct_ctx* ctx);
/* Number of boxes of an ensemble (1 for a plain box). */
int ct_box_count(const ct_ctx* ctx, int box_id);
/* Kick of every box of an ensemble; results[s] receives box s's kick_return. */
ct_status ct_kick_ensemble(ct_ctx* ctx, int box_id, const ct_kick_params* params, ct_kick_return* results);

/* Host <-> device transfers.  x,y,z: fixed32 positions (uint32, 2^-32 box units);
 * vxyz: float[3*n] interleaved velocities (the reference's particles_v layout);
 * rung: int8[n].  Download arguments may be NULL to skip a field; g/pot only exist after a
 * kick with save_force.  An upload replaces particle data in place and keeps the active range
 * set by ct_sort_by_rung (min_rung 0 resets it). */
ct_status ct_box_upload(ct_ctx* ctx, int box_id, const uint32_t* x, const uint32_t* y, const uint32_t* z, const float* vxyz, const int8_t* rung);
ct_status ct_box_download(ct_ctx* ctx, int box_id, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, int8_t* rung, float* gx, float* gy,
		float* gz, float* pot);

/* Device-pointer variants (same layout, memory on the context's device). */
ct_status ct_box_upload_device(ct_ctx* ctx, int box_id, const uint32_t* x, const uint32_t* y, const uint32_t* z, const float* vxyz,
		const int8_t* rung);
ct_status ct_box_download_device(ct_ctx* ctx, int box_id, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, int8_t* rung, float* gx,
		float* gy, float* gz, float* pot);

/* ---- the gravity step (particles_sort_by_rung, tree_create, kick, drift) */
ct_status ct_sort_by_rung(ct_ctx* ctx, int box_id, int min_rung, int64_t* rung_begin);
ct_status ct_tree_create(ct_ctx* ctx, int box_id, const ct_tree_params* params, int64_t* node_count);
ct_status ct_kick(ct_ctx* ctx, int box_id, const ct_kick_params* params, ct_kick_return* result);
ct_status ct_drift(ct_ctx* ctx, int box_id, int rung, float a, float dt, double drag);

/* ---- drift with the lightcone capture of cuda_drift (src/drift.cu:36-195) */

/* One crossing of the light cone (lc_entry, cosmictiger/lightcone.hpp:54-58): the crossing point
 * relative to the observer at the origin, fixed<int,31> (2^-31 box units, in [-1, 1]); the
 * particle's velocity (code units, after drag); its HEALPix nested pixel at nside. */
typedef struct {
	int32_t x, y, z;
	float vx, vy, vz;
	int32_t pix;
} ct_lc_entry;

/* Lightcone of the drift (cuda_drift's tau0, tau1, tau_max and options lc_map_size): crossings of
 * the period boundaries k * tau_max between tau0 and tau1 are recorded in the 8 periodic images
 * next to the observer, when tau_max - tau1 < 1 (src/drift.cu:38). */
typedef struct {
	float tau0;
	float tau1;
	float tau_max;
	int nside; /* 1 .. 8192 */
} ct_lc_params;

/* ct_drift plus the lightcone capture.  The crossings are appended to the box's lightcone buffer
 * (grown as needed; no crossing is dropped); *captured (optional) receives this call's count.
 * Waits for the drift to finish (the reference's cuda_drift synchronises the same way).
 * Replaces cuda_drift(rung, a, dt, tau0, tau1, tau_max, drag) with options do_lc (drift.cu:156). */
ct_status ct_drift_lightcone(ct_ctx* ctx, int box_id, int rung, float a, float dt, double drag, const ct_lc_params* lc, int64_t* captured);

/* Entries held in the box's lightcone buffer. */
ct_status ct_lightcone_count(ct_ctx* ctx, int box_id, int64_t* count);

/* Copies up to max_entries entries (host memory) and, with clear != 0, empties the buffer;
 * *count receives the number held before the call.  The order of entries within one drift is
 * unspecified (the reference's is per block of its kernel). */
ct_status ct_lightcone_download(ct_ctx* ctx, int box_id, ct_lc_entry* out, int64_t max_entries, int64_t* count, int clear);

/* Sets the buffer's capacity in entries (at least what it holds); the drift grows it as needed. */
ct_status ct_lightcone_reserve(ct_ctx* ctx, int box_id, int64_t entries);

/* ---- initial conditions: Zel'dovich / 2LPT displacements of a lattice
 * (initialize, src/initialize.cpp:261-355; the field of twolpt_generate, :436-540) */
typedef struct {
	int nfour;              /* particles per dimension = FFT grid (parts_dim = Nfour), even, 4 .. 1024 */
	double box_size;        /* box size in Mpc (code_to_cm / mpc_to_cm) */
	double omega_m;         /* matter density (omega_b + omega_c) */
	double z0;              /* starting redshift */
	double hubble;          /* h */
	double sigma8;          /* normalisation of the table */
	double H0;              /* Hubble constant in code time units (constants::H0 code_to_s h) */
	int twolpt;             /* add the second-order displacements */
	const float* table_k;   /* power.init rows (read_power_spectrum, initialize.cpp:870-898): */
	const float* table_p;   /*   k in h / Mpc, log-uniform; P in (Mpc / h)^3 */
	int ntable;
} ct_ic_params;

typedef struct {
	double D1, D2;          /* first- and second-order growth factors at z0 */
	double prefac1, prefac2; /* velocity factors */
	double norm;            /* sigma8 normalisation applied to the table */
	float dxmax[3];         /* largest first-order displacement per axis, mean spacings */
	float dxmax2[3];        /* largest second-order displacement per axis */
} ct_ic_return;

/* Fills a single box of nfour^3 particles with the lattice displaced by the Zel'dovich (and
 * 2LPT) field of the table, seeded per k-space row as the reference seeds it (GSL taus).
 * Replaces initialize(z0) with options Nfour, parts_dim, twolpt, sigma8, use_power_file. */
ct_status ct_initialize(ct_ctx* ctx, int box_id, const ct_ic_params* params, ct_ic_return* result);

/* ---- matter power spectrum (power_spectrum_compute, src/power.cpp:33-45; fft3d_power_spectrum,
 * src/fft.cpp:172-214): cloud-kernel density on an nfour^3 grid (nfour even, 4 .. 1024) after folding the box `fold`
 * times, transform, window deconvolution, mean |delta_k|^2 in log-spaced shells from 1 to
 * nfour / 2 (grid units).  k[i]: shell centre in 1 / Mpc (times fold); P[i]: mean power; Perr[i]
 * (optional): the reference's error estimate.  *nbins receives the number of shells
 * (max(nfour / 8, 64)); with k and P null only the count is returned. */
ct_status ct_power_spectrum(ct_ctx* ctx, int box_id, int nfour, int fold, double box_size, int max_bins, float* k, float* P, float* Perr,
		int* nbins);

/* ---- hierarchical (multistep) step: kick_step_hierarchical (src/driver.cpp:382-593) */
typedef struct {
	int minrung;      /* the step's minimum rung */
	int minrung0;     /* the run's base minimum rung (top-level clip, driver.cpp:442-462) */
	int max_rung;     /* highest rung after the previous step (its top kick's max_rung) */
	double a;         /* scale factor for the kicks and drifts of this step */
	double tau;       /* time at the start of the step (0: first call of a run) */
	double t0;        /* top-level step: rung r advances by t0 / 2^r */
	double theta;
	double hsoft;     /* softening support h, box units */
	int bucket;       /* leaf capacity */
	float eta;
	float GM;
	float max_dt;
	int do_phi;
	int nocrop;       /* disable the top-level clip */
	double drag;
	float sign;
} ct_step_params;

typedef struct {
	ct_kick_return kr;         /* the top-level kick's return (max_rung = next step's max_rung) */
	int minrung;               /* minimum rung for the next step (raised by the clip) */
	int max_rung;
	double particles_kicked;   /* sum over the ladder of active particles */
	int kicks;                 /* ladder levels visited */
	int particles_drifted_levels;
} ct_step_return;

ct_status ct_step_hierarchical(ct_ctx* ctx, int box_id, const ct_step_params* params, ct_step_return* result);
/* The active-range state of the hierarchical rung ladder: the start of the active range
 * (particles_current_range) and the saved starts of the enclosing ranges, innermost last
 * (particles_push/pop_rungs, src/particles.cpp:218-235) -- what particles_save writes after
 * the particles (src/particles.cpp:1220-1223), so that a run resumes where it stopped.
 * get: pass stack = NULL to learn the depth; set: restores both (begin <= box size). */
ct_status ct_box_get_rung_state(ct_ctx* ctx, int box_id, int64_t* rung_begin, int64_t* stack, int* depth);
ct_status ct_box_set_rung_state(ct_ctx* ctx, int box_id, int64_t rung_begin, const int64_t* stack, int depth);
/* Particle counts per rung 0..15 (particles_rung_counts, src/particles.cpp:583). */
ct_status ct_rung_counts(ct_ctx* ctx, int box_id, uint64_t* counts);

/* Tree export (breadth-first order) for inspection and parity checks. */
ct_status ct_tree_download(ct_ctx* ctx, int box_id, ct_node* nodes, int64_t max_nodes, int64_t* count);

/* Counters of the last tree/kick/drift on a box. */
ct_status ct_get_counters(ct_ctx* ctx, int box_id, ct_counters* out);

/* Wait for all work of the context. */
ct_status ct_synchronize(ct_ctx* ctx);

/* FP64 direct Ewald summation (accuracy reference, not part of the step): force and
 * potential of all box particles (unit mass each) on nsink sink positions, softened nearest
 * image plus the periodic correction, alpha = 2.  Results in double, unscaled by GM. */
ct_status ct_direct_ewald(ct_ctx* ctx, int box_id, int64_t nsink, const uint32_t* sx, const uint32_t* sy, const uint32_t* sz, double h, double* gx,
		double* gy, double* gz, double* pot);

/* Measured FP32 FMA throughput of the context's device in TFLOP/s (2 flops per FMA): the
 * denominator of the FP32 roofline of the interaction kernels. */
ct_status ct_fp32_peak(ct_ctx* ctx, double* tflops);

/* The context's CUDA stream (cudaStream_t), for callers that order their own work with it. */
void* ct_stream(ct_ctx* ctx);

/* Summation of the per-sink particle-particle sums: 1 (default) adds the partial sums of the
 * staged source batches with Neumaier compensation, 0 adds them plainly in FP32 (for precision
 * studies; the reference adds plainly, gravity.cu:331-343). */
ct_status ct_ctx_set_compensated(ct_ctx* ctx, int compensated);

/* Scheduling priority of the context's CUDA streams, in CUDA's convention (0 the default and
 * lowest; negative values higher; clamped to the device's range).  The context is drained and
 * its streams are replaced, so a handle from ct_stream taken before the call is stale after it.
 * The reference has no counterpart (one process per GPU); the serving loop gives the lane that
 * holds the oldest request the higher priority, so that work started first finishes first. */
ct_status ct_ctx_set_priority(ct_ctx* ctx, int priority);

/* Launch shape of the particle-particle and leaf-kick kernels, the knobs of the autotuner
 * (cosmictiger_b200/autotune.py).  The reference fixes them at build time: its P2P stages at
 * most KICK_PP_MAX = 928 source particles per pass (cosmictiger/kick.hpp:48), its M2P at most
 * KICK_C_MAX = 32 multipoles (kick.hpp:27), one warp per work item (src/kick.cu:179).
 *   p2p_stage       source particles staged per pass (the cell-list size): 64, 128 or 256
 *   warps_per_tile  warps sharing one sink tile's sources: 1 or 2
 *   tile_width      sinks per tile, for P2P and the leaf kick: 32, or 16 (every tile then
 *                   spreads each sink's sources / multipoles over two or more lanes)
 * Results differ from one shape to another only in the order of the per-sink sums (within
 * float rounding); each shape is deterministic.  Default {128, 1, 32}; others: CT_ERR_ARG. */
typedef struct {
	int p2p_stage;
	int warps_per_tile;
	int tile_width;
} ct_tuning;
ct_status ct_ctx_set_tuning(ct_ctx* ctx, const ct_tuning* tuning);
ct_status ct_ctx_get_tuning(const ct_ctx* ctx, ct_tuning* tuning);

/* ---- allocation-free variant (no counterpart in the reference)
 *
 * For callers that cannot allocate device memory when they partition rungs: a host driver
 * living inside a memory pool it does not own, an embedding application whose allocator
 * forbids cudaMalloc/cudaFree on its hot path, or code that must keep its device footprint
 * fixed after start-up.  Same result as ct_sort_by_rung (particles with rung < min_rung move to
 * [begin, *rung_begin), the rest to [*rung_begin, n), with the reference's exact two-pointer
 * permutation), but on device arrays the caller already holds (SoA velocities), on the
 * caller's stream, with no context and no allocation: all temporary storage is one
 * file-scope __device__ array of fixed size that every GPU loading the library keeps until
 * process exit (about 17 MB).
 *   - at most CT_NOALLOC_MAX_PARTICLES particles in [begin, n); more returns CT_ERR_CAPACITY
 *     (and a message on stderr) before any device work;
 *   - the first call on each device looks up the array's device address; make that first call
 *     before any stream capture;
 *   - every call shares the one array: calls that overlap on the GPU (other streams, other
 *     host threads) race and must be serialised by the caller;
 *   - min_rung == 0 resets *rung_begin to 0 without touching the arrays, like the reference.
 * Returns after synchronising `stream` (a cudaStream_t; NULL is the legacy default stream). */
#define CT_NOALLOC_MAX_PARTICLES (1 << 20)
ct_status ct_sort_by_rung_noalloc(int64_t begin, int64_t n, int min_rung, uint32_t* x, uint32_t* y, uint32_t* z, float* vx, float* vy, float* vz,
		int8_t* rung, int64_t* rung_begin, void* stream);

#ifdef __cplusplus
}
#endif
#endif
