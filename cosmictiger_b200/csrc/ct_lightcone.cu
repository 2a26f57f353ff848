// Drift with the lightcone capture of the reference's cuda_drift_kernel (src/drift.cu:36-154).
//
// The rung's particles move as k_drift moves them (the FP64 update, wrap and fixed32 store),
// and each crossing of the light cone in the 8 periodic images next to the observer is
// recorded: the point where the particle's straight path meets the cone of the next period
// boundary (i0 + 1) tau_max, its velocity and its HEALPix nested pixel.  The crossing tests
// and the solve keep the reference's expression forms in FP64 (this unit is compiled with
// the default FMA contraction, as the reference's drift.cu is), so that the recorded entries
// are the reference's, bit for bit.
//
// Two passes ahead of the plain drift, so that the FP64 work runs on full warps: about one
// particle in twenty crosses per drift, which would put a crossing in nearly every warp of a
// fused kernel.  Pass 1 writes the (particle, image) pairs that a float pre-test cannot rule
// out; the host sizes the entry buffer for them (nothing has moved, so an overfull candidate
// list is simply redone after it grows); pass 2 runs the exact test and the pixel one pair per
// lane and writes the entries; then k_drift moves the particles.  No crossing is dropped and
// no worst-case buffer is held.
#include "ct_internal.cuh"

#include <algorithm>
#include <climits>

namespace ct {
namespace {

constexpr int LC_TPB = 256;

// Bits 0..12 of v to the even positions 0..24.
__device__ __forceinline__ uint32_t spread13(uint32_t v) {
	v &= 0x1fffu;
	v = (v | (v << 8)) & 0x00ff00ffu;
	v = (v | (v << 4)) & 0x0f0f0f0fu;
	v = (v | (v << 2)) & 0x33333333u;
	v = (v | (v << 1)) & 0x55555555u;
	return v;
}

// HEALPix nested pixel of a direction (Gorski et al. 2005, ApJ 622:759), evaluated as the
// reference does (vec2pix_nest, src/healpix.cu:55-171): face and in-face coordinates at the
// finest resolution 8192, nested index by bit interleaving (x on the even bits), degraded to
// nside by integer division so that boundary rounding is the same at every nside.
__device__ int healpix_nest(int nside, double x, double y, double z) {
	constexpr int NS = 8192;
	const double piover2 = 0.5 * M_PI, twopi = 2.0 * M_PI;
	const double zn = z / sqrt(x * x + y * y + z * z);
	double phi = 0.0;
	if (x != 0.0 || y != 0.0) {
		phi = atan2(y, x);
		if (phi < 0.0) {
			phi += twopi;
		}
	}
	const double za = fabs(zn);
	const double tt = phi / piover2;
	int face, ix, iy;
	if (za <= 2. / 3.) {
		const int jp = (int) floor(NS * (0.5 + tt - zn * 0.75));
		const int jm = (int) floor(NS * (0.5 + tt + zn * 0.75));
		const int ifp = jp / NS, ifm = jm / NS;
		face = ifp == ifm ? ifp % 4 + 4 : (ifp < ifm ? ifp % 4 : ifm % 4 + 8);
		ix = jm % NS;
		iy = NS - jp % NS - 1;
	} else {
		int ntt = (int) floor(tt);
		ntt = ntt >= 4 ? 3 : ntt;
		const double tp = tt - ntt;
		const double tmp = sqrt(3. * (1. - za));
		const int jp = min((int) floor(NS * tp * tmp), NS - 1);
		const int jm = min((int) floor(NS * (1. - tp) * tmp), NS - 1);
		if (zn >= 0) {
			face = ntt;
			ix = NS - jm - 1;
			iy = NS - jp - 1;
		} else {
			face = ntt + 8;
			ix = jp;
			iy = jm;
		}
	}
	const int ipf = (int) (spread13(ix) | (spread13(iy) << 1));
	const int f = NS / nside;
	return ipf / (f * f) + face * nside * nside;
}

struct LcArgs {
	int64_t b;               // range start
	int64_t total;           // particles in the range
	uint32_t* x[3];
	float* v[3];
	const int8_t* rung;
	int which;
	double c1;               // dt / a
	double drag_c0;          // 1 / (1 + drag dt)
	int do_drag;
	double ainv, t0, t1, c0, tmax;  // 1 / a, tau0, tau1, 1 / tau_max, tau_max
	int nside;
	ct_lc_entry* out;
	unsigned long long* ctr;  // [0] candidates, [1] entries
};

// Crossing of periodic image `img` (x, y, z offsets -1 or 0; x slowest, the reference's loop
// order) between the particle's positions p0 and p1 (src/drift.cu:76-120).  On a crossing
// inside the unit sphere around the observer returns true with the crossing point in q.
__device__ __forceinline__ bool lc_crossing(const LcArgs& a, const double p0[3], const double p1[3], const float vel[3], int img, double q[3]) {
	const double ox = (double) ((img >> 2) - 1), oy = (double) (((img >> 1) & 1) - 1), oz = (double) ((img & 1) - 1);
	const double x0 = p0[0] + ox, y0 = p0[1] + oy, z0 = p0[2] + oz;
	const double x1 = p1[0] + ox, y1 = p1[1] + oy, z1 = p1[2] + oz;
	const double dist0 = sqrt(x0 * x0 + y0 * y0 + z0 * z0);
	const double dist1 = sqrt(x1 * x1 + y1 * y1 + z1 * z1);
	const double cone0 = a.t0 + dist0;  // tau + distance at the drift's two ends
	const double cone1 = a.t1 + dist1;
	const int i0 = (int) (cone0 * a.c0);
	const int i1 = (int) (cone1 * a.c0);
	if (!(i0 != i1 && (dist1 <= 1.0 || dist0 <= 1.0))) {
		return false;
	}
	// |X0 + v t| = ti - (tau0 + t): the path meets the cone of period boundary ti
	const float vx = vel[0] * a.ainv;
	const float vy = vel[1] * a.ainv;
	const float vz = vel[2] * a.ainv;
	const double ti = double((double) (i0 + 1)) * double(a.tmax);
	const double dti = ti - a.t0;
	const double dti2 = dti * dti;
	const double lag = a.t0 - ti;
	const double A = 1.0 - (vx * vx + vy * vy + vz * vz);
	const double B = 2.0 * (lag - (vx * x0 + vy * y0 + vz * z0));
	const double C = dti2 - (x0 * x0 + y0 * y0 + z0 * z0);
	const double t = -(B + sqrt(B * B - 4.0 * A * C)) / (2.0 * A);
	q[0] = x0 + vx * t;
	q[1] = y0 + vy * t;
	q[2] = z0 + vz * t;
	return q[0] * q[0] + q[1] * q[1] + q[2] * q[2] <= 1.0;
}

// Cheap necessary condition for a crossing of image `img`: the exact test needs the period
// index of tau + distance to change between the two ends of the drift and one end within
// distance 1.  Both ends lie within [min(tau0, tau1) + d0 - s, max(tau0, tau1) + d0 + s] for
// the start distance d0 and the drift length s, so an image whose interval (widened by
// LC_MARGIN, far above the float rounding of d0 and s) holds no multiple of tau_max, or whose
// d0 - s exceeds 1, cannot cross; the exact FP64 test decides every other image.
constexpr float LC_MARGIN = 1e-4f;

__device__ __forceinline__ bool lc_candidate(const LcArgs& a, const double p0[3], float s, int img) {
	const float x = (float) (p0[0] + (double) ((img >> 2) - 1));
	const float y = (float) (p0[1] + (double) (((img >> 1) & 1) - 1));
	const float z = (float) (p0[2] + (double) ((img & 1) - 1));
	const float d0 = sqrtf(x * x + y * y + z * z);
	const float w = s + LC_MARGIN;
	if (d0 - w > 1.0f) {
		return false;
	}
	const double lo = (fmin(a.t0, a.t1) + (double) (d0 - w)) * a.c0;
	const double hi = (fmax(a.t0, a.t1) + (double) (d0 + w)) * a.c0;
	// (the exact test truncates toward zero: below zero, leave the decision to it)
	return lo < 0.0 || floor(lo) != floor(hi);
}

// The drift's start and end points and the velocity after drag of particle i, as cuda_drift
// computes them (src/drift.cu:58-75): end = start + v dt / a in FP64, drag applied to v after.
__device__ __forceinline__ void lc_particle(const LcArgs& a, int64_t i, double p0[3], double p1[3], float vel[3]) {
#pragma unroll
	for (int d = 0; d < 3; d++) {
		p0[d] = fixed_to_double(a.x[d][i]);
		vel[d] = a.v[d][i];
		p1[d] = __dadd_rn(p0[d], __dmul_rn((double) vel[d], a.c1));
	}
	if (a.do_drag) {
#pragma unroll
		for (int d = 0; d < 3; d++) {
			vel[d] = (float) ((double) vel[d] * a.drag_c0);
		}
	}
}

// Pass 1: the (particle, image) pairs that pass the pre-test, as index * 8 + image.  A warp
// reserves its pairs with one atomic; pairs past the buffer are counted, not written (the host
// then grows the buffer and runs the pass again: nothing has moved yet).
__global__ void __launch_bounds__(LC_TPB) k_lc_candidates(LcArgs a, uint64_t* __restrict__ cand, unsigned long long cap) {
	const int lane = threadIdx.x & 31;
	const int64_t stride = (int64_t) gridDim.x * blockDim.x;
	// warp-uniform trip count: the reservation is a warp collective
	for (int64_t w0 = blockIdx.x * (int64_t) blockDim.x + (threadIdx.x - lane); w0 < a.total; w0 += stride) {
		const int64_t i = a.b + w0 + lane;
		unsigned mask = 0;
		if (w0 + lane < a.total && a.rung[i] == a.which) {
			double p0[3], p1[3];
			float vel[3];
			lc_particle(a, i, p0, p1, vel);
			// drift length, rounded up (relative 1e-6) past its float rounding
			const float sx = (float) (p1[0] - p0[0]), sy = (float) (p1[1] - p0[1]), sz = (float) (p1[2] - p0[2]);
			const float s = sqrtf(sx * sx + sy * sy + sz * sz) * 1.000001f;
			for (int img = 0; img < 8; img++) {
				if (lc_candidate(a, p0, s, img)) {
					mask |= 1u << img;
				}
			}
		}
		const int cnt = __popc(mask);
		int incl = cnt;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int y = __shfl_up_sync(0xffffffffu, incl, o);
			incl += lane >= o ? y : 0;
		}
		const int wtot = __shfl_sync(0xffffffffu, incl, 31);
		if (wtot == 0) {
			continue;
		}
		unsigned long long base = 0;
		if (lane == 0) {
			base = atomicAdd(a.ctr, (unsigned long long) wtot);
		}
		base = __shfl_sync(0xffffffffu, base, 0);
		unsigned long long k = base + (unsigned long long) (incl - cnt);
		for (int img = 0; img < 8; img++) {
			if (mask >> img & 1u) {
				if (k < cap) {
					cand[k] = ((uint64_t) i << 3) | (uint64_t) img;
				}
				k++;
			}
		}
	}
}

// Pass 2: the exact test of every candidate, one per lane; a crossing writes its entry.  The
// buffer holds at least the candidates' count past the entries already there.
__global__ void __launch_bounds__(LC_TPB) k_lc_entries(LcArgs a, const uint64_t* __restrict__ cand, int64_t ncand) {
	const int lane = threadIdx.x & 31;
	const int64_t stride = (int64_t) gridDim.x * blockDim.x;
	for (int64_t w0 = blockIdx.x * (int64_t) blockDim.x + (threadIdx.x - lane); w0 < ncand; w0 += stride) {
		bool hit = false;
		double q[3];
		float vel[3];
		if (w0 + lane < ncand) {
			const uint64_t r = cand[w0 + lane];
			double p0[3], p1[3];
			lc_particle(a, (int64_t) (r >> 3), p0, p1, vel);
			hit = lc_crossing(a, p0, p1, vel, (int) (r & 7), q);
		}
		const unsigned m = __ballot_sync(0xffffffffu, hit);
		if (m == 0) {
			continue;
		}
		unsigned long long base = 0;
		if (lane == 0) {
			base = atomicAdd(a.ctr + 1, (unsigned long long) __popc(m));
		}
		base = __shfl_sync(0xffffffffu, base, 0);
		if (hit) {
			ct_lc_entry e;
			// fixed<int,31> = double (fixed.hpp:97-101): truncation of 2^31 q
			e.x = __double2int_rz(2147483648.0 * q[0]);
			e.y = __double2int_rz(2147483648.0 * q[1]);
			e.z = __double2int_rz(2147483648.0 * q[2]);
			e.vx = vel[0];
			e.vy = vel[1];
			e.vz = vel[2];
			e.pix = healpix_nest(a.nside, q[0], q[1], q[2]);
			a.out[base + __popc(m & ((1u << lane) - 1u))] = e;
		}
	}
}

__global__ void k_lc_counters(unsigned long long* ctr, unsigned long long entries) {
	ctr[0] = 0;
	ctr[1] = entries;
}

// Entry buffer of at least `cap` entries holding the first `keep` entries of the old one.
ct_status lc_resize(Ctx* c, Box* b, int64_t cap, int64_t keep) {
	cap = std::max<int64_t>(cap, 1);
	ct_lc_entry* p = nullptr;
	CT_TRY(dalloc(c, (void**) &p, sizeof(ct_lc_entry) * cap, "lightcone entries"));
	if (keep > 0) {
		const cudaError_t e = cudaMemcpyAsync(p, b->lc, sizeof(ct_lc_entry) * keep, cudaMemcpyDeviceToDevice, c->stream);
		if (e != cudaSuccess) {
			dfree(c, p, sizeof(ct_lc_entry) * cap);
			return cuda_check(c, e, "lightcone entry copy");
		}
		CT_CUDA(c, cudaStreamSynchronize(c->stream));
	}
	dfree(c, b->lc, sizeof(ct_lc_entry) * b->lc_cap);
	b->lc = p;
	b->lc_cap = cap;
	return CT_OK;
}

int lc_grid(const Ctx* c, int64_t n) {
	return (int) std::max<int64_t>(1, std::min<int64_t>((n + LC_TPB - 1) / LC_TPB, (int64_t) c->nsm * 8));
}

Box* lc_box(Ctx* c, int id) {
	if (!c || id < 0 || id >= (int) c->boxes.size()) {
		return nullptr;
	}
	return c->boxes[id];
}

}  // namespace

void lightcone_release(Ctx* c, Box* b) {
	dfree(c, b->lc, sizeof(ct_lc_entry) * b->lc_cap);
	dfree(c, b->lc_cand, sizeof(uint64_t) * b->lc_cand_cap);
	dfree(c, b->d_lc_ctr, 4 * sizeof(unsigned long long));
	b->lc = nullptr;
	b->lc_cand = nullptr;
	b->d_lc_ctr = nullptr;
	b->lc_cap = b->lc_count = b->lc_last = b->lc_cand_cap = 0;
}

}  // namespace ct

using namespace ct;

extern "C" ct_status ct_drift_lightcone(ct_ctx* ctx, int box_id, int rung, float a, float dt, double drag, const ct_lc_params* lc, int64_t* captured) {
	Ctx* c = (Ctx*) ctx;
	Box* b = lc_box(c, box_id);
	if (!b || !lc || !(a > 0.f) || rung < 0 || rung > 127) {
		return fail(c, CT_ERR_ARG, "ct_drift_lightcone: bad arguments");
	}
	if (lc->nside < 1 || lc->nside > 8192) {
		return fail(c, CT_ERR_ARG, "ct_drift_lightcone: nside must be in [1, 8192]");
	}
	if (b->nsub != 1) {
		return fail(c, CT_ERR_ARG, "ct_drift_lightcone: the lightcone is captured for single boxes, not ensembles");
	}
	if (b->n >= ((int64_t) 1 << 32)) {
		return fail(c, CT_ERR_ARG, "ct_drift_lightcone: too many particles for 32-bit indices");
	}
	if (captured) {
		*captured = 0;
	}
	cudaSetDevice(c->device);
	// the kernel's arguments as cuda_drift passes them (float host values widened to double)
	const double da = a, ddt = dt, t0 = lc->tau0, t1 = lc->tau1, tmax = lc->tau_max;
	if (!(tmax - t1 < 1.0)) {
		// no capture in this drift (src/drift.cu:38)
		return drift_run(c, b, rung, a, dt, drag);
	}
	const int64_t np = b->n - b->rung_begin;
	if (np <= 0) {
		return drift_run(c, b, rung, a, dt, drag);
	}
	if (!b->d_lc_ctr) {
		CT_TRY(dalloc(c, (void**) &b->d_lc_ctr, 4 * sizeof(unsigned long long), "lightcone counters"));
	}
	// candidate room: twice the last drift's crossings, at least 1/64 of the particles
	const int64_t room = std::max<int64_t>(std::max<int64_t>(1 << 16, np / 64), 2 * b->lc_last);
	if (b->lc_cand_cap < room) {
		dfree(c, b->lc_cand, sizeof(uint64_t) * b->lc_cand_cap);
		b->lc_cand = nullptr;
		b->lc_cand_cap = 0;
		CT_TRY(dalloc(c, (void**) &b->lc_cand, sizeof(uint64_t) * room, "lightcone candidates"));
		b->lc_cand_cap = room;
	}
	LcArgs la;
	la.b = b->rung_begin;
	la.total = np;
	for (int d = 0; d < 3; d++) {
		la.x[d] = b->x[d];
		la.v[d] = b->v[d];
	}
	la.rung = b->rung;
	la.which = rung;
	la.c1 = ddt / da;
	la.do_drag = drag != 0.0;
	la.drag_c0 = la.do_drag ? 1.0 / (1.0 + drag * ddt) : 1.0;
	la.ainv = 1.0 / da;
	la.t0 = t0;
	la.t1 = t1;
	la.c0 = 1.0 / tmax;
	la.tmax = tmax;
	la.nside = lc->nside;
	la.ctr = b->d_lc_ctr;
	const int64_t before = b->lc_count;
	cudaStream_t st = c->stream;
	cudaEventRecord(c->ev[6], st);
	unsigned long long h[2] = { 0, 0 };
	for (int pass = 0;; pass++) {
		c->launches += 2;
		k_lc_counters<<<1, 1, 0, st>>>(b->d_lc_ctr, (unsigned long long) before);
		k_lc_candidates<<<lc_grid(c, np), LC_TPB, 0, st>>>(la, b->lc_cand, (unsigned long long) b->lc_cand_cap);
		CT_CUDA(c, cudaGetLastError());
		CT_CUDA(c, cudaMemcpyAsync(h, b->d_lc_ctr, sizeof(h), cudaMemcpyDeviceToHost, st));
		CT_CUDA(c, cudaStreamSynchronize(st));
		if ((int64_t) h[0] <= b->lc_cand_cap) {
			break;
		}
		if (pass >= 1) {
			// the count of a pass that fits is the count of the one before
			return fail(c, CT_ERR_CUDA, "ct_drift_lightcone: candidate count changed between passes");
		}
		const int64_t need = (int64_t) h[0] + (int64_t) h[0] / 4;
		dfree(c, b->lc_cand, sizeof(uint64_t) * b->lc_cand_cap);
		b->lc_cand = nullptr;
		b->lc_cand_cap = 0;
		CT_TRY(dalloc(c, (void**) &b->lc_cand, sizeof(uint64_t) * need, "lightcone candidates"));
		b->lc_cand_cap = need;
	}
	const int64_t ncand = (int64_t) h[0];
	if (b->lc_cap - b->lc_count < ncand) {
		CT_TRY(lc_resize(c, b, std::max<int64_t>(b->lc_count + ncand, 2 * b->lc_cap), b->lc_count));
	}
	la.out = b->lc;
	if (ncand > 0) {
		c->launches++;
		k_lc_entries<<<lc_grid(c, ncand), LC_TPB, 0, st>>>(la, b->lc_cand, ncand);
	}
	CT_TRY(drift_run(c, b, rung, a, dt, drag, false));
	CT_CUDA(c, cudaMemcpyAsync(h, b->d_lc_ctr, sizeof(h), cudaMemcpyDeviceToHost, st));
	cudaEventRecord(c->ev[7], st);
	CT_CUDA(c, cudaStreamSynchronize(st));
	c->drift_timed = true;
	b->lc_count = (int64_t) h[1];
	b->lc_last = b->lc_count - before;
	b->tree_valid = false;
	if (captured) {
		*captured = b->lc_count - before;
	}
	return CT_OK;
}

extern "C" ct_status ct_lightcone_count(ct_ctx* ctx, int box_id, int64_t* count) {
	Ctx* c = (Ctx*) ctx;
	Box* b = lc_box(c, box_id);
	if (!b || !count) {
		return fail(c, CT_ERR_ARG, "ct_lightcone_count: bad arguments");
	}
	*count = b->lc_count;
	return CT_OK;
}

extern "C" ct_status ct_lightcone_download(ct_ctx* ctx, int box_id, ct_lc_entry* out, int64_t max_entries, int64_t* count, int clear) {
	Ctx* c = (Ctx*) ctx;
	Box* b = lc_box(c, box_id);
	if (!b || max_entries < 0 || (max_entries > 0 && !out)) {
		return fail(c, CT_ERR_ARG, "ct_lightcone_download: bad arguments");
	}
	cudaSetDevice(c->device);
	if (count) {
		*count = b->lc_count;
	}
	const int64_t m = std::min(max_entries, b->lc_count);
	if (m > 0) {
		CT_CUDA(c, cudaMemcpyAsync(out, b->lc, sizeof(ct_lc_entry) * m, cudaMemcpyDeviceToHost, c->stream));
	}
	CT_CUDA(c, cudaStreamSynchronize(c->stream));
	if (clear) {
		b->lc_count = 0;
	}
	return CT_OK;
}

extern "C" ct_status ct_lightcone_reserve(ct_ctx* ctx, int box_id, int64_t entries) {
	Ctx* c = (Ctx*) ctx;
	Box* b = lc_box(c, box_id);
	if (!b || entries < 0) {
		return fail(c, CT_ERR_ARG, "ct_lightcone_reserve: bad arguments");
	}
	cudaSetDevice(c->device);
	const int64_t cap = std::max(entries, b->lc_count);
	if (cap == b->lc_cap) {
		return CT_OK;
	}
	CT_CUDA(c, cudaStreamSynchronize(c->stream));
	return lc_resize(c, b, cap, b->lc_count);
}
