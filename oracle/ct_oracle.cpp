// CPU oracle for the gravity step (test infrastructure only; see ct_oracle.h).
//
// Compiled with -ffp-contract=off: every float/double expression below is evaluated as
// written, which is how the reference's C++ reads (the tree geometry of src/tree.cpp and the
// opening tests of src/kick.cu).  The FMM operators come from the generated headers, whose
// outputs are pinned against the reference's own operators by tests/golden.
#include "ct_oracle.h"
#include "fmm_p7.h"
#include "fmm_p5.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// Dynamic parallel loop over [0, n) on nthreads host threads (<= 0: all cores).
template<class F>
void parallel_for(int n, int nthreads, F&& f) {
	if (nthreads <= 0) {
		nthreads = std::max(1u, std::thread::hardware_concurrency());
	}
	nthreads = std::min(nthreads, std::max(n, 1));
	std::atomic<int> next(0);
	auto body = [&]() {
		for (int i = next++; i < n; i = next++) {
			f(i);
		}
	};
	std::vector<std::thread> th;
	for (int t = 1; t < nthreads; t++) {
		th.emplace_back(body);
	}
	body();
	for (auto& t : th) {
		t.join();
	}
}

constexpr float FIXED2FLOAT = 1.0f / 4294967296.0f; // fixed.hpp:39
constexpr double FIXED2DOUBLE = 1.0 / 4294967296.0;

// fixed32 from double: truncation of 2^32 x, wrapping modulo 2^32 like the x86-64
// double -> 64-bit integer -> low 32 bits conversion (fixed.hpp:97-101).
inline uint32_t fixed32_from_double(double x) {
	return (uint32_t) (int64_t) (x * 4294967296.0);
}
// fixed<int,29> from double (range.hpp:358; fixed.hpp:97-101).
inline int32_t range_fixed_from_double(double x) {
	return (int32_t) (x * 536870912.0);
}
inline double fixed32_to_double(uint32_t i) {
	return double(i) * FIXED2DOUBLE;
}
// Periodic separation a - b, nearest image (fixed.hpp:303-305).
inline float fdist(uint32_t a, uint32_t b) {
	return float(int32_t(a - b)) * FIXED2FLOAT;
}
// distance(fixed32 b, range_fixed a) = -distance(a, b) (range.hpp:447-458).
inline float fdist_rf(uint32_t b, int32_t a) {
	float f = double(a) / 536870912.0 - fixed32_to_double(b);
	f -= double(f > 0.5);
	f += double(f < -0.5);
	return -f;
}
inline float sqrf(float a, float b, float c) {
	return a * a + b * b + c * c;
}

// Ferrer-type softening kernel of order 4 (gravity.hpp:73-96).
template<class T>
inline void gsoft(T& f, T& phi, T q2, T hinv, T h2inv, T h3inv) {
	const T Af[5] = { T(1155. / 128.), T(-693. / 32.), T(1485. / 64.), T(-385. / 32.), T(315. / 128.) };
	const T Aphi[6] = { T(693. / 256.), T(-1155. / 256.), T(693. / 128.), T(-495. / 128.), T(385. / 256.), T(-63. / 256.) };
	q2 *= h2inv;
	f = Af[4];
	for (int n = 3; n >= 0; n--) {
		f = std::fma(f, q2, Af[n]);
	}
	f *= h3inv;
	phi = Aphi[5];
	for (int n = 4; n >= 0; n--) {
		phi = std::fma(phi, q2, Aphi[n]);
	}
	phi *= hinv;
}
inline float self_phi() {
	return float(693. / 256.);
}

// ---------------------------------------------------------------- operator dispatch
struct Ops7 {
	static constexpr int NEXP = ct_p7::NEXP, NMULT = ct_p7::NMULT;
	template<class T> static void greens(T* D, T x, T y, T z) {
		ct_p7::greens(D, x, y, z);
	}
	template<class T> static void greens_add(T* L, T x, T y, T z) {
		ct_p7::greens_add(L, x, y, z);
	}
	static int ewald(float* D, float x, float y, float z) {
		return ct_p7::ewald_greens(D, x, y, z, tab());
	}
	template<class T> static void m2l(T* L, const T* M, const T* D, bool phi) {
		ct_p7::m2l(L, M, D, phi);
	}
	template<class T> static void m2l2(T* L, const T* M, const T* D, bool phi) {
		ct_p7::m2l_2(L, M, D, phi);
	}
	template<class T> static void p2m(T* M, T x, T y, T z) {
		ct_p7::p2m(M, x, y, z);
	}
	template<class T> static void m2m(T* M, const T* Ma, T x, T y, T z) {
		ct_p7::m2m(M, Ma, x, y, z);
	}
	template<class T> static void l2l(T* Lb, const T* La, T x, T y, T z, bool phi) {
		ct_p7::l2l(Lb, La, x, y, z, phi);
	}
	template<class T> static void l2p(T* Lb, const T* La, T x, T y, T z, bool phi) {
		ct_p7::l2p(Lb, La, x, y, z, phi);
	}
	static const ct_p7::EwaldTab& tab() {
		// function-local static: initialised once, thread-safe
		static const ct_p7::EwaldTab* t = [] {
			auto* p = new ct_p7::EwaldTab;
			ct_p7::ewald_build_host(*p);
			return p;
		}();
		return *t;
	}
};
struct Ops5 {
	static constexpr int NEXP = ct_p5::NEXP, NMULT = ct_p5::NMULT;
	template<class T> static void greens(T* D, T x, T y, T z) {
		ct_p5::greens(D, x, y, z);
	}
	template<class T> static void greens_add(T* L, T x, T y, T z) {
		ct_p5::greens_add(L, x, y, z);
	}
	static int ewald(float* D, float x, float y, float z) {
		return ct_p5::ewald_greens(D, x, y, z, tab());
	}
	template<class T> static void m2l(T* L, const T* M, const T* D, bool phi) {
		ct_p5::m2l(L, M, D, phi);
	}
	template<class T> static void m2l2(T* L, const T* M, const T* D, bool phi) {
		ct_p5::m2l_2(L, M, D, phi);
	}
	template<class T> static void p2m(T* M, T x, T y, T z) {
		ct_p5::p2m(M, x, y, z);
	}
	template<class T> static void m2m(T* M, const T* Ma, T x, T y, T z) {
		ct_p5::m2m(M, Ma, x, y, z);
	}
	template<class T> static void l2l(T* Lb, const T* La, T x, T y, T z, bool phi) {
		ct_p5::l2l(Lb, La, x, y, z, phi);
	}
	template<class T> static void l2p(T* Lb, const T* La, T x, T y, T z, bool phi) {
		ct_p5::l2p(Lb, La, x, y, z, phi);
	}
	static const ct_p5::EwaldTab& tab() {
		// function-local static: initialised once, thread-safe
		static const ct_p5::EwaldTab* t = [] {
			auto* p = new ct_p5::EwaldTab;
			ct_p5::ewald_build_host(*p);
			return p;
		}();
		return *t;
	}
};

// ---------------------------------------------------------------- tree build
struct BuildRet {
	double multi[37]; // kept in double until stored (tree.cpp stores float)
	float multi_f[37];
	uint32_t pos[3];
	int id;
	float radius;
	double box_b[3], box_e[3];
};

struct Builder {
	uint32_t* x[3];
	float* v;
	int8_t* r;
	double theta, h;
	int bucket;
	// nodes in depth-first order (parent, left subtree, right subtree); a subtree built on
	// another thread is spliced in after the left one, so the order does not depend on threads
	std::vector<ct_or_node> nodes;
	int fork_depth;  // right children above this depth are built on their own thread
	bool too_deep;  // a node at depth MAX_DEPTH - 1 still had to split (tree.cpp:285-286)
};

// Two-pointer partition of [b, e) at xmid along xdim (particles.cpp:979-1018).
int partition(Builder& B, int b, int e, double xm, int xdim) {
	int lo = b, hi = e;
	const uint32_t xmid = fixed32_from_double(xm);
	uint32_t* xd = B.x[xdim];
	while (lo < hi) {
		if (xd[lo] >= xmid) {
			while (lo != hi) {
				hi--;
				if (xd[hi] < xmid) {
					for (int d = 0; d < 3; d++) {
						std::swap(B.x[d][hi], B.x[d][lo]);
					}
					for (int d = 0; d < 3; d++) {
						std::swap(B.v[3 * hi + d], B.v[3 * lo + d]);
					}
					std::swap(B.r[hi], B.r[lo]);
					break;
				}
			}
		}
		lo++;
	}
	return hi;
}

template<class Ops>
BuildRet tree_create(Builder& B, uint64_t key, int pb, int pe, const double* box_b, const double* box_e, int depth) {
	BuildRet rc;
	const int index = (int) B.nodes.size();
	B.nodes.emplace_back();
	const int nparts = pe - pb;
	float box_r = 0.0f;
	for (int dim = 0; dim < 3; dim++) {
		const double s = 0.5 * (box_e[dim] - box_b[dim]);
		box_r = float(double(box_r) + s * s);
	}
	box_r = std::sqrt(box_r);
	const bool ewald_satisfied = (box_r < 0.25 * (B.theta / (1.0 + B.theta)) && box_r < 0.125 - 0.25 * B.h);
	int children[2] = { -1, -1 };
	double Xc[3];
	float radius;
	bool isleaf = true;
	const bool must_split = nparts > B.bucket || (!ewald_satisfied && nparts > 0);
	if (must_split && depth >= 127) {
		B.too_deep = true;
	}
	if (!B.too_deep && must_split) {
		isleaf = false;
		int xdim = 0;
		double max_span = -1.0;
		for (int dim = 0; dim < 3; dim++) {
			const double span = box_e[dim] - box_b[dim];
			if (span > max_span) {
				max_span = span;
				xdim = dim;
			}
		}
		const double xmid = 0.5 * (box_e[xdim] + box_b[xdim]);
		const int mid = partition(B, pb, pe, xmid, xdim);
		double lb[3], le[3], rb[3], re[3];
		for (int d = 0; d < 3; d++) {
			lb[d] = rb[d] = box_b[d];
			le[d] = re[d] = box_e[d];
		}
		le[xdim] = rb[xdim] = xmid;
		BuildRet rcl, rcr;
		if (depth < B.fork_depth && nparts > 65536) {
			// the reference forks the right child (tree.cpp:349-350); here the fork builds into a
			// builder of its own, whose nodes follow the left subtree's
			Builder R;
			for (int d = 0; d < 3; d++) {
				R.x[d] = B.x[d];
			}
			R.v = B.v;
			R.r = B.r;
			R.theta = B.theta;
			R.h = B.h;
			R.bucket = B.bucket;
			R.fork_depth = B.fork_depth;
			R.too_deep = false;
			std::thread t([&]() {
				rcr = tree_create<Ops>(R, (key << 1) + 1, mid, pe, rb, re, depth + 1);
			});
			rcl = tree_create<Ops>(B, key << 1, pb, mid, lb, le, depth + 1);
			t.join();
			const int off = (int) B.nodes.size();
			for (ct_or_node n : R.nodes) {
				if (n.child_left >= 0) {
					n.child_left += off;
				}
				if (n.child_right >= 0) {
					n.child_right += off;
				}
				B.nodes.push_back(n);
			}
			rcr.id += off;
			B.too_deep = B.too_deep || R.too_deep;
		} else {
			rcl = tree_create<Ops>(B, key << 1, pb, mid, lb, le, depth + 1);
			rcr = tree_create<Ops>(B, (key << 1) + 1, mid, pe, rb, re, depth + 1);
		}
		const float ml0 = rcl.multi_f[0], mr0 = rcr.multi_f[0];
		for (int dim = 0; dim < 3; dim++) {
			if (ml0 != 0.0f && mr0 != 0.0f) {
				rc.box_b[dim] = std::min(rcl.box_b[dim], rcr.box_b[dim]);
				rc.box_e[dim] = std::max(rcl.box_e[dim], rcr.box_e[dim]);
			} else if (ml0 != 0.0f) {
				rc.box_b[dim] = rcl.box_b[dim];
				rc.box_e[dim] = rcl.box_e[dim];
			} else {
				rc.box_b[dim] = rcr.box_b[dim];
				rc.box_e[dim] = rcr.box_e[dim];
			}
		}
		double Xl[3], Xr[3];
		for (int dim = 0; dim < 3; dim++) {
			Xl[dim] = fixed32_to_double(rcl.pos[dim]);
			Xr[dim] = fixed32_to_double(rcr.pos[dim]);
		}
		double Xc1[3], Xc2[3];
		double radius1 = 0.0, radius2;
		bool tried1 = false;
		if (nparts <= 64 * B.bucket && (rc.box_e[xdim] - rc.box_b[xdim] <= 0.5)) {
			tried1 = true;
			uint32_t xc[3];
			for (int dim = 0; dim < 3; dim++) {
				Xc1[dim] = 0.5 * (rc.box_b[dim] + rc.box_e[dim]);
				xc[dim] = fixed32_from_double(Xc1[dim]);
			}
			float r2max = 0.0f;
			for (int i = pb; i < pe; i++) {
				float dx[3];
				for (int dim = 0; dim < 3; dim++) {
					dx[dim] = float(int32_t(B.x[dim][i] - xc[dim])) * FIXED2FLOAT;
				}
				const float r2 = sqrf(dx[0], dx[1], dx[2]);
				r2max = std::max(r2max, r2);
			}
			radius1 = std::sqrt(r2max); // float sqrt (the reference resolves sqrt(float) to the float overload)
		}
		double N[3];
		double norminv = 0.0;
		for (int dim = 0; dim < 3; dim++) {
			N[dim] = Xl[dim] - Xr[dim];
			norminv += N[dim] * N[dim];
		}
		norminv = 1.0 / std::sqrt(norminv);
		for (int dim = 0; dim < 3; dim++) {
			N[dim] *= norminv;
			N[dim] = std::abs(N[dim]);
		}
		double r = 0.0;
		const double Rl = rcl.radius, Rr = rcr.radius;
		if (mr0 != 0.0f) {
			if (ml0 != 0.0f) {
				for (int dim = 0; dim < 3; dim++) {
					const double xmax = std::max(Xl[dim] + N[dim] * Rl, Xr[dim] + N[dim] * Rr);
					const double xmin = std::min(Xl[dim] - N[dim] * Rl, Xr[dim] - N[dim] * Rr);
					Xc2[dim] = (xmax + xmin) * 0.5;
					const double t = (xmax - xmin) * 0.5;
					r += t * t;
				}
			} else {
				for (int dim = 0; dim < 3; dim++) {
					Xc2[dim] = Xr[dim];
				}
				r = Rr * Rr;
			}
		} else {
			for (int dim = 0; dim < 3; dim++) {
				Xc2[dim] = Xl[dim];
			}
			r = Rl * Rl;
		}
		radius2 = std::sqrt(r);
		if (tried1 && radius1 < radius2) {
			for (int d = 0; d < 3; d++) {
				Xc[d] = Xc1[d];
			}
			radius = float(radius1);
		} else {
			for (int d = 0; d < 3; d++) {
				Xc[d] = Xc2[d];
			}
			radius = float(radius2);
		}
		r = 0.0;
		for (int dim = 0; dim < 3; dim++) {
			const double span = rc.box_e[dim] - rc.box_b[dim];
			r += (span * 0.5) * (span * 0.5);
		}
		r = std::sqrt(r);
		if (r < radius) {
			radius = float(r);
			for (int dim = 0; dim < 3; dim++) {
				Xc[dim] = (rc.box_b[dim] + rc.box_e[dim]) * 0.5;
			}
		}
		for (int dim = 0; dim < 3; dim++) {
			rc.pos[dim] = fixed32_from_double(Xc[dim]);
		}
		// M2M of both children to the new centre in double (tree.cpp:481-494)
		double Ml[37], Mr[37];
		Ops::m2m(Ml, rcl.multi, Xl[0] - Xc[0], Xl[1] - Xc[1], Xl[2] - Xc[2]);
		Ops::m2m(Mr, rcr.multi, Xr[0] - Xc[0], Xr[1] - Xc[1], Xr[2] - Xc[2]);
		for (int i = 0; i < Ops::NMULT; i++) {
			const float m = float(Ml[i] + Mr[i]);
			rc.multi_f[i] = m;
			rc.multi[i] = m;
		}
		children[0] = rcl.id;
		children[1] = rcr.id;
	} else {
		for (int dim = 0; dim < 3; dim++) {
			rc.box_b[dim] = box_e[dim];
			rc.box_e[dim] = box_b[dim];
		}
		for (int i = pb; i < pe; i++) {
			for (int dim = 0; dim < 3; dim++) {
				const double xx = fixed32_to_double(B.x[dim][i]);
				rc.box_e[dim] = std::max(rc.box_e[dim], xx);
				rc.box_b[dim] = std::min(rc.box_b[dim], xx);
			}
		}
		for (int dim = 0; dim < 3; dim++) {
			Xc[dim] = (rc.box_e[dim] + rc.box_b[dim]) * 0.5;
		}
		double r = 0.0;
		for (int i = pb; i < pe; i++) {
			double this_radius = 0.0;
			for (int dim = 0; dim < 3; dim++) {
				const double xx = fixed32_to_double(B.x[dim][i]);
				this_radius += (xx - Xc[dim]) * (xx - Xc[dim]);
			}
			r = std::max(r, this_radius);
		}
		radius = float(std::sqrt(r));
		double M[37];
		for (int i = 0; i < Ops::NMULT; i++) {
			M[i] = 0.0;
		}
		uint32_t Y[3];
		for (int dim = 0; dim < 3; dim++) {
			Y[dim] = fixed32_from_double(Xc[dim]);
		}
		for (int i = pb; i < pe; i++) {
			float dx[3];
			for (int dim = 0; dim < 3; dim++) {
				dx[dim] = float(int32_t(B.x[dim][i] - Y[dim])) * FIXED2FLOAT;
			}
			float m[37];
			Ops::p2m(m, dx[0], dx[1], dx[2]);
			for (int j = 0; j < Ops::NMULT; j++) {
				M[j] += double(m[j]);
			}
		}
		for (int i = 0; i < Ops::NMULT; i++) {
			rc.multi_f[i] = float(M[i]);
			rc.multi[i] = rc.multi_f[i];
		}
		for (int dim = 0; dim < 3; dim++) {
			rc.pos[dim] = fixed32_from_double(Xc[dim]);
		}
	}
	rc.radius = radius;
	rc.id = index;
	{
		ct_or_node& n = B.nodes[index];
		memset(&n, 0, sizeof(n));
		n.key = key;
		n.part_begin = pb;
		n.part_end = pe;
		n.child_left = children[0];
		n.child_right = children[1];
		for (int d = 0; d < 3; d++) {
			n.pos[d] = rc.pos[d];
			n.box_begin[d] = range_fixed_from_double(rc.box_b[d]);
			n.box_end[d] = range_fixed_from_double(rc.box_e[d]);
		}
		n.radius = radius;
		n.leaf = isleaf;
		n.depth = depth;
		for (int i = 0; i < Ops::NMULT; i++) {
			n.multi[i] = rc.multi_f[i];
		}
	}
	return rc;
}

// ---------------------------------------------------------------- kick
struct Force {
	float gx, gy, gz, phi;
};

struct KickCtx {
	const ct_or_kick_params* p;
	const ct_or_node* nodes;
	const uint32_t* x[3];
	float* v;
	int8_t* rung;
	float *gx, *gy, *gz, *pot;
};

struct KickAcc {
	int max_rung = 0;
	double pot = 0, kin = 0, dkin = 0, xmom = 0, ymom = 0, zmom = 0, nmom = 0;
	double flops = 0;
};

// box_intersects_sphere (range.hpp:459-466)
bool box_intersects_sphere(const ct_or_node& box, const uint32_t* x, float r) {
	float d2 = 0.0f;
	for (int dim = 0; dim < 3; dim++) {
		const float a = fdist_rf(x[dim], box.box_begin[dim]);
		const float b = fdist_rf(x[dim], box.box_end[dim]);
		const float d2begin = a * a;
		const float d2end = b * b;
		const int64_t xr = int64_t(x[dim] >> 3); // range_fixed(fixed32): raw >> (32-29)
		const int outside = (xr < box.box_begin[dim]) + (xr > box.box_end[dim]);
		d2 += float(outside) * std::min(d2begin, d2end);
	}
	return d2 < r * r;
}

// Flop convention of the reference (per-interaction counts returned by its operators and
// the hand counts in src/gravity.cu and src/kick.cu); used only for roofline reporting.
constexpr double FLOP_GREENS = 265, FLOP_M2L = 1583, FLOP_M2L_PHI = 119, FLOP_L2L_CUDA = 2650, FLOP_L2L_PHI = 332;

template<class Ops>
void do_kick(KickCtx& C, KickAcc& acc, const float* L, const ct_or_node& self, std::vector<Force>& force) {
	const auto& p = *C.p;
	const int nsink = self.part_end - self.part_begin;
	for (int i = 0; i < nsink; i++) {
		const int snki = self.part_begin + i;
		float dx[3];
		for (int d = 0; d < 3; d++) {
			dx[d] = fdist(C.x[d][snki], self.pos[d]);
		}
		float L2[5];
		Ops::l2p(L2, L, dx[0], dx[1], dx[2], p.do_phi != 0);
		Force& F = force[i];
		F.phi += 1e3f * L2[0];
		F.gx -= 1e6f * L2[1];
		F.gy -= 1e6f * L2[2];
		F.gz -= 1e6f * L2[3];
		F.gz *= p.GM;
		F.gy *= p.GM;
		F.gx *= p.GM;
		F.phi *= p.GM;
		float vx = C.v[3 * snki + 0], vy = C.v[3 * snki + 1], vz = C.v[3 * snki + 2];
		const float kin0 = 0.5 * sqrf(vx, vy, vz);
		const float sgn = p.sign * (p.top ? 1.f : -1.f);
		const float rdt = 1.0f / float(1 << p.min_rung);
		if (p.ascending) {
			const float dt = 0.5f * rdt * p.t0;
			if (!p.first_call) {
				vx = std::fma(sgn * F.gx, dt, vx);
				vy = std::fma(sgn * F.gy, dt, vy);
				vz = std::fma(sgn * F.gz, dt, vz);
			}
		}
		acc.kin += 0.5f * sqrf(vx, vy, vz);
		acc.xmom += vx;
		acc.ymom += vy;
		acc.zmom += vz;
		acc.nmom += std::sqrt(sqrf(vx, vy, vz));
		if (p.save_force) {
			C.gx[snki] = F.gx;
			C.gy[snki] = F.gy;
			C.gz[snki] = F.gz;
			C.pot[snki] = F.phi;
		}
		if (p.descending) {
			const float g2 = sqrf(F.gx, F.gy, F.gz);
			float dt = std::min(p.eta * std::sqrt(p.a * p.h * (1.0f / std::sqrt(g2))), p.t0);
			dt = std::min(p.max_dt, dt);
			int rung = C.rung[snki];
			rung = std::max(p.min_rung + int(int(std::ceil(std::log2(p.t0 / dt))) > p.min_rung), rung - 1);
			C.rung[snki] = int8_t(rung);
			acc.max_rung = std::max(rung, acc.max_rung);
			dt = 0.5f * rdt * p.t0;
			vx = std::fma(sgn * F.gx, dt, vx);
			vy = std::fma(sgn * F.gy, dt, vy);
			vz = std::fma(sgn * F.gz, dt, vz);
		}
		const float kin1 = 0.5 * sqrf(vx, vy, vz);
		C.v[3 * snki + 0] = vx;
		C.v[3 * snki + 1] = vy;
		C.v[3 * snki + 2] = vz;
		acc.pot += 0.5f * F.phi;
		acc.dkin += kin1 - kin0;
		acc.flops += 557 + p.do_phi * 178;
	}
}

template<class Ops>
void walk(KickCtx& C, KickAcc& acc, int selfi, const float* Lparent, const uint32_t* Lpos, std::vector<int> echecks, std::vector<int> dchecks) {
	const auto& p = *C.p;
	const ct_or_node* nodes = C.nodes;
	const ct_or_node& self = nodes[selfi];
	const bool do_phi = p.do_phi != 0;
	const float thetainv = 1.f / p.theta;
	const float h = p.h;
	float L[Ops::NEXP];
	{
		float dx[3];
		for (int d = 0; d < 3; d++) {
			dx[d] = fdist(self.pos[d], Lpos[d]);
		}
		Ops::l2l(L, Lparent, dx[0], dx[1], dx[2], do_phi);
		acc.flops += FLOP_L2L_CUDA + do_phi * FLOP_L2L_PHI;
	}
	const int nsinks = self.part_end - self.part_begin;
	std::vector<Force> force;
	if (self.leaf) {
		force.resize(nsinks);
		for (auto& f : force) {
			f.gx = f.gy = f.gz = 0.f;
			f.phi = self_phi() * (1.f / h);
		}
	}
	const float rs = self.radius;
	if (nsinks) {
		// Ewald check list: one pass (kick.cu:269-329)
		std::vector<int> cc, next;
		for (int c : echecks) {
			const ct_or_node& o = nodes[c];
			if (o.part_end - o.part_begin) {
				float dx[3];
				for (int d = 0; d < 3; d++) {
					dx[d] = fdist(self.pos[d], o.pos[d]);
				}
				float R2 = sqrf(dx[0], dx[1], dx[2]);
				const float t = std::max(0.5f - (rs + o.radius), 0.f);
				R2 = std::max(R2, t * t);
				const float dcc = (rs + o.radius) * thetainv;
				if (R2 > dcc * dcc) {
					cc.push_back(c);
				} else {
					next.push_back(c);
				}
			}
		}
		echecks.clear();
		for (int c : next) {
			echecks.push_back(nodes[c].child_left);
			echecks.push_back(nodes[c].child_right);
		}
		if (!cc.empty()) {
			float Lacc[Ops::NEXP] = { };
			for (int c : cc) {
				const ct_or_node& o = nodes[c];
				float dx[3], D[Ops::NEXP];
				for (int d = 0; d < 3; d++) {
					dx[d] = fdist(self.pos[d], o.pos[d]);
				}
				const int icnt = Ops::ewald(D, dx[0], dx[1], dx[2]);
				Ops::m2l(Lacc, o.multi, D, do_phi);
				acc.flops += 3 + 7 + 843.0 * icnt + 140 * 92 + 540 + FLOP_M2L + do_phi * FLOP_M2L_PHI;
			}
			for (int i = 0; i < Ops::NEXP; i++) {
				L[i] += Lacc[i];
			}
		}
	}
	std::vector<int> leaflist;
	if (nsinks) {
		// Direct check list (kick.cu:330-431)
		std::vector<int> cc, cp, pc, next;
		std::vector<int>& checks = dchecks;
		do {
			for (int c : checks) {
				const ct_or_node& o = nodes[c];
				const int onp = o.part_end - o.part_begin;
				if (!onp) {
					continue;
				}
				float dx[3];
				for (int d = 0; d < 3; d++) {
					dx[d] = fdist(self.pos[d], o.pos[d]);
				}
				const float R2 = sqrf(dx[0], dx[1], dx[2]);
				const float mind = rs + o.radius + h;
				const float dcc = std::max((rs + o.radius) * thetainv, mind);
				bool sw_cc = R2 > dcc * dcc, sw_cp = false, sw_pc = false;
				if (!sw_cc && o.leaf && self.leaf) {
					const float dcp = std::max((rs * thetainv + o.radius), mind);
					const float dpc = std::max((rs + o.radius * thetainv), mind);
					sw_pc = (R2 > dpc * dpc || !box_intersects_sphere(self, o.pos, std::max(thetainv * o.radius, h))) && nsinks >= 38;
					sw_cp = (R2 > dcp * dcp || !box_intersects_sphere(o, self.pos, std::max(thetainv * rs, h))) && onp >= 38;
					if (sw_pc && sw_cp) {
						if (nsinks < onp) {
							sw_cp = false;
						} else if (nsinks > onp) {
							sw_pc = false;
						} else {
							sw_cp = sw_pc = false;
						}
					}
				}
				if (sw_cc) {
					cc.push_back(c);
				} else if (sw_cp) {
					cp.push_back(c);
				} else if (sw_pc) {
					pc.push_back(c);
				} else if (o.leaf) {
					leaflist.push_back(c);
				} else {
					next.push_back(c);
				}
			}
			checks.clear();
			for (int c : next) {
				checks.push_back(nodes[c].child_left);
				checks.push_back(nodes[c].child_right);
			}
			next.clear();
		} while (!checks.empty() && self.leaf);
		// cuda_gravity_cc_direct
		if (!cc.empty()) {
			float Lacc[Ops::NEXP] = { };
			for (int c : cc) {
				const ct_or_node& o = nodes[c];
				float dx[3], D[Ops::NEXP];
				for (int d = 0; d < 3; d++) {
					dx[d] = fdist(self.pos[d], o.pos[d]);
				}
				Ops::greens(D, dx[0], dx[1], dx[2]);
				Ops::m2l(Lacc, o.multi, D, do_phi);
				acc.flops += 6 + FLOP_GREENS + FLOP_M2L + do_phi * FLOP_M2L_PHI;
			}
			for (int i = 0; i < Ops::NEXP; i++) {
				L[i] += Lacc[i];
			}
		}
		if (self.leaf) {
			// cuda_gravity_cp_direct: source particles into the local expansion
			if (!cp.empty()) {
				float Lacc[Ops::NEXP] = { };
				for (int c : cp) {
					const ct_or_node& o = nodes[c];
					for (int j = o.part_begin; j < o.part_end; j++) {
						float dx[3];
						for (int d = 0; d < 3; d++) {
							dx[d] = fdist(self.pos[d], C.x[d][j]);
						}
						Ops::greens_add(Lacc, dx[0], dx[1], dx[2]);
						acc.flops += Ops::NEXP + 6 + FLOP_GREENS;
					}
				}
				for (int i = 0; i < Ops::NEXP; i++) {
					L[i] += Lacc[i];
				}
			}
			// cuda_gravity_pc_direct: source multipoles at each sink
			for (int c : pc) {
				const ct_or_node& o = nodes[c];
				for (int k = 0; k < nsinks; k++) {
					const int s = self.part_begin + k;
					float dx[3], D[Ops::NEXP], L2[5] = { 0, 0, 0, 0, 0 };
					for (int d = 0; d < 3; d++) {
						dx[d] = fdist(C.x[d][s], o.pos[d]);
					}
					Ops::greens(D, dx[0], dx[1], dx[2]);
					Ops::m2l2(L2, o.multi, D, do_phi);
					force[k].gx -= 1e6f * L2[1];
					force[k].gy -= 1e6f * L2[2];
					force[k].gz -= 1e6f * L2[3];
					force[k].phi += 1e3f * L2[0];
					acc.flops += 6 + FLOP_GREENS + 520 + do_phi * FLOP_M2L_PHI + 4;
				}
			}
			// cuda_gravity_pp_direct
			if (!leaflist.empty()) {
				const float h2 = h * h;
				const float hinv = 1.f / h;
				const float h2inv = hinv * hinv;
				const float h3inv = h2inv * hinv;
				for (int k = 0; k < nsinks; k++) {
					const int s = self.part_begin + k;
					// pairwise terms in FP32 as the reference computes them; sums kept in FP64 so that
					// the oracle carries no accumulation error of its own
					double fx = 0.0, fy = 0.0, fz = 0.0, pot = 0.0;
					for (int c : leaflist) {
						const ct_or_node& o = nodes[c];
						for (int j = o.part_begin; j < o.part_end; j++) {
							const float dx0 = fdist(C.x[0][s], C.x[0][j]);
							const float dx1 = fdist(C.x[1][s], C.x[1][j]);
							const float dx2 = fdist(C.x[2][s], C.x[2][j]);
							const float r2 = sqrf(dx0, dx1, dx2);
							float r1inv, r3inv;
							if (r2 > h2) {
								r1inv = 1.0f / std::sqrt(r2);
								r3inv = r1inv * r1inv * r1inv;
							} else {
								gsoft(r3inv, r1inv, r2, hinv, h2inv, h3inv);
							}
							fx += double(dx0 * r3inv);
							fy += double(dx1 * r3inv);
							fz += double(dx2 * r3inv);
							pot -= double(r1inv);
						}
						acc.flops += 21.0 * (o.part_end - o.part_begin);
					}
					force[k].gx = float(double(force[k].gx) - fx);
					force[k].gy = float(double(force[k].gy) - fy);
					force[k].gz = float(double(force[k].gz) - fz);
					force[k].phi = float(double(force[k].phi) + pot);
				}
			}
		} else {
			for (int c : leaflist) {
				checks.push_back(c);
			}
		}
	}
	if (self.leaf) {
		if (nsinks) {
			do_kick<Ops>(C, acc, L, self, force);
		}
	} else {
		walk<Ops>(C, acc, self.child_left, L, self.pos, echecks, dchecks);
		walk<Ops>(C, acc, self.child_right, L, self.pos, echecks, dchecks);
	}
}

// Work items: the walk above a cut (nodes holding more than max_parts particles that are not
// leaves) hands each subtree below it, with its check lists and the expansion of its parent,
// to a work item (subtrees without particles too, which the reference hands to nobody,
// kick.cpp:178-181: they carry no particles and no work) -- the split the reference makes between its CPU top and its GPU kernel
// (kick.cpp:169-190), with the items ordered by their first particle as the reference's
// kick_workspace orders them (kick_workspace.cpp:308-310).  The top runs level by level, the
// nodes of one level on all threads.
template<class Ops>
struct WorkItem {
	int self;
	std::vector<float> L;  // the parent's expansion, about Lpos
	uint32_t pos[3];
	std::vector<int> e, d;
};

// One node above the cut: its expansion from the parent's (L2L) and its Ewald and direct
// check lists (the same list processing as walk() for a non-leaf node); the two children
// inherit the result.
template<class Ops>
void top_expand(KickCtx& C, KickAcc& acc, const WorkItem<Ops>& w, WorkItem<Ops>& left, WorkItem<Ops>& right) {
	const ct_or_node& self = C.nodes[w.self];
	const auto& p = *C.p;
	const ct_or_node* nodes = C.nodes;
	const bool do_phi = p.do_phi != 0;
	const float thetainv = 1.f / p.theta;
	const float h = p.h;
	float L[Ops::NEXP];
	float dx[3];
	for (int d = 0; d < 3; d++) {
		dx[d] = fdist(self.pos[d], w.pos[d]);
	}
	Ops::l2l(L, w.L.data(), dx[0], dx[1], dx[2], do_phi);
	acc.flops += FLOP_L2L_CUDA + do_phi * FLOP_L2L_PHI;
	const float rs = self.radius;
	std::vector<int> cc, next;
	for (int c : w.e) {
		const ct_or_node& o = nodes[c];
		if (o.part_end - o.part_begin) {
			for (int d = 0; d < 3; d++) {
				dx[d] = fdist(self.pos[d], o.pos[d]);
			}
			float R2 = sqrf(dx[0], dx[1], dx[2]);
			const float t = std::max(0.5f - (rs + o.radius), 0.f);
			R2 = std::max(R2, t * t);
			const float dcc = (rs + o.radius) * thetainv;
			if (R2 > dcc * dcc) {
				cc.push_back(c);
			} else {
				next.push_back(c);
			}
		}
	}
	std::vector<int> e2;
	for (int c : next) {
		e2.push_back(nodes[c].child_left);
		e2.push_back(nodes[c].child_right);
	}
	if (!cc.empty()) {
		float Lacc[Ops::NEXP] = { };
		for (int c : cc) {
			const ct_or_node& o = nodes[c];
			float D[Ops::NEXP];
			for (int d = 0; d < 3; d++) {
				dx[d] = fdist(self.pos[d], o.pos[d]);
			}
			const int icnt = Ops::ewald(D, dx[0], dx[1], dx[2]);
			Ops::m2l(Lacc, o.multi, D, do_phi);
			acc.flops += 3 + 7 + 843.0 * icnt + 140 * 92 + 540 + FLOP_M2L + do_phi * FLOP_M2L_PHI;
		}
		for (int i = 0; i < Ops::NEXP; i++) {
			L[i] += Lacc[i];
		}
	}
	cc.clear();
	next.clear();
	std::vector<int> leaf;
	for (int c : w.d) {
		const ct_or_node& o = nodes[c];
		if (!(o.part_end - o.part_begin)) {
			continue;
		}
		for (int d = 0; d < 3; d++) {
			dx[d] = fdist(self.pos[d], o.pos[d]);
		}
		const float R2 = sqrf(dx[0], dx[1], dx[2]);
		const float mind = rs + o.radius + h;
		const float dcc = std::max((rs + o.radius) * thetainv, mind);
		if (R2 > dcc * dcc) {
			cc.push_back(c);
		} else if (o.leaf) {
			leaf.push_back(c);
		} else {
			next.push_back(c);
		}
	}
	std::vector<int> d2;
	for (int c : next) {
		d2.push_back(nodes[c].child_left);
		d2.push_back(nodes[c].child_right);
	}
	for (int c : leaf) {
		d2.push_back(c);
	}
	if (!cc.empty()) {
		float Lacc[Ops::NEXP] = { };
		for (int c : cc) {
			const ct_or_node& o = nodes[c];
			float D[Ops::NEXP];
			for (int d = 0; d < 3; d++) {
				dx[d] = fdist(self.pos[d], o.pos[d]);
			}
			Ops::greens(D, dx[0], dx[1], dx[2]);
			Ops::m2l(Lacc, o.multi, D, do_phi);
			acc.flops += 6 + FLOP_GREENS + FLOP_M2L + do_phi * FLOP_M2L_PHI;
		}
		for (int i = 0; i < Ops::NEXP; i++) {
			L[i] += Lacc[i];
		}
	}
	for (WorkItem<Ops>* ch : { &left, &right }) {
		ch->L.assign(L, L + Ops::NEXP);
		for (int d = 0; d < 3; d++) {
			ch->pos[d] = self.pos[d];
		}
		ch->e = e2;
		ch->d = d2;
	}
	left.self = self.child_left;
	right.self = self.child_right;
}

struct PlanBase {
	virtual ~PlanBase() {
	}
	ct_or_kick_params p;
	KickCtx C;
	int order;
	KickAcc top;
	double top_seconds = 0.0;
	virtual int64_t size() const = 0;
	virtual void info(int32_t* self, int32_t* nparts, int64_t* dsum, int32_t* ne) const = 0;
	virtual void run(const int8_t* select, int nthreads, double* seconds, KickAcc& tot) = 0;
	virtual void list_sizes(int64_t* nd, int64_t* ne) const = 0;
	virtual void export_items(int32_t* self, float* L, int nexp, uint32_t* pos, int64_t* doff, int32_t* dlist, int64_t* eoff, int32_t* elist) const = 0;
};

template<class Ops>
struct Plan: PlanBase {
	std::vector<WorkItem<Ops>> items;
	int64_t size() const override {
		return (int64_t) items.size();
	}
	void build(int max_parts, int nthreads) {
		const auto t0 = std::chrono::steady_clock::now();
		std::vector<WorkItem<Ops>> level(1);
		level[0].self = 0;
		level[0].L.assign(Ops::NEXP, 0.f);
		for (int d = 0; d < 3; d++) {
			level[0].pos[d] = 0;
		}
		level[0].e.assign(1, 0);
		level[0].d.assign(1, 0);
		while (!level.empty()) {
			const int n = (int) level.size();
			std::vector<WorkItem<Ops>> kids(2 * (size_t) n);
			std::vector<char> expanded(n, 0);
			std::vector<KickAcc> accs(n);
			parallel_for(n, nthreads, [&](int i) {
				const ct_or_node& nd = C.nodes[level[i].self];
				if (nd.leaf || nd.part_end - nd.part_begin <= max_parts) {
					return;
				}
				top_expand<Ops>(C, accs[i], level[i], kids[2 * i], kids[2 * i + 1]);
				expanded[i] = 1;
			});
			std::vector<WorkItem<Ops>> nextl;
			for (int i = 0; i < n; i++) {
				top.flops += accs[i].flops;
				if (expanded[i]) {
					nextl.push_back(std::move(kids[2 * i]));
					nextl.push_back(std::move(kids[2 * i + 1]));
				} else {
					items.push_back(std::move(level[i]));
				}
			}
			level.swap(nextl);
		}
		std::stable_sort(items.begin(), items.end(), [&](const WorkItem<Ops>& a, const WorkItem<Ops>& b) {
			return C.nodes[a.self].part_begin < C.nodes[b.self].part_begin;
		});
		top_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	}
	void info(int32_t* self, int32_t* nparts, int64_t* dsum, int32_t* ne) const override {
		for (size_t i = 0; i < items.size(); i++) {
			const ct_or_node& nd = C.nodes[items[i].self];
			if (self) {
				self[i] = items[i].self;
			}
			if (nparts) {
				nparts[i] = nd.part_end - nd.part_begin;
			}
			if (dsum) {
				int64_t s = 0;
				for (int c : items[i].d) {
					s += C.nodes[c].part_end - C.nodes[c].part_begin;
				}
				dsum[i] = s;
			}
			if (ne) {
				ne[i] = (int32_t) items[i].e.size();
			}
		}
	}
	void list_sizes(int64_t* nd, int64_t* ne) const override {
		*nd = *ne = 0;
		for (const auto& w : items) {
			*nd += (int64_t) w.d.size();
			*ne += (int64_t) w.e.size();
		}
	}
	void export_items(int32_t* self, float* L, int nexp, uint32_t* pos, int64_t* doff, int32_t* dlist, int64_t* eoff, int32_t* elist) const override {
		int64_t d = 0, e = 0;
		for (size_t i = 0; i < items.size(); i++) {
			const auto& w = items[i];
			self[i] = w.self;
			for (int k = 0; k < nexp; k++) {
				L[i * nexp + k] = k < Ops::NEXP ? w.L[k] : 0.f;
			}
			for (int k = 0; k < 3; k++) {
				pos[3 * i + k] = w.pos[k];
			}
			doff[i] = d;
			eoff[i] = e;
			for (int c : w.d) {
				dlist[d++] = c;
			}
			for (int c : w.e) {
				elist[e++] = c;
			}
		}
		doff[items.size()] = d;
		eoff[items.size()] = e;
	}
	void run(const int8_t* select, int nthreads, double* seconds, KickAcc& tot) override {
		std::vector<int> todo;
		for (int i = 0; i < (int) items.size(); i++) {
			if (!select || select[i]) {
				todo.push_back(i);
			}
		}
		std::vector<KickAcc> accs(todo.size());
		parallel_for((int) todo.size(), nthreads, [&](int k) {
			const int i = todo[k];
			const auto t0 = std::chrono::steady_clock::now();
			walk<Ops>(C, accs[k], items[i].self, items[i].L.data(), items[i].pos, items[i].e, items[i].d);
			if (seconds) {
				seconds[i] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
			}
		});
		tot = top;
		for (auto& a : accs) {
			tot.max_rung = std::max(tot.max_rung, a.max_rung);
			tot.pot += a.pot;
			tot.kin += a.kin;
			tot.dkin += a.dkin;
			tot.xmom += a.xmom;
			tot.ymom += a.ymom;
			tot.zmom += a.zmom;
			tot.nmom += a.nmom;
			tot.flops += a.flops;
		}
	}
};

PlanBase* make_plan(int order, const ct_or_kick_params* p, int nnodes, const ct_or_node* nodes, const uint32_t* x, const uint32_t* y,
		const uint32_t* z, int max_parts, int nthreads) {
	if (nnodes <= 0) {
		return nullptr;
	}
	PlanBase* P;
	if (order == 5) {
		P = new Plan<Ops5>();
	} else {
		P = new Plan<Ops7>();
	}
	P->order = order;
	P->p = *p;
	P->C.p = &P->p;
	P->C.nodes = nodes;
	P->C.x[0] = x;
	P->C.x[1] = y;
	P->C.x[2] = z;
	P->C.v = nullptr;
	P->C.rung = nullptr;
	P->C.gx = P->C.gy = P->C.gz = P->C.pot = nullptr;
	if (nthreads <= 0) {
		nthreads = std::max(1u, std::thread::hardware_concurrency());
	}
	if (max_parts <= 0) {
		const int ntot = nodes[0].part_end - nodes[0].part_begin;
		max_parts = std::max(ntot / std::max(1, 16 * nthreads), 1);
	}
	if (order == 5) {
		static_cast<Plan<Ops5>*>(P)->build(max_parts, nthreads);
	} else {
		static_cast<Plan<Ops7>*>(P)->build(max_parts, nthreads);
	}
	return P;
}

void store_return(const KickAcc& tot, ct_or_kick_return* rc, double* flops) {
	if (rc) {
		rc->max_rung = tot.max_rung;
		rc->pot = tot.pot;
		rc->kin = tot.kin;
		rc->dkin = tot.dkin;
		rc->xmom = tot.xmom;
		rc->ymom = tot.ymom;
		rc->zmom = tot.zmom;
		rc->nmom = tot.nmom;
	}
	if (flops) {
		*flops = tot.flops;
	}
}

int plan_run(PlanBase* P, float* v, int8_t* rung, float* gx, float* gy, float* gz, float* pot, const int8_t* select, int nthreads,
		double* seconds, ct_or_kick_return* rc, double* flops) {
	if (P->p.save_force && (!gx || !gy || !gz || !pot)) {
		return -2;
	}
	P->C.v = v;
	P->C.rung = rung;
	P->C.gx = gx;
	P->C.gy = gy;
	P->C.gz = gz;
	P->C.pot = pot;
	KickAcc tot;
	P->run(select, nthreads, seconds, tot);
	store_return(tot, rc, flops);
	return 0;
}

// ---------------------------------------------------------------- FP64 direct Ewald
// Periodic potential of a unit mass minus the bare nearest-image 1/r term, and its gradient,
// alpha = 2: erf(alpha r)/r for the n=0 image, -erfc/r for the other images inside 2.6 box
// lengths, Fourier terms 0<|h|^2<=8 via per-sink sums, and the pi/alpha^2 background term.
void ewald_correction_real(double dx, double dy, double dz, double& phi, double* g, const ct_p7::EwaldTab& tab) {
	const double alpha = 2.0;
	const double twooversqrtpi = 1.1283791670955126;
	double r2 = dx * dx + dy * dy + dz * dz;
	double r = std::sqrt(r2);
	if (alpha * r < 0.05) {
		// erf(a r)/r = (2a/sqrt(pi)) (1 - a^2 r^2/3 + a^4 r^4/10 - a^6 r^6/42 + a^8 r^8/216)
		const double a2r2 = alpha * alpha * r2;
		phi += twooversqrtpi * alpha * (1.0 - a2r2 / 3.0 + a2r2 * a2r2 / 10.0 - a2r2 * a2r2 * a2r2 / 42.0 + a2r2 * a2r2 * a2r2 * a2r2 / 216.0);
		// gradient: x * (2a/sqrt(pi)) a^2 (-2/3 + 4 a^2 r^2/10 - 6 a^4 r^4 /42 + 8 a^6 r^6/216)
		const double c = twooversqrtpi * alpha * alpha * alpha * (-2.0 / 3.0 + 0.4 * a2r2 - a2r2 * a2r2 / 7.0 + a2r2 * a2r2 * a2r2 / 27.0);
		g[0] += c * dx;
		g[1] += c * dy;
		g[2] += c * dz;
	} else {
		const double e = std::erf(alpha * r);
		phi += e / r;
		const double dphidr = -e / r2 + twooversqrtpi * alpha * std::exp(-alpha * alpha * r2) / r;
		g[0] += dphidr * dx / r;
		g[1] += dphidr * dy / r;
		g[2] += dphidr * dz / r;
	}
	for (int i = 0; i < CT_EWALD_NREAL; i++) {
		const double x = dx - tab.real[i][0], y = dy - tab.real[i][1], z = dz - tab.real[i][2];
		const double s2 = x * x + y * y + z * z;
		if (s2 < 2.6 * 2.6) {
			const double s = std::sqrt(s2);
			const double ec = std::erfc(alpha * s);
			phi -= ec / s;
			const double dphids = ec / s2 + twooversqrtpi * alpha * std::exp(-alpha * alpha * s2) / s;
			g[0] += dphids * x / s;
			g[1] += dphids * y / s;
			g[2] += dphids * z / s;
		}
	}
	phi += M_PI / (alpha * alpha);
}

}  // namespace

// ---------------------------------------------------------------- C entry points
extern "C" {

#define CT_OR_DISPATCH(order, call7, call5) do { if ((order) == 5) { call5; } else { call7; } } while (0)

int ct_or_greens(int order, const float* X, float* D) {
	CT_OR_DISPATCH(order, ct_p7::greens(D, X[0], X[1], X[2]), ct_p5::greens(D, X[0], X[1], X[2]));
	return 0;
}
int ct_or_ewald_greens(int order, const float* X, float* D) {
	int ic = 0;
	CT_OR_DISPATCH(order, ic = Ops7::ewald(D, X[0], X[1], X[2]), ic = Ops5::ewald(D, X[0], X[1], X[2]));
	return ic;
}
int ct_or_ewald_greens_d(int order, const double* X, double* D) {
	int ic = 0;
	CT_OR_DISPATCH(order, ic = ct_p7::ewald_greens(D, X[0], X[1], X[2], Ops7::tab()), ic = ct_p5::ewald_greens(D, X[0], X[1], X[2], Ops5::tab()));
	return ic;
}
void ct_or_m2l(int order, const float* M, const float* D, float* L, int do_phi) {
	CT_OR_DISPATCH(order, ct_p7::m2l(L, M, D, do_phi != 0), ct_p5::m2l(L, M, D, do_phi != 0));
}
void ct_or_m2l2(int order, const float* M, const float* D, float* L, int do_phi) {
	CT_OR_DISPATCH(order, ct_p7::m2l_2(L, M, D, do_phi != 0), ct_p5::m2l_2(L, M, D, do_phi != 0));
}
void ct_or_p2m(int order, const float* X, float* M) {
	CT_OR_DISPATCH(order, ct_p7::p2m(M, X[0], X[1], X[2]), ct_p5::p2m(M, X[0], X[1], X[2]));
}
void ct_or_m2m_d(int order, const double* M, const double* X, double* Mout) {
	CT_OR_DISPATCH(order, ct_p7::m2m(Mout, M, X[0], X[1], X[2]), ct_p5::m2m(Mout, M, X[0], X[1], X[2]));
}
void ct_or_l2l(int order, const float* L, const float* X, float* Lout, int do_phi) {
	CT_OR_DISPATCH(order, ct_p7::l2l(Lout, L, X[0], X[1], X[2], do_phi != 0), ct_p5::l2l(Lout, L, X[0], X[1], X[2], do_phi != 0));
}
void ct_or_l2p(int order, const float* L, const float* X, float* Lout, int do_phi) {
	CT_OR_DISPATCH(order, ct_p7::l2p(Lout, L, X[0], X[1], X[2], do_phi != 0), ct_p5::l2p(Lout, L, X[0], X[1], X[2], do_phi != 0));
}
void ct_or_ewald_tables(int order, float* real_idx, float* four_idx, float* four_exp, float* D0) {
	auto copy = [&](const auto& t, int nexp, int nfull) {
		memcpy(real_idx, t.real, sizeof(t.real));
		memcpy(four_idx, t.four, sizeof(t.four));
		for (int i = 0; i < CT_EWALD_NFOUR; i++) {
			for (int k = 0; k < nexp; k++) {
				four_exp[i * nexp + k] = t.four_exp[i][k];
			}
		}
		for (int c = 0; c < nfull; c++) {
			D0[c] = t.D0[c];
		}
	};
	CT_OR_DISPATCH(order, copy(Ops7::tab(), ct_p7::NEXP, ct_p7::NFULL), copy(Ops5::tab(), ct_p5::NEXP, ct_p5::NFULL));
}

int ct_or_tree_build(int order, int n, int begin, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, int8_t* rung, double theta, double hsoft,
		int bucket, ct_or_node* nodes, int max_nodes, int nthreads) {
	Builder B;
	B.x[0] = x;
	B.x[1] = y;
	B.x[2] = z;
	B.v = vxyz;
	B.r = rung;
	B.theta = theta;
	B.h = hsoft;
	B.bucket = bucket;
	B.too_deep = false;
	if (nthreads <= 0) {
		nthreads = std::max(1u, std::thread::hardware_concurrency());
	}
	// about two subtrees per thread
	B.fork_depth = 0;
	while ((1 << B.fork_depth) < 2 * nthreads && nthreads > 1) {
		B.fork_depth++;
	}
	B.nodes.reserve(std::max(64, 2 * (n - begin) / std::max(bucket / 2, 1)));
	const double bb[3] = { 0, 0, 0 }, be[3] = { 1, 1, 1 };
	if (order == 5) {
		tree_create<Ops5>(B, 1, begin, n, bb, be, 0);
	} else {
		tree_create<Ops7>(B, 1, begin, n, bb, be, 0);
	}
	if (B.too_deep) {
		return -2;
	}
	if ((int64_t) B.nodes.size() > max_nodes) {
		return -1;
	}
	memcpy(nodes, B.nodes.data(), sizeof(ct_or_node) * B.nodes.size());
	return (int) B.nodes.size();
}

int ct_or_kick(int order, const ct_or_kick_params* p, int nnodes, const ct_or_node* nodes, const uint32_t* x, const uint32_t* y, const uint32_t* z,
		float* vxyz, int8_t* rung, float* gx, float* gy, float* gz, float* pot, ct_or_kick_return* rc, int nthreads, double* flops) {
	if (p->save_force && (!gx || !gy || !gz || !pot)) {
		return -2;
	}
	PlanBase* P = make_plan(order, p, nnodes, nodes, x, y, z, 0, nthreads);
	if (!P) {
		return -1;
	}
	const int err = plan_run(P, vxyz, rung, gx, gy, gz, pot, nullptr, nthreads, nullptr, rc, flops);
	delete P;
	return err;
}

void* ct_or_kick_plan_create(int order, const ct_or_kick_params* p, int nnodes, const ct_or_node* nodes, const uint32_t* x, const uint32_t* y,
		const uint32_t* z, int max_parts, int nthreads, int64_t* nitems, double* top_seconds) {
	PlanBase* P = make_plan(order, p, nnodes, nodes, x, y, z, max_parts, nthreads);
	if (P) {
		if (nitems) {
			*nitems = P->size();
		}
		if (top_seconds) {
			*top_seconds = P->top_seconds;
		}
	}
	return P;
}

void ct_or_kick_plan_items(const void* plan, int32_t* self, int32_t* nparts, int64_t* near_parts, int32_t* ewald_checks) {
	static_cast<const PlanBase*>(plan)->info(self, nparts, near_parts, ewald_checks);
}

int ct_or_kick_plan_run(void* plan, float* vxyz, int8_t* rung, float* gx, float* gy, float* gz, float* pot, const int8_t* select, int nthreads,
		double* item_seconds, ct_or_kick_return* rc, double* flops) {
	return plan_run(static_cast<PlanBase*>(plan), vxyz, rung, gx, gy, gz, pot, select, nthreads, item_seconds, rc, flops);
}

void ct_or_kick_plan_list_sizes(const void* plan, int64_t* ndirect, int64_t* newald) {
	static_cast<const PlanBase*>(plan)->list_sizes(ndirect, newald);
}

void ct_or_kick_plan_export(const void* plan, int32_t* self, float* L, int nexp, uint32_t* pos, int64_t* doff, int32_t* dlist, int64_t* eoff,
		int32_t* elist) {
	static_cast<const PlanBase*>(plan)->export_items(self, L, nexp, pos, doff, dlist, eoff, elist);
}

void ct_or_kick_plan_destroy(void* plan) {
	delete static_cast<PlanBase*>(plan);
}

void ct_or_drift(int n, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, const int8_t* rung, int which_rung, float a, float dt, double drag) {
	const double c1 = double(dt) / double(a);
	uint32_t* X[3] = { x, y, z };
	for (int i = 0; i < n; i++) {
		if (rung[i] != which_rung) {
			continue;
		}
		for (int d = 0; d < 3; d++) {
			const double x0 = fixed32_to_double(X[d][i]);
			double x1 = x0 + double(vxyz[3 * i + d]) * c1;
			x1 -= double(x1 >= 1.0);
			x1 += double(x1 < 0.0);
			X[d][i] = fixed32_from_double(x1);
		}
		if (drag != 0.0) {
			const double c0 = 1.0 / (1.0 + drag * double(dt));
			for (int d = 0; d < 3; d++) {
				vxyz[3 * i + d] *= c0;
			}
		}
	}
}

// Bits 0..12 of v to the even bit positions 0..24.
static uint32_t spread13(uint32_t v) {
	uint32_t r = 0;
	for (int b = 0; b < 13; b++) {
		r |= ((v >> b) & 1u) << (2 * b);
	}
	return r;
}

// The HEALPix construction (Gorski et al. 2005, ApJ 622:759), as the reference evaluates it
// (src/healpix.cu:55-171): face and in-face coordinates at the finest resolution 8192, the
// nested index by bit interleaving (x on even bits), degraded to nside by integer division.
int ct_or_healpix_nest(int nside, double x, double y, double z) {
	const int NS = 8192;
	const double piover2 = 0.5 * M_PI, twopi = 2.0 * M_PI;
	const double zn = z / std::sqrt(x * x + y * y + z * z);
	double phi = 0.0;
	if (x != 0.0 || y != 0.0) {
		phi = std::atan2(y, x);
		if (phi < 0.0) {
			phi += twopi;
		}
	}
	const double za = std::fabs(zn);
	const double tt = phi / piover2;
	int face, ix, iy;
	if (za <= 2. / 3.) {
		const int jp = (int) std::floor(NS * (0.5 + tt - zn * 0.75));
		const int jm = (int) std::floor(NS * (0.5 + tt + zn * 0.75));
		const int ifp = jp / NS, ifm = jm / NS;
		if (ifp == ifm) {
			face = ifp % 4 + 4;
		} else if (ifp < ifm) {
			face = ifp % 4;
		} else {
			face = ifm % 4 + 8;
		}
		ix = jm % NS;
		iy = NS - jp % NS - 1;
	} else {
		int ntt = (int) std::floor(tt);
		if (ntt >= 4) {
			ntt = 3;
		}
		const double tp = tt - ntt;
		const double tmp = std::sqrt(3. * (1. - za));
		const int jp = std::min((int) std::floor(NS * tp * tmp), NS - 1);
		const int jm = std::min((int) std::floor(NS * (1. - tp) * tmp), NS - 1);
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

// fixed<int,31> = double (fixed.hpp:97-101): truncation of 2^31 x, saturating as the GPU's
// conversion does at x = 1.
static int32_t fixed31_from_double(double x) {
	const double s = 2147483648.0 * x;
	if (s >= 2147483647.0) {
		return 2147483647;
	}
	return (int32_t) s;
}

int64_t ct_or_drift_lc(int n, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, const int8_t* rung, int which_rung, float a, float dt,
		double drag, float tau0, float tau1, float tau_max, int nside, ct_or_lc_entry* out, int64_t max_out) {
	// kernel arguments as cuda_drift passes them (src/drift.cu:156-195): floats widened to double
	const double da = a, ddt = dt, t0 = tau0, t1 = tau1, tmax = tau_max;
	const bool do_lc = tmax - t1 < 1.0;
	const double c0 = 1.0 / tmax;
	const double ainv = 1.0 / da;
	const double c1 = ddt / da;
	uint32_t* X[3] = { x, y, z };
	int64_t count = 0;
	for (int i = 0; i < n; i++) {
		if (rung[i] != which_rung) {
			continue;
		}
		float* vel = vxyz + 3 * i;
		double p0[3], p1[3];
		for (int d = 0; d < 3; d++) {
			p0[d] = fixed32_to_double(X[d][i]);
			p1[d] = p0[d] + double(vel[d]) * c1;
		}
		if (drag != 0.0) {
			const double dc = 1.0 / (1.0 + drag * ddt);
			for (int d = 0; d < 3; d++) {
				vel[d] *= dc;
			}
		}
		if (do_lc) {
			for (int xi = -1; xi <= 0; xi++) {
				for (int yi = -1; yi <= 0; yi++) {
					for (int zi = -1; zi <= 0; zi++) {
						const double A0[3] = { p0[0] + xi, p0[1] + yi, p0[2] + zi };
						const double A1[3] = { p1[0] + xi, p1[1] + yi, p1[2] + zi };
						const double dist0 = std::sqrt(A0[0] * A0[0] + A0[1] * A0[1] + A0[2] * A0[2]);
						const double dist1 = std::sqrt(A1[0] * A1[0] + A1[1] * A1[1] + A1[2] * A1[2]);
						const int i0 = (int) ((t0 + dist0) * c0);
						const int i1 = (int) ((t1 + dist1) * c0);
						if (i0 == i1 || !(dist1 <= 1.0 || dist0 <= 1.0)) {
							continue;
						}
						// where the particle's straight path meets the light cone of period
						// boundary (i0 + 1) tau_max: |X0 + v t| = ti - (tau0 + t), solved for t
						const float vx = float(vel[0] * ainv), vy = float(vel[1] * ainv), vz = float(vel[2] * ainv);
						const double ti = double(i0 + 1) * tmax;
						const double sq = (ti - t0) * (ti - t0);
						const double A = 1.0 - (vx * vx + vy * vy + vz * vz);
						const double B = 2.0 * ((t0 - ti) - (vx * A0[0] + vy * A0[1] + vz * A0[2]));
						const double C = sq - (A0[0] * A0[0] + A0[1] * A0[1] + A0[2] * A0[2]);
						const double t = -(B + std::sqrt(B * B - 4.0 * A * C)) / (2.0 * A);
						const double q[3] = { A0[0] + vx * t, A0[1] + vy * t, A0[2] + vz * t };
						if (q[0] * q[0] + q[1] * q[1] + q[2] * q[2] <= 1.0) {
							if (count < max_out) {
								ct_or_lc_entry& e = out[count];
								e.x = fixed31_from_double(q[0]);
								e.y = fixed31_from_double(q[1]);
								e.z = fixed31_from_double(q[2]);
								e.vx = vel[0];
								e.vy = vel[1];
								e.vz = vel[2];
								e.pix = ct_or_healpix_nest(nside, q[0], q[1], q[2]);
							}
							count++;
						}
					}
				}
			}
		}
		for (int d = 0; d < 3; d++) {
			double v = p1[d];
			v -= double(v >= 1.0);
			v += double(v < 0.0);
			X[d][i] = fixed32_from_double(v);
		}
	}
	return count;
}

int ct_or_sort_by_rung(int n, int begin, int minrung, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, int8_t* rung) {
	if (minrung == 0) {
		return 0;
	}
	int lo = begin, hi = n;
	while (lo < hi) {
		if (rung[lo] >= minrung) {
			while (lo != hi) {
				hi--;
				if (rung[hi] < minrung) {
					std::swap(x[hi], x[lo]);
					std::swap(y[hi], y[lo]);
					std::swap(z[hi], z[lo]);
					for (int d = 0; d < 3; d++) {
						std::swap(vxyz[3 * hi + d], vxyz[3 * lo + d]);
					}
					std::swap(rung[hi], rung[lo]);
					break;
				}
			}
		}
		lo++;
	}
	return hi;
}

void ct_or_direct_ewald(int n, const uint32_t* x, const uint32_t* y, const uint32_t* z, int nsink, const uint32_t* sx, const uint32_t* sy,
		const uint32_t* sz, double h, double* gx, double* gy, double* gz, double* pot, int nthreads) {
	const auto& tab = Ops7::tab();
	// Fourier part through per-vector sums over all sources: sum_j cos(2 pi h.(xi - xj)) =
	// cos(2 pi h.xi) C(h) + sin(2 pi h.xi) S(h).
	std::vector<double> Ch(CT_EWALD_NFOUR, 0.0), Sh(CT_EWALD_NFOUR, 0.0);
	for (int k = 0; k < CT_EWALD_NFOUR; k++) {
		double c = 0.0, s = 0.0;
		for (int j = 0; j < n; j++) {
			const double ph = 2.0 * M_PI * (tab.four[k][0] * fixed32_to_double(x[j]) + tab.four[k][1] * fixed32_to_double(y[j]) + tab.four[k][2] * fixed32_to_double(z[j]));
			c += std::cos(ph);
			s += std::sin(ph);
		}
		Ch[k] = c;
		Sh[k] = s;
	}
	const double hinv = 1.0 / h, h2inv = hinv * hinv, h3inv = h2inv * hinv;
	parallel_for(nsink, nthreads, [&](int i) {
		double phi = 0.0, g[3] = { 0, 0, 0 };
		for (int j = 0; j < n; j++) {
			const double dx = double(int32_t(sx[i] - x[j])) * FIXED2DOUBLE;
			const double dy = double(int32_t(sy[i] - y[j])) * FIXED2DOUBLE;
			const double dz = double(int32_t(sz[i] - z[j])) * FIXED2DOUBLE;
			const double r2 = dx * dx + dy * dy + dz * dz;
			// softened nearest image (the tree's P2P kernel, gravity.cu:331-338)
			if (r2 > h * h) {
				const double rinv = 1.0 / std::sqrt(r2);
				const double r3inv = rinv * rinv * rinv;
				g[0] -= dx * r3inv;
				g[1] -= dy * r3inv;
				g[2] -= dz * r3inv;
				phi -= rinv;
			} else {
				double f, p;
				gsoft<double>(f, p, r2, hinv, h2inv, h3inv);
				g[0] -= dx * f;
				g[1] -= dy * f;
				g[2] -= dz * f;
				phi -= p;
			}
			// smooth periodic correction: potential erf/r etc.; force = -gradient
			double pc = 0.0, gc[3] = { 0, 0, 0 };
			ewald_correction_real(dx, dy, dz, pc, gc, tab);
			phi += pc;
			g[0] -= gc[0];
			g[1] -= gc[1];
			g[2] -= gc[2];
		}
		// the self pair's softened term is excluded, as in the tree code (kick.cu:265)
		phi += double(self_phi()) * hinv;
		const double xi[3] = { fixed32_to_double(sx[i]), fixed32_to_double(sy[i]), fixed32_to_double(sz[i]) };
		for (int k = 0; k < CT_EWALD_NFOUR; k++) {
			const double hx = tab.four[k][0], hy = tab.four[k][1], hz = tab.four[k][2];
			const double h2 = hx * hx + hy * hy + hz * hz;
			const double c0 = -std::exp(-M_PI * M_PI * h2 / 4.0) / (M_PI * h2);
			const double ph = 2.0 * M_PI * (hx * xi[0] + hy * xi[1] + hz * xi[2]);
			const double cs = std::cos(ph), sn = std::sin(ph);
			phi += c0 * (cs * Ch[k] + sn * Sh[k]);
			// d/dxi of cos(ph - phj) = -2 pi h sin(ph - phj); sum_j sin(ph - phj) = sn C - cs S
			const double sd = sn * Ch[k] - cs * Sh[k];
			g[0] -= -c0 * 2.0 * M_PI * hx * sd;
			g[1] -= -c0 * 2.0 * M_PI * hy * sd;
			g[2] -= -c0 * 2.0 * M_PI * hz * sd;
		}
		gx[i] = g[0];
		gy[i] = g[1];
		gz[i] = g[2];
		pot[i] = phi;
	});
}

}
