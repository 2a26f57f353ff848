// Shared scaffolding for the generated FMM operator headers (fmm_p*.h):
// host/device qualifiers and type-generic fused multiply-add / sqrt.
#pragma once
#include <cmath>

#ifndef CT_HD
#ifdef __CUDACC__
#define CT_HD __host__ __device__ __forceinline__
#else
#define CT_HD inline
#endif
#endif

#ifdef __CUDACC__
#define CT_HD_FN __host__ __device__ inline
#else
#define CT_HD_FN inline
#endif

CT_HD_FN float ct_fma(float a, float b, float c) {
#ifdef __CUDA_ARCH__
	return __fmaf_rn(a, b, c);
#else
	return std::fma(a, b, c);
#endif
}
CT_HD_FN double ct_fma(double a, double b, double c) {
#ifdef __CUDA_ARCH__
	return __fma_rn(a, b, c);
#else
	return std::fma(a, b, c);
#endif
}
// Bit helpers for the Ewald image sets: population count, 1-based index of the lowest set
// bit, and a word of a six-word register array chosen without dynamic indexing.
CT_HD_FN int ct_popc(unsigned int m) {
#ifdef __CUDA_ARCH__
	return __popc(m);
#else
	return __builtin_popcount(m);
#endif
}
CT_HD_FN int ct_ffs(unsigned int m) {
#ifdef __CUDA_ARCH__
	return __ffs((int) m);
#else
	return __builtin_ffs((int) m);
#endif
}
CT_HD_FN unsigned int ct_word4(const unsigned int* a, int w) {
	return w == 0 ? a[0] : w == 1 ? a[1] : w == 2 ? a[2] : a[3];
}
CT_HD_FN float ct_sqrt(float a) {
#ifdef __CUDA_ARCH__
	return __fsqrt_rn(a);
#else
	return std::sqrt(a);
#endif
}
// 1 / sqrt(a) for a > 0, else 0: the Green's function's reciprocal distance.  On the device
// CUDA's rsqrtf (one MUFU operation, at most 2 ulp from the exact value, as the reference's
// fast-math build gets from its 1 / sqrt); on the host the correctly rounded 1 / sqrt.
CT_HD_FN float ct_rinv(float a) {
#ifdef __CUDA_ARCH__
	return a > 0.f ? rsqrtf(a) : 0.f;
#else
	return a > 0.f ? 1.f / std::sqrt(a) : 0.f;
#endif
}
CT_HD_FN double ct_rinv(double a) {
	return a > 0.0 ? 1.0 / std::sqrt(a) : 0.0;
}
CT_HD_FN double ct_sqrt(double a) {
#ifdef __CUDA_ARCH__
	return __dsqrt_rn(a);
#else
	return std::sqrt(a);
#endif
}

// Ewald sum sizes: real-space images with distance from the unit cell below 2.6 box
// lengths, and Fourier vectors with 0 < |h|^2 <= 8 (cosmictiger/ewald_indices.hpp:28-29).
#define CT_EWALD_NREAL 178
#define CT_EWALD_NFOUR 92
// The Ewald Green's function of the kick sums the real-space images within 2.3 box lengths of
// the separation, not 2.6: the terms beyond add less than the single-precision rounding of the
// sum (3,000 random separations in double: at most 2.8e-8 of an order's largest entry up to
// order 3, 3.0e-7 at orders 4-6, against single-precision errors of 8.8e-7 to 2.3e-5).  The
// CT_EWALD_NREAL_G images within that distance of the unit cell lead the image table.
#define CT_EWALD_RCUT_G 2.3
#define CT_EWALD_NREAL_G 116

CT_HD_FN float ct_exp_f(float a) {
	return expf(a);
}
CT_HD_FN double ct_exp_f(double a) {
	return exp(a);
}
template<class T>
CT_HD_FN void ct_sincos(T a, T* s, T* c) {
#ifdef __CUDA_ARCH__
	sincos(a, s, c);
#else
	*s = std::sin(a);
	*c = std::cos(a);
#endif
}

// exp(x) from its Taylor series through x^16 (used for small |x| near the origin of the
// Ewald sum, cosmictiger/math.hpp:169-206).
template<class T>
CT_HD_FN T ct_exp_series(T x) {
	// 1/k!, k = 16..0
	const double c[17] = { 4.7794773323873853e-14, 7.6471637318198164e-13, 1.1470745597729725e-11, 1.6059043836821613e-10, 2.08767569878681e-09,
			2.505210838544172e-08, 2.7557319223985888e-07, 2.7557319223985893e-06, 2.4801587301587302e-05, 0.00019841269841269841,
			0.0013888888888888889, 0.0083333333333333332, 0.041666666666666664, 0.16666666666666666, 0.5, 1.0, 1.0 };
	T w = T(c[0]);
	for (int i = 1; i < 17; i++) {
		w = ct_fma(w, x, T(c[i]));
	}
	return w;
}

// erf(x) from its Taylor series 2/sqrt(pi) sum_n (-1)^n x^(2n+1) / (n! (2n+1)), n = 0..14
// (cosmictiger/math.hpp:160-167).
template<class T>
CT_HD_FN T ct_erf_series(T x) {
	const double c[15] = { 1.1283791670955126, -0.37612638903183754, 0.11283791670955126, -0.026866170645131252, 0.0052239776254421878,
			-0.00085483270234508528, 0.00012055332981789664, -1.4925650358406251e-05, 1.6462114365889247e-06, -1.6365844691234924e-07,
			1.4807192815879218e-08, -1.2290555301717926e-09, 9.4227590646504108e-11, -6.7113668551641104e-12, 4.4632242632864774e-13 };
	const T x2 = x * x;
	T w = T(c[14]);
	for (int i = 13; i >= 0; i--) {
		w = ct_fma(w, x2, T(c[i]));
	}
	return w * x;
}

// Single-precision exp and sincos used inside the Ewald operator.  They are written here (not
// taken from the CUDA or C math library) so that host and device evaluate them with the same
// IEEE operation sequence and agree bit for bit:
//   exp:    Cody-Waite reduction y = k ln2 + r (ln2 split in two parts, |r| <= ln2/2), Taylor
//           polynomial of exp(r) through r^8 (truncation < 2e-9), exact scaling by 2^k;
//   sincos: Cody-Waite reduction by pi/2 (three-part split), Taylor polynomials of sin through
//           r^11 and cos through r^12 on |r| <= pi/4, quadrant selection.
CT_HD_FN float ct_exp_poly(float y) {
	if (y < -87.0f) {
		return 0.0f;
	}
	const float k = rintf(y * 1.44269504088896341f);
	float r = ct_fma(-k, 0.693145751953125f, y);
	r = ct_fma(-k, 1.428606765330187e-06f, r);
	float p = 1.0f / 40320.0f;
	p = ct_fma(p, r, 1.0f / 5040.0f);
	p = ct_fma(p, r, 1.0f / 720.0f);
	p = ct_fma(p, r, 1.0f / 120.0f);
	p = ct_fma(p, r, 1.0f / 24.0f);
	p = ct_fma(p, r, 1.0f / 6.0f);
	p = ct_fma(p, r, 0.5f);
	p = ct_fma(p, r, 1.0f);
	p = ct_fma(p, r, 1.0f);
	return ldexpf(p, (int) k);
}
CT_HD_FN void ct_sincos_poly(float x, float* s, float* c) {
	const float k = rintf(x * 0.636619772367581343f);
	float r = ct_fma(-k, 1.5707963705062866f, x);
	r = ct_fma(-k, -4.371138828673793e-08f, r);
	r = ct_fma(-k, -1.7763568394002505e-15f, r);
	const float r2 = r * r;
	float ps = -1.0f / 39916800.0f;
	ps = ct_fma(ps, r2, 1.0f / 362880.0f);
	ps = ct_fma(ps, r2, -1.0f / 5040.0f);
	ps = ct_fma(ps, r2, 1.0f / 120.0f);
	ps = ct_fma(ps, r2, -1.0f / 6.0f);
	const float sr = ct_fma(ps * r2, r, r);
	float pc = 1.0f / 479001600.0f;
	pc = ct_fma(pc, r2, -1.0f / 3628800.0f);
	pc = ct_fma(pc, r2, 1.0f / 40320.0f);
	pc = ct_fma(pc, r2, -1.0f / 720.0f);
	pc = ct_fma(pc, r2, 1.0f / 24.0f);
	pc = ct_fma(pc, r2, -0.5f);
	const float cr = ct_fma(pc, r2, 1.0f);
	const int q = ((int) k) & 3;
	const float S[4] = { sr, cr, -sr, -cr };
	const float C[4] = { cr, -sr, -cr, sr };
	*s = S[q];
	*c = C[q];
}
CT_HD_FN double ct_exp_poly(double y) {
	return exp(y);
}
CT_HD_FN void ct_sincos_poly(double x, double* s, double* c) {
#ifdef __CUDA_ARCH__
	sincos(x, s, c);
#else
	*s = std::sin(x);
	*c = std::cos(x);
#endif
}

// erfc(x) and exp(-x^2) by Abramowitz & Stegun 7.1.26 (|error| <= 1.5e-7), the form the
// reference uses on the device (cosmictiger/math.hpp:56-71).  On the device, in single
// precision, the reciprocal and the exponential are CUDA's fast intrinsics (__fdividef,
// __expf: a few ulp, far below the formula's own error), as the reference's --use_fast_math
// build makes them; the host keeps the correctly rounded division and its own exponential.
template<class T>
CT_HD_FN void ct_erfcexp(T x, T* ec, T* ex) {
	const T p = T(0.3275911), a1 = T(0.254829592), a2 = T(-0.284496736), a3 = T(1.421413741), a4 = T(-1.453152027), a5 = T(1.061405429);
#ifdef __CUDA_ARCH__
	T t;
	if constexpr (sizeof(T) == sizeof(float)) {
		t = __fdividef(1.0f, ct_fma(p, x, T(1)));
		*ex = __expf(-x * x);
	} else {
		t = T(1) / ct_fma(p, x, T(1));
		*ex = ct_exp_poly(-x * x);
	}
#else
	const T t = T(1) / ct_fma(p, x, T(1));
	*ex = ct_exp_poly(-x * x);
#endif
	T s = ct_fma(a5, t, a4);
	s = ct_fma(s, t, a3);
	s = ct_fma(s, t, a2);
	s = ct_fma(s, t, a1);
	*ec = s * t * *ex;
}

// distance and its reciprocal from the squared distance (> 0): on the device in single
// precision one MUFU reciprocal square root and a product, elsewhere the correctly rounded
// square root and division
template<class T>
CT_HD_FN void ct_dist(T r2, T* r, T* rinv) {
#ifdef __CUDA_ARCH__
	if constexpr (sizeof(T) == sizeof(float)) {
		*rinv = rsqrtf(r2);
		*r = r2 * *rinv;
		return;
	}
#endif
	*r = ct_sqrt(r2);
	*rinv = T(1) / *r;
}
