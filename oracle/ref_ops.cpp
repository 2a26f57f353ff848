// Test-only harness: compiles the reference's own generated FMM operators
// (cosmictiger/fmm_kernels.hpp, host SIMD instantiation) into a shared library
// with plain C entry points, so that the golden-vector script can record their
// outputs.  Built by oracle/Makefile into oracle/_ref/ from the sources under the
// reference tree; nothing in the product links or loads it.
//
// The reference instantiates its host operators on simd_float / simd_double
// (8 / 4 lanes, cosmictiger/simd.hpp:31-55).  Each entry point broadcasts one
// input to every lane and returns lane 0.
//
// ewald_const's accessors are declared by the reference (cosmictiger/ewald_indices.hpp:32-41)
// and defined in its CUDA file; oracle/ref_ewald_host.h defines them over tables built by a
// restatement of ewald_const::init_gpu (src/ewald_indices.cu:30-114).
#include <cosmictiger/fmm_kernels.hpp>
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "ref_ewald_host.h"

template<class V, class S, int N>
static void load(V& v, const S* p) {
	for (int i = 0; i < N; i++) {
		v[i] = p[i];
	}
}

extern "C" {

int ref_order() {
	return ORDER;
}

int ref_greens(const float* X, float* D) {
	array<simd_float, NDIM> x;
	for (int d = 0; d < NDIM; d++) {
		x[d] = X[d];
	}
	expansion<simd_float> Ds;
	const int fl = greens_function(Ds, x);
	for (int i = 0; i < EXPANSION_SIZE; i++) {
		D[i] = Ds[i][0];
	}
	return fl;
}

int ref_ewald_greens(const float* X, float* D) {
	ref_ewald_init();
	array<simd_float, NDIM> x;
	for (int d = 0; d < NDIM; d++) {
		x[d] = X[d];
	}
	expansion<simd_float> Ds;
	const int fl = ewald_greens_function(Ds, x);
	for (int i = 0; i < EXPANSION_SIZE; i++) {
		D[i] = Ds[i][0];
	}
	return fl;
}

int ref_m2l(const float* M, const float* D, float* L, int do_phi) {
	multipole<simd_float> Ms;
	expansion<simd_float> Ds, Ls;
	for (int i = 0; i < MULTIPOLE_SIZE; i++) {
		Ms[i] = M[i];
	}
	for (int i = 0; i < EXPANSION_SIZE; i++) {
		Ds[i] = D[i];
		Ls[i] = L[i];
	}
	const int fl = M2L(Ls, Ms, Ds, do_phi != 0);
	for (int i = 0; i < EXPANSION_SIZE; i++) {
		L[i] = Ls[i][0];
	}
	return fl;
}

int ref_m2l2(const float* M, const float* D, float* L, int do_phi) {
	multipole<simd_float> Ms;
	expansion<simd_float> Ds;
	expansion2<simd_float> Ls;
	for (int i = 0; i < MULTIPOLE_SIZE; i++) {
		Ms[i] = M[i];
	}
	for (int i = 0; i < EXPANSION_SIZE; i++) {
		Ds[i] = D[i];
	}
	for (int i = 0; i < 5; i++) {
		Ls[i] = L[i];
	}
	const int fl = M2L(Ls, Ms, Ds, do_phi != 0);
	for (int i = 0; i < 5; i++) {
		L[i] = Ls[i][0];
	}
	return fl;
}

void ref_p2m(const float* X, float* M) {
	array<simd_float, NDIM> x;
	for (int d = 0; d < NDIM; d++) {
		x[d] = X[d];
	}
	const auto Ms = P2M(x);
	for (int i = 0; i < MULTIPOLE_SIZE; i++) {
		M[i] = Ms[i][0];
	}
}

void ref_m2m_d(const double* M, const double* X, double* Mout) {
	multipole<simd_double> Ms;
	array<simd_double, NDIM> x;
	for (int i = 0; i < MULTIPOLE_SIZE; i++) {
		Ms[i] = M[i];
	}
	for (int d = 0; d < NDIM; d++) {
		x[d] = X[d];
	}
	const auto Mo = M2M<simd_double>(Ms, x);
	for (int i = 0; i < MULTIPOLE_SIZE; i++) {
		Mout[i] = Mo[i][0];
	}
}

void ref_l2l(const float* L, const float* X, float* Lout, int do_phi) {
	expansion<simd_float> Ls;
	array<simd_float, NDIM> x;
	for (int i = 0; i < EXPANSION_SIZE; i++) {
		Ls[i] = L[i];
	}
	for (int d = 0; d < NDIM; d++) {
		x[d] = X[d];
	}
	const auto Lo = L2L(Ls, x, do_phi != 0);
	for (int i = 0; i < EXPANSION_SIZE; i++) {
		Lout[i] = Lo[i][0];
	}
}

void ref_l2p(const float* L, const float* X, float* Lout, int do_phi) {
	expansion<simd_float> Ls;
	array<simd_float, NDIM> x;
	for (int i = 0; i < EXPANSION_SIZE; i++) {
		Ls[i] = L[i];
	}
	for (int d = 0; d < NDIM; d++) {
		x[d] = X[d];
	}
	const auto Lo = L2P(Ls, x, do_phi != 0);
	for (int i = 0; i < 5; i++) {
		Lout[i] = Lo[i][0];
	}
}

void ref_ewald_tables(float* real_idx, float* four_idx, float* four_exp, float* D0) {
	ref_ewald_init();
	for (int i = 0; i < NREAL; i++) {
		for (int d = 0; d < NDIM; d++) {
			real_idx[NDIM * i + d] = h_real[i][d];
		}
	}
	for (int i = 0; i < NFOUR; i++) {
		for (int d = 0; d < NDIM; d++) {
			four_idx[NDIM * i + d] = h_four[i][d];
		}
		for (int j = 0; j < EXPANSION_SIZE; j++) {
			four_exp[EXPANSION_SIZE * i + j] = h_four_exp[i][j];
		}
	}
	for (int n = 0; n < (LORDER + 2) * (LORDER + 1) * LORDER / 6; n++) {
		D0[n] = h_D0[n];
	}
}

}
