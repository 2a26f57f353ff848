// Test infrastructure only (oracle build).  The reference's Ewald tables on the host: its
// ewald_const accessors (declared in cosmictiger/ewald_indices.hpp:32-41, defined in its CUDA
// file src/ewald_indices.cu) defined over tables built by ref_ewald_init(), a restatement of
// ewald_const::init_gpu (src/ewald_indices.cu:30-114) in the same float/double mix.  Included
// by exactly one translation unit of each binary that needs them (oracle/ref_ops.cpp,
// oracle/kick_probe.cpp); the accessors build the tables on first use.
#pragma once
#include <cosmictiger/ewald_indices.hpp>
#include <cosmictiger/fmm_kernels.hpp>

#include <algorithm>
#include <cmath>
#include <cstdio>

static array<array<float, NDIM>, NREAL> h_real;
static array<array<float, NDIM>, NFOUR> h_four;
static array<tensor_trless_sym<float, LORDER>, NFOUR> h_four_exp;
static tensor_sym<float, LORDER> h_D0;
static bool h_init = false;

static void ref_ewald_init() {
	if (h_init) {
		return;
	}
	int count = 0;
	int n2max = 12;
	int nmax = int(std::sqrt(double(n2max))) + 1;
	for (int i = -nmax; i <= nmax; i++) {
		for (int j = -nmax; j <= nmax; j++) {
			for (int k = -nmax; k <= nmax; k++) {
				const int i2 = i * i + j * j + k * k;
				const double x = std::max(std::abs(i) - 0.5, 0.0);
				const double y = std::max(std::abs(j) - 0.5, 0.0);
				const double z = std::max(std::abs(k) - 0.5, 0.0);
				const double d = std::sqrt(x * x + y * y + z * z);
				if (d < EWALD_REAL_CUTOFF && i2 > 0) {
					h_real[count][0] = i;
					h_real[count][1] = j;
					h_real[count][2] = k;
					count++;
				}
			}
		}
	}
	if (count != NREAL) {
		fprintf(stderr, "ref_ewald_init: %d real vectors, expected %d\n", count, NREAL);
	}
	auto by_norm_desc = [](const array<float, NDIM>& a, const array<float, NDIM>& b) {
		return a[0] * a[0] + a[1] * a[1] + a[2] * a[2] > b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
	};
	std::stable_sort(h_real.begin(), h_real.end(), by_norm_desc);
	count = 0;
	n2max = 8;
	nmax = int(std::sqrt(double(n2max))) + 1;
	for (int i = -nmax; i <= nmax; i++) {
		for (int j = -nmax; j <= nmax; j++) {
			for (int k = -nmax; k <= nmax; k++) {
				const int h2 = i * i + j * j + k * k;
				if (h2 <= n2max && h2 > 0) {
					h_four[count][0] = i;
					h_four[count][1] = j;
					h_four[count][2] = k;
					count++;
				}
			}
		}
	}
	std::stable_sort(h_four.begin(), h_four.end(), by_norm_desc);
	for (int i = 0; i < NFOUR; i++) {
		array<float, NDIM> h = h_four[i];
		auto D0 = vector_to_sym_tensor<float, LORDER>(h);
		const float h2 = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
		const float c0 = -1.0 / h2 * std::exp(-M_PI * M_PI * h2 / 4.0) / M_PI;
		const int signs[4] = { 1, -1, -1, 1 };
		array<int, NDIM> n;
		for (n[0] = 0; n[0] < LORDER; n[0]++) {
			for (n[1] = 0; n[1] < LORDER - n[0]; n[1]++) {
				for (n[2] = 0; n[2] < LORDER - n[0] - n[1]; n[2]++) {
					const int n0 = n[0] + n[1] + n[2];
					D0(n) *= (signs[n0 % 4] * std::pow(2.0 * M_PI * SCALE_FACTOR_INV1, n0) * c0) * SCALE_FACTOR_INV1;
				}
			}
		}
		h_four_exp[i] = D0.detraceD();
	}
	for (int n = 0; n < (LORDER + 2) * (LORDER + 1) * LORDER / 6; n++) {
		h_D0[n] = 0.0;
	}
	constexpr double alpha = 2.0;
	for (int n = 0; n < LORDER; n += 2) {
		for (int m = 0; m < LORDER - n; m += 2) {
			for (int l = 0; l < LORDER - n - m; l += 2) {
				h_D0(n, m, l) = std::pow(SCALE_FACTOR_INV1, n + m + l + 1) * std::pow(-2.0, (n + m + l) / 2 + 1) / ((n + m + l + 1.0) * std::sqrt(M_PI))
						* std::pow(alpha, n + m + l + 1) * double_factorial(n - 1) * double_factorial(m - 1) * double_factorial(l - 1);
			}
		}
	}
	h_init = true;
}

int ewald_const::nfour() {
	return NFOUR;
}
int ewald_const::nreal() {
	return NREAL;
}
const tensor_sym<float, LORDER> ewald_const::D0() {
	ref_ewald_init();
	return h_D0;
}
const array<float, NDIM>& ewald_const::real_index(int i) {
	ref_ewald_init();
	return h_real[i];
}
const array<float, NDIM>& ewald_const::four_index(int i) {
	ref_ewald_init();
	return h_four[i];
}
const tensor_trless_sym<float, LORDER>& ewald_const::four_expansion(int i) {
	ref_ewald_init();
	return h_four_exp[i];
}
