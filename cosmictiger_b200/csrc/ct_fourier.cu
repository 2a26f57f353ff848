// Fourier-space work around the gravity step: the reference's initial-condition generator
// (Zel'dovich and 2LPT displacements of a lattice, src/initialize.cpp:261-355,436-898) and its
// matter power spectrum (src/power.cpp:33-77, src/power.cu:32-85, src/fft.cpp:172-330).
//
// Both follow the reference's conventions: grids of Nfour^3 points in x-major order, the
// half-complex layout N x N x (N/2 + 1) of a real-to-complex transform along z, the 6-point
// quintic-spline cloud kernel (CLOUD_MIN -2 .. CLOUD_MAX 3, fft.hpp:113-134) for mass
// assignment and interpolation with its window deconvolved in k-space, and the random field
// drawn row by row (one generator per (x, y) row of k-space) from GSL's "taus" generator
// (L'Ecuyer 1996), so that a seed gives the reference's field.  The transforms are cuFFT's
// (single precision, out of place); the reference's normalisations are applied around them.
#include "ct_internal.cuh"

#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace ct {
namespace {

constexpr int FT_TPB = 256;
constexpr int CLOUD_MIN = -2;
constexpr int CLOUD_MAX = 3;

// ---------------------------------------------------------------- the cloud kernel
// Quintic spline of support 3 (fft.hpp:116-131), with the reference's mixed float / double
// arithmetic.
__host__ __device__ inline float cloud_weight(float x) {
	x = fabsf(x);
	const float x2 = x * x;
	const float x3 = x * x2;
	const float x4 = x2 * x2;
	const float x5 = x3 * x2;
	if (x > 3.0f) {
		return 0.0f;
	} else if (x < 1.0f) {
		return (33.0f - 30.0 * x2 + 15.0f * x4 - 5.0f * x5) / 60.0f;
	} else if (x < 2.0f) {
		return (51.0 + 75.0 * x - 210 * x2 + 150 * x3 - 45 * x4 + 5 * x5) / 120.0;
	} else {
		return (243.0 - 405.0 * x + 270 * x2 - 90 * x3 + 15 * x4 - x5) / 120.0;
	}
}

__host__ __device__ inline double sinc(double x) {
	return x == 0.0 ? 1.0 : sin(x) / x;
}

// Inverse of the kernel's window at wavenumber kh (grid units): 1 / sinc(kh / 2)^6.
__host__ __device__ inline double cloud_filter(double kh) {
	const double s = sinc(0.5 * kh);
	const double s3 = s * (s * s);
	return 1.0 / (s3 * s3);
}

__device__ __forceinline__ int wrap(int i, int n) {
	i %= n;
	return i < 0 ? i + n : i;
}

// ---------------------------------------------------------------- GSL "taus"
// The maximally equidistributed combined Tausworthe generator of L'Ecuyer (Math. Comp. 65,
// 1996, 203-213): three 32-bit components, output their XOR.  Seeding as GSL's gsl_rng_taus
// does: seed 0 is taken as 1, the components are successive values of the LCG
// x -> 69069 x mod 2^32 from the seed, and six outputs are discarded.  uniform_pos divides an
// output by 2^32 and skips zero.
struct Taus {
	uint32_t s1, s2, s3;

	__host__ __device__ uint32_t next() {
		s1 = ((s1 & 4294967294u) << 12) ^ (((s1 << 13) ^ s1) >> 19);
		s2 = ((s2 & 4294967288u) << 4) ^ (((s2 << 2) ^ s2) >> 25);
		s3 = ((s3 & 4294967280u) << 17) ^ (((s3 << 3) ^ s3) >> 11);
		return s1 ^ s2 ^ s3;
	}
	__host__ __device__ void seed(uint32_t s) {
		if (s == 0) {
			s = 1;
		}
		s1 = 69069u * s;
		s2 = 69069u * s1;
		s3 = 69069u * s2;
		for (int i = 0; i < 6; i++) {
			next();
		}
	}
	__host__ __device__ double uniform_pos() {
		uint32_t v;
		do {
			v = next();
		} while (v == 0);
		return v / 4294967296.0;
	}
};

// ---------------------------------------------------------------- power table
// P(k) in Mpc^3 at k_i = exp(logkmin + i dlogk): cubic interpolation of log P in log k over
// four table points (power_spectrum_function::operator(), initialize.cpp:110-139).  Indices
// are clamped to the table (the reference reads past it when k is out of range; the host
// checks the range before generating).
struct PowerTable {
	const float* P;
	int n;
	float logkmin, dlogk;

	__host__ __device__ float operator()(float k) const {
		const float logk = logf(k);
		const float k0 = (logk - logkmin) / dlogk;
		int i0 = int(k0) - 1;
		i0 = i0 < 0 ? 0 : (i0 > n - 4 ? n - 4 : i0);
		const int i1 = i0 + 1, i2 = i0 + 2, i3 = i0 + 3;
		const float x = k0 - i1;
		const float y0 = logf(P[i0]);
		const float y1 = logf(P[i1]);
		const float y2 = logf(P[i2]);
		const float y3 = logf(P[i3]);
		const float k1 = (y2 - y0) * 0.5;
		const float k2 = (y3 - y1) * 0.5;
		const float a = y1;
		const float b = k1;
		const float c = -2 * k1 - k2 - 3 * y1 + 3 * y2;
		const float d = k1 + k2 + 2 * y1 - 2 * y2;
		return expf(a + b * x + c * x * x + d * x * x * x);
	}
};

// ---------------------------------------------------------------- k-space fields
// The Gaussian field for the displacement derivatives dim1, dim2 (3: none):
// Y(k) = n(k) sqrt(P(|k|)) box^-1.5 N^3 (-i k_dim1)(-i k_dim2) / k^2, n a unit complex normal,
// times the cloud kernel's inverse window (twolpt_generate, initialize.cpp:436-540).  Every
// (x, y) row of k-space has its own generator (seed (I0 N + I1) 1234 + 42, eight draws
// discarded) for kz > 0; the kz = 0 element takes the generator of the mirrored row and its
// conjugate on the lower half, which makes the kz = 0 plane Hermitian.  The seeds do not depend
// on dim1, dim2, so every field of one call draws the same numbers: the amplitude
// n(k) sqrt(P) box^-1.5 N^3 is made once (row generators, then one thread per mode) and each
// field is an elementwise pass over it.

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
	return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 filtered(float2 v, float kx, float ky, float kz, float box_size, int N) {
	const float fx = (float) cloud_filter(kx * box_size / N);
	const float fy = (float) cloud_filter(ky * box_size / N);
	const float fz = (float) cloud_filter(kz * box_size / N);
	v = make_float2(v.x * fx, v.y * fx);
	v = make_float2(v.x * fy, v.y * fy);
	return make_float2(v.x * fz, v.y * fz);
}

__device__ __forceinline__ float wavenumber(int I, int N, float box_size) {
	const int i = I < N / 2 ? I : I - N;
	return 2.f * (float) M_PI / box_size * float(i);
}

// The uniforms (x, y) of every mode, as floats, row by row (the generators are sequential).
__global__ void __launch_bounds__(FT_TPB) k_ic_uniforms(int N, float2* __restrict__ U) {
	const int NZ = N / 2 + 1;
	const int64_t rows = (int64_t) N * N;
	for (int64_t row = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; row < rows; row += (int64_t) gridDim.x * blockDim.x) {
		const int I0 = (int) (row / N), I1 = (int) (row % N);
		float2* out = U + row * NZ;
		Taus g;
		g.seed((uint32_t) (((int64_t) I0 * N + I1) * 1234 + 42));
		for (int l = 0; l < 8; l++) {
			g.uniform_pos();
		}
		for (int I2 = 1; I2 < NZ; I2++) {
			const double x = g.uniform_pos();
			const double y = g.uniform_pos();
			out[I2] = make_float2((float) x, (float) y);
		}
		// kz = 0: the mirrored row's generator (no draw for the k = 0 mode)
		const int J0 = I0 > N / 2 ? N - I0 : I0;
		const int J1 = I1 > N / 2 ? N - I1 : I1;
		g.seed((uint32_t) (((int64_t) J0 * N + J1) * 1234 + 42));
		for (int l = 0; l < 8; l++) {
			g.uniform_pos();
		}
		float2 u = make_float2(1.f, 0.f);
		if (I0 != 0 || I1 != 0) {
			const double x = g.uniform_pos();
			const double y = g.uniform_pos();
			u = make_float2((float) x, (float) y);
		}
		out[0] = u;
	}
}

// In place: uniforms -> amplitude n(k) sqrt(P(|k|)) factor (0 at k = 0).
__global__ void __launch_bounds__(FT_TPB) k_ic_amplitude(int N, float box_size, float factor, PowerTable power, float2* __restrict__ U) {
	const int NZ = N / 2 + 1;
	const int64_t total = (int64_t) N * N * NZ;
	for (int64_t e = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; e < total; e += (int64_t) gridDim.x * blockDim.x) {
		const int I2 = (int) (e % NZ);
		const int64_t row = e / NZ;
		const int I0 = (int) (row / N), I1 = (int) (row % N);
		if (I0 == 0 && I1 == 0 && I2 == 0) {
			U[e] = make_float2(0.f, 0.f);
			continue;
		}
		const float kx = wavenumber(I0, N, box_size), ky = wavenumber(I1, N, box_size), kz = wavenumber(I2, N, box_size);
		const float K0 = sqrtf(kx * kx + ky * ky + kz * kz);
		const float2 u = U[e];
		const float ang = 2.f * float(M_PI) * u.y;
		const float mag = sqrtf(-logf(fabsf(u.x)));
		float2 r = make_float2(cosf(ang) * mag, sinf(ang) * mag);
		const float sp = sqrtf(power(K0));
		r = make_float2(r.x * sp, r.y * sp);
		U[e] = make_float2(r.x * factor, r.y * factor);
	}
}

// One field: Y = A (-i k_dim1)(-i k_dim2) / k^2, conjugated (times the parity sign) on the lower
// half of the kz = 0 plane, times the inverse window.
__global__ void __launch_bounds__(FT_TPB) k_ic_field(int N, float box_size, int dim1, int dim2, const float2* __restrict__ A, cufftComplex* __restrict__ Y) {
	const int NZ = N / 2 + 1;
	const int64_t total = (int64_t) N * N * NZ;
	float sgn = 1.f;
	sgn *= dim1 != 3 ? -1.f : 1.f;
	sgn *= dim2 != 3 ? -1.f : 1.f;
	for (int64_t e = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; e < total; e += (int64_t) gridDim.x * blockDim.x) {
		const int I2 = (int) (e % NZ);
		const int64_t row = e / NZ;
		const int I0 = (int) (row / N), I1 = (int) (row % N);
		const float kx = wavenumber(I0, N, box_size), ky = wavenumber(I1, N, box_size), kz = wavenumber(I2, N, box_size);
		float2 v = make_float2(0.f, 0.f);
		if (I2 > 0 || I0 != 0 || I1 != 0) {
			const float k2 = kx * kx + ky * ky + kz * kz;
			const float2 K[4] = { make_float2(0.f, -kx), make_float2(0.f, -ky), make_float2(0.f, -kz), make_float2(1.f, 0.f) };
			v = cmul(A[e], K[dim1]);
			v = cmul(v, K[dim2]);
			v = make_float2(v.x / k2, v.y / k2);
			if (I2 == 0 && (I0 > N / 2 || (I0 == 0 && I1 > N / 2))) {
				v = make_float2(v.x * sgn, -v.y * sgn);
			}
		}
		v = filtered(v, kx, ky, kz, box_size, N);
		Y[e] = make_cuComplex(v.x, v.y);
	}
}

// Second-order displacement field of axis dim from the transformed 2LPT source:
// Y = -i k_dim delta2(k) / k^2 times the inverse window, 0 at k = 0 (twolpt_correction2,
// initialize.cpp:384-434).
__global__ void __launch_bounds__(FT_TPB) k_ic_correction(const cufftComplex* __restrict__ src, cufftComplex* __restrict__ Y, int N, float box_size, int dim) {
	const int NZ = N / 2 + 1;
	const int64_t total = (int64_t) N * N * NZ;
	for (int64_t e = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; e < total; e += (int64_t) gridDim.x * blockDim.x) {
		const int I2 = (int) (e % NZ);
		const int64_t row = e / NZ;
		const int I0 = (int) (row / N), I1 = (int) (row % N);
		const int i = I0 < N / 2 ? I0 : I0 - N;
		const int j = I1 < N / 2 ? I1 : I1 - N;
		const int k = I2 < N / 2 ? I2 : I2 - N;
		float2 v = make_float2(0.f, 0.f);
		if (i * i + j * j + k * k > 0) {
			const float kx = 2.f * (float) M_PI / box_size * float(i);
			const float ky = 2.f * (float) M_PI / box_size * float(j);
			const float kz = 2.f * (float) M_PI / box_size * float(k);
			const float k2 = kx * kx + ky * ky + kz * kz;
			const float K[3] = { kx, ky, kz };
			const cufftComplex s = src[e];
			// -i K y / k^2
			v = make_float2(K[dim] * s.y, -K[dim] * s.x);
			v = make_float2(v.x / k2, v.y / k2);
			v = filtered(v, kx, ky, kz, box_size, N);
		}
		Y[e] = make_cuComplex(v.x, v.y);
	}
}

// ---------------------------------------------------------------- real space
// The lattice (init_X0, initialize.cpp:650-798): particle (I0 N + I1) N + I2 at I / N, at rest,
// rung 0.
__global__ void __launch_bounds__(FT_TPB) k_ic_lattice(int N, uint32_t* __restrict__ x, uint32_t* __restrict__ y, uint32_t* __restrict__ z,
		float* __restrict__ v0, float* __restrict__ v1, float* __restrict__ v2, int8_t* __restrict__ rung) {
	const int64_t n = (int64_t) N * N * N;
	const double Ninv = 1.0 / N;
	for (int64_t p = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; p < n; p += (int64_t) gridDim.x * blockDim.x) {
		const int I2 = (int) (p % N);
		const int I1 = (int) ((p / N) % N);
		const int I0 = (int) (p / ((int64_t) N * N));
		x[p] = fixed_from_double(I0 * Ninv);
		y[p] = fixed_from_double(I1 * Ninv);
		z[p] = fixed_from_double(I2 * Ninv);
		v0[p] = v1[p] = v2[p] = 0.f;
		rung[p] = 0;
	}
}

// Displacement of axis dim (zeldovich_end, initialize.cpp:800-868): the field interpolated
// with the cloud kernel at each particle's lattice point, dx = -D field / box; the position
// moves by dx (periodic) and the velocity by prefac dx.  Particle (I0 N + I1) N + I2 sits at
// lattice point I, and the kernel's 6^3 weights there are products of per-axis weights that
// depend only on I0, I1, I2, so the 216-term sum is taken as three 6-term passes over the grid
// (double precision, as the reference accumulates): x and y into double grids, z fused with
// the update.  The largest dx in units of the mean spacing goes to dxmax (float bits: a
// positive float orders like its bits).
__device__ __forceinline__ void lattice_stencil(int I, int N, int& i1, double w[6]) {
	const double x0 = fixed_to_double(fixed_from_double(I * (1.0 / N)));
	i1 = (int) (x0 * N);
	const double t = x0 * N - i1;
#pragma unroll
	for (int j = 0; j < 6; j++) {
		w[j] = cloud_weight((float) (-(j + CLOUD_MIN) + t));
	}
}

// One pass along axis 0 (stride N^2) or 1 (stride N).
template<class Tin>
__global__ void __launch_bounds__(FT_TPB) k_ic_smooth(int N, int axis, const Tin* __restrict__ in, double* __restrict__ out) {
	const int64_t n = (int64_t) N * N * N;
	const int64_t stride = axis == 0 ? (int64_t) N * N : N;
	for (int64_t e = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; e < n; e += (int64_t) gridDim.x * blockDim.x) {
		const int I = axis == 0 ? (int) (e / ((int64_t) N * N)) : (int) ((e / N) % N);
		int i1;
		double w[6];
		lattice_stencil(I, N, i1, w);
		const int64_t base = e - (int64_t) I * stride;
		double acc = 0.0;
#pragma unroll
		for (int j = 0; j < 6; j++) {
			acc += w[j] * (double) in[base + (int64_t) wrap(i1 + j + CLOUD_MIN, N) * stride];
		}
		out[e] = acc;
	}
}

// The pass along z, scaled by the inverse transform's normalisation, and the update.
__global__ void __launch_bounds__(FT_TPB) k_ic_displace(int N, const double* __restrict__ B, double scale, int dim, float D, float prefac,
		double box_size_inv, uint32_t* __restrict__ X, float* __restrict__ V, unsigned int* dxmax) {
	const int64_t n = (int64_t) N * N * N;
	float mymax = 0.f;
	for (int64_t p = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; p < n; p += (int64_t) gridDim.x * blockDim.x) {
		const int I2 = (int) (p % N);
		int i1;
		double w[6];
		lattice_stencil(I2, N, i1, w);
		const int64_t base = p - I2;
		double dx = 0.0;
#pragma unroll
		for (int j = 0; j < 6; j++) {
			dx += w[j] * B[base + wrap(i1 + j + CLOUD_MIN, N)];
		}
		dx *= scale;
		dx *= -D * box_size_inv;
		double x = fixed_to_double(X[p]) + dx;
		if (x >= 1.0) {
			x -= 1.0;
		} else if (x < 0.0) {
			x += 1.0;
		}
		X[p] = fixed_from_double(x);
		V[p] += prefac * dx;
		mymax = fmaxf(mymax, (float) (dx * N));
	}
	for (int o = 16; o; o >>= 1) {
		mymax = fmaxf(mymax, __shfl_xor_sync(0xffffffffu, mymax, o));
	}
	if ((threadIdx.x & 31) == 0 && mymax > 0.f) {
		atomicMax(dxmax, __float_as_uint(mymax));
	}
}

// The 2LPT source (twolpt_phase, initialize.cpp:565-589): phases 0..8 bring the second
// derivatives (yy, zz, xx, zz, xx, yy, xy, xz, yz); an even phase up to 6 keeps its field, an
// odd one adds the product with the kept field, and phases 7 and 8 subtract their squares:
// delta2 = p_yy p_zz + p_xx p_zz + p_xx p_yy - p_xz^2 - p_yz^2 (the reference keeps p_xy at
// phase 6 without using it, so -p_xy^2 is not part of its source; reproduced as is).
__global__ void __launch_bounds__(FT_TPB) k_twolpt_phase(int64_t n, int phase, const float* __restrict__ R, float scale, float* __restrict__ part,
		float* __restrict__ delta2) {
	for (int64_t p = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; p < n; p += (int64_t) gridDim.x * blockDim.x) {
		const float r = R[p] * scale;
		if (phase > 6) {
			delta2[p] -= r * r;
		} else if (phase % 2 == 0) {
			part[p] = r;
		} else {
			delta2[p] += part[p] * r;
		}
	}
}

__global__ void k_fill(int64_t n, float* __restrict__ a, float v) {
	for (int64_t p = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; p < n; p += (int64_t) gridDim.x * blockDim.x) {
		a[p] = v;
	}
}

// ---------------------------------------------------------------- power spectrum
// Mass assignment with the cloud kernel on the N^3 grid after folding the box M times
// (accumulate_density_kernel, power.cu:32-61): x -> frac(M x), 216 weights per particle.
__global__ void __launch_bounds__(FT_TPB) k_density(int64_t n, const uint32_t* __restrict__ X, const uint32_t* __restrict__ Yp, const uint32_t* __restrict__ Z,
		int M, int N, float* __restrict__ rho) {
	for (int64_t p = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; p < n; p += (int64_t) gridDim.x * blockDim.x) {
		const float x = fmodf(M * (float(X[p]) * (1.f / 4294967296.f)), 1.0f);
		const float y = fmodf(M * (float(Yp[p]) * (1.f / 4294967296.f)), 1.0f);
		const float z = fmodf(M * (float(Z[p]) * (1.f / 4294967296.f)), 1.0f);
		const int j = (int) (x * N), k = (int) (y * N), l = (int) (z * N);
		const float x0 = x * N - j, y0 = y * N - k, z0 = z * N - l;
		float wy[6], wz[6];
		int cy[6], cz[6];
#pragma unroll
		for (int q = 0; q < 6; q++) {
			wy[q] = cloud_weight(y0 - (q + CLOUD_MIN));
			wz[q] = cloud_weight(z0 - (q + CLOUD_MIN));
			cy[q] = wrap(k + q + CLOUD_MIN, N);
			cz[q] = wrap(l + q + CLOUD_MIN, N);
		}
		for (int a = 0; a < 6; a++) {
			const float wx = cloud_weight(x0 - (a + CLOUD_MIN));
			const int64_t ox = (int64_t) wrap(j + a + CLOUD_MIN, N) * N;
#pragma unroll
			for (int b = 0; b < 6; b++) {
				const int64_t oy = (ox + cy[b]) * N;
				const float wxy = wx * wy[b];
#pragma unroll
				for (int c = 0; c < 6; c++) {
					atomicAdd(rho + oy + cz[c], wxy * wz[c]);
				}
			}
		}
	}
}

// Bin of |k| (grid units) among the log-spaced edges (search_kbins, fft.cpp:219-237): -1 below
// 0 or at / above the last edge.
__device__ __forceinline__ int k_bin(const float* kb, int nb, double k) {
	if (k < 0.0 || k >= kb[nb]) {
		return -1;
	}
	int lo = 0, hi = nb;
	while (hi - lo > 1) {
		const int mid = (lo + hi) / 2;
		if (k >= kb[mid]) {
			lo = mid;
		} else {
			hi = mid;
		}
	}
	return lo;
}

constexpr int MAX_BINS = 1024;

// Pass 1 (power_spectrum_compute, fft.cpp:240-304): each mode of the half-complex box,
// deconvolved by the kernel's window (in place), adds |Y|^2, 1 and |k| to its bin.
// Pass 2 (power_spectrum_compute2, :306-360): the mode is multiplied further by
// (sinc(pi i/N) sinc(pi j/N) sinc(pi k/N))^-3 and adds (|Y|^2 - P_bin)^2 to its bin.
__global__ void __launch_bounds__(FT_TPB) k_power_bins(cufftComplex* __restrict__ Y, int N, const float* __restrict__ kb, int nb, int pass,
		const double* __restrict__ pmean, double* __restrict__ out) {
	__shared__ double s_p[MAX_BINS], s_c[MAX_BINS], s_k[MAX_BINS];
	for (int b = threadIdx.x; b < nb; b += blockDim.x) {
		s_p[b] = s_c[b] = s_k[b] = 0.0;
	}
	__syncthreads();
	const int NZ = N / 2 + 1;
	const int64_t total = (int64_t) N * N * NZ;
	for (int64_t e = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; e < total; e += (int64_t) gridDim.x * blockDim.x) {
		const int I2 = (int) (e % NZ);
		const int64_t row = e / NZ;
		const int I0 = (int) (row / N), I1 = (int) (row % N);
		const int64_t i = I0 < N / 2 ? I0 : I0 - N;
		const int64_t j = I1 < N / 2 ? I1 : I1 - N;
		const int64_t k = I2 < N / 2 ? I2 : I2 - N;
		double c0;
		if (pass == 1) {
			c0 = cloud_filter(2.0 * M_PI * i / N) * cloud_filter(2.0 * M_PI * j / N) * cloud_filter(2.0 * M_PI * k / N);
		} else {
			c0 = pow(1.0 / (sinc(M_PI * i / N) * sinc(M_PI * j / N) * sinc(M_PI * k / N)), 3);
		}
		cufftComplex y = Y[e];
		y.x *= c0;
		y.y *= c0;
		Y[e] = y;
		const double kk = sqrt((double) (i * i + j * j + k * k));
		if (kk > 0) {
			const int bin = k_bin(kb, nb, kk);
			if (bin >= 0) {
				const float pwr = y.x * y.x + y.y * y.y;
				if (pass == 1) {
					atomicAdd(&s_p[bin], (double) pwr);
					atomicAdd(&s_c[bin], 1.0);
					atomicAdd(&s_k[bin], kk);
				} else {
					const double d = (double) (pwr - (float) pmean[bin]);
					atomicAdd(&s_p[bin], d * d);
				}
			}
		}
	}
	__syncthreads();
	for (int b = threadIdx.x; b < nb; b += blockDim.x) {
		if (s_p[b] != 0.0) {
			atomicAdd(&out[b], s_p[b]);
		}
		if (pass == 1 && s_c[b] != 0.0) {
			atomicAdd(&out[nb + b], s_c[b]);
			atomicAdd(&out[2 * nb + b], s_k[b]);
		}
	}
}

}  // namespace
}  // namespace ct

namespace ct {
namespace {

int ft_grid(const Ctx* c, int64_t n) {
	return (int) std::max<int64_t>(1, std::min<int64_t>((n + FT_TPB - 1) / FT_TPB, (int64_t) c->nsm * 8));
}

ct_status fft_check(Ctx* c, cufftResult r, const char* what) {
	if (r != CUFFT_SUCCESS) {
		return fail(c, r == CUFFT_ALLOC_FAILED ? CT_ERR_MEMORY : CT_ERR_CUDA, std::string(what) + ": cuFFT error " + std::to_string((int) r));
	}
	return CT_OK;
}

// Device buffers and cuFFT plans of one call, released on every return path.
struct FtScope {
	Ctx* c;
	std::vector<std::pair<void*, size_t>> bufs;
	cufftHandle plans[2] = { 0, 0 };
	bool have[2] = { false, false };

	explicit FtScope(Ctx* c_) : c(c_) {
	}
	~FtScope() {
		cudaStreamSynchronize(c->stream);
		for (int i = 0; i < 2; i++) {
			if (have[i]) {
				cufftDestroy(plans[i]);
			}
		}
		for (auto& b : bufs) {
			dfree(c, b.first, b.second);
		}
	}
	template<class T>
	ct_status alloc(T** p, size_t count, const char* what) {
		CT_TRY(dalloc(c, (void**) p, sizeof(T) * count, what));
		bufs.push_back({ (void*) *p, sizeof(T) * count });
		return CT_OK;
	}
	ct_status plan(int which, int N, cufftType type) {
		CT_TRY(fft_check(c, cufftPlan3d(&plans[which], N, N, N, type), "cufftPlan3d"));
		have[which] = true;
		return fft_check(c, cufftSetStream(plans[which], c->stream), "cufftSetStream");
	}
};

// cosmos_growth_factor (src/cosmology.cpp:80-87): the linear growth factor's fitting formula.
double growth_factor(double omega_m, float a) {
	const double omega_l = 1.f - omega_m;
	const double a3 = a * (a * a);
	const double deninv = 1.f / (omega_m + a3 * omega_l);
	const double Om = omega_m * deninv;
	const double Ol = a3 * omega_l * deninv;
	return a * 2.5 * Om / (pow(Om, 4.f / 7.f) - Ol + (1.f + 0.5f * Om) * (1.f + 0.014285714f * Ol));
}

// sigma8 normalisation of the table (power_spectrum_function::normalize and
// sigma8_integrand, initialize.cpp:141-172): Simpson's rule over 8192 log-k intervals of the
// top-hat variance at R = 8 / h Mpc, in float; the table is scaled in place and the factor
// returned.
float sigma8_normalize(PowerTable& t, std::vector<float>& P, float logkmax_table, double hubble, double sigma8) {
	auto integrand = [&](float x) -> float {
		const float R = 8 / (float) hubble;
		const float c0 = float(9) / (2. * float(M_PI) * float(M_PI)) / powf(R, 6);
		const float k = std::exp(x);
		const float p = t(k);
		const float tmp = (std::sin(k * R) - k * R * std::cos(k * R));
		return c0 * p * tmp * tmp * std::pow(k, -3);
	};
	const int N = 8 * 1024;
	float sum = 0.0;
	const float logkmax = logkmax_table - 2.5 * t.dlogk;
	const float logkmin = t.logkmin + 1.5 * t.dlogk;
	const float dlogk = (logkmax - logkmin) / N;
	sum = (1.0 / 3.0) * (integrand(logkmax) + integrand(logkmin)) * dlogk;
	for (int i = 1; i < N; i += 2) {
		const float logk = logkmin + i * dlogk;
		sum += (4.0 / 3.0) * integrand(logk) * dlogk;
	}
	for (int i = 2; i < N; i += 2) {
		const float logk = logkmin + i * dlogk;
		sum += (2.0 / 3.0) * integrand(logk) * dlogk;
	}
	sum = (sigma8 * sigma8) / sum;
	for (auto& q : P) {
		q *= sum;
	}
	return sum;
}

}  // namespace
}  // namespace ct

using namespace ct;

extern "C" ct_status ct_initialize(ct_ctx* ctx, int box_id, const ct_ic_params* p, ct_ic_return* ret) {
	Ctx* c = (Ctx*) ctx;
	if (!c || box_id < 0 || box_id >= (int) c->boxes.size() || !c->boxes[box_id] || !p) {
		return fail(c, CT_ERR_ARG, "ct_initialize: bad arguments");
	}
	Box* b = c->boxes[box_id];
	const int N = p->nfour;
	if (N < 4 || N > 1024 || N % 2 != 0) {
		// (cuFFT's 3-D plans take 32-bit sizes)
		return fail(c, CT_ERR_ARG, "ct_initialize: nfour must be even, 4 .. 1024");
	}
	const int64_t n = (int64_t) N * N * N;
	if (b->nsub != 1 || b->n != n) {
		return fail(c, CT_ERR_ARG, "ct_initialize: the box must be a single box of nfour^3 particles");
	}
	if (!p->table_k || !p->table_p || p->ntable < 8 || !(p->box_size > 0.0) || !(p->hubble > 0.0) || !(p->sigma8 > 0.0) || !(p->omega_m > 0.0) ||
			!(p->z0 > -1.0)) {
		return fail(c, CT_ERR_ARG, "ct_initialize: bad parameters or power table");
	}
	// the table as read_power_spectrum takes it (initialize.cpp:870-898): k h / Mpc -> 1 / Mpc,
	// P (Mpc / h)^3 -> Mpc^3, log-uniform in k
	const float h = (float) p->hubble;
	std::vector<float> P(p->ntable);
	float kmax = 0.0, kmin = 3.4e38f;
	for (int i = 0; i < p->ntable; i++) {
		const float k = p->table_k[i] * h;
		P[i] = p->table_p[i] / (h * h * h);
		if (!(k > 0.f) || !(P[i] > 0.f)) {
			return fail(c, CT_ERR_ARG, "ct_initialize: power table entries must be positive");
		}
		kmax = std::max(kmax, k);
		kmin = std::min(kmin, k);
	}
	PowerTable tab;
	tab.P = P.data();
	tab.n = p->ntable;
	tab.logkmin = std::log(kmin);
	const float logkmax = std::log(kmax);
	tab.dlogk = (logkmax - tab.logkmin) / (p->ntable - 1);
	const float box = (float) p->box_size;
	// the interpolation needs two table points below and three above each |k| of the grid
	const double kf = 2.0 * M_PI / box, kN = kf * std::sqrt(3.0) * (N / 2);
	if (std::log(kf) < tab.logkmin + 1.0 * tab.dlogk || std::log(kN) > logkmax - 2.0 * tab.dlogk) {
		return fail(c, CT_ERR_ARG, "ct_initialize: the power table does not cover the grid's wavenumbers " + std::to_string(kf) + " .. " +
				std::to_string(kN) + " / Mpc");
	}
	const float norm = sigma8_normalize(tab, P, logkmax, p->hubble, p->sigma8);
	// growth and velocity factors (initialize(), initialize.cpp:262-275)
	const float omega_m = (float) p->omega_m;
	const float a0 = 1.0 / (p->z0 + 1.0);
	const float D1 = growth_factor(omega_m, a0) / growth_factor(omega_m, 1.0);
	const float Om = omega_m / (omega_m + (a0 * a0 * a0) * (1.0 - omega_m));
	const float f1 = std::pow(Om, 5.f / 9.f);
	const float H0 = (float) p->H0;
	const float H = H0 * std::sqrt(omega_m / (a0 * a0 * a0) + 1.0 - omega_m);
	const float prefac1 = f1 * H * a0 * a0;
	const float D2 = -3.f * (D1 * D1) / 7.f;
	const float f2 = 2.f * std::pow(Om, 6.f / 11.f);
	const float prefac2 = f2 * H * a0 * a0;
	cudaSetDevice(c->device);
	cudaStream_t st = c->stream;
	FtScope S(c);
	const int NZ = N / 2 + 1;
	const int64_t ncx = (int64_t) N * N * NZ;
	float* dP = nullptr;
	float2* A = nullptr;
	cufftComplex* Y = nullptr;
	float* R = nullptr;
	double* G1 = nullptr;
	double* G2 = nullptr;
	unsigned int* dmax = nullptr;
	CT_TRY(S.alloc(&dP, P.size(), "power table"));
	CT_TRY(S.alloc(&A, ncx, "mode amplitudes"));
	CT_TRY(S.alloc(&Y, ncx, "k-space field"));
	CT_TRY(S.alloc(&R, n, "real-space field"));
	CT_TRY(S.alloc(&G1, n, "interpolation pass"));
	CT_TRY(S.alloc(&G2, n, "interpolation pass"));
	CT_TRY(S.alloc(&dmax, 6, "displacement maxima"));
	CT_TRY(S.plan(0, N, CUFFT_C2R));
	CT_CUDA(c, cudaMemcpyAsync(dP, P.data(), sizeof(float) * P.size(), cudaMemcpyHostToDevice, st));
	CT_CUDA(c, cudaMemsetAsync(dmax, 0, 6 * sizeof(unsigned int), st));
	PowerTable dtab = tab;
	dtab.P = dP;
	const float factor = std::pow(box, -1.5) * N * N * N;
	const double scale = 1.0 / ((double) N * N * N);  // cuFFT's inverse is unnormalised
	const float fscale = (float) scale;
	const double box_inv = 1.0 / box;
	const int gn = ft_grid(c, n), gx = ft_grid(c, ncx);
	c->launches += 3;
	k_ic_lattice<<<gn, FT_TPB, 0, st>>>(N, b->x[0], b->x[1], b->x[2], b->v[0], b->v[1], b->v[2], b->rung);
	k_ic_uniforms<<<ft_grid(c, (int64_t) N * N), FT_TPB, 0, st>>>(N, A);
	k_ic_amplitude<<<gx, FT_TPB, 0, st>>>(N, box, factor, dtab, A);
	// interpolation at the lattice points and update of axis dim
	auto displace = [&](int dim, float D, float prefac, unsigned int* mx) {
		c->launches += 3;
		k_ic_smooth<float><<<gn, FT_TPB, 0, st>>>(N, 0, R, G1);
		k_ic_smooth<double><<<gn, FT_TPB, 0, st>>>(N, 1, G1, G2);
		k_ic_displace<<<gn, FT_TPB, 0, st>>>(N, G2, scale, dim, D, prefac, box_inv, b->x[dim], b->v[dim], mx);
	};
	for (int dim = 0; dim < 3; dim++) {
		c->launches++;
		k_ic_field<<<gx, FT_TPB, 0, st>>>(N, box, dim, 3, A, Y);
		CT_TRY(fft_check(c, cufftExecC2R(S.plans[0], Y, R), "cufftExecC2R"));
		displace(dim, D1, prefac1, dmax + dim);
	}
	if (p->twolpt) {
		float* delta2 = nullptr;
		float* part = nullptr;
		cufftComplex* d2k = nullptr;
		CT_TRY(S.alloc(&delta2, n, "2LPT source"));
		CT_TRY(S.alloc(&part, n, "2LPT factor"));
		CT_TRY(S.alloc(&d2k, ncx, "2LPT source transform"));
		CT_TRY(S.plan(1, N, CUFFT_R2C));
		c->launches++;
		k_fill<<<gn, FT_TPB, 0, st>>>(n, delta2, 0.f);
		const int pairs[9][2] = { { 1, 1 }, { 2, 2 }, { 0, 0 }, { 2, 2 }, { 0, 0 }, { 1, 1 }, { 0, 1 }, { 0, 2 }, { 1, 2 } };
		for (int ph = 0; ph < 9; ph++) {
			c->launches += 2;
			k_ic_field<<<gx, FT_TPB, 0, st>>>(N, box, pairs[ph][0], pairs[ph][1], A, Y);
			CT_TRY(fft_check(c, cufftExecC2R(S.plans[0], Y, R), "cufftExecC2R"));
			k_twolpt_phase<<<gn, FT_TPB, 0, st>>>(n, ph, R, fscale, part, delta2);
		}
		CT_TRY(fft_check(c, cufftExecR2C(S.plans[1], delta2, d2k), "cufftExecR2C"));
		for (int dim = 0; dim < 3; dim++) {
			c->launches++;
			k_ic_correction<<<gx, FT_TPB, 0, st>>>(d2k, Y, N, box, dim);
			CT_TRY(fft_check(c, cufftExecC2R(S.plans[0], Y, R), "cufftExecC2R"));
			displace(dim, -D2, prefac2, dmax + 3 + dim);
		}
	}
	CT_CUDA(c, cudaGetLastError());
	unsigned int hm[6];
	CT_CUDA(c, cudaMemcpyAsync(hm, dmax, sizeof(hm), cudaMemcpyDeviceToHost, st));
	CT_CUDA(c, cudaStreamSynchronize(st));
	b->rung_begin = 0;
	b->rung_stack.clear();
	b->tree_valid = false;
	if (ret) {
		ret->D1 = D1;
		ret->D2 = D2;
		ret->prefac1 = prefac1;
		ret->prefac2 = prefac2;
		ret->norm = norm;
		for (int d = 0; d < 3; d++) {
			float a, q;
			memcpy(&a, hm + d, 4);
			memcpy(&q, hm + 3 + d, 4);
			ret->dxmax[d] = a;
			ret->dxmax2[d] = q;
		}
	}
	return CT_OK;
}

extern "C" ct_status ct_power_spectrum(ct_ctx* ctx, int box_id, int nfour, int fold, double box_size, int max_bins, float* k, float* P, float* Perr,
		int* nbins) {
	Ctx* c = (Ctx*) ctx;
	if (!c || box_id < 0 || box_id >= (int) c->boxes.size() || !c->boxes[box_id] || !nbins) {
		return fail(c, CT_ERR_ARG, "ct_power_spectrum: bad arguments");
	}
	Box* b = c->boxes[box_id];
	if (b->nsub != 1) {
		return fail(c, CT_ERR_ARG, "ct_power_spectrum: the spectrum is of a single box, not an ensemble");
	}
	const int N = nfour;
	if (N < 4 || N > 1024 || N % 2 != 0 || fold < 1 || !(box_size > 0.0)) {
		return fail(c, CT_ERR_ARG, "ct_power_spectrum: nfour must be even, 4 .. 1024; fold >= 1; box_size > 0");
	}
	// log-spaced bin edges in grid units from 1 to N / 2 (fft3d_power_spectrum, fft.cpp:172-214)
	std::vector<float> kb;
	const double Ns = std::max(N / 8.0, 64.0);
	const double lkmin = std::log(0.999999), lkmax = std::log(N / 2.0);
	const double dl = (lkmax - lkmin) / Ns;
	for (int i = 0; i <= Ns; i++) {
		kb.push_back(std::exp(lkmin + dl * i));
	}
	const int nb = (int) kb.size() - 1;
	*nbins = nb;
	if (!k || !P || max_bins < nb) {
		return k || P ? fail(c, CT_ERR_ARG, "ct_power_spectrum: room for " + std::to_string(nb) + " bins needed") : CT_OK;
	}
	cudaSetDevice(c->device);
	cudaStream_t st = c->stream;
	FtScope S(c);
	const int64_t ng = (int64_t) N * N * N, ncx = (int64_t) N * N * (N / 2 + 1);
	float* rho = nullptr;
	cufftComplex* Y = nullptr;
	float* dkb = nullptr;
	double* acc = nullptr;
	double* pmean = nullptr;
	CT_TRY(S.alloc(&rho, ng, "density grid"));
	CT_TRY(S.alloc(&Y, ncx, "density transform"));
	CT_TRY(S.alloc(&dkb, kb.size(), "k bins"));
	CT_TRY(S.alloc(&acc, 3 * nb, "bin sums"));
	CT_TRY(S.alloc(&pmean, nb, "bin means"));
	CT_TRY(S.plan(1, N, CUFFT_R2C));
	CT_CUDA(c, cudaMemcpyAsync(dkb, kb.data(), sizeof(float) * kb.size(), cudaMemcpyHostToDevice, st));
	CT_CUDA(c, cudaMemsetAsync(acc, 0, sizeof(double) * 3 * nb, st));
	// the grid starts at -1 (fft3d_init(N, -1), power.cpp:35) and gains the particles' weights
	c->launches += 2;
	k_fill<<<ft_grid(c, ng), FT_TPB, 0, st>>>(ng, rho, -1.0f);
	const int64_t np = b->n;
	if (np > 0) {
		c->launches++;
		k_density<<<ft_grid(c, np), FT_TPB, 0, st>>>(np, b->x[0], b->x[1], b->x[2], fold, N, rho);
	}
	CT_TRY(fft_check(c, cufftExecR2C(S.plans[1], rho, Y), "cufftExecR2C"));
	k_power_bins<<<ft_grid(c, ncx), FT_TPB, 0, st>>>(Y, N, dkb, nb, 1, nullptr, acc);
	std::vector<double> h(3 * nb);
	CT_CUDA(c, cudaMemcpyAsync(h.data(), acc, sizeof(double) * 3 * nb, cudaMemcpyDeviceToHost, st));
	CT_CUDA(c, cudaStreamSynchronize(st));
	std::vector<double> mean(nb, 0.0);
	for (int i = 0; i < nb; i++) {
		const double cnt = h[nb + i];
		mean[i] = cnt > 0 ? h[i] / cnt : 0.0;
		P[i] = (float) mean[i];
		k[i] = (float) (std::sqrt((double) kb[i] * kb[i + 1]) * (2.0 * M_PI / box_size) * fold);
	}
	CT_CUDA(c, cudaMemcpyAsync(pmean, mean.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, st));
	CT_CUDA(c, cudaMemsetAsync(acc, 0, sizeof(double) * nb, st));
	c->launches++;
	k_power_bins<<<ft_grid(c, ncx), FT_TPB, 0, st>>>(Y, N, dkb, nb, 2, pmean, acc);
	std::vector<double> dev(nb);
	CT_CUDA(c, cudaMemcpyAsync(dev.data(), acc, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
	CT_CUDA(c, cudaStreamSynchronize(st));
	for (int i = 0; i < nb; i++) {
		const double cnt = h[nb + i];
		float e = 0.f;
		if (cnt > 0) {
			if (cnt > 1) {
				e = (float) (std::sqrt(dev[i]) / std::sqrt(cnt - 1) / std::sqrt(cnt));
			} else {
				P[i] = 0.f;
			}
		}
		if (Perr) {
			Perr[i] = e;
		}
	}
	CT_CUDA(c, cudaGetLastError());
	return CT_OK;
}
