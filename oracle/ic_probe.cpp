// Test infrastructure only (oracle build; never part of the library).
//
// Runs the reference's own initial-condition generator, initialize() of src/initialize.cpp
// (Zel'dovich displacements and the 2LPT correction, src/initialize.cpp:261-355,436-898), and its
// matter power spectrum, power_spectrum_compute() of src/power.cpp with the binning of
// src/fft.cpp:172-360 and the density kernel of src/power.cu:31-67, with its distributed 3-D
// transform (src/fft.cpp) compiled where they lie, in one process: HPX is
// the single-threaded stand-in in stub/hpx, FFTW's one-line transforms are the plain discrete
// Fourier sums below (double accumulation, stored in single precision as FFTW stores them),
// GSL's "taus" generator is L'Ecuyer's published three-component Tausworthe recurrence (the
// algorithm gsl_rng_taus implements), and the power spectrum is read from power.init in the
// working directory, as the reference reads it (src/initialize.cpp:870-898).
//
//   ic_probe N box_mpc z0 omega_m hubble sigma8 twolpt table.txt out.bin
//   ic_probe power N fold box_mpc particles.bin out.bin
//
// table.txt holds "k P" lines (k in h/Mpc, P in (Mpc/h)^3); the probe copies it to ./power.init.
// out.bin: int64 n, then n uint32 x, y, z (fixed32 raw), then n float vx, vy, vz, then the
// float factors D1, D2, prefac1, prefac2 as initialize() computes them for z0.
// Code units: box = 1, H0 = 1 (code_to_s = 1 / (H0 [1/s] * hubble)).
// power mode: particles.bin holds int64 n, then n uint32 x, y, z (fixed32 raw); out.bin gets
// int64 m, then m float k, P, Perr (the power_spectrum_t the reference returns).
#include "ref_host.h"

#include <cosmictiger/boltzmann.hpp>
#include <cosmictiger/constants.hpp>
#include <cosmictiger/cosmology.hpp>
#include <cosmictiger/initialize.hpp>
#include <cosmictiger/power.hpp>
#include <cosmictiger/zero_order.hpp>
#include <fftw3.h>
#include <silo.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

// ---------------------------------------------------------------- GSL "taus" (L'Ecuyer 1996)
struct gsl_rng_type {
	int id;
};
struct gsl_rng {
	uint32_t s1, s2, s3;
};
static const gsl_rng_type taus_type { 1 };
const gsl_rng_type* gsl_rng_taus = &taus_type;

static uint32_t taus_next(gsl_rng* r) {
	// the three component recurrences of the maximally equidistributed combined Tausworthe
	// generator (L'Ecuyer, Math. Comp. 65 (1996) 203-213), combined by exclusive or
	r->s1 = ((r->s1 & 4294967294u) << 12) ^ (((r->s1 << 13) ^ r->s1) >> 19);
	r->s2 = ((r->s2 & 4294967288u) << 4) ^ (((r->s2 << 2) ^ r->s2) >> 25);
	r->s3 = ((r->s3 & 4294967280u) << 17) ^ (((r->s3 << 3) ^ r->s3) >> 11);
	return r->s1 ^ r->s2 ^ r->s3;
}
gsl_rng* gsl_rng_alloc(const gsl_rng_type*) {
	return new gsl_rng { 1, 1, 1 };
}
void gsl_rng_set(const gsl_rng* cr, unsigned long int seed) {
	// seeding: a zero seed becomes 1, the three states follow by the LCG x -> 69069 x (mod 2^32),
	// then six steps warm the generator up (the published seeding procedure of gsl_rng_taus)
	gsl_rng* r = const_cast<gsl_rng*>(cr);
	uint32_t s = (uint32_t) seed;
	if (s == 0) {
		s = 1;
	}
	r->s1 = 69069u * s;
	r->s2 = 69069u * r->s1;
	r->s3 = 69069u * r->s2;
	for (int i = 0; i < 6; i++) {
		taus_next(r);
	}
}
double gsl_rng_uniform(const gsl_rng* r) {
	return taus_next(const_cast<gsl_rng*>(r)) / 4294967296.0;
}
double gsl_rng_uniform_pos(const gsl_rng* r) {
	double x;
	do {
		x = gsl_rng_uniform(r);
	} while (x == 0.0);
	return x;
}
unsigned long int gsl_rng_get(const gsl_rng* r) {
	return taus_next(const_cast<gsl_rng*>(r));
}
void gsl_rng_free(gsl_rng* r) {
	delete r;
}

// ---------------------------------------------------------------- FFTW's one-line transforms
// Unnormalised sums X_k = sum_j x_j exp(sign 2 pi i j k / n) in double, stored as floats.
struct fftwf_plan_s {
	int n, kind, sign;  // kind: 0 complex, 1 real to complex, 2 complex to real
	void* in;
	void* out;
};
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex* in, fftwf_complex* out, int sign, unsigned) {
	return new fftwf_plan_s { n, 0, sign, in, out };
}
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float* in, fftwf_complex* out, unsigned) {
	return new fftwf_plan_s { n, 1, FFTW_FORWARD, in, out };
}
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex* in, float* out, unsigned) {
	return new fftwf_plan_s { n, 2, FFTW_BACKWARD, in, out };
}
void fftwf_execute(const fftwf_plan p) {
	const int n = p->n;
	std::vector<double> cr(n), ci(n);
	for (int j = 0; j < n; j++) {
		const double a = 2.0 * M_PI * j / n;
		cr[j] = std::cos(a);
		ci[j] = std::sin(a);
	}
	if (p->kind == 0) {
		const fftwf_complex* x = (const fftwf_complex*) p->in;
		std::vector<double> re(n), im(n);
		for (int k = 0; k < n; k++) {
			double sr = 0.0, si = 0.0;
			for (int j = 0; j < n; j++) {
				const int m = (int) (((int64_t) j * k) % n);
				const double c = cr[m], s = p->sign * ci[m];
				sr += x[j][0] * c - x[j][1] * s;
				si += x[j][0] * s + x[j][1] * c;
			}
			re[k] = sr;
			im[k] = si;
		}
		fftwf_complex* y = (fftwf_complex*) p->out;
		for (int k = 0; k < n; k++) {
			y[k][0] = (float) re[k];
			y[k][1] = (float) im[k];
		}
	} else if (p->kind == 1) {
		const float* x = (const float*) p->in;
		fftwf_complex* y = (fftwf_complex*) p->out;
		std::vector<double> re(n / 2 + 1), im(n / 2 + 1);
		for (int k = 0; k <= n / 2; k++) {
			double sr = 0.0, si = 0.0;
			for (int j = 0; j < n; j++) {
				const int m = (int) (((int64_t) j * k) % n);
				sr += x[j] * cr[m];
				si -= x[j] * ci[m];
			}
			re[k] = sr;
			im[k] = si;
		}
		for (int k = 0; k <= n / 2; k++) {
			y[k][0] = (float) re[k];
			y[k][1] = (float) im[k];
		}
	} else {
		// Hermitian input of n / 2 + 1 entries; the imaginary parts of the zero and (even n)
		// Nyquist entries are ignored, as a real-output transform ignores them
		const fftwf_complex* x = (const fftwf_complex*) p->in;
		std::vector<double> r(n);
		for (int j = 0; j < n; j++) {
			double s = x[0][0];
			for (int k = 1; k <= (n - 1) / 2; k++) {
				const int m = (int) (((int64_t) j * k) % n);
				s += 2.0 * (x[k][0] * cr[m] - x[k][1] * ci[m]);
			}
			if (n % 2 == 0) {
				s += x[n / 2][0] * ((j % 2) ? -1.0 : 1.0);
			}
			r[j] = s;
		}
		float* y = (float*) p->out;
		for (int j = 0; j < n; j++) {
			y[j] = (float) r[j];
		}
	}
}
void fftwf_destroy_plan(fftwf_plan p) {
	delete p;
}

// ---------------------------------------------------------------- the density kernel
// The reference's accumulate_density_kernel (src/power.cu:31-67), taken verbatim from its
// source into oracle/_ref/ic/power_kernel.inc by the build recipe, compiled here as a host
// function: its launch indices are the emulated block and thread below, and its atomic adds
// plain adds (one thread at a time).
namespace emu {
struct index3 {
	unsigned x = 0, y = 0, z = 0;
};
static index3 thread, block, grid;
}  // namespace emu
static inline float emu_atomic_add(float* p, float v) {
	const float old = *p;
	*p = old + v;
	return old;
}
#undef __global__
#define __global__ static
#define threadIdx emu::thread
#define blockIdx emu::block
#define gridDim emu::grid
#define atomicAdd emu_atomic_add
#define BLOCK_SIZE 256
#include "power_kernel.inc"
#undef threadIdx
#undef blockIdx
#undef gridDim
#undef atomicAdd

// The reference's launch wrapper (src/power.cu:69-84) on the host: a zeroed density box and
// the kernel over one block of BLOCK_SIZE threads, run thread by thread (the GPU's order of the
// atomic adds is not fixed either; sums differ by rounding only).
vector<float> accumulate_density_cuda(int M, int Ndim, range<int64_t> intbox) {
	vector<float> rho(intbox.volume(), 0.f);
	emu::grid.x = 1;
	emu::block.x = 0;
	for (unsigned t = 0; t < BLOCK_SIZE; t++) {
		emu::thread.x = t;
		accumulate_density_kernel(&particles_pos(XDIM, 0), &particles_pos(YDIM, 0), &particles_pos(ZDIM, 0), rho.data(), M, particles_size(), Ndim,
				intbox);
	}
	return rho;
}

// ---------------------------------------------------------------- not reached
// the Einstein-Boltzmann power spectrum (compute_power_spectrum), the alternative to power.init
void create_zero_order_universe(zero_order_universe*, std::function<double(double)>, double, cosmic_params) {
	abort();
}
void einstein_boltzmann_interpolation_function(interp_functor<double>*, interp_functor<double>*, cos_state*, zero_order_universe*, double, double, double, int,
		double, double, bool, double) {
	abort();
}
// Silo output of the transform (fft3d2silo, a debugging dump)
DBfile* DBCreateReal(const char*, int, int, const char*, int) {
	abort();
}
int DBPutQuadmesh(DBfile*, const char*, const char* const*, const void*, const int*, int, int, int, DBoptlist*) {
	abort();
}
int DBPutQuadvar1(DBfile*, const char*, const char*, const void*, const int*, int, const void*, int, int, int, DBoptlist*) {
	abort();
}
int DBClose(DBfile*) {
	abort();
}

static int power_main(int argc, char** argv) {
	if (argc != 7) {
		fprintf(stderr, "usage: ic_probe power N fold box_mpc particles.bin out.bin\n");
		return 2;
	}
	const int N = atoi(argv[2]);
	const int fold = atoi(argv[3]);
	ref_set_defaults();
	FILE* fp = fopen(argv[5], "rb");
	int64_t n = 0;
	if (!fp || fread(&n, sizeof(n), 1, fp) != 1) {
		return 2;
	}
	// the binning reads the grid size from parts_dim (src/fft.cpp:245,315), the transform from Nfour
	g_opts.Nfour = N;
	g_opts.parts_dim = N;
	g_opts.nparts = n;
	g_opts.code_to_cm = atof(argv[4]) * constants::mpc_to_cm;
	particles_resize(n);
	for (int d = 0; d < NDIM; d++) {
		std::vector<uint32_t> x(n);
		if (fread(x.data(), sizeof(uint32_t), n, fp) != (size_t) n) {
			return 2;
		}
		for (int64_t i = 0; i < n; i++) {
			particles_pos(d, i).set_integer(x[i]);
		}
	}
	fclose(fp);
	const power_spectrum_t ps = power_spectrum_compute(fold);
	fp = fopen(argv[6], "wb");
	if (!fp) {
		return 2;
	}
	const int64_t m = ps.P.size();
	fwrite(&m, sizeof(m), 1, fp);
	fwrite(ps.k.data(), sizeof(float), m, fp);
	fwrite(ps.P.data(), sizeof(float), m, fp);
	fwrite(ps.Perr.data(), sizeof(float), m, fp);
	fclose(fp);
	return 0;
}

int main(int argc, char** argv) {
	if (argc > 1 && std::string(argv[1]) == "power") {
		return power_main(argc, argv);
	}
	if (argc != 10) {
		fprintf(stderr, "usage: ic_probe N box_mpc z0 omega_m hubble sigma8 twolpt table.txt out.bin\n");
		return 2;
	}
	const int N = atoi(argv[1]);
	const double box = atof(argv[2]);
	const double z0 = atof(argv[3]);
	ref_set_defaults();
	g_opts.Nfour = N;
	g_opts.parts_dim = N;
	g_opts.nparts = (size_t) N * N * N;
	g_opts.omega_m = atof(argv[4]);
	g_opts.hubble = atof(argv[5]);
	g_opts.sigma8 = atof(argv[6]);
	g_opts.twolpt = atoi(argv[7]) != 0;
	g_opts.use_power_file = true;
	g_opts.use_glass = false;
	g_opts.close_pack = false;
	g_opts.code_to_cm = box * constants::mpc_to_cm;
	g_opts.code_to_s = 1.0 / (constants::H0 * g_opts.hubble);
	{
		FILE* in = fopen(argv[8], "rt");
		FILE* out = fopen("power.init", "wt");
		if (!in || !out) {
			fprintf(stderr, "ic_probe: cannot copy %s to ./power.init\n", argv[8]);
			return 2;
		}
		char buf[4096];
		size_t k;
		while ((k = fread(buf, 1, sizeof(buf), in)) > 0) {
			fwrite(buf, 1, k, out);
		}
		fclose(in);
		fclose(out);
	}
	initialize(z0);
	// the factors initialize() prints, in its own single-precision expressions
	// (src/initialize.cpp:264-273)
	const float omega_m = g_opts.omega_m;
	const float a0 = 1.0 / (z0 + 1.0);
	const float D1 = cosmos_growth_factor(omega_m, a0) / cosmos_growth_factor(omega_m, 1.0);
	const float Om = omega_m / (omega_m + (a0 * a0 * a0) * (1.0 - omega_m));
	const float H0 = constants::H0 * g_opts.code_to_s * g_opts.hubble;
	const float H = H0 * std::sqrt(omega_m / (a0 * a0 * a0) + 1.0 - omega_m);
	const float fac[4] = { D1, -3.f * D1 * D1 / 7.f, std::pow(Om, 5.f / 9.f) * H * a0 * a0, 2.f * std::pow(Om, 6.f / 11.f) * H * a0 * a0 };
	const int64_t n = particles_size();
	FILE* fp = fopen(argv[9], "wb");
	if (!fp) {
		return 2;
	}
	fwrite(&n, sizeof(n), 1, fp);
	for (int d = 0; d < NDIM; d++) {
		std::vector<uint32_t> x(n);
		for (int64_t i = 0; i < n; i++) {
			x[i] = particles_pos(d, i).raw();
		}
		fwrite(x.data(), sizeof(uint32_t), n, fp);
	}
	for (int d = 0; d < NDIM; d++) {
		std::vector<float> v(n);
		for (int64_t i = 0; i < n; i++) {
			v[i] = particles_vel(d, i);
		}
		fwrite(v.data(), sizeof(float), n, fp);
	}
	fwrite(fac, sizeof(float), 4, fp);
	fclose(fp);
	return 0;
}
