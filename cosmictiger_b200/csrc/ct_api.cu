// C ABI of the gravity step: contexts, boxes, transfers, drift, rung sort, direct Ewald.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>

#include "ct_internal.cuh"
#include "fmm_p7.h"

namespace ct {

ct_status fail(Ctx* c, ct_status code, const std::string& msg) {
	if (c) {
		c->err = msg;
	}
	return code;
}

ct_status cuda_check(Ctx* c, cudaError_t e, const char* what) {
	return fail(c, e == cudaErrorMemoryAllocation ? CT_ERR_MEMORY : CT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

ct_status dalloc(Ctx* c, void** p, size_t bytes, const char* what) {
	*p = nullptr;
	if (bytes == 0) {
		bytes = 16;
	}
	if (c->budget && c->used + bytes > c->budget) {
		return fail(c, CT_ERR_MEMORY, std::string("HBM budget exhausted allocating ") + what);
	}
	// stream-ordered, from the context's pool: no device-wide synchronisation, and memory freed
	// earlier in the context is reused without going back to the CUDA driver
	const cudaError_t e = cudaMallocFromPoolAsync(p, bytes, c->pool, c->stream);
	if (e != cudaSuccess) {
		cudaGetLastError();
		*p = nullptr;
		return fail(c, CT_ERR_MEMORY, std::string("device allocation failed for ") + what + ": " + cudaGetErrorString(e));
	}
	c->used += bytes;
	return CT_OK;
}

void dfree(Ctx* c, void* p, size_t bytes) {
	if (p) {
		cudaFreeAsync(p, c->stream);
		c->used -= std::min(c->used, bytes == 0 ? size_t(16) : bytes);
	}
}

void* scratch(Ctx* c, int slot, size_t bytes, ct_status* st) {
	if ((int) c->scratch.size() <= slot) {
		c->scratch.resize(slot + 1);
	}
	DevBuf& b = c->scratch[slot];
	if (b.bytes < bytes || !b.p) {
		if (b.p) {
			cudaStreamSynchronize(c->stream);
			dfree(c, b.p, b.bytes);
			b.p = nullptr;
			b.bytes = 0;
		}
		const size_t want = std::max(bytes + bytes / 4, (size_t) 4096);
		const ct_status s = dalloc(c, &b.p, want, "scratch");
		if (s != CT_OK) {
			*st = s;
			return nullptr;
		}
		b.bytes = want;
	}
	return b.p;
}

namespace {

Box* get_box(Ctx* c, int id) {
	if (!c || id < 0 || id >= (int) c->boxes.size()) {
		return nullptr;
	}
	return c->boxes[id];
}

int grid(Ctx* c, int64_t n, int tpb) {
	return (int) std::max<int64_t>(1, std::min<int64_t>((n + tpb - 1) / tpb, (int64_t) c->nsm * 8));
}

__global__ void k_aos_to_soa(int64_t n, const float* __restrict__ vxyz, float* v0, float* v1, float* v2) {
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		v0[i] = vxyz[3 * i];
		v1[i] = vxyz[3 * i + 1];
		v2[i] = vxyz[3 * i + 2];
	}
}

__global__ void k_soa_to_aos(int64_t n, const float* v0, const float* v1, const float* v2, float* __restrict__ vxyz) {
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		vxyz[3 * i] = v0[i];
		vxyz[3 * i + 1] = v1[i];
		vxyz[3 * i + 2] = v2[i];
	}
}

// Drift of one rung (src/drift.cu:36-154; lightcone capture excluded): FP64 position update,
// periodic wrap, truncating fixed32 store.  Particles of other rungs are not touched.
__global__ void __launch_bounds__(256) k_drift(int64_t b, int64_t n, uint32_t* __restrict__ x0, uint32_t* __restrict__ x1, uint32_t* __restrict__ x2,
		float* __restrict__ v0, float* __restrict__ v1, float* __restrict__ v2, const int8_t* __restrict__ rung, int which, double c1, double drag_c0,
		int do_drag) {
	for (int64_t i = b + blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		if (rung[i] != which) {
			continue;
		}
		uint32_t* X[3] = { x0, x1, x2 };
		float* V[3] = { v0, v1, v2 };
#pragma unroll
		for (int d = 0; d < 3; d++) {
			const double xo = fixed_to_double(X[d][i]);
			double x1d = __dadd_rn(xo, __dmul_rn((double) V[d][i], c1));
			x1d = __dsub_rn(x1d, (double) (x1d >= 1.0));
			x1d = __dadd_rn(x1d, (double) (x1d < 0.0));
			X[d][i] = fixed_from_double(x1d);
		}
		if (do_drag) {
#pragma unroll
			for (int d = 0; d < 3; d++) {
				V[d][i] = (float) ((double) V[d][i] * drag_c0);
			}
		}
	}
}

// ---- rung partition (src/particles.cpp:1029-1076): same exact permutation rule as the tree
// partition, with predicate rung < minrung on the left.
__global__ void k_rung_flags(int64_t b, int64_t e, const int8_t* rung, int minrung, int* lt) {
	for (int64_t i = b + blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < e; i += (int64_t) gridDim.x * blockDim.x) {
		lt[i - b] = rung[i] < minrung;
	}
}
__global__ void k_rung_mis(int64_t b, int64_t e, const int* lt, const int* m, int* misL, int* misR) {
	const int64_t s = b + *m;
	for (int64_t i = b + blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < e; i += (int64_t) gridDim.x * blockDim.x) {
		const int f = lt[i - b];
		misL[i - b] = (i < s) && !f;
		misR[i - b] = (i >= s) && f;
	}
}
__global__ void k_rung_pos(int64_t b, int64_t e, const int* misL, const int* misR, const int* exL, const int* exR, const int* totR, int* posL,
		int* posR) {
	for (int64_t i = b + blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < e; i += (int64_t) gridDim.x * blockDim.x) {
		const int64_t k = i - b;
		if (misL[k]) {
			posL[exL[k]] = (int) i;
		}
		if (misR[k]) {
			posR[*totR - 1 - exR[k]] = (int) i;
		}
	}
}
__global__ void k_rung_swap(const int* posL, const int* posR, const int* nmis, uint32_t* x0, uint32_t* x1, uint32_t* x2, float* v0, float* v1,
		float* v2, int8_t* rung) {
	const int n = *nmis;
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		const int a = posL[k], c = posR[k];
		uint32_t t = x0[a];
		x0[a] = x0[c];
		x0[c] = t;
		t = x1[a];
		x1[a] = x1[c];
		x1[c] = t;
		t = x2[a];
		x2[a] = x2[c];
		x2[c] = t;
		float f = v0[a];
		v0[a] = v0[c];
		v0[c] = f;
		f = v1[a];
		v1[a] = v1[c];
		v1[c] = f;
		f = v2[a];
		v2[a] = v2[c];
		v2[c] = f;
		const int8_t r = rung[a];
		rung[a] = rung[c];
		rung[c] = r;
	}
}

// ---- FP64 direct Ewald (accuracy reference)
__global__ void k_struct_factor(int64_t n, const uint32_t* x0, const uint32_t* x1, const uint32_t* x2, const float* four, double* CS) {
	const int h = blockIdx.y;
	const double hx = four[3 * h], hy = four[3 * h + 1], hz = four[3 * h + 2];
	double c = 0.0, s = 0.0;
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		const double ph = 6.283185307179586 * (hx * fixed_to_double(x0[i]) + hy * fixed_to_double(x1[i]) + hz * fixed_to_double(x2[i]));
		double sn, cs;
		sincos(ph, &sn, &cs);
		c += cs;
		s += sn;
	}
	for (int o = 16; o; o >>= 1) {
		c += __shfl_xor_sync(0xffffffffu, c, o);
		s += __shfl_xor_sync(0xffffffffu, s, o);
	}
	if ((threadIdx.x & 31) == 0) {
		atomicAdd(CS + 2 * h, c);
		atomicAdd(CS + 2 * h + 1, s);
	}
}

__device__ void ewald_pair_fp64(double dx, double dy, double dz, const float* real, double& phi, double* g) {
	const double alpha = 2.0, tsp = 1.1283791670955126;
	const double r2 = dx * dx + dy * dy + dz * dz;
	const double r = sqrt(r2);
	if (alpha * r < 0.05) {
		const double a2r2 = alpha * alpha * r2;
		phi += tsp * alpha * (1.0 - a2r2 / 3.0 + a2r2 * a2r2 / 10.0 - a2r2 * a2r2 * a2r2 / 42.0 + a2r2 * a2r2 * a2r2 * a2r2 / 216.0);
		const double c = tsp * alpha * alpha * alpha * (-2.0 / 3.0 + 0.4 * a2r2 - a2r2 * a2r2 / 7.0 + a2r2 * a2r2 * a2r2 / 27.0);
		g[0] += c * dx;
		g[1] += c * dy;
		g[2] += c * dz;
	} else {
		const double e = erf(alpha * r);
		phi += e / r;
		const double dp = (-e / r2 + tsp * alpha * exp(-alpha * alpha * r2) / r) / r;
		g[0] += dp * dx;
		g[1] += dp * dy;
		g[2] += dp * dz;
	}
	for (int i = 0; i < CT_EWALD_NREAL; i++) {
		const double x = dx - real[3 * i], y = dy - real[3 * i + 1], z = dz - real[3 * i + 2];
		const double s2 = x * x + y * y + z * z;
		if (s2 < 2.6 * 2.6) {
			const double s = sqrt(s2);
			const double ec = erfc(alpha * s);
			phi -= ec / s;
			const double dp = (ec / s2 + tsp * alpha * exp(-alpha * alpha * s2) / s) / s;
			g[0] += dp * x;
			g[1] += dp * y;
			g[2] += dp * z;
		}
	}
	phi += 3.141592653589793 / (alpha * alpha);
}

__global__ void __launch_bounds__(256) k_direct_ewald(int64_t n, const uint32_t* x0, const uint32_t* x1, const uint32_t* x2, const uint32_t* sx,
		const uint32_t* sy, const uint32_t* sz, double h, const float* real, double* out) {
	__shared__ double red[8][4];
	__shared__ float sreal[3 * CT_EWALD_NREAL];
	for (int i = threadIdx.x; i < 3 * CT_EWALD_NREAL; i += blockDim.x) {
		sreal[i] = real[i];
	}
	__syncthreads();
	const int s = blockIdx.x;
	const uint32_t X = sx[s], Y = sy[s], Z = sz[s];
	const double hinv = 1.0 / h, h2inv = hinv * hinv, h3inv = h2inv * hinv;
	double phi = 0.0, g[3] = { 0.0, 0.0, 0.0 };
	for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
		const double dx = (double) (int32_t) (X - x0[j]) * (1.0 / 4294967296.0);
		const double dy = (double) (int32_t) (Y - x1[j]) * (1.0 / 4294967296.0);
		const double dz = (double) (int32_t) (Z - x2[j]) * (1.0 / 4294967296.0);
		const double r2 = dx * dx + dy * dy + dz * dz;
		if (r2 > h * h) {
			const double rinv = 1.0 / sqrt(r2);
			const double r3 = rinv * rinv * rinv;
			g[0] -= dx * r3;
			g[1] -= dy * r3;
			g[2] -= dz * r3;
			phi -= rinv;
		} else {
			const double q2 = r2 * h2inv;
			double f = 315. / 128.;
			f = fma(f, q2, -385. / 32.);
			f = fma(f, q2, 1485. / 64.);
			f = fma(f, q2, -693. / 32.);
			f = fma(f, q2, 1155. / 128.);
			f *= h3inv;
			double p = -63. / 256.;
			p = fma(p, q2, 385. / 256.);
			p = fma(p, q2, -495. / 128.);
			p = fma(p, q2, 693. / 128.);
			p = fma(p, q2, -1155. / 256.);
			p = fma(p, q2, 693. / 256.);
			p *= hinv;
			g[0] -= dx * f;
			g[1] -= dy * f;
			g[2] -= dz * f;
			phi -= p;
		}
		double pc = 0.0, gc[3] = { 0.0, 0.0, 0.0 };
		ewald_pair_fp64(dx, dy, dz, sreal, pc, gc);
		phi += pc;
		g[0] -= gc[0];
		g[1] -= gc[1];
		g[2] -= gc[2];
	}
	double v[4] = { g[0], g[1], g[2], phi };
	for (int k = 0; k < 4; k++) {
		for (int o = 16; o; o >>= 1) {
			v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
		}
	}
	if ((threadIdx.x & 31) == 0) {
		for (int k = 0; k < 4; k++) {
			red[threadIdx.x >> 5][k] = v[k];
		}
	}
	__syncthreads();
	if (threadIdx.x < 4) {
		double t = 0.0;
		for (int w = 0; w < (int) (blockDim.x >> 5); w++) {
			t += red[w][threadIdx.x];
		}
		out[4 * s + threadIdx.x] = t;
	}
}

__global__ void k_direct_ewald_four(int nsink, const uint32_t* sx, const uint32_t* sy, const uint32_t* sz, const float* four, const double* CS, double h,
		double* out) {
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= nsink) {
		return;
	}
	const double xi[3] = { fixed_to_double(sx[s]), fixed_to_double(sy[s]), fixed_to_double(sz[s]) };
	double phi = 693.0 / 256.0 / h;  // the self pair's softened term is excluded (kick.cu:265)
	double g[3] = { 0, 0, 0 };
	for (int k = 0; k < CT_EWALD_NFOUR; k++) {
		const double hx = four[3 * k], hy = four[3 * k + 1], hz = four[3 * k + 2];
		const double h2 = hx * hx + hy * hy + hz * hz;
		const double c0 = -exp(-9.869604401089358 * h2 / 4.0) / (3.141592653589793 * h2);
		double sn, cs;
		sincos(6.283185307179586 * (hx * xi[0] + hy * xi[1] + hz * xi[2]), &sn, &cs);
		phi += c0 * (cs * CS[2 * k] + sn * CS[2 * k + 1]);
		const double sd = sn * CS[2 * k] - cs * CS[2 * k + 1];
		g[0] += c0 * 6.283185307179586 * hx * sd;
		g[1] += c0 * 6.283185307179586 * hy * sd;
		g[2] += c0 * 6.283185307179586 * hz * sd;
	}
	out[4 * s] += g[0];
	out[4 * s + 1] += g[1];
	out[4 * s + 2] += g[2];
	out[4 * s + 3] += phi;
}

// FP32 FMA throughput probe: 16 independent FMA chains per thread in registers.
__global__ void __launch_bounds__(256) k_fma_peak(float* out, int iters, float b, float c) {
	float a[16];
#pragma unroll
	for (int k = 0; k < 16; k++) {
		a[k] = threadIdx.x * 1e-3f + k;
	}
	for (int i = 0; i < iters; i++) {
#pragma unroll
		for (int k = 0; k < 16; k++) {
			a[k] = fmaf(a[k], b, c);
		}
	}
	float s = 0.f;
#pragma unroll
	for (int k = 0; k < 16; k++) {
		s += a[k];
	}
	if (s == 1234.5f) {
		out[threadIdx.x] = s;
	}
}

}  // namespace

ct_status drift_run(Ctx* c, Box* b, int rung, float a, float dt, double drag, bool events) {
	const double c1 = (double) dt / (double) a;
	const double c0 = drag != 0.0 ? 1.0 / (1.0 + drag * (double) dt) : 1.0;
	const int64_t np = b->n - b->rung_begin;
	if (events) {
		cudaEventRecord(c->ev[6], c->stream);
	}
	if (np > 0) {
		c->launches++;
		k_drift<<<grid(c, np, 256), 256, 0, c->stream>>>(b->rung_begin, b->n, b->x[0], b->x[1], b->x[2], b->v[0], b->v[1], b->v[2], b->rung, rung, c1, c0,
				drag != 0.0);
	}
	if (events) {
		cudaEventRecord(c->ev[7], c->stream);
		c->drift_timed = true;
	}
	CT_CUDA(c, cudaGetLastError());
	b->tree_valid = false;
	return CT_OK;
}

ct_status sort_by_rung_run(Ctx* c, Box* b, int minrung) {
	cudaStream_t st = c->stream;
	if (minrung == 0) {
		// particles_sort_by_rung(0) only resets the active range (particles.cpp:1035-1036);
		// saved ranges on the rung stack stay for the caller's pops
		b->rung_begin = 0;
		b->tree_valid = false;
		return CT_OK;
	}
	const int64_t beg = b->rung_begin, e = b->n, n = e - beg;
	if (n <= 0) {
		return CT_OK;
	}
	ct_status s = CT_OK;
	int* lt = (int*) scratch(c, 21, sizeof(int) * n, &s);
	int* misL = (int*) scratch(c, 22, sizeof(int) * n, &s);
	int* misR = (int*) scratch(c, 23, sizeof(int) * n, &s);
	int* exL = (int*) scratch(c, 24, sizeof(int) * n, &s);
	int* exR = (int*) scratch(c, 25, sizeof(int) * n, &s);
	int* posL = (int*) scratch(c, 26, sizeof(int) * n, &s);
	int* posR = (int*) scratch(c, 27, sizeof(int) * n, &s);
	int* tot = (int*) scratch(c, 28, sizeof(int) * 4, &s);
	CT_TRY(s);
	size_t need = 0, need2 = 0;
	cub::DeviceReduce::Sum(nullptr, need, lt, tot, (int) n, st);
	cub::DeviceScan::ExclusiveSum(nullptr, need2, misL, exL, (int) n, st);
	void* tmp = scratch(c, 29, std::max(need, need2) + 256, &s);
	CT_TRY(s);
	need = std::max(need, need2);
	c->launches++;
	k_rung_flags<<<grid(c, n, 256), 256, 0, st>>>(beg, e, b->rung, minrung, lt);
	CT_CUDA(c, cub::DeviceReduce::Sum(tmp, need, lt, tot, (int) n, st));
	c->launches++;
	k_rung_mis<<<grid(c, n, 256), 256, 0, st>>>(beg, e, lt, tot, misL, misR);
	CT_CUDA(c, cub::DeviceScan::ExclusiveSum(tmp, need, misL, exL, (int) n, st));
	CT_CUDA(c, cub::DeviceReduce::Sum(tmp, need, misL, tot + 1, (int) n, st));
	CT_CUDA(c, cub::DeviceScan::ExclusiveSum(tmp, need, misR, exR, (int) n, st));
	CT_CUDA(c, cub::DeviceReduce::Sum(tmp, need, misR, tot + 2, (int) n, st));
	c->launches++;
	k_rung_pos<<<grid(c, n, 256), 256, 0, st>>>(beg, e, misL, misR, exL, exR, tot + 2, posL, posR);
	c->launches++;
	k_rung_swap<<<grid(c, n, 256), 256, 0, st>>>(posL, posR, tot + 1, b->x[0], b->x[1], b->x[2], b->v[0], b->v[1], b->v[2], b->rung);
	int* h = (int*) c->pinned;
	CT_CUDA(c, cudaMemcpyAsync(h, tot, sizeof(int), cudaMemcpyDeviceToHost, st));
	CT_CUDA(c, cudaStreamSynchronize(st));
	b->rung_begin = beg + h[0];
	b->tree_valid = false;
	return CT_OK;
}

ct_status direct_ewald_run(Ctx* c, Box* b, int64_t nsink, const uint32_t* sx, const uint32_t* sy, const uint32_t* sz, double h, double* gx,
		double* gy, double* gz, double* pot) {
	cudaStream_t st = c->stream;
	// the index table is the same for every call: built once, read-only afterwards (calls from
	// several host threads on different contexts share it)
	static ct_p7::EwaldTab tab;
	static std::once_flag tab_once;
	std::call_once(tab_once, [] { ct_p7::ewald_build_indices(tab); });
	ct_status s = CT_OK;
	float* dreal = (float*) scratch(c, 30, sizeof(tab.real) + sizeof(tab.four), &s);
	uint32_t* dsk = (uint32_t*) scratch(c, 31, sizeof(uint32_t) * 3 * nsink, &s);
	double* dout = (double*) scratch(c, 32, sizeof(double) * 4 * nsink + 2 * CT_EWALD_NFOUR * sizeof(double), &s);
	CT_TRY(s);
	float* dfour = dreal + 3 * CT_EWALD_NREAL;
	double* CS = dout + 4 * nsink;
	CT_CUDA(c, cudaMemcpyAsync(dreal, tab.real, sizeof(tab.real), cudaMemcpyHostToDevice, st));
	CT_CUDA(c, cudaMemcpyAsync(dfour, tab.four, sizeof(tab.four), cudaMemcpyHostToDevice, st));
	CT_CUDA(c, cudaMemcpyAsync(dsk, sx, sizeof(uint32_t) * nsink, cudaMemcpyHostToDevice, st));
	CT_CUDA(c, cudaMemcpyAsync(dsk + nsink, sy, sizeof(uint32_t) * nsink, cudaMemcpyHostToDevice, st));
	CT_CUDA(c, cudaMemcpyAsync(dsk + 2 * nsink, sz, sizeof(uint32_t) * nsink, cudaMemcpyHostToDevice, st));
	CT_CUDA(c, cudaMemsetAsync(CS, 0, 2 * CT_EWALD_NFOUR * sizeof(double), st));
	const int64_t n = b->n;
	dim3 gsf((unsigned) std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 64)), CT_EWALD_NFOUR);
	c->launches++;
	k_struct_factor<<<gsf, 256, 0, st>>>(n, b->x[0], b->x[1], b->x[2], dfour, CS);
	for (int64_t s0 = 0; s0 < nsink; s0 += 65535) {
		const int ns = (int) std::min<int64_t>(65535, nsink - s0);
		c->launches++;
		k_direct_ewald<<<ns, 256, 0, st>>>(n, b->x[0], b->x[1], b->x[2], dsk + s0, dsk + nsink + s0, dsk + 2 * nsink + s0, h, dreal, dout + 4 * s0);
	}
	c->launches++;
	k_direct_ewald_four<<<(int) ((nsink + 127) / 128), 128, 0, st>>>((int) nsink, dsk, dsk + nsink, dsk + 2 * nsink, dfour, CS, h, dout);
	CT_CUDA(c, cudaGetLastError());
	std::vector<double> hout(4 * nsink);
	CT_CUDA(c, cudaMemcpyAsync(hout.data(), dout, sizeof(double) * 4 * nsink, cudaMemcpyDeviceToHost, st));
	CT_CUDA(c, cudaStreamSynchronize(st));
	for (int64_t i = 0; i < nsink; i++) {
		gx[i] = hout[4 * i];
		gy[i] = hout[4 * i + 1];
		gz[i] = hout[4 * i + 2];
		pot[i] = hout[4 * i + 3];
	}
	return CT_OK;
}

}  // namespace ct

using namespace ct;

extern "C" {

ct_status ct_ctx_create(ct_ctx** out, int device, size_t hbm_budget_bytes, int order) {
	if (!out || (order != 7 && order != 5)) {
		return CT_ERR_ARG;
	}
	*out = nullptr;
	Ctx* c = new (std::nothrow) Ctx();
	if (!c) {
		return CT_ERR_MEMORY;
	}
	c->device = device;
	c->order = order;
	c->budget = hbm_budget_bytes;
	cudaError_t e = cudaSetDevice(device);
	if (e != cudaSuccess) {
		delete c;
		return CT_ERR_CUDA;
	}
	cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
	if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
		delete c;
		return CT_ERR_CUDA;
	}
	// the context's device memory pool, keeping freed memory for reuse until the context ends
	cudaMemPoolProps props = {};
	props.allocType = cudaMemAllocationTypePinned;
	props.handleTypes = cudaMemHandleTypeNone;
	props.location.type = cudaMemLocationTypeDevice;
	props.location.id = device;
	if (cudaMemPoolCreate(&c->pool, &props) != cudaSuccess) {
		cudaGetLastError();
		cudaStreamDestroy(c->stream);
		delete c;
		return CT_ERR_CUDA;
	}
	uint64_t keep = UINT64_MAX;
	cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
	for (int i = 0; i < 16; i++) {
		cudaEventCreate(&c->ev[i]);
	}
	for (int i = 0; i < 2; i++) {
		if (cudaStreamCreateWithFlags(&c->side[i], cudaStreamNonBlocking) != cudaSuccess ||
				cudaEventCreateWithFlags(&c->join_ev[i], cudaEventDisableTiming) != cudaSuccess) {
			ct_ctx_destroy((ct_ctx*) c);
			return CT_ERR_CUDA;
		}
	}
	if (cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming) != cudaSuccess) {
		ct_ctx_destroy((ct_ctx*) c);
		return CT_ERR_CUDA;
	}
	c->pinned_bytes = 1 << 16;
	if (cudaMallocHost(&c->pinned, c->pinned_bytes) != cudaSuccess) {
		delete c;
		return CT_ERR_MEMORY;
	}
	if (dalloc(c, (void**) &c->d_flags, 64 * sizeof(int), "flags") != CT_OK || dalloc(c, (void**) &c->d_counters, 32 * sizeof(double), "counters") != CT_OK) {
		ct_ctx_destroy((ct_ctx*) c);
		return CT_ERR_MEMORY;
	}
	cudaMemsetAsync(c->d_flags, 0, 64 * sizeof(int), c->stream);
	const ct_status s = ewald_init(c);
	if (s != CT_OK) {
		ct_ctx_destroy((ct_ctx*) c);
		return s;
	}
	*out = (ct_ctx*) c;
	return CT_OK;
}

void ct_ctx_destroy(ct_ctx* ctx) {
	Ctx* c = (Ctx*) ctx;
	if (!c) {
		return;
	}
	cudaSetDevice(c->device);
	if (c->stream) {
		cudaStreamSynchronize(c->stream);
	}
	for (size_t i = 0; i < c->boxes.size(); i++) {
		if (c->boxes[i]) {
			ct_box_destroy(ctx, (int) i);
		}
	}
	kick_buffers_release(c);
	for (auto& s : c->scratch) {
		dfree(c, s.p, s.bytes);
	}
	dfree(c, c->d_flags, 64 * sizeof(int));
	dfree(c, c->d_counters, 32 * sizeof(double));
	if (c->pinned) {
		cudaFreeHost(c->pinned);
	}
	for (int i = 0; i < 16; i++) {
		cudaEventDestroy(c->ev[i]);
	}
	for (int i = 0; i < 2; i++) {
		if (c->side[i]) {
			cudaStreamSynchronize(c->side[i]);
			cudaStreamDestroy(c->side[i]);
		}
		if (c->join_ev[i]) {
			cudaEventDestroy(c->join_ev[i]);
		}
	}
	if (c->fork_ev) {
		cudaEventDestroy(c->fork_ev);
	}
	if (c->stream) {
		cudaStreamSynchronize(c->stream);
	}
	if (c->pool) {
		cudaMemPoolDestroy(c->pool);  // returns the pool's memory to the CUDA driver
	}
	if (c->stream) {
		cudaStreamDestroy(c->stream);
	}
	delete c;
}

const char* ct_last_error(const ct_ctx* ctx) {
	const Ctx* c = (const Ctx*) ctx;
	return c ? c->err.c_str() : "no context";
}

unsigned long long ct_launch_count(const ct_ctx* ctx) {
	return ctx ? ((const Ctx*) ctx)->launches : 0;
}

int ct_order(const ct_ctx* ctx) {
	return ctx ? ((const Ctx*) ctx)->order : 0;
}

static ct_status box_create_impl(Ctx* c, int nsub, const int64_t* counts, int* box_id) {
	int64_t n = 0;
	for (int s = 0; s < nsub; s++) {
		if (counts[s] < 0) {
			return fail(c, CT_ERR_ARG, "negative particle count");
		}
		n += counts[s];
	}
	if (n > (int64_t) INT32_MAX / 2) {
		return fail(c, CT_ERR_ARG, "too many particles for 32-bit indices");
	}
	cudaSetDevice(c->device);
	Box* b = new (std::nothrow) Box();
	if (!b) {
		return fail(c, CT_ERR_MEMORY, "host allocation");
	}
	b->n = n;
	b->nsub = nsub;
	b->sub_off.assign(nsub + 1, 0);
	for (int s = 0; s < nsub; s++) {
		b->sub_off[s + 1] = b->sub_off[s] + counts[s];
	}
	memset(&b->counters, 0, sizeof(b->counters));
	ct_status s = dalloc(c, (void**) &b->d_sub_off, sizeof(int64_t) * (nsub + 1), "box offsets");
	if (s == CT_OK) {
		s = dalloc(c, (void**) &b->d_sub_sums, sizeof(double) * 9 * nsub, "box sums");
	}
	if (s == CT_OK) {
		s = dalloc(c, (void**) &b->d_sub_maxrung, sizeof(int) * nsub, "box max rungs");
	}
	if (s == CT_OK && cudaMemcpyAsync(b->d_sub_off, b->sub_off.data(), sizeof(int64_t) * (nsub + 1), cudaMemcpyHostToDevice, c->stream) != cudaSuccess) {
		s = fail(c, CT_ERR_CUDA, "copy of box offsets");
	}
	for (int d = 0; d < 3 && s == CT_OK; d++) {
		s = dalloc(c, (void**) &b->x[d], sizeof(uint32_t) * n, "positions");
		if (s == CT_OK) {
			s = dalloc(c, (void**) &b->v[d], sizeof(float) * n, "velocities");
		}
	}
	if (s == CT_OK) {
		s = dalloc(c, (void**) &b->rung, n + 16, "rungs");
	}
	if (s != CT_OK) {
		for (int d = 0; d < 3; d++) {
			dfree(c, b->x[d], sizeof(uint32_t) * n);
			dfree(c, b->v[d], sizeof(float) * n);
		}
		dfree(c, b->d_sub_off, sizeof(int64_t) * (nsub + 1));
		dfree(c, b->d_sub_sums, sizeof(double) * 9 * nsub);
		dfree(c, b->d_sub_maxrung, sizeof(int) * nsub);
		delete b;
		return s;
	}
	b->cap = n;
	b->sub_cap = nsub;
	int id = -1;
	for (size_t i = 0; i < c->boxes.size(); i++) {
		if (!c->boxes[i]) {
			id = (int) i;
			break;
		}
	}
	if (id < 0) {
		id = (int) c->boxes.size();
		c->boxes.push_back(nullptr);
	}
	c->boxes[id] = b;
	*box_id = id;
	return CT_OK;
}

ct_status ct_box_create(ct_ctx* ctx, int64_t n, int* box_id) {
	Ctx* c = (Ctx*) ctx;
	if (!c || n < 0 || !box_id) {
		return fail(c, CT_ERR_ARG, "ct_box_create: bad arguments");
	}
	return box_create_impl(c, 1, &n, box_id);
}

ct_status ct_ensemble_create(ct_ctx* ctx, int nbox, const int64_t* counts, int* box_id) {
	Ctx* c = (Ctx*) ctx;
	if (!c || nbox < 1 || !counts || !box_id) {
		return fail(c, CT_ERR_ARG, "ct_ensemble_create: bad arguments");
	}
	return box_create_impl(c, nbox, counts, box_id);
}

ct_status ct_ensemble_set_params(ct_ctx* ctx, int box_id, const float* h, const float* GM) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b || !h || !GM) {
		return fail(c, CT_ERR_ARG, "ct_ensemble_set_params: bad arguments");
	}
	for (int s = 0; s < b->nsub; s++) {
		if (!(h[s] > 0.f) || !(GM[s] > 0.f)) {
			return fail(c, CT_ERR_ARG, "ct_ensemble_set_params: softening and GM must be positive");
		}
	}
	cudaSetDevice(c->device);
	if (!b->d_sub_h) {
		CT_TRY(dalloc(c, (void**) &b->d_sub_h, sizeof(float) * b->sub_cap, "box softening"));
		CT_TRY(dalloc(c, (void**) &b->d_sub_GM, sizeof(float) * b->sub_cap, "box GM"));
	}
	b->sub_h_host.assign(h, h + b->nsub);
	CT_CUDA(c, cudaMemcpyAsync(b->d_sub_h, h, sizeof(float) * b->nsub, cudaMemcpyHostToDevice, c->stream));
	CT_CUDA(c, cudaMemcpyAsync(b->d_sub_GM, GM, sizeof(float) * b->nsub, cudaMemcpyHostToDevice, c->stream));
	return CT_OK;
}

// Device-to-device moves between plain boxes and the slots of an ensemble.
static ct_status ensemble_move(Ctx* c, int ens_id, const int* boxes, int count, bool gather) {
	Box* e = get_box(c, ens_id);
	if (!e || !boxes || count != e->nsub) {
		return fail(c, CT_ERR_ARG, "ensemble gather/scatter: bad arguments");
	}
	cudaSetDevice(c->device);
	cudaStream_t st = c->stream;
	for (int s = 0; s < count; s++) {
		Box* b = get_box(c, boxes[s]);
		const int64_t off = e->sub_off[s], n = e->sub_off[s + 1] - e->sub_off[s];
		if (!b || b->n != n || b->nsub != 1) {
			return fail(c, CT_ERR_ARG, "ensemble gather/scatter: box size differs from its slot");
		}
		for (int d = 0; d < 3; d++) {
			if (gather) {
				CT_CUDA(c, cudaMemcpyAsync(e->x[d] + off, b->x[d], sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
				CT_CUDA(c, cudaMemcpyAsync(e->v[d] + off, b->v[d], sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
			} else {
				CT_CUDA(c, cudaMemcpyAsync(b->x[d], e->x[d] + off, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
				CT_CUDA(c, cudaMemcpyAsync(b->v[d], e->v[d] + off, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
			}
		}
		if (gather) {
			CT_CUDA(c, cudaMemcpyAsync(e->rung + off, b->rung, n, cudaMemcpyDeviceToDevice, st));
		} else {
			CT_CUDA(c, cudaMemcpyAsync(b->rung, e->rung + off, n, cudaMemcpyDeviceToDevice, st));
			b->tree_valid = false;
			b->rung_begin = 0;
		}
	}
	if (gather) {
		e->tree_valid = false;
		e->rung_begin = 0;
	}
	return CT_OK;
}

ct_status ct_ensemble_reshape(ct_ctx* ctx, int box_id, int nbox, const int64_t* counts) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b || nbox < 1 || !counts) {
		return fail(c, CT_ERR_ARG, "ct_ensemble_reshape: bad arguments");
	}
	int64_t n = 0;
	for (int s = 0; s < nbox; s++) {
		if (counts[s] < 0) {
			return fail(c, CT_ERR_ARG, "ct_ensemble_reshape: negative particle count");
		}
		n += counts[s];
	}
	if (n > (int64_t) INT32_MAX / 2) {
		return fail(c, CT_ERR_ARG, "ct_ensemble_reshape: too many particles for 32-bit indices");
	}
	cudaSetDevice(c->device);
	CT_CUDA(c, cudaStreamSynchronize(c->stream));
	if (n > b->cap) {
		// particle arrays grow with headroom; their contents are replaced by the caller
		const int64_t cap = std::max<int64_t>(n, b->cap + b->cap / 2);
		for (int d = 0; d < 3; d++) {
			dfree(c, b->x[d], sizeof(uint32_t) * b->cap);
			dfree(c, b->v[d], sizeof(float) * b->cap);
			dfree(c, b->g[d], sizeof(float) * b->g_cap);
			b->x[d] = nullptr;
			b->g[d] = nullptr;
			b->v[d] = nullptr;
		}
		dfree(c, b->pot, sizeof(float) * b->g_cap);
		dfree(c, b->rung, b->cap + 16);
		b->pot = nullptr;
		b->rung = nullptr;
		b->g_cap = 0;
		b->cap = 0;
		for (int d = 0; d < 3; d++) {
			CT_TRY(dalloc(c, (void**) &b->x[d], sizeof(uint32_t) * cap, "positions"));
			CT_TRY(dalloc(c, (void**) &b->v[d], sizeof(float) * cap, "velocities"));
		}
		CT_TRY(dalloc(c, (void**) &b->rung, cap + 16, "rungs"));
		b->cap = cap;
	}
	if (nbox > b->sub_cap) {
		const int sc = std::max(nbox, b->sub_cap + b->sub_cap / 2);
		dfree(c, b->d_sub_off, sizeof(int64_t) * (b->sub_cap + 1));
		dfree(c, b->d_sub_sums, sizeof(double) * 9 * b->sub_cap);
		dfree(c, b->d_sub_maxrung, sizeof(int) * b->sub_cap);
		dfree(c, b->d_sub_h, sizeof(float) * b->sub_cap);
		dfree(c, b->d_sub_GM, sizeof(float) * b->sub_cap);
		dfree(c, b->d_sub_first, sizeof(int) * b->sub_cap);
		b->d_sub_off = nullptr;
		b->d_sub_sums = nullptr;
		b->d_sub_maxrung = nullptr;
		b->d_sub_h = b->d_sub_GM = nullptr;
		b->d_sub_first = nullptr;
		b->sub_cap = 0;
		CT_TRY(dalloc(c, (void**) &b->d_sub_off, sizeof(int64_t) * (sc + 1), "box offsets"));
		CT_TRY(dalloc(c, (void**) &b->d_sub_sums, sizeof(double) * 9 * sc, "box sums"));
		CT_TRY(dalloc(c, (void**) &b->d_sub_maxrung, sizeof(int) * sc, "box max rungs"));
		b->sub_cap = sc;
	}
	b->n = n;
	b->nsub = nbox;
	b->sub_off.assign(nbox + 1, 0);
	for (int s = 0; s < nbox; s++) {
		b->sub_off[s + 1] = b->sub_off[s] + counts[s];
	}
	CT_CUDA(c, cudaMemcpyAsync(b->d_sub_off, b->sub_off.data(), sizeof(int64_t) * (nbox + 1), cudaMemcpyHostToDevice, c->stream));
	// the per-box softening, GM and first-call flags of the old layout no longer apply
	if (b->d_sub_h) {
		b->sub_h_host.clear();
		dfree(c, b->d_sub_h, sizeof(float) * b->sub_cap);
		dfree(c, b->d_sub_GM, sizeof(float) * b->sub_cap);
		b->d_sub_h = b->d_sub_GM = nullptr;
	}
	if (b->d_sub_first) {
		dfree(c, b->d_sub_first, sizeof(int) * b->sub_cap);
		b->d_sub_first = nullptr;
	}
	b->rung_begin = 0;
	b->rung_stack.clear();
	b->tree_valid = false;
	b->have_force = false;
	return CT_OK;
}

ct_status ct_ensemble_set_first_call(ct_ctx* ctx, int box_id, const int* first_call) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b || !first_call) {
		return fail(c, CT_ERR_ARG, "ct_ensemble_set_first_call: bad arguments");
	}
	cudaSetDevice(c->device);
	if (!b->d_sub_first) {
		CT_TRY(dalloc(c, (void**) &b->d_sub_first, sizeof(int) * b->sub_cap, "box first-call flags"));
	}
	CT_CUDA(c, cudaMemcpyAsync(b->d_sub_first, first_call, sizeof(int) * b->nsub, cudaMemcpyHostToDevice, c->stream));
	return CT_OK;
}

ct_status ct_ensemble_gather(ct_ctx* ctx, int ens_id, const int* boxes, int count) {
	return ensemble_move((Ctx*) ctx, ens_id, boxes, count, true);
}

ct_status ct_ensemble_scatter(ct_ctx* ctx, int ens_id, const int* boxes, int count) {
	return ensemble_move((Ctx*) ctx, ens_id, boxes, count, false);
}

size_t ct_bytes_in_use(const ct_ctx* ctx) {
	return ctx ? ((const Ctx*) ctx)->used : 0;
}

int ct_box_count(const ct_ctx* ctx, int box_id) {
	Box* b = get_box((Ctx*) ctx, box_id);
	return b ? b->nsub : -1;
}

ct_status ct_box_destroy(ct_ctx* ctx, int box_id) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b) {
		return fail(c, CT_ERR_ARG, "ct_box_destroy: no such box");
	}
	cudaStreamSynchronize(c->stream);
	lightcone_release(c, b);
	const int64_t n = b->cap;
	for (int d = 0; d < 3; d++) {
		dfree(c, b->x[d], sizeof(uint32_t) * n);
		dfree(c, b->v[d], sizeof(float) * n);
		dfree(c, b->g[d], sizeof(float) * b->g_cap);
	}
	dfree(c, b->pot, sizeof(float) * b->g_cap);
	dfree(c, b->rung, n + 16);
	const int64_t cap = b->node_cap;
	dfree(c, b->nodes, sizeof(NodeW) * cap);
	dfree(c, b->nbox, sizeof(int32_t) * 6 * cap);
	dfree(c, b->multi, sizeof(float) * NMULT_STRIDE * cap);
	dfree(c, b->key, sizeof(uint64_t) * cap);
	dfree(c, b->depth, sizeof(int32_t) * cap);
	dfree(c, b->parent, sizeof(int32_t) * cap);
	dfree(c, b->gbox, sizeof(double) * 6 * cap);
	dfree(c, b->tbox, sizeof(double) * 6 * cap);
	dfree(c, b->d_sub_off, sizeof(int64_t) * (b->sub_cap + 1));
	dfree(c, b->d_sub_sums, sizeof(double) * 9 * b->sub_cap);
	dfree(c, b->d_sub_maxrung, sizeof(int) * b->sub_cap);
	dfree(c, b->d_sub_h, sizeof(float) * b->sub_cap);
	dfree(c, b->d_sub_GM, sizeof(float) * b->sub_cap);
	dfree(c, b->d_sub_first, sizeof(int) * b->sub_cap);
	delete b;
	c->boxes[box_id] = nullptr;
	return CT_OK;
}

int64_t ct_box_size(const ct_ctx* ctx, int box_id) {
	Box* b = get_box((Ctx*) ctx, box_id);
	return b ? b->n : -1;
}

static ct_status upload_impl(Ctx* c, Box* b, const uint32_t* x, const uint32_t* y, const uint32_t* z, const float* vxyz, const int8_t* rung,
		cudaMemcpyKind kind) {
	cudaStream_t st = c->stream;
	const int64_t n = b->n;
	const uint32_t* src[3] = { x, y, z };
	for (int d = 0; d < 3; d++) {
		if (src[d]) {
			CT_CUDA(c, cudaMemcpyAsync(b->x[d], src[d], sizeof(uint32_t) * n, kind, st));
		}
	}
	if (vxyz && n > 0) {
		ct_status s = CT_OK;
		float* tmp = (float*) scratch(c, 33, sizeof(float) * 3 * n, &s);
		CT_TRY(s);
		CT_CUDA(c, cudaMemcpyAsync(tmp, vxyz, sizeof(float) * 3 * n, kind, st));
		c->launches++;
		k_aos_to_soa<<<grid(c, n, 256), 256, 0, st>>>(n, tmp, b->v[0], b->v[1], b->v[2]);
	}
	if (rung) {
		CT_CUDA(c, cudaMemcpyAsync(b->rung, rung, n, kind, st));
	}
	CT_CUDA(c, cudaGetLastError());
	// particle data are replaced in place; the active range of the last ct_sort_by_rung (and
	// the hierarchical step's range stack) is kept
	b->tree_valid = false;
	return CT_OK;
}

static ct_status download_impl(Ctx* c, Box* b, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, int8_t* rung, float* gx, float* gy, float* gz,
		float* pot, cudaMemcpyKind kind) {
	cudaStream_t st = c->stream;
	const int64_t n = b->n;
	uint32_t* dst[3] = { x, y, z };
	for (int d = 0; d < 3; d++) {
		if (dst[d]) {
			CT_CUDA(c, cudaMemcpyAsync(dst[d], b->x[d], sizeof(uint32_t) * n, kind, st));
		}
	}
	if (vxyz && n > 0) {
		ct_status s = CT_OK;
		float* tmp = (float*) scratch(c, 33, sizeof(float) * 3 * n, &s);
		CT_TRY(s);
		c->launches++;
		k_soa_to_aos<<<grid(c, n, 256), 256, 0, st>>>(n, b->v[0], b->v[1], b->v[2], tmp);
		CT_CUDA(c, cudaMemcpyAsync(vxyz, tmp, sizeof(float) * 3 * n, kind, st));
	}
	if (rung) {
		CT_CUDA(c, cudaMemcpyAsync(rung, b->rung, n, kind, st));
	}
	float* gd[4] = { gx, gy, gz, pot };
	float* gs[4] = { b->g[0], b->g[1], b->g[2], b->pot };
	for (int d = 0; d < 4; d++) {
		if (gd[d]) {
			if (!gs[d]) {
				return fail(c, CT_ERR_STATE, "forces were not saved (kick with save_force first)");
			}
			CT_CUDA(c, cudaMemcpyAsync(gd[d], gs[d], sizeof(float) * n, kind, st));
		}
	}
	CT_CUDA(c, cudaStreamSynchronize(st));
	return CT_OK;
}

ct_status ct_box_upload(ct_ctx* ctx, int box_id, const uint32_t* x, const uint32_t* y, const uint32_t* z, const float* vxyz, const int8_t* rung) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b) {
		return fail(c, CT_ERR_ARG, "ct_box_upload: no such box");
	}
	cudaSetDevice(c->device);
	CT_TRY(upload_impl(c, b, x, y, z, vxyz, rung, cudaMemcpyHostToDevice));
	CT_CUDA(c, cudaStreamSynchronize(c->stream));
	return CT_OK;
}

ct_status ct_box_upload_device(ct_ctx* ctx, int box_id, const uint32_t* x, const uint32_t* y, const uint32_t* z, const float* vxyz, const int8_t* rung) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b) {
		return fail(c, CT_ERR_ARG, "ct_box_upload_device: no such box");
	}
	cudaSetDevice(c->device);
	return upload_impl(c, b, x, y, z, vxyz, rung, cudaMemcpyDeviceToDevice);
}

ct_status ct_box_download(ct_ctx* ctx, int box_id, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, int8_t* rung, float* gx, float* gy, float* gz,
		float* pot) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b) {
		return fail(c, CT_ERR_ARG, "ct_box_download: no such box");
	}
	cudaSetDevice(c->device);
	return download_impl(c, b, x, y, z, vxyz, rung, gx, gy, gz, pot, cudaMemcpyDeviceToHost);
}

ct_status ct_box_download_device(ct_ctx* ctx, int box_id, uint32_t* x, uint32_t* y, uint32_t* z, float* vxyz, int8_t* rung, float* gx, float* gy,
		float* gz, float* pot) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b) {
		return fail(c, CT_ERR_ARG, "ct_box_download_device: no such box");
	}
	cudaSetDevice(c->device);
	return download_impl(c, b, x, y, z, vxyz, rung, gx, gy, gz, pot, cudaMemcpyDeviceToDevice);
}

ct_status ct_sort_by_rung(ct_ctx* ctx, int box_id, int min_rung, int64_t* rung_begin) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b || min_rung < 0 || min_rung > 15) {
		return fail(c, CT_ERR_ARG, "ct_sort_by_rung: bad arguments");
	}
	if (b->nsub > 1 && min_rung > 0) {
		return fail(c, CT_ERR_ARG, "ct_sort_by_rung: an ensemble is kicked with all particles active (min_rung 0)");
	}
	cudaSetDevice(c->device);
	CT_TRY(sort_by_rung_run(c, b, min_rung));
	if (rung_begin) {
		*rung_begin = b->rung_begin;
	}
	return CT_OK;
}

ct_status ct_tree_create(ct_ctx* ctx, int box_id, const ct_tree_params* params, int64_t* node_count) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b || !params || params->bucket < 1 || !(params->theta > 0.0) || params->hsoft < 0.0) {
		return fail(c, CT_ERR_ARG, "ct_tree_create: bad arguments");
	}
	cudaSetDevice(c->device);
	cudaEventRecord(c->ev[8], c->stream);
	CT_TRY(tree_build(c, b, params));
	cudaEventRecord(c->ev[9], c->stream);
	cudaEventSynchronize(c->ev[9]);
	b->counters.ms_tree = elapsed_ms(c->ev[8], c->ev[9]);
	if (node_count) {
		*node_count = b->nnodes;
	}
	return CT_OK;
}

ct_status ct_kick(ct_ctx* ctx, int box_id, const ct_kick_params* params, ct_kick_return* result) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b || !params || !(params->theta > 0.f) || !(params->h > 0.f) || params->min_rung < 0 || params->min_rung > 15) {
		return fail(c, CT_ERR_ARG, "ct_kick: bad arguments");
	}
	if (!b->tree_valid) {
		return fail(c, CT_ERR_STATE, "ct_kick: no valid tree (call ct_tree_create after every upload/drift/sort)");
	}
	if (std::fabs((double) params->theta - b->tparams.theta) > 1e-6 * b->tparams.theta) {
		return fail(c, CT_ERR_ARG, "ct_kick: theta differs from the one the tree was built with");
	}
	cudaSetDevice(c->device);
	if (params->save_force && (!b->pot || b->g_cap < b->n)) {
		for (int d = 0; d < 3; d++) {
			dfree(c, b->g[d], sizeof(float) * b->g_cap);
			b->g[d] = nullptr;
		}
		dfree(c, b->pot, sizeof(float) * b->g_cap);
		b->pot = nullptr;
		b->g_cap = 0;
		for (int d = 0; d < 3; d++) {
			CT_TRY(dalloc(c, (void**) &b->g[d], sizeof(float) * b->cap, "forces"));
		}
		CT_TRY(dalloc(c, (void**) &b->pot, sizeof(float) * b->cap, "potentials"));
		b->g_cap = b->cap;
	}
	return kick_run(c, b, params, result);
}

ct_status ct_kick_ensemble(ct_ctx* ctx, int box_id, const ct_kick_params* params, ct_kick_return* results) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b || !results) {
		return fail(c, CT_ERR_ARG, "ct_kick_ensemble: bad arguments");
	}
	ct_kick_return total;
	CT_TRY(ct_kick(ctx, box_id, params, &total));
	if (b->nsub == 1) {
		results[0] = total;
		return CT_OK;
	}
	std::vector<double> sums(9 * b->nsub);
	std::vector<int> mr(b->nsub);
	CT_CUDA(c, cudaMemcpyAsync(sums.data(), b->d_sub_sums, sizeof(double) * 9 * b->nsub, cudaMemcpyDeviceToHost, c->stream));
	CT_CUDA(c, cudaMemcpyAsync(mr.data(), b->d_sub_maxrung, sizeof(int) * b->nsub, cudaMemcpyDeviceToHost, c->stream));
	CT_CUDA(c, cudaStreamSynchronize(c->stream));
	for (int s = 0; s < b->nsub; s++) {
		ct_kick_return& r = results[s];
		const double* q = sums.data() + 9 * s;
		r.pot = q[0];
		r.kin = q[1];
		r.dkin = q[2];
		r.xmom = q[3];
		r.ymom = q[4];
		r.zmom = q[5];
		r.nmom = q[6];
		r.max_rung = mr[s];
	}
	return CT_OK;
}

ct_status ct_drift(ct_ctx* ctx, int box_id, int rung, float a, float dt, double drag) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b || !(a > 0.f) || rung < 0 || rung > 127) {
		return fail(c, CT_ERR_ARG, "ct_drift: bad arguments");
	}
	cudaSetDevice(c->device);
	CT_TRY(drift_run(c, b, rung, a, dt, drag));
	return CT_OK;
}

ct_status ct_tree_download(ct_ctx* ctx, int box_id, ct_node* nodes, int64_t max_nodes, int64_t* count) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b || !count) {
		return fail(c, CT_ERR_ARG, "ct_tree_download: bad arguments");
	}
	if (!b->tree_valid) {
		return fail(c, CT_ERR_STATE, "ct_tree_download: no valid tree");
	}
	*count = b->nnodes;
	if (!nodes) {
		return CT_OK;
	}
	if (max_nodes < b->nnodes) {
		return fail(c, CT_ERR_ARG, "ct_tree_download: output too small");
	}
	cudaSetDevice(c->device);
	const int64_t nn = b->nnodes;
	std::vector<NodeW> w(nn);
	std::vector<int32_t> bx(6 * nn), dep(nn);
	std::vector<float> mu(NMULT_STRIDE * nn);
	std::vector<uint64_t> key(nn);
	cudaStream_t st = c->stream;
	CT_CUDA(c, cudaMemcpyAsync(w.data(), b->nodes, sizeof(NodeW) * nn, cudaMemcpyDeviceToHost, st));
	CT_CUDA(c, cudaMemcpyAsync(bx.data(), b->nbox, sizeof(int32_t) * 6 * nn, cudaMemcpyDeviceToHost, st));
	CT_CUDA(c, cudaMemcpyAsync(dep.data(), b->depth, sizeof(int32_t) * nn, cudaMemcpyDeviceToHost, st));
	CT_CUDA(c, cudaMemcpyAsync(mu.data(), b->multi, sizeof(float) * NMULT_STRIDE * nn, cudaMemcpyDeviceToHost, st));
	CT_CUDA(c, cudaMemcpyAsync(key.data(), b->key, sizeof(uint64_t) * nn, cudaMemcpyDeviceToHost, st));
	CT_CUDA(c, cudaStreamSynchronize(st));
	const int nm = c->order == 5 ? 17 : 37;
	for (int64_t i = 0; i < nn; i++) {
		ct_node& o = nodes[i];
		memset(&o, 0, sizeof(o));
		o.key = key[i];
		o.part_begin = w[i].pbeg;
		o.part_end = w[i].pend;
		o.child_left = w[i].child;
		o.child_right = w[i].child >= 0 ? w[i].child + 1 : -1;
		o.pos[0] = w[i].x;
		o.pos[1] = w[i].y;
		o.pos[2] = w[i].z;
		o.radius = w[i].radius;
		for (int d = 0; d < 3; d++) {
			o.box_begin[d] = bx[6 * i + d];
			o.box_end[d] = bx[6 * i + 3 + d];
		}
		o.leaf = w[i].flags & 1;
		o.depth = dep[i];
		for (int k = 0; k < nm; k++) {
			o.multi[k] = mu[NMULT_STRIDE * i + k];
		}
	}
	return CT_OK;
}

ct_status ct_get_counters(ct_ctx* ctx, int box_id, ct_counters* out) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b || !out) {
		return fail(c, CT_ERR_ARG, "ct_get_counters: bad arguments");
	}
	if (c->drift_timed && cudaEventQuery(c->ev[7]) == cudaSuccess) {
		b->counters.ms_drift = elapsed_ms(c->ev[6], c->ev[7]);
	}
	*out = b->counters;
	return CT_OK;
}

ct_status ct_synchronize(ct_ctx* ctx) {
	Ctx* c = (Ctx*) ctx;
	if (!c) {
		return CT_ERR_ARG;
	}
	CT_CUDA(c, cudaStreamSynchronize(c->stream));
	return CT_OK;
}

ct_status ct_ctx_set_compensated(ct_ctx* ctx, int compensated) {
	Ctx* c = (Ctx*) ctx;
	if (!c) {
		return CT_ERR_ARG;
	}
	c->compensated = compensated != 0;
	return CT_OK;
}

ct_status ct_ctx_set_priority(ct_ctx* ctx, int priority) {
	Ctx* c = (Ctx*) ctx;
	if (!c) {
		return CT_ERR_ARG;
	}
	cudaSetDevice(c->device);
	int least = 0, greatest = 0;
	CT_CUDA(c, cudaDeviceGetStreamPriorityRange(&least, &greatest));
	const int p = std::min(least, std::max(greatest, priority));  // greatest is the numerically smallest
	if (p == c->priority) {
		return CT_OK;
	}
	// new streams first (on failure the context keeps its old ones), then drain and swap
	cudaStream_t ns[3] = { nullptr, nullptr, nullptr };
	for (int i = 0; i < 3; i++) {
		if (cudaStreamCreateWithPriority(&ns[i], cudaStreamNonBlocking, p) != cudaSuccess) {
			for (int k = 0; k < i; k++) {
				cudaStreamDestroy(ns[k]);
			}
			return fail(c, CT_ERR_CUDA, "cudaStreamCreateWithPriority failed");
		}
	}
	cudaStream_t old[3] = { c->stream, c->side[0], c->side[1] };
	for (int i = 0; i < 3; i++) {
		cudaStreamSynchronize(old[i]);
	}
	c->stream = ns[0];
	c->side[0] = ns[1];
	c->side[1] = ns[2];
	for (int i = 0; i < 3; i++) {
		cudaStreamDestroy(old[i]);
	}
	c->priority = p;
	return CT_OK;
}

ct_status ct_ctx_set_tuning(ct_ctx* ctx, const ct_tuning* t) {
	Ctx* c = (Ctx*) ctx;
	if (!c || !t) {
		return CT_ERR_ARG;
	}
	const bool ok = (t->p2p_stage == 64 || t->p2p_stage == 128 || t->p2p_stage == 256) && (t->warps_per_tile == 1 || t->warps_per_tile == 2) &&
			(t->tile_width == 16 || t->tile_width == 32);
	if (!ok) {
		return fail(c, CT_ERR_ARG, "ct_ctx_set_tuning: p2p_stage 64/128/256, warps_per_tile 1/2, tile_width 16/32");
	}
	c->tune = *t;
	return CT_OK;
}

ct_status ct_ctx_get_tuning(const ct_ctx* ctx, ct_tuning* t) {
	const Ctx* c = (const Ctx*) ctx;
	if (!c || !t) {
		return CT_ERR_ARG;
	}
	*t = c->tune;
	return CT_OK;
}

ct_status ct_fp32_peak(ct_ctx* ctx, double* tflops) {
	Ctx* c = (Ctx*) ctx;
	if (!c || !tflops) {
		return CT_ERR_ARG;
	}
	cudaSetDevice(c->device);
	ct_status s = CT_OK;
	float* out = (float*) scratch(c, 34, 1024 * sizeof(float), &s);
	CT_TRY(s);
	const int blocks = c->nsm * 8, iters = 8192;
	double best = 0.0;
	for (int rep = 0; rep < 4; rep++) {
		cudaEventRecord(c->ev[10], c->stream);
		c->launches++;
		k_fma_peak<<<blocks, 256, 0, c->stream>>>(out, iters, 0.9999999f, 1e-7f);
		cudaEventRecord(c->ev[11], c->stream);
		CT_CUDA(c, cudaEventSynchronize(c->ev[11]));
		const float ms = elapsed_ms(c->ev[10], c->ev[11]);
		const double fl = 2.0 * 16.0 * iters * 256.0 * blocks;
		if (rep > 0) {
			best = std::max(best, fl / (ms * 1e-3) / 1e12);
		}
	}
	*tflops = best;
	return CT_OK;
}

void* ct_stream(ct_ctx* ctx) {
	return ctx ? (void*) ((Ctx*) ctx)->stream : nullptr;
}

ct_status ct_direct_ewald(ct_ctx* ctx, int box_id, int64_t nsink, const uint32_t* sx, const uint32_t* sy, const uint32_t* sz, double h, double* gx,
		double* gy, double* gz, double* pot) {
	Ctx* c = (Ctx*) ctx;
	Box* b = get_box(c, box_id);
	if (!b || nsink <= 0 || !sx || !sy || !sz || !gx || !gy || !gz || !pot || !(h > 0.0)) {
		return fail(c, CT_ERR_ARG, "ct_direct_ewald: bad arguments");
	}
	cudaSetDevice(c->device);
	return direct_ewald_run(c, b, nsink, sx, sy, sz, h, gx, gy, gz, pot);
}

}  // extern "C"
