// Rung partition without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need the rung
// partition: a host driver that runs inside a memory pool it does not own, an embedding
// application whose allocator forbids cudaMalloc/cudaFree on its hot path, or code that must
// keep the device footprint fixed after start-up.  For them this file provides
// ct_sort_by_rung_noalloc: the same exact partition as ct_sort_by_rung (particles with
// rung < min_rung first, the reference's two-pointer permutation), on arrays the caller
// already holds on the device, with all temporary storage in one file-scope __device__ array.
//
// The array (g_rung_scratch) is part of the library image: every GPU that loads the library
// holds it until the process exits.  Host code must not pass the symbol itself to a kernel
// (on the host it names a stand-in, not device memory); its device address is obtained once
// per device with cudaGetSymbolAddress and cached.
#include <cub/cub.cuh>

#include <cstdio>
#include <mutex>

#include "ct_internal.cuh"

namespace {

constexpr int64_t kMaxParticles = CT_NOALLOC_MAX_PARTICLES;
constexpr size_t kCubBytes = size_t(1) << 20;                                  // CUB temporary storage
constexpr size_t kArrayBytes = sizeof(int) * (size_t) kMaxParticles;          // one int per particle
constexpr size_t kScratchBytes = 4 * kArrayBytes + kCubBytes + 256;           // exL, exR, posL, posR, CUB, counters

static __device__ __align__(256) unsigned char g_rung_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = { nullptr };

// Device address of g_rung_scratch on the current device (set up on first use per device).
ct_status scratch_address(unsigned char** out) {
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
		return CT_ERR_CUDA;
	}
	std::lock_guard<std::mutex> lock(g_mutex);
	if (!g_scratch_addr[dev]) {
		void* p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_rung_scratch);
		if (e != cudaSuccess || !p) {
			fprintf(stderr, "ct_sort_by_rung_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
			return CT_ERR_CUDA;
		}
		g_scratch_addr[dev] = (unsigned char*) p;
	}
	*out = g_scratch_addr[dev];
	return CT_OK;
}

struct BelowRung {
	const int8_t* rung;
	int min_rung;
	__host__ __device__ int operator()(int64_t i) const {
		return rung[i] < min_rung;
	}
};

// Misplaced elements relative to the split s = begin + m: left side holding rung >= min_rung,
// or right side holding rung < min_rung.
struct Misplaced {
	const int8_t* rung;
	int min_rung;
	int64_t begin;
	const int* m;
	int right;
	__host__ __device__ int operator()(int64_t i) const {
		const int64_t s = begin + *m;
		const int64_t p = begin + i;
		const bool lt = rung[p] < min_rung;
		return right ? (p >= s && lt) : (p < s && !lt);
	}
};

__global__ void k_na_positions(int64_t begin, int64_t cnt, const int8_t* rung, int min_rung, const int* m, const int* exL, const int* exR,
		const int* totR, int* posL, int* posR) {
	const int64_t s = begin + *m;
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < cnt; i += (int64_t) gridDim.x * blockDim.x) {
		const int64_t p = begin + i;
		const bool lt = rung[p] < min_rung;
		// offsets from begin (below the 2^20 capacity), so that no index wraps however far
		// into the caller's arrays the range starts
		if (p < s && !lt) {
			posL[exL[i]] = (int) i;
		}
		if (p >= s && lt) {
			posR[*totR - 1 - exR[i]] = (int) i;
		}
	}
}

__global__ void k_na_swap(int64_t begin, const int* posL, const int* posR, const int* nmis, uint32_t* x, uint32_t* y, uint32_t* z, float* vx,
		float* vy, float* vz, int8_t* rung) {
	const int n = *nmis;
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
		const int64_t a = begin + posL[k], b = begin + posR[k];
		uint32_t t = x[a];
		x[a] = x[b];
		x[b] = t;
		t = y[a];
		y[a] = y[b];
		y[b] = t;
		t = z[a];
		z[a] = z[b];
		z[b] = t;
		float f = vx[a];
		vx[a] = vx[b];
		vx[b] = f;
		f = vy[a];
		vy[a] = vy[b];
		vy[b] = f;
		f = vz[a];
		vz[a] = vz[b];
		vz[b] = f;
		const int8_t r = rung[a];
		rung[a] = rung[b];
		rung[b] = r;
	}
}

}  // namespace

extern "C" ct_status ct_sort_by_rung_noalloc(int64_t begin, int64_t n, int min_rung, uint32_t* x, uint32_t* y, uint32_t* z, float* vx, float* vy,
		float* vz, int8_t* rung, int64_t* rung_begin, void* stream) {
	if (!rung_begin || begin < 0 || n < begin || min_rung < 0 || min_rung > 15) {
		return CT_ERR_ARG;
	}
	if (min_rung == 0) {
		// particles_sort_by_rung(0) resets the active range to all particles (particles.cpp:1035)
		*rung_begin = 0;
		return CT_OK;
	}
	const int64_t cnt = n - begin;
	if (cnt > kMaxParticles) {
		fprintf(stderr, "ct_sort_by_rung_noalloc: %lld particles exceed the fixed scratch capacity of %lld\n", (long long) cnt, (long long) kMaxParticles);
		return CT_ERR_CAPACITY;
	}
	if (cnt == 0) {
		*rung_begin = begin;
		return CT_OK;
	}
	if (!x || !y || !z || !vx || !vy || !vz || !rung) {
		return CT_ERR_ARG;
	}
	unsigned char* base = nullptr;
	const ct_status s0 = scratch_address(&base);
	if (s0 != CT_OK) {
		return s0;
	}
	cudaStream_t st = (cudaStream_t) stream;
	int* exL = (int*) base;
	int* exR = (int*) (base + kArrayBytes);
	int* posL = (int*) (base + 2 * kArrayBytes);
	int* posR = (int*) (base + 3 * kArrayBytes);
	void* cub_tmp = base + 4 * kArrayBytes;
	int* counters = (int*) (base + 4 * kArrayBytes + kCubBytes);  // [0] m, [1] misplaced-left, [2] misplaced-right
	cub::CountingInputIterator<int64_t> idx(0);
	cub::TransformInputIterator<int, BelowRung, cub::CountingInputIterator<int64_t>> below(idx, BelowRung { rung + begin, min_rung });
	cub::TransformInputIterator<int, Misplaced, cub::CountingInputIterator<int64_t>> misL(idx, Misplaced { rung, min_rung, begin, counters, 0 });
	cub::TransformInputIterator<int, Misplaced, cub::CountingInputIterator<int64_t>> misR(idx, Misplaced { rung, min_rung, begin, counters, 1 });
	size_t need = 0, b1 = 0, b2 = 0;
	if (cub::DeviceReduce::Sum(nullptr, b1, below, counters, (int) cnt, st) != cudaSuccess ||
			cub::DeviceScan::ExclusiveSum(nullptr, b2, misL, exL, (int) cnt, st) != cudaSuccess) {
		return CT_ERR_CUDA;
	}
	need = b1 > b2 ? b1 : b2;
	if (need > kCubBytes) {
		return CT_ERR_CAPACITY;
	}
	size_t tb = kCubBytes;
	cudaError_t e = cub::DeviceReduce::Sum(cub_tmp, tb, below, counters, (int) cnt, st);
	tb = kCubBytes;
	if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(cub_tmp, tb, misL, exL, (int) cnt, st);
	tb = kCubBytes;
	if (e == cudaSuccess) e = cub::DeviceReduce::Sum(cub_tmp, tb, misL, counters + 1, (int) cnt, st);
	tb = kCubBytes;
	if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(cub_tmp, tb, misR, exR, (int) cnt, st);
	tb = kCubBytes;
	if (e == cudaSuccess) e = cub::DeviceReduce::Sum(cub_tmp, tb, misR, counters + 2, (int) cnt, st);
	if (e != cudaSuccess) {
		return CT_ERR_CUDA;
	}
	const int grid = (int) ((cnt + 255) / 256 < 4096 ? (cnt + 255) / 256 : 4096);
	k_na_positions<<<grid, 256, 0, st>>>(begin, cnt, rung, min_rung, counters, exL, exR, counters + 2, posL, posR);
	k_na_swap<<<grid, 256, 0, st>>>(begin, posL, posR, counters + 1, x, y, z, vx, vy, vz, rung);
	int m = 0;
	e = cudaGetLastError();
	if (e == cudaSuccess) e = cudaMemcpyAsync(&m, counters, sizeof(int), cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess) e = cudaStreamSynchronize(st);
	if (e != cudaSuccess) {
		return CT_ERR_CUDA;
	}
	*rung_begin = begin + m;
	return CT_OK;
}
