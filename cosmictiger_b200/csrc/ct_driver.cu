// One hierarchical (multistep) gravity step: the rung ladder of kick_step_hierarchical
// (src/driver.cpp:382-593) as a host loop over the box's device-resident state.
//
// The ladder visits rungs from the highest present down to min_rung ("ascending": closing
// half kicks of the finer sub-steps) and back up ("descending": opening half kicks, rung
// assignment, drift of each rung).  Each visit sorts the active range by rung
// (particles_sort_by_rung), builds the tree over the active particles only, kicks them and,
// when descending, drifts the rung.  The active-range stack (particles_push/pop_rungs,
// src/particles.cpp:218-235) persists between steps in the box.  The top-level clip
// (driver.cpp:442-462): when more than a quarter of the particles sit above the base rung, the
// base rung is raised for the rest of the run.
#include <algorithm>
#include <vector>

#include "ct_internal.cuh"

namespace ct {
namespace {

__global__ void k_rung_hist(int64_t n, const int8_t* rung, unsigned long long* hist) {
	__shared__ unsigned long long sh[16];
	if (threadIdx.x < 16) {
		sh[threadIdx.x] = 0;
	}
	__syncthreads();
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		const int r = rung[i];
		atomicAdd(&sh[r < 0 ? 0 : (r > 15 ? 15 : r)], 1ull);
	}
	__syncthreads();
	if (threadIdx.x < 16 && sh[threadIdx.x]) {
		atomicAdd(hist + threadIdx.x, sh[threadIdx.x]);
	}
}

// particles_set_minrung (src/particles.cpp:628-648): rung = max(rung, minrung)
__global__ void k_set_minrung(int64_t n, int8_t* rung, int minrung) {
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		if (rung[i] < minrung) {
			rung[i] = (int8_t) minrung;
		}
	}
}

int grid_of(Ctx* c, int64_t n) {
	return (int) std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t) c->nsm * 8));
}

}  // namespace

ct_status rung_counts(Ctx* c, Box* b, uint64_t* counts) {
	ct_status s = CT_OK;
	unsigned long long* d = (unsigned long long*) scratch(c, 50, 16 * sizeof(unsigned long long), &s);
	CT_TRY(s);
	CT_CUDA(c, cudaMemsetAsync(d, 0, 16 * sizeof(unsigned long long), c->stream));
	c->launches++;
	k_rung_hist<<<grid_of(c, b->n), 256, 0, c->stream>>>(b->n, b->rung, d);
	CT_CUDA(c, cudaMemcpyAsync(counts, d, 16 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
	CT_CUDA(c, cudaStreamSynchronize(c->stream));
	return CT_OK;
}

ct_status step_hierarchical(Ctx* c, Box* b, const ct_step_params* p, ct_step_return* out) {
	if (b->nsub != 1) {
		return fail(c, CT_ERR_ARG, "ct_step_hierarchical: runs on a single box");
	}
	int minrung = p->minrung;
	int max_rung = std::max(p->max_rung, minrung);
	std::vector<int> levels;
	for (int i = max_rung; i > minrung; i--) {
		levels.push_back(i);
	}
	levels.push_back(minrung);
	bool ascending = true;
	bool clip_top = false;
	ct_step_return R;
	memset(&R, 0, sizeof(R));
	for (size_t li = 0; li < levels.size(); li++) {
		const int level = levels[li];
		bool top = false;
		if (level == minrung) {
			ascending = false;
			top = true;
		}
		if (!ascending && !top) {
			b->rung_stack.push_back(b->rung_begin);  // particles_push_rungs
		}
		if (!ascending) {
			CT_TRY(sort_by_rung_run(c, b, level));
		}
		R.particles_kicked += (double) (b->n - b->rung_begin);
		if (top && minrung == p->minrung0) {
			uint64_t counts[16];
			CT_TRY(rung_counts(c, b, counts));
			int maxr = 0;
			for (int k = 0; k < 16; k++) {
				if (counts[k]) {
					maxr = k;
				}
			}
			if (maxr > p->minrung0) {
				uint64_t fast = 0;
				const uint64_t slow = counts[p->minrung0];
				for (int k = p->minrung0 + 1; k < 16; k++) {
					fast += counts[k];
				}
				if (3 * fast > slow) {
					clip_top = !p->nocrop;
				}
			}
		}
		ct_tree_params tp;
		tp.min_rung = level;
		tp.theta = p->theta;
		tp.hsoft = p->hsoft;
		tp.bucket = p->bucket;
		CT_TRY(tree_build(c, b, &tp));
		ct_kick_params kp;
		memset(&kp, 0, sizeof(kp));
		kp.top = (clip_top && level == p->minrung0 + 1) ? 1 : top;
		kp.sign = p->sign;
		kp.ascending = ascending || top;
		kp.descending = (clip_top && top) ? 0 : (!ascending || top);
		kp.save_force = 0;
		kp.GM = p->GM;
		kp.eta = p->eta;
		kp.h = (float) p->hsoft;
		kp.a = (float) p->a;
		kp.first_call = p->tau == 0.0;
		kp.min_rung = level;
		kp.do_phi = p->do_phi && top;
		kp.t0 = (float) p->t0;
		kp.max_dt = p->max_dt;
		kp.theta = (float) p->theta;
		ct_kick_return kr;
		CT_TRY(kick_run(c, b, &kp, &kr));
		R.kicks++;
		if (clip_top && top) {
			c->launches++;
			k_set_minrung<<<grid_of(c, b->n), 256, 0, c->stream>>>(b->n, b->rung, p->minrung0 + 1);
			CT_CUDA(c, cudaGetLastError());
		}
		if (top) {
			R.kr = kr;
		}
		if (clip_top && top) {
			levels.push_back(p->minrung0 + 1);
		} else if (!ascending || top) {
			max_rung = kr.max_rung;
			R.kr.max_rung = max_rung;
			if (max_rung > level) {
				levels.push_back(level + 1);
			}
		}
		if ((!ascending || top) && !(clip_top && top)) {
			const double dt = (1.0 / double(1 << level)) * p->t0;  // rung_dt[level] * t0
			CT_TRY(drift_run(c, b, level, (float) p->a, (float) dt, p->drag));
			R.particles_drifted_levels++;
		}
		if (ascending && !top) {
			if (b->rung_stack.empty()) {
				return fail(c, CT_ERR_STATE, "ct_step_hierarchical: rung stack underflow (max_rung above the previous step's rungs)");
			}
			b->rung_begin = b->rung_stack.back();  // particles_pop_rungs
			b->rung_stack.pop_back();
		}
	}
	if (clip_top) {
		minrung++;
	}
	R.minrung = minrung;
	R.max_rung = max_rung;
	b->tree_valid = false;
	if (out) {
		*out = R;
	}
	return CT_OK;
}

}  // namespace ct

using namespace ct;

extern "C" ct_status ct_rung_counts(ct_ctx* ctx, int box_id, uint64_t* counts) {
	Ctx* c = (Ctx*) ctx;
	if (!c || box_id < 0 || box_id >= (int) c->boxes.size() || !c->boxes[box_id] || !counts) {
		return fail(c, CT_ERR_ARG, "ct_rung_counts: bad arguments");
	}
	cudaSetDevice(c->device);
	return rung_counts(c, c->boxes[box_id], counts);
}

extern "C" ct_status ct_box_get_rung_state(ct_ctx* ctx, int box_id, int64_t* rung_begin, int64_t* stack, int* depth) {
	Ctx* c = (Ctx*) ctx;
	if (!c || box_id < 0 || box_id >= (int) c->boxes.size() || !c->boxes[box_id] || !depth) {
		return fail(c, CT_ERR_ARG, "ct_box_get_rung_state: bad arguments");
	}
	const Box* b = c->boxes[box_id];
	if (rung_begin) {
		*rung_begin = b->rung_begin;
	}
	if (stack) {
		if (*depth < (int) b->rung_stack.size()) {
			return fail(c, CT_ERR_ARG, "ct_box_get_rung_state: stack buffer too small");
		}
		for (size_t i = 0; i < b->rung_stack.size(); i++) {
			stack[i] = b->rung_stack[i];
		}
	}
	*depth = (int) b->rung_stack.size();
	return CT_OK;
}

extern "C" ct_status ct_box_set_rung_state(ct_ctx* ctx, int box_id, int64_t rung_begin, const int64_t* stack, int depth) {
	Ctx* c = (Ctx*) ctx;
	if (!c || box_id < 0 || box_id >= (int) c->boxes.size() || !c->boxes[box_id] || depth < 0 || (depth > 0 && !stack)) {
		return fail(c, CT_ERR_ARG, "ct_box_set_rung_state: bad arguments");
	}
	Box* b = c->boxes[box_id];
	if (rung_begin < 0 || rung_begin > b->n) {
		return fail(c, CT_ERR_ARG, "ct_box_set_rung_state: active range start outside the box");
	}
	for (int i = 0; i < depth; i++) {
		if (stack[i] < 0 || stack[i] > b->n) {
			return fail(c, CT_ERR_ARG, "ct_box_set_rung_state: saved range start outside the box");
		}
	}
	b->rung_begin = rung_begin;
	b->rung_stack.assign(stack, stack + depth);
	b->tree_valid = false;
	return CT_OK;
}

extern "C" ct_status ct_step_hierarchical(ct_ctx* ctx, int box_id, const ct_step_params* params, ct_step_return* result) {
	Ctx* c = (Ctx*) ctx;
	if (!c || box_id < 0 || box_id >= (int) c->boxes.size() || !c->boxes[box_id] || !params) {
		return fail(c, CT_ERR_ARG, "ct_step_hierarchical: bad arguments");
	}
	if (params->minrung < 0 || params->minrung > 15 || params->max_rung > 15 || !(params->theta > 0) || !(params->hsoft > 0) || params->bucket < 1) {
		return fail(c, CT_ERR_ARG, "ct_step_hierarchical: bad parameters");
	}
	cudaSetDevice(c->device);
	Box* b = c->boxes[box_id];
	cudaEventRecord(c->ev[13], c->stream);
	const ct_status s = step_hierarchical(c, b, params, result);
	cudaEventRecord(c->ev[14], c->stream);
	return s;
}
