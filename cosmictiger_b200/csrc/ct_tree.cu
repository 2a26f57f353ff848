// Tree construction on the device, level by level (compiled with -fmad=false so that every
// float/double expression is evaluated exactly as written, matching the reference's C++).
//
// Reference: tree_create (src/tree.cpp:273-601) builds the tree recursively on the host,
// splitting each node at the midpoint of its box's longest dimension with the in-place
// two-pointer partition particles_sort (src/particles.cpp:979-1018).  Here all nodes of one
// depth are split together:
//   1. classify: leaf or split, split dimension and midpoint (tree.cpp:314-348);
//   2. partition every split node's range with the exact permutation of the two-pointer
//      loop: with m = #(x < xmid), the k-th element >= xmid in [b, b+m) (counted from the left)
//      swaps with the k-th element < xmid in [b+m, e) (counted from the right);
//   3. create the children.
// The upsweep then runs deepest level first: leaf tight boxes, centres, radii and P2M
// (tree.cpp:498-571), interior unions, the two centre/radius candidates and M2M in double
// (tree.cpp:355-497).  Particles are reordered by moving x, y, z and an index; velocities
// and rungs are gathered through the index at the end (same final arrays as swapping all
// fields in the reference's loop).
#include <cub/cub.cuh>

#include "ct_internal.cuh"
#include "ct_ops.cuh"

namespace ct {
namespace {

constexpr int TPB = 256;
constexpr int PER_T = 8;
constexpr int TILE = TPB * PER_T;

struct BuildScratch {
	int32_t* idx;        // particle index being permuted [n]
	int32_t* posL;       // partition scratch [n]
	int32_t* posR;       // partition scratch [n]
	int32_t* split;      // per node of the level: 1 if split
	int32_t* rank;       // exclusive scan of split
	int32_t* ntiles;     // tiles per node of the level
	int32_t* tile_off;   // exclusive scan of ntiles
	int32_t* xdim;       // split dimension per node of the level
	uint32_t* xmidf;     // fixed32 midpoint per node of the level
	double* xmid;        // double midpoint per node of the level
	int32_t* node_m;     // # below midpoint per node of the level
	int32_t* node_nmis;  // # swaps per node of the level
	int32_t* tile_node;  // per tile: node (local index in level)
	int32_t* tile_lt;    // per tile: # below midpoint
	int32_t* tile_offL;  // per tile: # misplaced-left in earlier tiles of the node
	int32_t* tile_offR;  // per tile: # misplaced-right in later tiles of the node
	int32_t* totals;     // [0] nsplit, [1] ntiles (device)
	void* cub_tmp;
	size_t cub_bytes;
};

__device__ __forceinline__ int block_sum_int(int v, int* sh) {
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	for (int o = 16; o; o >>= 1) {
		v += __shfl_down_sync(0xffffffffu, v, o);
	}
	__syncthreads();
	if (lane == 0) {
		sh[w] = v;
	}
	__syncthreads();
	int t = 0;
	for (int i = 0; i < (int) (blockDim.x >> 5); i++) {
		t += sh[i];
	}
	__syncthreads();
	return t;
}

// Exclusive block scan of ints; returns the block total through *total.
__device__ __forceinline__ int block_excl_scan(int v, int* sh, int* total) {
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	int inc = v;
	for (int o = 1; o < 32; o <<= 1) {
		const int t = __shfl_up_sync(0xffffffffu, inc, o);
		if (lane >= o) {
			inc += t;
		}
	}
	__syncthreads();
	if (lane == 31) {
		sh[w] = inc;
	}
	__syncthreads();
	int base = 0, tot = 0;
	for (int i = 0; i < (int) (blockDim.x >> 5); i++) {
		if (i < w) {
			base += sh[i];
		}
		tot += sh[i];
	}
	__syncthreads();
	*total = tot;
	return base + inc - v;
}

// One root per sub-box: node s covers the unit box and particles [off[s], off[s+1]), except
// that a single box starts at the active range [pbeg, pend).
__global__ void k_init_roots(int nroot, const int64_t* off, NodeW* nodes, double* gbox, uint64_t* key, int32_t* depth, int32_t* parent, int32_t pbeg,
		int32_t pend) {
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= nroot) {
		return;
	}
	NodeW r;
	r.x = r.y = r.z = 0;
	r.radius = 0.f;
	r.pbeg = nroot == 1 ? pbeg : (int32_t) off[s];
	r.pend = nroot == 1 ? pend : (int32_t) off[s + 1];
	r.child = -1;
	r.flags = 1;
	nodes[s] = r;
	for (int d = 0; d < 3; d++) {
		gbox[6 * s + d] = 0.0;
		gbox[6 * s + 3 + d] = 1.0;
	}
	key[s] = 1;
	depth[s] = 0;
	parent[s] = -1;
}

__global__ void k_iota(int32_t* idx, int64_t n) {
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		idx[i] = (int32_t) i;
	}
}

// Leaf or split (tree.cpp:314-348).
__global__ void k_classify(int64_t lb, int nl, const NodeW* nodes, const double* gbox, const int32_t* depth, double theta, double hsoft, int bucket,
		BuildScratch s, int* flags) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nl; i += gridDim.x * blockDim.x) {
		const int64_t ni = lb + i;
		const NodeW nd = nodes[ni];
		const int nparts = nd.pend - nd.pbeg;
		const double* gb = gbox + 6 * ni;
		float box_r = 0.0f;
		for (int dim = 0; dim < 3; dim++) {
			const double h = 0.5 * (gb[3 + dim] - gb[dim]);
			box_r += h * h;
		}
		box_r = sqrtf(box_r);
		const bool ewald_satisfied = (box_r < 0.25 * (theta / (1.0 + theta)) && box_r < 0.125 - 0.25 * hsoft);
		bool split = nparts > bucket || (!ewald_satisfied && nparts > 0);
		if (split && depth[ni] >= MAX_DEPTH - 1) {
			atomicOr(flags + 2, 1);
			split = false;
		}
		int xdim = 0;
		double max_span = -1.0;
		for (int dim = 0; dim < 3; dim++) {
			const double span = gb[3 + dim] - gb[dim];
			if (span > max_span) {
				max_span = span;
				xdim = dim;
			}
		}
		const double xm = 0.5 * (gb[3 + xdim] + gb[xdim]);
		s.split[i] = split;
		s.ntiles[i] = split ? (nparts + TILE - 1) / TILE : 0;
		s.xdim[i] = xdim;
		s.xmid[i] = xm;
		s.xmidf[i] = fixed_from_double(xm);
	}
}

__global__ void k_tile_map(int nl, BuildScratch s) {
	const int lane = threadIdx.x & 31;
	const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int nw = (gridDim.x * blockDim.x) >> 5;
	for (int i = wid; i < nl; i += nw) {
		const int nt = s.ntiles[i];
		const int t0 = s.tile_off[i];
		for (int t = lane; t < nt; t += 32) {
			s.tile_node[t0 + t] = i;
		}
	}
}

__device__ __forceinline__ void tile_range(const NodeW& nd, int t, int t0, int* tb, int* te) {
	*tb = nd.pbeg + (t - t0) * TILE;
	*te = min(*tb + TILE, nd.pend);
}

// P1: elements below the midpoint per tile.
__global__ void __launch_bounds__(TPB) k_count(int64_t lb, int ntile, const NodeW* nodes, const uint32_t* x0, const uint32_t* x1, const uint32_t* x2,
		BuildScratch s) {
	__shared__ int sh[32];
	const uint32_t* xs[3] = { x0, x1, x2 };
	for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
		const int i = s.tile_node[t];
		const NodeW nd = nodes[lb + i];
		int tb, te;
		tile_range(nd, t, s.tile_off[i], &tb, &te);
		const uint32_t* xd = xs[s.xdim[i]];
		const uint32_t xm = s.xmidf[i];
		int c = 0;
		const int p0 = tb + threadIdx.x * PER_T;
		for (int j = 0; j < PER_T; j++) {
			const int p = p0 + j;
			if (p < te) {
				c += xd[p] < xm;
			}
		}
		c = block_sum_int(c, sh);
		if (threadIdx.x == 0) {
			s.tile_lt[t] = c;
		}
	}
}

// P2: per split node, midpoint count m and per-tile offsets of misplaced elements.
__global__ void __launch_bounds__(TPB) k_node_scan(int64_t lb, int nl, const NodeW* nodes, const uint32_t* x0, const uint32_t* x1, const uint32_t* x2,
		BuildScratch s) {
	__shared__ int sh[32];
	__shared__ int s_strad[3];
	const uint32_t* xs[3] = { x0, x1, x2 };
	for (int i = blockIdx.x; i < nl; i += gridDim.x) {
		if (!s.split[i]) {
			continue;
		}
		const NodeW nd = nodes[lb + i];
		const int t0 = s.tile_off[i];
		const int nt = s.ntiles[i];
		int m = 0;
		for (int k = threadIdx.x; k < nt; k += TPB) {
			m += s.tile_lt[t0 + k];
		}
		m = block_sum_int(m, sh);
		const int sp = nd.pbeg + m;
		const uint32_t* xd = xs[s.xdim[i]];
		const uint32_t xm = s.xmidf[i];
		// the tile holding the split point strictly inside it
		const int ts = (sp - nd.pbeg) / TILE;
		int sL = 0, sR = 0;
		if (ts < nt) {
			int tb, te;
			tile_range(nd, t0 + ts, t0, &tb, &te);
			if (tb < sp && sp < te) {
				const int p0 = tb + threadIdx.x * PER_T;
				for (int j = 0; j < PER_T; j++) {
					const int p = p0 + j;
					if (p < te) {
						const bool lt = xd[p] < xm;
						sL += (p < sp) && !lt;
						sR += (p >= sp) && lt;
					}
				}
			}
		}
		sL = block_sum_int(sL, sh);
		sR = block_sum_int(sR, sh);
		if (threadIdx.x == 0) {
			s_strad[0] = sL;
			s_strad[1] = sR;
		}
		__syncthreads();
		// prefix of misplaced-left (left to right) and inclusive prefix of misplaced-right
		int carryL = 0, carryR = 0;
		for (int k0 = 0; k0 < nt; k0 += TPB) {
			const int k = k0 + threadIdx.x;
			int mL = 0, mR = 0;
			if (k < nt) {
				int tb, te;
				tile_range(nd, t0 + k, t0, &tb, &te);
				const int lt = s.tile_lt[t0 + k];
				if (te <= sp) {
					mL = (te - tb) - lt;
				} else if (tb >= sp) {
					mR = lt;
				} else {
					mL = s_strad[0];
					mR = s_strad[1];
				}
			}
			int totL, totR;
			const int exL = block_excl_scan(mL, sh, &totL);
			const int exR = block_excl_scan(mR, sh, &totR);
			if (k < nt) {
				s.tile_offL[t0 + k] = carryL + exL;
				s.tile_offR[t0 + k] = carryR + exR + mR;  // inclusive, fixed below
			}
			carryL += totL;
			carryR += totR;
		}
		__syncthreads();
		for (int k = threadIdx.x; k < nt; k += TPB) {
			s.tile_offR[t0 + k] = carryR - s.tile_offR[t0 + k];  // misplaced-right in later tiles
		}
		if (threadIdx.x == 0) {
			s.node_m[i] = m;
			s.node_nmis[i] = carryL;
		}
		__syncthreads();
	}
}

// P3: positions of the misplaced elements, ranked from the left (left region) and from the
// right (right region).
__global__ void __launch_bounds__(TPB) k_positions(int64_t lb, int ntile, const NodeW* nodes, const uint32_t* x0, const uint32_t* x1,
		const uint32_t* x2, BuildScratch s) {
	__shared__ int sh[32];
	const uint32_t* xs[3] = { x0, x1, x2 };
	for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
		const int i = s.tile_node[t];
		const NodeW nd = nodes[lb + i];
		int tb, te;
		tile_range(nd, t, s.tile_off[i], &tb, &te);
		const int sp = nd.pbeg + s.node_m[i];
		const uint32_t* xd = xs[s.xdim[i]];
		const uint32_t xm = s.xmidf[i];
		const int p0 = tb + threadIdx.x * PER_T;
		unsigned mskL = 0, mskR = 0;
		for (int j = 0; j < PER_T; j++) {
			const int p = p0 + j;
			if (p < te) {
				const bool lt = xd[p] < xm;
				if (p < sp && !lt) {
					mskL |= 1u << j;
				}
				if (p >= sp && lt) {
					mskR |= 1u << j;
				}
			}
		}
		int totL, totR;
		const int exL = block_excl_scan(__popc(mskL), sh, &totL);
		const int exR = block_excl_scan(__popc(mskR), sh, &totR);
		const int baseL = s.tile_offL[t] + exL;
		const int baseR = s.tile_offR[t];
		int cL = 0, cR = 0;
		for (int j = 0; j < PER_T; j++) {
			const int p = p0 + j;
			if (mskL & (1u << j)) {
				s.posL[nd.pbeg + baseL + cL] = p;
				cL++;
			}
			if (mskR & (1u << j)) {
				cR++;
				// misplaced-right elements of this tile after p: totR - (exR + cR)
				s.posR[nd.pbeg + baseR + (totR - (exR + cR))] = p;
			}
		}
	}
}

// P4: the swaps.
__global__ void __launch_bounds__(TPB) k_swap(int64_t lb, int ntile, const NodeW* nodes, uint32_t* x0, uint32_t* x1, uint32_t* x2, BuildScratch s) {
	for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
		const int i = s.tile_node[t];
		const NodeW nd = nodes[lb + i];
		int tb, te;
		tile_range(nd, t, s.tile_off[i], &tb, &te);
		const int nmis = s.node_nmis[i];
		for (int p = tb + threadIdx.x; p < te; p += TPB) {
			const int k = p - nd.pbeg;
			if (k < nmis) {
				const int a = s.posL[nd.pbeg + k];
				const int b = s.posR[nd.pbeg + k];
				uint32_t t0 = x0[a];
				x0[a] = x0[b];
				x0[b] = t0;
				t0 = x1[a];
				x1[a] = x1[b];
				x1[b] = t0;
				t0 = x2[a];
				x2[a] = x2[b];
				x2[b] = t0;
				const int32_t ti = s.idx[a];
				s.idx[a] = s.idx[b];
				s.idx[b] = ti;
			}
		}
	}
}

__global__ void k_children(int64_t lb, int nl, int64_t cb, NodeW* nodes, double* gbox, uint64_t* key, int32_t* depth, int32_t* parent, BuildScratch s) {
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nl; i += gridDim.x * blockDim.x) {
		const int64_t ni = lb + i;
		NodeW nd = nodes[ni];
		if (!s.split[i]) {
			nd.child = -1;
			nd.flags = 1;
			nodes[ni] = nd;
			continue;
		}
		const int64_t l = cb + 2 * (int64_t) s.rank[i];
		const int64_t r = l + 1;
		nd.child = (int32_t) l;
		nd.flags = 0;
		nodes[ni] = nd;
		const int mid = nd.pbeg + s.node_m[i];
		NodeW c;
		c.x = c.y = c.z = 0;
		c.radius = 0.f;
		c.child = -1;
		c.flags = 1;
		c.pbeg = nd.pbeg;
		c.pend = mid;
		nodes[l] = c;
		c.pbeg = mid;
		c.pend = nd.pend;
		nodes[r] = c;
		const int xd = s.xdim[i];
		for (int d = 0; d < 6; d++) {
			gbox[6 * l + d] = gbox[6 * ni + d];
			gbox[6 * r + d] = gbox[6 * ni + d];
		}
		gbox[6 * l + 3 + xd] = s.xmid[i];
		gbox[6 * r + xd] = s.xmid[i];
		key[l] = key[ni] << 1;
		key[r] = (key[ni] << 1) + 1;
		depth[l] = depth[r] = depth[ni] + 1;
		parent[l] = parent[r] = (int32_t) ni;
	}
}

__global__ void k_gather_particles(int64_t b, int64_t n, const int32_t* idx, const float* v0, const float* v1, const float* v2, const int8_t* r,
		float* o0, float* o1, float* o2, int8_t* orr) {
	for (int64_t i = b + blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		const int j = idx[i];
		o0[i] = v0[j];
		o1[i] = v1[j];
		o2[i] = v2[j];
		orr[i] = r[j];
	}
}

// ---------------------------------------------------------------- upsweep
template<class T>
__device__ __forceinline__ T warp_max(T v) {
	for (int o = 16; o; o >>= 1) {
		v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
	}
	return v;
}
template<class T>
__device__ __forceinline__ T warp_min(T v) {
	for (int o = 16; o; o >>= 1) {
		v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
	}
	return v;
}
template<class T>
__device__ __forceinline__ T warp_sum(T v) {
	for (int o = 16; o; o >>= 1) {
		v += __shfl_xor_sync(0xffffffffu, v, o);
	}
	return v;
}

constexpr int UTPB = 128;

// A warp per node (tree.cpp:351-571): tight box, expansion centre and radius, multipole (P2M of
// the particles for a leaf, M2M of the two children in double for an interior node).
template<class Ops>
__global__ void __launch_bounds__(UTPB) k_upsweep(int64_t lb, int64_t le, NodeW* nodes, int32_t* nbox, float* multi, double* tbox, const double* gbox,
		const uint32_t* x0, const uint32_t* x1, const uint32_t* x2, int bucket) {
	constexpr int NM = Ops::NMULT;
	const uint32_t* xs[3] = { x0, x1, x2 };
	const int lane = threadIdx.x & 31;
	const int64_t gw = (blockIdx.x * (int64_t) blockDim.x + threadIdx.x) >> 5;
	const int64_t nw = ((int64_t) gridDim.x * blockDim.x) >> 5;
	for (int64_t ni = lb + gw; ni < le; ni += nw) {
		const NodeW nd = nodes[ni];
		const int nparts = nd.pend - nd.pbeg;
		const double* gb = gbox + 6 * ni;
		if (nd.child < 0) {
			// ---- leaf (tree.cpp:498-571)
			double mn[3], mx[3];
			for (int d = 0; d < 3; d++) {
				mn[d] = gb[3 + d];
				mx[d] = gb[d];
			}
			for (int p = nd.pbeg + lane; p < nd.pend; p += 32) {
				for (int d = 0; d < 3; d++) {
					const double xx = fixed_to_double(xs[d][p]);
					mx[d] = fmax(mx[d], xx);
					mn[d] = fmin(mn[d], xx);
				}
			}
			for (int d = 0; d < 3; d++) {
				mn[d] = warp_min(mn[d]);
				mx[d] = warp_max(mx[d]);
			}
			double Xc[3];
			for (int d = 0; d < 3; d++) {
				Xc[d] = (mx[d] + mn[d]) * 0.5;
			}
			double r = 0.0;
			for (int p = nd.pbeg + lane; p < nd.pend; p += 32) {
				double this_radius = 0.0;
				for (int d = 0; d < 3; d++) {
					const double dx = fixed_to_double(xs[d][p]) - Xc[d];
					this_radius += dx * dx;
				}
				r = fmax(r, this_radius);
			}
			r = warp_max(r);
			// P2M about fixed32(Xc), summed in double
			uint32_t Y[3];
			for (int d = 0; d < 3; d++) {
				Y[d] = fixed_from_double(Xc[d]);
			}
			double M[NM];
			for (int k = 0; k < NM; k++) {
				M[k] = 0.0;
			}
			for (int p = nd.pbeg + lane; p < nd.pend; p += 32) {
				float m[NM];
				Ops::p2m(m, fixed_dist(x0[p], Y[0]), fixed_dist(x1[p], Y[1]), fixed_dist(x2[p], Y[2]));
				for (int k = 0; k < NM; k++) {
					M[k] += (double) m[k];
				}
			}
			for (int k = 0; k < NM; k++) {
				M[k] = warp_sum(M[k]);
			}
			if (lane == 0) {
				NodeW o = nd;
				o.x = Y[0];
				o.y = Y[1];
				o.z = Y[2];
				o.radius = (float) sqrt(r);
				nodes[ni] = o;
				for (int d = 0; d < 3; d++) {
					tbox[6 * ni + d] = mn[d];
					tbox[6 * ni + 3 + d] = mx[d];
					nbox[6 * ni + d] = range_fixed_from_double(mn[d]);
					nbox[6 * ni + 3 + d] = range_fixed_from_double(mx[d]);
				}
			}
#pragma unroll
			for (int k = 0; k < NM; k++) {
				if (lane == (k & 31)) {
					multi[NMULT_STRIDE * ni + k] = (float) M[k];
				}
			}
		} else {
			// ---- interior node (tree.cpp:351-497)
			const int64_t L = nd.child, R = nd.child + 1;
			const NodeW nl = nodes[L], nr = nodes[R];
			const float ml0 = multi[NMULT_STRIDE * L], mr0 = multi[NMULT_STRIDE * R];
			double bb[3], be[3];
			for (int d = 0; d < 3; d++) {
				const double lb_ = tbox[6 * L + d], le_ = tbox[6 * L + 3 + d];
				const double rb_ = tbox[6 * R + d], re_ = tbox[6 * R + 3 + d];
				if (ml0 != 0.0f && mr0 != 0.0f) {
					bb[d] = fmin(lb_, rb_);
					be[d] = fmax(le_, re_);
				} else if (ml0 != 0.0f) {
					bb[d] = lb_;
					be[d] = le_;
				} else {
					bb[d] = rb_;
					be[d] = re_;
				}
			}
			int xdim = 0;
			{
				double max_span = -1.0;
				for (int d = 0; d < 3; d++) {
					const double span = gb[3 + d] - gb[d];
					if (span > max_span) {
						max_span = span;
						xdim = d;
					}
				}
			}
			const bool tried1 = nparts <= 64 * bucket && (be[xdim] - bb[xdim] <= 0.5);
			double Xc1[3];
			float r2max = 0.0f;
			if (tried1) {
				uint32_t xc[3];
				for (int d = 0; d < 3; d++) {
					Xc1[d] = 0.5 * (bb[d] + be[d]);
					xc[d] = fixed_from_double(Xc1[d]);
				}
				for (int p = nd.pbeg + lane; p < nd.pend; p += 32) {
					const float dx = fixed_dist(x0[p], xc[0]);
					const float dy = fixed_dist(x1[p], xc[1]);
					const float dz = fixed_dist(x2[p], xc[2]);
					const float r2 = dx * dx + dy * dy + dz * dz;
					r2max = fmaxf(r2max, r2);
				}
				r2max = warp_max(r2max);
			}
			double sX[3];
			{
				const double Xl[3] = { fixed_to_double(nl.x), fixed_to_double(nl.y), fixed_to_double(nl.z) };
				const double Xr[3] = { fixed_to_double(nr.x), fixed_to_double(nr.y), fixed_to_double(nr.z) };
				const double radius1 = tried1 ? (double) sqrtf(r2max) : 0.0;
				double N[3];
				double norminv = 0.0;
				for (int d = 0; d < 3; d++) {
					N[d] = Xl[d] - Xr[d];
					norminv += N[d] * N[d];
				}
				norminv = 1.0 / sqrt(norminv);
				for (int d = 0; d < 3; d++) {
					N[d] *= norminv;
					N[d] = fabs(N[d]);
				}
				double r = 0.0, Xc2[3];
				const double Rl = nl.radius, Rr = nr.radius;
				if (mr0 != 0.0f) {
					if (ml0 != 0.0f) {
						for (int d = 0; d < 3; d++) {
							const double a = Xl[d] + N[d] * Rl, b = Xr[d] + N[d] * Rr;
							const double xmax = (a < b) ? b : a;  // std::max
							const double c = Xl[d] - N[d] * Rl, e = Xr[d] - N[d] * Rr;
							const double xmin = (e < c) ? e : c;  // std::min
							Xc2[d] = (xmax + xmin) * 0.5;
							const double t = (xmax - xmin) * 0.5;
							r += t * t;
						}
					} else {
						for (int d = 0; d < 3; d++) {
							Xc2[d] = Xr[d];
						}
						r = Rr * Rr;
					}
				} else {
					for (int d = 0; d < 3; d++) {
						Xc2[d] = Xl[d];
					}
					r = Rl * Rl;
				}
				const double radius2 = sqrt(r);
				double Xc[3];
				float radius;
				if (tried1 && radius1 < radius2) {
					for (int d = 0; d < 3; d++) {
						Xc[d] = Xc1[d];
					}
					radius = (float) radius1;
				} else {
					for (int d = 0; d < 3; d++) {
						Xc[d] = Xc2[d];
					}
					radius = (float) radius2;
				}
				r = 0.0;
				for (int d = 0; d < 3; d++) {
					const double span = be[d] - bb[d];
					r += (span * 0.5) * (span * 0.5);
				}
				r = sqrt(r);
				if (r < radius) {
					radius = (float) r;
					for (int d = 0; d < 3; d++) {
						Xc[d] = (bb[d] + be[d]) * 0.5;
					}
				}
				for (int d = 0; d < 3; d++) {
					sX[d] = Xc[d];
				}
				NodeW o = nd;
				o.x = fixed_from_double(Xc[0]);
				o.y = fixed_from_double(Xc[1]);
				o.z = fixed_from_double(Xc[2]);
				o.radius = radius;
				if (lane == 0) {
					nodes[ni] = o;
					for (int d = 0; d < 3; d++) {
						tbox[6 * ni + d] = bb[d];
						tbox[6 * ni + 3 + d] = be[d];
						nbox[6 * ni + d] = range_fixed_from_double(bb[d]);
						nbox[6 * ni + 3 + d] = range_fixed_from_double(be[d]);
					}
				}
			}
			// M2M of both children in double (tree.cpp:481-494): lane 0 the left, lane 1 the right,
			// then left + right
			double Mo[NM];
			for (int k = 0; k < NM; k++) {
				Mo[k] = 0.0;
			}
			if (lane < 2) {
				const int64_t c = lane == 0 ? L : R;
				const NodeW cn = lane == 0 ? nl : nr;
				double Ma[NM];
				for (int k = 0; k < NM; k++) {
					Ma[k] = (double) multi[NMULT_STRIDE * c + k];
				}
				Ops::m2m(Mo, Ma, fixed_to_double(cn.x) - sX[0], fixed_to_double(cn.y) - sX[1], fixed_to_double(cn.z) - sX[2]);
			}
			for (int k = 0; k < NM; k++) {
				const double right = __shfl_down_sync(0xffffffffu, Mo[k], 1);
				if (lane == 0) {
					multi[NMULT_STRIDE * ni + k] = (float) (Mo[k] + right);
				}
			}
		}
	}
}

template<class T>
ct_status grow(Ctx* c, T** p, int64_t old_n, int64_t new_n, int per, const char* what) {
	T* q = nullptr;
	CT_TRY(dalloc(c, (void**) &q, sizeof(T) * per * new_n, what));
	if (*p) {
		CT_CUDA(c, cudaMemcpyAsync(q, *p, sizeof(T) * per * old_n, cudaMemcpyDeviceToDevice, c->stream));
		CT_CUDA(c, cudaStreamSynchronize(c->stream));
		dfree(c, *p, sizeof(T) * per * old_n);
	}
	*p = q;
	return CT_OK;
}

ct_status ensure_nodes(Ctx* c, Box* b, int64_t need) {
	if (need <= b->node_cap) {
		return CT_OK;
	}
	int64_t cap = std::max<int64_t>(need, b->node_cap * 3 / 2);
	cap = std::max<int64_t>(cap, 1024);
	const int64_t old = b->node_cap;
	CT_TRY(grow(c, &b->nodes, old, cap, 1, "tree nodes"));
	CT_TRY(grow(c, &b->nbox, old, cap, 6, "node boxes"));
	CT_TRY(grow(c, &b->multi, old, cap, NMULT_STRIDE, "multipoles"));
	CT_TRY(grow(c, &b->key, old, cap, 1, "node keys"));
	CT_TRY(grow(c, &b->depth, old, cap, 1, "node depth"));
	CT_TRY(grow(c, &b->parent, old, cap, 1, "node parent"));
	CT_TRY(grow(c, &b->gbox, old, cap, 6, "node geometric box"));
	CT_TRY(grow(c, &b->tbox, old, cap, 6, "node tight box"));
	b->node_cap = cap;
	return CT_OK;
}

int grid_for(Ctx* c, int64_t work, int tpb, int per_sm = 8) {
	const int64_t g = (work + tpb - 1) / tpb;
	return (int) std::max<int64_t>(1, std::min<int64_t>(g, (int64_t) c->nsm * per_sm));
}

template<class Ops>
ct_status tree_build_t(Ctx* c, Box* b, const ct_tree_params* p) {
	cudaStream_t st = c->stream;
	const int64_t n = b->n;
	const int64_t pb = b->rung_begin;
	const int64_t np = n - pb;
	b->tree_valid = false;
	if (np > INT32_MAX / 2) {
		return fail(c, CT_ERR_ARG, "box too large for 32-bit particle indices");
	}
	// node capacity: the reference's arena, max(8 N / bucket, 2^21) (tree.cpp:247) is an
	// upper estimate; start smaller and grow per level as needed.
	CT_TRY(ensure_nodes(c, b, std::max<int64_t>(4 * np / std::max(p->bucket, 1) + 4096, 8192)));
	ct_status s1 = CT_OK;
	BuildScratch s;
	const int64_t npad = std::max<int64_t>(np, 1);
	s.idx = (int32_t*) scratch(c, 0, sizeof(int32_t) * n, &s1);
	s.posL = (int32_t*) scratch(c, 1, sizeof(int32_t) * n, &s1);
	s.posR = (int32_t*) scratch(c, 2, sizeof(int32_t) * n, &s1);
	CT_TRY(s1);
	(void) npad;
	c->launches++;
	k_iota<<<grid_for(c, n, 256), 256, 0, st>>>(s.idx, n);
	c->launches++;
	const int nroot = b->nsub;
	CT_TRY(ensure_nodes(c, b, nroot + 1));
	k_init_roots<<<(nroot + 127) / 128, 128, 0, st>>>(nroot, b->d_sub_off, b->nodes, b->gbox, b->key, b->depth, b->parent, (int32_t) pb, (int32_t) n);
	CT_CUDA(c, cudaMemsetAsync(c->d_flags, 0, 4 * sizeof(int), st));
	std::vector<int64_t> levels;
	levels.push_back(0);
	int64_t lb = 0, le = nroot;
	int32_t* h_tot = (int32_t*) c->pinned;
	while (le > lb) {
		levels.push_back(le);
		const int nl = (int) (le - lb);
		// per-level scratch (node- and tile-sized arrays)
		const int64_t max_tiles = (np + TILE - 1) / TILE + nl + 1;
		s.split = (int32_t*) scratch(c, 3, sizeof(int32_t) * (nl + 1), &s1);
		s.rank = (int32_t*) scratch(c, 4, sizeof(int32_t) * (nl + 1), &s1);
		s.ntiles = (int32_t*) scratch(c, 5, sizeof(int32_t) * (nl + 1), &s1);
		s.tile_off = (int32_t*) scratch(c, 6, sizeof(int32_t) * (nl + 1), &s1);
		s.xdim = (int32_t*) scratch(c, 7, sizeof(int32_t) * nl, &s1);
		s.xmidf = (uint32_t*) scratch(c, 8, sizeof(uint32_t) * nl, &s1);
		s.xmid = (double*) scratch(c, 9, sizeof(double) * nl, &s1);
		s.node_m = (int32_t*) scratch(c, 10, sizeof(int32_t) * nl, &s1);
		s.node_nmis = (int32_t*) scratch(c, 11, sizeof(int32_t) * nl, &s1);
		s.tile_node = (int32_t*) scratch(c, 12, sizeof(int32_t) * max_tiles, &s1);
		s.tile_lt = (int32_t*) scratch(c, 13, sizeof(int32_t) * max_tiles, &s1);
		s.tile_offL = (int32_t*) scratch(c, 14, sizeof(int32_t) * max_tiles, &s1);
		s.tile_offR = (int32_t*) scratch(c, 15, sizeof(int32_t) * max_tiles, &s1);
		s.totals = c->d_flags + 8;
		CT_TRY(s1);
		size_t need = 0;
		cub::DeviceScan::ExclusiveSum(nullptr, need, s.split, s.rank, nl + 1, st);
		s.cub_bytes = need;
		s.cub_tmp = scratch(c, 16, need + 256, &s1);
		CT_TRY(s1);
		c->launches++;
		k_classify<<<grid_for(c, nl, 256), 256, 0, st>>>(lb, nl, b->nodes, b->gbox, b->depth, p->theta, p->hsoft, p->bucket, s, c->d_flags);
		CT_CUDA(c, cudaMemsetAsync(s.split + nl, 0, sizeof(int32_t), st));
		CT_CUDA(c, cudaMemsetAsync(s.ntiles + nl, 0, sizeof(int32_t), st));
		CT_CUDA(c, cub::DeviceScan::ExclusiveSum(s.cub_tmp, need, s.split, s.rank, nl + 1, st));
		CT_CUDA(c, cub::DeviceScan::ExclusiveSum(s.cub_tmp, need, s.ntiles, s.tile_off, nl + 1, st));
		CT_CUDA(c, cudaMemcpyAsync(h_tot, s.rank + nl, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
		CT_CUDA(c, cudaMemcpyAsync(h_tot + 1, s.tile_off + nl, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
		CT_CUDA(c, cudaStreamSynchronize(st));
		const int nsplit = h_tot[0];
		const int ntile = h_tot[1];
		if (nsplit > 0) {
			CT_TRY(ensure_nodes(c, b, le + 2 * (int64_t) nsplit));
			c->launches++;
			k_tile_map<<<grid_for(c, (int64_t) nl * 32, 256), 256, 0, st>>>(nl, s);
			const int gt = std::min(ntile, c->nsm * 16);
			c->launches++;
			k_count<<<gt, TPB, 0, st>>>(lb, ntile, b->nodes, b->x[0], b->x[1], b->x[2], s);
			c->launches++;
			k_node_scan<<<std::min(nl, c->nsm * 16), TPB, 0, st>>>(lb, nl, b->nodes, b->x[0], b->x[1], b->x[2], s);
			c->launches++;
			k_positions<<<gt, TPB, 0, st>>>(lb, ntile, b->nodes, b->x[0], b->x[1], b->x[2], s);
			c->launches++;
			k_swap<<<gt, TPB, 0, st>>>(lb, ntile, b->nodes, b->x[0], b->x[1], b->x[2], s);
		}
		c->launches++;
		k_children<<<grid_for(c, nl, 256), 256, 0, st>>>(lb, nl, le, b->nodes, b->gbox, b->key, b->depth, b->parent, s);
		CT_CUDA(c, cudaGetLastError());
		lb = le;
		le = le + 2 * (int64_t) nsplit;
	}
	b->level_start = levels;  // level k = [levels[k], levels[k+1])
	b->nnodes = le;
	// apply the permutation to velocities and rungs
	{
		ct_status s2 = CT_OK;
		float* t0 = (float*) scratch(c, 17, sizeof(float) * n, &s2);
		float* t1 = (float*) scratch(c, 18, sizeof(float) * n, &s2);
		float* t2 = (float*) scratch(c, 19, sizeof(float) * n, &s2);
		int8_t* tr = (int8_t*) scratch(c, 20, n + 16, &s2);
		CT_TRY(s2);
		CT_CUDA(c, cudaMemcpyAsync(t0 + pb, b->v[0] + pb, sizeof(float) * np, cudaMemcpyDeviceToDevice, st));
		CT_CUDA(c, cudaMemcpyAsync(t1 + pb, b->v[1] + pb, sizeof(float) * np, cudaMemcpyDeviceToDevice, st));
		CT_CUDA(c, cudaMemcpyAsync(t2 + pb, b->v[2] + pb, sizeof(float) * np, cudaMemcpyDeviceToDevice, st));
		CT_CUDA(c, cudaMemcpyAsync(tr + pb, b->rung + pb, np, cudaMemcpyDeviceToDevice, st));
		if (np > 0) {
			c->launches++;
			k_gather_particles<<<grid_for(c, np, 256), 256, 0, st>>>(pb, n, s.idx, t0, t1, t2, tr, b->v[0], b->v[1], b->v[2], b->rung);
		}
	}
	// upsweep, deepest level first
	for (int k = (int) levels.size() - 2; k >= 0; k--) {
		const int64_t a = levels[k], e = levels[k + 1];
		if (e > a) {
			c->launches++;
			k_upsweep<Ops><<<(int) std::min<int64_t>((e - a + UTPB / 32 - 1) / (UTPB / 32), (int64_t) c->nsm * 16), UTPB, 0, st>>>(a, e, b->nodes, b->nbox,
					b->multi, b->tbox, b->gbox,
					b->x[0], b->x[1], b->x[2], p->bucket);
		}
	}
	CT_CUDA(c, cudaGetLastError());
	CT_CUDA(c, cudaMemcpyAsync(h_tot, c->d_flags, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
	CT_CUDA(c, cudaStreamSynchronize(st));
	if (h_tot[2]) {
		return fail(c, CT_ERR_CAPACITY, "tree depth exceeded the maximum of 128 (coincident particles?)");
	}
	b->tparams = *p;
	b->tree_valid = true;
	return CT_OK;
}

}  // namespace

ct_status tree_build(Ctx* c, Box* b, const ct_tree_params* p) {
	if (c->order == 5) {
		return tree_build_t<Ops5>(c, b, p);
	}
	return tree_build_t<Ops7>(c, b, p);
}

}  // namespace ct
