// The kick: dual tree walk, interactions and the leaf kick on the device.
//
// Reference: cuda_kick_kernel (src/kick.cu:179-506) walks each work item's subtree depth-first
// in one warp and evaluates interactions as it goes; the host walks the top of the tree
// (src/kick.cpp:150-507).  Here the walk is breadth-first over the whole tree, one warp per
// node, with the reference's opening criteria and list semantics:
//   Ewald list  (kick.cu:269-329): CC if max(R^2, (0.5-(rs+ro))^2) > ((rs+ro)/theta)^2,
//                otherwise the children are checked one level down;
//   direct list (kick.cu:330-431): CC if R > max((rs+ro)/theta, rs+ro+h); for leaf-leaf pairs
//                P2L (CP) / M2P (PC) by the dpc/dcp and box tests with MIN_PARTS_PCCP;
//                remaining leaves are P2P, other nodes are opened; a leaf re-checks the
//                children it opens until none remain; a non-leaf passes children and leaves
//                down to both of its children.
// Every node's lists land contiguously in global memory (per-warp staging), so that the
// interaction kernels that follow read them with one pass per node:
//   k_m2l        Ewald and direct M2L plus P2L into the node's own expansion delta (warp per
//                node, lanes over sources, butterfly reduction; gravity.cu:44-155,213-244);
//   k_l2l        top-down L2L: L(node) = L2L(L(parent)) + delta (kick.cu:246-258);
//   k_leaf       M2P, P2P (sources staged in shared memory as floats relative to the leaf
//                centre, compensated per-batch accumulation), L2P and the kick
//                (gravity.cu:157-211,246-404, kick.cu:53-177).
#include <cub/cub.cuh>
#include <cstdlib>
#include <mutex>

#include "ct_internal.cuh"
#include "ct_ops.cuh"

namespace ct {

__constant__ ct_p7::EwaldTab c_tab7;
__constant__ ct_p5::EwaldTab c_tab5;

template<class Ops> __device__ __forceinline__ const typename Ops::Tab& ewald_tab();
template<> __device__ __forceinline__ const ct_p7::EwaldTab& ewald_tab<Ops7>() {
	return c_tab7;
}
template<> __device__ __forceinline__ const ct_p5::EwaldTab& ewald_tab<Ops5>() {
	return c_tab5;
}

// The Ewald tables as the generated operator reads them, for kernels whose threads walk the
// real images in different orders: the real-image vectors (indexed differently by every
// thread) from a shared-memory copy, the Fourier terms and the r -> 0 limit (indexed alike by
// all threads of a warp) from the __constant__ tables.
template<class Tab>
struct EwaldView {
	const float (*real)[3];
	const decltype(Tab::four)& four;
	const float (*four_exp)[sizeof(Tab::four_exp[0]) / sizeof(float)];  // rows of the Fourier tensors (shared memory in the kernel)
	const decltype(Tab::D0)& D0;
};

namespace {

// ---------------------------------------------------------------- Ewald tables (FP64 on the device)
__global__ void k_ewald_four7(ct_p7::EwaldTab* t) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < CT_EWALD_NFOUR) {
		double E[ct_p7::NEXP];
		ct_p7::ewald_four_entry(E, t->four[i][0], t->four[i][1], t->four[i][2]);
		for (int k = 0; k < ct_p7::NEXP; k++) {
			t->four_exp[i][k] = (float) E[k];
		}
	}
	if (i < ct_p7::NFULL) {
		t->D0[i] = (float) ct_p7::ewald_d0_entry(i);
	}
}
__global__ void k_ewald_four5(ct_p5::EwaldTab* t) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < CT_EWALD_NFOUR) {
		double E[ct_p5::NEXP];
		ct_p5::ewald_four_entry(E, t->four[i][0], t->four[i][1], t->four[i][2]);
		for (int k = 0; k < ct_p5::NEXP; k++) {
			t->four_exp[i][k] = (float) E[k];
		}
	}
	if (i < ct_p5::NFULL) {
		t->D0[i] = (float) ct_p5::ewald_d0_entry(i);
	}
}

// ---------------------------------------------------------------- walk
constexpr int WALK_TPB = 128;
constexpr int NLIST = 8;  // per-warp staging arrays
enum {
	S_ECC = 0, S_EOUT, S_DCC, S_CP, S_PC, S_LEAF, S_NEXT0, S_NEXT1
};

struct WalkOut {
	// per node, indexed by node id: {offset, count} pairs
	int2* ecc;   // Ewald CC sources
	int2* dcc;   // direct CC sources
	int2* cp;    // leaves: P2L source leaves
	int2* pc;    // leaves: M2P source nodes
	int2* pp;    // leaves: P2P source leaves
	int2* eout;  // non-leaves: Ewald checks passed to the children
	int2* dout;  // non-leaves: direct checks passed to the children
	int* ecc_list;
	int* dcc_list;
	int* cp_list;
	int* pc_list;
	int* pp_list;
	int* pass_cur;   // pass-down lists of this level (eout/dout)
	int* pass_prev;  // pass-down lists of the level above
	unsigned long long* cursor;  // [0] ecc [1] dcc [2] cp [3] pc [4] pp [5] pass (this level)
	long long cap_cc, cap_leaf, cap_pass;
	int* stage;   // per-warp staging, NLIST * stage_cap ints per warp
	int stage_cap;
	int* flags;   // [0] overflow [1] dropped Ewald check
};

struct WalkParams {
	float thetainv;
	float h;
	int nroot;  // nodes [0, nroot) are the roots of independent boxes
	const int64_t* sub_off;
	const float* sub_h;  // per-box softening of an ensemble, or null
};

__device__ __forceinline__ float sqrf3(float a, float b, float c) {
	return __fadd_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)), __fmul_rn(c, c));
}

// distance(fixed32 b, range_fixed a) of range.hpp:447-458, negated argument order
__device__ __forceinline__ float dist_rf(uint32_t b, int32_t a) {
	float f = __dsub_rn(__dmul_rn((double) a, 1.0 / 536870912.0), fixed_to_double(b));
	f = (float) __dsub_rn((double) f, (double) (f > 0.5f));
	f = (float) __dadd_rn((double) f, (double) (f < -0.5f));
	return -f;
}

// box_intersects_sphere (range.hpp:459-466)
__device__ __forceinline__ bool box_sphere(const int32_t* bx, uint32_t x, uint32_t y, uint32_t z, float r) {
	const uint32_t X[3] = { x, y, z };
	float d2 = 0.0f;
	for (int d = 0; d < 3; d++) {
		const float a = dist_rf(X[d], bx[d]);
		const float b = dist_rf(X[d], bx[3 + d]);
		const float d2b = __fmul_rn(a, a), d2e = __fmul_rn(b, b);
		const int32_t xr = (int32_t) (X[d] >> 3);
		const int outside = (xr < bx[d]) + (xr > bx[3 + d]);
		d2 = __fadd_rn(d2, __fmul_rn((float) outside, fminf(d2b, d2e)));
	}
	return d2 < __fmul_rn(r, r);
}

// Warp-compacted append of `n` (0..2) values per lane to a staging array.
__device__ __forceinline__ void stage_push(int* arr, int& cnt, int cap, int lane, int n, int v0, int v1, int* ovf) {
	const unsigned m1 = __ballot_sync(0xffffffffu, n >= 1);
	const unsigned m2 = __ballot_sync(0xffffffffu, n >= 2);
	const unsigned lt = (1u << lane) - 1u;
	const int off = __popc(m1 & lt) + __popc(m2 & lt);
	const int tot = __popc(m1) + __popc(m2);
	if (n >= 1) {
		const int p = cnt + off;
		if (p < cap) {
			arr[p] = v0;
		} else {
			*ovf = 1;
		}
		if (n >= 2) {
			if (p + 1 < cap) {
				arr[p + 1] = v1;
			} else {
				*ovf = 1;
			}
		}
	}
	cnt += tot;
}

// Copy a staged list to global memory; returns {offset, count}.
__device__ __forceinline__ int2 flush(const int* src, int cnt, int cap, int* dst, unsigned long long* cursor, long long dcap, int lane, int* ovf) {
	cnt = min(cnt, cap);
	unsigned long long off = 0;
	if (lane == 0 && cnt) {
		off = atomicAdd(cursor, (unsigned long long) cnt);
	}
	off = __shfl_sync(0xffffffffu, off, 0);
	if ((long long) (off + cnt) > dcap) {
		if (lane == 0) {
			atomicOr(ovf, 1);
		}
		return make_int2(0, 0);
	}
	for (int i = lane; i < cnt; i += 32) {
		dst[off + i] = src[i];
	}
	return make_int2((int) off, cnt);
}

__global__ void __launch_bounds__(WALK_TPB) k_walk(int64_t lb, int64_t le, const NodeW* __restrict__ nodes, const int32_t* __restrict__ nbox,
		const int32_t* __restrict__ parent, WalkOut o, WalkParams p) {
	const int lane = threadIdx.x & 31;
	const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int nw = (gridDim.x * blockDim.x) >> 5;
	int* st = o.stage + (size_t) gw * NLIST * o.stage_cap;
	const int cap = o.stage_cap;
	int* sl[NLIST];
	for (int k = 0; k < NLIST; k++) {
		sl[k] = st + k * cap;
	}
	int ovf = 0, dropped = 0;
	const float thetainv = p.thetainv;
	for (int64_t si = lb + gw; si < le; si += nw) {
		const NodeW self = nodes[si];
		const float h = p.sub_h ? p.sub_h[box_of(p.sub_off, p.nroot, self.pbeg)] : p.h;
		const int nsinks = self.pend - self.pbeg;
		const bool sleaf = self.flags & 1;
		int2 z2 = make_int2(0, 0);
		if (nsinks == 0) {
			if (lane == 0) {
				o.ecc[si] = z2;
				o.dcc[si] = z2;
				if (sleaf) {
					o.cp[si] = z2;
					o.pc[si] = z2;
					o.pp[si] = z2;
				} else {
					o.eout[si] = z2;
					o.dout[si] = z2;
				}
			}
			continue;
		}
		// input check lists: the parent's pass-down lists, or {root} at the root
		const int* ein;
		const int* din;
		int ne, nd;
		int root_list = (int) si;
		if (si < p.nroot) {
			ein = din = &root_list;
			ne = nd = 1;
		} else {
			const int pa = parent[si];
			const int2 e = o.eout[pa], d = o.dout[pa];
			ein = o.pass_prev + e.x;
			ne = e.y;
			din = o.pass_prev + d.x;
			nd = d.y;
		}
		int32_t sbox[6];
		if (sleaf) {
			for (int d = 0; d < 6; d++) {
				sbox[d] = nbox[6 * si + d];
			}
		}
		const float rs = self.radius;
		// ---- Ewald list: one pass
		int n_ecc = 0, n_eout = 0;
		for (int j0 = 0; j0 < ne; j0 += 32) {
			const int j = j0 + lane;
			int cc = 0, nx = 0, c = 0, c0 = 0;
			if (j < ne) {
				c = ein[j];
				const NodeW ot = nodes[c];
				if (ot.pend > ot.pbeg) {
					const float dx = fixed_dist(self.x, ot.x), dy = fixed_dist(self.y, ot.y), dz = fixed_dist(self.z, ot.z);
					float R2 = sqrf3(dx, dy, dz);
					const float t = fmaxf(__fsub_rn(0.5f, __fadd_rn(rs, ot.radius)), 0.f);
					R2 = fmaxf(R2, __fmul_rn(t, t));
					const float dcc = __fmul_rn(__fadd_rn(rs, ot.radius), thetainv);
					cc = R2 > __fmul_rn(dcc, dcc);
					if (!cc) {
						if (ot.child >= 0 && !sleaf) {
							nx = 2;
							c0 = ot.child;
						} else {
							dropped = 1;
						}
					}
				}
			}
			stage_push(sl[S_ECC], n_ecc, cap, lane, cc, c, 0, &ovf);
			stage_push(sl[S_EOUT], n_eout, cap, lane, nx, c0, c0 + 1, &ovf);
		}
		// ---- direct list (leaf: iterate over the children it opens)
		int n_dcc = 0, n_cp = 0, n_pc = 0, n_leaf = 0, n_next = 0;
		const int* cur = din;
		int ncur = nd;
		int which = 0;
		while (true) {
			int* nxt = sl[S_NEXT0 + which];
			n_next = 0;
			for (int j0 = 0; j0 < ncur; j0 += 32) {
				const int j = j0 + lane;
				int kind = -1, c = 0;  // 0 cc 1 cp 2 pc 3 leaf 4 next
				int c0 = 0;
				if (j < ncur) {
					c = cur[j];
					const NodeW ot = nodes[c];
					const int onp = ot.pend - ot.pbeg;
					if (onp) {
						const float dx = fixed_dist(self.x, ot.x), dy = fixed_dist(self.y, ot.y), dz = fixed_dist(self.z, ot.z);
						const float R2 = sqrf3(dx, dy, dz);
						const float rsum = __fadd_rn(rs, ot.radius);
						const float mind = __fadd_rn(rsum, h);
						const float dcc = fmaxf(__fmul_rn(rsum, thetainv), mind);
						const bool oleaf = ot.flags & 1;
						bool sw_cc = R2 > __fmul_rn(dcc, dcc), sw_cp = false, sw_pc = false;
						if (!sw_cc && oleaf && sleaf) {
							const float dcp = fmaxf(__fadd_rn(__fmul_rn(rs, thetainv), ot.radius), mind);
							const float dpc = fmaxf(__fadd_rn(rs, __fmul_rn(ot.radius, thetainv)), mind);
							sw_pc = (R2 > __fmul_rn(dpc, dpc) || !box_sphere(sbox, ot.x, ot.y, ot.z, fmaxf(__fmul_rn(thetainv, ot.radius), h)))
									&& nsinks >= MIN_PARTS_PCCP;
							int32_t obox[6];
							for (int d = 0; d < 6; d++) {
								obox[d] = nbox[6 * (int64_t) c + d];
							}
							sw_cp = (R2 > __fmul_rn(dcp, dcp) || !box_sphere(obox, self.x, self.y, self.z, fmaxf(__fmul_rn(thetainv, rs), h)))
									&& onp >= MIN_PARTS_PCCP;
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
							kind = 0;
						} else if (sw_cp) {
							kind = 1;
						} else if (sw_pc) {
							kind = 2;
						} else if (oleaf) {
							kind = 3;
						} else {
							kind = 4;
							c0 = ot.child;
						}
					}
				}
				stage_push(sl[S_DCC], n_dcc, cap, lane, kind == 0, c, 0, &ovf);
				stage_push(sl[S_CP], n_cp, cap, lane, kind == 1, c, 0, &ovf);
				stage_push(sl[S_PC], n_pc, cap, lane, kind == 2, c, 0, &ovf);
				stage_push(sl[S_LEAF], n_leaf, cap, lane, kind == 3, c, 0, &ovf);
				stage_push(nxt, n_next, cap, lane, kind == 4 ? 2 : 0, c0, c0 + 1, &ovf);
			}
			__syncwarp();
			if (sleaf && n_next > 0) {
				cur = nxt;
				ncur = min(n_next, cap);
				which ^= 1;
				continue;
			}
			break;
		}
		__syncwarp();
		// ---- flush to global lists
		const int2 ecc = flush(sl[S_ECC], n_ecc, cap, o.ecc_list, o.cursor + 0, o.cap_cc, lane, o.flags);
		const int2 dcc = flush(sl[S_DCC], n_dcc, cap, o.dcc_list, o.cursor + 1, o.cap_cc, lane, o.flags);
		if (lane == 0) {
			o.ecc[si] = ecc;
			o.dcc[si] = dcc;
		}
		if (sleaf) {
			const int2 cp = flush(sl[S_CP], n_cp, cap, o.cp_list, o.cursor + 2, o.cap_leaf, lane, o.flags);
			const int2 pc = flush(sl[S_PC], n_pc, cap, o.pc_list, o.cursor + 3, o.cap_leaf, lane, o.flags);
			const int2 pp = flush(sl[S_LEAF], n_leaf, cap, o.pp_list, o.cursor + 4, o.cap_leaf, lane, o.flags);
			if (lane == 0) {
				o.cp[si] = cp;
				o.pc[si] = pc;
				o.pp[si] = pp;
			}
		} else {
			// Ewald pass-down: children of the opened checks
			const int2 eo = flush(sl[S_EOUT], n_eout, cap, o.pass_cur, o.cursor + 5, o.cap_pass, lane, o.flags);
			// direct pass-down: children of opened checks, then the leaf checks (kick.cu:424-430)
			const int nn = min(n_next, cap), nl = min(n_leaf, cap);
			unsigned long long off = 0;
			if (lane == 0 && nn + nl) {
				off = atomicAdd(o.cursor + 5, (unsigned long long) (nn + nl));
			}
			off = __shfl_sync(0xffffffffu, off, 0);
			int2 dout = make_int2(0, 0);
			if ((long long) (off + nn + nl) > o.cap_pass) {
				if (lane == 0) {
					atomicOr(o.flags, 1);
				}
			} else {
				const int* nxt = sl[S_NEXT0 + which];
				for (int i = lane; i < nn; i += 32) {
					o.pass_cur[off + i] = nxt[i];
				}
				for (int i = lane; i < nl; i += 32) {
					o.pass_cur[off + nn + i] = sl[S_LEAF][i];
				}
				dout = make_int2((int) off, nn + nl);
			}
			if (lane == 0) {
				o.eout[si] = eo;
				o.dout[si] = dout;
			}
		}
		__syncwarp();
	}
	if (ovf) {
		atomicOr(o.flags, 1);
	}
	if (dropped) {
		atomicOr(o.flags + 1, 1);
	}
}

// ---------------------------------------------------------------- M2L / P2L
template<int N>
__device__ __forceinline__ void warp_reduce_arr(float* L) {
	for (int o = 16; o; o >>= 1) {
		for (int i = 0; i < N; i++) {
			L[i] += __shfl_xor_sync(0xffffffffu, L[i], o);
		}
	}
}

// Ewald M2L for every node: dL = sum over the Ewald CC list.
// Work units of a warp in a resident grid: lane 0 takes the next `chunk` units from the
// counter, so that warps that finish early take more (tile costs vary with the leaf's size and
// lists) and no partly filled last wave of blocks is left.
__device__ __forceinline__ int64_t warp_take(unsigned long long* next, int chunk) {
	unsigned long long v = 0;
	if ((threadIdx.x & 31) == 0) {
		v = atomicAdd(next, (unsigned long long) chunk);
	}
	return (int64_t) __shfl_sync(0xffffffffu, v, 0);
}
// The node-indexed interaction kernels (Ewald M2L, direct M2L, P2L) visit the nodes of their
// kind in `order`, longest lists first (nodes without a list of the kind sort last), and each
// warp of a resident grid takes the next node from `next` when it is done with one: list
// lengths vary by orders of magnitude, and a static interleave left the busiest SM with
// 1.2-1.5x the mean SM's work.  Each node's sum is still made by one warp in list order, so
// the results do not depend on the schedule.
__device__ __forceinline__ int64_t next_node(unsigned long long* next, const int32_t* __restrict__ order, int64_t nn) {
	const int64_t k = warp_take(next, 1);
	return k < nn ? (int64_t) order[k] : -1;
}

template<class Ops>
__global__ void __launch_bounds__(128, 4) k_m2l_ewald(int64_t nn, const int32_t* __restrict__ order, unsigned long long* next, const NodeW* __restrict__ nodes,
		const float* __restrict__ multi, const int2* __restrict__ ecc, const int* __restrict__ ecc_list, float* __restrict__ dL, int do_phi, double* counters) {
	constexpr int NE = Ops::NEXP, NM = Ops::NMULT;
	__shared__ float s_real[CT_EWALD_NREAL][3];
	__shared__ float s_L[4][32][51];
	// the Fourier terms' derivative tensors of the first half of the table (one of each +h/-h
	// pair) in shared memory, read by a rolled loop: the unrolled loop over constant-memory
	// operands made the kernel long enough to stall on instruction fetch (the 128-box
	// ensemble's M2L phase 85 -> 52 ms)
	__shared__ __align__(16) float s_fexp[CT_EWALD_NFOUR / 2][NE];
	const auto& ct = ewald_tab<Ops>();
	for (int i = threadIdx.x; i < CT_EWALD_NREAL * 3; i += blockDim.x) {
		s_real[i / 3][i % 3] = ct.real[i / 3][i % 3];
	}
	for (int i = threadIdx.x; i < (CT_EWALD_NFOUR / 2) * NE; i += blockDim.x) {
		s_fexp[i / NE][i % NE] = ct.four_exp[i / NE][i % NE];
	}
	__syncthreads();
	const EwaldView<typename Ops::Tab> view { s_real, ct.four, s_fexp, ct.D0 };
	const int lane = threadIdx.x & 31;
	double icnt_tot = 0;
	for (;;) {
		const int64_t si = next_node(next, order, nn);
		if (si < 0) {
			break;
		}
		const int2 lst = ecc[si];
		if (lst.y == 0) {
			break;  // the rest of the order holds no Ewald list either (dL is zeroed before the launch)
		}
		const NodeW self = nodes[si];
		// this lane's expansion sum in shared memory (rows of 51 floats: lanes on distinct banks),
		// which leaves the registers to the Green's function
		float* L = &s_L[threadIdx.x >> 5][lane][0];
		for (int i = 0; i < NE; i++) {
			L[i] = 0.f;
		}
		for (int j = lane; j < lst.y; j += 32) {
			const int c = ecc_list[lst.x + j];
			const NodeW ot = nodes[c];
			float M[NM], D[NE];
			const int ic = Ops::ewald(D, fixed_dist(self.x, ot.x), fixed_dist(self.y, ot.y), fixed_dist(self.z, ot.z), view);
			icnt_tot += ic;
			const float4* mp = (const float4*) (multi + (size_t) NMULT_STRIDE * c);
#pragma unroll
			for (int k = 0; k < (NM + 3) / 4; k++) {
				const float4 v = __ldg(mp + k);
				if (4 * k + 0 < NM) M[4 * k + 0] = v.x;
				if (4 * k + 1 < NM) M[4 * k + 1] = v.y;
				if (4 * k + 2 < NM) M[4 * k + 2] = v.z;
				if (4 * k + 3 < NM) M[4 * k + 3] = v.w;
			}
			Ops::m2l(L, M, D, do_phi != 0);
		}
		__syncwarp();
		// entry n summed over the 32 lanes' rows by lane n % 32
		for (int n = lane; n < NE; n += 32) {
			float t = 0.f;
			for (int q = 0; q < 32; q++) {
				t += s_L[threadIdx.x >> 5][q][n];
			}
			dL[NEXP_STRIDE * si + n] = t;
		}
		__syncwarp();
	}
	icnt_tot += __shfl_xor_sync(0xffffffffu, icnt_tot, 16);
	icnt_tot += __shfl_xor_sync(0xffffffffu, icnt_tot, 8);
	icnt_tot += __shfl_xor_sync(0xffffffffu, icnt_tot, 4);
	icnt_tot += __shfl_xor_sync(0xffffffffu, icnt_tot, 2);
	icnt_tot += __shfl_xor_sync(0xffffffffu, icnt_tot, 1);
	if (lane == 0 && icnt_tot > 0) {
		atomicAdd(counters + 0, icnt_tot);
	}
}

// Asynchronous 16-byte global -> shared copies (cp.async; L1-allocating, the multipoles of
// a source node are read by many sink nodes): one group per stage, waited for per thread.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
	const unsigned s = (unsigned) __cvta_generic_to_shared(smem);
	asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
	asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template<int N>
__device__ __forceinline__ void cp_async_wait() {
	asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Shared memory of k_m2l_direct: per warp the 32 lanes' expansion rows (51 floats: lanes on
// distinct banks) and two stages of one source per lane (its centre and radius, 16 bytes, and
// its multipole row, 160 bytes).
constexpr int M2L_STAGE = 44;  // floats per lane and stage
constexpr size_t M2L_DIRECT_SMEM = sizeof(float) * (4 * 32 * 51 + 4 * 2 * 32 * M2L_STAGE);

// Direct M2L: dL += sum over the direct CC list (gravity.cu:44-73).  Lanes take the sources
// 32 apart; each lane copies its next source (centre and multipole) into shared memory while
// it evaluates the current one, so that the gathers from global memory overlap the arithmetic.
template<class Ops>
__global__ void __launch_bounds__(128, 3) k_m2l_direct(int64_t nn, const int32_t* __restrict__ order, unsigned long long* next, const NodeW* __restrict__ nodes,
		const float* __restrict__ multi, const int2* __restrict__ dcc, const int* __restrict__ dcc_list, float* __restrict__ dL, int do_phi) {
	constexpr int NE = Ops::NEXP, NM = Ops::NMULT;
	extern __shared__ __align__(16) float m2l_smem[];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	float* s_L = m2l_smem;  // [4][32][51]
	float* my_stage = m2l_smem + 4 * 32 * 51 + ((w * 2) * 32 + lane) * M2L_STAGE;  // stage b at + b * 32 * M2L_STAGE
	auto stage = [&](int c, int b) {
		float* d = my_stage + b * 32 * M2L_STAGE;
		cp_async16(d, nodes + c);
		const float* mp = multi + (size_t) NMULT_STRIDE * c;
#pragma unroll
		for (int k = 0; k < (NM + 3) / 4; k++) {
			cp_async16(d + 4 + 4 * k, mp + 4 * k);
		}
	};
	for (;;) {
		const int64_t si = next_node(next, order, nn);
		if (si < 0) {
			break;
		}
		const int2 lst = dcc[si];
		if (lst.y == 0) {
			break;  // the rest of the order holds no direct list either
		}
		const NodeW self = nodes[si];
		float* L = s_L + (w * 32 + lane) * 51;
		for (int i = 0; i < NE; i++) {
			L[i] = 0.f;
		}
		int b = 0;
		if (lane < lst.y) {
			stage(dcc_list[lst.x + lane], 0);
		}
		cp_async_commit();
		for (int j = lane; j < lst.y; j += 32) {
			if (j + 32 < lst.y) {
				stage(dcc_list[lst.x + j + 32], b ^ 1);
			}
			cp_async_commit();
			cp_async_wait<1>();  // this stage's copies (all but the group just committed)
			const float* d = my_stage + b * 32 * M2L_STAGE;
			const uint4 oc = *(const uint4*) d;
			float M[NM], D[NE];
#pragma unroll
			for (int k = 0; k < (NM + 3) / 4; k++) {
				const float4 v = *(const float4*) (d + 4 + 4 * k);
				if (4 * k + 0 < NM) M[4 * k + 0] = v.x;
				if (4 * k + 1 < NM) M[4 * k + 1] = v.y;
				if (4 * k + 2 < NM) M[4 * k + 2] = v.z;
				if (4 * k + 3 < NM) M[4 * k + 3] = v.w;
			}
			Ops::greens(D, fixed_dist(self.x, oc.x), fixed_dist(self.y, oc.y), fixed_dist(self.z, oc.z));
			Ops::m2l(L, M, D, do_phi != 0);
			b ^= 1;
		}
		cp_async_wait<0>();
		__syncwarp();
		// entry n summed over the 32 lanes' rows by lane n % 32
		for (int n = lane; n < NE; n += 32) {
			float t = 0.f;
			for (int q = 0; q < 32; q++) {
				t += s_L[(w * 32 + q) * 51 + n];
			}
			dL[NEXP_STRIDE * si + n] += t;
		}
		__syncwarp();
	}
}

// P2L (gravity.cu:134-144): every particle of the leaf's CP source leaves adds its Green's
// function to the leaf's expansion, dL += sum D(x_leaf - x_p).  The source leaves' particles
// are taken as one flat sequence (32 leaves at a time, prefix sums of their sizes in
// registers), so lanes stay busy across leaf boundaries; each lane prefetches its next
// particle's position while it evaluates the current one.
template<class Ops>
__global__ void __launch_bounds__(128, 5) k_p2l(int64_t nn, const int32_t* __restrict__ order, unsigned long long* next, const NodeW* __restrict__ nodes,
		const int2* __restrict__ cp, const int* __restrict__ cp_list, const uint32_t* __restrict__ x0, const uint32_t* __restrict__ x1,
		const uint32_t* __restrict__ x2, float* __restrict__ dL, double* counters) {
	constexpr int NE = Ops::NEXP;
	const int lane = threadIdx.x & 31;
	double ncp = 0;
	for (;;) {
		const int64_t si = next_node(next, order, nn);
		if (si < 0) {
			break;
		}
		const int2 cpl = cp[si];
		if (cpl.y == 0 || !(nodes[si].flags & 1)) {
			break;  // the rest of the order holds no P2L list either (only leaves have one)
		}
		const NodeW self = nodes[si];
		float L[NE];
		for (int i = 0; i < NE; i++) {
			L[i] = 0.f;
		}
		for (int qb = 0; qb < cpl.y; qb += 32) {
			int beg = 0, cnt = 0;
			if (qb + lane < cpl.y) {
				const NodeW s = nodes[cp_list[cpl.x + qb + lane]];
				beg = s.pbeg;
				cnt = s.pend - s.pbeg;
			}
			int inc = cnt;  // inclusive prefix of the sizes over lanes
#pragma unroll
			for (int o = 1; o < 32; o <<= 1) {
				const int t = __shfl_up_sync(0xffffffffu, inc, o);
				inc += lane >= o ? t : 0;
			}
			const int total = __shfl_sync(0xffffffffu, inc, 31);
			const int start = inc - cnt;  // this lane's leaf: flat indices [start, inc)
			const int first = beg - start;  // particle index = first[owner] + flat index
			ncp += total;
			// particle of flat index gb + lane: the leaves ending at or before gb (one ballot)
			// plus the leaves starting inside (gb, gb + lane] (one OR-reduction of start bits)
			// give the owner lane (leaves holding particles start at distinct flat indices)
			auto particle = [&](int gb) {
				const int o0 = __popc(__ballot_sync(0xffffffffu, inc <= gb));
				const int rel = start - gb;
				const unsigned starts = __reduce_or_sync(0xffffffffu, (cnt > 0 && rel > 0 && rel < 32) ? (1u << rel) : 0u);
				const int owner = o0 + __popc(starts & ((2u << lane) - 1u));
				return __shfl_sync(0xffffffffu, first, owner & 31) + gb + lane;
			};
			int k = particle(0);
			uint32_t px = 0, py = 0, pz = 0;
			if (lane < total) {
				px = x0[k];
				py = x1[k];
				pz = x2[k];
			}
			for (int gb = 0; gb < total; gb += 32) {
				const uint32_t cx = px, cy = py, cz = pz;
				const bool have = gb + lane < total;
				if (gb + 32 < total) {
					k = particle(gb + 32);
					if (gb + 32 + lane < total) {
						px = x0[k];
						py = x1[k];
						pz = x2[k];
					}
				}
				if (have) {
					Ops::greens_add(L, fixed_dist(self.x, cx), fixed_dist(self.y, cy), fixed_dist(self.z, cz));
				}
			}
		}
		warp_reduce_arr<NE>(L);
		if (lane == 0) {
			for (int i = 0; i < NE; i++) {
				dL[NEXP_STRIDE * si + i] += L[i];
			}
		}
	}
	if (lane == 0 && ncp > 0) {
		atomicAdd(counters + 1, ncp);
	}
}

// Sort keys of the three node orders: the bit length of the node's list length of each kind (P2L
// lists count only at leaves), and the node indices to be sorted with them.  Sorting by the bit
// length (a stable sort) puts the longest lists first and keeps tree order among lists of
// similar length, so that warps working at the same time read nearby source nodes.
constexpr int ORDER_KEY_BITS = 6;  // bit lengths 0..32
__global__ void k_order_keys(int64_t nn, const NodeW* __restrict__ nodes, const int2* __restrict__ ecc, const int2* __restrict__ dcc,
		const int2* __restrict__ cp, uint32_t* __restrict__ key, int32_t* __restrict__ idx) {
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < nn; i += (int64_t) gridDim.x * blockDim.x) {
		const uint32_t le = (uint32_t) ecc[i].y, ld = (uint32_t) dcc[i].y, lp = (nodes[i].flags & 1) ? (uint32_t) cp[i].y : 0u;
		key[i] = 32u - __clz(le);
		key[nn + i] = 32u - __clz(ld);
		key[2 * nn + i] = 32u - __clz(lp);
		idx[i] = (int32_t) i;
	}
}

// ---------------------------------------------------------------- L2L (top-down, one level)
template<class Ops>
__global__ void k_l2l(int64_t lb, int64_t le, const NodeW* __restrict__ nodes, const int32_t* __restrict__ parent, const float* __restrict__ dL,
		const float* __restrict__ dL2, const float* __restrict__ dL3, float* __restrict__ Lx, int do_phi) {
	constexpr int NE = Ops::NEXP;
	for (int64_t i = lb + blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < le; i += (int64_t) gridDim.x * blockDim.x) {
		float out[NE], d[NE];
		// the node's M2L and P2L sums, added in the order one stream would add them
		for (int k = 0; k < NE; k++) {
			d[k] = (dL[NEXP_STRIDE * i + k] + dL2[NEXP_STRIDE * i + k]) + dL3[NEXP_STRIDE * i + k];
		}
		if (parent[i] < 0) {  // a root: the expansion starts at zero
			for (int k = 0; k < NE; k++) {
				out[k] = d[k];
			}
		} else {
			const int pa = parent[i];
			const NodeW nd = nodes[i], pn = nodes[pa];
			float La[NE];
			const float* src = Lx + NEXP_STRIDE * (int64_t) pa;
			for (int k = 0; k < NE; k++) {
				La[k] = src[k];
			}
			Ops::l2l(out, La, fixed_dist(nd.x, pn.x), fixed_dist(nd.y, pn.y), fixed_dist(nd.z, pn.z), do_phi != 0);
			for (int k = 0; k < NE; k++) {
				out[k] += d[k];
			}
		}
		float* dst = Lx + NEXP_STRIDE * i;
		for (int k = 0; k < NE; k++) {
			dst[k] = out[k];
		}
	}
}

// Neumaier-compensated running sum of per-batch partial forces.
__device__ __forceinline__ void ksum(float& s, float& comp, float v) {
	const float t = s + v;
	if (fabsf(s) >= fabsf(v)) {
		comp += (s - t) + v;
	} else {
		comp += (v - t) + s;
	}
	s = t;
}

// ---------------------------------------------------------------- leaf path
// P2P (a warp per 32-sink tile of a leaf; the particles of its P2P source leaves staged per
// warp in shared memory as offsets from the leaf centre), then M2P + L2P + kick per tile.
constexpr int P2P_TPB = 256;

struct P2PArgs {
	int nsub;
	const int64_t* sub_off;
	const float* sub_h;
	const NodeW* nodes;
	const int32_t* nbox;  // tight boxes of the nodes
	const int2* items;  // (leaf node, tile)
	int64_t nitems;
	const int2* pp;
	const int* pp_list;
	const uint32_t* x[3];
	float4* F;          // per particle: P2P sums (sum dx r^-3, ..., -sum r^-1)
	float h;
	int compensated;
	double* pairs;
	double* near_pairs;
	unsigned long long* next;  // work counter: warps take tiles in list order
	int tw;                    // sinks per tile (32, or 16: every tile through the SMALL path)
};

// Approximate reciprocal square root (the MUFU unit), flushing denormals: pair separations
// are at least one fixed32 unit, r^2 >= 2^-64, far above the denormal range.
__device__ __forceinline__ float rsqrt_ftz(float x) {
	float y;
	asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
	return y;
}

// r^-1 and r^-3 of a pair, or the Ferrer-softened values inside h (gravity.hpp:73-96).
__device__ __forceinline__ void pair_kernel(float r2, float h2, float hinv, float h2inv, float h3inv, float& r1inv, float& r3inv) {
	if (r2 > h2) {
		r1inv = rsqrt_ftz(r2);
		r3inv = r1inv * r1inv * r1inv;
	} else {
		const float q2 = r2 * h2inv;
		float f = 315.f / 128.f;
		f = fmaf(f, q2, -385.f / 32.f);
		f = fmaf(f, q2, 1485.f / 64.f);
		f = fmaf(f, q2, -693.f / 32.f);
		f = fmaf(f, q2, 1155.f / 128.f);
		r3inv = f * h3inv;
		float ph = -63.f / 256.f;
		ph = fmaf(ph, q2, 385.f / 256.f);
		ph = fmaf(ph, q2, -495.f / 128.f);
		ph = fmaf(ph, q2, 693.f / 128.f);
		ph = fmaf(ph, q2, -1155.f / 256.f);
		ph = fmaf(ph, q2, 693.f / 256.f);
		r1inv = ph * hinv;
	}
}

// Smallest distance between two leaves' tight boxes (fixed<int,29> raw, 6 per node) under the
// periodic wrap, squared, in box units.
__device__ __forceinline__ float box_gap2(const int32_t* a, const int32_t* b) {
	float g2 = 0.f;
#pragma unroll
	for (int d = 0; d < 3; d++) {
		// centre distance (wrapped to the nearest image) minus the two half widths
		const int64_t ca = (int64_t) a[d] + a[3 + d], cb = (int64_t) b[d] + b[3 + d];  // 2 x centre
		int64_t dc = ca - cb;                                                          // 2^30 = one box
		if (dc > ((int64_t) 1 << 29)) {
			dc -= (int64_t) 1 << 30;
		} else if (dc < -((int64_t) 1 << 29)) {
			dc += (int64_t) 1 << 30;
		}
		const int64_t adc = dc < 0 ? -dc : dc;
		const int64_t w = ((int64_t) a[3 + d] - a[d]) + ((int64_t) b[3 + d] - b[d]);
		const int64_t gap = adc - w;  // 2 x gap, 2^-30 units
		if (gap > 0) {
			const float gf = (float) gap * (1.0f / 1073741824.0f);
			g2 += gf * gf;
		}
	}
	return g2;
}

// Packed pairs of floats for the sm_100 f32x2 instructions: one instruction applies the same
// IEEE round-to-nearest operation to both halves, so each half is bit-identical to the scalar
// operation while the instruction issues once.
struct f2 {
	uint64_t v;
};
__device__ __forceinline__ f2 f2_pack(float lo, float hi) {
	f2 r;
	asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
	return r;
}
__device__ __forceinline__ void f2_unpack(f2 a, float& lo, float& hi) {
	asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
}
__device__ __forceinline__ f2 f2_sub(f2 a, f2 b) {
	f2 r;
	asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
	return r;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) {
	f2 r;
	asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
	return r;
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) {
	f2 r;
	asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
	return r;
}

// Staged sources of one warp: positions relative to the sink leaf's centre, x and y of source
// pairs interleaved (x_2i, x_2i+1, y_2i, y_2i+1) and z by quads, so that a pair of sources
// arrives as aligned register pairs for the f32x2 instructions.
template<int STAGE>
struct P2PStage {
	float4 xy[STAGE / 2];
	float4 z[STAGE / 4];
};

template<int STAGE>
__device__ __forceinline__ void stage_put(P2PStage<STAGE>* st, int j, float x, float y, float z) {
	float* xy = reinterpret_cast<float*>(st->xy);
	xy[4 * (j >> 1) + (j & 1)] = x;
	xy[4 * (j >> 1) + 2 + (j & 1)] = y;
	reinterpret_cast<float*>(st->z)[j] = z;
}

// One staged source against one sink with the per-pair softening test.
template<int STAGE>
__device__ __forceinline__ void p2p_checked(const P2PStage<STAGE>* st, int j, float kx, float ky, float kz, float h2, float hinv, float h2inv, float h3inv,
		float& fx, float& fy, float& fz, float& pt) {
	const float* xy = reinterpret_cast<const float*>(st->xy);
	const float dx = kx - xy[4 * (j >> 1) + (j & 1)];
	const float dy = ky - xy[4 * (j >> 1) + 2 + (j & 1)];
	const float dz = kz - reinterpret_cast<const float*>(st->z)[j];
	const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
	float r1, r3;
	pair_kernel(r2, h2, hinv, h2inv, h3inv, r1, r3);
	fx = fmaf(dx, r3, fx);
	fy = fmaf(dy, r3, fy);
	fz = fmaf(dz, r3, fz);
	pt -= r1;
}

// Sum over staged sources [0, cnt) for one sink.  CHECK: pairs may fall inside the softening
// length (per-pair test); otherwise every pair is known to be farther than h and sources go
// two at a time through f32x2 (even sources in the low half, odd in the high half).
//
// Sources [jb, je) of the chunk (jb a multiple of 4): the whole chunk for a full tile, a slice
// for one replica of a small tile.
template<bool CHECK, int STAGE>
__device__ __forceinline__ void p2p_chunk(const P2PStage<STAGE>* __restrict__ st, int jb, int je, float kx, float ky, float kz, float h2, float hinv,
		float h2inv, float h3inv, float& fx, float& fy, float& fz, float& pt) {
	int j = jb;
	const f2 KX = f2_pack(kx, kx), KY = f2_pack(ky, ky), KZ = f2_pack(kz, kz);
	f2 ax = f2_pack(0.f, 0.f), ay = ax, az = ax, ap = ax;
	// four sources (two f32x2 pairs) starting at q, a multiple of 4.  With CHECK, a quad with
	// a pair inside the softening length goes through the scalar per-pair test instead (rare:
	// near source leaves mostly hold pairs farther apart than h).
	auto quad = [&](int q) {
		const float4 xy0 = st->xy[q >> 1];
		const float4 xy1 = st->xy[(q >> 1) + 1];
		const float4 zz = st->z[q >> 2];
		const f2 dx0 = f2_sub(KX, f2_pack(xy0.x, xy0.y)), dy0 = f2_sub(KY, f2_pack(xy0.z, xy0.w)), dz0 = f2_sub(KZ, f2_pack(zz.x, zz.y));
		const f2 dx1 = f2_sub(KX, f2_pack(xy1.x, xy1.y)), dy1 = f2_sub(KY, f2_pack(xy1.z, xy1.w)), dz1 = f2_sub(KZ, f2_pack(zz.z, zz.w));
		const f2 q0 = f2_fma(dx0, dx0, f2_fma(dy0, dy0, f2_mul(dz0, dz0)));
		const f2 q1 = f2_fma(dx1, dx1, f2_fma(dy1, dy1, f2_mul(dz1, dz1)));
		float a0, b0, a1, b1;
		f2_unpack(q0, a0, b0);
		f2_unpack(q1, a1, b1);
		if (CHECK && !(fminf(fminf(a0, b0), fminf(a1, b1)) > h2)) {
			for (int t = 0; t < 4; t++) {
				p2p_checked(st, q + t, kx, ky, kz, h2, hinv, h2inv, h3inv, fx, fy, fz, pt);
			}
			return;
		}
		const f2 r10 = f2_pack(rsqrt_ftz(a0), rsqrt_ftz(b0));
		const f2 r11 = f2_pack(rsqrt_ftz(a1), rsqrt_ftz(b1));
		const f2 r30 = f2_mul(f2_mul(r10, r10), r10);
		const f2 r31 = f2_mul(f2_mul(r11, r11), r11);
		ax = f2_fma(dx0, r30, ax);
		ay = f2_fma(dy0, r30, ay);
		az = f2_fma(dz0, r30, az);
		ap = f2_sub(ap, r10);
		ax = f2_fma(dx1, r31, ax);
		ay = f2_fma(dy1, r31, ay);
		az = f2_fma(dz1, r31, az);
		ap = f2_sub(ap, r11);
	};
	if (!CHECK && jb == 0 && je == STAGE) {
		// a full chunk: constant offsets; unrolled by 8 quads, not fully (the fully unrolled
		// chunk, ~1,500 instructions, stalled warps on instruction fetch: 36.1 -> 35.0 ms at 256^3)
#pragma unroll 8
		for (int q = 0; q < STAGE; q += 4) {
			quad(q);
		}
		j = STAGE;
	} else {
#pragma unroll 2
		for (; j + 3 < je; j += 4) {
			quad(j);
		}
	}
	float lo, hi;
	f2_unpack(ax, lo, hi);
	fx += lo + hi;
	f2_unpack(ay, lo, hi);
	fy += lo + hi;
	f2_unpack(az, lo, hi);
	fz += lo + hi;
	f2_unpack(ap, lo, hi);
	pt += lo + hi;
	for (; j < je; j++) {
		p2p_checked(st, j, kx, ky, kz, h2, hinv, h2inv, h3inv, fx, fy, fz, pt);
	}
}

// The two warps of pair `pair` (warps 2 pair and 2 pair + 1 of the block) meet here: a named
// barrier of 64 threads (ids 1.., id 0 being __syncthreads').
__device__ __forceinline__ void pair_sync(int pair) {
	asm volatile("bar.sync %0, 64;" ::"r"(1 + pair) : "memory");
}

// SMALL: tiles of at most 16 sinks.  S' = S rounded up to a power of two lanes hold the sinks
// (lanes past S repeat a sink and are not written); the 32 / S' groups of S' lanes (replicas)
// each take a contiguous slice of every staged chunk and are added by a butterfly at the end.
// STAGE: sources staged per chunk (the cell-list size).  WPT: warps per tile; with 2, the
// warps of a pair take one tile together, each every other chunk of its sources, and the
// second warp's sums are added to the first's in a fixed order (deterministic).
template<bool SMALL, int STAGE, int WPT>
__global__ void __launch_bounds__(P2P_TPB, 3) k_p2p(P2PArgs a) {
	static_assert(WPT == 1 || WPT == 2, "one or two warps per tile");
	__shared__ P2PStage<STAGE> stage[P2P_TPB / 32];
	__shared__ float4 comb[WPT > 1 ? P2P_TPB / 64 : 1][2][32];
	__shared__ long long pair_tile[P2P_TPB / 64];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const int pw = WPT > 1 ? (w & 1) : 0, pair = w >> 1;
	P2PStage<STAGE>* my = &stage[w];
	double npairs = 0.0, nnear = 0.0;
	// a resident grid; each warp (pair of warps) takes the next tile when it is done with one
	for (;;) {
		int64_t it;
		if (WPT == 1) {
			it = warp_take(a.next, 1);
		} else {
			if (pw == 0) {
				const int64_t t = warp_take(a.next, 1);
				if (lane == 0) {
					pair_tile[pair] = t;
				}
			}
			pair_sync(pair);
			it = pair_tile[pair];
		}
		if (it >= a.nitems) {
			break;
		}
		const int2 item = a.items[it];
		const NodeW self = a.nodes[item.x];
		const float h = a.sub_h ? a.sub_h[box_of(a.sub_off, a.nsub, self.pbeg)] : a.h;
		const float h2 = h * h, hinv = 1.f / h, h2inv = hinv * hinv, h3inv = h2inv * hinv;
		// a source leaf needs the per-pair softening test only if its box comes within h of the
		// sink leaf's box (margin far above the boxes' truncation and float rounding)
		const float near2 = h2 * 1.01f;
		int sl = lane, rep = 0, Sp = 32;
		if (SMALL) {
			const int S = max(1, min(a.tw, self.pend - (self.pbeg + a.tw * item.y)));  // 1..16
			Sp = S <= 1 ? 1 : 1 << (32 - __clz(S - 1));
			sl = lane & (Sp - 1);
			rep = lane / Sp;
			sl = sl < S ? sl : sl - S;  // sl < Sp < 2S
		}
		const int k = self.pbeg + a.tw * item.y + sl;
		const bool active = SMALL ? (rep == 0 && (lane & (Sp - 1)) == sl) : k < self.pend;
		float kx = 0.f, ky = 0.f, kz = 0.f;
		if (SMALL || active) {
			kx = fixed_dist(a.x[0][k], self.x);
			ky = fixed_dist(a.x[1][k], self.y);
			kz = fixed_dist(a.x[2][k], self.z);
		}
		float sx = 0.f, sy = 0.f, sz = 0.f, sp = 0.f, cx = 0.f, cy = 0.f, cz = 0.f, cp = 0.f;
		const int2 ppl = a.pp[item.x];
		int64_t np = 0, nn = 0;
		for (int qb = 0; qb < ppl.y; qb += 32) {
			// lanes take 32 source leaves at a time: particle range and class (near: the leaf's
			// box comes within h of the sink leaf's box, so pairs need the softening test)
			int beg = 0, cnt = 0;
			bool near = false;
			if (qb + lane < ppl.y) {
				const int sl = a.pp_list[ppl.x + qb + lane];
				const int2 pr = *reinterpret_cast<const int2*>(&a.nodes[sl].pbeg);
				beg = pr.x;
				cnt = pr.y - pr.x;
				near = box_gap2(a.nbox + 6 * (int64_t) item.x, a.nbox + 6 * (int64_t) sl) <= near2;
			}
			// far leaves first, then near ones; the particles of one class form a single flat
			// sequence (prefix sums of the leaf sizes over lanes), staged STAGE at a time
			for (int cls = 0; cls < 2; cls++) {
				const bool check = cls != 0;
				const int c = near == check ? cnt : 0;
				int inc = c;
#pragma unroll
				for (int o = 1; o < 32; o <<= 1) {
					const int t = __shfl_up_sync(0xffffffffu, inc, o);
					inc += lane >= o ? t : 0;
				}
				const int total = __shfl_sync(0xffffffffu, inc, 31);
				const int first = beg - (inc - c);  // particle index = first[owner] + flat index
				for (int gb = (WPT > 1 ? pw * STAGE : 0); gb < total; gb += WPT * STAGE) {
					const int n = min(STAGE, total - gb);
#pragma unroll
					for (int j = lane; j < STAGE; j += 32) {
						const int g = gb + j;
						// owner lane of flat index g: the lanes whose inclusive prefix is <= g
						int l = 0;
#pragma unroll
						for (int st = 16; st; st >>= 1) {
							l += __shfl_sync(0xffffffffu, inc, l + st - 1) <= g ? st : 0;
						}
						const int pi = __shfl_sync(0xffffffffu, first, l) + g;
						if (g < total) {
							stage_put(my, j, fixed_dist(a.x[0][pi], self.x), fixed_dist(a.x[1][pi], self.y), fixed_dist(a.x[2][pi], self.z));
						}
					}
					__syncwarp();
					float fx = 0.f, fy = 0.f, fz = 0.f, pt = 0.f;
					int jb = 0, je = n;
					if (SMALL) {
						const int R = 32 / Sp;
						const int sub = ((n + R - 1) / R + 3) & ~3;
						jb = min(n, rep * sub);
						je = min(n, jb + sub);
					}
					if (check) {
						p2p_chunk<true, STAGE>(my, jb, je, kx, ky, kz, h2, hinv, h2inv, h3inv, fx, fy, fz, pt);
					} else {
						p2p_chunk<false, STAGE>(my, jb, je, kx, ky, kz, h2, hinv, h2inv, h3inv, fx, fy, fz, pt);
					}
					__syncwarp();
					if (a.compensated) {
						ksum(sx, cx, fx);
						ksum(sy, cy, fy);
						ksum(sz, cz, fz);
						ksum(sp, cp, pt);
					} else {
						sx += fx;
						sy += fy;
						sz += fz;
						sp += pt;
					}
					np += n;
					nn += check ? n : 0;
				}
			}
		}
		float tx = sx + cx, ty = sy + cy, tz = sz + cz, tp = sp + cp;
		if (WPT > 1) {
			// the second warp's sums added to the first's (this order in every run)
			if (pw == 1) {
				comb[pair][0][lane] = make_float4(tx, ty, tz, tp);
			}
			pair_sync(pair);
			if (pw == 0) {
				const float4 o = comb[pair][0][lane];
				tx += o.x;
				ty += o.y;
				tz += o.z;
				tp += o.w;
			}
		}
		if (SMALL) {
			for (int o = Sp; o < 32; o <<= 1) {
				tx += __shfl_xor_sync(0xffffffffu, tx, o);
				ty += __shfl_xor_sync(0xffffffffu, ty, o);
				tz += __shfl_xor_sync(0xffffffffu, tz, o);
				tp += __shfl_xor_sync(0xffffffffu, tp, o);
			}
		}
		if (active) {
			if (pw == 0) {
				a.F[k] = make_float4(tx, ty, tz, tp);
			}
			npairs += (double) np;
			nnear += (double) nn;
		}
	}
	for (int o = 16; o; o >>= 1) {
		npairs += __shfl_xor_sync(0xffffffffu, npairs, o);
		nnear += __shfl_xor_sync(0xffffffffu, nnear, o);
	}
	if (lane == 0 && npairs > 0) {
		atomicAdd(a.pairs, npairs);
		atomicAdd(a.near_pairs, nnear);
	}
}

// Tiles with more than 16 sinks to `big`, the others to `small` (order within each list is
// immaterial: every tile computes its own sinks).
__global__ void k_split_tiles(const int2* __restrict__ items, int64_t nitems, const NodeW* __restrict__ nodes, int tw, int2* big, int2* small,
		unsigned long long* counts) {
	for (int64_t it = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; it < nitems; it += (int64_t) gridDim.x * blockDim.x) {
		const int2 item = items[it];
		const NodeW nd = nodes[item.x];
		const int S = min(tw, nd.pend - (nd.pbeg + tw * item.y));
		if (S > 16) {
			big[atomicAdd(counts, 1ull)] = item;
		} else {
			small[atomicAdd(counts + 1, 1ull)] = item;
		}
	}
}

struct KickTileArgs {
	int nsub;               // > 1: per-box sums for an ensemble
	const int64_t* sub_off; // particle offsets of the boxes (nsub + 1)
	double* sub_sums;       // 9 per box
	int* sub_maxrung;
	const float* sub_h;
	const float* sub_GM;
	const int* sub_first;
	const NodeW* nodes;
	const float* multi;
	const float* Lx;
	const int2* items;
	int64_t nitems;
	const int2* pc;
	const int* pc_list;
	const float4* F;
	const uint32_t* x[3];
	float* v[3];
	int8_t* rung;
	float* g[3];
	float* pot;
	ct_kick_params kp;
	double* sums;
	int* max_rung;
	unsigned long long* next;  // work counter (resident grid, tiles taken in list order)
	int tw;                    // sinks per tile (32 or 16)
};

// M2P, L2P and the kick for one tile (at most 32 sinks) per warp (gravity.cu:157-211, kick.cu:53-177).
// Sums of the kick return go to one set per box: block-reduced for a single box, per tile
// (warp-reduced, atomically added to the tile's box) for an ensemble.
template<class Ops>
__global__ void __launch_bounds__(128, 3) k_leaf_kick(KickTileArgs a) {
	constexpr int NE = Ops::NEXP, NM = Ops::NMULT;
	__shared__ double s_red[4][9];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const auto& kp = a.kp;
	double acc[9];
	for (int q = 0; q < 9; q++) {
		acc[q] = 0.0;
	}
	int maxr = 0;
	for (int64_t it = warp_take(a.next, 1); it < a.nitems; it = warp_take(a.next, 1)) {
		const int2 item = a.items[it];
		const NodeW self = a.nodes[item.x];
		const int bx = a.nsub > 1 ? box_of(a.sub_off, a.nsub, self.pbeg) : 0;
		const float hh = a.sub_h ? a.sub_h[bx] : kp.h;
		const float GM = a.sub_GM ? a.sub_GM[bx] : kp.GM;
		const bool first_call = a.sub_first ? a.sub_first[bx] != 0 : kp.first_call != 0;
		const float hinv = 1.f / hh;
		// S sinks in this tile; with at most 16, R = 32 / S lanes (replicas) share each sink's
		// M2P list (replica r takes every R-th source node); every lane holds a real sink
		const int S = max(1, min(a.tw, self.pend - (self.pbeg + a.tw * item.y)));
		const int R = S <= 16 ? 32 / S : 1;
		const int sink = lane % S, rep = lane / S;
		const int k = self.pbeg + a.tw * item.y + sink;
		const bool active = rep == 0;
		const uint32_t X[3] = { a.x[0][k], a.x[1][k], a.x[2][k] };
		float Fx = 0.f, Fy = 0.f, Fz = 0.f, Fp = rep == 0 ? (693.f / 256.f) * hinv : 0.f;
		const int2 pcl = a.pc[item.x];
		for (int q = rep < R ? rep : 0; q < pcl.y; q += R) {
			const int c = a.pc_list[pcl.x + q];
			const NodeW ot = a.nodes[c];
			float M[NM], D[NE], L2[5] = { 0.f, 0.f, 0.f, 0.f, 0.f };
			const float4* mp = (const float4*) (a.multi + (size_t) NMULT_STRIDE * c);
#pragma unroll
			for (int i = 0; i < (NM + 3) / 4; i++) {
				const float4 v = __ldg(mp + i);
				if (4 * i + 0 < NM) M[4 * i + 0] = v.x;
				if (4 * i + 1 < NM) M[4 * i + 1] = v.y;
				if (4 * i + 2 < NM) M[4 * i + 2] = v.z;
				if (4 * i + 3 < NM) M[4 * i + 3] = v.w;
			}
			Ops::greens(D, fixed_dist(X[0], ot.x), fixed_dist(X[1], ot.y), fixed_dist(X[2], ot.z));
			Ops::m2l2(L2, M, D, kp.do_phi != 0);
			Fx -= 1e6f * L2[1];
			Fy -= 1e6f * L2[2];
			Fz -= 1e6f * L2[3];
			Fp += 1e3f * L2[0];
		}
		if (R > 1) {
			// replica 0 adds the other replicas' sums, in replica order (lane sink + t S <= 31)
			const float ox = Fx, oy = Fy, oz = Fz, op = Fp;
			for (int t = 1; t < R; t++) {
				const int src = sink + t * S;
				Fx += __shfl_sync(0xffffffffu, ox, src);
				Fy += __shfl_sync(0xffffffffu, oy, src);
				Fz += __shfl_sync(0xffffffffu, oz, src);
				Fp += __shfl_sync(0xffffffffu, op, src);
			}
		}
		double ia[9];
		for (int q = 0; q < 9; q++) {
			ia[q] = 0.0;
		}
		int imax = 0;
		if (active) {
			ia[8] = pcl.y;
			const float4 P = a.F[k];
			Fx -= P.x;
			Fy -= P.y;
			Fz -= P.z;
			Fp += P.w;
			float La[NE], L2[5];
			const float* Lsrc = a.Lx + (size_t) NEXP_STRIDE * item.x;
			for (int i = 0; i < NE; i++) {
				La[i] = Lsrc[i];
			}
			Ops::l2p(L2, La, fixed_dist(X[0], self.x), fixed_dist(X[1], self.y), fixed_dist(X[2], self.z), kp.do_phi != 0);
			Fp += 1e3f * L2[0];
			Fx -= 1e6f * L2[1];
			Fy -= 1e6f * L2[2];
			Fz -= 1e6f * L2[3];
			Fz *= GM;
			Fy *= GM;
			Fx *= GM;
			Fp *= GM;
			float vx = a.v[0][k], vy = a.v[1][k], vz = a.v[2][k];
			const float kin0 = (float) (0.5 * (double) (vx * vx + vy * vy + vz * vz));
			const float sgn = kp.sign * (kp.top ? 1.f : -1.f);
			const float rdt = 1.0f / (float) (1 << kp.min_rung);
			if (kp.ascending) {
				const float dt = 0.5f * rdt * kp.t0;
				if (!first_call) {
					vx = fmaf(sgn * Fx, dt, vx);
					vy = fmaf(sgn * Fy, dt, vy);
					vz = fmaf(sgn * Fz, dt, vz);
				}
			}
			ia[1] = 0.5f * (vx * vx + vy * vy + vz * vz);
			ia[3] = vx;
			ia[4] = vy;
			ia[5] = vz;
			ia[6] = sqrtf(vx * vx + vy * vy + vz * vz);
			if (kp.save_force) {
				a.g[0][k] = Fx;
				a.g[1][k] = Fy;
				a.g[2][k] = Fz;
				a.pot[k] = Fp;
			}
			if (kp.descending) {
				const float g2 = Fx * Fx + Fy * Fy + Fz * Fz;
				float dt = fminf(kp.eta * sqrtf(kp.a * hh * rsqrtf(g2)), kp.t0);
				dt = fminf(kp.max_dt, dt);
				int r = a.rung[k];
				r = max(kp.min_rung + int((int) ceilf(log2f(kp.t0 / dt)) > kp.min_rung), r - 1);
				r = max(0, min(r, 15));
				a.rung[k] = (int8_t) r;
				imax = r;
				dt = 0.5f * rdt * kp.t0;
				vx = fmaf(sgn * Fx, dt, vx);
				vy = fmaf(sgn * Fy, dt, vy);
				vz = fmaf(sgn * Fz, dt, vz);
			}
			const float kin1 = (float) (0.5 * (double) (vx * vx + vy * vy + vz * vz));
			a.v[0][k] = vx;
			a.v[1][k] = vy;
			a.v[2][k] = vz;
			ia[0] = 0.5f * Fp;
			ia[2] = kin1 - kin0;
		}
		if (a.nsub > 1) {
			for (int q = 0; q < 9; q++) {
				for (int o = 16; o; o >>= 1) {
					ia[q] += __shfl_xor_sync(0xffffffffu, ia[q], o);
				}
			}
			for (int o = 16; o; o >>= 1) {
				imax = max(imax, __shfl_xor_sync(0xffffffffu, imax, o));
			}
			if (lane == 0) {
				const int lo = bx;
				for (int q = 0; q < 9; q++) {
					atomicAdd(a.sub_sums + 9 * lo + q, ia[q]);
				}
				atomicMax(a.sub_maxrung + lo, imax);
			} else {
				// every lane now holds the warp's totals: only lane 0 carries them into the
				// context-wide sums below
				for (int q = 0; q < 9; q++) {
					ia[q] = 0.0;
				}
			}
		}
		for (int q = 0; q < 9; q++) {
			acc[q] += ia[q];
		}
		maxr = max(maxr, imax);
	}
	for (int q = 0; q < 9; q++) {
		double v = acc[q];
		for (int o = 16; o; o >>= 1) {
			v += __shfl_xor_sync(0xffffffffu, v, o);
		}
		if (lane == 0) {
			s_red[w][q] = v;
		}
	}
	for (int o = 16; o; o >>= 1) {
		maxr = max(maxr, __shfl_xor_sync(0xffffffffu, maxr, o));
	}
	__syncthreads();
	if (threadIdx.x < 9) {
		double v = 0;
		for (int q = 0; q < 4; q++) {
			v += s_red[q][threadIdx.x];
		}
		atomicAdd(a.sums + threadIdx.x, v);
	}
	if (lane == 0 && maxr > 0) {
		atomicMax(a.max_rung, maxr);
	}
}

// Tiles of tw sinks of every leaf: counts, then (leaf, tile) items at the scanned offsets.
__global__ void k_tile_count(int64_t nleaves, const int64_t* leaves, const NodeW* nodes, int tw, int* ntiles) {
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < nleaves; i += (int64_t) gridDim.x * blockDim.x) {
		const NodeW nd = nodes[leaves[i]];
		ntiles[i] = (nd.pend - nd.pbeg + tw - 1) / tw;
	}
}
__global__ void k_tile_fill(int64_t nleaves, const int64_t* leaves, const int* ntiles, const int* off, int2* items) {
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < nleaves; i += (int64_t) gridDim.x * blockDim.x) {
		const int o = off[i];
		for (int t = 0; t < ntiles[i]; t++) {
			items[o + t] = make_int2((int) leaves[i], t);
		}
	}
}

__global__ void k_collect_leaves(int64_t nn, const NodeW* nodes, int64_t* leaves, unsigned long long* count) {
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < nn; i += (int64_t) gridDim.x * blockDim.x) {
		const NodeW nd = nodes[i];
		if ((nd.flags & 1) && nd.pend > nd.pbeg) {
			const unsigned long long p = atomicAdd(count, 1ull);
			leaves[p] = i;
		}
	}
}

// ---------------------------------------------------------------- host driver
}  // namespace

// Blocks of `tpb` threads of `kernel` resident on the whole GPU (its register and shared
// memory use decide; at least one per SM).
template<class K>
int resident_blocks(const Ctx* c, K kernel, int tpb, size_t dyn_smem = 0) {
	int nb = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, tpb, dyn_smem) != cudaSuccess || nb < 1) {
		cudaGetLastError();
		nb = 1;
	}
	return nb * c->nsm;
}

// One launch of the P2P kernel instance the context's tuning names (cell-list size, warps per
// tile): a resident grid, at most one block per 8 tiles.
template<bool SMALL, int STAGE, int WPT>
void launch_p2p_t(const Ctx* c, const P2PArgs& pa, int64_t ntiles, cudaStream_t st) {
	const int64_t want = (ntiles * WPT + 7) / 8;
	const int nb = (int) std::max<int64_t>(1, std::min<int64_t>(want, (int64_t) resident_blocks(c, k_p2p<SMALL, STAGE, WPT>, P2P_TPB)));
	k_p2p<SMALL, STAGE, WPT><<<nb, P2P_TPB, 0, st>>>(pa);
}
template<bool SMALL>
void launch_p2p(const Ctx* c, const P2PArgs& pa, int64_t ntiles, cudaStream_t st) {
	const int s = c->tune.p2p_stage, w = c->tune.warps_per_tile;
	if (s == 64) {
		w == 2 ? launch_p2p_t<SMALL, 64, 2>(c, pa, ntiles, st) : launch_p2p_t<SMALL, 64, 1>(c, pa, ntiles, st);
	} else if (s == 256) {
		w == 2 ? launch_p2p_t<SMALL, 256, 2>(c, pa, ntiles, st) : launch_p2p_t<SMALL, 256, 1>(c, pa, ntiles, st);
	} else {
		w == 2 ? launch_p2p_t<SMALL, 128, 2>(c, pa, ntiles, st) : launch_p2p_t<SMALL, 128, 1>(c, pa, ntiles, st);
	}
}

struct KickBuffers {
	int2* per_node = nullptr;  // 7 arrays of nnodes
	size_t per_node_n = 0;
	int* cc = nullptr;         // ecc + dcc lists
	size_t cc_n = 0;
	long long cap_cc = 0;
	int* leafl = nullptr;      // cp + pc + pp lists
	size_t leaf_n = 0;
	long long cap_leaf = 0;
	int* pass = nullptr;       // two pass-down buffers
	size_t pass_n = 0;
	long long cap_pass = 0;
	int* stage = nullptr;
	size_t stage_n = 0;
	int stage_cap = 0;
	int nwarps = 0;
	float* dL = nullptr;  // Ewald M2L sums (then L2L adds the next two)
	size_t dL_n = 0;
	float* dL2 = nullptr;  // direct M2L sums
	size_t dL2_n = 0;
	float* dL3 = nullptr;  // P2L sums
	size_t dL3_n = 0;
	float* Lx = nullptr;
	size_t Lx_n = 0;
	int64_t* leaves = nullptr;
	size_t leaves_n = 0;
};

namespace {


KickBuffers& kbuf(Ctx* c) {
	if (!c->kick) {
		c->kick = new KickBuffers();
	}
	return *c->kick;
}

template<class T>
ct_status ensure(Ctx* c, T** p, size_t& have, size_t need, const char* what) {
	if (need <= have && *p) {
		return CT_OK;
	}
	if (*p) {
		dfree(c, *p, sizeof(T) * have);
		*p = nullptr;
	}
	const size_t n = std::max(need, have * 3 / 2);
	CT_TRY(dalloc(c, (void**) p, sizeof(T) * n, what));
	have = n;
	return CT_OK;
}

template<class Ops>
ct_status kick_t(Ctx* c, Box* b, const ct_kick_params* kp, ct_kick_return* out) {
	cudaStream_t st = c->stream;
	KickBuffers& K = kbuf(c);
	const int64_t nn = b->nnodes;
	const int64_t np = b->n - b->rung_begin;
	// per-node list descriptors
	CT_TRY(ensure(c, &K.per_node, K.per_node_n, (size_t) 7 * nn, "walk descriptors"));
	CT_TRY(ensure(c, &K.dL, K.dL_n, (size_t) NEXP_STRIDE * nn, "expansion deltas"));
	CT_TRY(ensure(c, &K.dL2, K.dL2_n, (size_t) NEXP_STRIDE * nn, "expansion deltas (direct M2L)"));
	CT_TRY(ensure(c, &K.dL3, K.dL3_n, (size_t) NEXP_STRIDE * nn, "expansion deltas (P2L)"));
	CT_TRY(ensure(c, &K.Lx, K.Lx_n, (size_t) NEXP_STRIDE * nn, "local expansions"));
	CT_TRY(ensure(c, &K.leaves, K.leaves_n, (size_t) nn, "leaf index"));
	K.nwarps = c->nsm * 16 * (WALK_TPB / 32) / 4;  // 4 blocks of 4 warps per SM
	if (K.stage_cap == 0) {
		K.stage_cap = 4096;
	}
	if (K.cap_cc == 0) {
		K.cap_cc = std::max<long long>(1 << 20, 256LL * nn);
		K.cap_leaf = std::max<long long>(1 << 20, 128LL * nn);
		K.cap_pass = std::max<long long>(1 << 20, 256LL * nn);
	}
	double* counters = c->d_counters;
	for (int attempt = 0; attempt < 6; attempt++) {
		// (re)allocate list storage at the current capacities
		CT_TRY(ensure(c, &K.cc, K.cc_n, (size_t) 2 * K.cap_cc, "CC lists"));
		CT_TRY(ensure(c, &K.leafl, K.leaf_n, (size_t) 3 * K.cap_leaf, "leaf lists"));
		CT_TRY(ensure(c, &K.pass, K.pass_n, (size_t) 2 * K.cap_pass, "pass-down lists"));
		CT_TRY(ensure(c, &K.stage, K.stage_n, (size_t) K.nwarps * NLIST * K.stage_cap, "walk staging"));
		WalkOut o;
		o.ecc = K.per_node;
		o.dcc = K.per_node + nn;
		o.cp = K.per_node + 2 * nn;
		o.pc = K.per_node + 3 * nn;
		o.pp = K.per_node + 4 * nn;
		o.eout = K.per_node + 5 * nn;
		o.dout = K.per_node + 6 * nn;
		o.ecc_list = K.cc;
		o.dcc_list = K.cc + K.cap_cc;
		o.cp_list = K.leafl;
		o.pc_list = K.leafl + K.cap_leaf;
		o.pp_list = K.leafl + 2 * K.cap_leaf;
		o.cap_cc = K.cap_cc;
		o.cap_leaf = K.cap_leaf;
		o.cap_pass = K.cap_pass;  // buffers hold at least 2x / 3x these
		o.stage = K.stage;
		o.stage_cap = K.stage_cap;
		o.flags = c->d_flags;
		o.cursor = (unsigned long long*) (c->d_flags + 16);
		CT_CUDA(c, cudaMemsetAsync(c->d_flags, 0, 64 * sizeof(int), st));
		WalkParams wp;
		wp.thetainv = 1.f / kp->theta;
		wp.h = kp->h;
		wp.nroot = b->nsub;
		wp.sub_off = b->d_sub_off;
		wp.sub_h = b->d_sub_h;
		cudaEventRecord(c->ev[0], st);
		const int nlev = (int) b->level_start.size() - 1;
		for (int k = 0; k < nlev; k++) {
			const int64_t lb = b->level_start[k], le = b->level_start[k + 1];
			o.pass_cur = K.pass + (k & 1) * K.cap_pass;
			o.pass_prev = K.pass + ((k + 1) & 1) * K.cap_pass;
			// pass-down cursor restarts every level (its buffer alternates)
			CT_CUDA(c, cudaMemsetAsync(o.cursor + 5, 0, sizeof(unsigned long long), st));
			const int64_t nwn = std::min<int64_t>((le - lb + 3) / 4, (int64_t) K.nwarps / 4);
			c->launches++;
			k_walk<<<(int) std::max<int64_t>(nwn, 1), WALK_TPB, 0, st>>>(lb, le, b->nodes, b->nbox, b->parent, o, wp);
		}
		CT_CUDA(c, cudaGetLastError());
		cudaEventRecord(c->ev[1], st);
		int* hf = (int*) c->pinned;
		CT_CUDA(c, cudaMemcpyAsync(hf, c->d_flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
		CT_CUDA(c, cudaStreamSynchronize(st));
		if (hf[1]) {
			return fail(c, CT_ERR_STATE, "an Ewald check failed the opening test against a leaf; the tree was built with a different theta");
		}
		if (hf[0]) {
			// overflow: grow everything and retry
			K.stage_cap *= 2;
			K.cap_cc *= 2;
			K.cap_leaf *= 2;
			K.cap_pass *= 2;
			continue;
		}
		// ---- interactions
		CT_CUDA(c, cudaMemsetAsync(counters, 0, 16 * sizeof(double), st));
		// node orders of the three node-indexed kernels, longest lists first (radix sort of the
		// list lengths' bit lengths; nodes without a list of a kind sort last)
		ct_status s3 = CT_OK;
		uint32_t* okey = (uint32_t*) scratch(c, 46, sizeof(uint32_t) * 6 * nn, &s3);
		int32_t* oidx = (int32_t*) scratch(c, 47, sizeof(int32_t) * 4 * nn, &s3);
		unsigned long long* onext = (unsigned long long*) scratch(c, 48, 3 * sizeof(unsigned long long), &s3);
		CT_TRY(s3);
		size_t sort_bytes = 0;
		CT_CUDA(c, cub::DeviceRadixSort::SortPairsDescending(nullptr, sort_bytes, okey, okey + 3 * nn, oidx, oidx + nn, (int) nn, 0, ORDER_KEY_BITS, st));
		void* sort_tmp = scratch(c, 49, sort_bytes + 256, &s3);
		CT_TRY(s3);
		c->launches++;
		k_order_keys<<<(int) std::max<int64_t>(1, std::min<int64_t>((nn + 255) / 256, c->nsm * 8)), 256, 0, st>>>(nn, b->nodes, o.ecc, o.dcc, o.cp, okey,
				oidx);
		for (int k = 0; k < 3; k++) {
			size_t tb = sort_bytes;
			CT_CUDA(c, cub::DeviceRadixSort::SortPairsDescending(sort_tmp, tb, okey + k * nn, okey + (3 + k) * nn, oidx, oidx + (1 + k) * nn, (int) nn, 0,
					ORDER_KEY_BITS, st));
		}
		CT_CUDA(c, cudaMemsetAsync(onext, 0, 3 * sizeof(unsigned long long), st));
		const size_t dl_bytes = sizeof(float) * NEXP_STRIDE * nn;
		CT_CUDA(c, cudaMemsetAsync(K.dL, 0, dl_bytes, st));
		// The three kernels run side by side on three streams, each into its own expansion
		// deltas; L2L adds them in this order, dL + dL2 + dL3, the order of one stream.  Each is
		// a resident grid (blocks per SM from the occupancy query) whose warps take nodes from
		// the kind's order.
		CT_CUDA(c, cudaEventRecord(c->fork_ev, st));
		for (int k = 0; k < 2; k++) {
			CT_CUDA(c, cudaStreamWaitEvent(c->side[k], c->fork_ev, 0));
		}
		c->launches++;
		k_m2l_ewald<Ops><<<resident_blocks(c, k_m2l_ewald<Ops>, 128), 128, 0, st>>>(nn, oidx + nn, onext, b->nodes, b->multi, o.ecc, o.ecc_list, K.dL,
				kp->do_phi, counters);
		CT_CUDA(c, cudaMemsetAsync(K.dL2, 0, dl_bytes, c->side[0]));
		c->launches++;
		CT_CUDA(c, cudaFuncSetAttribute(k_m2l_direct<Ops>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) M2L_DIRECT_SMEM));
		k_m2l_direct<Ops><<<resident_blocks(c, k_m2l_direct<Ops>, 128, M2L_DIRECT_SMEM), 128, M2L_DIRECT_SMEM, c->side[0]>>>(nn, oidx + 2 * nn, onext + 1,
				b->nodes, b->multi, o.dcc, o.dcc_list, K.dL2, kp->do_phi);
		CT_CUDA(c, cudaMemsetAsync(K.dL3, 0, dl_bytes, c->side[1]));
		c->launches++;
		k_p2l<Ops><<<resident_blocks(c, k_p2l<Ops>, 128), 128, 0, c->side[1]>>>(nn, oidx + 3 * nn, onext + 2, b->nodes, o.cp, o.cp_list, b->x[0], b->x[1],
				b->x[2], K.dL3, counters);
		for (int k = 0; k < 2; k++) {
			CT_CUDA(c, cudaEventRecord(c->join_ev[k], c->side[k]));
			CT_CUDA(c, cudaStreamWaitEvent(st, c->join_ev[k], 0));
		}
		cudaEventRecord(c->ev[2], st);
		for (int k = 0; k < nlev; k++) {
			const int64_t lb = b->level_start[k], le = b->level_start[k + 1];
			const int64_t g = (le - lb + 127) / 128;
			c->launches++;
			k_l2l<Ops><<<(int) std::max<int64_t>(1, std::min<int64_t>(g, c->nsm * 16)), 128, 0, st>>>(lb, le, b->nodes, b->parent, K.dL, K.dL2, K.dL3,
					K.Lx, kp->do_phi);
		}
		cudaEventRecord(c->ev[3], st);
		// leaves
		unsigned long long* lcount = (unsigned long long*) (c->d_flags + 40);
		CT_CUDA(c, cudaMemsetAsync(lcount, 0, sizeof(unsigned long long), st));
		c->launches++;
		k_collect_leaves<<<(int) std::max<int64_t>(1, std::min<int64_t>((nn + 255) / 256, c->nsm * 8)), 256, 0, st>>>(nn, b->nodes, K.leaves, lcount);
		CT_CUDA(c, cudaMemcpyAsync(hf, lcount, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
		CT_CUDA(c, cudaStreamSynchronize(st));
		const int64_t nleaves = (int64_t) * (unsigned long long*) hf;
		cudaEventRecord(c->ev[4], st);
		cudaEventRecord(c->ev[5], st);
		cudaEventRecord(c->ev[12], st);  // no leaves: zero P2P and leaf-kick times
		if (nleaves > 0) {
			// 32-sink tiles of the leaves
			ct_status s2 = CT_OK;
			int* ntl = (int*) scratch(c, 40, sizeof(int) * (nleaves + 1), &s2);
			int* off = (int*) scratch(c, 41, sizeof(int) * (nleaves + 1), &s2);
			CT_TRY(s2);
			size_t need = 0;
			cub::DeviceScan::ExclusiveSum(nullptr, need, ntl, off, (int) nleaves + 1, st);
			void* tmp = scratch(c, 42, need + 256, &s2);
			CT_TRY(s2);
			c->launches++;
			const int tw = c->tune.tile_width;
			k_tile_count<<<(int) std::max<int64_t>(1, std::min<int64_t>((nleaves + 255) / 256, c->nsm * 8)), 256, 0, st>>>(nleaves, K.leaves, b->nodes, tw,
					ntl);
			CT_CUDA(c, cudaMemsetAsync(ntl + nleaves, 0, sizeof(int), st));
			CT_CUDA(c, cub::DeviceScan::ExclusiveSum(tmp, need, ntl, off, (int) nleaves + 1, st));
			CT_CUDA(c, cudaMemcpyAsync(hf, off + nleaves, sizeof(int), cudaMemcpyDeviceToHost, st));
			CT_CUDA(c, cudaStreamSynchronize(st));
			const int64_t nitems = hf[0];
			int2* items = (int2*) scratch(c, 43, sizeof(int2) * (nitems + 1), &s2);
			float4* F = (float4*) scratch(c, 44, sizeof(float4) * b->n, &s2);
			CT_TRY(s2);
			c->launches++;
			k_tile_fill<<<(int) std::max<int64_t>(1, std::min<int64_t>((nleaves + 255) / 256, c->nsm * 8)), 256, 0, st>>>(nleaves, K.leaves, ntl, off, items);
			P2PArgs pa;
			pa.nsub = b->nsub;
			pa.sub_off = b->d_sub_off;
			pa.sub_h = b->d_sub_h;
			pa.nodes = b->nodes;
			pa.nbox = b->nbox;
			pa.items = items;
			pa.nitems = nitems;
			pa.pp = o.pp;
			pa.pp_list = o.pp_list;
			for (int d = 0; d < 3; d++) {
				pa.x[d] = b->x[d];
			}
			pa.F = F;
			pa.h = kp->h;
			pa.compensated = c->compensated;
			pa.pairs = counters + 4 + 7;
			pa.near_pairs = counters + 13;
			pa.tw = tw;
			// full tiles and tiles of at most 16 sinks go to separate launches
			int2* tiles2 = (int2*) scratch(c, 45, sizeof(int2) * 2 * (nitems + 1), &s2);
			CT_TRY(s2);
			unsigned long long* tcount = (unsigned long long*) (c->d_flags + 44);
			CT_CUDA(c, cudaMemsetAsync(tcount, 0, 2 * sizeof(unsigned long long), st));
			unsigned long long* wnext = (unsigned long long*) (c->d_flags + 52);  // work counters of the two launches
			CT_CUDA(c, cudaMemsetAsync(wnext, 0, 2 * sizeof(unsigned long long), st));

			c->launches++;
			k_split_tiles<<<(int) std::max<int64_t>(1, std::min<int64_t>((nitems + 255) / 256, c->nsm * 8)), 256, 0, st>>>(items, nitems, b->nodes, tw,
					tiles2, tiles2 + nitems + 1, tcount);
			CT_CUDA(c, cudaMemcpyAsync(hf, tcount, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
			CT_CUDA(c, cudaStreamSynchronize(st));
			const int64_t nbig = (int64_t) ((unsigned long long*) hf)[0], nsmall = (int64_t) ((unsigned long long*) hf)[1];
			cudaEventRecord(c->ev[4], st);
			if (nbig > 0) {
				pa.items = tiles2;
				pa.nitems = nbig;
				pa.next = wnext;
				c->launches++;
				launch_p2p<false>(c, pa, nbig, st);
			}
			if (nsmall > 0) {
				pa.items = tiles2 + nitems + 1;
				pa.nitems = nsmall;
				pa.next = wnext + 1;
				c->launches++;
				launch_p2p<true>(c, pa, nsmall, st);
			}
			cudaEventRecord(c->ev[5], st);
			KickTileArgs ka;
			ka.nsub = b->nsub;
			ka.sub_off = b->d_sub_off;
			ka.sub_sums = b->d_sub_sums;
			ka.sub_maxrung = b->d_sub_maxrung;
			ka.sub_h = b->d_sub_h;
			ka.sub_GM = b->d_sub_GM;
			ka.sub_first = b->d_sub_first;
			if (b->nsub > 1) {
				CT_CUDA(c, cudaMemsetAsync(b->d_sub_sums, 0, sizeof(double) * 9 * b->nsub, st));
				CT_CUDA(c, cudaMemsetAsync(b->d_sub_maxrung, 0, sizeof(int) * b->nsub, st));
			}
			ka.nodes = b->nodes;
			ka.multi = b->multi;
			ka.Lx = K.Lx;
			ka.items = items;
			ka.nitems = nitems;
			ka.pc = o.pc;
			ka.pc_list = o.pc_list;
			ka.F = F;
			for (int d = 0; d < 3; d++) {
				ka.x[d] = b->x[d];
				ka.v[d] = b->v[d];
				ka.g[d] = b->g[d];
			}
			ka.rung = b->rung;
			ka.pot = b->pot;
			ka.kp = *kp;
			ka.sums = counters + 4;
			ka.max_rung = c->d_flags + 48;
			ka.next = (unsigned long long*) (c->d_flags + 62);
			ka.tw = tw;
			CT_CUDA(c, cudaMemsetAsync(ka.next, 0, sizeof(unsigned long long), st));
			c->launches++;
			k_leaf_kick<Ops><<<(int) std::max<int64_t>(1, std::min<int64_t>((nitems + 3) / 4, (int64_t) resident_blocks(c, k_leaf_kick<Ops>, 128))), 128, 0,
					st>>>(ka);
			cudaEventRecord(c->ev[12], st);
		}
		CT_CUDA(c, cudaGetLastError());
		double* hd = (double*) c->pinned;
		CT_CUDA(c, cudaMemcpyAsync(hd, counters, 16 * sizeof(double), cudaMemcpyDeviceToHost, st));
		CT_CUDA(c, cudaMemcpyAsync(hd + 16, c->d_flags + 48, sizeof(int), cudaMemcpyDeviceToHost, st));
		unsigned long long* hcur = (unsigned long long*) (hd + 20);
		CT_CUDA(c, cudaMemcpyAsync(hcur, o.cursor, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
		CT_CUDA(c, cudaStreamSynchronize(st));
		ct_kick_return r;
		r.pot = hd[4];
		r.kin = hd[5];
		r.dkin = hd[6];
		r.xmom = hd[7];
		r.ymom = hd[8];
		r.zmom = hd[9];
		r.nmom = hd[10];
		r.max_rung = *(int*) (hd + 16);
		if (out) {
			*out = r;
		}
		ct_counters& C = b->counters;
		C.cc_ewald = (double) hcur[0];
		C.cc_direct = (double) hcur[1];
		C.pc_pairs = hd[12];
		C.pp_pairs = hd[11];
		C.pp_near = hd[13];
		C.cp_pairs = hd[1];
		C.nodes = (double) nn;
		C.leaves = (double) nleaves;
		const double icnt = hd[0];
		const bool phi = kp->do_phi != 0;
		C.flops_pp = FLOP_PP * C.pp_pairs;
		// the reference's per-interaction counts (fmm_kernels.hpp:315,724,1486; gravity.cu:62,140,197,343;
		// kick.cu:153,257)
		C.flops_cc = C.cc_direct * (6 + FLOP_GREENS + FLOP_M2L + phi * FLOP_M2L_PHI) +
				C.cc_ewald * (3 + 7 + 140 * 92 + 540 + FLOP_M2L + phi * FLOP_M2L_PHI) + 843.0 * icnt;
		C.flops = C.flops_pp + C.flops_cc + C.cp_pairs * (Ops::NEXP + 6 + FLOP_GREENS) + C.pc_pairs * (6 + FLOP_GREENS + FLOP_M2L2 + phi * FLOP_M2L_PHI + 4)
				+ (double) nn * (FLOP_L2L + phi * FLOP_L2L_PHI) + (double) np * (FLOP_KICK + phi * FLOP_KICK_PHI);
		C.ms_walk = elapsed_ms(c->ev[0], c->ev[1]);
		C.ms_m2l = elapsed_ms(c->ev[1], c->ev[2]);
		C.ms_l2l = elapsed_ms(c->ev[2], c->ev[3]);
		C.ms_leaf = elapsed_ms(c->ev[4], c->ev[5]);  // the P2P kernels
		if (nleaves > 0) {
			C.ms_leafkick = elapsed_ms(c->ev[5], c->ev[12]);
		}
		b->have_force = kp->save_force != 0;
		return CT_OK;
	}
	return fail(c, CT_ERR_CAPACITY, "interaction lists overflowed after repeated regrowth");
}

}  // namespace

// The tables live in __constant__ memory, one copy per device shared by every context on it:
// they are written once per device and order (the first context created there), so that a
// context created later never rewrites them while another context's kernels read them, and
// the host-side index table is built once per process.
template<class Tab, class Build, class Four>
ct_status ewald_init_order(Ctx* c, const Tab& sym, int which, Build build, Four four) {
	static std::mutex m;
	static bool written[64][2] = {};
	static Tab h;
	static std::once_flag h_once;
	std::call_once(h_once, [&] { build(h); });
	int dev = 0;
	CT_CUDA(c, cudaGetDevice(&dev));
	std::lock_guard<std::mutex> lock(m);
	if (dev >= 0 && dev < 64 && written[dev][which]) {
		return CT_OK;
	}
	cudaStream_t st = c->stream;
	Tab* d = nullptr;
	CT_TRY(dalloc(c, (void**) &d, sizeof(h), "Ewald tables"));
	CT_CUDA(c, cudaMemcpyAsync(d, &h, sizeof(h), cudaMemcpyHostToDevice, st));
	c->launches++;
	four<<<1, 128, 0, st>>>(d);
	CT_CUDA(c, cudaMemcpyToSymbolAsync(sym, d, sizeof(h), 0, cudaMemcpyDeviceToDevice, st));
	CT_CUDA(c, cudaStreamSynchronize(st));
	dfree(c, d, sizeof(h));
	if (dev >= 0 && dev < 64) {
		written[dev][which] = true;
	}
	return CT_OK;
}

ct_status ewald_init(Ctx* c) {
	if (c->order == 5) {
		return ewald_init_order(c, c_tab5, 0, [](ct_p5::EwaldTab& t) { ct_p5::ewald_build_indices(t); }, k_ewald_four5);
	}
	return ewald_init_order(c, c_tab7, 1, [](ct_p7::EwaldTab& t) { ct_p7::ewald_build_indices(t); }, k_ewald_four7);
}

void kick_buffers_release(Ctx* c) {
	KickBuffers* K = c->kick;
	if (!K) {
		return;
	}
	dfree(c, K->per_node, sizeof(int2) * K->per_node_n);
	dfree(c, K->cc, sizeof(int) * K->cc_n);
	dfree(c, K->leafl, sizeof(int) * K->leaf_n);
	dfree(c, K->pass, sizeof(int) * K->pass_n);
	dfree(c, K->stage, sizeof(int) * K->stage_n);
	dfree(c, K->dL, sizeof(float) * K->dL_n);
	dfree(c, K->dL2, sizeof(float) * K->dL2_n);
	dfree(c, K->dL3, sizeof(float) * K->dL3_n);
	dfree(c, K->Lx, sizeof(float) * K->Lx_n);
	dfree(c, K->leaves, sizeof(int64_t) * K->leaves_n);
	delete K;
	c->kick = nullptr;
}

ct_status kick_run(Ctx* c, Box* b, const ct_kick_params* p, ct_kick_return* out) {
	if (c->order == 5) {
		return kick_t<Ops5>(c, b, p, out);
	}
	return kick_t<Ops7>(c, b, p, out);
}

}  // namespace ct
