// Test infrastructure only (oracle build; never part of the library).
//
// Runs the reference's own hierarchical step, kick_step_hierarchical (src/driver.cpp:382-593),
// compiled where it lies, with its own tree build and rung partition (src/tree.cpp,
// src/particles.cpp), for several steps on particles read from a file.  The two calls of the
// ladder that need a GPU in the reference are served by this project's CPU restatement
// (oracle/libct_oracle.so): kick() by ct_or_kick over the oracle's tree of the same particles
// (checked node by node against the reference's), drift() by ct_or_drift -- both pinned
// against the reference's CUDA kernels elsewhere (tests/test_reference_kick.py).  What this probe checks is the ladder itself: the
// levels, pushes and pops of the active range, the kick flags (ascending, descending, top,
// first call, the clipped top), the drifts per rung and the rung sorts, as the reference's
// code runs them.  One locality: domains_begin / domains_end move no particle (every particle
// is inside the single domain, src/domain.cpp:337-390) and are empty here; the universe is
// static (cosmos_ainv returns 1 / a: no expansion, a = 1 throughout).
//
//   ladder_probe <in> <out> <steps> <theta> <hsoft> <bucket> <GM> <eta> <t0>
//   in:  int64 n, then n x, n y, n z (uint32), n x 3 velocities (float), n rungs (int8)
//   out: per step: int32 minrung, int32 max_rung, int64 active-range start, then n x, n y, n z,
//        n x 3 velocities and n rungs after the step
#include "ref_host.h"

#include <cosmictiger/domain.hpp>
#include <cosmictiger/drift.hpp>
#include <cosmictiger/kick.hpp>

#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <utility>

std::pair<kick_return, tree_create_return> kick_step_hierarchical(int& minrung, int max_rung, double scale, double adot, double tau, double t0, double theta,
		energies_t* energies, int minrung0, bool do_phi, hpx::future<void>* lc_fut, bool nocrop, double drag);

// ---------------------------------------------------------------- services of the ladder
void domains_begin(int) {
}
void domains_end() {
}
double cosmos_ainv(double&, double& a, double) {
	return 1.0 / a;
}
void reset_gravity_counters() {
}
void set_gravity_counter_use(bool) {
}
void hpx_yield() {
}

static std::vector<ct_or_node> g_ref, g_nodes;

// The kick runs over the oracle's tree of the active particles: the same nodes as the
// reference's tree just built (checked field by field here; the particles, already in the
// reference's tree order, do not move) with the oracle's own multipoles, whose float
// rounding differs from the reference's vectorised P2M/M2M by about 1e-7 -- enough to move
// kicked velocities by an ulp.  The kick being compared elsewhere, the ladder here is run on
// the oracle's kick over the oracle's multipoles, as oracle_lib.step_hierarchical runs it.
kick_return kick(kick_params p, expansion<float>, array<fixed32, NDIM>, tree_id self, vector<tree_id>, vector<tree_id>, std::shared_ptr<kick_workspace>) {
	g_ref.clear();
	ref_emit_tree(self, 1, 0, g_ref);
	const part_int n = particles_size();
	const part_int rb = particles_current_range().first;
	uint32_t* px = (uint32_t*) &particles_pos(XDIM, 0);
	uint32_t* py = (uint32_t*) &particles_pos(YDIM, 0);
	uint32_t* pz = (uint32_t*) &particles_pos(ZDIM, 0);
	const std::vector<uint32_t> before(px, px + n);
	g_nodes.assign(g_ref.size() + 1024, ct_or_node());
	const int cnt = ct_or_tree_build(7, (int) n, (int) rb, px, py, pz, (float*) particles_vel_data(), (int8_t*) &particles_rung(0), g_opts.theta, g_opts.hsoft,
			g_opts.bucket_size, g_nodes.data(), (int) g_nodes.size(), 0);
	bool same = cnt == (int) g_ref.size() && std::equal(before.begin(), before.end(), px);
	for (int i = 0; same && i < cnt; i++) {
		const ct_or_node& a = g_nodes[i];
		const ct_or_node& b = g_ref[i];
		same = a.key == b.key && a.part_begin == b.part_begin && a.part_end == b.part_end && a.child_left == b.child_left && a.child_right == b.child_right &&
				a.leaf == b.leaf && a.depth == b.depth && !memcmp(a.pos, b.pos, sizeof(a.pos)) && !memcmp(&a.radius, &b.radius, sizeof(a.radius)) &&
				!memcmp(a.box_begin, b.box_begin, sizeof(a.box_begin)) && !memcmp(a.box_end, b.box_end, sizeof(a.box_end));
	}
	if (!same) {
		fprintf(stderr, "ladder_probe: the oracle's tree differs from the reference's (%d against %d nodes)\n", cnt, (int) g_ref.size());
		exit(4);
	}
	g_nodes.resize(cnt);
	ct_or_kick_params q;
	q.sign = p.sign;
	q.min_rung = p.min_rung;
	q.a = p.a;
	q.t0 = p.t0;
	q.theta = p.theta;
	q.h = p.h;
	q.eta = p.eta;
	q.GM = p.GM;
	q.max_dt = p.max_dt;
	q.save_force = 0;
	q.first_call = p.first_call;
	q.ascending = p.ascending;
	q.descending = p.descending;
	q.top = p.top;
	q.do_phi = p.do_phi;
	ct_or_kick_return r;
	double flops = 0.0;
	const int rc = ct_or_kick(7, &q, (int) g_nodes.size(), g_nodes.data(), (const uint32_t*) &particles_pos(XDIM, 0), (const uint32_t*) &particles_pos(YDIM, 0),
			(const uint32_t*) &particles_pos(ZDIM, 0), (float*) particles_vel_data(), (int8_t*) &particles_rung(0), nullptr, nullptr, nullptr, nullptr, &r, 0,
			&flops);
	if (rc != 0) {
		fprintf(stderr, "ladder_probe: the oracle's kick failed (%d)\n", rc);
		exit(1);
	}
	kick_return kr;
	kr.max_rung = r.max_rung;
	kr.pot = r.pot;
	kr.kin = r.kin;
	kr.dkin = r.dkin;
	kr.xmom = r.xmom;
	kr.ymom = r.ymom;
	kr.zmom = r.zmom;
	kr.nmom = r.nmom;
	return kr;
}

// the reference's drift moves the particles of rung `rung` in the active range by
// cuda_drift(rung, scale, dt, ...) (src/drift.cpp:33-37, src/drift.cu:155-195), whose drag is
// that of glass creation (off here)
void drift(double scale, double dt, double, double, double, int rung, double) {
	const part_int n = particles_size();
	const part_int b = particles_current_range().first;
	ct_or_drift((int) (n - b), (uint32_t*) &particles_pos(XDIM, b), (uint32_t*) &particles_pos(YDIM, b), (uint32_t*) &particles_pos(ZDIM, b),
			(float*) (particles_vel_data() + b), (const int8_t*) &particles_rung(b), rung, (float) scale, (float) dt, 0.0);
}

int main(int argc, char** argv) {
	if (argc != 10) {
		fprintf(stderr, "usage: ladder_probe <in> <out> <steps> <theta> <hsoft> <bucket> <GM> <eta> <t0>\n");
		return 2;
	}
	const int steps = atoi(argv[3]);
	const double theta = atof(argv[4]);
	ref_set_defaults();
	g_opts.hsoft = atof(argv[5]);
	g_opts.bucket_size = atoi(argv[6]);
	g_opts.GM = atof(argv[7]);
	g_opts.eta = atof(argv[8]);
	const double t0 = atof(argv[9]);
	g_opts.theta = theta;
	g_opts.create_glass = false;
	g_opts.plummer = false;
	g_opts.do_lc = false;
	g_opts.nsteps = 64;
	FILE* f = fopen(argv[1], "rb");
	int64_t n = 0;
	if (!f || fread(&n, sizeof(n), 1, f) != 1 || n <= 0) {
		fprintf(stderr, "ladder_probe: cannot read %s\n", argv[1]);
		return 1;
	}
	std::vector<uint32_t> X[NDIM];
	std::vector<float> V(3 * n);
	std::vector<int8_t> R(n);
	bool ok = true;
	for (int d = 0; d < NDIM; d++) {
		X[d].resize(n);
		ok = ok && fread(X[d].data(), sizeof(uint32_t), n, f) == (size_t) n;
	}
	ok = ok && fread(V.data(), sizeof(float), 3 * n, f) == (size_t) (3 * n) && fread(R.data(), 1, n, f) == (size_t) n;
	fclose(f);
	if (!ok) {
		fprintf(stderr, "ladder_probe: short read\n");
		return 1;
	}
	g_opts.nparts = n;
	particles_resize(n);
	for (part_int i = 0; i < n; i++) {
		for (int d = 0; d < NDIM; d++) {
			particles_pos(d, i).raw() = X[d][i];
			particles_vel(d, i) = V[3 * i + d];
		}
		particles_rung(i) = R[i];
	}
	particles_sort_by_rung(0);
	FILE* g = fopen(argv[2], "wb");
	if (!g) {
		fprintf(stderr, "ladder_probe: cannot write %s\n", argv[2]);
		return 1;
	}
	int minrung = 0, max_rung = 0;
	double tau = 0.0;
	for (int s = 0; s < steps; s++) {
		energies_t energies;
		const auto res = kick_step_hierarchical(minrung, max_rung, 1.0, 0.0, tau, t0, theta, &energies, 0, true, nullptr, false, 0.0);
		max_rung = res.first.max_rung;
		tau += t0;
		const int32_t head[2] = { minrung, max_rung };
		const int64_t rb = particles_current_range().first;
		ok = fwrite(head, sizeof(head), 1, g) == 1 && fwrite(&rb, sizeof(rb), 1, g) == 1;
		for (int d = 0; d < NDIM && ok; d++) {
			for (part_int i = 0; i < n; i++) {
				X[d][i] = particles_pos(d, i).raw();
			}
			ok = fwrite(X[d].data(), sizeof(uint32_t), n, g) == (size_t) n;
		}
		for (part_int i = 0; i < n && ok; i++) {
			for (int d = 0; d < NDIM; d++) {
				V[3 * i + d] = particles_vel(d, i);
			}
			R[i] = particles_rung(i);
		}
		ok = ok && fwrite(V.data(), sizeof(float), 3 * n, g) == (size_t) (3 * n) && fwrite(R.data(), 1, n, g) == (size_t) n;
		if (!ok) {
			fprintf(stderr, "ladder_probe: cannot write %s\n", argv[2]);
			return 1;
		}
	}
	return fclose(g) == 0 ? 0 : 1;
}
