// Test infrastructure only (oracle build; never part of the library).
//
// The reference's CPU top of the kick and the GPU work items it hands over: kick()
// (src/kick.cpp:150-507, with its multipole interactions of src/gravity.cpp) over a tree built
// by the reference's tree_create (src/tree.cpp), compiled where they lie against the
// single-threaded HPX stand-in.  Every node holding at most max_parts particles goes to the
// GPU workspace as a work item (kick.cpp:170-189); the workspace here is a stand-in that records
// the items -- subtree root, incoming expansion, its centre, direct and Ewald check lists -- in
// place of copying them to the device (kick_workspace.cpp:68-327), and releases the root's
// return once all particles are covered, as the device kick's completion does (kick_set_rc).
//
//   kick_probe <in> <out> <theta> <hsoft> <bucket> <blocks>
//
// in: int64 n, uint32 x[n], y[n], z[n].  blocks: the device's kick block count (kick.cu's
// kick_block_count), which sets max_parts = min(CUDA_KICK_PARTS_MAX, max(n / blocks, bucket)).
// out: int64 nnodes, ct_or_node[nnodes] (the tree, depth first, left child first), the
// positions after the build (uint32 x[n], y[n], z[n]), int64 max_parts, int64 nitems, then per
// item in the workspace's order (first particle, kick_workspace.cpp:308-310): int32 self,
// float L[EXPANSION_SIZE], uint32 pos[3], int32 nd, int32 dlist[nd], int32 ne, int32 elist[ne]
// (nodes as indices of the depth-first list).
#include "ref_ewald_host.h"
#include "ref_host.h"

#include <cosmictiger/kick.hpp>
#include <cosmictiger/kick_workspace.hpp>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>

static int g_blocks = 1;
int kick_block_count() {
	return g_blocks;
}

// ---------------------------------------------------------------- recording workspace
static std::vector<kick_workitem> g_items;
static part_int g_total = 0, g_covered = 0;
static bool g_released = false;

static void covered(part_int n) {
	g_covered += n;
	if (g_covered == g_total && !g_released) {
		g_released = true;
		kick_set_rc(kick_return());
	}
}
kick_workspace::kick_workspace(kick_params p, part_int n) {
	params = p;
	total_parts = n;
	nparts = 0;
	g_total = n;
	g_covered = 0;
	g_released = false;
	g_items.clear();
}
kick_workspace::~kick_workspace() {
}
void kick_workspace::clear_buffers() {
}
void kick_workspace::add_work(std::shared_ptr<kick_workspace>, expansion<float> L, array<fixed32, NDIM> pos, tree_id self, vector<tree_id>&& dchecklist,
		vector<tree_id>&& echecklist) {
	kick_workitem w;
	w.L = L;
	w.pos = pos;
	w.self = self;
	w.dchecklist = std::move(dchecklist);
	w.echecklist = std::move(echecklist);
	g_items.push_back(std::move(w));
	covered(tree_get_node(self)->nparts());
}
void kick_workspace::add_parts(std::shared_ptr<kick_workspace>, part_int n) {
	covered(n);
}
void kick_workspace::to_gpu() {
}

// ---------------------------------------------------------------- node numbering
static void number_nodes(tree_id id, std::unordered_map<int, int>& dfs, int& next) {
	dfs[id.index] = next++;
	const tree_node* nd = tree_get_node(id);
	if (!nd->leaf) {
		number_nodes(nd->children[LEFT], dfs, next);
		number_nodes(nd->children[RIGHT], dfs, next);
	}
}

int main(int argc, char** argv) {
	if (argc != 7) {
		fprintf(stderr, "usage: kick_probe <in> <out> <theta> <hsoft> <bucket> <blocks>\n");
		return 2;
	}
	ref_set_defaults();
	const double theta = atof(argv[3]);
	g_opts.hsoft = atof(argv[4]);
	g_opts.bucket_size = atoi(argv[5]);
	g_blocks = atoi(argv[6]);
	g_opts.theta = theta;
	g_opts.cuda = true;
	FILE* f = fopen(argv[1], "rb");
	int64_t n = 0;
	if (!f || fread(&n, sizeof(n), 1, f) != 1 || n <= 0) {
		fprintf(stderr, "kick_probe: cannot read %s\n", argv[1]);
		return 1;
	}
	std::vector<uint32_t> X[NDIM];
	for (int d = 0; d < NDIM; d++) {
		X[d].resize(n);
		if (fread(X[d].data(), sizeof(uint32_t), n, f) != (size_t) n) {
			return 1;
		}
	}
	fclose(f);
	g_opts.nparts = n;
	particles_resize(n);
	for (part_int i = 0; i < n; i++) {
		for (int d = 0; d < NDIM; d++) {
			particles_pos(d, i).raw() = X[d][i];
			particles_vel(d, i) = 0.f;
		}
		particles_rung(i) = 0;
	}
	particles_sort_by_rung(0);
	tree_create_params tp(0, theta, g_opts.hsoft);
	const tree_create_return trc = tree_create(tp);
	std::vector<ct_or_node> nodes;
	ref_emit_tree(trc.id, 1, 0, nodes);
	std::unordered_map<int, int> dfs;
	int next = 0;
	number_nodes(trc.id, dfs, next);
	// the driver's first call of a step (driver.cpp:490-528): zero expansion at the origin, the
	// root as both check lists, all particles active
	kick_params kp;
	kp.gpu = true;
	kp.min_rung = 0;
	kp.min_level = tp.min_level;
	kp.theta = theta;
	kp.h = g_opts.hsoft;
	kp.GM = 1.0f / n;
	kp.eta = 0.2f;
	kp.a = 1.0f;
	kp.t0 = 1.0f;
	kp.first_call = true;
	kp.save_force = false;
	kp.ascending = kp.descending = kp.top = true;
	kp.do_phi = true;
	kp.node_load = 0.f;
	expansion<float> L;
	for (int i = 0; i < EXPANSION_SIZE; i++) {
		L[i] = 0.0f;
	}
	array<fixed32, NDIM> pos;
	for (int d = 0; d < NDIM; d++) {
		pos[d] = 0.f;
	}
	vector<tree_id> checklist(1, trc.id);
	kick(kp, L, pos, trc.id, checklist, checklist, nullptr);
	std::stable_sort(g_items.begin(), g_items.end(), [](const kick_workitem& a, const kick_workitem& b) {
		return tree_get_node(a.self)->part_range.first < tree_get_node(b.self)->part_range.first;
	});
	const auto rng = particles_current_range();
	const int64_t max_parts = std::min((int64_t) CUDA_KICK_PARTS_MAX, (int64_t) std::max((int64_t) (rng.second - rng.first) / g_blocks,
			(int64_t) g_opts.bucket_size));
	FILE* g = fopen(argv[2], "wb");
	if (!g) {
		return 1;
	}
	const int64_t cnt = nodes.size();
	fwrite(&cnt, sizeof(cnt), 1, g);
	fwrite(nodes.data(), sizeof(ct_or_node), nodes.size(), g);
	for (int d = 0; d < NDIM; d++) {
		for (part_int i = 0; i < n; i++) {
			X[d][i] = particles_pos(d, i).raw();
		}
		fwrite(X[d].data(), sizeof(uint32_t), n, g);
	}
	fwrite(&max_parts, sizeof(max_parts), 1, g);
	const int64_t nitems = g_items.size();
	fwrite(&nitems, sizeof(nitems), 1, g);
	for (const auto& w : g_items) {
		const int32_t self = dfs.at(w.self.index);
		fwrite(&self, sizeof(self), 1, g);
		for (int i = 0; i < EXPANSION_SIZE; i++) {
			const float l = w.L[i];
			fwrite(&l, sizeof(l), 1, g);
		}
		for (int d = 0; d < NDIM; d++) {
			const uint32_t p = w.pos[d].raw();
			fwrite(&p, sizeof(p), 1, g);
		}
		for (const auto* list : { &w.dchecklist, &w.echecklist }) {
			const int32_t m = list->size();
			fwrite(&m, sizeof(m), 1, g);
			for (const auto& id : *list) {
				const int32_t k = dfs.at(id.index);
				fwrite(&k, sizeof(k), 1, g);
			}
		}
	}
	if (fclose(g) != 0) {
		return 1;
	}
	return g_released ? 0 : 4;
}
