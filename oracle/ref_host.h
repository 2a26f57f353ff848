// Test infrastructure only (oracle build).  Shared pieces of the probes that run the
// reference's host sources in one process: see oracle/ref_host.cpp.
#pragma once
#include <cosmictiger/options.hpp>
#include <cosmictiger/particles.hpp>
#include <cosmictiger/tree.hpp>
#include <cosmictiger/range.hpp>
#include <gsl/gsl_rng.h>

#include <cstdint>
#include <vector>

#include "ct_oracle.h"

// the options every reference function reads (get_options()); ref_set_defaults() sets the
// reference's defaults for the cache and allocation line sizes and turns groups, tracers and
// saved forces off
extern options g_opts;
void ref_set_defaults();

// the reference's tree below `id` in ct_or_node records: depth first, left child first, heap keys
void ref_emit_tree(tree_id id, uint64_t key, int depth, std::vector<ct_or_node>& out);
