// Test infrastructure only (oracle build): part of the single-threaded HPX stand-in, see hpx/hpx.hpp.
#pragma once
#include <hpx/hpx.hpp>
