// Test infrastructure only (oracle build). Stand-in for a Thrust header that current CCCL no longer ships; the reference's
// cosmictiger/cuda.hpp includes it only for a pinned-allocator alias.
#pragma once
#include <memory>
namespace thrust { namespace system { namespace cuda { namespace experimental {
template<class T> using pinned_allocator = std::allocator<T>;
} } } }
