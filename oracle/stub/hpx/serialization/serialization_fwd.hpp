// Test infrastructure only (oracle build). Stand-in for the one HPX header the reference's CUDA sources include (through tree.hpp):
// the serialization macro is not needed when the kick runs in a single process.
#pragma once
#define HPX_SERIALIZATION_SPLIT_MEMBER()
