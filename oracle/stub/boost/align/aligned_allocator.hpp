// Test infrastructure only (oracle build).  The one Boost.Align template the reference's
// src/gravity.cpp uses (boost::alignment::aligned_allocator<T, Alignment>), as a standard
// allocator over C++17 aligned new, so that the source compiles where it lies for the probes.
#pragma once
#include <cstddef>
#include <new>

namespace boost {
namespace alignment {
template<class T, std::size_t Alignment = alignof(T)>
class aligned_allocator {
public:
	using value_type = T;
	static constexpr std::size_t align = Alignment < alignof(T) ? alignof(T) : Alignment;
	template<class U>
	struct rebind {
		using other = aligned_allocator<U, Alignment>;
	};
	aligned_allocator() noexcept = default;
	template<class U>
	aligned_allocator(const aligned_allocator<U, Alignment>&) noexcept {
	}
	T* allocate(std::size_t n) {
		return static_cast<T*>(::operator new(n * sizeof(T), std::align_val_t(align)));
	}
	void deallocate(T* p, std::size_t) noexcept {
		::operator delete(p, std::align_val_t(align));
	}
	template<class U>
	bool operator==(const aligned_allocator<U, Alignment>&) const noexcept {
		return true;
	}
	template<class U>
	bool operator!=(const aligned_allocator<U, Alignment>&) const noexcept {
		return false;
	}
};
}  // namespace alignment
}  // namespace boost
