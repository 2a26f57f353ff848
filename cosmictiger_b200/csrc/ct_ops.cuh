// Order dispatch for the generated operators: kernels are templated on one of these.
#pragma once
#include "fmm_p5.h"
#include "fmm_p7.h"

namespace ct {

#define CT_OPS_STRUCT(NAME, NS)                                                                          \
	struct NAME {                                                                                        \
		static constexpr int ORDER = NS::ORDER;                                                          \
		static constexpr int NEXP = NS::NEXP;                                                            \
		static constexpr int NMULT = NS::NMULT;                                                          \
		static constexpr int NFULL = NS::NFULL;                                                          \
		using Tab = NS::EwaldTab;                                                                        \
		template<class T> __host__ __device__ __forceinline__ static void greens(T* D, T x, T y, T z) {  \
			NS::greens(D, x, y, z);                                                                      \
		}                                                                                                \
		template<class T> __host__ __device__ __forceinline__ static void greens_add(T* L, T x, T y, T z) { \
			NS::greens_add(L, x, y, z);                                                                  \
		}                                                                                                \
		template<class T, class TabT> __host__ __device__ __forceinline__ static int ewald(T* D, T x, T y, T z, const TabT& t) { \
			return NS::ewald_greens(D, x, y, z, t);                                                      \
		}                                                                                                \
		template<class T> __host__ __device__ __forceinline__ static void m2l(T* L, const T* M, const T* D, bool p) { \
			NS::m2l(L, M, D, p);                                                                         \
		}                                                                                                \
		template<class T> __host__ __device__ __forceinline__ static void m2l2(T* L, const T* M, const T* D, bool p) { \
			NS::m2l_2(L, M, D, p);                                                                       \
		}                                                                                                \
		template<class T> __host__ __device__ __forceinline__ static void p2m(T* M, T x, T y, T z) {     \
			NS::p2m(M, x, y, z);                                                                         \
		}                                                                                                \
		template<class T> __host__ __device__ __forceinline__ static void m2m(T* M, const T* Ma, T x, T y, T z) { \
			NS::m2m(M, Ma, x, y, z);                                                                     \
		}                                                                                                \
		template<class T> __host__ __device__ __forceinline__ static void l2l(T* Lb, const T* La, T x, T y, T z, bool p) { \
			NS::l2l(Lb, La, x, y, z, p);                                                                 \
		}                                                                                                \
		template<class T> __host__ __device__ __forceinline__ static void l2p(T* Lb, const T* La, T x, T y, T z, bool p) { \
			NS::l2p(Lb, La, x, y, z, p);                                                                 \
		}                                                                                                \
	};

CT_OPS_STRUCT(Ops7, ct_p7)
CT_OPS_STRUCT(Ops5, ct_p5)

// Reference flop convention per interaction (returned counts of cosmictiger/fmm_kernels.hpp
// and the hand counts of src/gravity.cu / src/kick.cu); used only for reporting.
constexpr double FLOP_PP = 21;          // gravity.cu:343
constexpr double FLOP_GREENS = 265;     // fmm_kernels.hpp:306 (262 + 3 scale)
constexpr double FLOP_M2L = 1583;       // fmm_kernels.hpp:1890
constexpr double FLOP_M2L_PHI = 119;
constexpr double FLOP_M2L2 = 520;       // gravity.cu:197-203
constexpr double FLOP_L2L = 2650;       // kick.cu:257
constexpr double FLOP_L2L_PHI = 332;
constexpr double FLOP_KICK = 557;       // kick.cu:153
constexpr double FLOP_KICK_PHI = 178;

}  // namespace ct
