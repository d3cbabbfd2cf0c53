// Unequal-time Green's functions G(0,t), G(t,t), G(t,0) for every slice
// (reference src/greens.c:247-494, calc_ue_g).
#pragma once

#include "common.cuh"

namespace dq {

template <typename T>
struct UneqState {
	static bool supported(int, int) { return false; }
	int alloc(int, int, int, int) { return 0; }
	void release() {}
	template <typename G>
	int compute(G &) { return -10; }
	struct Buf { T *p = nullptr; };
	Buf G0t, Gtt, Gt0;
};

}  // namespace dq
