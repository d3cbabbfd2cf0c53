// Scalar types and small device helpers shared by the DQMC kernels.
//
// The engine computes in FP64 throughout (double), or complex128 when the
// hopping matrix carries Peierls phases (zd below, the layout of C99
// double complex: re then im).  Kernels are templates over the scalar.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dq {

struct __align__(16) zd {
	double x, y;
};

__host__ __device__ inline zd mkz(double a, double b) { return zd{a, b}; }
__host__ __device__ inline zd operator+(zd a, zd b) { return zd{a.x + b.x, a.y + b.y}; }
__host__ __device__ inline zd operator-(zd a, zd b) { return zd{a.x - b.x, a.y - b.y}; }
__host__ __device__ inline zd operator-(zd a) { return zd{-a.x, -a.y}; }
__host__ __device__ inline zd operator+(zd a) { return a; }
__host__ __device__ inline zd operator*(zd a, zd b) {
	return zd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__host__ __device__ inline zd operator*(double s, zd a) { return zd{s * a.x, s * a.y}; }
__host__ __device__ inline zd operator*(zd a, double s) { return zd{s * a.x, s * a.y}; }
__host__ __device__ inline zd operator+(zd a, double s) { return zd{a.x + s, a.y}; }
__host__ __device__ inline zd operator+(double s, zd a) { return zd{a.x + s, a.y}; }
__host__ __device__ inline zd operator-(double s, zd a) { return zd{s - a.x, -a.y}; }
__host__ __device__ inline zd operator-(zd a, double s) { return zd{a.x - s, a.y}; }
__host__ __device__ inline zd &operator+=(zd &a, zd b) { a.x += b.x; a.y += b.y; return a; }
__host__ __device__ inline zd &operator-=(zd &a, zd b) { a.x -= b.x; a.y -= b.y; return a; }
__host__ __device__ inline zd &operator*=(zd &a, zd b) { a = a * b; return a; }
__host__ __device__ inline zd &operator*=(zd &a, double s) { a.x *= s; a.y *= s; return a; }
__host__ __device__ inline zd operator/(zd a, zd b) {
	// Smith's algorithm keeps the intermediate products in range
	if (fabs(b.x) >= fabs(b.y)) {
		const double r = b.y / b.x, den = b.x + b.y * r;
		return zd{(a.x + a.y * r) / den, (a.y - a.x * r) / den};
	}
	const double r = b.x / b.y, den = b.x * r + b.y;
	return zd{(a.x * r + a.y) / den, (a.y * r - a.x) / den};
}
__host__ __device__ inline zd operator/(zd a, double s) { return zd{a.x / s, a.y / s}; }
__host__ __device__ inline zd operator/(double s, zd b) { return zd{s, 0.0} / b; }

// uniform helpers over double and zd
__host__ __device__ inline double re(double a) { return a; }
__host__ __device__ inline double re(zd a) { return a.x; }
__host__ __device__ inline double im(double) { return 0.0; }
__host__ __device__ inline double im(zd a) { return a.y; }
__host__ __device__ inline double conjv(double a) { return a; }
__host__ __device__ inline zd conjv(zd a) { return zd{a.x, -a.y}; }
__host__ __device__ inline double abs2(double a) { return a * a; }
__host__ __device__ inline double abs2(zd a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ inline double absv(double a) { return fabs(a); }
__host__ __device__ inline double absv(zd a) { return hypot(a.x, a.y); }
template <typename T> __host__ __device__ inline T from_re(double a);
template <> __host__ __device__ inline double from_re<double>(double a) { return a; }
template <> __host__ __device__ inline zd from_re<zd>(double a) { return zd{a, 0.0}; }
template <typename T> __host__ __device__ inline T zero() { return from_re<T>(0.0); }
template <typename T> __host__ __device__ inline T one() { return from_re<T>(1.0); }
__host__ __device__ inline double fma_(double a, double b, double c) { return fma(a, b, c); }
__host__ __device__ inline zd fma_(zd a, zd b, zd c) {
	return zd{fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y))};
}
// phase a/|a| (1 for a == 0)
__host__ __device__ inline double phase_of(double a) { return a < 0.0 ? -1.0 : 1.0; }
__host__ __device__ inline zd phase_of(zd a) {
	const double m = hypot(a.x, a.y);
	return m > 0.0 ? zd{a.x / m, a.y / m} : zd{1.0, 0.0};
}

__host__ __device__ inline void split(const double &v, double &r, double &i) { r = v; i = 0.0; }
__host__ __device__ inline void split(const zd &v, double &r, double &i) { r = v.x; i = v.y; }

template <typename T> struct is_cplx { static constexpr bool value = false; };
template <> struct is_cplx<zd> { static constexpr bool value = true; };

__device__ inline double shfl(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }
__device__ inline zd shfl(zd v, int src) {
	return zd{__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src)};
}
__device__ inline double shfl_xor(double v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
__device__ inline zd shfl_xor(zd v, int o) {
	return zd{__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o)};
}
__device__ inline double warp_sum(double v) {
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}
__device__ inline zd warp_sum(zd v) {
	for (int o = 16; o > 0; o >>= 1) {
		v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
		v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
	}
	return v;
}

// Warp-level FP64 tensor-core MMA, m8n8k4 (row-major A 8x4, col-major B 4x8):
// lane l holds a = A[l/4][l%4], b = B[l%4][l/4], c = C[l/4][2(l%4)+{0,1}].
__device__ inline void dmma(double &c0, double &c1, double a, double b) {
	asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
	             : "+d"(c0), "+d"(c1)
	             : "d"(a), "d"(b));
}

// error word set by kernels instead of trapping; read by the host after a step
enum : unsigned {
	DQ_ERR_NONE = 0,
	DQ_ERR_SIZE = 1u << 0,     // a size beyond what the kernel was built for
	DQ_ERR_SINGULAR = 1u << 1, // zero pivot in the final solve
	DQ_ERR_NAN = 1u << 2,      // non-finite value detected
	DQ_ERR_TIMEOUT = 1u << 3,  // a bounded wait on another CTA ran out
};

}  // namespace dq
