// Per-device cache of the kernels' dynamic shared-memory limits, and the
// tensor maps of the TMA-fed GEMM.
#include <cudaTypedefs.h>

#include <map>
#include <mutex>
#include <utility>

#include "launch.cuh"

namespace dq {

// cuTensorMapEncodeTiled from the driver, looked up once
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
	static std::once_flag once;
	static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
	std::call_once(once, []() {
		void *p = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
		    q == cudaDriverEntryPointSuccess)
			fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
	});
	return fn;
}

bool tma_map_operand(CUtensorMap *map, int *tz, int *tw, const void *base, int elem_doubles, int rows,
		int cols, long long ld, const Addr &ad, int batch, int box_rows, int box_cols)
{
	PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
	if (!fn || !base || ad.tab || ad.div < 1 || rows < 1 || cols < 1 || batch < 1) return false;
	const unsigned long long es = 8ull * (unsigned long long)elem_doubles;   // bytes per element
	const unsigned long long s1 = (unsigned long long)ld * es;
	if (((uintptr_t)base & 15) || (s1 & 15) || ld < rows) return false;
	if (ad.hi < 0 || ad.lo < 0 || ((unsigned long long)ad.hi * es) % 16 || ((unsigned long long)ad.lo * es) % 16)
		return false;
	// (rows, columns, b % div, b / div); a coordinate whose stride is 0 is
	// not a dimension of the map (extent 1, coordinate 0)
	const bool zu = ad.lo != 0 && ad.div > 1, wu = ad.hi != 0;
	const unsigned long long fill = s1 * (unsigned long long)cols;          // stride of unused dims
	cuuint64_t dim[4] = {(cuuint64_t)rows * elem_doubles, (cuuint64_t)cols,
	                     zu ? (cuuint64_t)ad.div : 1, wu ? (cuuint64_t)((batch - 1) / ad.div + 1) : 1};
	cuuint64_t str[3] = {s1, zu ? (unsigned long long)ad.lo * es : fill,
	                     wu ? (unsigned long long)ad.hi * es : fill * 2};
	for (int i = 0; i < 3; i++)
		if (str[i] == 0 || str[i] % 16 || str[i] >= (1ull << 40)) return false;
	cuuint32_t box[4] = {(cuuint32_t)(box_rows * elem_doubles), (cuuint32_t)box_cols, 1, 1};
	if (box[0] > 256 || box[1] > 256 || (box[0] * 8) % 16) return false;
	cuuint32_t est[4] = {1, 1, 1, 1};
	const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void *>(base), dim, str, box, est,
	                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
	                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if (r != CUDA_SUCCESS) return false;
	*tz = zu ? 1 : 0;
	*tw = wu ? 1 : 0;
	return true;
}

cudaError_t raise_smem_ptr(const void *kern, size_t bytes, bool carve)
{
	static std::mutex mu;
	static std::map<std::pair<int, const void *>, size_t> cur;
	int dev = 0;
	const cudaError_t ge = cudaGetDevice(&dev);
	if (ge != cudaSuccess) return ge;
	std::lock_guard<std::mutex> lk(mu);
	const auto key = std::make_pair(dev, kern);
	if (carve && !cur.count(key)) {
		const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
		                                           (int)cudaSharedmemCarveoutMaxShared);
		if (e != cudaSuccess) return e;
	}
	size_t &c = cur[key];
	if (bytes <= c) return cudaSuccess;
	const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
	if (e == cudaSuccess) c = bytes;
	return e;
}

}  // namespace dq
