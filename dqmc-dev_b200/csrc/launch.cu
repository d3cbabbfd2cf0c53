// Per-device cache of the kernels' dynamic shared-memory limits.
#include <map>
#include <mutex>
#include <utility>

#include "launch.cuh"

namespace dq {

cudaError_t raise_smem_ptr(const void *kern, size_t bytes)
{
	static std::mutex mu;
	static std::map<std::pair<int, const void *>, size_t> cur;
	int dev = 0;
	const cudaError_t ge = cudaGetDevice(&dev);
	if (ge != cudaSuccess) return ge;
	std::lock_guard<std::mutex> lk(mu);
	size_t &c = cur[std::make_pair(dev, kern)];
	if (bytes <= c) return cudaSuccess;
	const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
	if (e == cudaSuccess) c = bytes;
	return e;
}

}  // namespace dq
