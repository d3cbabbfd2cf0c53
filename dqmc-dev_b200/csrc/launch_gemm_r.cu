// Batched GEMM launchers, real scalars.
#include "launch_gemm.cuh"

namespace dq {
template int launch_gemm<double>(const GemmArgs<double> &, cudaStream_t);
}
