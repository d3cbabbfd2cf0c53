// Batched GEMM launchers, complex scalars.
#include "launch_gemm.cuh"

namespace dq {
template int launch_gemm<zd>(const GemmArgs<zd> &, cudaStream_t);
}
