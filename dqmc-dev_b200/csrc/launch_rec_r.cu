// Recombine launchers, real scalars.
#include "launch_qr.cuh"

namespace dq {
template int launch_rec<double>(const RecArgs<double> &, cudaStream_t);
}
