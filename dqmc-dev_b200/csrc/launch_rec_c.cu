// Recombine launchers, complex scalars.
#include "launch_qr.cuh"

namespace dq {
template int launch_rec<zd>(const RecArgs<zd> &, cudaStream_t);
}
