// Column-pivoted QR launchers, complex scalars.
#include "launch_qr.cuh"

namespace dq {
template int launch_qr_pivot<zd>(const QrArgs<zd> &, cudaStream_t);
}
