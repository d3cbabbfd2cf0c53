// Pre-sorted QR launchers, complex scalars.
#include "launch_qr.cuh"

namespace dq {
template int launch_qr_presort<zd>(const QrArgs<zd> &, cudaStream_t);
}
