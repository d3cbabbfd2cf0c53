// Pre-sorted QR launchers, real scalars.
#include "launch_qr.cuh"

namespace dq {
template int launch_qr_presort<double>(const QrArgs<double> &, cudaStream_t);
}
