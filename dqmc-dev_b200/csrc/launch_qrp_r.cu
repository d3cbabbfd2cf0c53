// Column-pivoted QR launchers, real scalars.
#include "launch_qr.cuh"

namespace dq {
template int launch_qr_pivot<double>(const QrArgs<double> &, cudaStream_t);
}
