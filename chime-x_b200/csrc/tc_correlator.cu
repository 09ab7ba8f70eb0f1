// tc_correlator.cu -- tcgen05 kind::i8 correlator (placeholder until the
// tensor-core kernel lands; the plain path uses the SIMT kernel meanwhile).
#include "chimex_internal.h"

namespace chx {

bool tc_supported(int, int) { return false; }

cudaError_t launch_correlate_tc(const TcArgs &, int, cudaStream_t) {
    return cudaErrorNotSupported;
}

}  // namespace chx
