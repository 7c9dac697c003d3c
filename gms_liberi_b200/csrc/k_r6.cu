// k_r6.cu -- explicit instantiation of the int2222 quartet class (quartet.cuh).
#include "quartet.cuh"

namespace liberi {
template cudaError_t launch_t<2, 2, 2, 2>(const ClassArgs &, int, int, cudaStream_t);
}  // namespace liberi
