// k_r4.cu -- explicit instantiation of the int2220 quartet class (quartet.cuh).
#include "quartet.cuh"

namespace liberi {
template cudaError_t launch_t<2, 2, 2, 0>(const ClassArgs &, int, int, cudaStream_t);
}  // namespace liberi
