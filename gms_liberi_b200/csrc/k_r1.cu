// k_r1.cu -- explicit instantiation of the int2211 quartet class (quartet.cuh).
#include "quartet.cuh"

namespace liberi {
template cudaError_t launch_t<2, 2, 1, 1>(const ClassArgs &, int, int, cudaStream_t);
}  // namespace liberi
