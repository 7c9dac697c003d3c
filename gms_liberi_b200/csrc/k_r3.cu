// k_r3.cu -- explicit instantiation of the int2120, int2111 quartet classes (quartet.cuh).
#include "quartet.cuh"

namespace liberi {
template cudaError_t launch_t<2, 1, 2, 0>(const ClassArgs &, int, int, cudaStream_t);
template cudaError_t launch_t<2, 1, 1, 1>(const ClassArgs &, int, int, cudaStream_t);
}  // namespace liberi
