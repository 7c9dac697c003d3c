// k_d1.cu -- explicit instantiation of the int1111, int0002, int0012, int0102 quartet classes (quartet.cuh).
#include "quartet.cuh"

namespace liberi {
template cudaError_t launch_t<1, 1, 1, 1>(const ClassArgs &, int, int, cudaStream_t);
template cudaError_t launch_t<2, 0, 0, 0>(const ClassArgs &, int, int, cudaStream_t);
template cudaError_t launch_t<2, 1, 0, 0>(const ClassArgs &, int, int, cudaStream_t);
template cudaError_t launch_t<2, 0, 1, 0>(const ClassArgs &, int, int, cudaStream_t);
}  // namespace liberi
