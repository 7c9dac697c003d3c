// k_sp.cu -- explicit instantiation of the int0000, int0001, int0011, int0111, int0101 quartet classes (quartet.cuh).
#include "quartet.cuh"

namespace liberi {
template cudaError_t launch_t<0, 0, 0, 0>(const ClassArgs &, int, int, cudaStream_t);
template cudaError_t launch_t<1, 0, 0, 0>(const ClassArgs &, int, int, cudaStream_t);
template cudaError_t launch_t<1, 1, 0, 0>(const ClassArgs &, int, int, cudaStream_t);
template cudaError_t launch_t<1, 1, 1, 0>(const ClassArgs &, int, int, cudaStream_t);
template cudaError_t launch_t<1, 0, 1, 0>(const ClassArgs &, int, int, cudaStream_t);
}  // namespace liberi
