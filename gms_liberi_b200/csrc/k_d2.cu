// k_d2.cu -- explicit instantiation of the int0112, int0022, int0122, int1102, int0202 quartet classes (quartet.cuh).
#include "quartet.cuh"

namespace liberi {
template cudaError_t launch_t<2, 1, 1, 0>(const ClassArgs &, int, int, cudaStream_t);
template cudaError_t launch_t<2, 2, 0, 0>(const ClassArgs &, int, int, cudaStream_t);
template cudaError_t launch_t<2, 2, 1, 0>(const ClassArgs &, int, int, cudaStream_t);
template cudaError_t launch_t<1, 1, 2, 0>(const ClassArgs &, int, int, cudaStream_t);
template cudaError_t launch_t<2, 0, 2, 0>(const ClassArgs &, int, int, cudaStream_t);
}  // namespace liberi
