// k_d1.cu -- explicit instantiation of the int0002, int0012, int0102, int0112 quartet classes (quartet.cuh).
#include "quartet.cuh"

namespace liberi {
template cudaError_t launch_t<0, 0, 2, 0>(const ClassArgs &, long long, int, int, cudaStream_t);
template cudaError_t launch_t<0, 0, 2, 1>(const ClassArgs &, long long, int, int, cudaStream_t);
template cudaError_t launch_t<1, 0, 2, 0>(const ClassArgs &, long long, int, int, cudaStream_t);
template cudaError_t launch_t<1, 0, 2, 1>(const ClassArgs &, long long, int, int, cudaStream_t);
}  // namespace liberi
