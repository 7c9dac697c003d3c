// k_r2.cu -- explicit instantiation of the int2121 quartet class (quartet.cuh).
#include "quartet.cuh"

namespace liberi {
template cudaError_t launch_t<2, 1, 2, 1>(const ClassArgs &, int, int, cudaStream_t);
}  // namespace liberi
