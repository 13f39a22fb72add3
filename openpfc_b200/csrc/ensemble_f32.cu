// FP32 instantiation of the ensemble stage kernels (see ensemble.cuh).
#include "ensemble.cuh"
namespace opfc {
template int ens_launch_stage<float>(int, int, int, int, int, int, const EnsArgs &, cudaStream_t);
}
