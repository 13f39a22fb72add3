// FP64 instantiation of the pass kernels (see kernels.cuh).
#include "kernels.cuh"
namespace opfc {
OPFC_INSTANTIATE(double)
}
