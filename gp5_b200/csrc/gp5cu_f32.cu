// Complex64 instantiation of the kernels and launchers (FP64 reductions).
#include "launch_impl.cuh"

namespace gp5 {
template struct Launch<float>;
}
