// Complex128 instantiation of the kernels and launchers.
#include "launch_impl.cuh"

namespace gp5 {
template struct Launch<double>;
}
