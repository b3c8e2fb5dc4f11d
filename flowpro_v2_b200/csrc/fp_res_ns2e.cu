// Kernels of the 2D compressible Euler model (NavierStokes with isFlowViscous = false).
#include "fp_residual_impl.cuh"

namespace fp {
const Launchers* launchers_ns2_euler(int order) {
    static const Launchers t[4] = {Launch<NS2E, 2, 1>::table(), Launch<NS2E, 2, 2>::table(), Launch<NS2E, 2, 3>::table(),
                                   Launch<NS2E, 2, 4>::table()};
    return order >= 1 && order <= 4 ? &t[order - 1] : nullptr;
}
}  // namespace fp
