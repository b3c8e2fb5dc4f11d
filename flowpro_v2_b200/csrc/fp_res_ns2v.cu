// Kernels of the 2D compressible Navier-Stokes model (NavierStokes with isFlowViscous = true).
#include "fp_residual_impl.cuh"

namespace fp {
const Launchers* launchers_ns2_viscous(int order) {
    static const Launchers t[4] = {Launch<NS2V, 2, 1>::table(), Launch<NS2V, 2, 2>::table(), Launch<NS2V, 2, 3>::table(),
                                   Launch<NS2V, 2, 4>::table()};
    return order >= 1 && order <= 4 ? &t[order - 1] : nullptr;
}
const Launchers* launchers_ns2_euler(int order);
const Launchers* launchers_ns2(int viscous, int order) {
    return viscous ? launchers_ns2_viscous(order) : launchers_ns2_euler(order);
}
}  // namespace fp
