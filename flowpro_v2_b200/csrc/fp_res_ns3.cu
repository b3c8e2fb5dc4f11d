// Kernels of the 3D compressible Euler / Navier-Stokes models on tetrahedra.
#include "fp_residual_impl.cuh"

namespace fp {
const Launchers* launchers_ns3(int viscous, int order) {
    static const Launchers e[3] = {Launch<NS3E, 3, 1>::table(), Launch<NS3E, 3, 2>::table(), Launch<NS3E, 3, 3>::table()};
    static const Launchers v[3] = {Launch<NS3V, 3, 1>::table(), Launch<NS3V, 3, 2>::table(), Launch<NS3V, 3, 3>::table()};
    if (order < 1 || order > 3) return nullptr;
    return viscous ? &v[order - 1] : &e[order - 1];
}
}  // namespace fp
