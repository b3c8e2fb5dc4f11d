// Kernels of the isentropic Euler model (AdiabaticEulers) on triangles and tetrahedra.
#include "fp_residual_impl.cuh"

namespace fp {
const Launchers* launchers_adiabatic(int dim, int order) {
    static const Launchers t2[4] = {Launch<AD2, 2, 1>::table(), Launch<AD2, 2, 2>::table(), Launch<AD2, 2, 3>::table(),
                                    Launch<AD2, 2, 4>::table()};
    static const Launchers t3[3] = {Launch<AD3, 3, 1>::table(), Launch<AD3, 3, 2>::table(), Launch<AD3, 3, 3>::table()};
    if (dim == 2 && order >= 1 && order <= 4) return &t2[order - 1];
    if (dim == 3 && order >= 1 && order <= 3) return &t3[order - 1];
    return nullptr;
}
}  // namespace fp
