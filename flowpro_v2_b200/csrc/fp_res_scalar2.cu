// Kernels of the scalar advection(-diffusion) test equation of the reference tests.
#include "fp_residual_impl.cuh"

namespace fp {
const Launchers* launchers_scalar2(int viscous, int order) {
    static const Launchers a[4] = {Launch<SC2A, 2, 1>::table(), Launch<SC2A, 2, 2>::table(), Launch<SC2A, 2, 3>::table(),
                                   Launch<SC2A, 2, 4>::table()};
    static const Launchers d[4] = {Launch<SC2D, 2, 1>::table(), Launch<SC2D, 2, 2>::table(), Launch<SC2D, 2, 3>::table(),
                                   Launch<SC2D, 2, 4>::table()};
    if (order < 1 || order > 4) return nullptr;
    return viscous ? &d[order - 1] : &a[order - 1];
}
}  // namespace fp
