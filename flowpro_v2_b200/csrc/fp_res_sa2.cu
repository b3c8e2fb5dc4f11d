// Kernels of the 2D Spalart-Allmaras RANS model.
#include "fp_residual_impl.cuh"

namespace fp {
const Launchers* launchers_sa2(int order) {
    static const Launchers t[3] = {Launch<SA2, 2, 2>::table(), Launch<SA2, 2, 3>::table(), Launch<SA2, 2, 4>::table()};
    return order >= 2 && order <= 4 ? &t[order - 2] : nullptr;
}
}  // namespace fp
