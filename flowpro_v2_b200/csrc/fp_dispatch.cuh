// Model configurations compiled into the library.
#pragma once
#include "fp_kernels.cuh"

namespace fp {

using NS2E = NS<2, false>;   // 2D Euler
using NS2V = NS<2, true>;    // 2D Navier-Stokes
using NS3E = NS<3, false>;   // 3D Euler
using NS3V = NS<3, true>;    // 3D Navier-Stokes
using SA2 = SA<2>;           // 2D Spalart-Allmaras
using SC2A = Scalar<2, false>;  // scalar advection (reference tests)
using SC2D = Scalar<2, true>;   // scalar advection-diffusion (reference tests)
using AD2 = Adiabatic<2>;       // 2D isentropic Euler (AdiabaticEulers)
using AD3 = Adiabatic<3>;       // 3D isentropic Euler

}  // namespace fp
