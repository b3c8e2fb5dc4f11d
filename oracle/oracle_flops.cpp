// CPU ORACLE (test infrastructure): the oracle built with a counting floating-point type
// (flop_real.hpp) as build/liboracle_flops.so.  Same C entry points as liboracle.so, plus
// or_flops_reset / or_flops_get: the operations the restated reference algorithm performs, e.g.
// in one residual evaluation (DGpure.residuum with residuumWall, DGpure.java:108-356), which
// is the algorithmic FLOP count the residual kernels' FP64 roofline is measured against.
// Built without OpenMP (one thread, so the counters need no atomics).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <limits>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../flowpro_v2_b200/csrc/gauss_rules.h"
#include "flop_real.hpp"

// the phase hooks of Element::residuum (oracle_dg.hpp)
#define ORC_FACE_PHASE(interior) (orc_flops::g_phase = (interior) ? 1 : 2)
#define ORC_VOLUME_PHASE() (orc_flops::g_phase = 0)

#define double orc_flops::Real
#include "oracle_capi.cpp"
#undef double

orc_flops::Counters orc_flops::g_counts[3];
int orc_flops::g_phase = 0;

extern "C" {
void or_flops_reset() {
    for (auto& c : orc_flops::g_counts) c = orc_flops::Counters();
    orc_flops::g_phase = 0;
}
// out[3][6]: per phase (volume and the rest, interior faces, boundary faces): additions (and
// subtractions, negations), multiplications, divisions, square roots, other library functions,
// trivial operations (an exact zero operand)
void or_flops_get(unsigned long long* out) {
    for (int p = 0; p < 3; p++) {
        const orc_flops::Counters& c = orc_flops::g_counts[p];
        unsigned long long* o = out + 6 * p;
        o[0] = c.add;
        o[1] = c.mul;
        o[2] = c.div;
        o[3] = c.sqrt;
        o[4] = c.fn;
        o[5] = c.triv;
    }
}
}
