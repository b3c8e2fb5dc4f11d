// Host-side solver state shared by the single-case and batched solver loops:
// BDF coefficients and FlowPro's State + CFLSetup.
#pragma once
#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

namespace fp {

// BDF coefficients, BDF2.coefficients (BDF2.java:298-308); dto <= 0: BDF1 start
inline void bdf_coef(int order, double dt, double dto, double* a) {
    if (order == 2 && dto > 0) {
        a[0] = (2 * dt + dto) / (dt * (dt + dto));
        a[1] = -(dt + dto) / (dt * dto);
        a[2] = dt / (dto * (dt + dto));
    } else {
        a[0] = 1 / dt;
        a[1] = -1 / dt;
        a[2] = 0;
    }
}

// State + CFLSetup (State.java:145-240, CFLSetup.java:34-63)
struct State {
    int steps = 0;
    double t = 0, currentCFL = 0, residuum = std::numeric_limits<double>::max(), dt = 0, dt0 = 0;
    std::vector<double> equationResiduum, normalisation;
    int nNorm = 0;
    double cfl = 1, maxCFL = 1e4, resOld = -1;
    bool vary = false, fixed = false;
    double getCFL(double actual, double res) {
        if (!vary) return std::min(actual + cfl / 20, cfl);
        bool known = res > 0 && res < std::numeric_limits<double>::max();
        if (actual <= 0) {
            resOld = known ? res : -1;
            return cfl;
        }
        double factor = 1;
        if (known && resOld > 0) factor = std::max(0.5, std::min(resOld / res, 2.0));
        resOld = known ? res : -1;
        return std::max(std::min(actual, cfl), std::min(actual * factor, maxCFL));
    }
    void updateCFL() {
        if (fixed)
            dt = std::min(2 * dt, dt0);
        else
            currentCFL = getCFL(currentCFL, residuum);
    }
    void reduceCFL() {
        if (fixed) {
            dt /= 2;
        } else {
            resOld = -1;
            currentCFL /= 1.5;
        }
    }
    bool hopeless() const { return fixed ? dt < dt0 / 1024 : (currentCFL > 0 && currentCFL < cfl / 20); }
    void setResiduum(const std::vector<double>& norms) {
        size_t ne = norms.size();
        if (normalisation.size() != ne) {
            normalisation.assign(ne, 0.0);
            nNorm = 0;
        }
        if (nNorm < 5) {
            for (size_t m = 0; m < ne; m++) normalisation[m] = std::max(normalisation[m], norms[m]);
            nNorm++;
        }
        double mx = 0;
        for (double r : normalisation) mx = std::max(mx, r);
        equationResiduum.assign(ne, 0.0);
        residuum = 0;
        for (size_t m = 0; m < ne; m++) {
            double nrm = normalisation[m] > 0 ? normalisation[m] : mx;
            equationResiduum[m] = nrm > 0 ? norms[m] / nrm : norms[m];
            if (std::isnan(equationResiduum[m]))
                residuum = NAN;
            else if (!std::isnan(residuum))
                residuum = std::max(residuum, equationResiduum[m]);
        }
    }
};

}  // namespace fp
