// Solver output files in the reference's text formats, written by the host loops of
// fp_solve_implicit / fp_solve_explicit when fp_solver_output names a directory:
//
//   residuum.txt   one row per finished step: residuum, t, CPU ms and the relative residua
//                  of the equations (MasterSolver.appendResiduum, MasterSolver.java:94-111);
//                  emptied when a new computation starts (FlowProMain.java:691-700)
//   W.txt          integral averages of the solution per element (Mesh.getAvgW,
//                  Element.calculateAvgW, Element.java:647-655; Mat.save, Mat.java:982-991)
//   We.txt         basis coefficients per element, equation-major (Mesh.getW)
//   artificialViscosity.txt   eps + dampInner per element and equation (Mesh.java:337-345)
//   state.txt      t, steps, CPU, transfer, residuum, CFL, dt, residuumNormalisation, order
//                  as Java properties (State.save, State.java:113-136)
//   STOP           asks the running computation to stop after the current step; the file is
//                  deleted (MasterSolver.isStopRequested, MasterSolver.java:60-67)
//
// Numbers are written as Java's Double.toString writes them: the shortest decimal that reads
// back to the same double, in plain notation for 1e-3 <= |x| < 1e7 and as d.dddE<n> otherwise.
// These are Java 19's digits; Java 17 (the reference's target) prints one or two extra digits
// for some values, which read back to the same double.
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fp_ctx.h"

namespace fp {

namespace {

// shortest round-trip digits of a > 0 and the decimal exponent of the first one:
// a = 0.d1 d2 ... x 10^point
void shortest_digits(double a, std::string& digits, int& point) {
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof buf, a, std::chars_format::scientific);
    std::string s(buf, r.ptr);  // d[.ddd]e[+-]XX
    const size_t epos = s.find('e');
    const int ex = std::atoi(s.c_str() + epos + 1);
    digits.clear();
    for (size_t i = 0; i < epos; i++)
        if (s[i] != '.') digits += s[i];
    while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
    point = ex + 1;
    if (digits.size() == 1) {
        // one significant digit: Double.toString prints at least two, the two-digit decimal
        // closest to the value when it reads back to it (4.9E-324 for the smallest subnormal)
        auto r2 = std::to_chars(buf, buf + sizeof buf, a, std::chars_format::scientific, 1);
        std::string s2(buf, r2.ptr);
        if (std::strtod(s2.c_str(), nullptr) == a) {
            const size_t e2 = s2.find('e');
            std::string d2;
            for (size_t i = 0; i < e2; i++)
                if (s2[i] != '.') d2 += s2[i];
            while (d2.size() > 1 && d2.back() == '0') d2.pop_back();
            digits = d2;
            point = std::atoi(s2.c_str() + e2 + 1) + 1;
        }
    }
}

std::string join(const std::string& dir, const char* name) {
    if (dir.empty()) return name;
    return dir.back() == '/' ? dir + name : dir + "/" + name;
}

}  // namespace

std::string java_double(double x) {
    if (std::isnan(x)) return "NaN";
    if (std::isinf(x)) return x > 0 ? "Infinity" : "-Infinity";
    if (x == 0.0) return std::signbit(x) ? "-0.0" : "0.0";
    const double a = std::fabs(x);
    std::string digits;
    int point = 0;
    shortest_digits(a, digits, point);
    std::string out = x < 0 ? "-" : "";
    if (a >= 1e-3 && a < 1e7) {
        if (point <= 0)
            out += "0." + std::string(-point, '0') + digits;
        else if (point >= (int)digits.size())
            out += digits + std::string(point - digits.size(), '0') + ".0";
        else
            out += digits.substr(0, point) + "." + digits.substr(point);
    } else {
        out += digits.substr(0, 1) + "." + (digits.size() > 1 ? digits.substr(1) : "0") + "E" + std::to_string(point - 1);
    }
    return out;
}

int io_reset_residuum(const std::string& dir) {
    FILE* f = std::fopen(join(dir, "residuum.txt").c_str(), "w");
    if (!f) return FP_ERR_ARG;
    std::fclose(f);
    return FP_OK;
}

int io_append_residuum(const std::string& dir, double residuum, double t, double cpu, const std::vector<double>& eq) {
    FILE* f = std::fopen(join(dir, "residuum.txt").c_str(), "a");
    if (!f) return FP_ERR_ARG;
    std::string line = java_double(residuum) + " " + java_double(t) + " " + java_double(cpu);
    for (double r : eq) line += " " + java_double(r);
    line += "\n";
    std::fputs(line.c_str(), f);
    std::fclose(f);
    return FP_OK;
}

int io_save_rows(const std::string& dir, const char* name, const double* a, size_t rows, size_t cols) {
    FILE* f = std::fopen(join(dir, name).c_str(), "w");
    if (!f) return FP_ERR_ARG;
    std::string line;
    for (size_t i = 0; i < rows; i++) {
        line.clear();
        for (size_t j = 0; j < cols; j++) line += java_double(a[i * cols + j]) + " ";
        line += "\n";
        std::fputs(line.c_str(), f);
    }
    std::fclose(f);
    return FP_OK;
}

int io_save_state(const std::string& dir, const IoState& s) {
    FILE* f = std::fopen(join(dir, "state.txt").c_str(), "w");
    if (!f) return FP_ERR_ARG;
    std::string out = "#FlowPro state\n";
    out += "t=" + java_double(s.t) + "\n";
    out += "steps=" + std::to_string(s.steps) + "\n";
    out += "CPU=" + std::to_string(s.cpu_ms) + "\n";
    out += "transfer=0\n";
    out += "residuum=" + java_double(s.residuum) + "\n";
    out += "CFL=" + java_double(s.cfl) + "\n";
    out += "dt=" + java_double(s.dt) + "\n";
    if (!s.normalisation.empty()) {
        std::string v;
        for (double r : s.normalisation) v += (v.empty() ? "" : ",") + java_double(r);
        out += "residuumNormalisation=" + v + "\n";
    }
    out += "order=" + std::to_string(s.order) + "\n";
    std::fputs(out.c_str(), f);
    std::fclose(f);
    return FP_OK;
}

bool io_stop_requested(const std::string& dir) {
    const std::string p = join(dir, "STOP");
    FILE* f = std::fopen(p.c_str(), "r");
    if (!f) return false;
    std::fclose(f);
    std::remove(p.c_str());
    return true;
}

}  // namespace fp

extern "C" int fp_java_double(double x, char* buf, int n) {
    if (!buf || n <= 0) return FP_ERR_ARG;
    const std::string s = fp::java_double(x);
    if ((int)s.size() + 1 > n) return FP_ERR_ARG;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return FP_OK;
}
