// Host-side set-up structures shared by the set-up code, the kernels' launch
// wrappers and the C-ABI layer.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/flowgpu.h"

namespace fp {

// Compile-time element configuration (element type x order); quadrature sizes are
// those of FlowPro's rules (QuadratureCentral: order k -> line k points, triangle of
// degree 2k-1 (2k if negative weights), tetrahedron of degree 2k-1).
constexpr int nbasis_of(int dim, int order) {
    return dim == 2 ? order * (order + 1) / 2 : (3 * (order - 1) * order + 2) / 2;
}
constexpr int nqv_of(int dim, int order) {
    return dim == 2 ? (order == 1 ? 1 : order == 2 ? 6 : order == 3 ? 7 : 16)
                    : (order == 1 ? 1 : order == 2 ? 6 : 14);
}
constexpr int nqf_of(int dim, int order) {
    return dim == 2 ? order : (order == 1 ? 1 : order == 2 ? 6 : 7);
}
constexpr int nperm_of(int dim) { return dim == 2 ? 2 : 6; }

// Geometry fields per element, stored field-major: geo[field * ld + e]
template <int DIM>
struct GeoLayout {
    static constexpr int NF = DIM + 1;
    static constexpr int JINV = 0;                    // Jinv[d'][d] (dim*dim): dphi/dx_d = sum_d' Jinv[d'][d] dphi/dxi_d'
    static constexpr int JAC = JINV + DIM * DIM;      // volume Jacobian as FlowPro defines it (|det|/2 in 2D, |det| in 3D)
    static constexpr int NRM = JAC + 1;               // n[k][d] outward unit normals
    static constexpr int JF = NRM + NF * DIM;         // face Jacobian per face
    static constexpr int DL = JF + NF;                // DDG distance dL per face
    static constexpr int X0 = DL + NF;                // x(xi) = X0 + J xi
    static constexpr int JM = X0 + DIM;               // J[i][j] = dx_i/dxi_j
    static constexpr int SIZE = JM + DIM * DIM;       // elemSize
    static constexpr int AREA = SIZE + 1;             // area (volume)
    static constexpr int NFIELDS = AREA + 1;
};

// Reference tables of one (element type, order), all doubles, packed:
//   vol:   w[q], phi[q][j], dphi[q][j][d], interp[q][v], xi[q][d]
//   faceL: wf[p], phiL[k][p][j], dphiL[k][p][j][d], finterp[p][vf], xiL[k][p][d]
//   faceR: phiR[k'][perm][p][j], dphiR[k'][perm][p][j][d]
//   misc:  Is[j] (basis means), Mref[i][j] (reference mass matrix, sum_q w phi_i phi_j), MinvRef,
//          one[j] (coefficients of the constant 1), trun[i][j] (projection onto linear functions)
struct RefTables {
    int dim = 2, order = 1, nb = 1, nqv = 1, nqf = 1, nf = 3, nv = 3, nvf = 2, nperm = 2;
    int o_w, o_phi, o_dphi, o_interp, o_xi;
    int o_wf, o_phiL, o_dphiL, o_finterp, o_xiL;
    int o_phiR, o_dphiR;
    int o_Is, o_Mref, o_MinvRef, o_one, o_trun;
    std::vector<double> data;
};

struct HostMesh {
    int dim = 2, nElem = 0, nVert = 0, nf = 3, nv = 3, ld = 0;
    fp_model_params model{};
    fp_num_params num{};
    RefTables tab;
    std::vector<double> geo;          // [NFIELDS][ld]
    std::vector<int> tt;              // [nf][ld] neighbour or negative BC code
    std::vector<int> fcode;           // [nf][ld] k' * nperm + perm for interior faces
    std::vector<double> vwd;          // [nv][ld] wall distance at the element vertices
    std::vector<double> vu;           // [nv*dim][ld] mesh velocity at the element vertices (empty: static)
    std::vector<int> order;           // element indexes in DOF order (RCM)
    std::vector<int> rank;            // position of element e in the DOF order
    std::vector<double> area, elemSize, xs;  // host copies for checks
    // face list of the face-based residual (each face once, owner = lower element index)
    int nFaces = 0, ldf = 0;
    bool faceMode = false;            // every neighbour quadrature point matched an owner point
    std::vector<int> fl, fk, fr, fc;  // [ldf] owner, owner's face, neighbour (or BC code), neighbour code
    std::vector<int> qmap;            // [nperm][nqf] neighbour-side quadrature index of owner point p
    std::vector<int> efc;             // [nf][ld] (face << 1) | side
};

// set-up functions (fp_setup.cpp)
int build_ref_tables(int dim, int order, RefTables& t, std::string& err);
int build_host_mesh(const fp_mesh_desc& desc, const fp_model_params& model, const fp_num_params& num,
                    HostMesh& hm, std::string& err);
int model_from_properties(const char* props, fp_model_params& m, fp_num_params& n, std::string& err);
std::vector<int> reverse_cuthill_mckee(int nElem, int nf, const int* tt);
int create_neighbor_matrix(int dim, int nElem, const int* elements, int nBound, const int* boundary, int* tt);
void const_init_condition(const fp_model_params& m, double* w);

}  // namespace fp
