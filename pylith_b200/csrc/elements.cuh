// Reference elements and geometry for the cell-loop kernels.
//
// What PETSc's PetscFE/PetscFEGeom provide to DMPlexComputeResidual (basis tabulation at
// quadrature points, J, |J|, J^{-1}; topology/FieldOps.cc:42-129): here as compile-time
// element descriptions. Quadrature: P1 tetrahedron, centroid rule (integrates the constant
// and linear integrands of P1 elasticity exactly); Q1 hexahedron, 2x2x2 Gauss-Legendre;
// Q2 hexahedron, 3x3x3 Gauss-Legendre with trilinear geometry from the 8 corners. Node
// orders are those of pylith_b200/meshing.py.
#pragma once

#include "common.cuh"

namespace plb {

enum CellKind { TET4 = 0, HEX8 = 1, HEX27 = 2 };

template <int CELL>
struct ElementTraits;

template <>
struct ElementTraits<TET4> {
    static constexpr int nen = 4;
    static constexpr int nq = 1;
};
template <>
struct ElementTraits<HEX8> {
    static constexpr int nen = 8;
    static constexpr int nq = 8;
};
template <>
struct ElementTraits<HEX27> {
    static constexpr int nen = 27;
    static constexpr int nq = 27;
};

// Hexahedron corner c in {0..7}: lattice offsets (0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),...
PL_HD int hex_cx(int c) { return ((c + 1) >> 1) & 1; }
PL_HD int hex_cy(int c) { return (c >> 1) & 1; }
PL_HD int hex_cz(int c) { return c >> 2; }

// 1-D Gauss points on [-1, 1]
PL_HD double gauss2_x(int i) { return i == 0 ? -0.57735026918962576451 : 0.57735026918962576451; }
PL_HD double gauss3_x(int i) {
    return i == 0 ? -0.77459666924148337704 : (i == 1 ? 0.0 : 0.77459666924148337704);
}
PL_HD double gauss3_w(int i) { return i == 1 ? (8.0 / 9.0) : (5.0 / 9.0); }

// Linear 1-D Lagrange basis on {-1, 1}: value and derivative of node a at x.
PL_HD double lin_v(int a, double x) { return a == 0 ? 0.5 * (1.0 - x) : 0.5 * (1.0 + x); }
PL_HD double lin_d(int a) { return a == 0 ? -0.5 : 0.5; }
// Quadratic 1-D Lagrange basis on {-1, 0, 1}.
PL_HD double quad_v(int a, double x) {
    return a == 0 ? 0.5 * x * (x - 1.0) : (a == 1 ? 1.0 - x * x : 0.5 * x * (x + 1.0));
}
PL_HD double quad_d(int a, double x) { return a == 0 ? x - 0.5 : (a == 1 ? -2.0 * x : x + 0.5); }

struct Geom {
    double inv[3][3];  // dxi/dx
    double wdetJ;
    double detJ;
};

// 3x3 inverse by cofactors; returns det.
template <typename R>
PL_HD R invert3(const R J[3][3], R inv[3][3]) {
    const R c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const R c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const R c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const R det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    const R r = R(1) / det;
    inv[0][0] = c00 * r;
    inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * r;
    inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * r;
    inv[1][0] = c01 * r;
    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * r;
    inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * r;
    inv[2][0] = c02 * r;
    inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * r;
    inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * r;
    return det;
}

// Reference-coordinate gradient of the trilinear corner basis at Gauss point (qi,qj,qk) of an
// n-point rule.
template <int NQD>
PL_HD void hex_corner_dN(int c, int qi, int qj, int qk, double d[3]) {
    const double x = NQD == 2 ? gauss2_x(qi) : gauss3_x(qi);
    const double y = NQD == 2 ? gauss2_x(qj) : gauss3_x(qj);
    const double z = NQD == 2 ? gauss2_x(qk) : gauss3_x(qk);
    const int a = hex_cx(c), b = hex_cy(c), e = hex_cz(c);
    d[0] = lin_d(a) * lin_v(b, y) * lin_v(e, z);
    d[1] = lin_v(a, x) * lin_d(b) * lin_v(e, z);
    d[2] = lin_v(a, x) * lin_v(b, y) * lin_d(e);
}

PL_HD double hex_corner_N(int c, double x, double y, double z) {
    return lin_v(hex_cx(c), x) * lin_v(hex_cy(c), y) * lin_v(hex_cz(c), z);
}

// Trilinear geometry at a Gauss point of a hexahedron from its 8 corner coordinates.
template <int NQD>
PL_HD void hex_geometry(const double X[8][3], int qi, int qj, int qk, double w, Geom* g) {
    double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        double d[3];
        hex_corner_dN<NQD>(c, qi, qj, qk, d);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) J[i][j] += X[c][i] * d[j];
    }
    g->detJ = invert3(J, g->inv);
    g->wdetJ = w * g->detJ;
}

// Trilinear geometry at the cell centre (reference point (0,0,0)): where basis-order-0 derived
// fields are evaluated (PETSc's order-0 Lagrange dual basis is the value at the centroid).
PL_HD void hex_geometry_centre(const double X[8][3], Geom* g) {
    double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const double d[3] = {lin_d(hex_cx(c)) * 0.25, lin_d(hex_cy(c)) * 0.25, lin_d(hex_cz(c)) * 0.25};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) J[i][j] += X[c][i] * d[j];
    }
    g->detJ = invert3(J, g->inv);
    g->wdetJ = 8.0 * g->detJ;
}

// Affine tetrahedron geometry: reference vertices (0,0,0),(1,0,0),(0,1,0),(0,0,1).
PL_HD void tet_geometry(const double X[4][3], Geom* g) {
    double J[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        J[i][0] = X[1][i] - X[0][i];
        J[i][1] = X[2][i] - X[0][i];
        J[i][2] = X[3][i] - X[0][i];
    }
    g->detJ = invert3(J, g->inv);
    g->wdetJ = g->detJ / 6.0;
}

// Physical gradient of tet basis function n: rows of J^{-1} (n = 1..3), minus their sum (n = 0).
PL_HD void tet_grad(const Geom& g, int n, double out[3]) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        out[j] = n == 0 ? -(g.inv[0][j] + g.inv[1][j] + g.inv[2][j]) : g.inv[n - 1][j];
    }
}

}  // namespace plb
