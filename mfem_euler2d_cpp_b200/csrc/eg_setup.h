// Host-side setup and diagnostics of the simple-wave problem (C++).
#pragma once
#include <string>
#include <vector>

#include "../../include/euler2d_cuda.h"

namespace eg {
namespace host {
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w);
double lagrange(const std::vector<double> &nodes, int i, double x);
double dlagrange(const std::vector<double> &nodes, int i, double x);
void fill_desc(eg_desc &d, int nx, int ny, int k, double alpha_deg, double gamma, double safety);
void exact(double gamma, double x, double y, double time, double alpha, double out[4]);
void initial(const eg_desc &d, std::vector<double> &u);
void errors(const eg_desc &d, const double *u, double time, double out[4]);
void integral(const eg_desc &d, const double *u, double out[4]);
void differences(const eg_desc &d, const double *u, const double *v, double out[4]);
// Problem::Save (src/problem.cpp:762-790): prefix.mesh (the Cartesian quadrilateral mesh in
// MFEM mesh v1.0 text), prefix_{rho,rhou,rhov,energy}.gf (one L2 Gauss-Legendre grid function
// per component, element-major DOFs) and prefix_coefficients.csv. Returns false when a file
// cannot be opened.
bool save_solution(const eg_desc &d, const double *u, const std::string &prefix);
}  // namespace host
}  // namespace eg
