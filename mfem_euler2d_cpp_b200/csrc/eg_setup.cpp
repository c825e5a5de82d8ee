// Host-side problem setup and diagnostics (outside the Newton timer):
// Gauss-Legendre tables of the Qk collocation (src/problem.cpp:91-222), the
// rotated simple wave (src/physics.cpp:64-93), the initial L2 projection
// (src/problem.cpp:329-349), exact-solution errors (704-726), conserved
// integrals (727-738) and DG/HDG L2 differences (739-761).
#include "eg_setup.h"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <stdexcept>

namespace eg {
namespace host {

static constexpr double kPi = 3.141592653589793238462643383279502884;

// Gauss-Legendre nodes/weights on [0,1], ascending; Newton iteration on the
// Legendre three-term recurrence in extended precision, mirrored so the rule
// is exactly symmetric.
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
  x.assign(n, 0.);
  w.assign(n, 0.);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    long double z = std::cos(3.14159265358979323846264338327950288L * (i + 0.75L) / (n + 0.5L));
    long double dp = 0;
    for (int it = 0; it < 100; ++it) {
      long double p0 = 1, p1 = 0;
      for (int j = 1; j <= n; ++j) {
        const long double p2 = p1;
        p1 = p0;
        p0 = ((2 * j - 1) * z * p1 - (j - 1) * p2) / j;
      }
      dp = n * (z * p0 - p1) / (z * z - 1);
      const long double dz = p0 / dp;
      z -= dz;
      if (std::abs(dz) < 1e-19L) break;
    }
    {
      long double p0 = 1, p1 = 0;
      for (int j = 1; j <= n; ++j) {
        const long double p2 = p1;
        p1 = p0;
        p0 = ((2 * j - 1) * z * p1 - (j - 1) * p2) / j;
      }
      dp = n * (z * p0 - p1) / (z * z - 1);
    }
    const long double wt = 1.0L / ((1 - z * z) * dp * dp);
    x[n - 1 - i] = double((1 + z) / 2);
    x[i] = double((1 - z) / 2);
    w[n - 1 - i] = double(wt);
    w[i] = double(wt);
  }
  if (n % 2 == 1) x[n / 2] = 0.5;
}

double lagrange(const std::vector<double> &nodes, int i, double x) {
  double v = 1.;
  for (int m = 0; m < int(nodes.size()); ++m)
    if (m != i) v *= (x - nodes[m]) / (nodes[i] - nodes[m]);
  return v;
}
double dlagrange(const std::vector<double> &nodes, int i, double x) {
  double s = 0.;
  const int n = int(nodes.size());
  for (int k = 0; k < n; ++k) {
    if (k == i) continue;
    double v = 1. / (nodes[i] - nodes[k]);
    for (int m = 0; m < n; ++m)
      if (m != i && m != k) v *= (x - nodes[m]) / (nodes[i] - nodes[m]);
    s += v;
  }
  return s;
}

static double zap(double v) { return std::abs(v) < 1e-14 ? 0. : v; }

void fill_desc(eg_desc &d, int nx, int ny, int k, double alpha_deg, double gamma, double safety) {
  if (k < 0 || k > 8) throw std::invalid_argument("k must be in 0..8");
  if (nx < 2 || ny < 2) throw std::invalid_argument("nx, ny must be >= 2");
  if (!(alpha_deg > 0 && alpha_deg < 90)) throw std::invalid_argument("0 < alpha < 90 required");
  d = eg_desc{};
  const int q = k + 1, p = q * q;
  d.nx = nx;
  d.ny = ny;
  d.k = k;
  d.gamma = gamma;
  d.safety = safety;
  d.alpha = alpha_deg * kPi / 180;
  d.lx = 2 / std::cos(d.alpha);
  d.ly = 2 / std::sin(d.alpha);
  d.hx = d.lx / nx;
  d.hy = d.ly / ny;
  d.area = d.hx * d.hy;
  std::vector<double> x, w;
  gauss_legendre(q, x, w);
  for (int j = 0; j < q; ++j) {
    d.ew[j] = w[j];
    d.ex[j] = x[j];
  }
  for (int iy = 0; iy < q; ++iy)
    for (int ix = 0; ix < q; ++ix) {
      const int i = iy * q + ix;
      d.w[i] = w[ix] * w[iy];
      d.mass[i] = d.w[i];
      d.inv_mass[i] = 1.0 / d.w[i];
      d.tensor_node[i] = i;
    }
  for (int a = 0; a < q; ++a)
    for (int i = 0; i < q; ++i) {
      const double dv = dlagrange(x, i, x[a]) * lagrange(x, 0, x[0]);
      d.tensor_dx[a * q + i] = std::abs(dv) < 1e-14 ? 0. : dv / d.hx;
      const double dy = lagrange(x, 0, x[0]) * dlagrange(x, i, x[a]);
      d.tensor_dy[a * q + i] = std::abs(dy) < 1e-14 ? 0. : dy / d.hy;
    }
  for (int s = 0; s < 4; ++s)
    for (int j = 0; j < q; ++j)
      for (int l = 0; l < q; ++l) {
        double v;
        if (s < 2) {
          v = lagrange(x, l, double(s)) * lagrange(x, j, x[j]);
        } else {
          v = lagrange(x, j, x[j]) * lagrange(x, l, double(s - 2));
        }
        d.face_basis[(s * q + j) * q + l] = zap(v);
      }
}

// ------------------------------------------------------------ exact wave
void exact(double gamma, double x, double y, double time, double alpha, double out[4]) {
  const double gm1 = gamma - 1.;
  const double drift = (3. - gamma) / 2., amplitude = (gamma + 1.) / 4.;
  if (!(time >= 0 && time * kPi * amplitude < 1))
    throw std::runtime_error("Exact solution requires T < 4/((gamma+1)*pi)");
  double phase = std::cos(alpha) * x + std::sin(alpha) * y;
  phase -= 2 * std::floor((phase + 1) / 2);
  phase -= time * drift;
  phase -= 2 * std::floor((phase + 1) / 2);
  double lo = phase - time * amplitude, hi = phase + time * amplitude, z = phase;
  for (int i = 0; i < 80; i++) {
    const double r = z + time * amplitude * std::sin(kPi * z) - phase;
    if (std::abs(r) < 2e-15) break;
    if (r > 0) {
      hi = z;
    } else {
      lo = z;
    }
    const double q = z - r / (1 + time * amplitude * kPi * std::cos(kPi * z));
    z = (q >= lo && q <= hi) ? q : .5 * (lo + hi);
  }
  const double jm = std::sin(kPi * z), v = 1 + .5 * jm;
  const double sound = gm1 * (2. - jm) / 4.;
  const double rho = std::pow(sound * sound / gamma, 1. / gm1);
  const double pressure = std::pow(rho, gamma);
  out[0] = rho;
  out[1] = rho * v * std::cos(alpha);
  out[2] = rho * v * std::sin(alpha);
  out[3] = pressure / gm1 + .5 * rho * v * v;
}

// Lower-left corner of cell e from the shifted Cartesian mesh, evaluated as
// the element-centre transform minus half a cell (src/problem.cpp:48-72).
static void cell_origin(const eg_desc &d, int e, double &ox, double &oy) {
  const int ix = e % d.nx, iy = e / d.nx;
  auto vx = [&](int i) { return d.lx * i / d.nx - .5 * d.lx; };
  auto vy = [&](int j) { return d.ly * j / d.ny - .5 * d.ly; };
  const double x0 = vx(ix), x1 = vx(ix + 1), y0 = vy(iy), y1 = vy(iy + 1);
  const double cx = x0 * .25 + x1 * .25 + x1 * .25 + x0 * .25;
  const double cy = y0 * .25 + y0 * .25 + y1 * .25 + y1 * .25;
  ox = cx - .5 * d.hx;
  oy = cy - .5 * d.hy;
}

struct FineRule {
  std::vector<double> x, y, w;
};
// Square Gauss-Legendre rule of order max(24, 2k+8): 13 x 13 points for k <= 8.
static FineRule fine_rule(int k) {
  const int order = std::max(24, 2 * k + 8);
  const int n = (order | 1) / 2 + 1;
  std::vector<double> x, w;
  gauss_legendre(n, x, w);
  FineRule r;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      r.x.push_back(x[i]);
      r.y.push_back(x[j]);
      r.w.push_back(w[i] * w[j]);
    }
  return r;
}

static void shape(const std::vector<double> &nodes, double x, double y, std::vector<double> &sh) {
  const int q = int(nodes.size());
  sh.resize(q * q);
  for (int j = 0; j < q; ++j) {
    const double ly = lagrange(nodes, j, y);
    for (int i = 0; i < q; ++i) sh[j * q + i] = lagrange(nodes, i, x) * ly;
  }
}

void initial(const eg_desc &d, std::vector<double> &u) {
  const int q = d.k + 1, p = q * q, m = 4 * p, n = d.nx * d.ny;
  std::vector<double> nodes(d.ex, d.ex + q);
  u.assign((size_t)n * m, 0.);
  const FineRule r = fine_rule(d.k);
  const int nq = int(r.w.size());
  std::vector<std::vector<double>> shapes(nq);
  for (int qp = 0; qp < nq; ++qp) shape(nodes, r.x[qp], r.y[qp], shapes[qp]);
  for (int e = 0; e < n; ++e) {
    double ox, oy;
    cell_origin(d, e, ox, oy);
    double *ue = u.data() + (size_t)e * m;
    for (int qp = 0; qp < nq; ++qp) {
      double v[4];
      exact(d.gamma, ox + d.hx * r.x[qp], oy + d.hy * r.y[qp], 0, d.alpha, v);
      const std::vector<double> &sh = shapes[qp];
      for (int i = 0; i < p; ++i)
        for (int c = 0; c < 4; ++c) ue[4 * i + c] += r.w[qp] * sh[i] * v[c];
    }
    for (int i = 0; i < p; ++i)
      for (int c = 0; c < 4; ++c) ue[4 * i + c] *= d.inv_mass[i];
  }
}

void errors(const eg_desc &d, const double *u, double time, double out[4]) {
  const int q = d.k + 1, p = q * q, m = 4 * p, n = d.nx * d.ny;
  std::vector<double> nodes(d.ex, d.ex + q);
  const FineRule r = fine_rule(d.k);
  const int nq = int(r.w.size());
  std::vector<std::vector<double>> shapes(nq);
  for (int qp = 0; qp < nq; ++qp) shape(nodes, r.x[qp], r.y[qp], shapes[qp]);
  double a[4] = {0, 0, 0, 0};
  for (int e = 0; e < n; ++e) {
    double ox, oy;
    cell_origin(d, e, ox, oy);
    const double *ue = u + (size_t)e * m;
    for (int qp = 0; qp < nq; ++qp) {
      double v[4];
      exact(d.gamma, ox + d.hx * r.x[qp], oy + d.hy * r.y[qp], time, d.alpha, v);
      const std::vector<double> &sh = shapes[qp];
      for (int c = 0; c < 4; ++c) {
        double z = 0;
        for (int i = 0; i < p; ++i) z += sh[i] * ue[4 * i + c];
        a[c] += d.area * r.w[qp] * (z - v[c]) * (z - v[c]);
      }
    }
  }
  for (int c = 0; c < 4; ++c) out[c] = std::sqrt(a[c]);
}

void integral(const eg_desc &d, const double *u, double out[4]) {
  const int q = d.k + 1, p = q * q, m = 4 * p, n = d.nx * d.ny;
  double a[4] = {0, 0, 0, 0};
  for (int e = 0; e < n; ++e)
    for (int i = 0; i < p; ++i)
      for (int c = 0; c < 4; ++c) a[c] += d.area * d.w[i] * u[(size_t)e * m + 4 * i + c];
  for (int c = 0; c < 4; ++c) out[c] = a[c];
}

void differences(const eg_desc &d, const double *u, const double *v, double out[4]) {
  const int q = d.k + 1, p = q * q, m = 4 * p, n = d.nx * d.ny;
  std::vector<double> nodes(d.ex, d.ex + q);
  const FineRule r = fine_rule(d.k);
  const int nq = int(r.w.size());
  std::vector<std::vector<double>> shapes(nq);
  for (int qp = 0; qp < nq; ++qp) shape(nodes, r.x[qp], r.y[qp], shapes[qp]);
  double a[4] = {0, 0, 0, 0};
  for (int e = 0; e < n; ++e)
    for (int qp = 0; qp < nq; ++qp)
      for (int c = 0; c < 4; ++c) {
        double diff = 0.;
        for (int i = 0; i < p; ++i)
          diff += shapes[qp][i] * (u[(size_t)e * m + 4 * i + c] - v[(size_t)e * m + 4 * i + c]);
        a[c] += d.area * r.w[qp] * diff * diff;
      }
  for (int c = 0; c < 4; ++c) out[c] = std::sqrt(a[c]);
}

// The mesh is the reference's MakeCartesian2D(nx, ny, QUADRILATERAL, lx, ly) in row-major order
// (no space-filling-curve reordering), shifted to the centred box (src/problem.cpp:47-51): vertex
// (i, j) is i + j (nx + 1) at (lx i / nx - lx / 2, ly j / ny - ly / 2),
// element (i, j) is i + j nx with its corners counter-clockwise from the lower left, and the
// boundary segments run bottom (attribute 1), right (2), top (3), left (4), each oriented with the
// domain on its left. The grid functions hold u[e m + 4 i + c] at DOF e p + i, the element-local
// numbering of an L2 space (FiniteElementSpace::GetElementDofs).
bool save_solution(const eg_desc &d, const double *u, const std::string &prefix) {
  const int nx = d.nx, ny = d.ny, q = d.k + 1, p = q * q, m = 4 * p, n = nx * ny;
  auto vid = [nx](int i, int j) { return i + j * (nx + 1); };
  {
    std::ofstream ms(prefix + ".mesh");
    if (!ms) return false;
    ms << "MFEM mesh v1.0\n\n"
          "#\n# MFEM Geometry Types (see mesh/geom.hpp):\n#\n# POINT       = 0\n"
          "# SEGMENT     = 1\n# TRIANGLE    = 2\n# SQUARE      = 3\n# TETRAHEDRON = 4\n"
          "# CUBE        = 5\n# PRISM       = 6\n# PYRAMID     = 7\n#\n\n"
       << "dimension\n2\n\nelements\n" << n << '\n';
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        ms << "1 3 " << vid(i, j) << ' ' << vid(i + 1, j) << ' ' << vid(i + 1, j + 1) << ' '
           << vid(i, j + 1) << '\n';
    ms << "\nboundary\n" << 2 * (nx + ny) << '\n';
    for (int i = 0; i < nx; ++i) ms << "1 1 " << vid(i + 1, 0) << ' ' << vid(i, 0) << '\n';
    for (int j = 0; j < ny; ++j) ms << "2 1 " << vid(nx, j + 1) << ' ' << vid(nx, j) << '\n';
    for (int i = 0; i < nx; ++i) ms << "3 1 " << vid(i, ny) << ' ' << vid(i + 1, ny) << '\n';
    for (int j = 0; j < ny; ++j) ms << "4 1 " << vid(0, j) << ' ' << vid(0, j + 1) << '\n';
    ms << "\nvertices\n" << (nx + 1) * (ny + 1) << "\n2\n" << std::setprecision(17);
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i)
        ms << d.lx * i / nx - .5 * d.lx << ' ' << d.ly * j / ny - .5 * d.ly << '\n';
    if (!ms) return false;
  }
  static const char *names[] = {"rho", "rhou", "rhov", "energy"};
  for (int c = 0; c < 4; ++c) {
    std::ofstream fs(prefix + "_" + names[c] + ".gf");
    if (!fs) return false;
    fs << "FiniteElementSpace\nFiniteElementCollection: L2_2D_P" << d.k
       << "\nVDim: 1\nOrdering: 0\n\n" << std::setprecision(17);
    for (int e = 0; e < n; ++e)
      for (int i = 0; i < p; ++i) fs << u[(size_t)e * m + 4 * i + c] << '\n';
    if (!fs) return false;
  }
  std::ofstream cs(prefix + "_coefficients.csv");
  if (!cs) return false;
  cs << "element,node,rho,rhou,rhov,energy\n" << std::setprecision(17);
  for (int e = 0; e < n; ++e)
    for (int i = 0; i < p; ++i) {
      cs << e << ',' << i;
      for (int c = 0; c < 4; ++c) cs << ',' << u[(size_t)e * m + 4 * i + c];
      cs << '\n';
    }
  return bool(cs);
}

}  // namespace host
}  // namespace eg
