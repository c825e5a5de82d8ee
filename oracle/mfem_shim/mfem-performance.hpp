// MFEM-subset shim: test infrastructure for the oracle only.
//
// The reference solver (YueWu2002/mfem_euler2d_cpp) is written against MFEM
// (pinned in its RESULTS.md:258-259 as "MFEM commit 54d7f64513"), which is not
// vendored with it and is not installed here. This header restates, in our own
// code, the published semantics of exactly the MFEM symbols the reference uses
// (include/euler.hpp:8 and the call sites listed beside each class below), so
// that the UNMODIFIED reference sources compile into the CPU oracle binary
// `oracle/_ref/euler2d_ref`. Nothing in the CUDA product links this file.
//
// Conventions restated from MFEM's public documentation:
//  * Vector / DenseMatrix hold real_t=double; DenseMatrix is column-major.
//  * Gauss-Legendre rules on [0,1]; a segment rule of order o has o/2+1 points;
//    square rules are tensor products with x running fastest.
//  * L2 Qk elements with Gauss-Legendre nodes use lexicographic node order
//    (x fastest); shape functions are Lagrange polynomials at the nodes.
//  * LUFactors: right-looking LU with row partial pivoting (first maximum wins),
//    unit lower L, pivots stored as the row swapped with each step.
//  * Mesh::MakeCartesian2D numbers elements row-major (x fastest) when
//    sfc_ordering is false.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <iomanip>
#include <map>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace mfem {
using real_t = double;

// ----------------------------------------------------------------- Array<T>
template <typename T>
class Array {
  std::vector<T> v_;

 public:
  Array() = default;
  explicit Array(int n) : v_(n) {}
  int Size() const { return int(v_.size()); }
  void SetSize(int n) { v_.resize(n); }
  T &operator[](int i) { return v_[i]; }
  const T &operator[](int i) const { return v_[i]; }
  T *GetData() { return v_.data(); }
};

// ------------------------------------------------------------------- Vector
// Owning or non-owning (view) dense vector. SetSize keeps the storage when the
// requested size fits the current capacity, so views stay views.
class Vector {
  double *data_ = nullptr;
  int size_ = 0, capacity_ = 0;
  bool own_ = false;

  void release() {
    if (own_) delete[] data_;
    data_ = nullptr;
    size_ = capacity_ = 0;
    own_ = false;
  }

 public:
  Vector() = default;
  explicit Vector(int s) { SetSize(s); }
  Vector(double *d, int s) : data_(d), size_(s), capacity_(s), own_(false) {}
  Vector(const Vector &v) {
    SetSize(v.size_);
    if (size_) std::memcpy(data_, v.data_, sizeof(double) * size_);
  }
  Vector(Vector &&v) noexcept
      : data_(v.data_), size_(v.size_), capacity_(v.capacity_), own_(v.own_) {
    v.data_ = nullptr;
    v.size_ = v.capacity_ = 0;
    v.own_ = false;
  }
  ~Vector() { release(); }
  Vector &operator=(const Vector &v) {
    if (this != &v) {
      SetSize(v.size_);
      if (size_) std::memmove(data_, v.data_, sizeof(double) * size_);
    }
    return *this;
  }
  Vector &operator=(Vector &&v) noexcept {
    if (this != &v) {
      release();
      data_ = v.data_;
      size_ = v.size_;
      capacity_ = v.capacity_;
      own_ = v.own_;
      v.data_ = nullptr;
      v.size_ = v.capacity_ = 0;
      v.own_ = false;
    }
    return *this;
  }
  Vector &operator=(double c) {
    for (int i = 0; i < size_; ++i) data_[i] = c;
    return *this;
  }
  void SetSize(int s) {
    if (s == size_) return;
    if (s <= capacity_) {
      size_ = s;
      return;
    }
    double *fresh = new double[s]();
    release();
    data_ = fresh;
    size_ = capacity_ = s;
    own_ = true;
  }
  int Size() const { return size_; }
  double *GetData() const { return data_; }
  double &operator[](int i) { return data_[i]; }
  const double &operator[](int i) const { return data_[i]; }
  double &operator()(int i) { return data_[i]; }
  const double &operator()(int i) const { return data_[i]; }
  Vector &operator+=(const Vector &v) {
    for (int i = 0; i < size_; ++i) data_[i] += v.data_[i];
    return *this;
  }
  Vector &operator-=(const Vector &v) {
    for (int i = 0; i < size_; ++i) data_[i] -= v.data_[i];
    return *this;
  }
  Vector &operator+=(double c) {
    for (int i = 0; i < size_; ++i) data_[i] += c;
    return *this;
  }
  Vector &operator*=(double c) {
    for (int i = 0; i < size_; ++i) data_[i] *= c;
    return *this;
  }
  // this += a*v
  Vector &Add(double a, const Vector &v) {
    for (int i = 0; i < size_; ++i) data_[i] += a * v.data_[i];
    return *this;
  }
  double Norml2() const {
    double s = 0.;
    for (int i = 0; i < size_; ++i) s += data_[i] * data_[i];
    return std::sqrt(s);
  }
  double Normlinf() const {
    double s = 0.;
    for (int i = 0; i < size_; ++i) s = std::max(s, std::abs(data_[i]));
    return s;
  }
};

// -------------------------------------------------- fixed-size TVector/TMatrix
// Aggregates with inline storage; TMatrix is column-major.
template <int S, typename data_t = real_t, bool align = false>
struct TVector {
  data_t data[S];
  data_t &operator[](int i) { return data[i]; }
  const data_t &operator[](int i) const { return data[i]; }
  void Set(data_t d) {
    for (int i = 0; i < S; ++i) data[i] = d;
  }
};
template <int N1, int N2, typename data_t = real_t, bool align = false>
struct TMatrix : public TVector<N1 * N2, data_t, align> {
  data_t &operator()(int i, int j) { return this->data[i + N1 * j]; }
  const data_t &operator()(int i, int j) const { return this->data[i + N1 * j]; }
};

// --------------------------------------------------------------- DenseMatrix
class DenseMatrix {
  double *data_ = nullptr;
  int h_ = 0, w_ = 0, capacity_ = 0;
  bool own_ = false;

  void release() {
    if (own_) delete[] data_;
    data_ = nullptr;
    capacity_ = 0;
    own_ = false;
  }

 public:
  DenseMatrix() = default;
  explicit DenseMatrix(int s) { SetSize(s, s); }
  DenseMatrix(int h, int w) { SetSize(h, w); }
  DenseMatrix(double *d, int h, int w) : data_(d), h_(h), w_(w), capacity_(h * w), own_(false) {}
  DenseMatrix(const DenseMatrix &m) {
    SetSize(m.h_, m.w_);
    if (h_ * w_) std::memcpy(data_, m.data_, sizeof(double) * h_ * w_);
  }
  DenseMatrix(DenseMatrix &&m) noexcept
      : data_(m.data_), h_(m.h_), w_(m.w_), capacity_(m.capacity_), own_(m.own_) {
    m.data_ = nullptr;
    m.h_ = m.w_ = m.capacity_ = 0;
    m.own_ = false;
  }
  ~DenseMatrix() { release(); }
  DenseMatrix &operator=(const DenseMatrix &m) {
    if (this != &m) {
      SetSize(m.h_, m.w_);
      if (h_ * w_) std::memmove(data_, m.data_, sizeof(double) * h_ * w_);
    }
    return *this;
  }
  DenseMatrix &operator=(DenseMatrix &&m) noexcept {
    if (this != &m) {
      release();
      data_ = m.data_;
      h_ = m.h_;
      w_ = m.w_;
      capacity_ = m.capacity_;
      own_ = m.own_;
      m.data_ = nullptr;
      m.h_ = m.w_ = m.capacity_ = 0;
      m.own_ = false;
    }
    return *this;
  }
  DenseMatrix &operator=(double c) {
    for (int i = 0; i < h_ * w_; ++i) data_[i] = c;
    return *this;
  }
  DenseMatrix &operator*=(double c) {
    for (int i = 0; i < h_ * w_; ++i) data_[i] *= c;
    return *this;
  }
  // Storage is reused when it fits; a new allocation starts zeroed.
  void SetSize(int h, int w) {
    if (h == h_ && w == w_) return;
    if (h * w > capacity_) {
      double *fresh = new double[size_t(h) * w]();
      release();
      data_ = fresh;
      capacity_ = h * w;
      own_ = true;
    }
    h_ = h;
    w_ = w;
  }
  void SetSize(int s) { SetSize(s, s); }
  int Height() const { return h_; }
  int Width() const { return w_; }
  double *GetData() const { return data_; }
  double &operator()(int i, int j) { return data_[i + size_t(h_) * j]; }
  const double &operator()(int i, int j) const { return data_[i + size_t(h_) * j]; }
  // y = A x
  void Mult(const double *x, double *y) const {
    for (int i = 0; i < h_; ++i) y[i] = 0.;
    for (int j = 0; j < w_; ++j) {
      const double xj = x[j];
      const double *col = data_ + size_t(h_) * j;
      for (int i = 0; i < h_; ++i) y[i] += col[i] * xj;
    }
  }
  void Mult(const Vector &x, Vector &y) const { Mult(x.GetData(), y.GetData()); }
  // y = A^T x
  void MultTranspose(const double *x, double *y) const {
    for (int j = 0; j < w_; ++j) {
      const double *col = data_ + size_t(h_) * j;
      double s = 0.;
      for (int i = 0; i < h_; ++i) s += col[i] * x[i];
      y[j] = s;
    }
  }
  // y += a A x
  void AddMult_a(double a, const Vector &x, Vector &y) const {
    const double *xp = x.GetData();
    double *yp = y.GetData();
    for (int j = 0; j < w_; ++j) {
      const double xj = a * xp[j];
      const double *col = data_ + size_t(h_) * j;
      for (int i = 0; i < h_; ++i) yp[i] += col[i] * xj;
    }
  }
  // this += c A
  void Add(double c, const DenseMatrix &a) {
    for (int i = 0; i < h_ * w_; ++i) data_[i] += c * a.data_[i];
  }
};

// C += a A B
inline void AddMult_a(double a, const DenseMatrix &A, const DenseMatrix &B, DenseMatrix &C) {
  const int m = C.Height(), n = C.Width(), kk = A.Width();
  for (int j = 0; j < n; ++j) {
    for (int l = 0; l < kk; ++l) {
      const double blj = a * B(l, j);
      for (int i = 0; i < m; ++i) C(i, j) += A(i, l) * blj;
    }
  }
}

// ---------------------------------------------------------------- LUFactors
// In-place LU of a column-major m x m matrix with row partial pivoting.
class LUFactors {
 public:
  double *data;
  int *ipiv;
  LUFactors() : data(nullptr), ipiv(nullptr) {}
  LUFactors(double *d, int *p) : data(d), ipiv(p) {}

  bool Factor(int m, double tol = 0.0) {
    double *a = data;
    for (int i = 0; i < m; ++i) {
      int piv = i;
      double best = std::abs(a[i + i * m]);
      for (int j = i + 1; j < m; ++j) {
        const double b = std::abs(a[j + i * m]);
        if (b > best) {
          best = b;
          piv = j;
        }
      }
      ipiv[i] = piv;
      if (piv != i) {
        for (int j = 0; j < m; ++j) std::swap(a[i + j * m], a[piv + j * m]);
      }
      if (!(std::abs(a[i + i * m]) > tol)) return false;
      const double inv = 1.0 / a[i + i * m];
      for (int j = i + 1; j < m; ++j) a[j + i * m] *= inv;
      for (int k = i + 1; k < m; ++k) {
        const double aik = a[i + k * m];
        for (int j = i + 1; j < m; ++j) a[j + k * m] -= aik * a[j + i * m];
      }
    }
    return true;
  }
  // X <- A^{-1} X for n right-hand sides (X is m x n, column-major).
  void Solve(int m, int n, double *X) const {
    const double *a = data;
    for (int k = 0; k < n; ++k) {
      double *x = X + size_t(k) * m;
      for (int i = 0; i < m; ++i) std::swap(x[i], x[ipiv[i]]);
      for (int j = 0; j < m; ++j) {
        const double xj = x[j];
        for (int i = j + 1; i < m; ++i) x[i] -= a[i + j * m] * xj;
      }
      for (int j = m - 1; j >= 0; --j) {
        const double xj = x[j] / a[j + j * m];
        x[j] = xj;
        for (int i = 0; i < j; ++i) x[i] -= a[i + j * m] * xj;
      }
    }
  }
  // X <- X A^{-1} (X is n x m, column-major).
  void RightSolve(int m, int n, double *X) const {
    const double *a = data;
    // X <- X U^{-1}
    for (int k = 0; k < m; ++k) {
      double *xk = X + size_t(k) * n;
      for (int j = 0; j < k; ++j) {
        const double ujk = a[j + k * m];
        const double *xj = X + size_t(j) * n;
        for (int i = 0; i < n; ++i) xk[i] -= xj[i] * ujk;
      }
      const double inv = 1.0 / a[k + k * m];
      for (int i = 0; i < n; ++i) xk[i] *= inv;
    }
    // X <- X L^{-1}
    for (int k = m - 1; k >= 0; --k) {
      double *xk = X + size_t(k) * n;
      for (int j = k + 1; j < m; ++j) {
        const double ljk = a[j + k * m];
        const double *xj = X + size_t(j) * n;
        for (int i = 0; i < n; ++i) xk[i] -= xj[i] * ljk;
      }
    }
    // X <- X P (undo the row interchanges as column interchanges, last first)
    for (int k = m - 1; k >= 0; --k) {
      if (ipiv[k] != k) {
        double *xa = X + size_t(k) * n, *xb = X + size_t(ipiv[k]) * n;
        for (int i = 0; i < n; ++i) std::swap(xa[i], xb[i]);
      }
    }
  }
};

// ---------------------------------------------------------------- Operator
class Operator {
 protected:
  int height, width;

 public:
  explicit Operator(int s = 0) : height(s), width(s) {}
  Operator(int h, int w) : height(h), width(w) {}
  virtual ~Operator() = default;
  int Height() const { return height; }
  int Width() const { return width; }
  virtual void Mult(const Vector &x, Vector &y) const = 0;
};
class Solver : public Operator {
 public:
  using Operator::Operator;
};

// -------------------------------------------------------- DenseMatrixInverse
class DenseMatrixInverse : public Solver {
  const DenseMatrix *source_ = nullptr;
  DenseMatrix lu_;
  std::vector<int> piv_;

 public:
  explicit DenseMatrixInverse(const DenseMatrix &m) : Solver(m.Height()), source_(&m) { Factor(); }
  explicit DenseMatrixInverse(const DenseMatrix *m) : Solver(m->Height()), source_(m) {}
  void Factor() {
    lu_ = *source_;
    height = width = lu_.Height();
    piv_.assign(height, 0);
    LUFactors f(lu_.GetData(), piv_.data());
    if (!f.Factor(height)) throw std::runtime_error("DenseMatrixInverse: singular matrix");
  }
  void GetInverseMatrix(DenseMatrix &inv) const {
    const int m = height;
    inv.SetSize(m, m);
    inv = 0.;
    for (int i = 0; i < m; ++i) inv(i, i) = 1.;
    LUFactors f(const_cast<double *>(lu_.GetData()), const_cast<int *>(piv_.data()));
    f.Solve(m, m, inv.GetData());
  }
  void Mult(const Vector &x, Vector &y) const override {
    y.SetSize(height);
    std::copy_n(x.GetData(), height, y.GetData());
    LUFactors f(const_cast<double *>(lu_.GetData()), const_cast<int *>(piv_.data()));
    f.Solve(height, 1, y.GetData());
  }
};

// -------------------------------------------------------------- SparseMatrix
// CSR with sorted columns. The (n) constructor collects entries until
// Finalize(), summing duplicates.
class SparseMatrix : public Operator {
  std::vector<int> I_, J_;
  std::vector<double> A_;
  std::vector<std::map<int, double>> rows_;
  bool finalized_ = true;

 public:
  explicit SparseMatrix(int n) : Operator(n), rows_(n), finalized_(false) {}
  SparseMatrix(int *i, int *j, double *data, int h, int w) : Operator(h, w) {
    const int nnz = i[h];
    I_.assign(i, i + h + 1);
    J_.assign(j, j + nnz);
    A_.assign(data, data + nnz);
    delete[] i;
    delete[] j;
    delete[] data;
  }
  void Add(int i, int j, double v) {
    if (finalized_) throw std::runtime_error("SparseMatrix::Add after Finalize");
    rows_[i][j] += v;
  }
  void Finalize() {
    if (finalized_) return;
    I_.assign(1, 0);
    for (auto &r : rows_) {
      for (auto &e : r) {
        J_.push_back(e.first);
        A_.push_back(e.second);
      }
      I_.push_back(int(J_.size()));
    }
    rows_.clear();
    finalized_ = true;
  }
  int NumNonZeroElems() const { return finalized_ ? I_.back() : 0; }
  const int *GetI() const { return I_.data(); }
  const int *GetJ() const { return J_.data(); }
  const double *GetData() const { return A_.data(); }
  void Mult(const Vector &x, Vector &y) const override {
    y.SetSize(height);
    for (int r = 0; r < height; ++r) {
      double s = 0.;
      for (int k = I_[r]; k < I_[r + 1]; ++k) s += A_[k] * x[J_[k]];
      y[r] = s;
    }
  }
  void ToDenseMatrix(DenseMatrix &d) const {
    d.SetSize(height, width);
    d = 0.;
    for (int r = 0; r < height; ++r)
      for (int k = I_[r]; k < I_[r + 1]; ++k) d(r, J_[k]) += A_[k];
  }
};

// ------------------------------------------------------------------ BlockILU
// Block ILU(0) on the block sparsity pattern of a CSR matrix, natural order,
// with explicit inverses of the factored diagonal blocks.
class BlockILU : public Solver {
 public:
  enum class Reordering { MINIMUM_DISCARDED_FILL, NONE };

 private:
  int b_ = 1, nb_ = 0;
  std::vector<int> row_, col_, diag_;
  std::vector<DenseMatrix> blk_;
  std::vector<DenseMatrix> dinv_;

  int find(int i, int j) const {
    auto it = std::lower_bound(col_.begin() + row_[i], col_.begin() + row_[i + 1], j);
    return (it != col_.begin() + row_[i + 1] && *it == j) ? int(it - col_.begin()) : -1;
  }

 public:
  BlockILU(const SparseMatrix &a, int block, Reordering reordering = Reordering::NONE, int k_fill = 0)
      : Solver(a.Height()), b_(block) {
    if (reordering != Reordering::NONE || k_fill != 0)
      throw std::runtime_error("BlockILU shim supports only NONE ordering with zero fill");
    nb_ = a.Height() / b_;
    const int *I = a.GetI(), *J = a.GetJ();
    const double *A = a.GetData();
    std::vector<std::vector<int>> pat(nb_);
    for (int r = 0; r < a.Height(); ++r)
      for (int k = I[r]; k < I[r + 1]; ++k) pat[r / b_].push_back(J[k] / b_);
    row_.assign(1, 0);
    for (int i = 0; i < nb_; ++i) {
      pat[i].push_back(i);
      std::sort(pat[i].begin(), pat[i].end());
      pat[i].erase(std::unique(pat[i].begin(), pat[i].end()), pat[i].end());
      for (int j : pat[i]) {
        if (j == i) diag_.push_back(int(col_.size()));
        col_.push_back(j);
      }
      row_.push_back(int(col_.size()));
    }
    blk_.assign(col_.size(), DenseMatrix(b_));
    for (auto &m : blk_) m = 0.;
    for (int r = 0; r < a.Height(); ++r)
      for (int k = I[r]; k < I[r + 1]; ++k) {
        const int id = find(r / b_, J[k] / b_);
        blk_[id](r % b_, J[k] % b_) += A[k];
      }
    dinv_.resize(nb_);
    DenseMatrix tmp(b_);
    for (int i = 0; i < nb_; ++i) {
      for (int ik = row_[i]; ik < diag_[i]; ++ik) {
        const int k = col_[ik];
        tmp = 0.;
        AddMult_a(1.0, blk_[ik], dinv_[k], tmp);
        blk_[ik] = tmp;
        for (int kj = diag_[k] + 1; kj < row_[k + 1]; ++kj) {
          const int ij = find(i, col_[kj]);
          if (ij >= 0) AddMult_a(-1.0, blk_[ik], blk_[kj], blk_[ij]);
        }
      }
      DenseMatrixInverse inv(blk_[diag_[i]]);
      inv.GetInverseMatrix(dinv_[i]);
    }
  }
  void Mult(const Vector &b, Vector &x) const override {
    x.SetSize(height);
    Vector y(height);
    for (int i = 0; i < nb_; ++i) {
      Vector yi(y.GetData() + i * b_, b_);
      std::copy_n(b.GetData() + i * b_, b_, yi.GetData());
      for (int ij = row_[i]; ij < diag_[i]; ++ij) {
        Vector yj(y.GetData() + col_[ij] * b_, b_);
        blk_[ij].AddMult_a(-1.0, yj, yi);
      }
    }
    for (int i = nb_ - 1; i >= 0; --i) {
      Vector yi(y.GetData() + i * b_, b_);
      for (int ij = diag_[i] + 1; ij < row_[i + 1]; ++ij) {
        Vector xj(x.GetData() + col_[ij] * b_, b_);
        blk_[ij].AddMult_a(-1.0, xj, yi);
      }
      Vector xi(x.GetData() + i * b_, b_);
      dinv_[i].Mult(yi, xi);
    }
  }
};

// MDF ordering is an MFEM-internal routine; it is not restated here.
inline void MinimumDiscardedFillOrdering(SparseMatrix &, Array<int> &) {
  throw std::runtime_error("MDF ordering is unavailable in the MFEM-subset oracle shim");
}

// ---------------------------------------------------------- geometry/enums
struct Geometry {
  enum Type { POINT = 0, SEGMENT = 1, TRIANGLE = 2, SQUARE = 3 };
};
struct Element {
  enum Type { POINT, SEGMENT, TRIANGLE, QUADRILATERAL };
};
struct BasisType {
  enum { GaussLegendre = 0, GaussLobatto = 1 };
};

// ------------------------------------------------------- integration rules
struct IntegrationPoint {
  double x = 0, y = 0, z = 0, weight = 0;
  void Set2(double x1, double x2) {
    x = x1;
    y = x2;
  }
};
class IntegrationRule {
  std::vector<IntegrationPoint> pts_;
  int order_ = 0;

 public:
  IntegrationRule() = default;
  IntegrationRule(std::vector<IntegrationPoint> p, int order) : pts_(std::move(p)), order_(order) {}
  int GetNPoints() const { return int(pts_.size()); }
  int GetOrder() const { return order_; }
  IntegrationPoint &IntPoint(int i) { return pts_[i]; }
  const IntegrationPoint &IntPoint(int i) const { return pts_[i]; }
};

namespace shim_detail {
// Gauss-Legendre nodes/weights on [0,1], ascending, mirrored for exact symmetry.
// Newton iteration on the three-term Legendre recurrence in extended precision.
inline void GaussLegendre(int n, std::vector<double> &x, std::vector<double> &w) {
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
    // z > 0 is the i-th largest root; map to [0,1] (ascending index n-1-i).
    const long double wt = 1.0L / ((1 - z * z) * dp * dp);  // = (2/((1-z^2)P'^2))/2
    x[n - 1 - i] = double((1 + z) / 2);
    x[i] = double((1 - z) / 2);
    w[n - 1 - i] = double(wt);
    w[i] = double(wt);
  }
  if (n % 2 == 1) x[n / 2] = 0.5;
}
}  // namespace shim_detail

class IntegrationRules {
  std::map<std::pair<int, int>, std::unique_ptr<IntegrationRule>> cache_;

 public:
  const IntegrationRule &Get(int geom, int order) {
    auto key = std::make_pair(geom, order);
    auto it = cache_.find(key);
    if (it != cache_.end()) return *it->second;
    const int n = (order | 1) / 2 + 1;
    std::vector<double> x, w;
    shim_detail::GaussLegendre(n, x, w);
    std::vector<IntegrationPoint> pts;
    if (geom == Geometry::SEGMENT) {
      for (int i = 0; i < n; ++i) {
        IntegrationPoint p;
        p.x = x[i];
        p.weight = w[i];
        pts.push_back(p);
      }
    } else if (geom == Geometry::SQUARE) {
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          IntegrationPoint p;
          p.x = x[i];
          p.y = x[j];
          p.weight = w[i] * w[j];
          pts.push_back(p);
        }
    } else {
      throw std::runtime_error("IntRules shim: unsupported geometry");
    }
    auto &slot = cache_[key];
    slot = std::make_unique<IntegrationRule>(std::move(pts), 2 * n - 1);
    return *slot;
  }
};
inline IntegrationRules IntRules;

// ----------------------------------------------------------- finite elements
// Lagrange basis at Gauss-Legendre nodes: segment (dim 1) or tensor square
// (dim 2, lexicographic, x fastest).
class FiniteElement {
  int dim_ = 1, order_ = 0, n1_ = 1;
  std::vector<double> nodes_;

  double lagrange(int i, double x) const {
    double v = 1.;
    for (int m = 0; m < n1_; ++m)
      if (m != i) v *= (x - nodes_[m]) / (nodes_[i] - nodes_[m]);
    return v;
  }
  double dlagrange(int i, double x) const {
    double s = 0.;
    for (int k = 0; k < n1_; ++k) {
      if (k == i) continue;
      double v = 1. / (nodes_[i] - nodes_[k]);
      for (int m = 0; m < n1_; ++m)
        if (m != i && m != k) v *= (x - nodes_[m]) / (nodes_[i] - nodes_[m]);
      s += v;
    }
    return s;
  }

 public:
  FiniteElement(int dim, int order) : dim_(dim), order_(order), n1_(order + 1) {
    std::vector<double> w;
    shim_detail::GaussLegendre(n1_, nodes_, w);
  }
  int GetDim() const { return dim_; }
  int GetOrder() const { return order_; }
  int GetDof() const { return dim_ == 1 ? n1_ : n1_ * n1_; }
  void CalcShape(const IntegrationPoint &ip, Vector &shape) const {
    if (dim_ == 1) {
      for (int i = 0; i < n1_; ++i) shape[i] = lagrange(i, ip.x);
      return;
    }
    for (int j = 0; j < n1_; ++j) {
      const double ly = lagrange(j, ip.y);
      for (int i = 0; i < n1_; ++i) shape[j * n1_ + i] = lagrange(i, ip.x) * ly;
    }
  }
  void CalcDShape(const IntegrationPoint &ip, DenseMatrix &dshape) const {
    if (dim_ == 1) {
      for (int i = 0; i < n1_; ++i) dshape(i, 0) = dlagrange(i, ip.x);
      return;
    }
    for (int j = 0; j < n1_; ++j) {
      const double ly = lagrange(j, ip.y), dly = dlagrange(j, ip.y);
      for (int i = 0; i < n1_; ++i) {
        dshape(j * n1_ + i, 0) = dlagrange(i, ip.x) * ly;
        dshape(j * n1_ + i, 1) = lagrange(i, ip.x) * dly;
      }
    }
  }
};

class FiniteElementCollection {
 public:
  virtual ~FiniteElementCollection() = default;
  virtual const FiniteElement *FiniteElementForGeometry(int geom) const = 0;
  virtual const char *Name() const = 0;
};
class L2_FECollection : public FiniteElementCollection {
  int order_, dim_;
  std::unique_ptr<FiniteElement> segment_, square_;
  std::string name_;

 public:
  L2_FECollection(int order, int dim, int btype = BasisType::GaussLegendre)
      : order_(order), dim_(dim) {
    if (btype != BasisType::GaussLegendre)
      throw std::runtime_error("L2_FECollection shim supports Gauss-Legendre nodes only");
    segment_ = std::make_unique<FiniteElement>(1, order);
    if (dim >= 2) square_ = std::make_unique<FiniteElement>(2, order);
    name_ = "L2_" + std::to_string(dim) + "D_P" + std::to_string(order);
  }
  const FiniteElement *FiniteElementForGeometry(int geom) const override {
    if (geom == Geometry::SEGMENT) return segment_.get();
    if (geom == Geometry::SQUARE && square_) return square_.get();
    throw std::runtime_error("L2_FECollection shim: unsupported geometry");
  }
  const char *Name() const override { return name_.c_str(); }
  int GetOrder() const { return order_; }
};

// ------------------------------------------------------------------- Mesh
class ElementTransformation {
  const double *v_[4] = {nullptr, nullptr, nullptr, nullptr};
  IntegrationPoint ip_;
  DenseMatrix jac_{2, 2};

 public:
  void SetVertices(const double *a, const double *b, const double *c, const double *d) {
    v_[0] = a;
    v_[1] = b;
    v_[2] = c;
    v_[3] = d;
  }
  void SetIntPoint(const IntegrationPoint *ip) {
    ip_ = *ip;
    const double s = ip_.x, t = ip_.y;
    for (int r = 0; r < 2; ++r) {
      jac_(r, 0) = (1 - t) * (v_[1][r] - v_[0][r]) + t * (v_[2][r] - v_[3][r]);
      jac_(r, 1) = (1 - s) * (v_[3][r] - v_[0][r]) + s * (v_[2][r] - v_[1][r]);
    }
  }
  void Transform(const IntegrationPoint &ip, Vector &x) const {
    const double s = ip.x, t = ip.y;
    x.SetSize(2);
    for (int r = 0; r < 2; ++r)
      x[r] = v_[0][r] * (1 - s) * (1 - t) + v_[1][r] * s * (1 - t) + v_[2][r] * s * t +
             v_[3][r] * (1 - s) * t;
  }
  const DenseMatrix &Jacobian() const { return jac_; }
};

class Mesh {
  std::vector<std::array<double, 3>> vertices_;
  std::vector<std::array<int, 4>> elements_;
  std::vector<std::array<int, 3>> boundary_;  // attribute, v0, v1
  ElementTransformation tr_;

 public:
  Mesh() = default;
  Mesh(Mesh &&) = default;
  Mesh &operator=(Mesh &&) = default;
  static Mesh MakeCartesian2D(int nx, int ny, int type, bool /*generate_edges*/, double sx,
                              double sy, bool sfc_ordering = true) {
    if (type != Element::QUADRILATERAL || sfc_ordering)
      throw std::runtime_error("Mesh shim: only row-major quadrilateral Cartesian meshes");
    Mesh m;
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i)
        m.vertices_.push_back({sx * i / nx, sy * j / ny, 0.});
    auto vid = [nx](int i, int j) { return i + j * (nx + 1); };
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        m.elements_.push_back({vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)});
    for (int i = 0; i < nx; ++i) m.boundary_.push_back({1, vid(i + 1, 0), vid(i, 0)});
    for (int j = 0; j < ny; ++j) m.boundary_.push_back({2, vid(nx, j + 1), vid(nx, j)});
    for (int i = 0; i < nx; ++i) m.boundary_.push_back({3, vid(i, ny), vid(i + 1, ny)});
    for (int j = 0; j < ny; ++j) m.boundary_.push_back({4, vid(0, j), vid(0, j + 1)});
    return m;
  }
  int GetNV() const { return int(vertices_.size()); }
  int GetNE() const { return int(elements_.size()); }
  double *GetVertex(int v) { return vertices_[v].data(); }
  ElementTransformation *GetElementTransformation(int e) {
    const auto &el = elements_[e];
    tr_.SetVertices(vertices_[el[0]].data(), vertices_[el[1]].data(), vertices_[el[2]].data(),
                    vertices_[el[3]].data());
    return &tr_;
  }
  void Print(std::ostream &os) const {
    os << "MFEM mesh v1.0\n\ndimension\n2\n\nelements\n" << elements_.size() << '\n';
    for (const auto &e : elements_) os << "1 3 " << e[0] << ' ' << e[1] << ' ' << e[2] << ' ' << e[3] << '\n';
    os << "\nboundary\n" << boundary_.size() << '\n';
    for (const auto &b : boundary_) os << b[0] << " 1 " << b[1] << ' ' << b[2] << '\n';
    os << "\nvertices\n" << vertices_.size() << "\n2\n" << std::setprecision(17);
    for (const auto &v : vertices_) os << v[0] << ' ' << v[1] << '\n';
  }
};

class FiniteElementSpace {
  Mesh *mesh_;
  const FiniteElementCollection *fec_;

 public:
  FiniteElementSpace(Mesh *m, const FiniteElementCollection *f) : mesh_(m), fec_(f) {}
  const FiniteElement *GetFE(int) const { return fec_->FiniteElementForGeometry(Geometry::SQUARE); }
  int GetNDofs() const { return mesh_->GetNE() * GetFE(0)->GetDof(); }
  const FiniteElementCollection *FEColl() const { return fec_; }
  void GetElementDofs(int e, Array<int> &dofs) const {
    const int p = GetFE(0)->GetDof();
    dofs.SetSize(p);
    for (int i = 0; i < p; ++i) dofs[i] = e * p + i;
  }
};

class GridFunction : public Vector {
  FiniteElementSpace *fes_;

 public:
  explicit GridFunction(FiniteElementSpace *f) : Vector(f->GetNDofs()), fes_(f) { *this = 0.; }
  using Vector::operator=;
  void Save(std::ostream &os) const {
    os << "FiniteElementSpace\nFiniteElementCollection: " << fes_->FEColl()->Name()
       << "\nVDim: 1\nOrdering: 0\n\n";
    for (int i = 0; i < Size(); ++i) os << (*this)[i] << '\n';
  }
};
}  // namespace mfem
