// Minimal stand-ins for the handful of MFEM types that the reference's
// assembly sources name (solver/problem_common.inc, solver/asm_data.inc,
// solver/asm_gpu.inc), so that those files compile unchanged from the
// reference tree without MFEM.  Test infrastructure only.
//
// Only the members the CPU reassembler (reassemble_element/reassemble_all,
// build_csr_symbolic) and the GPU classes actually execute carry real code:
// Array<int>, Vector::GetData, DenseMatrix element access and the
// MFEM_VERIFY check.  Everything that belongs to MFEM's element and mesh
// machinery (used only by extract_asm_data / extract_ref_rule, which the
// shim never calls: the oracle feeds AsmData directly) aborts if reached.
#pragma once

#include <complex>
#include <cstdio>
#include <cstdlib>
#include <vector>

#define MFEM_VERIFY(cond, msg)                                              \
  do {                                                                      \
    if (!(cond)) {                                                          \
      std::fprintf(stderr, "MFEM_VERIFY failed: %s (%s:%d)\n", msg,         \
                   __FILE__, __LINE__);                                     \
      std::abort();                                                         \
    }                                                                       \
  } while (0)

namespace mfem {

[[noreturn]] inline void shim_unreachable(const char *what) {
  std::fprintf(stderr, "mfem shim: %s is not available\n", what);
  std::abort();
}

template <typename T>
class Array {
 public:
  Array() = default;
  explicit Array(int n) : d_(n) {}
  int Size() const { return (int)d_.size(); }
  T &operator[](int i) { return d_[i]; }
  const T &operator[](int i) const { return d_[i]; }
  void Append(const T &v) { d_.push_back(v); }
  T *GetData() { return d_.data(); }
  const T *GetData() const { return d_.data(); }

 private:
  std::vector<T> d_;
};

class Vector {
 public:
  Vector() = default;
  explicit Vector(int n) : own_(n), p_(own_.data()), n_(n) {}
  Vector(double *p, int n) : p_(p), n_(n) {}
  void SetSize(int n) {
    own_.assign(n, 0.0);
    p_ = own_.data();
    n_ = n;
  }
  Vector &operator=(double v) {
    for (int i = 0; i < n_; ++i) p_[i] = v;
    return *this;
  }
  double &operator()(int i) { return p_[i]; }
  double operator()(int i) const { return p_[i]; }
  double *GetData() { return p_; }
  const double *GetData() const { return p_; }
  int Size() const { return n_; }

 private:
  std::vector<double> own_;
  double *p_ = nullptr;
  int n_ = 0;
};

class DenseMatrix {
 public:
  DenseMatrix() = default;
  explicit DenseMatrix(int n) { SetSize(n, n); }
  DenseMatrix(int r, int c) { SetSize(r, c); }
  void SetSize(int n) { SetSize(n, n); }
  void SetSize(int r, int c) {
    r_ = r;
    c_ = c;
    d_.assign((size_t)r * c, 0.0);
  }
  DenseMatrix &operator=(double v) {
    for (double &x : d_) x = v;
    return *this;
  }
  // column-major, like MFEM
  double &operator()(int i, int j) { return d_[(size_t)j * r_ + i]; }
  double operator()(int i, int j) const { return d_[(size_t)j * r_ + i]; }

 private:
  int r_ = 0, c_ = 0;
  std::vector<double> d_;
};

struct IntegrationPoint {
  double x = 0, y = 0, z = 0, weight = 0;
  void Set3(double a, double b, double c) { x = a; y = b; z = c; }
};

class IntegrationRule {
 public:
  int GetNPoints() const { shim_unreachable("IntegrationRule"); }
  const IntegrationPoint &IntPoint(int) const { shim_unreachable("IntegrationRule"); }
};

struct Geometry {
  enum Type { TETRAHEDRON = 4 };
};

struct IntegrationRules {
  const IntegrationRule &Get(int, int) const { shim_unreachable("IntRules"); }
};
static IntegrationRules IntRules;

// Affine element map x = v0 + J xi, enough for the reference's coefficient
// classes (ScatterSource::Eval calls Attribute and Transform); the Jacobian
// queries of the MFEM extraction stay unavailable.
class ElementTransformation {
 public:
  int Attribute = 0;
  bool affine = false;
  double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // row-major
  double v0[3] = {0, 0, 0};
  void SetIntPoint(const IntegrationPoint *) { shim_unreachable("ElementTransformation"); }
  const DenseMatrix &Jacobian() { shim_unreachable("ElementTransformation"); }
  double Weight() { shim_unreachable("ElementTransformation"); }
  void Transform(const IntegrationPoint &ip, Vector &x) {
    if (!affine) shim_unreachable("ElementTransformation::Transform");
    const double xi[3] = {ip.x, ip.y, ip.z};
    for (int i = 0; i < 3; ++i)
      x(i) = v0[i] + J[3 * i] * xi[0] + J[3 * i + 1] * xi[1] + J[3 * i + 2] * xi[2];
  }
};

class FiniteElement {
 public:
  int GetDof() const { shim_unreachable("FiniteElement"); }
  void CalcVShape(const IntegrationPoint &, DenseMatrix &) const { shim_unreachable("FiniteElement"); }
  void CalcCurlShape(const IntegrationPoint &, DenseMatrix &) const { shim_unreachable("FiniteElement"); }
};

class DofTransformation {
 public:
  const Array<int> &GetFaceOrientations() const { shim_unreachable("DofTransformation"); }
};

class Mesh {
 public:
  int GetNE() const { shim_unreachable("Mesh"); }
  int GetAttribute(int) const { shim_unreachable("Mesh"); }
  ElementTransformation *GetElementTransformation(int) { shim_unreachable("Mesh"); }
};

class FiniteElementSpace {
 public:
  int GetVSize() const { shim_unreachable("FiniteElementSpace"); }
  const FiniteElement *GetFE(int) const { shim_unreachable("FiniteElementSpace"); }
  void GetElementDofs(int, Array<int> &, DofTransformation &) const {
    shim_unreachable("FiniteElementSpace");
  }
};

inline void CalcInverse(const DenseMatrix &, DenseMatrix &) { shim_unreachable("CalcInverse"); }

class MatrixCoefficient {
 public:
  explicit MatrixCoefficient(int) {}
  virtual ~MatrixCoefficient() = default;
  virtual void Eval(DenseMatrix &, ElementTransformation &, const IntegrationPoint &) = 0;
};

class VectorCoefficient {
 public:
  explicit VectorCoefficient(int) {}
  virtual ~VectorCoefficient() = default;
  virtual void Eval(Vector &, ElementTransformation &, const IntegrationPoint &) = 0;
};

}  // namespace mfem
