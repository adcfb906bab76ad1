// mfem.hpp -- minimal stand-in for the parts of MFEM that the reference's
// hot-path sources touch, so that those sources (ChandrashekarFlux.cpp,
// BasicOperations.cpp, NavierStokesFlux.cpp, DGSEMIntegrator.cpp,
// LiftingScheme.cpp, LiftingBR1.cpp, Indicator.cpp,
// PerssonPeraireIndicator.cpp, ModalBasis.cpp) compile unmodified from where
// they lie and can be run as the parity pin of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY (built into oracle/_ref/, never into the product).
//
// MFEM itself is an empty submodule in the reference checkout, so every class
// here is written from MFEM's documented semantics for the calls the
// reference makes.  The ones that change floating-point results are kept
// faithful: Vector(double*, int) wraps storage without owning it (the
// reference relies on that aliasing), operator/= multiplies by the
// reciprocal, DenseMatrix is column-major and its products accumulate in
// MFEM's kernel order, CalcOrtho and AddMult_a_VWt follow MFEM's formulas, and
// Gauss-Lobatto rules/basis are on [0,1] with nodes lexicographic, x fastest.
// Affine and multilinear (bilinear quadrilateral / trilinear hexahedron)
// elements with aligned faces are modelled.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#define MFEM_ASSERT(x, msg)
#define MFEM_VERIFY(x, msg)                                          \
    do {                                                             \
        if (!(x)) throw std::runtime_error("MFEM_VERIFY failed");    \
    } while (0)
#define MFEM_ABORT(msg) throw std::runtime_error("MFEM_ABORT");
#define MFEM_WARNING(msg) \
    do {                  \
    } while (0)

namespace mfem {

using real_t = double;
inline real_t infinity() { return std::numeric_limits<real_t>::infinity(); }

// ------------------------------------------------------------------ Array
template <class T>
class Array {
    std::vector<T> d_;

public:
    Array() = default;
    explicit Array(int n) : d_(n) {}
    int Size() const { return (int)d_.size(); }
    void SetSize(int n) { d_.resize(n); }
    void Reserve(int n) { d_.reserve(n); }
    T &operator[](int i) { return d_[i]; }
    const T &operator[](int i) const { return d_[i]; }
    int Append(const T &v) { d_.push_back(v); return Size(); }
    int Append(const Array<T> &a) { d_.insert(d_.end(), a.d_.begin(), a.d_.end()); return Size(); }
    Array &operator=(const T &v) { std::fill(d_.begin(), d_.end(), v); return *this; }
    T *GetData() { return d_.data(); }
    const T *GetData() const { return d_.data(); }
    void Sort() { std::sort(d_.begin(), d_.end()); }
    void Unique() { d_.erase(std::unique(d_.begin(), d_.end()), d_.end()); }
    T Max() const { return *std::max_element(d_.begin(), d_.end()); }
};

template <class T>
class Array2D {
    int M_ = 0, N_ = 0;
    std::vector<T> d_;

public:
    Array2D() = default;
    Array2D(int m, int n) : M_(m), N_(n), d_((size_t)m * n) {}
    T &operator()(int i, int j) { return d_[(size_t)i * N_ + j]; }
    const T &operator()(int i, int j) const { return d_[(size_t)i * N_ + j]; }
    int NumRows() const { return M_; }
    int NumCols() const { return N_; }
    void GetRow(int i, Array<T> &row) const {
        row.SetSize(N_);
        for (int j = 0; j < N_; ++j) row[j] = (*this)(i, j);
    }
};

// ----------------------------------------------------------------- Vector
class Vector {
protected:
    real_t *data_ = nullptr;
    int size_ = 0;
    int cap_ = 0;
    bool own_ = false;

    void alloc(int n) {
        if (own_) delete[] data_;
        data_ = n > 0 ? new real_t[n]() : nullptr;
        cap_ = n;
        own_ = true;
        size_ = n;
    }

public:
    Vector() = default;
    explicit Vector(int n) { alloc(n); }
    Vector(real_t *p, int n) : data_(p), size_(n), cap_(n), own_(false) {}   // wraps, no ownership
    Vector(const Vector &v) {
        alloc(v.size_);
        if (size_) std::memcpy(data_, v.data_, sizeof(real_t) * size_);
    }
    ~Vector() {
        if (own_) delete[] data_;
    }
    void SetSize(int n) {
        if (n == size_) return;
        if (own_ && n <= cap_) { size_ = n; return; }
        alloc(n);
    }
    void SetDataAndSize(real_t *p, int n) {
        if (own_) delete[] data_;
        data_ = p;
        size_ = cap_ = n;
        own_ = false;
    }
    int Size() const { return size_; }
    real_t *GetData() const { return data_; }
    real_t *begin() const { return data_; }
    real_t *end() const { return data_ + size_; }
    real_t &operator()(int i) { return data_[i]; }
    const real_t &operator()(int i) const { return data_[i]; }
    real_t &operator[](int i) { return data_[i]; }
    const real_t &operator[](int i) const { return data_[i]; }
    Vector &operator=(const Vector &v) {
        if (this == &v) return *this;
        SetSize(v.size_);
        for (int i = 0; i < size_; ++i) data_[i] = v.data_[i];
        return *this;
    }
    Vector &operator=(real_t c) {
        for (int i = 0; i < size_; ++i) data_[i] = c;
        return *this;
    }
    Vector &operator*=(real_t c) {
        for (int i = 0; i < size_; ++i) data_[i] *= c;
        return *this;
    }
    Vector &operator/=(real_t c) {   // MFEM: multiply by the reciprocal
        const real_t m = 1.0 / c;
        for (int i = 0; i < size_; ++i) data_[i] *= m;
        return *this;
    }
    Vector &operator+=(const Vector &v) {
        for (int i = 0; i < size_; ++i) data_[i] += v.data_[i];
        return *this;
    }
    Vector &operator-=(const Vector &v) {
        for (int i = 0; i < size_; ++i) data_[i] -= v.data_[i];
        return *this;
    }
    Vector &Add(real_t a, const Vector &v) {
        for (int i = 0; i < size_; ++i) data_[i] += a * v.data_[i];
        return *this;
    }
    real_t operator*(const Vector &v) const {   // dot product
        real_t s = 0.0;
        for (int i = 0; i < size_; ++i) s += data_[i] * v.data_[i];
        return s;
    }
    void Neg() {
        for (int i = 0; i < size_; ++i) data_[i] = -data_[i];
    }
    void Reciprocal() {
        for (int i = 0; i < size_; ++i) data_[i] = 1.0 / data_[i];
    }
    real_t Norml2() const {   // scaled 2-norm as MFEM (hypot-style)
        if (size_ == 0) return 0.0;
        if (size_ == 1) return std::abs(data_[0]);
        real_t scale = 0.0, sum = 0.0;
        for (int i = 0; i < size_; ++i) {
            if (data_[i] != 0.0) {
                const real_t a = std::abs(data_[i]);
                if (scale <= a) {
                    const real_t r = scale / a;
                    sum = 1.0 + sum * (r * r);
                    scale = a;
                    continue;
                }
                const real_t r = a / scale;
                sum += r * r;
            }
        }
        return scale * std::sqrt(sum);
    }
    void GetSubVector(const Array<int> &dofs, Vector &elem) const {
        elem.SetSize(dofs.Size());
        for (int i = 0; i < dofs.Size(); ++i) elem(i) = data_[dofs[i]];
    }
    void GetSubVector(const Array<int> &dofs, real_t *elem) const {
        for (int i = 0; i < dofs.Size(); ++i) elem[i] = data_[dofs[i]];
    }
    void SetSubVector(const Array<int> &dofs, const Vector &elem) {
        for (int i = 0; i < dofs.Size(); ++i) data_[dofs[i]] = elem(i);
    }
    void SetSubVector(const Array<int> &dofs, const real_t *elem) {
        for (int i = 0; i < dofs.Size(); ++i) data_[dofs[i]] = elem[i];
    }
    void SetSubVector(const Array<int> &dofs, real_t value) {
        for (int i = 0; i < dofs.Size(); ++i) data_[dofs[i]] = value;
    }
    void AddElementVector(const Array<int> &dofs, const Vector &elem) {
        for (int i = 0; i < dofs.Size(); ++i) data_[dofs[i]] += elem(i);
    }
    void AddElementVector(const Array<int> &dofs, const real_t *elem) {
        for (int i = 0; i < dofs.Size(); ++i) data_[dofs[i]] += elem[i];
    }
};

inline void add(const Vector &v1, const Vector &v2, Vector &v) {
    v.SetSize(v1.Size());
    for (int i = 0; i < v.Size(); ++i) v(i) = v1(i) + v2(i);
}
inline void add(const Vector &v1, real_t alpha, const Vector &v2, Vector &v) {
    v.SetSize(v1.Size());
    for (int i = 0; i < v.Size(); ++i) v(i) = v1(i) + alpha * v2(i);
}
inline void add(real_t a, const Vector &x, real_t b, const Vector &y, Vector &z) {
    z.SetSize(x.Size());
    for (int i = 0; i < z.Size(); ++i) z(i) = a * x(i) + b * y(i);
}
inline void subtract(real_t a, const Vector &x, const Vector &y, Vector &z) {
    z.SetSize(x.Size());
    for (int i = 0; i < z.Size(); ++i) z(i) = a * (x(i) - y(i));
}

// ------------------------------------------------------------ DenseMatrix
class DenseMatrix {
protected:
    real_t *data_ = nullptr;
    int h_ = 0, w_ = 0, cap_ = 0;
    bool own_ = false;

    void alloc(int h, int w) {
        if (own_) delete[] data_;
        const int n = h * w;
        data_ = n > 0 ? new real_t[n]() : nullptr;
        cap_ = n;
        own_ = true;
        h_ = h;
        w_ = w;
    }

public:
    DenseMatrix() = default;
    explicit DenseMatrix(int n) { alloc(n, n); }
    DenseMatrix(int h, int w) { alloc(h, w); }
    DenseMatrix(real_t *d, int h, int w) : data_(d), h_(h), w_(w), cap_(h * w), own_(false) {}
    DenseMatrix(const DenseMatrix &m) {
        alloc(m.h_, m.w_);
        if (h_ * w_) std::memcpy(data_, m.data_, sizeof(real_t) * h_ * w_);
    }
    ~DenseMatrix() {
        if (own_) delete[] data_;
    }
    void UseExternalData(real_t *d, int h, int w) {
        if (own_) delete[] data_;
        data_ = d;
        h_ = h;
        w_ = w;
        cap_ = h * w;
        own_ = false;
    }
    void SetSize(int n) { SetSize(n, n); }
    void SetSize(int h, int w) {
        if (h == h_ && w == w_) return;
        if (own_ && h * w <= cap_) { h_ = h; w_ = w; return; }
        alloc(h, w);
    }
    int Height() const { return h_; }
    int Width() const { return w_; }
    int NumRows() const { return h_; }
    int NumCols() const { return w_; }
    real_t *Data() const { return data_; }
    real_t *GetData() const { return data_; }
    real_t &operator()(int i, int j) { return data_[i + (size_t)j * h_]; }
    const real_t &operator()(int i, int j) const { return data_[i + (size_t)j * h_]; }
    DenseMatrix &operator=(real_t c) {
        for (int i = 0; i < h_ * w_; ++i) data_[i] = c;
        return *this;
    }
    DenseMatrix &operator=(const DenseMatrix &m) {
        if (this == &m) return *this;
        SetSize(m.h_, m.w_);
        for (int i = 0; i < h_ * w_; ++i) data_[i] = m.data_[i];
        return *this;
    }
    DenseMatrix &operator+=(const DenseMatrix &m) {
        for (int i = 0; i < h_ * w_; ++i) data_[i] += m.data_[i];
        return *this;
    }
    DenseMatrix &operator*=(real_t c) {
        for (int i = 0; i < h_ * w_; ++i) data_[i] *= c;
        return *this;
    }
    void Neg() {
        for (int i = 0; i < h_ * w_; ++i) data_[i] = -data_[i];
    }
    void GetRow(int r, Vector &row) const {
        row.SetSize(w_);
        for (int j = 0; j < w_; ++j) row(j) = (*this)(r, j);
    }
    void GetColumn(int c, Vector &col) const {
        col.SetSize(h_);
        for (int i = 0; i < h_; ++i) col(i) = (*this)(i, c);
    }
    void GetColumnReference(int c, Vector &col) { col.SetDataAndSize(data_ + (size_t)c * h_, h_); }
    void SetRow(int r, const Vector &row) {
        for (int j = 0; j < w_; ++j) (*this)(r, j) = row(j);
    }
    void SetCol(int c, const Vector &col) {
        for (int i = 0; i < h_; ++i) (*this)(i, c) = col(i);
    }
    // y = A x, accumulated column by column (mfem kernels::Mult)
    void Mult(const real_t *x, real_t *y) const {
        if (w_ == 0) {
            for (int r = 0; r < h_; ++r) y[r] = 0.0;
            return;
        }
        const real_t *d_col = data_;
        real_t x_col = x[0];
        for (int r = 0; r < h_; ++r) y[r] = x_col * d_col[r];
        d_col += h_;
        for (int c = 1; c < w_; ++c) {
            x_col = x[c];
            for (int r = 0; r < h_; ++r) y[r] += x_col * d_col[r];
            d_col += h_;
        }
    }
    void Mult(const Vector &x, Vector &y) const { Mult(x.GetData(), y.GetData()); }
    void AddMult(const Vector &x, Vector &y) const {
        const real_t *d_col = data_;
        for (int c = 0; c < w_; ++c) {
            const real_t x_col = x[c];
            for (int r = 0; r < h_; ++r) y[r] += x_col * d_col[r];
            d_col += h_;
        }
    }
    void MultTranspose(const Vector &x, Vector &y) const {
        for (int i = 0; i < w_; ++i) {
            real_t d = 0.0;
            for (int j = 0; j < h_; ++j) d += (*this)(j, i) * x[j];
            y[i] = d;
        }
    }
    void Transpose() {   // square, in place
        for (int i = 0; i < h_; ++i)
            for (int j = i + 1; j < w_; ++j) std::swap((*this)(i, j), (*this)(j, i));
    }
    // Gauss-Jordan inverse with partial pivoting (square)
    void Invert() {
        const int n = h_;
        std::vector<real_t> A(data_, data_ + n * n), I(n * n, 0.0);
        for (int i = 0; i < n; ++i) I[i + i * n] = 1.0;
        auto a = [&](int i, int j) -> real_t & { return A[i + j * n]; };
        auto b = [&](int i, int j) -> real_t & { return I[i + j * n]; };
        for (int c = 0; c < n; ++c) {
            int piv = c;
            for (int r = c + 1; r < n; ++r)
                if (std::abs(a(r, c)) > std::abs(a(piv, c))) piv = r;
            for (int k = 0; k < n; ++k) {
                std::swap(a(c, k), a(piv, k));
                std::swap(b(c, k), b(piv, k));
            }
            const real_t d = 1.0 / a(c, c);
            for (int k = 0; k < n; ++k) { a(c, k) *= d; b(c, k) *= d; }
            for (int r = 0; r < n; ++r) {
                if (r == c) continue;
                const real_t f = a(r, c);
                if (f == 0.0) continue;
                for (int k = 0; k < n; ++k) { a(r, k) -= f * a(c, k); b(r, k) -= f * b(c, k); }
            }
        }
        std::copy(I.begin(), I.end(), data_);
    }
};

// a = b * c (mfem kernels::Mult order)
inline void Mult(const DenseMatrix &b, const DenseMatrix &c, DenseMatrix &a) {
    const int ah = b.Height(), aw = c.Width(), bw = b.Width();
    for (int i = 0; i < ah * aw; ++i) a.Data()[i] = 0.0;
    for (int j = 0; j < aw; ++j)
        for (int k = 0; k < bw; ++k)
            for (int i = 0; i < ah; ++i) a(i, j) += b(i, k) * c(k, j);
}
// ABt = A * B^T (mfem kernels::MultABt order)
inline void MultABt(const DenseMatrix &A, const DenseMatrix &B, DenseMatrix &ABt) {
    const int ah = A.Height(), bh = B.Height(), aw = A.Width();
    for (int i = 0; i < ah * bh; ++i) ABt.Data()[i] = 0.0;
    for (int k = 0; k < aw; ++k)
        for (int j = 0; j < bh; ++j) {
            const real_t bjk = B(j, k);
            for (int i = 0; i < ah; ++i) ABt(i, j) += A(i, k) * bjk;
        }
}
// VWt += a v w^T
inline void AddMult_a_VWt(const real_t a, const Vector &v, const Vector &w, DenseMatrix &VWt) {
    for (int j = 0; j < w.Size(); ++j) {
        const real_t awj = a * w(j);
        for (int i = 0; i < v.Size(); ++i) VWt(i, j) += v(i) * awj;
    }
}
// Scaled normal of a face from its Jacobian (mfem::CalcOrtho)
inline void CalcOrtho(const DenseMatrix &J, Vector &n) {
    if (J.Height() == 2) {
        n(0) = J(1, 0);
        n(1) = -J(0, 0);
    } else {
        n(0) = J(1, 0) * J(2, 1) - J(2, 0) * J(1, 1);
        n(1) = J(2, 0) * J(0, 1) - J(0, 0) * J(2, 1);
        n(2) = J(0, 0) * J(1, 1) - J(1, 0) * J(0, 1);
    }
}

class DenseTensor {
    std::vector<real_t> d_;
    int m_ = 0, n_ = 0, k_ = 0;
    DenseMatrix Mk_;

public:
    DenseTensor() = default;
    DenseTensor(int i, int j, int k) { SetSize(i, j, k); }
    void SetSize(int i, int j, int k) {
        m_ = i; n_ = j; k_ = k;
        d_.assign((size_t)i * j * k, 0.0);
    }
    int SizeI() const { return m_; }
    int SizeJ() const { return n_; }
    int SizeK() const { return k_; }
    DenseMatrix &operator()(int k) {   // one shared slice object, as MFEM
        Mk_.UseExternalData(d_.data() + (size_t)k * m_ * n_, m_, n_);
        return Mk_;
    }
    real_t &operator()(int i, int j, int k) { return d_[i + (size_t)m_ * (j + (size_t)n_ * k)]; }
};

// -------------------------------------------------------- quadrature / basis
struct Geometry {
    enum Type { INVALID = -1, POINT = 0, SEGMENT, TRIANGLE, SQUARE, TETRAHEDRON, CUBE, PRISM, PYRAMID };
};
struct Quadrature1D {
    enum { Invalid = -1, GaussLegendre = 0, GaussLobatto = 1 };
};
struct BasisType {
    enum { Invalid = -1, GaussLegendre = 0, GaussLobatto = 1, Positive = 2 };
    static int CheckNodal(int b) { return b; }
};

struct IntegrationPoint {
    real_t x = 0.0, y = 0.0, z = 0.0, weight = 0.0;
    int index = 0;
    void Get(real_t *p, const int dim) const {
        p[0] = x;
        if (dim > 1) {
            p[1] = y;
            if (dim > 2) p[2] = z;
        }
    }
    void Set2(real_t x1, real_t x2) { x = x1; y = x2; }
    void Set3(real_t x1, real_t x2, real_t x3) { x = x1; y = x2; z = x3; }
};

class IntegrationRule {
    std::vector<IntegrationPoint> p_;

public:
    IntegrationRule() = default;
    explicit IntegrationRule(int n) : p_(n) {}
    int GetNPoints() const { return (int)p_.size(); }
    IntegrationPoint &IntPoint(int i) { return p_[i]; }
    const IntegrationPoint &IntPoint(int i) const { return p_[i]; }
    const IntegrationPoint *begin() const { return p_.data(); }
    const IntegrationPoint *end() const { return p_.data() + p_.size(); }
};

// Gauss-Lobatto nodes/weights on [0,1] (n points), long-double Newton.
void GaussLobattoRule(int n, std::vector<real_t> &x, std::vector<real_t> &w);
const IntegrationRule &TensorGL(int geom, int n);

class IntegrationRules {
public:
    IntegrationRules(int refined = 0, int type = Quadrature1D::GaussLegendre) { (void)refined; (void)type; }
    // GL rule with n points integrates degree 2n-3 exactly
    const IntegrationRule &Get(int geom, int order) const { return TensorGL(geom, order / 2 + 2); }
};

class Poly_1D {
public:
    static void CalcLegendre(const int p, const real_t x, real_t *u) {
        real_t z;
        u[0] = 1.;
        if (p == 0) return;
        u[1] = z = 2. * x - 1.;
        for (int n = 1; n < p; n++) u[n + 1] = ((2 * n + 1) * z * u[n] - n * u[n - 1]) / (n + 1);
    }
    static void CalcLegendre(const int p, const real_t x, real_t *u, real_t *d) {
        real_t z;
        u[0] = 1.;
        d[0] = 0.;
        if (p == 0) return;
        u[1] = z = 2. * x - 1.;
        d[1] = 2.;
        for (int n = 1; n < p; n++) {
            u[n + 1] = ((2 * n + 1) * z * u[n] - n * u[n - 1]) / (n + 1);
            d[n + 1] = (4 * n + 2) * u[n] + d[n - 1];
        }
    }
};

// Tensor-product Lagrange element on Gauss-Lobatto nodes of [0,1]^dim.
class FiniteElement {
    int dim_ = 0, order_ = 0;
    std::vector<real_t> x_;
    IntegrationRule nodes_;

public:
    FiniteElement(int dim, int order);
    int GetDim() const { return dim_; }
    int GetOrder() const { return order_; }
    int GetDof() const { return nodes_.GetNPoints(); }
    int GetGeomType() const { return dim_ == 1 ? Geometry::SEGMENT : dim_ == 2 ? Geometry::SQUARE : Geometry::CUBE; }
    const IntegrationRule &GetNodes() const { return nodes_; }
    void CalcShape(const IntegrationPoint &ip, Vector &shape) const;
};

class DG_FECollection {
    int order_, dim_, btype_;
    std::unique_ptr<FiniteElement> fe_;

public:
    DG_FECollection(int p, int dim, int btype = BasisType::GaussLegendre)
        : order_(p), dim_(dim), btype_(btype), fe_(new FiniteElement(dim, p)) {}
    int GetBasisType() const { return btype_; }
    const FiniteElement *FiniteElementForGeometry(int) const { return fe_.get(); }
    const FiniteElement *FE() const { return fe_.get(); }
    int GetOrder() const { return order_; }
};

// ------------------------------------------------------- transformations
// The element map is affine (x = x0 + J xi) or multilinear in the element's
// corners (MFEM's IsoparametricTransformation with the order-1 H1 basis):
// SetIntPoint evaluates J = dx/dxi there and, as MFEM does on demand, its
// adjugate (CalcAdjugate) and determinant (Weight).
class ElementTransformation {
public:
    int ElementNo = 0;
    int dim = 0;
    DenseMatrix J, adj;
    real_t detJ = 0.0;
    real_t x0[3] = {0, 0, 0};
    bool multilinear = false;
    real_t corner[8][3] = {};          // corner b at reference vertex (b & 1, b >> 1 & 1, b >> 2 & 1)
    const IntegrationPoint *ip = nullptr;
    void SetIntPoint(const IntegrationPoint *p) {
        ip = p;
        if (multilinear) eval(*p);
    }
    const IntegrationPoint &GetIntPoint() const { return *ip; }
    real_t Weight() { return detJ; }
    const DenseMatrix &Jacobian() { return J; }
    const DenseMatrix &AdjugateJacobian() { return adj; }
    void Transform(const IntegrationPoint &p, Vector &x) {
        real_t xi[3] = {p.x, p.y, p.z};
        x.SetSize(dim);
        if (multilinear) {
            for (int r = 0; r < dim; ++r) x(r) = 0.0;
            for (int b = 0; b < (1 << dim); ++b) {
                real_t phi = 1.0;
                for (int q = 0; q < dim; ++q) phi *= ((b >> q) & 1) ? xi[q] : 1.0 - xi[q];
                for (int r = 0; r < dim; ++r) x(r) += phi * corner[b][r];
            }
            return;
        }
        for (int r = 0; r < dim; ++r) {
            real_t s = x0[r];
            for (int c = 0; c < dim; ++c) s += J(r, c) * xi[c];
            x(r) = s;
        }
    }

private:
    void eval(const IntegrationPoint &p) {
        const real_t xi[3] = {p.x, p.y, p.z};
        for (int r = 0; r < dim; ++r)
            for (int c = 0; c < dim; ++c) J(r, c) = 0.0;
        for (int b = 0; b < (1 << dim); ++b)
            for (int c = 0; c < dim; ++c) {
                real_t dphi = ((b >> c) & 1) ? 1.0 : -1.0;
                for (int q = 0; q < dim; ++q)
                    if (q != c) dphi *= ((b >> q) & 1) ? xi[q] : 1.0 - xi[q];
                for (int r = 0; r < dim; ++r) J(r, c) += dphi * corner[b][r];
            }
        if (dim == 2) {   // CalcAdjugate, DenseMatrix::Det
            adj(0, 0) = J(1, 1); adj(0, 1) = -J(0, 1);
            adj(1, 0) = -J(1, 0); adj(1, 1) = J(0, 0);
            detJ = J(0, 0) * J(1, 1) - J(0, 1) * J(1, 0);
        } else {
            adj(0, 0) = J(1, 1) * J(2, 2) - J(1, 2) * J(2, 1);
            adj(0, 1) = J(0, 2) * J(2, 1) - J(0, 1) * J(2, 2);
            adj(0, 2) = J(0, 1) * J(1, 2) - J(0, 2) * J(1, 1);
            adj(1, 0) = J(1, 2) * J(2, 0) - J(1, 0) * J(2, 2);
            adj(1, 1) = J(0, 0) * J(2, 2) - J(0, 2) * J(2, 0);
            adj(1, 2) = J(0, 2) * J(1, 0) - J(0, 0) * J(1, 2);
            adj(2, 0) = J(1, 0) * J(2, 1) - J(1, 1) * J(2, 0);
            adj(2, 1) = J(0, 1) * J(2, 0) - J(0, 0) * J(2, 1);
            adj(2, 2) = J(0, 0) * J(1, 1) - J(0, 1) * J(1, 0);
            detJ = J(0, 0) * adj(0, 0) + J(0, 1) * adj(1, 0) + J(0, 2) * adj(2, 0);
        }
    }
};

class FaceElementTransformations {
public:
    int ElementNo = -1;   // the face number
    int Elem1No = -1, Elem2No = -1;
    int lf1 = 0, lf2 = 0, dim = 0;
    real_t orient = 1.0;  // sign that makes CalcOrtho point out of elem1
    ElementTransformation *T1 = nullptr, *T2 = nullptr;
    DenseMatrix Jf;
    IntegrationPoint eip1, eip2;
    // maps the face point into both elements, sets their transformations there
    // and the face Jacobian (element 1's tangential columns, oriented)
    void SetAllIntPoints(const IntegrationPoint *face_ip);
    ElementTransformation &GetElement1Transformation() { return *T1; }
    ElementTransformation &GetElement2Transformation() { return *T2; }
    const IntegrationPoint &GetElement1IntPoint() { return eip1; }
    const IntegrationPoint &GetElement2IntPoint() { return eip2; }
    const DenseMatrix &Jacobian() { return Jf; }
    // the physical point of the face point last set by SetAllIntPoints
    void Transform(const IntegrationPoint &, Vector &x) { T1->Transform(eip1, x); }
};

// ------------------------------------------------------------ coefficients
// MFEM's function coefficients: a std::function of the physical point (and,
// with SetTime, of the time), from FaceElementTransformations::Transform.
inline void mfem_error(const char *msg) { throw std::runtime_error(msg); }
class FunctionCoefficient {
public:
    explicit FunctionCoefficient(std::function<real_t(const Vector &)> f) : f_(std::move(f)) {}
    void SetTime(real_t t) { t_ = t; }
    real_t Eval(FaceElementTransformations &T, const IntegrationPoint &ip) {
        Vector x;
        T.Transform(ip, x);
        return f_(x);
    }

private:
    std::function<real_t(const Vector &)> f_;
    real_t t_ = 0.0;
};
class VectorFunctionCoefficient {
public:
    VectorFunctionCoefficient(int vdim, std::function<void(const Vector &, Vector &)> f)
        : vdim_(vdim), f_(std::move(f)) {}
    void SetTime(real_t t) { t_ = t; }
    void Eval(Vector &v, FaceElementTransformations &T, const IntegrationPoint &ip) {
        Vector x;
        T.Transform(ip, x);
        v.SetSize(vdim_);
        f_(x, v);
    }

private:
    int vdim_;
    std::function<void(const Vector &, Vector &)> f_;
    real_t t_ = 0.0;
};

// ------------------------------------------------------------ mesh / spaces
struct Connection {
    int from, to;
    Connection(int f = 0, int t = 0) : from(f), to(t) {}
    bool operator<(const Connection &o) const { return from < o.from || (from == o.from && to < o.to); }
    bool operator==(const Connection &o) const { return from == o.from && to == o.to; }
};
class Table {
public:
    Table() = default;
    Table(int, Array<Connection> &) {}
};
inline void Transpose(const Table &, Table &, int = -1) {}

class Mesh {
public:
    int dim = 0;
    std::vector<ElementTransformation> trans;
    std::vector<std::unique_ptr<FaceElementTransformations>> faces;
    int GetNE() const { return (int)trans.size(); }
    int GetNBE() const { return 0; }
    int SpaceDimension() const { return dim; }
    int Dimension() const { return dim; }
    void GetBdrElementAdjacentElement(int, int &el, int &info) const { el = -1; info = -1; }
    ElementTransformation *GetElementTransformation(int e) { return &trans[e]; }
    int GetNumFaces() const { return (int)faces.size(); }
    FaceElementTransformations *GetInteriorFaceTransformations(int f) { return faces[f].get(); }
};
class ParMesh : public Mesh {};

class ParFiniteElementSpace {
public:
    ParMesh *mesh = nullptr;
    const DG_FECollection *fec = nullptr;
    int vdim = 1;
    ParFiniteElementSpace(ParMesh *m, const DG_FECollection *f, int vd = 1) : mesh(m), fec(f), vdim(vd) {}
    int GetVDim() const { return vdim; }
    int GetNE() const { return mesh->GetNE(); }
    const FiniteElement *GetFE(int) const { return fec->FE(); }
    int GetElementOrder(int) const { return fec->GetOrder(); }
    Mesh *GetMesh() const { return mesh; }
    int GetNDofs() const { return GetNE() * fec->FE()->GetDof(); }
    int GetVSize() const { return vdim * GetNDofs(); }
    ElementTransformation *GetElementTransformation(int e) const { return mesh->GetElementTransformation(e); }
    void GetElementDofs(int e, Array<int> &dofs) const {
        const int nd = fec->FE()->GetDof();
        dofs.SetSize(nd);
        for (int i = 0; i < nd; ++i) dofs[i] = e * nd + i;
    }
    void GetElementVDofs(int e, Array<int> &vdofs) const {   // Ordering::byNODES
        const int nd = fec->FE()->GetDof(), N = GetNDofs();
        vdofs.SetSize(nd * vdim);
        for (int f = 0; f < vdim; ++f)
            for (int i = 0; i < nd; ++i) vdofs[f * nd + i] = f * N + e * nd + i;
    }
};

class ParGridFunction : public Vector {
public:
    ParFiniteElementSpace *fes = nullptr;
    explicit ParGridFunction(ParFiniteElementSpace *f) : Vector(f->GetVSize()), fes(f) {}
    using Vector::operator=;
};

class NonlinearFormIntegrator {
public:
    virtual void AssembleElementVector(const FiniteElement &, ElementTransformation &, const Vector &, Vector &) {}
    virtual void AssembleFaceVector(const FiniteElement &, const FiniteElement &, FaceElementTransformations &,
                                    const Vector &, Vector &) {}
    virtual ~NonlinearFormIntegrator() = default;
};

// mfem::EulerFlux / FluxFunction: only the members the reference reads.
class EulerFlux {
public:
    const int num_equations;
    const int dim;
    EulerFlux(const int dim_, const real_t) : num_equations(dim_ + 2), dim(dim_) {}
    real_t ComputeFlux(const Vector &, ElementTransformation &, DenseMatrix &) const { return 0.0; }
    real_t ComputeFluxDotN(const Vector &, const Vector &, FaceElementTransformations &, Vector &) const { return 0.0; }
};

}   // namespace mfem
