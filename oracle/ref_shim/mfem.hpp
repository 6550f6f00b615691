// mfem.hpp — a small stand-in for the parts of the MFEM API that Prandtl's
// hot-path sources use, written for this project so those sources can be
// compiled unmodified (in place, from the reference tree) and run as a
// parity check.  TEST INFRASTRUCTURE ONLY: nothing in the product uses it.
//
// Scope: affine, axis-aligned Cartesian quads/hexes, or nodal (curved,
// skewed, unstructured) ones given by their DG nodes' coordinates; L2 Gauss-Lobatto nodal
// elements; Gauss-Lobatto integration rules on [0,1]; dense linear algebra on
// column-major matrices.  Semantics that change results are kept as MFEM
// documents them:
//   * Vector(double *data, int n) and DenseMatrix(double *data, int h, int w)
//     are non-owning views, and GetData() on a const object returns a mutable
//     pointer, so in-place edits through a view reach the caller's storage;
//   * DenseMatrix::GetColumnReference makes a view of one column;
//   * DenseMatrix storage is column-major;
//   * Vector::operator/=(c) scales by the reciprocal of c.
// Everything else (summation order inside Mult/MultTranspose, the dense
// inverse, the GLL rule) is this file's own implementation of the
// mathematics, so results match real MFEM to rounding, not bit for bit.
#pragma once

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#define MFEM_ASSERT(x, msg)
#define MFEM_VERIFY(x, msg)                                                                        \
    do {                                                                                           \
        if (!(x)) { std::cerr << "stand-in MFEM check failed\n"; std::abort(); }                    \
    } while (0)
#define MFEM_ABORT(msg)                                                                            \
    do {                                                                                           \
        std::cerr << "stand-in MFEM abort\n";                                                      \
        std::abort();                                                                              \
    } while (0);
#define MFEM_HOST_DEVICE
#define MFEM_WARNING(msg) do { } while (0)

namespace mfem {

typedef double real_t;
inline real_t infinity() { return std::numeric_limits<real_t>::infinity(); }
inline void mfem_error(const char *msg)
{
    std::cerr << "stand-in MFEM error: " << msg << "\n";
    std::abort();
}

template <class T> class Array {
    std::vector<T> v_;

public:
    Array() {}
    explicit Array(int n) : v_(n) {}
    int Size() const { return (int)v_.size(); }
    void SetSize(int n) { v_.resize(n); }
    void Reserve(int n) { v_.reserve(n); }
    T &operator[](int i) { return v_[i]; }
    const T &operator[](int i) const { return v_[i]; }
    void Append(const T &x) { v_.push_back(x); }
    void Append(const Array<T> &a) { v_.insert(v_.end(), a.v_.begin(), a.v_.end()); }
    void Prepend(const T &x) { v_.insert(v_.begin(), x); }
    Array &operator=(const T &x) { std::fill(v_.begin(), v_.end(), x); return *this; }
    T Max() const { return *std::max_element(v_.begin(), v_.end()); }
    void Sort() { std::sort(v_.begin(), v_.end()); }
    void Unique() { v_.erase(std::unique(v_.begin(), v_.end()), v_.end()); }
    T *GetData() { return v_.data(); }
    const T *Read(bool = true) const { return v_.data(); }
};

template <class T> class Array2D {
    int M_ = 0, N_ = 0;
    std::vector<T> v_;

public:
    Array2D() {}
    Array2D(int m, int n) : M_(m), N_(n), v_((size_t)m * n) {}
    T &operator()(int i, int j) { return v_[(size_t)i * N_ + j]; }
    const T &operator()(int i, int j) const { return v_[(size_t)i * N_ + j]; }
    int NumRows() const { return M_; }
    int NumCols() const { return N_; }
    void GetRow(int i, Array<T> &row) const
    {
        row.SetSize(N_);
        for (int j = 0; j < N_; j++) row[j] = (*this)(i, j);
    }
};

class Vector {
    real_t *data_ = nullptr;
    int size_ = 0;
    int cap_ = 0;
    bool own_ = false;

    void alloc(int n)
    {
        if (own_) delete[] data_;
        data_ = n > 0 ? new real_t[n]() : nullptr;
        size_ = cap_ = n;
        own_ = true;
    }

public:
    Vector() {}
    explicit Vector(int n) { alloc(n); }
    Vector(real_t *d, int n) : data_(d), size_(n), cap_(n), own_(false) {}
    Vector(const Vector &o)
    {
        alloc(o.size_);
        if (size_) std::memcpy(data_, o.data_, sizeof(real_t) * size_);
    }
    ~Vector()
    {
        if (own_) delete[] data_;
    }
    void SetSize(int n)
    {
        if (n == size_) return;
        if (n <= cap_) { size_ = n; return; }
        alloc(n);
    }
    void SetDataAndSize(real_t *d, int n)
    {
        if (own_) delete[] data_;
        data_ = d;
        size_ = cap_ = n;
        own_ = false;
    }
    void NewDataAndSize(real_t *d, int n) { SetDataAndSize(d, n); }
    int Size() const { return size_; }
    real_t *GetData() const { return data_; }
    operator real_t *() const { return data_; }
    real_t &operator()(int i) { return data_[i]; }
    const real_t &operator()(int i) const { return data_[i]; }
    real_t &operator[](int i) { return data_[i]; }
    const real_t &operator[](int i) const { return data_[i]; }
    real_t *begin() const { return data_; }
    real_t *end() const { return data_ + size_; }
    Vector &operator=(const Vector &o)
    {
        if (this == &o) return *this;
        SetSize(o.size_);
        if (size_) std::memmove(data_, o.data_, sizeof(real_t) * size_);
        return *this;
    }
    Vector &operator=(const real_t *d)
    {
        if (size_) std::memmove(data_, d, sizeof(real_t) * size_);
        return *this;
    }
    Vector &operator=(real_t c)
    {
        for (int i = 0; i < size_; i++) data_[i] = c;
        return *this;
    }
    Vector &operator*=(real_t c)
    {
        for (int i = 0; i < size_; i++) data_[i] *= c;
        return *this;
    }
    Vector &operator/=(real_t c)
    {
        const real_t m = 1.0 / c;
        for (int i = 0; i < size_; i++) data_[i] *= m;
        return *this;
    }
    Vector &operator+=(const Vector &o)
    {
        for (int i = 0; i < size_; i++) data_[i] += o.data_[i];
        return *this;
    }
    Vector &operator-=(const Vector &o)
    {
        for (int i = 0; i < size_; i++) data_[i] -= o.data_[i];
        return *this;
    }
    Vector &operator+=(real_t c)
    {
        for (int i = 0; i < size_; i++) data_[i] += c;
        return *this;
    }
    void Neg()
    {
        for (int i = 0; i < size_; i++) data_[i] = -data_[i];
    }
    // this += a * v
    void Add(real_t a, const Vector &v)
    {
        for (int i = 0; i < size_; i++) data_[i] += a * v.data_[i];
    }
    void Reciprocal()
    {
        for (int i = 0; i < size_; i++) data_[i] = 1.0 / data_[i];
    }
    real_t operator*(const Vector &o) const
    {
        real_t s = 0.0;
        for (int i = 0; i < size_; i++) s += data_[i] * o.data_[i];
        return s;
    }
    real_t Norml2() const
    {
        // Overflow-safe two-norm: running scale and sum of squared ratios.
        if (size_ == 0) return 0.0;
        if (size_ == 1) return std::abs(data_[0]);
        real_t scale = 0.0, sum = 0.0;
        for (int i = 0; i < size_; i++) {
            if (data_[i] == 0.0) continue;
            const real_t a = std::abs(data_[i]);
            if (scale <= a) {
                const real_t r = scale / a;
                sum = 1.0 + sum * (r * r);
                scale = a;
            } else {
                const real_t r = a / scale;
                sum += r * r;
            }
        }
        return scale * std::sqrt(sum);
    }
    void GetSubVector(const Array<int> &dofs, Vector &elem) const
    {
        elem.SetSize(dofs.Size());
        for (int i = 0; i < dofs.Size(); i++) elem(i) = data_[dofs[i]];
    }
    void GetSubVector(const Array<int> &dofs, real_t *elem) const
    {
        for (int i = 0; i < dofs.Size(); i++) elem[i] = data_[dofs[i]];
    }
    void SetSubVector(const Array<int> &dofs, real_t value)
    {
        for (int i = 0; i < dofs.Size(); i++) data_[dofs[i]] = value;
    }
    void SetSubVector(const Array<int> &dofs, const Vector &elem)
    {
        for (int i = 0; i < dofs.Size(); i++) data_[dofs[i]] = elem(i);
    }
    void SetSubVector(const Array<int> &dofs, const real_t *elem)
    {
        for (int i = 0; i < dofs.Size(); i++) data_[dofs[i]] = elem[i];
    }
    void AddElementVector(const Array<int> &dofs, const Vector &elem)
    {
        for (int i = 0; i < dofs.Size(); i++) data_[dofs[i]] += elem(i);
    }
    void AddElementVector(const Array<int> &dofs, const real_t *elem)
    {
        for (int i = 0; i < dofs.Size(); i++) data_[dofs[i]] += elem[i];
    }
    void Print(std::ostream &os = std::cout) const
    {
        for (int i = 0; i < size_; i++) os << data_[i] << (i + 1 < size_ ? " " : "\n");
    }
};

// v = v1 + v2
inline void add(const Vector &v1, const Vector &v2, Vector &v)
{
    v.SetSize(v1.Size());
    for (int i = 0; i < v.Size(); i++) v(i) = v1(i) + v2(i);
}
// z = a * (x - y)
inline void subtract(real_t a, const Vector &x, const Vector &y, Vector &z)
{
    z.SetSize(x.Size());
    for (int i = 0; i < z.Size(); i++) z(i) = a * (x(i) - y(i));
}

class DenseMatrix {
    real_t *data_ = nullptr;
    int h_ = 0, w_ = 0, cap_ = 0;
    bool own_ = false;

    void alloc(int h, int w)
    {
        if (own_) delete[] data_;
        int n = h * w;
        data_ = n > 0 ? new real_t[n]() : nullptr;
        h_ = h;
        w_ = w;
        cap_ = n;
        own_ = true;
    }

public:
    DenseMatrix() {}
    explicit DenseMatrix(int n) { alloc(n, n); }
    DenseMatrix(int h, int w) { alloc(h, w); }
    DenseMatrix(real_t *d, int h, int w) : data_(d), h_(h), w_(w), cap_(h * w), own_(false) {}
    DenseMatrix(const DenseMatrix &o)
    {
        alloc(o.h_, o.w_);
        if (cap_) std::memcpy(data_, o.data_, sizeof(real_t) * h_ * w_);
    }
    ~DenseMatrix()
    {
        if (own_) delete[] data_;
    }
    void SetSize(int n) { SetSize(n, n); }
    void SetSize(int h, int w)
    {
        if (h == h_ && w == w_) return;
        if (h * w <= cap_) { h_ = h; w_ = w; return; }
        alloc(h, w);
    }
    void UseExternalData(real_t *d, int h, int w)
    {
        if (own_) delete[] data_;
        data_ = d;
        h_ = h;
        w_ = w;
        cap_ = h * w;
        own_ = false;
    }
    void ClearExternalData()
    {
        if (!own_) { data_ = nullptr; h_ = w_ = cap_ = 0; }
    }
    int Height() const { return h_; }
    int Width() const { return w_; }
    int NumRows() const { return h_; }
    int NumCols() const { return w_; }
    real_t *GetData() const { return data_; }
    real_t *Data() const { return data_; }
    real_t &operator()(int i, int j) { return data_[i + (size_t)j * h_]; }
    const real_t &operator()(int i, int j) const { return data_[i + (size_t)j * h_]; }
    DenseMatrix &operator=(real_t c)
    {
        for (int i = 0; i < h_ * w_; i++) data_[i] = c;
        return *this;
    }
    DenseMatrix &operator=(const DenseMatrix &o)
    {
        if (this == &o) return *this;
        SetSize(o.h_, o.w_);
        std::memmove(data_, o.data_, sizeof(real_t) * h_ * w_);
        return *this;
    }
    DenseMatrix &operator*=(real_t c)
    {
        for (int i = 0; i < h_ * w_; i++) data_[i] *= c;
        return *this;
    }
    DenseMatrix &operator+=(const DenseMatrix &o)
    {
        for (int i = 0; i < h_ * w_; i++) data_[i] += o.data_[i];
        return *this;
    }
    void Neg()
    {
        for (int i = 0; i < h_ * w_; i++) data_[i] = -data_[i];
    }
    void GetRow(int r, Vector &row) const
    {
        row.SetSize(w_);
        for (int j = 0; j < w_; j++) row(j) = (*this)(r, j);
    }
    void SetRow(int r, const Vector &row)
    {
        for (int j = 0; j < w_; j++) (*this)(r, j) = row(j);
    }
    void SetRow(int r, real_t c)
    {
        for (int j = 0; j < w_; j++) (*this)(r, j) = c;
    }
    void GetColumn(int c, Vector &col) const
    {
        col.SetSize(h_);
        for (int i = 0; i < h_; i++) col(i) = (*this)(i, c);
    }
    void SetCol(int c, const Vector &col)
    {
        for (int i = 0; i < h_; i++) (*this)(i, c) = col(i);
    }
    void SetCol(int c, real_t v)
    {
        for (int i = 0; i < h_; i++) (*this)(i, c) = v;
    }
    void GetColumnReference(int c, Vector &col) { col.SetDataAndSize(data_ + (size_t)c * h_, h_); }
    // y = A x, columns visited in order
    void Mult(const real_t *x, real_t *y) const
    {
        for (int i = 0; i < h_; i++) y[i] = 0.0;
        for (int j = 0; j < w_; j++)
            for (int i = 0; i < h_; i++) y[i] += x[j] * (*this)(i, j);
    }
    void Mult(const Vector &x, Vector &y) const
    {
        y.SetSize(h_);
        Mult(x.GetData(), y.GetData());
    }
    void AddMult(const Vector &x, Vector &y) const
    {
        for (int j = 0; j < w_; j++)
            for (int i = 0; i < h_; i++) y(i) += x(j) * (*this)(i, j);
    }
    // y = A^T x
    void MultTranspose(const Vector &x, Vector &y) const
    {
        y.SetSize(w_);
        for (int j = 0; j < w_; j++) {
            real_t s = 0.0;
            for (int i = 0; i < h_; i++) s += x(i) * (*this)(i, j);
            y(j) = s;
        }
    }
    void Transpose()
    {
        std::vector<real_t> t((size_t)h_ * w_);
        for (int i = 0; i < h_; i++)
            for (int j = 0; j < w_; j++) t[j + (size_t)i * w_] = (*this)(i, j);
        std::swap(h_, w_);
        std::memcpy(data_, t.data(), sizeof(real_t) * h_ * w_);
    }
    // In-place inverse by Gauss-Jordan elimination with partial pivoting.
    void Invert()
    {
        const int n = h_;
        std::vector<real_t> A((size_t)n * n), I((size_t)n * n, 0.0);
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) A[(size_t)i * n + j] = (*this)(i, j);
        for (int i = 0; i < n; i++) I[(size_t)i * n + i] = 1.0;
        for (int c = 0; c < n; c++) {
            int p = c;
            for (int r = c + 1; r < n; r++)
                if (std::abs(A[(size_t)r * n + c]) > std::abs(A[(size_t)p * n + c])) p = r;
            if (p != c)
                for (int k = 0; k < n; k++) {
                    std::swap(A[(size_t)p * n + k], A[(size_t)c * n + k]);
                    std::swap(I[(size_t)p * n + k], I[(size_t)c * n + k]);
                }
            const real_t inv = 1.0 / A[(size_t)c * n + c];
            for (int k = 0; k < n; k++) {
                A[(size_t)c * n + k] *= inv;
                I[(size_t)c * n + k] *= inv;
            }
            for (int r = 0; r < n; r++) {
                if (r == c) continue;
                const real_t f = A[(size_t)r * n + c];
                if (f == 0.0) continue;
                for (int k = 0; k < n; k++) {
                    A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
                    I[(size_t)r * n + k] -= f * I[(size_t)c * n + k];
                }
            }
        }
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) (*this)(i, j) = I[(size_t)i * n + j];
    }
    real_t Weight() const
    {
        if (h_ == w_) {
            if (h_ == 1) return data_[0];
            if (h_ == 2) return (*this)(0, 0) * (*this)(1, 1) - (*this)(0, 1) * (*this)(1, 0);
            const DenseMatrix &a = *this;
            return a(0, 0) * (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) - a(0, 1) * (a(1, 0) * a(2, 2) - a(1, 2) * a(2, 0)) +
                   a(0, 2) * (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0));
        }
        return 0.0;
    }
};

// VWt += a * v w^T
inline void AddMult_a_VWt(const real_t a, const Vector &v, const Vector &w, DenseMatrix &VWt)
{
    for (int j = 0; j < w.Size(); j++) {
        const real_t awj = a * w(j);
        for (int i = 0; i < v.Size(); i++) VWt(i, j) += awj * v(i);
    }
}
// ABt = A B^T
inline void MultABt(const DenseMatrix &A, const DenseMatrix &B, DenseMatrix &ABt)
{
    ABt.SetSize(A.Height(), B.Height());
    for (int i = 0; i < A.Height(); i++)
        for (int j = 0; j < B.Height(); j++) {
            real_t s = 0.0;
            for (int k = 0; k < A.Width(); k++) s += A(i, k) * B(j, k);
            ABt(i, j) = s;
        }
}
// a = b c
inline void Mult(const DenseMatrix &b, const DenseMatrix &c, DenseMatrix &a)
{
    a.SetSize(b.Height(), c.Width());
    for (int i = 0; i < b.Height(); i++)
        for (int j = 0; j < c.Width(); j++) {
            real_t s = 0.0;
            for (int k = 0; k < b.Width(); k++) s += b(i, k) * c(k, j);
            a(i, j) = s;
        }
}
// Normal of a face from its Jacobian: 2D rotates the tangent, 3D takes the
// cross product of the two tangents; |n| is the face measure.
inline void CalcOrtho(const DenseMatrix &J, Vector &n)
{
    if (J.Height() == 2) {
        n(0) = J(1, 0);
        n(1) = -J(0, 0);
    } else {
        n(0) = J(1, 0) * J(2, 1) - J(2, 0) * J(1, 1);
        n(1) = J(2, 0) * J(0, 1) - J(0, 0) * J(2, 1);
        n(2) = J(0, 0) * J(1, 1) - J(1, 0) * J(0, 1);
    }
}

// Column-major 3-tensor with k-slices returned as matrix views.
class DenseTensor {
    std::vector<real_t> d_;
    int I_ = 0, J_ = 0, K_ = 0;
    std::vector<DenseMatrix> slices_;

public:
    void SetSize(int i, int j, int k)
    {
        I_ = i;
        J_ = j;
        K_ = k;
        d_.assign((size_t)i * j * k, 0.0);
        slices_.clear();
        slices_.reserve(k);
        for (int s = 0; s < k; s++) slices_.emplace_back(d_.data() + (size_t)s * i * j, i, j);
    }
    DenseMatrix &operator()(int k) { return slices_[k]; }
    const DenseMatrix &operator()(int k) const { return slices_[k]; }
    int SizeI() const { return I_; }
    int SizeJ() const { return J_; }
    int SizeK() const { return K_; }
};

struct Connection;
class Table {
    std::vector<std::vector<int>> rows_;

public:
    Table() {}
    Table(int nrows, Array<Connection> &list);
    int Size() const { return (int)rows_.size(); }
    void GetRow(int i, Array<int> &row) const
    {
        row.SetSize((int)rows_[i].size());
        for (int j = 0; j < row.Size(); j++) row[j] = rows_[i][j];
    }
};
struct Connection {
    int from, to;
    Connection() : from(0), to(0) {}
    Connection(int f, int t) : from(f), to(t) {}
    bool operator<(const Connection &o) const { return from < o.from || (from == o.from && to < o.to); }
    bool operator==(const Connection &o) const { return from == o.from && to == o.to; }
};

struct Quadrature1D {
    enum { GaussLegendre = 0, GaussLobatto = 1 };
};
struct BasisType {
    enum { GaussLegendre = 0, GaussLobatto = 1 };
    static void CheckNodal(int) {}
};

struct Geometry {
    enum Type { INVALID = -1, POINT = 0, SEGMENT, TRIANGLE, SQUARE, TETRAHEDRON, CUBE, PRISM, PYRAMID };
};

class IntegrationPoint {
public:
    real_t x = 0, y = 0, z = 0, weight = 0;
    int index = 0;
    void Get(real_t *p, int dim) const
    {
        p[0] = x;
        if (dim > 1) p[1] = y;
        if (dim > 2) p[2] = z;
    }
    void Set(const real_t *p, int dim)
    {
        x = p[0];
        if (dim > 1) y = p[1];
        if (dim > 2) z = p[2];
    }
};

class IntegrationRule {
    std::vector<IntegrationPoint> pts_;

public:
    IntegrationRule() {}
    explicit IntegrationRule(int n) : pts_(n) {}
    int GetNPoints() const { return (int)pts_.size(); }
    int Size() const { return (int)pts_.size(); }
    IntegrationPoint &IntPoint(int i) { return pts_[i]; }
    const IntegrationPoint &IntPoint(int i) const { return pts_[i]; }
    const IntegrationPoint *begin() const { return pts_.data(); }
    const IntegrationPoint *end() const { return pts_.data() + pts_.size(); }
    void SetSize(int n) { pts_.resize(n); }
};

// Gauss-Lobatto rule with n points on [0,1], mirrored about 1/2.
void StandInGaussLobatto(int n, std::vector<real_t> &x, std::vector<real_t> &w);

class IntegrationRules {
    int type_;
    std::vector<std::unique_ptr<IntegrationRule>> cache_;

public:
    IntegrationRules(int = 0, int type = Quadrature1D::GaussLegendre) : type_(type) {}
    const IntegrationRule &Get(int geom, int order);
};

// Lagrange basis through nodes x (n of them) at t: values L and derivatives dL.
inline void StandInLagrange(const std::vector<real_t> &x, real_t t, real_t *L, real_t *dL)
{
    const int n = (int)x.size();
    for (int j = 0; j < n; j++) {
        real_t v = 1.0, dv = 0.0;
        for (int m = 0; m < n; m++) {
            if (m == j) continue;
            real_t prod = 1.0 / (x[j] - x[m]);
            for (int q = 0; q < n; q++)
                if (q != j && q != m) prod *= (t - x[q]) / (x[j] - x[q]);
            dv += prod;
            v *= (t - x[m]) / (x[j] - x[m]);
        }
        L[j] = v;
        dL[j] = dv;
    }
}

// An element's map from [0,1]^dim: affine and axis-aligned (origin x0,
// extents h), or nodal — the degree-N interpolant of its DG nodes' physical
// coordinates X (X[k * dof + n], the LGL nodes x1d), whose Jacobian,
// adjugate and determinant are evaluated at the integration point set last,
// as MFEM's IsoparametricTransformation does for a curved mesh.
class ElementTransformation {
public:
    int ElementNo = 0;
    int dim = 2;
    real_t x0[3] = {0, 0, 0}, h[3] = {1, 1, 1};
    bool nodal = false;
    std::vector<real_t> X, x1d;
    DenseMatrix Jm, Adj;
    const IntegrationPoint *ip = nullptr;
    ElementTransformation() : Jm(3, 3), Adj(3, 3) {}
    void SetupNodal(int d, int e, const std::vector<real_t> &nodes1d, const real_t *coords, int ndof)
    {
        dim = d;
        ElementNo = e;
        nodal = true;
        x1d = nodes1d;
        X.assign(coords, coords + (size_t)d * ndof);
        Jm.SetSize(d, d);
        Adj.SetSize(d, d);
    }
    void EvalNodal(const IntegrationPoint &p)
    {
        const int Np = (int)x1d.size();
        std::vector<real_t> L[3], dL[3];
        real_t r[3] = {p.x, p.y, p.z};
        for (int q = 0; q < dim; q++) {
            L[q].assign(Np, 0.0);
            dL[q].assign(Np, 0.0);
            StandInLagrange(x1d, r[q], L[q].data(), dL[q].data());
        }
        int dof = 1;
        for (int q = 0; q < dim; q++) dof *= Np;
        Jm = 0.0;
        for (int n = 0; n < dof; n++) {
            const int idx[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
            for (int c = 0; c < dim; c++) {
                real_t g = 1.0;
                for (int q = 0; q < dim; q++) g *= q == c ? dL[q][idx[q]] : L[q][idx[q]];
                for (int k = 0; k < dim; k++) Jm(k, c) += g * X[(size_t)k * dof + n];
            }
        }
        if (dim == 2) {
            Adj(0, 0) = Jm(1, 1);
            Adj(0, 1) = -Jm(0, 1);
            Adj(1, 0) = -Jm(1, 0);
            Adj(1, 1) = Jm(0, 0);
        } else {
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
                    Adj(i, j) = Jm(j1, i1) * Jm(j2, i2) - Jm(j1, i2) * Jm(j2, i1);
                }
        }
    }
    void Setup(int d, int e, const real_t *origin, const real_t *hh)
    {
        dim = d;
        ElementNo = e;
        Jm.SetSize(d, d);
        Adj.SetSize(d, d);
        Jm = 0.0;
        Adj = 0.0;
        for (int i = 0; i < d; i++) {
            x0[i] = origin[i];
            h[i] = hh[i];
            Jm(i, i) = hh[i];
        }
        if (d == 2) {
            Adj(0, 0) = Jm(1, 1);
            Adj(1, 1) = Jm(0, 0);
        } else {
            Adj(0, 0) = Jm(1, 1) * Jm(2, 2);
            Adj(1, 1) = Jm(0, 0) * Jm(2, 2);
            Adj(2, 2) = Jm(0, 0) * Jm(1, 1);
        }
    }
    void SetIntPoint(const IntegrationPoint *p)
    {
        ip = p;
        if (nodal) EvalNodal(*p);
    }
    const IntegrationPoint &GetIntPoint() const { return *ip; }
    real_t Weight() { return Jm.Weight(); }
    const DenseMatrix &Jacobian() { return Jm; }
    const DenseMatrix &AdjugateJacobian() { return Adj; }
    void Transform(const IntegrationPoint &p, Vector &phys)
    {
        phys.SetSize(dim);
        real_t r[3] = {p.x, p.y, p.z};
        if (!nodal) {
            for (int i = 0; i < dim; i++) phys(i) = x0[i] + h[i] * r[i];
            return;
        }
        const int Np = (int)x1d.size();
        std::vector<real_t> L[3], dL[3];
        for (int q = 0; q < dim; q++) {
            L[q].assign(Np, 0.0);
            dL[q].assign(Np, 0.0);
            StandInLagrange(x1d, r[q], L[q].data(), dL[q].data());
        }
        int dof = 1;
        for (int q = 0; q < dim; q++) dof *= Np;
        for (int i = 0; i < dim; i++) phys(i) = 0.0;
        for (int n = 0; n < dof; n++) {
            const int idx[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
            real_t g = 1.0;
            for (int q = 0; q < dim; q++) g *= L[q][idx[q]];
            for (int i = 0; i < dim; i++) phys(i) += g * X[(size_t)i * dof + n];
        }
    }
};

// Face between element 1 and element 2 of an axis-aligned Cartesian mesh.
// Face point (s0[, s1]) sits at tangential coordinates (s0, s1) of both
// elements; the face Jacobian is oriented so CalcOrtho points out of element 1.
// General faces (nodal elements): element 1's face f1 = 2 d + side in its own
// frame, element 2's face f2 and the orientation o of the neighbour's
// tangential coordinates (swap if o & 1, then a -> 1 - a if o & 2, b -> 1 - b
// if o & 4); the face Jacobian is element 1's tangent columns at the point,
// ordered so that CalcOrtho points out of element 1, as MFEM orients it.
class FaceElementTransformations {
public:
    int Elem1No = 0, Elem2No = 0, ElementNo = 0;
    int dim = 2, dir = 0;
    int side1 = 1;  // 1: element 1's +dir face, 0: its -dir face
    bool general = false;
    int f2 = 0, orient = 0;
    ElementTransformation T1, T2;
    IntegrationPoint ip1, ip2;
    DenseMatrix FJ;
    void SetAllIntPointsGeneral(const IntegrationPoint *fp)
    {
        const int d1 = dir, d2 = f2 / 2, s2 = f2 % 2;
        real_t t[2] = {fp->x, dim == 3 ? fp->y : 0.0};
        real_t p1[3] = {0, 0, 0}, p2[3] = {0, 0, 0};
        int q = 0;
        for (int d = 0; d < dim; d++) p1[d] = d == d1 ? (side1 ? 1.0 : 0.0) : t[q++];
        real_t a = t[0], b = t[1];
        if (orient & 1) std::swap(a, b);
        if (orient & 2) a = 1.0 - a;
        if (orient & 4) b = 1.0 - b;
        real_t u[2] = {a, b};
        q = 0;
        for (int d = 0; d < dim; d++) p2[d] = d == d2 ? (s2 ? 1.0 : 0.0) : u[q++];
        ip1.Set(p1, dim);
        ip2.Set(p2, dim);
        T1.SetIntPoint(&ip1);
        if (Elem2No >= 0) T2.SetIntPoint(&ip2);
        const DenseMatrix &J = T1.Jacobian();
        if (dim == 2) {
            FJ.SetSize(2, 1);
            const int c = d1 == 0 ? 1 : 0;
            const real_t sg = (d1 == 0) == (side1 == 1) ? 1.0 : -1.0;
            FJ(0, 0) = sg * J(0, c);
            FJ(1, 0) = sg * J(1, c);
        } else {
            FJ.SetSize(3, 2);
            int c0 = (d1 + 1) % 3, c1 = (d1 + 2) % 3;
            if (!side1) std::swap(c0, c1);
            for (int k = 0; k < 3; k++) {
                FJ(k, 0) = J(k, c0);
                FJ(k, 1) = J(k, c1);
            }
        }
    }
    void SetAllIntPoints(const IntegrationPoint *fp)
    {
        if (general) return SetAllIntPointsGeneral(fp);
        real_t t[2] = {fp->x, fp->y};
        real_t p1[3], p2[3];
        int q = 0;
        for (int d = 0; d < dim; d++) {
            if (d == dir) {
                p1[d] = side1 ? 1.0 : 0.0;
                p2[d] = side1 ? 0.0 : 1.0;
            } else {
                p1[d] = p2[d] = t[q++];
            }
        }
        ip1.Set(p1, dim);
        ip2.Set(p2, dim);
        T1.SetIntPoint(&ip1);
        T2.SetIntPoint(&ip2);
    }
    ElementTransformation &GetElement1Transformation() { return T1; }
    ElementTransformation &GetElement2Transformation() { return T2; }
    const IntegrationPoint &GetElement1IntPoint() { return ip1; }
    const IntegrationPoint &GetElement2IntPoint() { return ip2; }
    const DenseMatrix &Jacobian() { return FJ; }
    // physical point of the face point set by SetAllIntPoints
    void Transform(const IntegrationPoint &, Vector &phys) { T1.Transform(ip1, phys); }
};

// Scalar function of the physical point (boundary data).
class FunctionCoefficient {
public:
    FunctionCoefficient(std::function<real_t(const Vector &)> f) : F(std::move(f)) {}
    void SetTime(real_t tt) { t = tt; }
    template <class Tr> real_t Eval(Tr &T, const IntegrationPoint &ip)
    {
        Vector x;
        T.Transform(ip, x);
        return F(x);
    }

private:
    std::function<real_t(const Vector &)> F;
    real_t t = 0.0;
};

// Vector-valued function of the physical point (boundary states).
class VectorFunctionCoefficient {
public:
    VectorFunctionCoefficient(int vd, std::function<void(const Vector &, Vector &)> f) : vdim(vd), F(std::move(f)) {}
    void SetTime(real_t tt) { t = tt; }
    template <class Tr> void Eval(Vector &V, Tr &T, const IntegrationPoint &ip)
    {
        Vector x;
        T.Transform(ip, x);
        V.SetSize(vdim);
        F(x, V);
    }

private:
    int vdim;
    std::function<void(const Vector &, Vector &)> F;
    real_t t = 0.0;
};

class FiniteElement {
public:
    int dim = 2, order = 1, dof = 0;
    Geometry::Type geom = Geometry::SQUARE;
    std::vector<real_t> nodes1d;
    IntegrationRule nodes;
    int GetDof() const { return dof; }
    int GetOrder() const { return order; }
    Geometry::Type GetGeomType() const { return geom; }
    const IntegrationRule &GetNodes() const { return nodes; }
    // Tensor-product Lagrange basis through the 1D Gauss-Lobatto nodes.
    void CalcShape(const IntegrationPoint &ip, Vector &shape) const
    {
        const int Np = order + 1;
        std::vector<real_t> L[3];
        real_t r[3] = {ip.x, ip.y, ip.z};
        for (int d = 0; d < dim; d++) {
            L[d].assign(Np, 1.0);
            for (int j = 0; j < Np; j++)
                for (int k = 0; k < Np; k++)
                    if (k != j) L[d][j] *= (r[d] - nodes1d[k]) / (nodes1d[j] - nodes1d[k]);
        }
        shape.SetSize(dof);
        for (int n = 0; n < dof; n++) {
            int i = n % Np, j = (n / Np) % Np, k = n / (Np * Np);
            real_t s = L[0][i];
            if (dim > 1) s *= L[1][j];
            if (dim > 2) s *= L[2][k];
            shape(n) = s;
        }
    }
};

class DG_FECollection {
    FiniteElement fe_;
    int btype_;

public:
    DG_FECollection(int order, int dim, int btype = BasisType::GaussLobatto);
    const FiniteElement *FiniteElementForGeometry(Geometry::Type) const { return &fe_; }
    int GetBasisType() const { return btype_; }
};

struct Poly_1D {
    // Shifted Legendre polynomials on [0,1] by the three-term recurrence.
    static void CalcLegendre(const int p, const real_t x, real_t *u)
    {
        real_t z;
        u[0] = 1.0;
        if (p == 0) return;
        u[1] = z = 2.0 * x - 1.0;
        for (int n = 1; n < p; n++) u[n + 1] = ((2 * n + 1) * z * u[n] - n * u[n - 1]) / (n + 1);
    }
    static void CalcLegendre(const int p, const real_t x, real_t *u, real_t *d)
    {
        CalcLegendre(p, x, u);
        d[0] = 0.0;
        for (int n = 1; n <= p; n++) d[n] = 0.0;  // derivatives are not used here
    }
};

class Mesh {
public:
    int dim = 2, ne = 0;
    std::vector<ElementTransformation> T;
    int GetNE() const { return ne; }
    int Dimension() const { return dim; }
    int SpaceDimension() const { return dim; }
    int GetNBE() const { return 0; }
    void GetBdrElementAdjacentElement(int, int &e, int &info) const { e = -1; info = 0; }
    ElementTransformation *GetElementTransformation(int e) { return &T[e]; }
    int GetBdrAttribute(int) const { return 1; }
    FaceElementTransformations *GetBdrFaceTransformations(int) { return nullptr; }
    Array<int> bdr_attributes;
};
typedef Mesh ParMesh;

class ParFiniteElementSpace {
public:
    Mesh *mesh = nullptr;
    const FiniteElement *fe = nullptr;
    int vdim = 1;
    int ndof = 1;  // dofs per element
    int GetVDim() const { return vdim; }
    int GetNE() const { return mesh->ne; }
    Mesh *GetMesh() const { return mesh; }
    const FiniteElement *GetFE(int) const { return fe; }
    int GetElementOrder(int) const { return fe->order; }
    int GetNDofs() const { return mesh->ne * ndof; }
    int GetVSize() const { return vdim * GetNDofs(); }
    int GetTrueVSize() const { return GetVSize(); }
    ElementTransformation *GetElementTransformation(int e) const { return &mesh->T[e]; }
    void GetElementDofs(int e, Array<int> &dofs) const
    {
        dofs.SetSize(ndof);
        for (int i = 0; i < ndof; i++) dofs[i] = e * ndof + i;
    }
    // byNODES: all dofs of component 0, then component 1, ...
    void GetElementVDofs(int e, Array<int> &vdofs) const
    {
        vdofs.SetSize(ndof * vdim);
        for (int v = 0; v < vdim; v++)
            for (int i = 0; i < ndof; i++) vdofs[v * ndof + i] = v * GetNDofs() + e * ndof + i;
    }
    void GetElementVDofs(int e, Array<int> &vdofs, int) const { GetElementVDofs(e, vdofs); }
    void GetFaceNbrElementVDofs(int, Array<int> &) const {}
    const FiniteElement *GetFaceNbrFE(int) const { return fe; }
};
typedef ParFiniteElementSpace FiniteElementSpace;

class ParGridFunction : public Vector {
public:
    ParGridFunction() {}
    explicit ParGridFunction(ParFiniteElementSpace *f) : Vector(f->GetVSize()) {}
    ParGridFunction &operator=(const Vector &v)
    {
        Vector::operator=(v);
        return *this;
    }
    ParGridFunction &operator=(real_t c)
    {
        Vector::operator=(c);
        return *this;
    }
    void ExchangeFaceNbrData() {}
    Vector &FaceNbrData() { return *this; }
};
typedef ParGridFunction GridFunction;

class NonlinearFormIntegrator {
public:
    virtual ~NonlinearFormIntegrator() = default;
    virtual void AssembleElementVector(const FiniteElement &, ElementTransformation &, const Vector &, Vector &) {}
    virtual void AssembleFaceVector(const FiniteElement &, const FiniteElement &, FaceElementTransformations &,
                                    const Vector &, Vector &)
    {
    }
};

// Base of NavierStokesFlux: only the members and hooks its sources touch.
class FluxFunction {
public:
    const int num_equations, dim;
    FluxFunction(int neq, int d) : num_equations(neq), dim(d) {}
    virtual ~FluxFunction() = default;
};
class EulerFlux : public FluxFunction {
public:
    const real_t specific_heat_ratio;
    EulerFlux(int dim, real_t gamma) : FluxFunction(dim + 2, dim), specific_heat_ratio(gamma) {}
    real_t ComputeFlux(const Vector &, ElementTransformation &, DenseMatrix &) const { return 0.0; }
    real_t ComputeFluxDotN(const Vector &, const Vector &, FaceElementTransformations &, Vector &) const
    {
        return 0.0;
    }
};

// Declarations that Prandtl sources name but the pinned paths never run.
void Transpose(const Table &A, Table &At, int ncols_A = -1);
inline Table::Table(int nrows, Array<Connection> &list) : rows_(nrows)
{
    for (int i = 0; i < list.Size(); i++) rows_[list[i].from].push_back(list[i].to);
}

}  // namespace mfem
