// mfem_mock.hpp — the few MFEM declarations the adapter header uses, so the
// CPU tests can compile and link include/prandtl_b200_mfem.hpp without MFEM.
#pragma once
namespace mfem {
class Vector {
public:
    Vector(double *d, int n) : data_(d), size_(n) {}
    double *GetData() const { return data_; }
    int Size() const { return size_; }

private:
    double *data_;
    int size_;
};
class Operator {
public:
    explicit Operator(int s) : height(s), width(s) {}
    virtual ~Operator() {}
    virtual void Mult(const Vector &x, Vector &y) const = 0;
    int Height() const { return height; }

protected:
    int height, width;
};
class TimeDependentOperator : public Operator {
public:
    explicit TimeDependentOperator(int n, double t0 = 0.0) : Operator(n), t(t0) {}

protected:
    double t;
};
class ODESolver {
public:
    virtual ~ODESolver() {}
    virtual void Init(TimeDependentOperator &f_) { f = &f_; }
    virtual void Step(Vector &x, double &t, double &dt) = 0;

protected:
    TimeDependentOperator *f = nullptr;
};
}  // namespace mfem
