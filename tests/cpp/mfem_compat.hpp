// Minimal signatures of mfem::Vector / Operator / TimeDependentOperator, enough
// to compile the DGSEMOperatorGPU adapter where MFEM is not installed.
#pragma once
#include <vector>
namespace mfem {
class Vector {
    std::vector<double> d_;
public:
    Vector() = default;
    explicit Vector(int n) : d_(n) {}
    int Size() const { return (int)d_.size(); }
    double *GetData() const { return const_cast<double *>(d_.data()); }
    double &operator()(int i) { return d_[i]; }
};
class Operator {
protected:
    int height, width;
public:
    explicit Operator(int s = 0) : height(s), width(s) {}
    virtual ~Operator() = default;
    int Height() const { return height; }
    virtual void Mult(const Vector &x, Vector &y) const = 0;
};
class TimeDependentOperator : public Operator {
protected:
    double t = 0.0;
public:
    explicit TimeDependentOperator(int n = 0) : Operator(n) {}
    virtual void SetTime(const double t_) { t = t_; }
    double GetTime() const { return t; }
};
}   // namespace mfem
