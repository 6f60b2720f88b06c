// Minimal stand-in for the reference's missing `ks/maths.h` (an empty git
// submodule in the reference checkout): the Eigen vector/matrix subset that
// the reference's hot-path sources use, written from scratch so that those
// sources compile unmodified for the oracle build (oracle/Makefile).
//
// Evaluation is eager and coefficient by coefficient, with the operation
// order of oracle/dmap_oracle.h: dot = (a0*b0 + a1*b1) + a2*b2, M*v row by
// row in the same order, 2x2 inverse through 1/det, 3x3 inverse by cofactors.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>

namespace Eigen
{

template <typename T, int R, int C>
struct Matrix;

template <typename T, int R, int C>
struct ColRef
{
    Matrix<T, R, C> *m;
    int j;
    template <int R2>
    ColRef &operator=(const Matrix<T, R2, 1> &v)
    {
        for (int i = 0; i < R; ++i)
            (*m)(i, j) = v[i];
        return *this;
    }
    operator Matrix<T, R, 1>() const
    {
        Matrix<T, R, 1> v;
        for (int i = 0; i < R; ++i)
            v[i] = (*m)(i, j);
        return v;
    }
};

template <typename T, int R, int C>
struct Matrix
{
    T v[R * C]; // column major

    Matrix() : v{} {}
    Matrix(T x, T y)
    {
        static_assert(R * C == 2, "two coefficients");
        v[0] = x;
        v[1] = y;
    }
    Matrix(T x, T y, T z)
    {
        static_assert(R * C == 3, "three coefficients");
        v[0] = x;
        v[1] = y;
        v[2] = z;
    }
    Matrix(const ColRef<T, R, 1> &) = delete;

    static Matrix Zero() { return Matrix(); }
    static Matrix Constant(T c)
    {
        Matrix m;
        for (int k = 0; k < R * C; ++k)
            m.v[k] = c;
        return m;
    }
    static Matrix UnitX()
    {
        Matrix m;
        m.v[0] = T(1);
        return m;
    }
    static Matrix UnitY()
    {
        Matrix m;
        m.v[1] = T(1);
        return m;
    }

    T &operator[](int k) { return v[k]; }
    const T &operator[](int k) const { return v[k]; }
    T &operator()(int i, int j) { return v[j * R + i]; }
    const T &operator()(int i, int j) const { return v[j * R + i]; }
    T &coeffRef(int i, int j) { return (*this)(i, j); }
    T coeff(int i, int j) const { return (*this)(i, j); }
    T x() const { return v[0]; }
    T y() const { return v[1]; }
    T z() const { return v[2]; }

    ColRef<T, R, C> col(int j) { return ColRef<T, R, C>{this, j}; }
    Matrix<T, R, 1> col(int j) const
    {
        Matrix<T, R, 1> c;
        for (int i = 0; i < R; ++i)
            c[i] = (*this)(i, j);
        return c;
    }
    struct RowView
    {
        Matrix<T, C, 1> r;
        Matrix<T, C, 1> transpose() const { return r; }
    };
    RowView row(int i) const
    {
        RowView rv;
        for (int j = 0; j < C; ++j)
            rv.r[j] = (*this)(i, j);
        return rv;
    }

    // Reductions over all coefficients, left to right.
    T sum() const
    {
        T s = v[0];
        for (int k = 1; k < R * C; ++k)
            s = s + v[k];
        return s;
    }
    T dot(const Matrix &b) const
    {
        T s = v[0] * b.v[0];
        for (int k = 1; k < R * C; ++k)
            s = s + v[k] * b.v[k];
        return s;
    }
    T squaredNorm() const { return dot(*this); }
    T norm() const { return std::sqrt(squaredNorm()); }
    Matrix normalized() const
    {
        T z = squaredNorm();
        if (z > T(0)) {
            T n = std::sqrt(z);
            Matrix r;
            for (int k = 0; k < R * C; ++k)
                r.v[k] = v[k] / n;
            return r;
        }
        return *this;
    }
    void normalize() { *this = normalized(); }
    Matrix cross(const Matrix &b) const
    {
        static_assert(R * C == 3, "cross of 3-vectors");
        return Matrix(v[1] * b.v[2] - v[2] * b.v[1], v[2] * b.v[0] - v[0] * b.v[2], v[0] * b.v[1] - v[1] * b.v[0]);
    }
    Matrix cwiseAbs() const
    {
        Matrix r;
        for (int k = 0; k < R * C; ++k)
            r.v[k] = std::abs(v[k]);
        return r;
    }
    Matrix cwiseMin(const Matrix &b) const
    {
        Matrix r;
        for (int k = 0; k < R * C; ++k)
            r.v[k] = std::min(v[k], b.v[k]);
        return r;
    }
    Matrix cwiseMax(const Matrix &b) const
    {
        Matrix r;
        for (int k = 0; k < R * C; ++k)
            r.v[k] = std::max(v[k], b.v[k]);
        return r;
    }
    Matrix cwiseMin(T b) const { return cwiseMin(Constant(b)); }
    Matrix cwiseMax(T b) const { return cwiseMax(Constant(b)); }
    Matrix cwiseProduct(const Matrix &b) const
    {
        Matrix r;
        for (int k = 0; k < R * C; ++k)
            r.v[k] = v[k] * b.v[k];
        return r;
    }
    T maxCoeff() const
    {
        T m = v[0];
        for (int k = 1; k < R * C; ++k)
            m = std::max(m, v[k]);
        return m;
    }
    T minCoeff() const
    {
        T m = v[0];
        for (int k = 1; k < R * C; ++k)
            m = std::min(m, v[k]);
        return m;
    }
    bool allFinite() const
    {
        for (int k = 0; k < R * C; ++k)
            if (!std::isfinite(v[k]))
                return false;
        return true;
    }
    template <typename U>
    Matrix<U, R, C> cast() const
    {
        Matrix<U, R, C> r;
        for (int k = 0; k < R * C; ++k)
            r.v[k] = (U)v[k];
        return r;
    }

    T determinant() const
    {
        static_assert(R == 2 && C == 2, "2x2 determinant");
        return (*this)(0, 0) * (*this)(1, 1) - (*this)(1, 0) * (*this)(0, 1);
    }
    Matrix inverse() const
    {
        Matrix r;
        if constexpr (R == 2 && C == 2) {
            T invdet = T(1) / determinant();
            r(0, 0) = (*this)(1, 1) * invdet;
            r(1, 0) = -(*this)(1, 0) * invdet;
            r(0, 1) = -(*this)(0, 1) * invdet;
            r(1, 1) = (*this)(0, 0) * invdet;
        } else {
            static_assert(R == 3 && C == 3, "2x2 or 3x3 inverse");
            auto cof = [&](int i, int j) {
                int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
                return (*this)(i1, j1) * (*this)(i2, j2) - (*this)(i1, j2) * (*this)(i2, j1);
            };
            T c0 = cof(0, 0), c1 = cof(1, 0), c2 = cof(2, 0);
            T det = (c0 * (*this)(0, 0) + c1 * (*this)(1, 0)) + c2 * (*this)(2, 0);
            T invdet = T(1) / det;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    r(i, j) = cof(j, i) * invdet;
        }
        return r;
    }

    Matrix operator-() const
    {
        Matrix r;
        for (int k = 0; k < R * C; ++k)
            r.v[k] = -v[k];
        return r;
    }
    Matrix &operator+=(const Matrix &b)
    {
        for (int k = 0; k < R * C; ++k)
            v[k] = v[k] + b.v[k];
        return *this;
    }
    Matrix &operator-=(const Matrix &b)
    {
        for (int k = 0; k < R * C; ++k)
            v[k] = v[k] - b.v[k];
        return *this;
    }
    Matrix &operator*=(T s)
    {
        for (int k = 0; k < R * C; ++k)
            v[k] = v[k] * s;
        return *this;
    }
    Matrix &operator/=(T s)
    {
        for (int k = 0; k < R * C; ++k)
            v[k] = v[k] / s;
        return *this;
    }
    bool operator==(const Matrix &b) const
    {
        for (int k = 0; k < R * C; ++k)
            if (!(v[k] == b.v[k]))
                return false;
        return true;
    }
    bool operator!=(const Matrix &b) const { return !(*this == b); }
};

template <typename T, int R, int C>
Matrix<T, R, C> operator+(Matrix<T, R, C> a, const Matrix<T, R, C> &b)
{
    return a += b;
}
template <typename T, int R, int C>
Matrix<T, R, C> operator-(Matrix<T, R, C> a, const Matrix<T, R, C> &b)
{
    return a -= b;
}
template <typename T, int R, int C>
Matrix<T, R, C> operator*(T s, const Matrix<T, R, C> &a)
{
    Matrix<T, R, C> r;
    for (int k = 0; k < R * C; ++k)
        r.v[k] = s * a.v[k];
    return r;
}
template <typename T, int R, int C>
Matrix<T, R, C> operator*(const Matrix<T, R, C> &a, T s)
{
    Matrix<T, R, C> r;
    for (int k = 0; k < R * C; ++k)
        r.v[k] = a.v[k] * s;
    return r;
}
template <typename T, int R, int C>
Matrix<T, R, C> operator/(const Matrix<T, R, C> &a, T s)
{
    Matrix<T, R, C> r;
    for (int k = 0; k < R * C; ++k)
        r.v[k] = a.v[k] / s;
    return r;
}
// Matrix products: coefficient (i, k) = sum over j, left to right.
template <typename T, int R, int K, int C>
Matrix<T, R, C> operator*(const Matrix<T, R, K> &a, const Matrix<T, K, C> &b)
{
    Matrix<T, R, C> r;
    for (int i = 0; i < R; ++i)
        for (int c = 0; c < C; ++c) {
            T s = a(i, 0) * b(0, c);
            for (int j = 1; j < K; ++j)
                s = s + a(i, j) * b(j, c);
            r(i, c) = s;
        }
    return r;
}

typedef Matrix<double, 2, 2> Matrix2d;
typedef Matrix<double, 3, 3> Matrix3d;
typedef Matrix<double, 2, 1> Vector2d;
typedef Matrix<double, 3, 1> Vector3d;
typedef Matrix<int, 3, 1> Vector3i;

} // namespace Eigen

namespace ks
{
using vec2d = Eigen::Matrix<double, 2, 1>;
using vec3d = Eigen::Matrix<double, 3, 1>;
using vec2 = Eigen::Matrix<float, 2, 1>;
using vec3 = Eigen::Matrix<float, 3, 1>;
using vec2i = Eigen::Matrix<int, 2, 1>;
using color3 = Eigen::Matrix<float, 3, 1>;
} // namespace ks
