// gb_math.cuh -- scalar policies and 3-vector / 3x3 algebra for the kernels.
//
// Every kernel is written once over a scalar type S:
//   float    FP32 bulk arithmetic of the mixed-precision mode;
//   double   FP64 with FMA contraction allowed (the fast all-FP64 mode);
//   dstrict  FP64 whose + - * / sqrt are the IEEE round-to-nearest
//            intrinsics, so the compiler cannot contract them into FMAs.
//            Written in the reference's operation order, dstrict arithmetic
//            reproduces the reference's CPU results bit for bit wherever no
//            transcendental function (pow, sin, cos, log) is involved.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define GB_HD __host__ __device__ __forceinline__
#define GB_D __device__ __forceinline__

namespace gb
{

struct dstrict
{
    double v;
    dstrict() = default;
    GB_HD constexpr dstrict(double x)
        : v(x)
    {
    }
    GB_HD explicit operator double() const
    {
        return v;
    }
};

GB_D dstrict operator+(dstrict a, dstrict b)
{
    return dstrict(__dadd_rn(a.v, b.v));
}
GB_D dstrict operator-(dstrict a, dstrict b)
{
    return dstrict(__dsub_rn(a.v, b.v));
}
GB_D dstrict operator*(dstrict a, dstrict b)
{
    return dstrict(__dmul_rn(a.v, b.v));
}
GB_D dstrict operator/(dstrict a, dstrict b)
{
    return dstrict(__ddiv_rn(a.v, b.v));
}
GB_D dstrict operator-(dstrict a)
{
    return dstrict(-a.v);
}
GB_D dstrict& operator+=(dstrict& a, dstrict b)
{
    a = a + b;
    return a;
}
GB_D dstrict& operator-=(dstrict& a, dstrict b)
{
    a = a - b;
    return a;
}
GB_D dstrict& operator*=(dstrict& a, dstrict b)
{
    a = a * b;
    return a;
}
GB_D dstrict& operator/=(dstrict& a, dstrict b)
{
    a = a / b;
    return a;
}
GB_D bool operator<(dstrict a, dstrict b)
{
    return a.v < b.v;
}
GB_D bool operator>(dstrict a, dstrict b)
{
    return a.v > b.v;
}
GB_D bool operator<=(dstrict a, dstrict b)
{
    return a.v <= b.v;
}
GB_D bool operator>=(dstrict a, dstrict b)
{
    return a.v >= b.v;
}
GB_D bool operator==(dstrict a, dstrict b)
{
    return a.v == b.v;
}
GB_D bool operator!=(dstrict a, dstrict b)
{
    return a.v != b.v;
}

// ---- scalar functions, overloaded per policy -------------------------------
GB_D float s_sqrt(float x)
{
    return sqrtf(x);
}
GB_D double s_sqrt(double x)
{
    return sqrt(x);
}
GB_D dstrict s_sqrt(dstrict x)
{
    return dstrict(__dsqrt_rn(x.v));
}
GB_D float s_fabs(float x)
{
    return fabsf(x);
}
GB_D double s_fabs(double x)
{
    return fabs(x);
}
GB_D dstrict s_fabs(dstrict x)
{
    return dstrict(fabs(x.v));
}
GB_D float s_pow(float x, float y)
{
    return powf(x, y);
}
GB_D double s_pow(double x, double y)
{
    return pow(x, y);
}
GB_D dstrict s_pow(dstrict x, dstrict y)
{
    return dstrict(pow(x.v, y.v));
}
GB_D float s_sin(float x)
{
    return sinf(x);
}
GB_D double s_sin(double x)
{
    return sin(x);
}
GB_D dstrict s_sin(dstrict x)
{
    return dstrict(sin(x.v));
}
GB_D float s_cos(float x)
{
    return cosf(x);
}
GB_D double s_cos(double x)
{
    return cos(x);
}
GB_D dstrict s_cos(dstrict x)
{
    return dstrict(cos(x.v));
}
GB_D float s_copysign(float a, float b)
{
    return copysignf(a, b);
}
GB_D double s_copysign(double a, double b)
{
    return copysign(a, b);
}
GB_D dstrict s_copysign(dstrict a, dstrict b)
{
    return dstrict(copysign(a.v, b.v));
}
GB_D double to_d(float x)
{
    return (double)x;
}
GB_D double to_d(double x)
{
    return x;
}
GB_D double to_d(dstrict x)
{
    return x.v;
}

// storage type of a policy (what its arrays hold in memory)
template <typename S>
struct storage
{
    using type = S;
};
template <>
struct storage<dstrict>
{
    using type = double;
};
template <typename S>
using store_t = typename storage<S>::type;

template <typename S>
GB_D S from_store(store_t<S> x)
{
    return S(x);
}

// ---- constants: Grains/Base/include/Basic.hh:103-128, the double values.  The
// FP32 mode uses the same values (they are absolute SI thresholds; the
// reference's coarser float tolerances change the contact set) -------------
template <typename S>
GB_D S k_eps()
{
    return S(1e-10);
}
template <typename S>
GB_D S k_loweps()
{
    return S(1e-5);
}
template <typename S>
GB_D S k_higheps()
{
    return S(1e-15);
}
template <typename S>
GB_D S k_pi()
{
    return S(3.1415926535897932385);
}

// ---- 3-vectors -----------------------------------------------------------
template <typename S>
struct V3
{
    S x, y, z;
};

template <typename S>
GB_HD V3<S> mk(S x, S y, S z)
{
    V3<S> r;
    r.x = x;
    r.y = y;
    r.z = z;
    return r;
}
template <typename S>
GB_HD V3<S> zero3()
{
    return mk<S>(S(0.0), S(0.0), S(0.0));
}
template <typename S>
GB_D V3<S> operator+(const V3<S>& a, const V3<S>& b)
{
    return mk<S>(a.x + b.x, a.y + b.y, a.z + b.z);
}
template <typename S>
GB_D V3<S> operator-(const V3<S>& a, const V3<S>& b)
{
    return mk<S>(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <typename S>
GB_D V3<S> operator-(const V3<S>& a)
{
    return mk<S>(-a.x, -a.y, -a.z);
}
template <typename S>
GB_D V3<S> operator*(S d, const V3<S>& a)
{
    return mk<S>(d * a.x, d * a.y, d * a.z);
}
template <typename S>
GB_D V3<S> operator/(const V3<S>& a, S d)
{
    return mk<S>(a.x / d, a.y / d, a.z / d);
}
// dot product as VectorMath.hh:116-126: out = 0; out += a_i b_i
template <typename S>
GB_D S dot(const V3<S>& a, const V3<S>& b)
{
    S o = S(0.0);
    o   = o + a.x * b.x;
    o   = o + a.y * b.y;
    o   = o + a.z * b.z;
    return o;
}
template <typename S>
GB_D V3<S> cross(const V3<S>& a, const V3<S>& b)
{
    return mk<S>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename S>
GB_D S norm2(const V3<S>& a)
{
    return a.x * a.x + a.y * a.y + a.z * a.z;
}
template <typename S>
GB_D S norm(const V3<S>& a)
{
    return s_sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
}
template <typename S>
GB_D V3<S> round3(V3<S> a, S tol)
{
    a.x = s_fabs(a.x) < tol ? S(0.0) : a.x;
    a.y = s_fabs(a.y) < tol ? S(0.0) : a.y;
    a.z = s_fabs(a.z) < tol ? S(0.0) : a.z;
    return a;
}
template <typename S>
GB_D bool eq3(const V3<S>& a, const V3<S>& b)
{
    return a.x == b.x && a.y == b.y && a.z == b.z;
}
template <typename D, typename S>
GB_D V3<D> cvt3(const V3<S>& a)
{
    return mk<D>(D(to_d(a.x)), D(to_d(a.y)), D(to_d(a.z)));
}

// ---- 3x3 matrices, row-major m[9] (Grains Matrix3) ---------------------------
template <typename S>
struct M3
{
    S m[9];
};
// M v (MatrixMath.hh:127-138)
template <typename S>
GB_D V3<S> mul(const M3<S>& M, const V3<S>& v)
{
    return mk<S>(M.m[0] * v.x + M.m[1] * v.y + M.m[2] * v.z,
                 M.m[3] * v.x + M.m[4] * v.y + M.m[5] * v.z,
                 M.m[6] * v.x + M.m[7] * v.y + M.m[8] * v.z);
}
// v M = M^T v (MatrixMath.hh:144-155)
template <typename S>
GB_D V3<S> mul_t(const M3<S>& M, const V3<S>& v)
{
    return mk<S>(M.m[0] * v.x + M.m[3] * v.y + M.m[6] * v.z,
                 M.m[1] * v.x + M.m[4] * v.y + M.m[7] * v.z,
                 M.m[2] * v.x + M.m[5] * v.y + M.m[8] * v.z);
}
// A B (MatrixMath.hh:160-175)
template <typename S>
GB_D M3<S> mul(const M3<S>& A, const M3<S>& B)
{
    M3<S> C;
#pragma unroll
    for(int r = 0; r < 3; ++r)
#pragma unroll
        for(int c = 0; c < 3; ++c)
            C.m[3 * r + c] = A.m[3 * r] * B.m[c] + A.m[3 * r + 1] * B.m[3 + c]
                             + A.m[3 * r + 2] * B.m[6 + c];
    return C;
}
template <typename S>
GB_D M3<S> transpose(const M3<S>& A)
{
    M3<S> T;
    T.m[0] = A.m[0];
    T.m[1] = A.m[3];
    T.m[2] = A.m[6];
    T.m[3] = A.m[1];
    T.m[4] = A.m[4];
    T.m[5] = A.m[7];
    T.m[6] = A.m[2];
    T.m[7] = A.m[5];
    T.m[8] = A.m[8];
    return T;
}

// Rotation matrix of a unit quaternion (w, x, y, z).
template <typename S>
GB_D M3<S> quat_to_matrix(S w, S x, S y, S z)
{
    M3<S>   R;
    const S one = S(1.0), two = S(2.0);
    R.m[0] = one - two * (y * y + z * z);
    R.m[1] = two * (x * y - w * z);
    R.m[2] = two * (x * z + w * y);
    R.m[3] = two * (x * y + w * z);
    R.m[4] = one - two * (x * x + z * z);
    R.m[5] = two * (y * z - w * x);
    R.m[6] = two * (x * z - w * y);
    R.m[7] = two * (y * z + w * x);
    R.m[8] = one - two * (x * x + y * y);
    return R;
}

// Affine transform: basis + origin (Grains Transform3).
template <typename S>
struct Tr
{
    M3<S> R;
    V3<S> o;
};
template <typename S>
GB_D V3<S> apply(const Tr<S>& t, const V3<S>& v)
{
    return mul(t.R, v) + t.o; // Transform3::operator() (Transform3.cpp:334-337)
}

} // namespace gb
