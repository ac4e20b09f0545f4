// Compiles the reference's Matrix3.cpp where it lies.  Two of its members do
// not compile as shipped: scale() assigns through `this` in a const member
// (Grains/Geometry/src/Matrix3.cpp:155-166) and operator*=(Vector3) calls a
// 3-argument setValue that Matrix3 does not declare (Matrix3.cpp:224-231).
// Neither is on the DEM time-step path.  Explicit specializations declared
// before the reference definitions keep the reference's explicit
// instantiation (`template class Matrix3<T>;`) from instantiating them.
#include <cstdlib>

#include "Matrix3.hh"

template <>
void Matrix3<float>::scale(const Vector3<float>&) const
{
    std::abort();
}
template <>
void Matrix3<double>::scale(const Vector3<double>&) const
{
    std::abort();
}
template <>
Matrix3<float>& Matrix3<float>::operator*=(const Vector3<float>&)
{
    std::abort();
}
template <>
Matrix3<double>& Matrix3<double>::operator*=(const Vector3<double>&)
{
    std::abort();
}

#include "Matrix3.cpp"
