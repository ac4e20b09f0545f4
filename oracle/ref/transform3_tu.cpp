// Compiles the reference's Transform3.cpp where it lies.  Its XML constructor
// calls Matrix3::isRotation, which Matrix3 does not declare
// (Grains/Geometry/src/Transform3.cpp:73); the harness never builds a
// transform from XML, so that constructor is explicitly specialized away.
#include <cstdlib>

#include "Transform3.hh"

template <>
Transform3<float>::Transform3(DOMNode*)
{
    std::abort();
}
template <>
Transform3<double>::Transform3(DOMNode*)
{
    std::abort();
}

#include "Transform3.cpp"
