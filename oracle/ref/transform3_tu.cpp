// Compiles the reference's Transform3.cpp where it lies.  Its XML constructor
// calls Matrix3::isRotation, which Matrix3 does not declare
// (Grains/Geometry/src/Transform3.cpp:73), so that constructor is explicitly
// specialized here: the same steps (Transform3.cpp:44-96 -- origin from
// <Centre>, basis from <AngularPosition> as a 3x3 matrix, as angles in
// degrees, or no rotation) with the rotation check written out as an
// orthonormality test (|M M^T - I| and |det M - 1| below 1e-10).
#include <cmath>
#include <iostream>
#include <sstream>

#include "ReaderXML.hh"
#include "Transform3.hh"

namespace
{
template <typename T>
bool is_rotation(Matrix3<T> const& m)
{
    for(int r = 0; r < 3; ++r)
        for(int c = 0; c < 3; ++c)
        {
            double s = 0.0;
            for(int k = 0; k < 3; ++k)
                s += (double)m[r][k] * (double)m[c][k];
            if(std::fabs(s - (r == c ? 1.0 : 0.0)) > 1e-10)
                return false;
        }
    const double det = (double)m[0][0] * ((double)m[1][1] * m[2][2] - (double)m[1][2] * m[2][1])
                       - (double)m[0][1] * ((double)m[1][0] * m[2][2] - (double)m[1][2] * m[2][0])
                       + (double)m[0][2] * ((double)m[1][0] * m[2][1] - (double)m[1][1] * m[2][0]);
    return std::fabs(det - 1.0) <= 1e-10;
}

template <typename T>
void from_xml(Transform3<T>& t, DOMNode* root)
{
    DOMNode* pos = ReaderXML::getNode(root, "Centre");
    if(pos)
        t.setOrigin(Vector3<T>(T(ReaderXML::getNodeAttr_Double(pos, "X")),
                               T(ReaderXML::getNodeAttr_Double(pos, "Y")),
                               T(ReaderXML::getNodeAttr_Double(pos, "Z"))));
    DOMNode*          angPos = ReaderXML::getNode(root, "AngularPosition");
    const std::string type   = ReaderXML::getNodeAttr_String(angPos, "Type");
    if(type == "Matrix")
    {
        Matrix3<T>         mat;
        std::istringstream in(ReaderXML::getNodeValue_String(angPos));
        in >> mat;
        t.setBasis(mat);
        if(!is_rotation(mat))
        {
            std::cout << "A matrix in one of the AngularPosition XML nodes is"
                      << " not a rotation matrix !!!" << std::endl;
            std::exit(1);
        }
    }
    else if(type == "Angles")
        t.setBasis(RADS_PER_DEG<T> * T(ReaderXML::getNodeAttr_Double(angPos, "aX")),
                   RADS_PER_DEG<T> * T(ReaderXML::getNodeAttr_Double(angPos, "aY")),
                   RADS_PER_DEG<T> * T(ReaderXML::getNodeAttr_Double(angPos, "aZ")));
    else
        t.setBasis(T(0), T(0), T(0));
}
} // namespace

template <>
Transform3<float>::Transform3(DOMNode* root)
{
    from_xml(*this, root);
}
template <>
Transform3<double>::Transform3(DOMNode* root)
{
    from_xml(*this, root);
}

#include "Transform3.cpp"
