// xml_drive -- TEST INFRASTRUCTURE: runs Grains3D from an XML input through
// the Xerces-free ReaderXML (grains3dgpu_b200/xml/ReaderXML.cpp), with the
// reference's own host path (GrainsCPU) or with GrainsB200
// (include/grains_b200_grains.hh), for tests/test_xml_cpu.py and
// tests/test_gpu_xml.py.
//
//   xml_drive tree FILE                 the parsed tree, one node per line
//   xml_drive materials FILE            material ids per particle / obstacle:
//                                       GrainsParameters' map (the fix)
//   xml_drive insert FILE OUT [--fix-insertion]
//                                       construction + insertion only (no GPU)
//   xml_drive run cpu|b200 FILE OUT [--no-fix-materials] [--fix-insertion]
//                                       the whole simulation
// OUT receives n (int64), then 12 n transform doubles (Transform3 buffer
// order), 6 n velocity doubles (v, omega) and 12 doubles per obstacle of the
// final state; stdout ends with one line "particles N contacts K".
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "GrainsCPU.hh"
#include "GrainsParameters.hh"
#include "ReaderXML.hh"

#include "grains_b200_grains.hh"

namespace
{
// ComponentManagerCPU::updateLinks clears one cell past the end of its cell
// list (ComponentManagerCPU.cpp:281-282); as in the harness, spare capacity
// keeps that write inside the allocation.
struct SpareCellsCPU : ComponentManagerCPU<double>
{
    SpareCellsCPU(uint np, uint no, uint nc)
        : ComponentManagerCPU<double>(np, no, nc)
    {
        this->m_cell.reserve(this->m_cell.size() + 4);
    }
};

struct ProbeCPU : GrainsCPU<double>
{
    ComponentManager<double>* components() const { return m_components; }
    // the host manager Construction made, rebuilt with spare cell capacity
    void spare_cells()
    {
        using GP = GrainsParameters<double>;
        auto* m  = new SpareCellsCPU(GP::m_numParticles, GP::m_numObstacles, GP::m_numCells);
        m->initializeParticles(m_components->getTransform());
        m->initializeObstacles(m_components->getTransformObstacles());
        delete m_components;
        m_components = m;
    }
};

int dump_tree(DOMNode const* n, int depth)
{
    if(n->getNodeType() == DOMNode::TEXT_NODE)
    {
        std::string t = n->getNodeValue();
        const size_t b = t.find_first_not_of(" \t\r\n");
        if(b == std::string::npos)
            std::printf("%*s#ws\n", 2 * depth, "");
        else
        {
            const size_t e = t.find_last_not_of(" \t\r\n");
            std::printf("%*s#text %s\n", 2 * depth, "", t.substr(b, e - b + 1).c_str());
        }
        return 0;
    }
    std::printf("%*s<%s", 2 * depth, "", n->getNodeName().c_str());
    for(auto const& a : n->m_attrs)
        std::printf(" %s=[%s]", a.first.c_str(), a.second.c_str());
    std::printf(">\n");
    DOMNodeList const* c = n->getChildNodes();
    for(XMLSize_t i = 0; i < c->getLength(); ++i)
        dump_tree(c->item(i), depth + 1);
    return 0;
}

int write_state(ComponentManager<double> const* cm, char const* out)
{
    const std::vector<Transform3<double>> tr  = cm->getTransform();
    const std::vector<Kinematics<double>> kin = cm->getVelocity();
    const std::vector<Transform3<double>> obs = cm->getTransformObstacles();
    std::ofstream                         f(out, std::ios::binary);
    const long long                       n = (long long)tr.size();
    f.write((char const*)&n, sizeof(n));
    auto put = [&](Transform3<double> const& t) {
        // the Transform3 buffer order: basis row-major, then the origin
        const Matrix3<double> m = t.getBasis();
        const Vector3<double> o = t.getOrigin();
        double                b[12];
        for(int r = 0; r < 3; ++r)
            for(int c = 0; c < 3; ++c)
                b[3 * r + c] = m[r][c];
        for(int k = 0; k < 3; ++k)
            b[9 + k] = o[k];
        f.write((char const*)b, sizeof(b));
    };
    for(auto const& t : tr)
        put(t);
    for(auto const& k : kin)
    {
        const Vector3<double> v = k.getTranslationalComponent(), w = k.getAngularComponent();
        const double          b[6] = {v[X], v[Y], v[Z], w[X], w[Y], w[Z]};
        f.write((char const*)b, sizeof(b));
    }
    for(auto const& t : obs)
        put(t);
    return f.good() ? 0 : 3;
}

bool has(int argc, char** argv, char const* flag)
{
    for(int i = 0; i < argc; ++i)
        if(std::strcmp(argv[i], flag) == 0)
            return true;
    return false;
}
} // namespace

int main(int argc, char** argv)
{
    if(argc < 3)
    {
        std::fprintf(stderr, "usage: xml_drive tree|materials|insert|run ...\n");
        return 2;
    }
    const std::string mode = argv[1];
    ReaderXML::initialize();
    try
    {
        if(mode == "tree")
        {
            DOMElement* root = ReaderXML::getRoot(argv[2]);
            if(!root)
                return 1;
            return dump_tree(root, 0);
        }
        if(mode == "materials")
        {
            DOMElement* root = ReaderXML::getRoot(argv[2]);
            if(!root)
                return 1;
            GrainsB200<double> g;
            g.initialize(root);
            std::vector<int32_t> p, o;
            GrainsB200<double>::materialIds(root, p, o);
            std::printf("particles");
            for(int32_t m : p)
                std::printf(" %d", m);
            std::printf("\nobstacles");
            for(int32_t m : o)
                std::printf(" %d", m);
            std::printf("\nmaterials %zu\n", GrainsParameters<double>::m_materialMap.size());
            return 0;
        }
        if(mode == "insert" && argc >= 4)
        {
            DOMElement* root = ReaderXML::getRoot(argv[2]);
            if(!root)
                return 1;
            GrainsB200<double>::Options o;
            o.fixInsertionWindow = has(argc, argv, "--fix-insertion");
            GrainsB200<double> g(o);
            g.initialize(root);
            std::vector<Transform3<double>> tr;
            std::vector<Kinematics<double>> kin;
            g.insert(tr, kin);
            const int rc = write_state(g.components(), argv[3]);
            std::printf("particles %zu contacts 0\n", tr.size());
            return rc;
        }
        if(mode == "run" && argc >= 5)
        {
            const std::string engine = argv[2];
            DOMElement*       root   = ReaderXML::getRoot(argv[3]);
            if(!root)
                return 1;
            if(engine == "cpu")
            {
                ProbeCPU g;
                g.initialize(root);
                g.spare_cells();
                g.simulate();
                g.finalize();
                const int rc = write_state(g.components(), argv[4]);
                std::printf("\nparticles %u contacts -1\n",
                            g.components()->getNumberOfParticles());
                return rc;
            }
            if(engine == "b200")
            {
                GrainsB200<double>::Options o;
                o.fixMaterialIds     = !has(argc, argv, "--no-fix-materials");
                o.fixInsertionWindow = has(argc, argv, "--fix-insertion");
                GrainsB200<double> g(o);
                g.initialize(root);
                g.simulate();
                g.finalize();
                const int rc = write_state(g.components(), argv[4]);
                std::printf("\nparticles %u contacts %lld\n",
                            g.components()->getNumberOfParticles(), g.contactsCounted());
                return rc;
            }
        }
    }
    catch(std::exception const& e)
    {
        std::fprintf(stderr, "xml_drive: %s\n", e.what());
        return 4;
    }
    std::fprintf(stderr, "xml_drive: bad arguments\n");
    return 2;
}
