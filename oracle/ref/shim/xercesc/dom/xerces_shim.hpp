// Minimal stand-ins for the Xerces-C DOM types named by the reference's
// headers (Grains/XML/include/ReaderXML.hh:4-8).  Xerces itself is absent; the
// harness never parses XML, so these only need to declare the names.
#pragma once
#include <cstddef>
#define XERCES_CPP_NAMESPACE_USE
typedef std::size_t XMLSize_t;
class DOMNode
{
public:
    virtual ~DOMNode() {}
};
class DOMElement : public DOMNode
{
};
class DOMNodeList
{
public:
    XMLSize_t getLength() const { return 0; }
    DOMNode*  item(XMLSize_t) const { return nullptr; }
};
class DOMBuilder
{
};
