// gb_dom.hh -- the document tree behind the Xerces-free ReaderXML
// (grains3dgpu_b200/xml/ReaderXML.cpp).
//
// Grains3D reads its input through ReaderXML (Grains/XML/include/
// ReaderXML.hh:21-110), whose signatures name four Xerces-C DOM types:
// DOMNode, DOMElement, DOMNodeList and DOMBuilder.  Outside ReaderXML the
// reference only calls DOMNodeList::getLength() and DOMNodeList::item(i)
// (Grains.cpp:142-209, :390-392; Insertion.cpp:50-52;
// ContactForceModelBuilderFactory.cpp:44-46).  These classes provide exactly
// that, over a plain tree parsed by gb::xml::parse, so that the reference's
// XML constructors build a simulation without Xerces.  The headers
// xercesc/dom/{DOMNode,DOMElement,DOMNodeList,DOMBuilder}.hpp in this
// directory include this one; put this directory first on the include path
// where Xerces' headers would be.
//
// The tree keeps what a Xerces DOM builder with default features keeps and
// the reference relies on: element and text children in document order,
// whitespace-only text between elements included (ConvexBuilderFactory
// takes the second child node of <Convex>, ReaderXML::getNodeNext), and
// attributes with entity references resolved.  Comments, processing
// instructions and the document type declaration are dropped.
#pragma once

#include <cstddef>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#define XERCES_CPP_NAMESPACE_USE
typedef std::size_t XMLSize_t;

class DOMNode;

// An ordered list of nodes that its owner keeps alive (Xerces' DOMNodeList).
class DOMNodeList
{
public:
    XMLSize_t getLength() const { return m_items.size(); }
    DOMNode*  item(XMLSize_t i) const { return i < m_items.size() ? m_items[i] : nullptr; }

    std::vector<DOMNode*> m_items;
};

class DOMNode
{
public:
    enum NodeType : short
    {
        ELEMENT_NODE = 1,
        TEXT_NODE    = 3
    };

    virtual ~DOMNode() = default;

    short                  getNodeType() const { return m_type; }
    // element: its tag; text node: "#text" (as in Xerces)
    std::string const&     getNodeName() const { return m_name; }
    // text node: its characters; element: empty
    std::string const&     getNodeValue() const { return m_value; }
    DOMNodeList const*     getChildNodes() const { return &m_children; }
    DOMNode*               getFirstChild() const { return m_children.item(0); }
    // the value of attribute `name`, or nullptr when the element has none
    std::string const*     getAttribute(std::string const& name) const
    {
        for(auto const& a : m_attrs)
            if(a.first == name)
                return &a.second;
        return nullptr;
    }

    short                                            m_type = ELEMENT_NODE;
    std::string                                      m_name;
    std::string                                      m_value;
    std::vector<std::pair<std::string, std::string>> m_attrs;
    DOMNodeList                                      m_children;      // element and text nodes
    std::vector<std::unique_ptr<DOMNode>>            m_owned;         // the same, owned
};

class DOMElement : public DOMNode
{
};

// Xerces' parser handle; ReaderXML keeps a pointer to one.
class DOMBuilder
{
};

namespace gb
{
namespace xml
{
// Parses an XML document; returns its root element, or nullptr with `error`
// set (line number and reason) when the text is not well-formed.
std::unique_ptr<DOMElement> parse(std::string const& text, std::string* error);

// All descendant elements of `root` named `name`, in document order (the
// element itself excluded), as Xerces' getElementsByTagName lists them.
void elements_by_tag(DOMNode const* root, std::string const& name, std::vector<DOMNode*>& out);
} // namespace xml
} // namespace gb
