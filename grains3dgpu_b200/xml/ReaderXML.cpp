// ReaderXML.cpp -- Grains3D's XML reader (Grains/XML/include/ReaderXML.hh:21-110)
// without Xerces-C.
//
// The reference reads every input through the static methods of ReaderXML,
// implemented over a Xerces DOM builder (Grains/XML/src/ReaderXML.cpp).  This
// file implements the same methods, with the same meaning, over the tree of
// gb_dom.hh and a small parser of its own, so that Grains<T>::initialize
// (Grains/Base/src/Grains.cpp:37-401) and every XML constructor it calls
// (RigidBody, Convex builders, Transform3, LinkedCell parameters, contact
// force models, time integrators, insertion, post-processing writers) run on
// a machine without Xerces.  Build it in place of Grains/XML/src/ReaderXML.cpp,
// with this file's directory ahead of Xerces' on the include path (the DOM
// headers xercesc/dom/*.hpp here replace Xerces').
//
// Behaviour, method by method, against the reference's:
//   getNode(DOMElement*, name)   first descendant element with that tag
//                                (getElementsByTagName()->item(0))
//   getNode(DOMNode*, name)      first child element with that name
//   getNodeAttr_Double/Int       atof/atoi of the attribute's text
//   getNodeAttr_String           the attribute's text
//   hasNodeAttr                  whether the attribute exists
//   getNodeName                  the element's tag ("#text" for text)
//   getNodeNext                  the second child node, text included
//   getNodeValue_Double/String   the first child's text
//   getNodes(DOMElement*, name)  every descendant element with that tag
//   getNodes(DOMNode*)           the child elements
//   getRoot(file)                the document element, or NULL (with a
//                                message) when the file cannot be read or is
//                                not well-formed XML
// Where the reference dereferences a missing attribute or child (a null
// pointer), these throw std::runtime_error naming the element and the
// attribute instead.  Node lists and documents live until terminate().
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>

#include "ReaderXML.hh"

namespace gb
{
namespace xml
{
namespace
{
struct Parser
{
    std::string const& s;
    size_t             i = 0;
    std::string        err;

    explicit Parser(std::string const& text)
        : s(text)
    {
    }

    int line_at(size_t pos) const
    {
        int l = 1;
        for(size_t k = 0; k < pos && k < s.size(); ++k)
            l += s[k] == '\n';
        return l;
    }
    bool fail(std::string const& why)
    {
        if(err.empty())
            err = "line " + std::to_string(line_at(i)) + ": " + why;
        return false;
    }
    bool starts(char const* t) const { return s.compare(i, std::char_traits<char>::length(t), t) == 0; }
    static bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }
    static bool is_name_char(char c)
    {
        return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9') || c == '_'
               || c == '-' || c == '.' || c == ':' || (unsigned char)c >= 0x80;
    }
    void skip_space()
    {
        while(i < s.size() && is_space(s[i]))
            ++i;
    }
    bool skip_until(char const* end)
    {
        const size_t p = s.find(end, i);
        if(p == std::string::npos)
            return fail(std::string("unterminated construct, no '") + end + "'");
        i = p + std::char_traits<char>::length(end);
        return true;
    }
    // <!DOCTYPE ...> with an optional [internal subset]
    bool skip_doctype()
    {
        int depth = 0;
        for(; i < s.size(); ++i)
        {
            if(s[i] == '[')
                ++depth;
            else if(s[i] == ']')
                --depth;
            else if(s[i] == '>' && depth == 0)
            {
                ++i;
                return true;
            }
        }
        return fail("unterminated DOCTYPE");
    }
    bool name(std::string& out)
    {
        const size_t b = i;
        while(i < s.size() && is_name_char(s[i]))
            ++i;
        if(i == b)
            return fail("a name was expected");
        out.assign(s, b, i - b);
        return true;
    }
    // the characters of [b, e) with entity and character references resolved
    bool decode(size_t b, size_t e, std::string& out)
    {
        out.clear();
        for(size_t k = b; k < e; ++k)
        {
            if(s[k] != '&')
            {
                out += s[k];
                continue;
            }
            const size_t semi = s.find(';', k);
            if(semi == std::string::npos || semi > e)
                return fail("unterminated entity reference");
            const std::string ent = s.substr(k + 1, semi - k - 1);
            if(ent == "lt")
                out += '<';
            else if(ent == "gt")
                out += '>';
            else if(ent == "amp")
                out += '&';
            else if(ent == "quot")
                out += '"';
            else if(ent == "apos")
                out += '\'';
            else if(!ent.empty() && ent[0] == '#')
            {
                const unsigned long cp = ent.size() > 1 && (ent[1] == 'x' || ent[1] == 'X')
                                             ? std::strtoul(ent.c_str() + 2, nullptr, 16)
                                             : std::strtoul(ent.c_str() + 1, nullptr, 10);
                // UTF-8 encoding of the code point
                if(cp < 0x80)
                    out += (char)cp;
                else if(cp < 0x800)
                {
                    out += (char)(0xC0 | (cp >> 6));
                    out += (char)(0x80 | (cp & 0x3F));
                }
                else if(cp < 0x10000)
                {
                    out += (char)(0xE0 | (cp >> 12));
                    out += (char)(0x80 | ((cp >> 6) & 0x3F));
                    out += (char)(0x80 | (cp & 0x3F));
                }
                else
                {
                    out += (char)(0xF0 | (cp >> 18));
                    out += (char)(0x80 | ((cp >> 12) & 0x3F));
                    out += (char)(0x80 | ((cp >> 6) & 0x3F));
                    out += (char)(0x80 | (cp & 0x3F));
                }
            }
            else
                return fail("unknown entity &" + ent + ";");
            k = semi;
        }
        return true;
    }
    static void add_text(DOMNode& parent, std::string const& text)
    {
        if(text.empty())
            return;
        // adjacent text (around a dropped comment, or a CDATA section) is one node
        if(!parent.m_owned.empty() && parent.m_owned.back()->m_type == DOMNode::TEXT_NODE)
        {
            parent.m_owned.back()->m_value += text;
            return;
        }
        auto t     = std::make_unique<DOMNode>();
        t->m_type  = DOMNode::TEXT_NODE;
        t->m_name  = "#text";
        t->m_value = text;
        parent.m_children.m_items.push_back(t.get());
        parent.m_owned.push_back(std::move(t));
    }
    // an element from its '<'; `depth` bounds the nesting
    bool element(DOMElement& el, int depth)
    {
        if(depth > 512)
            return fail("elements nested deeper than 512");
        ++i; // '<'
        if(!name(el.m_name))
            return false;
        for(;;)
        {
            skip_space();
            if(i >= s.size())
                return fail("unterminated start tag <" + el.m_name + ">");
            if(starts("/>"))
            {
                i += 2;
                return true;
            }
            if(s[i] == '>')
            {
                ++i;
                break;
            }
            std::string an, av;
            if(!name(an))
                return false;
            skip_space();
            if(i >= s.size() || s[i] != '=')
                return fail("'=' expected after attribute " + an);
            ++i;
            skip_space();
            if(i >= s.size() || (s[i] != '"' && s[i] != '\''))
                return fail("quoted value expected for attribute " + an);
            const char   q = s[i++];
            const size_t e = s.find(q, i);
            if(e == std::string::npos)
                return fail("unterminated value of attribute " + an);
            if(!decode(i, e, av))
                return false;
            i = e + 1;
            if(el.getAttribute(an))
                return fail("attribute " + an + " given twice on <" + el.m_name + ">");
            el.m_attrs.emplace_back(an, av);
        }
        // content
        for(;;)
        {
            if(i >= s.size())
                return fail("element <" + el.m_name + "> is not closed");
            if(starts("</"))
            {
                i += 2;
                std::string en;
                if(!name(en))
                    return false;
                if(en != el.m_name)
                    return fail("</" + en + "> closes <" + el.m_name + ">");
                skip_space();
                if(i >= s.size() || s[i] != '>')
                    return fail("'>' expected after </" + en);
                ++i;
                return true;
            }
            if(starts("<!--"))
            {
                if(!skip_until("-->"))
                    return false;
                continue;
            }
            if(starts("<![CDATA["))
            {
                const size_t b = i + 9;
                const size_t e = s.find("]]>", b);
                if(e == std::string::npos)
                    return fail("unterminated CDATA section");
                add_text(el, s.substr(b, e - b));
                i = e + 3;
                continue;
            }
            if(starts("<?"))
            {
                if(!skip_until("?>"))
                    return false;
                continue;
            }
            if(s[i] == '<')
            {
                auto child = std::make_unique<DOMElement>();
                if(!element(*child, depth + 1))
                    return false;
                el.m_children.m_items.push_back(child.get());
                el.m_owned.push_back(std::move(child));
                continue;
            }
            const size_t e = s.find('<', i);
            const size_t stop = e == std::string::npos ? s.size() : e;
            std::string  text;
            if(!decode(i, stop, text))
                return false;
            add_text(el, text);
            i = stop;
        }
    }
    std::unique_ptr<DOMElement> document()
    {
        if(starts("\xEF\xBB\xBF")) // UTF-8 byte-order mark
            i += 3;
        std::unique_ptr<DOMElement> root;
        for(;;)
        {
            skip_space();
            if(i >= s.size())
                break;
            if(starts("<?"))
            {
                if(!skip_until("?>"))
                    return nullptr;
            }
            else if(starts("<!--"))
            {
                if(!skip_until("-->"))
                    return nullptr;
            }
            else if(starts("<!DOCTYPE"))
            {
                if(!skip_doctype())
                    return nullptr;
            }
            else if(s[i] == '<' && !root)
            {
                root = std::make_unique<DOMElement>();
                if(!element(*root, 0))
                    return nullptr;
            }
            else
            {
                fail(root ? "content after the document element" : "a document element was expected");
                return nullptr;
            }
        }
        if(!root)
            fail("the document has no element");
        return root;
    }
};
} // namespace

std::unique_ptr<DOMElement> parse(std::string const& text, std::string* error)
{
    Parser p(text);
    auto   root = p.document();
    if(!p.err.empty())
    {
        if(error)
            *error = p.err;
        return nullptr;
    }
    return root;
}

void elements_by_tag(DOMNode const* root, std::string const& name, std::vector<DOMNode*>& out)
{
    for(DOMNode* c : root->m_children.m_items)
        if(c->m_type == DOMNode::ELEMENT_NODE)
        {
            if(c->m_name == name)
                out.push_back(c);
            elements_by_tag(c, name, out);
        }
}
} // namespace xml
} // namespace gb

// ---- ReaderXML ------------------------------------------------------------------
namespace
{
// documents and node lists handed out by ReaderXML, freed by terminate()
std::vector<std::unique_ptr<DOMElement>>  g_documents;
std::vector<std::unique_ptr<DOMNodeList>> g_lists;
DOMBuilder                                g_builder;

DOMNodeList* keep(std::vector<DOMNode*>&& items)
{
    g_lists.push_back(std::make_unique<DOMNodeList>());
    g_lists.back()->m_items = std::move(items);
    return g_lists.back().get();
}

std::string const& attribute(DOMNode* root, string const& name)
{
    if(!root)
        throw std::runtime_error("ReaderXML: attribute \"" + name + "\" of a missing node");
    std::string const* v = root->getAttribute(name);
    if(!v)
        throw std::runtime_error("ReaderXML: <" + root->m_name + "> has no attribute \"" + name + "\"");
    return *v;
}

std::string const& first_child_text(DOMNode* root)
{
    if(!root || !root->getFirstChild())
        throw std::runtime_error("ReaderXML: <" + std::string(root ? root->m_name : "?")
                                 + "> has no content");
    return root->getFirstChild()->m_value;
}
} // namespace

DOMBuilder* ReaderXML::m_parser = nullptr;

void ReaderXML::initialize()
{
    m_parser = &g_builder;
}

void ReaderXML::terminate()
{
    g_lists.clear();
    g_documents.clear();
    m_parser = nullptr;
}

DOMNode* ReaderXML::getNode(DOMElement* root, string const& name)
{
    if(!root)
        return nullptr;
    std::vector<DOMNode*> found;
    gb::xml::elements_by_tag(root, name, found);
    return found.empty() ? nullptr : found.front();
}

DOMNode* ReaderXML::getNode(DOMNode* root, string const& name)
{
    if(!root)
        return nullptr;
    for(DOMNode* c : root->m_children.m_items)
        if(c->m_type == DOMNode::ELEMENT_NODE && c->m_name == name)
            return c;
    return nullptr;
}

double ReaderXML::getNodeAttr_Double(DOMNode* root, string const& name)
{
    return std::atof(attribute(root, name).c_str());
}

int ReaderXML::getNodeAttr_Int(DOMNode* root, string const& name)
{
    return std::atoi(attribute(root, name).c_str());
}

string ReaderXML::getNodeAttr_String(DOMNode* root, string const& name)
{
    return attribute(root, name);
}

bool ReaderXML::hasNodeAttr(DOMNode* root, string const& name)
{
    return root && root->getAttribute(name) != nullptr;
}

string ReaderXML::getNodeName(DOMNode const* root)
{
    if(!root)
        throw std::runtime_error("ReaderXML: name of a missing node");
    return root->m_name;
}

DOMNode* ReaderXML::getNodeNext(DOMNode* root)
{
    return root ? root->m_children.item(1) : nullptr;
}

double ReaderXML::getNodeValue_Double(DOMNode* root)
{
    return std::atof(first_child_text(root).c_str());
}

string ReaderXML::getNodeValue_String(DOMNode* root)
{
    return first_child_text(root);
}

DOMNodeList* ReaderXML::getNodes(DOMElement* root, string const& name)
{
    std::vector<DOMNode*> found;
    if(root)
        gb::xml::elements_by_tag(root, name, found);
    return keep(std::move(found));
}

DOMNodeList* ReaderXML::getNodes(DOMNode* root)
{
    std::vector<DOMNode*> found;
    if(root)
        for(DOMNode* c : root->m_children.m_items)
            if(c->m_type == DOMNode::ELEMENT_NODE)
                found.push_back(c);
    return keep(std::move(found));
}

DOMElement* ReaderXML::getRoot(string const& xmlFile)
{
    std::ifstream in(xmlFile, std::ios::binary);
    if(!in)
    {
        std::cerr << "XML exception: cannot read " << xmlFile << std::endl;
        return nullptr;
    }
    std::stringstream buf;
    buf << in.rdbuf();
    std::string err;
    auto        root = gb::xml::parse(buf.str(), &err);
    if(!root)
    {
        std::cerr << "XML exception: " << xmlFile << ", " << err << std::endl;
        return nullptr;
    }
    g_documents.push_back(std::move(root));
    return g_documents.back().get();
}
