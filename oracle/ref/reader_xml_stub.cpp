// ReaderXML without Xerces: the harness builds every object from plain
// arrays, so none of these is reached.  They exist only so that the XML
// constructors the reference instantiates can link; each aborts if called.
#include <cstdlib>

#include "ReaderXML.hh"

DOMBuilder* ReaderXML::m_parser = nullptr;

void         ReaderXML::initialize() { std::abort(); }
void         ReaderXML::terminate() { std::abort(); }
DOMNode*     ReaderXML::getNode(DOMElement*, string const&) { std::abort(); }
DOMNode*     ReaderXML::getNode(DOMNode*, string const&) { std::abort(); }
double       ReaderXML::getNodeAttr_Double(DOMNode*, string const&) { std::abort(); }
int          ReaderXML::getNodeAttr_Int(DOMNode*, string const&) { std::abort(); }
string       ReaderXML::getNodeAttr_String(DOMNode*, string const&) { std::abort(); }
bool         ReaderXML::hasNodeAttr(DOMNode*, string const&) { std::abort(); }
string       ReaderXML::getNodeName(DOMNode const*) { std::abort(); }
DOMNode*     ReaderXML::getNodeNext(DOMNode*) { std::abort(); }
double       ReaderXML::getNodeValue_Double(DOMNode*) { std::abort(); }
string       ReaderXML::getNodeValue_String(DOMNode*) { std::abort(); }
DOMNodeList* ReaderXML::getNodes(DOMElement*, string const&) { std::abort(); }
DOMNodeList* ReaderXML::getNodes(DOMNode*) { std::abort(); }
DOMElement*  ReaderXML::getRoot(string const&) { std::abort(); }
