// Xerces-free stand-in: the DOM of gb_dom.hh (see there).
#pragma once
#include "../../gb_dom.hh"
