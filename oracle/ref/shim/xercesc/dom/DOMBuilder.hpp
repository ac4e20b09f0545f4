// Forwards to the DOM stand-ins used by the oracle harness.
#include "xerces_shim.hpp"
