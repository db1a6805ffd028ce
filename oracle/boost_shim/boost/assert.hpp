// std-based stand-in for <boost/assert.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
