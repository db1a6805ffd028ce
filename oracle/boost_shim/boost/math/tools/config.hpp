// std-based stand-in for <boost/math/tools/config.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
