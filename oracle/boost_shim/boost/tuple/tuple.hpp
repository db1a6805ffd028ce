// std-based stand-in for <boost/tuple/tuple.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
