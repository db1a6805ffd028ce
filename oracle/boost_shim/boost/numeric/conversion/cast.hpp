// std-based stand-in for <boost/numeric/conversion/cast.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
