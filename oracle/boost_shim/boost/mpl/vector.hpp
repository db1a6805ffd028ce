// std-based stand-in for <boost/mpl/vector.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
