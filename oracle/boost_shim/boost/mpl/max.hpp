// std-based stand-in for <boost/mpl/max.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
