// std-based stand-in for <boost/mpl/integral_c.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
