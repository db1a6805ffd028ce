// std-based stand-in for <boost/mpl/equal_to.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
