// std-based stand-in for <boost/mpl/int.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
