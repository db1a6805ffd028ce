// std-based stand-in for <boost/mpl/pair.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
