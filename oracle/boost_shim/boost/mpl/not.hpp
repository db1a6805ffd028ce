// std-based stand-in for <boost/mpl/not.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
