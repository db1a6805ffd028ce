// std-based stand-in for <boost/mpl/less_equal.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
