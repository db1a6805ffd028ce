// std-based stand-in for <boost/mpl/erase_key.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
