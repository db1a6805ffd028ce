// std-based stand-in for <boost/utility/enable_if.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
