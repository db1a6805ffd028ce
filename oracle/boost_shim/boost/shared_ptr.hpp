// std-based stand-in for <boost/shared_ptr.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
