// std-based stand-in for <boost/noncopyable.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
