// std-based stand-in for <boost/static_assert.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
