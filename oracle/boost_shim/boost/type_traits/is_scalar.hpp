// std-based stand-in for <boost/type_traits/is_scalar.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
