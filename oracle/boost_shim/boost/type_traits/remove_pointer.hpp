// std-based stand-in for <boost/type_traits/remove_pointer.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
