// std-based stand-in for <boost/type_traits/make_signed.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
