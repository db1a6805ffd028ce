// std-based stand-in for <boost/mpl/if.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
