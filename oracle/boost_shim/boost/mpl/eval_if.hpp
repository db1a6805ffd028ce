// std-based stand-in for <boost/mpl/eval_if.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
