// std-based stand-in for <boost/unordered_set.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
#include <unordered_set>
namespace boost { using std::unordered_set; }
