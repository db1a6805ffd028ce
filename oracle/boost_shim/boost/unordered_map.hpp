// std-based stand-in for <boost/unordered_map.hpp>; see _shim_core.hpp.
#include <boost/_shim_core.hpp>
#include <unordered_map>
namespace boost { using std::unordered_map; }
