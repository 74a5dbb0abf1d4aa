/* Stand-in: boost::bind as std::bind (see thread.hpp). */
#pragma once
#include <functional>
namespace boost {
using std::bind;
}
