/* Stand-in: boost::ref / cref as the standard library's (see thread.hpp). */
#pragma once
#include <functional>
namespace boost {
using std::cref;
using std::ref;
}
