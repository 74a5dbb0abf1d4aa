/* Stand-in: boost::array as std::array (the reference only names the type). */
#pragma once
#include <array>
namespace boost { using std::array; }
