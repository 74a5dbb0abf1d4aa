/* Stand-in: boost::optional appears only in declarations on the paths compiled here. */
#pragma once
namespace boost { template <class T> class optional; }
