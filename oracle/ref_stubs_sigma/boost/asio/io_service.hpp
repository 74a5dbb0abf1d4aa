/* Stand-in: the io_service names the reference's thread pool is written with; it runs posted work
 * at once (the depth-noise model is called single-threaded from this build). */
#pragma once
#include <cstddef>
namespace boost {
namespace asio {
class io_service {
  public:
    struct work {
        explicit work(io_service&) {}
    };
    std::size_t run() { return 0; }
    template <class F> void post(F f) { f(); }
};
}  // namespace asio
}  // namespace boost
