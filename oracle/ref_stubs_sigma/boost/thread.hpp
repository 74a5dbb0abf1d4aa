/* Stand-in for the reference's build of src/staticDepthNoiseModeling.cpp and its thread pool
 * (src/threadPool.cpp, src/parallelism.cpp): the Boost.Thread names they are written with, as the
 * standard library's.  The depth-noise model is run single-threaded from this build. */
#pragma once
#include <functional>
#include <future>
#include <mutex>
#include <thread>
#include <vector>
namespace boost {
using mutex = std::mutex;
using thread = std::thread;
class thread_group {
  public:
    template <class F> void create_thread(F f) { ts_.emplace_back(f); }
    std::size_t size() const { return ts_.size(); }
    ~thread_group()
    {
        for (auto& t : ts_)
            if (t.joinable()) t.detach();
    }

  private:
    std::vector<std::thread> ts_;
};
template <class R> using packaged_task = std::packaged_task<R()>;
template <class R> using unique_future = std::future<R>;
template <class It> void wait_for_all(It a, It b)
{
    for (; a != b; ++a) a->wait();
}
}  // namespace boost
