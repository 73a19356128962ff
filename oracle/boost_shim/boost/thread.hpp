// Test infrastructure: boost::thread_group over std::thread, for the
// reference's host code (one worker thread per device).
#pragma once
#include <thread>
#include <vector>
namespace boost {
class thread_group {
public:
    template <class F> void create_thread(F f) { threads_.emplace_back(f); }
    void join_all() {
        for (auto& t : threads_)
            if (t.joinable()) t.join();
        threads_.clear();
    }
    ~thread_group() { join_all(); }
private:
    std::vector<std::thread> threads_;
};
}
