// Minimal stand-in for tbb::concurrent_queue, enough for SupraLib/ContainerFactory.cpp to compile in
// the oracle's reference checker (test infrastructure; TBB is not installed in this environment).
#pragma once
#include <deque>
#include <mutex>
namespace tbb {
template <typename T>
class concurrent_queue {
public:
    concurrent_queue() = default;
    concurrent_queue(const concurrent_queue& o) : q_(o.q_) {}
    void push(const T& v) { std::lock_guard<std::mutex> l(m_); q_.push_back(v); }
    bool try_pop(T& v) {
        std::lock_guard<std::mutex> l(m_);
        if (q_.empty()) return false;
        v = q_.front();
        q_.pop_front();
        return true;
    }
    bool empty() const { return q_.empty(); }
private:
    std::deque<T> q_;
    mutable std::mutex m_;
};
}  // namespace tbb
