// Minimal stand-in for tbb::concurrent_unordered_map (oracle reference checker only).
#pragma once
#include <map>
#include <mutex>
namespace tbb {
template <typename K, typename V>
class concurrent_unordered_map {
public:
    typedef typename std::map<K, V>::iterator iterator;
    V& operator[](const K& k) { std::lock_guard<std::mutex> l(m_); return m_map[k]; }
    iterator begin() { return m_map.begin(); }
    iterator end() { return m_map.end(); }
private:
    std::map<K, V> m_map;
    std::mutex m_;
};
}  // namespace tbb
