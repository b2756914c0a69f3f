// Stand-in for the part of TBB that the reference's sources use
// (include/core/MipMap.hpp, src/acceleration/HLBVHAcceleration.cpp,
// include/core/Block.hpp, src/core/Block.cpp): blocked_range, parallel_for
// over one range, task_arena::current_thread_index and mutex with its
// scoped_lock.  parallel_for runs the range on the calling thread: the MIP
// construction and the HLBVH treelets give the same results for any
// partition (the HLBVH orders its leaves by an atomic counter, so a serial
// build is the deterministic one).  The render loop over image blocks that
// src/Main.cpp runs with tbb::parallel_for is driven by oracle/ref_shim/
// ref_render.cpp on host threads of its own.
#pragma once
#include <cstddef>
#include <mutex>

namespace tbb {
template <typename T>
class blocked_range {
public:
    blocked_range(T b, T e, size_t = 1) : b_(b), e_(e) {}
    T begin() const { return b_; }
    T end() const { return e_; }
private:
    T b_, e_;
};
template <typename Range, typename F>
void parallel_for(const Range &r, const F &f) { f(r); }
namespace task_arena {
inline int current_thread_index() { return 0; }
}
class mutex {
public:
    class scoped_lock {
    public:
        scoped_lock() = default;
        explicit scoped_lock(mutex &m) : m_(&m) { m_->m_.lock(); }
        ~scoped_lock() { if (m_) m_->m_.unlock(); }
        void acquire(mutex &m) { m_ = &m; m_->m_.lock(); }
        void release() { if (m_) m_->m_.unlock(); m_ = nullptr; }
        scoped_lock(const scoped_lock &) = delete;
        scoped_lock &operator=(const scoped_lock &) = delete;
    private:
        mutex *m_ = nullptr;
    };
    void lock() { m_.lock(); }
    void unlock() { m_.unlock(); }
private:
    std::mutex m_;
};
}  // namespace tbb
