// Serial stand-in for the part of TBB that the reference's MipMap uses
// (include/core/MipMap.hpp): blocked_range, parallel_for over one range,
// task_arena::current_thread_index.  The reference build for the parity
// library runs the MIP construction on one thread; the results do not depend
// on the partition (every output texel is computed by one thread in a fixed
// order).
#pragma once
#include <cstddef>

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
}  // namespace tbb
