/* Minimal stand-in for boost::lockfree::queue. The reference includes it from
 * hilbertjoin/egojoin.h:18 and instantiates one in mainJoin.cpp:48, but under
 * -DCOUNT_ONLY nothing is ever pushed or popped (the pair-queue path is dead
 * code). push/pop report failure so any accidental use is visible. */
#ifndef HJ_SHIM_BOOST_LOCKFREE_QUEUE_HPP
#define HJ_SHIM_BOOST_LOCKFREE_QUEUE_HPP
#include <cstddef>
namespace boost { namespace lockfree {
template <class T> class queue {
public:
    explicit queue(std::size_t) {}
    bool push(const T &) { return false; }
    bool pop(T &) { return false; }
};
} }
#endif
