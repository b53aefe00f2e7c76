/* Empty stand-in: the reference includes <boost/atomic.hpp> (hilbertjoin/egojoin.h:19)
 * but its count-only build (-DCOUNT_ONLY) uses nothing from it. */
#ifndef HJ_SHIM_BOOST_ATOMIC_HPP
#define HJ_SHIM_BOOST_ATOMIC_HPP
#endif
