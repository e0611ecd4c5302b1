/* Shim: boost::shared_ptr is std::shared_ptr for the oracle build. */
#ifndef BBT_SHIM_BOOST_SHARED_PTR_HPP
#define BBT_SHIM_BOOST_SHARED_PTR_HPP
#include <memory>
namespace boost { using std::shared_ptr; }
#endif
