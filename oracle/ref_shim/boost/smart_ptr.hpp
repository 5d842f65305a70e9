// Test-infrastructure shim: boost::shared_ptr mapped onto std::shared_ptr for
// building the reference's kriging sources without boost.
#ifndef ORACLE_SHIM_BOOST_SMART_PTR_HPP
#define ORACLE_SHIM_BOOST_SMART_PTR_HPP
#include <memory>
namespace boost { using std::shared_ptr; }
#endif
